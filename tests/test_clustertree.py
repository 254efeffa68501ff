"""Cluster tree and block partition against the reference's (golden_hmat.npz,
made by tests/golden/make_golden_hmat.py): integer arrays bit-exact, node
boxes exact."""
import hashlib

import numpy as np
import pytest

from conftest import golden
from mnpbem_b200.clustertree import BlockPartition, ClusterTree, make_kaware_fadmiss
from mnpbem_b200.geometry import ComParticle, trirod, trisphere
from mnpbem_b200.materials import EpsConst, EpsDrude


def _particle(case):
    eps = [EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)]
    if case == 'sph':
        return ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1)
    if case == 'rod':
        return ComParticle(eps, [trirod(20.0, 80.0, (31, 21, 41))], [[2, 1]], 1)
    if case == 'dimer':
        s = trisphere(144, 10.0)
        return ComParticle(eps, [s.shift([-6.0, 0, 0]), s.shift([6.0, 0, 0])],
                           [[2, 1], [2, 1]], 1, 2)
    if case == 'big':
        return ComParticle(eps, [trirod(20.0, 80.0, (97, 47, 171))], [[2, 1]], 1)
    raise KeyError(case)


def _ipart(cp):
    if len(cp.p) <= 1:
        return None
    return np.concatenate([np.full(q.nfaces, i, dtype=np.int64) for i, q in enumerate(cp.p)])


def _arrays(cp, cleaf, enei):
    tree = ClusterTree(cp.pos, cleaf=cleaf, ipart_arr=_ipart(cp))
    part = BlockPartition(tree, make_kaware_fadmiss(2.0 * np.pi / enei, eta0=2.5))
    return dict(ind=tree.ind, cind=tree.cind, son=tree.son, mid=tree.mid, rad=tree.rad,
                ipart=tree.ipart, row1=part.row1, col1=part.col1, row2=part.row2,
                col2=part.col2)


def _sha(a):
    h = hashlib.sha256()
    a = np.ascontiguousarray(a)
    h.update(str(a.dtype).encode())
    h.update(a.tobytes())
    return h.hexdigest()


@pytest.mark.parametrize('case', ['sph', 'rod', 'dimer'])
def test_tree_and_partition_exact(case):
    g = golden('golden_hmat')
    n, cleaf, enei = g[case + '_meta']
    cp = _particle(case)
    assert cp.n == int(n)
    got = _arrays(cp, int(cleaf), float(enei))
    for name, a in got.items():
        ref = g[case + '_' + name]
        assert a.shape == ref.shape, name
        assert np.array_equal(a, ref), name


def test_tree_and_partition_25k_faces():
    g = golden('golden_hmat')
    n, cleaf, enei = g['big_meta']
    cp = _particle('big')
    assert cp.n == int(n) == 25152
    got = _arrays(cp, int(cleaf), float(enei))
    for name, a in got.items():
        assert _sha(np.asarray(a)) == str(g['big_sha_' + name]), name


def test_partition_covers_matrix_once():
    cp = _particle('dimer')
    tree = ClusterTree(cp.pos, cleaf=32, ipart_arr=_ipart(cp))
    part = BlockPartition(tree, make_kaware_fadmiss(2.0 * np.pi / 600.0))
    cover = np.zeros((cp.n, cp.n), dtype=np.int32)
    for blk in np.vstack([part.dense, part.lowrank]):
        r0, m, c0, k = blk
        cover[r0:r0 + m, c0:c0 + k] += 1
    assert np.all(cover == 1)
    # low-rank blocks never straddle the two particles
    ip = _ipart(cp)[tree.ind[:, 0]]
    for r0, m, c0, k in part.lowrank:
        assert np.unique(ip[r0:r0 + m]).size == 1 and np.unique(ip[c0:c0 + k]).size == 1
