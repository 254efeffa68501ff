"""Work records of the H-matrix product kernels (hmatrix.row_records,
vtx_records and the packed row items), checked on the CPU: a NumPy walk of
the records that follows the kernels' indexing (hm_vtx_kernel,
hm_vtx_reduce_kernel, hm_rows_kernel with its 32-column stages,
hm_reduce_kernel) must give the product of the dense matrix assembled
directly from the block rectangles, for random ranks (zero included) and
random factors on a rod and on a two-particle tree."""
import numpy as np
import pytest
import torch

from mnpbem_b200.clustertree import BlockPartition, ClusterTree, make_kaware_fadmiss
from mnpbem_b200.hmatrix import HTopology, row_records, vtx_records

XS = 32          # x columns per stage of hm_rows_kernel


def _offsets(sizes):
    return np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)


def _setup(pos, cleaf, k, ipart, seed):
    rng = np.random.default_rng(seed)
    tree = ClusterTree(pos, cleaf, ipart)
    part = BlockPartition(tree, make_kaware_fadmiss(k))
    topo = HTopology(part, 100, torch.device('cpu'))
    lr, dn = part.lowrank.astype(np.int64), part.dense.astype(np.int64)
    rank = rng.integers(0, 41, size=lr.shape[0]).astype(np.int64)
    if rank.size:
        rank[0] = 0
        rank[-1] = 40
    offU = _offsets(lr[:, 1] * rank)
    offV = _offsets(lr[:, 3] * rank)
    offT = _offsets(rank)
    offTP = _offsets(topo.vseg_count * rank)
    cz = lambda m: rng.standard_normal(m) + 1j * rng.standard_normal(m)
    D = cz(max(1, topo.dense_entries))
    U = cz(max(1, int((lr[:, 1] * rank).sum())))
    V = cz(max(1, int((lr[:, 3] * rank).sum())))
    return tree, part, topo, rank, offU, offV, offT, offTP, D, U, V, dn, lr


def _dense(n, topo, rank, offU, offV, D, U, V, dn, lr):
    A = np.zeros((n, n), dtype=complex)
    for b, (r0, m, c0, w) in enumerate(dn):
        A[r0:r0 + m, c0:c0 + w] = D[topo.offD_h[b]:topo.offD_h[b] + m * w].reshape(w, m).T
    for b, (r0, m, c0, w) in enumerate(lr):
        r = rank[b]
        Ub = U[offU[b]:offU[b] + m * r].reshape(r, m).T          # column-major m x r
        Vb = V[offV[b]:offV[b] + w * r].reshape(w, r)            # (j, q) at q + j r
        A[r0:r0 + m, c0:c0 + w] = Ub @ Vb.T
    return A


def _walk(topo, rank, offU, offV, offT, offTP, D, U, V, Xc, nc):
    n = topo.n
    rent = row_records(topo, rank, offU, offT)
    vent = vtx_records(topo, rank, offV, offTP)
    TP = np.zeros((max(1, int((topo.vseg_count * rank).sum())) * 4 + 4,), dtype=complex)
    if topo.nlr:
        for v in vent:
            r, cnt = int(v['r']), int(v['cnt'])
            for q in range(r):
                for c in range(nc):
                    TP[(v['out'] + q) * 4 + c] = sum(
                        V[v['v'] + j * r + q] * Xc[c, v['xo'] + j] for j in range(cnt))
    T = np.zeros((max(1, int(rank.sum())) * nc,), dtype=complex)
    vptr = topo.vptr.numpy()
    for b in range(topo.nlr):
        r = rank[b]
        nseg = vptr[b + 1] - vptr[b]
        for q in range(r):
            for c in range(nc):
                T[offT[b] * nc + q * nc + c] = sum(
                    TP[((offTP[b] + sg * r) + q) * 4 + c] for sg in range(nseg))
    items = topo.items.numpy()
    chunks = topo.chunks.numpy()
    leaf = topo.leaf_rows.numpy()
    cptr = topo.cptr.numpy()
    partial = np.zeros((len(items), 32, nc), dtype=complex)
    for it, (k, e0, e1, packed) in enumerate(items):
        r0, nlive = packed >> 6, packed & 63
        assert e1 - e0 <= 32
        assert r0 == chunks[k][1] and nlive == min(32, leaf[chunks[k][0]][1] - r0)
        for e in range(e0, e1):
            rec = rent[e]
            base = D if rec['kind'] == 0 else U
            for j0 in range(0, int(rec['cnt']), XS):            # the kernel's stages
                for j in range(j0, min(j0 + XS, int(rec['cnt']))):
                    for c in range(nc):
                        x = Xc[c, rec['xo'] + j] if rec['kind'] == 0 else \
                            T[(rec['xo'] + j) * nc + c]
                        for i in range(nlive):
                            partial[it, i, c] += base[rec['a'] + r0 + i + j * rec['lda']] * x
    Yc = np.zeros((nc, n), dtype=complex)
    for k, (L, r0) in enumerate(chunks):
        rows = min(32, leaf[L][1] - r0)
        for i in range(rows):
            Yc[:, leaf[L][0] + r0 + i] = partial[cptr[k]:cptr[k + 1], i, :].sum(axis=0)
    return Yc


@pytest.mark.parametrize('case', ['rod', 'two_particles'])
def test_records_walk_equals_dense_product(case):
    from mnpbem_b200.geometry import trirod, trisphere
    if case == 'rod':
        pos = trirod(20.0, 80.0, (11, 11, 21)).pos
        ipart = None
        cleaf, k = 16, 2 * np.pi / 300.0
    else:
        a, b = trisphere(144, 10.0).pos, trisphere(144, 10.0).pos + [25.0, 0, 0]
        pos = np.concatenate([a, b])
        ipart = np.repeat([0, 1], [a.shape[0], b.shape[0]])
        cleaf, k = 40, 2 * np.pi / 500.0
    tree, part, topo, rank, offU, offV, offT, offTP, D, U, V, dn, lr = \
        _setup(pos, cleaf, k, ipart, seed=3)
    assert topo.nlr > 0 and topo.ndense > 0
    n = topo.n
    nc = 3
    rng = np.random.default_rng(5)
    Xc = rng.standard_normal((nc, n)) + 1j * rng.standard_normal((nc, n))
    A = _dense(n, topo, rank, offU, offV, D, U, V, dn, lr)
    Yc = _walk(topo, rank, offU, offV, offT, offTP, D, U, V, Xc, nc)
    want = (A @ Xc.T).T
    assert np.abs(Yc - want).max() < 1e-10 * np.abs(want).max()
