"""Point sets and the point-face classifier on the host (no GPU): the
medium grouping of ``ComPoint`` and the refinement pairs of
``refinematrix(points, particle)`` against the reference
(golden_dipole.npz, made by running the reference)."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200.greenfun import refinematrix_csr
from mnpbem_b200.points import ComPoint, Point, DipoleRet, point_media, is_point_set

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


@pytest.fixture(scope='module')
def setup():
    v, f = M.load_mesh('trisphere_144_20')
    cp = M.ComParticle([M.EpsConst(1.5), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    return cp, golden('golden_dipole')


def test_compoint_groups_by_medium(setup):
    cp, z = setup
    pt = ComPoint(cp, z['pos_in'])
    pos, med = point_media(pt)
    assert np.array_equal(pos, z['pt_pos'])
    assert np.array_equal(med, z['pt_inout'])
    assert pt.n == 5 and pt.np == 2 and list(pt.inout) == [1, 2]
    assert [list(i) for i in pt.index] == [[0, 1, 2], [3, 4]]
    assert is_point_set(pt) and not is_point_set(cp)
    # medium filter and minimum distance
    assert ComPoint(cp, z['pos_in'], medium=2).n == 2
    near = ComPoint(cp, np.array([[0.0, 0.0, 10.05], [0.0, 0.0, 30.0]]), mindist=3.0)
    assert near.n == 1 and np.allclose(near.pos, [[0.0, 0.0, 30.0]])
    # direct construction
    d = ComPoint(cp.eps, [Point(np.zeros((2, 3))), np.ones((1, 3))], [2, 1])
    assert d.n == 3 and np.array_equal(point_media(d)[1], [2, 2, 1])


def test_point_refinement_pairs(setup):
    cp, z = setup
    rptr, cols, kinds = refinematrix_csr(z['pt_pos'], np.asarray(cp.pos), None,
                                         np.asarray(cp.bradius()))
    rows = np.repeat(np.arange(5), np.diff(rptr))
    ours = sorted(zip(rows.tolist(), cols.tolist()))
    ref = sorted(zip(z['ir_rows'].tolist(), z['ir_cols'].tolist()))
    assert ours == ref
    assert np.all(kinds == 1)


def test_dipole_moments_layout(setup):
    cp, z = setup
    pt = ComPoint(cp, z['pos_in'])
    d = DipoleRet(pt)
    assert d.dip.shape == (5, 3, 3) and np.array_equal(d.dip[2], np.eye(3))
    d = DipoleRet(pt, np.array([[0.0, 0.0, 1.0]]))
    assert d.dip.shape == (5, 3, 1)
    full = np.arange(15, dtype=float).reshape(5, 3)
    d = DipoleRet(pt, full, full=True)
    assert d.dip.shape == (5, 3, 1) and np.array_equal(d.dip[:, :, 0], full)
