"""Green-function entries of one region pair, potentials and fields at the
faces, against the reference (golden_fields.npz, golden_tiny.npz,
golden_dimer.npz made by running the reference).

Tolerances (max-norm relative, as the other parity tests): matrix entries
1e-11 (the self-term Taylor sums carry ~1e-12 absolute rounding), potentials
and fields of a solution 1e-10."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import bem, excitation
from mnpbem_b200.greenfun import CompGreenStat

pytestmark = pytest.mark.gpu

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope='module')
def sphere(gpu_ok):
    v, f = M.load_mesh('trisphere_32_10')
    cp = M.ComParticle([M.EpsConst(1.0), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    return cp, bem.BEMRet(cp), golden('golden_fields'), golden('golden_tiny')


def test_cartesian_derivatives(sphere):
    cp, b, z, _ = sphere
    assert rel(b.g.eval(0, 0, 'Gp', 550.0), z['Gp_00']) < 1e-11
    assert rel(b.g.eval(0, 0, 'H1p', 550.0), z['H1p_00']) < 1e-11
    assert rel(b.g.eval(1, 1, 'H2p', 550.0), z['H2p_11']) < 1e-11
    assert b.g.eval(0, 1, 'Gp', 550.0) == 0          # no block connects


def test_eval_block(sphere):
    cp, b, z, _ = sphere
    assert rel(b.g.eval_block(0, 0, 'F', 550.0, 10, 25), z['blkF_00']) < 1e-11
    assert rel(b.g.eval_block(0, 0, 'H1p', 550.0, 10, 25), z['blkH1p_00']) < 1e-11
    assert b.g.eval_block(0, 1, 'G', 550.0, 0, 7).shape == (60, 7)
    with pytest.raises(ValueError):
        b.g.eval_block(0, 0, 'G', 550.0, 10, 61)


def test_eval_selected_entries(sphere):
    """eval(..., ind): row-major linear indices i * n + j.  The reference's
    own _eval2 raises on a single particle (compgreen_ret.py:885), so the
    entries are pinned against its full matrices."""
    cp, b, _, t = sphere
    ind = np.array([0, 1, 59, 61, 62, 130, 777, 1800, 2519, 3599, 121, 1234, 2000, 3000, 3540])
    assert rel(b.g.eval(0, 0, 'G', 550.0, ind), t['G1_550'].ravel()[ind]) < 1e-11
    assert rel(b.g.eval(1, 1, 'H2', 550.0, ind), t['H2_550'].ravel()[ind]) < 1e-11
    gp = b.g.eval(0, 0, 'Gp', 550.0, ind)
    full = b.g.eval(0, 0, 'Gp', 550.0)
    assert gp.shape == (len(ind), 3)
    assert rel(gp, full.transpose(0, 2, 1).reshape(-1, 3)[ind]) < 1e-14
    assert not np.any(b.g.eval(0, 1, 'G', 550.0, ind))
    with pytest.raises(IndexError):
        b.g.eval(0, 0, 'G', 550.0, [3600])


def test_static_green_function(sphere):
    cp, b, z, _ = sphere
    gs = CompGreenStat(cp)
    assert rel(gs.G, z['stat_G']) < 1e-12
    assert rel(gs.F, z['stat_F']) < 1e-12
    G, Gp = gs.eval('G', 'Gp')
    assert rel(G, z['stat_G']) < 1e-12
    assert rel(Gp, z['stat_Gp']) < 1e-11
    assert rel(gs.eval('H1p'), z['stat_H1p']) < 1e-11
    ind = np.array([0, 5, 61, 3599])
    assert rel(gs.eval(ind, 'G'), z['stat_G'].ravel()[ind]) < 1e-12
    assert rel(gs.eval_block('G', 500.0, 3, 9), z['stat_G'][:, 3:9]) < 1e-12


def test_potential_and_field_sphere(sphere):
    cp, b, z, _ = sphere
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    sig, _ = b.solve(exc.potential(cp, 550.0))
    for inout in (1, 2):
        s = str(inout)
        pot = b.potential(sig, inout)
        assert rel(getattr(pot, 'phi' + s), z['sph_phi_in%d' % inout]) < 1e-10
        assert rel(getattr(pot, 'phi' + s + 'p'), z['sph_phip_in%d' % inout]) < 1e-10
        assert rel(getattr(pot, 'a' + s), z['sph_a_in%d' % inout]) < 1e-10
        assert rel(getattr(pot, 'a' + s + 'p'), z['sph_ap_in%d' % inout]) < 1e-10
        f = b.field(sig, inout)
        assert f.e.shape == z['sph_e_in%d' % inout].shape
        assert rel(f.e, z['sph_e_in%d' % inout]) < 1e-10
        assert rel(f.h, z['sph_h_in%d' % inout]) < 1e-10


def test_potential_and_field_dimer(gpu_ok):
    """Two particles: the region-pair blocks connect across particles."""
    z = golden('golden_fields')
    v, f = M.load_mesh('trisphere_144_10')
    s1 = M.Particle(v, f, interp='curv').shift([-6.0, 0.0, 0.0])
    s2 = M.Particle(v, f, interp='curv').shift([6.0, 0.0, 0.0])
    cp = M.ComParticle([M.EpsConst(1.77), DRUDE], [s1, s2], [[2, 1], [2, 1]], 1, 2)
    b = bem.BEMRet(cp)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sig, _ = b.solve(exc.potential(cp, 600.0))
    for inout in (1, 2):
        s = str(inout)
        pot = b.potential(sig, inout)
        assert rel(getattr(pot, 'phi' + s), z['dim_phi_in%d' % inout]) < 1e-10
        assert rel(getattr(pot, 'a' + s + 'p'), z['dim_ap_in%d' % inout]) < 1e-10
        fl = b.field(sig, inout)
        assert fl.e.shape == (cp.n, 3)
        assert rel(fl.e, z['dim_e_in%d' % inout]) < 1e-10
        assert rel(fl.h, z['dim_h_in%d' % inout]) < 1e-10
