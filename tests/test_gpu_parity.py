"""End-to-end parity of the CUDA path with the reference (golden fixtures
made by running the reference) and with the CPU oracle.

Tolerances: FP64 GPU path vs reference -- sigma 1e-10 relative (max-norm),
currents h 1e-8, Green matrices 1e-12, extinction/scattering 1e-10."""
import numpy as np
import pytest
import torch

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import bem, excitation

pytestmark = pytest.mark.gpu

EPS = [M.EpsConst(1.0), M.EpsDrude(10.0, 9.065, 0.0708)]


def _cp(key):
    v, f = M.load_mesh(key)
    s = M.Particle(v, f, interp='curv' if f.shape[1] == 9 else 'flat')
    return M.ComParticle(EPS, [s], [[2, 1]]), s


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.fixture(scope='module')
def tiny():
    cp, s = _cp('trisphere_32_10')
    return cp, bem.BEMRet(cp), golden('golden_tiny')


def test_refined_coefficients_tiny(gpu_ok, tiny):
    cp, b, z = tiny
    t = b.tables
    assert np.array_equal(t.h_rows, z['ref_rows']) and np.array_equal(t.h_cols, z['ref_cols'])
    assert rel(t.g.cpu().numpy(), z['ref_g'].real) < 1e-14
    assert rel(t.f_raw.cpu().numpy(), z['ref_f_raw'].real) < 1e-11
    assert rel(t.f.cpu().numpy(), z['ref_f'].real) < 1e-11


def test_green_matrices_tiny(gpu_ok, tiny):
    cp, b, z = tiny
    for key, (i, j), nm in [('G', (0, 0), 'G1_550'), ('G', (1, 1), 'G2_550'),
                            ('H1', (0, 0), 'H1_550'), ('H2', (1, 1), 'H2_550')]:
        assert rel(b.g.eval(i, j, key, 550.0), z[nm]) < 1e-11, nm
    assert b.g.eval(0, 1, 'G', 550.0) == 0


def test_bemret_tiny_two_pols(gpu_ok, tiny):
    cp, b, z = tiny
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    for i, lam in enumerate(z['lams']):
        sig, _ = b.solve(exc.potential(cp, lam))
        assert rel(sig.sig1, z['sig1_%d' % i]) < 1e-10
        assert rel(sig.sig2, z['sig2_%d' % i]) < 1e-10
        assert rel(sig.h1, z['h1_%d' % i]) < 1e-8
        assert rel(sig.h2, z['h2_%d' % i]) < 1e-8
        assert np.allclose(exc.extinction(sig), z['ext_%d' % i], rtol=1e-10)
        assert np.allclose(exc.scattering(sig)[0], z['sca_%d' % i], rtol=1e-10)


def test_bemret_spectrum_batched_matches_single(gpu_ok, tiny):
    cp, b, z = tiny
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=2)
    for i, sg in enumerate(sols):
        assert rel(sg.sig2, z['sig2_%d' % i]) < 1e-10
        assert rel(sg.h1, z['h1_%d' % i]) < 1e-8


def test_bemstat_tiny(gpu_ok, tiny):
    cp, b, z = tiny
    st = bem.BEMStat(cp)
    assert rel(st.F, z['stat_F']) < 1e-13
    ex = excitation.PlaneWaveStat([[1, 0, 0]])
    sig, _ = st.solve(ex.potential(cp, 550.0))
    assert rel(sig.sig, z['stat_sig_550']) < 1e-12


def test_c0_spectrum_41_wavelengths(gpu_ok):
    """trisphere(144, 20): the full 41-wavelength spectrum against the reference."""
    cp, s = _cp('trisphere_144_20')
    z = golden('golden_c0')
    b = bem.BEMRet(cp)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=41)
    ext = np.array([exc.extinction(sg) for sg in sols])
    sca = np.array([exc.scattering(sg)[0] for sg in sols])
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-10
    assert np.max(np.abs(sca - z['sca']) / np.abs(z['sca'])) < 1e-10
    i470 = list(z['lams']).index(470.0)
    assert rel(sols[i470].sig2, z['sig2_470']) < 1e-10
    # quasistatic spectrum
    st = bem.BEMStat(cp)
    ex = excitation.PlaneWaveStat([[1, 0, 0]])
    for lam, e_ref in zip(z['stat_lams'], z['stat_ext']):
        sig, _ = st.solve(ex.potential(cp, lam))
        assert abs(ex.extinction(sig) - e_ref) < 1e-10 * abs(e_ref)


def test_rod_flat_quads(gpu_ok):
    """trirod(20, 80): flat mesh dominated by quadrilaterals."""
    cp, s = _cp('trirod_20_80_31_21_41')
    z = golden('golden_rod')
    b = bem.BEMRet(cp)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sig, _ = b.solve(exc.potential(cp, float(z['lam'])))
    assert abs(exc.extinction(sig) - float(z['ext'])) < 1e-9 * abs(float(z['ext']))
    assert abs(exc.scattering(sig)[0] - float(z['sca'])) < 1e-9 * abs(float(z['sca']))


def test_c1_2884_faces(gpu_ok):
    """trisphere(1444, 40) (2884 faces): extinction at 3 wavelengths, BEMStat too."""
    cp, s = _cp('trisphere_1444_40')
    z = golden('golden_c1')
    b = bem.BEMRet(cp)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=3)
    ext = np.array([exc.extinction(sg) for sg in sols])
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-10
    st = bem.BEMStat(cp)
    ex = excitation.PlaneWaveStat([[1, 0, 0]])
    for lam, e_ref in zip(z['stat_lams'], z['stat_ext']):
        sig, _ = st.solve(ex.potential(cp, lam))
        assert abs(ex.extinction(sig) - e_ref) < 1e-10 * abs(e_ref)


def test_native_library_was_used(gpu_ok):
    from mnpbem_b200 import _lib
    assert _lib.launch_count() > 0


def test_c0_refined_coefficient_subset(gpu_ok):
    """trisphere(144, 20) (284 curved faces): every 23rd refined pair of the
    reference (g and the closure-corrected f, greenret_refined.py:122-516,
    compgreen_ret.py:376-400), matched pair by pair (row, col)."""
    cp, s = _cp('trisphere_144_20')
    z = golden('golden_c0')
    b = bem.BEMRet(cp)
    t = b.tables
    key = {(int(r), int(c)): i for i, (r, c) in enumerate(zip(t.h_rows, t.h_cols))}
    idx = np.array([key[(int(r), int(c))] for r, c in zip(z['ref_rows'], z['ref_cols'])])
    assert len(idx) == len(z['ref_sub']) > 400
    g = t.g.cpu().numpy()[idx]
    f = t.f.cpu().numpy()[idx]
    assert rel(g, z['ref_g'].real) < 1e-13
    assert rel(f, z['ref_f'].real) < 1e-11
    # self pairs (polar quadrature) and near pairs (face quadrature) both present
    kinds = t.h_kinds[idx]
    assert (kinds == 2).sum() > 10 and (kinds == 1).sum() > 100


@pytest.fixture(scope='module')
def c1sig():
    cp, s = _cp('trisphere_1444_40')
    return cp, golden('golden_c1_sig')


def test_c1_fp64_sigma_five_wavelengths(gpu_ok, c1sig):
    """trisphere(1444, 40) (2884 faces): the plain FP64 GPU path against the
    reference BEMRet at 400, 470 (resonance), 520, 600, 800 nm -- sigma within
    1e-10 (max-norm relative), h within 1e-9, extinction and scattering within
    1e-10."""
    cp, z = c1sig
    b = bem.BEMRet(cp)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=5)
    for i, sg in enumerate(sols):
        assert rel(sg.sig1, z['sig1_%d' % i]) < 1e-10, i
        assert rel(sg.sig2, z['sig2_%d' % i]) < 1e-10, i
        assert rel(sg.h1, z['h1_%d' % i]) < 1e-9, i
        assert rel(sg.h2, z['h2_%d' % i]) < 1e-9, i
    ext = np.array([exc.extinction(sg) for sg in sols]).ravel()
    sca = np.array([exc.scattering(sg)[0] for sg in sols]).ravel()
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-10
    assert np.max(np.abs(sca - z['sca']) / np.abs(z['sca'])) < 1e-10
