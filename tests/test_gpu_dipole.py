"""Dipole excitations, point Green functions and decay rates against the
reference (golden_dipole.npz, made by running the reference on CPU).

Tolerances, max-norm relative: closed-form potentials and fields 1e-11;
point-face Green-function entries 1e-11; the FP64 solution 1e-10 and what is
derived from it (fields at the points, decay rates, scattering) 1e-9; the
mixed-precision spectrum path 1e-6 (its FP64 refinement stops at a forward
error of 1e-11 relative to the TF32 start, the decay rates amplify it by the
near-field enhancement)."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import bem
from mnpbem_b200.compstruct import CompStruct
from mnpbem_b200.greenfun import CompGreenRet
from mnpbem_b200.points import ComPoint, DipoleRet, CompGreenRetPoints

pytestmark = pytest.mark.gpu

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope='module')
def setup(gpu_ok):
    v, f = M.load_mesh('trisphere_144_20')
    cp = M.ComParticle([M.EpsConst(1.5), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    z = golden('golden_dipole')
    pt = ComPoint(cp, z['pos_in'])
    return cp, pt, DipoleRet(pt), z


def golden_sig(cp, z, i):
    return CompStruct(cp, float(z['lams'][i]), sig1=z['sig1_%d' % i], sig2=z['sig2_%d' % i],
                      h1=z['h1_%d' % i], h2=z['h2_%d' % i])


def test_potentials(setup):
    cp, pt, exc, z = setup
    for i, lam in enumerate(z['lams']):
        pot = exc.potential(cp, float(lam))
        for key in ('phi1', 'phi1p', 'a1', 'a1p', 'phi2', 'phi2p', 'a2', 'a2p'):
            assert rel(getattr(pot, key), z['%s_%d' % (key, i)]) < 1e-11, (key, lam)


def test_point_green_entries(setup):
    cp, pt, exc, z = setup
    g = CompGreenRet(pt, cp)
    assert isinstance(g, CompGreenRetPoints) and g.nref == len(z['ir_rows'])
    for i, lam in enumerate(z['lams']):
        assert rel(g.eval(0, 1, 'G', float(lam)), z['G_%d' % i]) < 1e-11
        assert rel(g.eval(0, 1, 'Gp', float(lam)), z['Gp_%d' % i]) < 1e-11
        assert rel(g.eval(0, 1, 'H2p', float(lam)), z['Gp_%d' % i]) < 1e-11
    assert g.eval(0, 0, 'F', 500.0) == 0


def test_solution_and_fields_at_points(setup):
    cp, pt, exc, z = setup
    b = bem.BEMRet(cp)
    sig, _ = b.solve(exc.potential(cp, float(z['lams'][0])))
    for key in ('sig1', 'sig2', 'h1', 'h2'):
        assert rel(getattr(sig, key), z['%s_0' % key]) < 1e-10, key
    f = CompGreenRet(pt, cp).field(golden_sig(cp, z, 0))
    assert rel(f.e, z['pe_0']) < 1e-10
    assert rel(f.h, z['ph_0']) < 1e-10


def test_decay_rates_and_scattering(setup):
    cp, pt, exc, z = setup
    b = bem.BEMRet(cp)
    for i, lam in enumerate(z['lams']):
        sig, _ = b.solve(exc.potential(cp, float(lam)))
        tot, rad, rad0 = exc.decayrate(sig)
        assert rel(tot, z['tot_%d' % i]) < 1e-9, lam
        assert rel(rad, z['rad_%d' % i]) < 1e-9, lam
        assert rel(rad0, z['rad0_%d' % i]) < 1e-13, lam
        sca, _ = exc.scattering(sig)
        assert rel(sca, z['sca_%d' % i]) < 1e-9, lam


def test_dipole_fields_at_faces(setup):
    cp, pt, exc, z = setup
    for i, lam in enumerate(z['lams']):
        f = exc.field(cp, float(lam), inout=2)
        assert f.e.shape == (cp.n, 3, 5, 3)
        assert rel(f.e[:, :, :3], z['de_%d' % i]) < 1e-11
        assert rel(f.h[:, :, :3], z['dh_%d' % i]) < 1e-11
        assert not np.any(f.e[:, :, 3:])            # inside points: not connected


def test_multi_rhs_equals_sequential(setup):
    """As the reference's test_multirhs_dipole: three moments in one solve
    equal three single-moment solves."""
    cp, pt, exc, z = setup
    b = bem.BEMRet(cp)
    sig3, _ = b.solve(exc.potential(cp, 600.0))
    s1 = np.asarray(sig3.sig1).reshape(cp.n, 5, 3)
    for d in range(3):
        one = DipoleRet(pt, np.eye(3)[d:d + 1])
        si, _ = b.solve(one.potential(cp, 600.0))
        assert np.abs(np.asarray(si.sig1).reshape(cp.n, 5) - s1[:, :, d]).max() <= \
            1e-12 * np.abs(s1).max()


def test_mixed_spectrum_decay_rates(setup):
    cp, pt, exc, z = setup
    b = bem.BEMRet(cp, precision='mixed')
    sols = b.solve_spectrum(exc, [float(x) for x in z['lams']], batch=2)
    for i, sig in enumerate(sols):
        tot, rad, _ = exc.decayrate(sig)
        assert rel(tot, z['tot_%d' % i]) < 1e-6
        assert rel(rad, z['rad_%d' % i]) < 1e-6
    assert rel(sols[0].sig2, z['sig2_0']) < 1e-6
