"""Electron-beam excitation (EELS) against the reference (golden_eels.npz,
made by running the reference on CPU): aloof, mixed and penetrating beams
through a 284-face gold sphere at 520 and 650 nm.

Tolerances, max-norm relative: potentials and beam fields 1e-12 (K0/K1 by
the trapezoidal rule agree with AMOS to ~1e-15); loss and photon-loss
probabilities of the reference's own solution 1e-10; loss of the GPU's FP64
solution 1e-7 (the surface loss is a small difference of face sums, up to
~100 times smaller than its terms at 650 nm)."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import bem
from mnpbem_b200.compstruct import CompStruct
from mnpbem_b200.eels import EELSRet

pytestmark = pytest.mark.gpu

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)
SETS = ['A', 'B', 'C']


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope='module')
def setup(gpu_ok):
    v, f = M.load_mesh('trisphere_144_20')
    cp = M.ComParticle([M.EpsConst(1.0), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    z = golden('golden_eels')
    return cp, z, {s: EELSRet(cp, z[s + '_impact_in'], 0.5, float(z['vel'])) for s in SETS}


def ref_sig(cp, z, pre, lam):
    return CompStruct(cp, lam, sig1=z[pre + 'sig1'], sig2=z[pre + 'sig2'], h1=z[pre + 'h1'],
                      h2=z[pre + 'h2'])


@pytest.mark.parametrize('name', SETS)
def test_potentials(setup, name):
    cp, z, ex = setup
    for i, lam in enumerate(z['lams']):
        pot = ex[name].potential(cp, float(lam))
        for key in ('phi1', 'phi1p', 'a1', 'a1p', 'phi2', 'phi2p', 'a2', 'a2p'):
            ref = z['%s_%d_%s' % (name, i, key)]
            if not np.any(ref):
                assert not np.any(getattr(pot, key)), (name, lam, key)
            else:
                assert rel(getattr(pot, key), ref) < 1e-12, (name, lam, key)


@pytest.mark.parametrize('name', SETS)
def test_loss_and_rad_of_reference_solution(setup, name):
    cp, z, ex = setup
    for i, lam in enumerate(z['lams']):
        pre = '%s_%d_' % (name, i)
        sig = ref_sig(cp, z, pre, float(lam))
        psurf, pbulk = ex[name].loss(sig)
        assert rel(psurf, z[pre + 'psurf']) < 1e-10, (name, lam)
        if np.any(z[pre + 'pbulk']):
            assert rel(pbulk, z[pre + 'pbulk']) < 1e-12
        prad, _ = ex[name].rad(sig)
        assert rel(prad, z[pre + 'prad']) < 1e-10, (name, lam)


@pytest.mark.parametrize('name', SETS)
def test_beam_fields(setup, name):
    cp, z, ex = setup
    for i, lam in enumerate(z['lams']):
        f = ex[name].field(cp, float(lam), inout=2)
        assert rel(f.e, z['%s_%d_e' % (name, i)]) < 1e-12
        assert rel(f.h, z['%s_%d_h' % (name, i)]) < 1e-12


def test_solve_and_loss(setup):
    cp, z, ex = setup
    b = bem.BEMRet(cp)
    for name in SETS:
        for i, lam in enumerate(z['lams']):
            pre = '%s_%d_' % (name, i)
            sig, _ = b.solve(ex[name].potential(cp, float(lam)))
            assert rel(sig.sig2, z[pre + 'sig2']) < 1e-10, (name, lam)
            psurf, _ = ex[name].loss(sig)
            assert rel(psurf, z[pre + 'psurf']) < 1e-7, (name, lam)


def test_spectrum_path(setup):
    """Beam potentials generated on the GPU for a batch of wavelengths feed
    the mixed-precision spectrum solver directly."""
    cp, z, ex = setup
    b = bem.BEMRet(cp, precision='mixed')
    sols = b.solve_spectrum(ex['C'], [float(x) for x in z['lams']], batch=2)
    for i, sig in enumerate(sols):
        psurf, _ = ex['C'].loss(sig)
        assert rel(psurf, z['C_%d_psurf' % i]) < 1e-5
