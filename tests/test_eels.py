"""Electron-beam set-up on the host (no GPU): crossing points, beam
segments inside the particle, faces integrated with quadrature, path lengths
and bulk losses against the reference (golden_eels.npz, made by running the
reference), and the Legendre-Gauss-Lobatto rule of the wire integrals."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200.eels import EELSRet, ene2vel, lgl_nodes

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


@pytest.fixture(scope='module')
def setup():
    v, f = M.load_mesh('trisphere_144_20')
    cp = M.ComParticle([M.EpsConst(1.0), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    return cp, golden('golden_eels')


@pytest.mark.parametrize('name', ['A', 'B', 'C'])
def test_beam_setup(setup, name):
    cp, z = setup
    assert z['vel'] == ene2vel(200e3)
    e = EELSRet(cp, z[name + '_impact_in'], 0.5, float(z['vel']))
    assert np.array_equal(e.impact, z[name + '_impact'])
    assert np.allclose(e._z, z[name + '_z'], rtol=0, atol=1e-12)
    assert np.array_equal(e._indimp, z[name + '_indimp'])
    assert np.array_equal(e._indmat, z[name + '_indmat'])
    assert np.array_equal(e._indquad, z[name + '_indquad'])
    assert np.allclose(e.path(), z[name + '_path'], rtol=1e-13, atol=0)
    for i, lam in enumerate(z['lams']):
        pb = e.bulkloss(float(lam))
        ref = z['%s_%d_pbulk' % (name, i)]
        assert np.allclose(pb, ref, rtol=1e-12, atol=0)


def test_lobatto_rule():
    x, w = lgl_nodes(10)
    assert x[0] == 1.0 and x[-1] == -1.0 and np.all(np.diff(x) < 0)
    for deg in range(20):                       # exact through degree 2n - 1 = 19
        exact = 0.0 if deg % 2 else 2.0 / (deg + 1)
        assert abs(w @ x ** deg - exact) < 1e-14


@pytest.mark.parametrize('name', ['A', 'B', 'C'])
def test_stat_beam_setup_and_bulkloss(setup, name):
    """EELSStat shares the beam set-up; its bulk loss (eels_stat.py:195-228)
    against the reference's (golden_eels_stat.npz)."""
    from mnpbem_b200.eels import EELSStat
    cp, _ = setup
    z = golden('golden_eels_stat')
    e = EELSStat(cp, z[name + '_impact_in'], 0.5, float(z['vel']))
    assert e.name == 'eels' and e.needs == {'sim': 'stat'}
    assert np.array_equal(e._indimp, z[name + '_indimp'])
    for i, lam in enumerate(z['lams']):
        pb = e.bulkloss(float(lam))
        ref = z['%s_%d_pbulk' % (name, i)]
        assert np.allclose(pb, ref, rtol=1e-12, atol=0)
