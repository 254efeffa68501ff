"""Quasistatic dipole excitations, point Green function fields and decay
rates against the reference (golden_dipole_stat.npz, made by running the
reference on CPU): five dipole positions (three outside a 284-face gold
sphere, one of them 2 nm above the surface, two inside) with the unit
moment triple, at 500 and 620 nm.

Tolerances, max-norm relative: closed-form potentials and fields 1e-12; the
FP64 BEMStat solution 1e-10; fields of the reference's solution at the
points 1e-11; decay rates from the GPU solution 1e-9.

The reference's ``DipoleStat.farfield`` raises (it imports a module that
does not exist); the far field here is checked against the closed form it
states (dipole_stat.py:415-510), restated in NumPy below."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import bem
from mnpbem_b200.compstruct import CompStruct
from mnpbem_b200.excitation import pinfty
from mnpbem_b200.greenfun import CompGreenStat
from mnpbem_b200.materials import eps_k
from mnpbem_b200.points import ComPoint, CompGreenStatPoints, DipoleStat

pytestmark = pytest.mark.gpu

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope='module')
def setup(gpu_ok):
    v, f = M.load_mesh('trisphere_144_20')
    cp = M.ComParticle([M.EpsConst(1.5), DRUDE], [M.Particle(v, f, interp='curv')], [[2, 1]])
    z = golden('golden_dipole_stat')
    pt = ComPoint(cp, z['pos_in'])
    assert np.array_equal(np.asarray(pt.pos), z['pt_pos'])
    return cp, pt, DipoleStat(pt), z


def test_potential_and_field(setup):
    cp, pt, exc, z = setup
    for i, lam in enumerate(z['lams']):
        assert rel(exc(cp, float(lam)).phip, z['%d_phip' % i]) < 1e-12
        assert rel(exc.field(cp, float(lam)).e, z['%d_e_faces' % i]) < 1e-12


def test_point_field_of_reference_solution(setup):
    cp, pt, exc, z = setup
    g = CompGreenStat(pt, cp)
    assert isinstance(g, CompGreenStatPoints)
    for i, lam in enumerate(z['lams']):
        sig = CompStruct(cp, float(lam), sig=z['%d_sig' % i])
        assert rel(g.field(sig).e, z['%d_e_pts' % i]) < 1e-11
        # the same field from the assembled entries
        Gp = g.eval('H2p')
        e = -np.einsum('pcj,jk->pck', Gp, z['%d_sig' % i].reshape(cp.n, -1))
        assert rel(e.reshape(z['%d_e_pts' % i].shape), z['%d_e_pts' % i]) < 1e-11


def test_solve_and_decayrate(setup):
    cp, pt, exc, z = setup
    b = bem.BEMStat(cp)
    for i, lam in enumerate(z['lams']):
        sig, _ = b.solve(exc(cp, float(lam)))
        assert sig.sig.shape == z['%d_sig' % i].shape
        assert rel(sig.sig, z['%d_sig' % i]) < 1e-10
        tot, rad, rad0 = exc.decayrate(sig)
        assert rel(tot, z['%d_tot' % i]) < 1e-9, lam
        assert rel(rad, z['%d_rad' % i]) < 1e-9, lam
        assert rel(rad0, z['%d_rad0' % i]) < 1e-12, lam


def test_farfield_closed_form(setup):
    cp, pt, exc, z = setup
    lam = 550.0
    ff = exc.farfield(None, lam)
    dirs = pinfty()[0]
    epsm, k = eps_k(cp.eps[0], lam)
    pos = np.asarray(pt.pos)
    scr = epsm / np.asarray(pt.eps1(lam))
    dip = exc.dip * scr[:, None, None]                               # (npt, 3, ndip)
    g = np.exp(-1j * k * dirs @ pos.T)                               # (ndir, npt)
    h = np.cross(dirs[:, None, None, :], dip.transpose(0, 2, 1)[None], axis=-1) * \
        g[:, :, None, None]                                          # (ndir, npt, ndip, 3)
    e = np.cross(h, dirs[:, None, None, :], axis=-1) * k ** 2 / epsm
    h = h * k ** 2 / np.sqrt(epsm)
    assert rel(ff.e, e.transpose(0, 3, 1, 2)) < 1e-12
    assert rel(ff.h, h.transpose(0, 3, 1, 2)) < 1e-12
