"""The oracle and the host geometry against fixtures made by the reference.

``tests/golden/make_golden.py`` ran the reference (PyMNPBEM) to write the
fixtures; these tests pin the CPU restatement (``oracle/``) and the package's
host-side geometry to them.
"""
import hashlib

import numpy as np
import pytest

from conftest import golden
from mnpbem_b200.geometry import Particle, ComParticle, load_mesh
from oracle import bem_oracle as O

DRUDE = lambda e: O.eps_drude(10.0, 9.065, 0.0708, e)
VAC = lambda e: O.eps_const(1.0, e)


def _sphere(key):
    v, f = load_mesh(key)
    return Particle(v, f, interp='curv')


def _digest(r, c, v):
    h = hashlib.sha256()
    for a in (r, c, v):
        h.update(np.ascontiguousarray(a, dtype=np.int64).tobytes())
    return h.hexdigest()


def test_geometry_bitexact_tiny():
    z = golden('golden_tiny')
    s = _sphere('trisphere_32_10')
    for k in ['pos', 'nvec', 'tvec1', 'tvec2', 'area']:
        assert np.array_equal(getattr(s, k), z['geom_' + k]), k
    assert np.array_equal(s.bradius(), z['geom_bradius'])


@pytest.mark.parametrize('fn,key', [('golden_c1', 'trisphere_1444_40'),
                                    ('golden_rod', 'trirod_20_80_31_21_41')])
def test_near_pairs_bitexact_large(fn, key):
    z = golden(fn)
    v, f = load_mesh(key)
    s = Particle(v, f, interp='curv' if f.shape[1] == 9 else 'flat')
    ir = O.refinematrix(s.pos, s.pos, s.bradius(), s.bradius())
    r, c = np.nonzero(ir)
    assert len(r) == int(z['near_count'])
    assert _digest(r, c, ir[r, c]) == str(z['near_digest'])


def test_refined_coefficients_and_matrices_tiny():
    z = golden('golden_tiny')
    s = _sphere('trisphere_32_10')
    cp = ComParticle([VAC, DRUDE], [s], [[2, 1]])
    ir = O.refinematrix(s.pos, s.pos, s.bradius(), s.bradius())
    r, c = np.nonzero(ir)
    assert np.array_equal(r, z['near_rows']) and np.array_equal(c, z['near_cols'])
    assert np.array_equal(ir[r, c], z['near_vals'])
    rows, cols, g, fraw = O.refined_coefficients(s, ir)
    assert np.array_equal(g, z['ref_g'])
    assert np.array_equal(fraw, z['ref_f_raw'])
    gr = O.RetGreen(cp)
    assert np.allclose(gr.f, z['ref_f'], rtol=0, atol=1e-14 * np.abs(z['ref_f']).max())
    b = O.BEMRetOracle(gr, [VAC, DRUDE], (2, 1)).init(550.0)
    for nm in ['G1', 'G2', 'H1', 'H2']:
        ref = z[nm + '_550']
        assert np.max(np.abs(getattr(b, nm) - ref)) <= 1e-14 * np.abs(ref).max(), nm


def test_bemret_solution_tiny():
    z = golden('golden_tiny')
    s = _sphere('trisphere_32_10')
    cp = ComParticle([VAC, DRUDE], [s], [[2, 1]])
    b = O.BEMRetOracle(O.RetGreen(cp), [VAC, DRUDE], (2, 1))
    pol = np.array([[1, 0, 0], [0, 1, 0.]])
    dirs = np.array([[0, 0, 1], [0, 0, 1.]])
    for i, lam in enumerate(z['lams']):
        b.init(lam)
        em, km = VAC(lam)
        pot = O.planewave_ret_potential(s, cp.inout_faces, 1, em, lam, pol, dirs)
        sol = b.solve_vars(*b.excitation(*pot))
        for nm, val in zip(['sig1', 'h1', 'sig2', 'h2'], sol):
            ref = z[nm + '_%d' % i]
            tol = 1e-12 if nm.startswith('sig') else 1e-10
            assert np.max(np.abs(val - ref)) <= tol * np.abs(ref).max(), (lam, nm)
        ext = O.extinction(s, cp.inout_faces, 1, km, lam, sol, pol, dirs)
        assert np.allclose(ext, z['ext_%d' % i], rtol=1e-12)


def test_bemstat_tiny():
    z = golden('golden_tiny')
    s = _sphere('trisphere_32_10')
    cp = ComParticle([VAC, DRUDE], [s], [[2, 1]])
    st = O.BEMStatOracle(cp)
    assert np.array_equal(st.F, z['stat_F'])
    e1 = DRUDE(550.0)[0]
    sig = st.solve(np.full(s.n, e1), np.ones(s.n, complex), -s.nvec @ np.array([1, 0, 0.]))
    assert np.max(np.abs(sig - z['stat_sig_550'])) <= 1e-13 * np.abs(z['stat_sig_550']).max()
