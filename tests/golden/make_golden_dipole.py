"""Golden dipole excitations, point Green functions and decay rates, made by
running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_dipole.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_dipole.py

Geometry: trisphere(144, 20) (284 curved faces), Drude gold in a host of
eps = 1.5.  Five dipole positions given to ``ComPoint(p, pos)``
(mnpbem/geometry/compoint.py:186), which groups them by medium: three
outside (one 2 nm above the surface, where point-face pairs are refined,
one 5 nm off, one far), two inside the gold.  Dipole moments: the default
unit triple (ndip = 3), so every excitation has K = 15 columns.

For 500 and 620 nm, ``golden_dipole.npz`` holds:

* ``DipoleRet.potential`` (mnpbem/simulation/dipole_ret.py:319): phi1,
  phi1p, a1, a1p, phi2, phi2p, a2, a2p at the faces;
* the dense ``BEMRet`` (mnpbem/bem/bem_ret.py:1569) solution sig1, sig2,
  h1, h2 (500 nm only);
* ``DipoleRet.decayrate`` (dipole_ret.py:517): tot, rad, rad0, and
  ``DipoleRet.scattering`` (dipole_ret.py:674): sca;
* ``CompGreenRet(pt, p).field(sig)`` (greenfun/compgreen_ret.py:912): e, h at
  the points;
* the dipoles' own fields at the faces from the outside points
  (``DipoleRet._dipolefield``, dipole_ret.py:238; the public ``field`` at
  dipole_ret.py:163 raises IndexError for groups of several points);
* ``CompGreenRet(pt, p).eval`` of G and Gp for face side 2 (the host).

Plus the ComPoint order (``pt_pos``, ``pt_inout``) and the point-face
refinement pairs of ``refinematrix(pt, p)`` (greenfun/refine_utils.py:29).  Only ``tests/`` read the
output; nothing at run time imports the reference.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
EPS_HOST = 1.5
LAMS = (500.0, 620.0)
POS = np.array([[0.0, 0.0, 12.0],      # 2 nm above the surface: refined pairs
                [15.0, 0.0, 0.0],      # 5 nm off
                [10.0, 30.0, 40.0],    # far
                [0.0, 0.0, 3.0],       # inside
                [2.0, -4.0, 1.0]])     # inside


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


def main(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.geometry.compoint import ComPoint
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.simulation.dipole_ret import DipoleRet
    from mnpbem.greenfun.compgreen_ret import CompGreenRet

    eps = [EpsConst(EPS_HOST), EpsDrude(*DRUDE)]
    cp = ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1, interp='curv')
    pt = ComPoint(cp, POS)
    out = {'n': cp.n, 'lams': np.array(LAMS), 'pos_in': POS,
           'pt_pos': np.asarray(pt.pos),
           'pt_inout': np.repeat(np.asarray(pt.inout), [q.n for q in pt.p])}
    from mnpbem.greenfun.refine_utils import refinematrix
    ir = refinematrix(pt, cp).tocoo()
    out['ir_rows'], out['ir_cols'], out['ir_kind'] = ir.row, ir.col, ir.data
    exc = DipoleRet(pt)
    bem = BEMRet(cp)
    g = CompGreenRet(pt, cp)
    for i, lam in enumerate(LAMS):
        pot = exc.potential(cp, lam)
        for key in ('phi1', 'phi1p', 'a1', 'a1p', 'phi2', 'phi2p', 'a2', 'a2p'):
            out['%s_%d' % (key, i)] = np.asarray(getattr(pot, key))
        sig, bem = bem.solve(pot)
        if i == 0:
            for key in ('sig1', 'sig2', 'h1', 'h2'):
                out['%s_%d' % (key, i)] = np.asarray(getattr(sig, key))
        tot, rad, rad0 = exc.decayrate(sig)
        out['tot_%d' % i], out['rad_%d' % i], out['rad0_%d' % i] = tot, rad, rad0
        out['sca_%d' % i] = np.asarray(exc.scattering(sig)[0])
        f = g.field(sig)
        out['pe_%d' % i], out['ph_%d' % i] = np.asarray(f.e), np.asarray(f.h)
        # the dipoles' own fields at the faces from the outside points; the
        # public DipoleRet.field raises IndexError for groups of more than one
        # point (dipole_ret.py:233 indexes with two 1-D arrays), so its field
        # function is called directly for the connected (host) group
        io = out['pt_inout']
        e_h, k_h = eps[0](lam)
        de, dh = exc._dipolefield(np.asarray(cp.pos), np.asarray(pt.pos)[io == 1],
                                  exc.dip[io == 1], e_h, k_h)
        out['de_%d' % i], out['dh_%d' % i] = np.asarray(de), np.asarray(dh)
        out['G_%d' % i] = np.asarray(g.eval(0, 1, 'G', lam))
        out['Gp_%d' % i] = np.asarray(g.eval(0, 1, 'Gp', lam))
        print('lambda', lam, 'tot', tot[:, 0], 'rad', rad[:, 0], flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_dipole.npz'), **out)
    print('wrote golden_dipole.npz')


if __name__ == '__main__':
    main(reference_root())
