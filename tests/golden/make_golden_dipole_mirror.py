"""Golden quasistatic mirror-symmetry dipole excitations and decay rates,
made by running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_dipole_mirror.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_dipole_mirror.py

Geometry: the two mirror cases of ``make_golden_mirror.py`` (a 20 nm sphere
as trispheresegment pieces, ``ComParticleMirror(eps, [p], [[2, 1]], sym,
(1,))`` with sym 'xy' and 'x'), Drude gold in vacuum.  Two dipole
positions outside the sphere, ``ComPoint(p, pos)``, the unit moment triple.

For 500 and 600 nm, ``golden_dipole_mirror.npz`` holds ``DipoleStatMirror``
(mnpbem/simulation/dipole_stat_mirror.py:15) potentials phip with their
symmetry values, the ``BEMStatMirror`` (mnpbem/bem/bem_stat_mirror.py:140)
surface charges, and ``decayrate`` (tot, rad, rad0); and the retarded
``DipoleRetMirror`` (mnpbem/simulation/dipole_ret_mirror.py:15) with
``BEMRetMirror`` (mnpbem/bem/bem_ret_mirror.py): potentials phi2p and a2p,
surface charges sig2 and currents h2 of every symmetry value, and
``decayrate`` (tot, rad).  Only ``tests/`` read the output.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
LAMS = (500.0, 600.0)
CASES = {'xy': ((0.0, np.pi / 2, 9), (0.0, np.pi, 17)),
         'x': ((-np.pi / 2, np.pi / 2, 9), (0.0, np.pi, 13))}
POS = np.array([[3.0, 4.0, 14.0], [13.0, 2.0, -3.0]])


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


def main(ref_root):
    import warnings
    warnings.simplefilter('ignore')
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trispheresegment
    from mnpbem.geometry.comparticle_mirror import ComParticleMirror
    from mnpbem.geometry.compoint import ComPoint
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_stat_mirror import BEMStatMirror
    from mnpbem.simulation.dipole_stat_mirror import DipoleStatMirror

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    out = {'lams': np.array(LAMS), 'pos_in': POS}
    for sym, (ph, th) in CASES.items():
        p = trispheresegment(np.linspace(*ph), np.linspace(*th), 20.0)
        cpm = ComParticleMirror(eps, [p], [[2, 1]], sym, (1,))
        pt = ComPoint(cpm, POS)
        out[sym + '_pt_pos'] = np.asarray(pt.pos)
        dip = DipoleStatMirror(pt)
        bem = BEMStatMirror(cpm)
        for i, lam in enumerate(LAMS):
            exc = dip(cpm, lam)
            sig, bem = bem.solve(exc)
            for v, (e, s) in enumerate(zip(exc.val, sig.val)):
                pre = 'stat_%s_%d_%d_' % (sym, i, v)
                out[pre + 'phip'] = np.asarray(e.phip)
                out[pre + 'symval'] = np.asarray(e.symval)
                out[pre + 'sig'] = np.asarray(s.sig)
            tot, rad, rad0 = dip.decayrate(sig)
            pre = 'stat_%s_%d_' % (sym, i)
            out[pre + 'tot'], out[pre + 'rad'], out[pre + 'rad0'] = tot, rad, rad0
            print(sym, lam, 'tot', tot[:, 0], flush=True)
    from mnpbem.bem.bem_ret_mirror import BEMRetMirror
    from mnpbem.simulation.dipole_ret_mirror import DipoleRetMirror
    for sym, (ph, th) in CASES.items():
        p = trispheresegment(np.linspace(*ph), np.linspace(*th), 20.0)
        cpm = ComParticleMirror(eps, [p], [[2, 1]], sym, (1,))
        pt = ComPoint(cpm, POS)
        dip = DipoleRetMirror(pt)
        bem = BEMRetMirror(cpm)
        for i, lam in enumerate(LAMS):
            exc = dip(cpm, lam)
            sig, bem = bem.solve(exc)
            for v, (e, s) in enumerate(zip(exc.val, sig.val)):
                pre = 'ret_%s_%d_%d_' % (sym, i, v)
                out[pre + 'phi2p'] = np.asarray(e.phi2p)
                out[pre + 'a2p'] = np.asarray(e.a2p)
                out[pre + 'symval'] = np.asarray(e.symval)
                out[pre + 'sig2'] = np.asarray(s.sig2)
                out[pre + 'h2'] = np.asarray(s.h2)
            tot, rad = dip.decayrate(sig)[:2]
            pre = 'ret_%s_%d_' % (sym, i)
            out[pre + 'tot'], out[pre + 'rad'] = tot, rad
            print('ret', sym, lam, 'tot', tot[:, 0], flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_dipole_mirror.npz'), **out)
    print('wrote golden_dipole_mirror.npz')


if __name__ == '__main__':
    main(reference_root())
