"""Golden quasistatic dipole excitations, point Green function fields and
decay rates, made by running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_dipole_stat.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_dipole_stat.py

Geometry: trisphere(144, 20) (284 faces), Drude gold in a host of
eps = 1.5.  Five dipole positions given to ``ComPoint(p, pos)``
(mnpbem/geometry/compoint.py:186): three outside (one 2 nm above the
surface, where point-face pairs are refined, one 5 nm off, one far), two
inside the gold.  Dipole moments: the default unit triple (ndip = 3).

For 500 and 620 nm, ``golden_dipole_stat.npz`` holds ``DipoleStat``
(mnpbem/simulation/dipole_stat.py:24) ``potential`` phip and ``field`` e at
the faces, the dense ``BEMStat`` solution sig, ``decayrate`` (tot, rad,
rad0) and ``CompGreenStat(pt, p).field(sig)`` (greenfun/compgreen_stat.py:974)
e at the points.  (``DipoleStat.farfield`` of the reference imports a module
that does not exist, ``mnpbem.particle``, and raises; it has no fixture.)
Only ``tests/`` read the output.
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
    import warnings
    warnings.simplefilter('ignore')
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.geometry.compoint import ComPoint
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_stat import BEMStat
    from mnpbem.greenfun import CompGreenStat
    from mnpbem.simulation.dipole_stat import DipoleStat

    eps = [EpsConst(EPS_HOST), EpsDrude(*DRUDE)]
    cp = ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1)
    pt = ComPoint(cp, POS)
    dip = DipoleStat(pt)
    bem = BEMStat(cp)
    out = {'n': cp.n, 'lams': np.array(LAMS), 'pos_in': POS, 'pt_pos': np.asarray(pt.pos)}
    for i, lam in enumerate(LAMS):
        pre = '%d_' % i
        exc = dip(cp, lam)
        out[pre + 'phip'] = np.asarray(exc.phip)
        out[pre + 'e_faces'] = np.asarray(dip.field(cp, lam).e)
        sig, bem = bem.solve(exc)
        out[pre + 'sig'] = np.asarray(sig.sig)
        tot, rad, rad0 = dip.decayrate(sig)
        out[pre + 'tot'], out[pre + 'rad'], out[pre + 'rad0'] = tot, rad, rad0
        g = CompGreenStat(pt, cp)
        out[pre + 'e_pts'] = np.asarray(g.field(sig).e)
        print(lam, 'tot', tot[:, 0], flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_dipole_stat.npz'), **out)
    print('wrote golden_dipole_stat.npz')


if __name__ == '__main__':
    main(reference_root())
