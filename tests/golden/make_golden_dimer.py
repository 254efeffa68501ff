"""Generate the dimer golden fixture by running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_dimer.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_dimer.py

Two gold Drude spheres trisphere(144, 10 nm) 2 nm apart on the x axis (centres
at x = -6 and +6 nm), inout [[2, 1], [2, 1]], in a host medium of eps = 1.77,
three plane waves (pol x / dir z, pol y / dir z, pol z / dir x).  BEMRet
(dense, FP64): extinction and scattering of the three excitations at 500, 600
and 700 nm, and sigma/h at 600 nm -- the two-particle connectivity of the
Green-function assembly and the embedding-medium wavenumbers of the
excitation and far field.

Output: ``golden_dimer.npz``.  Only ``tests/`` read it.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
EPS_HOST = 1.77
LAMS = (500.0, 600.0, 700.0)


def main(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    s1 = trisphere(144, 10.0).shift([-6.0, 0.0, 0.0])
    s2 = trisphere(144, 10.0).shift([6.0, 0.0, 0.0])
    cp = ComParticle([EpsConst(EPS_HOST), EpsDrude(*DRUDE)], [s1, s2], [[2, 1], [2, 1]], 1, 2)
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0], [1.0, 0, 0]])
    exc = PlaneWaveRet(pol, dirs)
    bem = BEMRet(cp)
    out = {'lams': np.array(LAMS)}
    ext, sca = [], []
    for enei in LAMS:
        sig, bem = bem.solve(exc.potential(cp, enei))
        ext.append(np.asarray(exc.extinction(sig)))
        sca.append(np.asarray(exc.scattering(sig)[0] if isinstance(exc.scattering(sig), tuple)
                              else exc.scattering(sig)))
        if enei == 600.0:
            for name in ('sig1', 'sig2', 'h1', 'h2'):
                out[name] = np.asarray(getattr(sig, name))
    out['ext'] = np.array(ext)
    out['sca'] = np.array(sca)
    print('ext', out['ext'])
    print('sca', out['sca'])
    np.savez_compressed(os.path.join(HERE, 'golden_dimer.npz'), **out)
    print('wrote golden_dimer.npz')


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


if __name__ == '__main__':
    main(reference_root())
