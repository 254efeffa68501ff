"""Golden solutions of the 2884-face sphere, made by running the reference
(PyMNPBEM) on CPU.

    python tests/golden/make_golden_c1sig.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_c1sig.py

Output ``golden_c1_sig.npz``: trisphere(1444, 40) (2884 curved faces), Drude
gold (eps0 = 10, wp = 9.065 eV, gamma = 0.0708 eV) in vacuum, plane wave pol x
/ dir z, reference ``BEMRet`` (mnpbem/bem/bem_ret.py:1569) at 400, 470 (the
dipole resonance), 520, 600 and 800 nm: sig1, sig2, h1, h2, extinction
(planewave_ret.py:437) and scattering (planewave_ret.py:391).

Only ``tests/`` read the output; nothing at run time imports the reference.
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
LAMS = (400.0, 470.0, 520.0, 600.0, 800.0)


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
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    s = trisphere(1444, 40.0)
    cp = ComParticle([EpsConst(1.0), EpsDrude(*DRUDE)], [s], [[2, 1]], 1)
    t0 = time.time()
    bem = BEMRet(cp)
    out = {'n': s.nfaces, 'lams': np.array(LAMS), 'ctor_s': time.time() - t0}
    exc = PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    ext, sca = [], []
    for i, lam in enumerate(LAMS):
        t0 = time.time()
        sig, bem = bem.solve(exc.potential(cp, lam))
        out['sig1_%d' % i] = np.asarray(sig.sig1)
        out['sig2_%d' % i] = np.asarray(sig.sig2)
        out['h1_%d' % i] = np.asarray(sig.h1)
        out['h2_%d' % i] = np.asarray(sig.h2)
        ext.append(float(np.asarray(exc.extinction(sig)).ravel()[0]))
        sca.append(float(np.asarray(exc.scattering(sig)[0]).ravel()[0]))
        print('lambda', lam, 'ext', ext[-1], 'sca', sca[-1], '%.1fs' % (time.time() - t0),
              flush=True)
    out.update(ext=np.array(ext), sca=np.array(sca))
    np.savez_compressed(os.path.join(HERE, 'golden_c1_sig.npz'), **out)
    print('wrote golden_c1_sig.npz')


if __name__ == '__main__':
    main(reference_root())
