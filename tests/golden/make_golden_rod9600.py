"""Golden iterative (H-matrix) solution of a 9600-face gold rod, made by
running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_rod9600.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_rod9600.py

The 25,152-face rod of the iterative benchmark does not fit the reference's
dense caches in 62 GB of host memory, so the reference is run on the largest
rod of the same family that does: trirod(20, 80, [61, 31, 101]) = 9600 flat
faces, Drude gold in vacuum, plane wave along the rod axis (pol x, dir z).

Output ``golden_rod9600.npz``:

* ``BEMRetIter`` (mnpbem/bem/bem_ret_iter.py:1636) with hmatrix=True, cleaf 64,
  htol 1e-6, preconditioner 'none', GMRES tol 1e-6, at 600 nm: sig1, sig2, h1,
  h2, extinction, scattering, the number of operator applications GMRES made
  and the ranks of the G1 low-rank blocks;
* the dense ``BEMRet`` (mnpbem/bem/bem_ret.py:1569) extinction and scattering
  at the same wavelength (how far the H-matrix solve sits from dense).

Only ``tests/`` read the output; nothing at run time imports the reference.
"""

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
ENEI = 600.0


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
    from mnpbem.geometry.mesh_generators import trirod
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret_iter import BEMRetIter
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    rod = trirod(20.0, 80.0, [61, 31, 101])
    cp = ComParticle(eps, [rod], [[2, 1]], 1)
    out = {'n': rod.nfaces, 'enei': ENEI}
    exc = PlaneWaveRet(np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 0.0, 1.0]]))

    t0 = time.time()
    bem = BEMRetIter(cp, hmatrix=True, cleaf=64, htol=1e-6, preconditioner='none', tol=1e-6,
                     maxit=200)
    count = {'n': 0}
    orig = bem._afun

    def counted(v):
        count['n'] += 1
        return orig(v)

    bem._afun = counted
    sig, _ = bem.solve(exc.potential(cp, ENEI))
    out['iter_sig1'] = np.asarray(sig.sig1)
    out['iter_sig2'] = np.asarray(sig.sig2)
    out['iter_h1'] = np.asarray(sig.h1)
    out['iter_h2'] = np.asarray(sig.h2)
    out['iter_ext'] = np.asarray(exc.extinction(sig))
    out['iter_sca'] = np.asarray(exc.scattering(sig)[0])
    out['iter_matvecs'] = np.array(count['n'])
    out['iter_G1_rank'] = np.array([u.shape[1] for u in bem._G1.lhs], dtype=np.int64)
    out['iter_s'] = time.time() - t0
    print('iterative: matvecs', count['n'], 'ext', out['iter_ext'], 'sca', out['iter_sca'],
          '%.1fs' % out['iter_s'], flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_rod9600.npz'), **out)
    del bem

    t0 = time.time()
    bemd = BEMRet(cp)
    sig, _ = bemd.solve(exc.potential(cp, ENEI))
    out['dense_ext'] = np.asarray(exc.extinction(sig))
    out['dense_sca'] = np.asarray(exc.scattering(sig)[0])
    out['dense_s'] = time.time() - t0
    print('dense: ext', out['dense_ext'], 'sca', out['dense_sca'], '%.1fs' % out['dense_s'],
          flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_rod9600.npz'), **out)
    print('wrote golden_rod9600.npz')


if __name__ == '__main__':
    main(reference_root())
