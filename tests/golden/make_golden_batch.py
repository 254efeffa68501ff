"""Golden spectra of a small uneven particle set, made by running the
reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_batch.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_batch.py

Five gold Drude particles in a host of eps = 1.77, each solved by the
reference's dense ``BEMRet`` (mnpbem/bem/bem_ret.py:1569) at 450, 550 and
700 nm for three plane waves (pol x / dir z, pol y / dir z, pol z / dir x):

* two spheres trisphere(144, 18) and trisphere(144, 31.5) (284 faces each),
* two rods of 448 flat faces with the same grid (17, 9, 13) but different
  diameter / length (12 / 40 nm and 20 / 70 nm), their meshes taken from
  ``mnpbem_b200.geometry.rod_mesh`` so both codes solve the same surface,
* a dimer of two trisphere(144, 14) with a 2 nm gap (568 faces).

Equal face counts put the two spheres, and the two rods, into one batch of
the batched GPU solver.  Output ``golden_batch.npz``: ext and sca
(particle, wavelength, polarisation) and sig2 of the first polarisation of
every particle at 550 nm.  Only ``tests/`` read it.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRUDE = (10.0, 9.065, 0.0708)
EPS_HOST = 1.77
LAMS = (450.0, 550.0, 700.0)
SPHERES = ((144, 18.0), (144, 31.5))
RODS = ((12.0, 40.0, (17, 9, 13)), (20.0, 70.0, (17, 9, 13)))
DIMER = (144, 14.0, 2.0)


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


def main(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ROOT)
    from mnpbem_b200.geometry import rod_mesh          # mesh arrays only
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere
    from mnpbem.geometry.particle import Particle
    from mnpbem.geometry.comparticle import ComParticle
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret import BEMRet
    from mnpbem.simulation.planewave_ret import PlaneWaveRet

    eps = [EpsConst(EPS_HOST), EpsDrude(*DRUDE)]
    parts = []
    for nv, d in SPHERES:
        parts.append(ComParticle(eps, [trisphere(nv, d)], [[2, 1]], 1))
    for d, h, n in RODS:
        v, f = rod_mesh(d, h, n)
        parts.append(ComParticle(eps, [Particle(v, f)], [[2, 1]], 1))
    nv, d, gap = DIMER
    c = 0.5 * (d + gap)
    parts.append(ComParticle(eps, [trisphere(nv, d).shift([-c, 0, 0]),
                                   trisphere(nv, d).shift([c, 0, 0])], [[2, 1], [2, 1]], 1, 2))
    exc = PlaneWaveRet(np.array([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]]),
                       np.array([[0, 0, 1.0], [0, 0, 1.0], [1.0, 0, 0]]))
    ext = np.zeros((len(parts), len(LAMS), 3))
    sca = np.zeros_like(ext)
    out = {'lams': np.array(LAMS), 'faces': np.array([p.n for p in parts])}
    for i, cp in enumerate(parts):
        bem = BEMRet(cp)
        for j, lam in enumerate(LAMS):
            sig, bem = bem.solve(exc.potential(cp, lam))
            ext[i, j] = np.asarray(exc.extinction(sig))
            s = exc.scattering(sig)
            sca[i, j] = np.asarray(s[0] if isinstance(s, tuple) else s)
            if lam == 550.0:
                out['sig2_%d' % i] = np.asarray(sig.sig2)[:, 0]
        print('particle', i, cp.n, 'faces, ext', ext[i, :, 0], flush=True)
    out.update(ext=ext, sca=sca)
    np.savez_compressed(os.path.join(HERE, 'golden_batch.npz'), **out)
    print('wrote golden_batch.npz')


if __name__ == '__main__':
    main(reference_root())
