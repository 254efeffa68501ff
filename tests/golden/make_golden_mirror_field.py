"""Golden fields of mirror-symmetric solutions, made by running the
reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_mirror_field.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_mirror_field.py

The two mirror cases of ``make_golden_mirror.py`` (quarter sphere, sym 'xy';
half sphere, sym 'x'), Drude gold in vacuum, ``PlaneWaveRetMirror`` pol x and
pol y along +z at 500 nm, solved by ``BEMRetMirror``; for every symmetry
value the solution (sig1, h1, sig2, h2, symval) and
``CompGreenRetMirror(p, p).field(sig, inout)`` (greenfun/compgreen_ret_mirror.py:
104-160) e and h for inout 1 and 2.  Only ``tests/`` read the output.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
LAM = 500.0
CASES = {'xy': ((0.0, np.pi / 2, 9), (0.0, np.pi, 17)),
         'x': ((-np.pi / 2, np.pi / 2, 9), (0.0, np.pi, 13))}


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
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret_mirror import BEMRetMirror
    from mnpbem.greenfun.compgreen_ret_mirror import CompGreenRetMirror
    from mnpbem.simulation.planewave_ret_mirror import PlaneWaveRetMirror

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    out = {'lam': LAM}
    for sym, (ph, th) in CASES.items():
        p = trispheresegment(np.linspace(*ph), np.linspace(*th), 20.0)
        cpm = ComParticleMirror(eps, [p], [[2, 1]], sym, (1,))
        exc = PlaneWaveRetMirror(np.array([[1.0, 0, 0], [0, 1.0, 0]]),
                                 np.array([[0, 0, 1.0], [0, 0, 1.0]]))
        sig, _ = BEMRetMirror(cpm).solve(exc(cpm, LAM))
        g = CompGreenRetMirror(cpm, cpm)
        for v, s in enumerate(sig.val):
            pre = '%s_%d_' % (sym, v)
            for key in ('sig1', 'h1', 'sig2', 'h2', 'symval'):
                out[pre + key] = np.asarray(getattr(s, key))
        for inout in (1, 2):
            f = g.field(sig, inout)
            for v, fv in enumerate(f.val):
                pre = '%s_%d_%d_' % (sym, v, inout)
                out[pre + 'e'], out[pre + 'h'] = np.asarray(fv.e), np.asarray(fv.h)
        print(sym, 'done', flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_mirror_field.npz'), **out)
    print('wrote golden_mirror_field.npz')


if __name__ == '__main__':
    main(reference_root())
