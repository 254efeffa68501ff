"""Golden mirror-symmetry solutions, made by running the reference (PyMNPBEM)
on CPU.

    python tests/golden/make_golden_mirror.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_mirror.py

Two irreducible parts of a 20 nm sphere, Drude gold in vacuum, each closed
together with its mirror images (closed_args (1,)):

* ``xy``: trispheresegment(linspace(0, pi/2, 9), linspace(0, pi, 17), 20),
  the x >= 0, y >= 0 quarter (128 faces; 512 in the full sphere);
* ``x``: trispheresegment(linspace(-pi/2, pi/2, 9), linspace(0, pi, 13), 20),
  the x >= 0 half (96 faces; 192 in the full sphere).

``ComParticleMirror`` (mnpbem/geometry/comparticle_mirror.py:110),
``BEMRetMirror`` (mnpbem/bem/bem_ret_mirror.py:147) and
``PlaneWaveRetMirror`` (mnpbem/simulation/planewave_ret_mirror.py:8) with
pol x and pol y along +z, at 500 and 600 nm; and the quasistatic
``BEMStatMirror`` (mnpbem/bem/bem_stat_mirror.py:140) with
``PlaneWaveStatMirror`` (mnpbem/simulation/planewave_stat_mirror.py:9), pol x
and pol y, at the same wavelengths (keys ``stat_*``: sig and symval per
symmetry value, extinction, scattering, absorption).  ``golden_mirror.npz`` holds
the irreducible mesh (verts2, faces2), the full particle's centroids and
normals, per wavelength and symmetry component sig1, sig2, h1, h2 and the
symmetry values, and the extinction and scattering cross sections.  Only
``tests/`` read the output.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
LAMS = (500.0, 600.0)
CASES = {'xy': ((0.0, np.pi / 2, 9), (0.0, np.pi, 17)),
         'x': ((-np.pi / 2, np.pi / 2, 9), (0.0, np.pi, 13))}


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
    from mnpbem.geometry.mesh_generators import trispheresegment
    from mnpbem.geometry.comparticle_mirror import ComParticleMirror
    from mnpbem.materials.eps_const import EpsConst
    from mnpbem.materials.eps_drude import EpsDrude
    from mnpbem.bem.bem_ret_mirror import BEMRetMirror
    from mnpbem.simulation.planewave_ret_mirror import PlaneWaveRetMirror

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    pol = np.array([[1.0, 0, 0], [0, 1.0, 0]])
    dirs = np.array([[0, 0, 1.0], [0, 0, 1.0]])
    out = {'lams': np.array(LAMS)}
    for sym, (ph, th) in CASES.items():
        p = trispheresegment(np.linspace(*ph), np.linspace(*th), 20.0)
        cpm = ComParticleMirror(eps, [p], [[2, 1]], sym, (1,))
        out[sym + '_verts2'] = np.asarray(p.verts2)
        out[sym + '_faces2'] = np.asarray(p.faces2)
        out[sym + '_full_pos'] = np.asarray(cpm.pfull.pos)
        out[sym + '_full_nvec'] = np.asarray(cpm.pfull.nvec)
        bem = BEMRetMirror(cpm)
        exc = PlaneWaveRetMirror(pol, dirs)
        for i, lam in enumerate(LAMS):
            sig, bem = bem.solve(exc.potential(cpm, lam))
            for v, s in enumerate(sig.val):
                pre = '%s_%d_%d_' % (sym, i, v)
                for key in ('sig1', 'sig2', 'h1', 'h2'):
                    out[pre + key] = np.asarray(getattr(s, key))
                out[pre + 'symval'] = np.asarray(s.symval)
            out['%s_%d_ext' % (sym, i)] = np.asarray(exc.extinction(sig))
            sca = exc.scattering(sig)
            out['%s_%d_sca' % (sym, i)] = np.asarray(sca[0] if isinstance(sca, tuple) else sca)
            print(sym, lam, 'ext', out['%s_%d_ext' % (sym, i)], flush=True)
    from mnpbem.bem.bem_stat_mirror import BEMStatMirror
    from mnpbem.simulation.planewave_stat_mirror import PlaneWaveStatMirror
    for sym, (ph, th) in CASES.items():
        p = trispheresegment(np.linspace(*ph), np.linspace(*th), 20.0)
        cpm = ComParticleMirror(eps, [p], [[2, 1]], sym, (1,))
        bem = BEMStatMirror(cpm)
        exc = PlaneWaveStatMirror(pol)
        for i, lam in enumerate(LAMS):
            sig, bem = bem.solve(exc.potential(cpm, lam))
            for v, sv in enumerate(sig.val):
                out['stat_%s_%d_%d_sig' % (sym, i, v)] = np.asarray(sv.sig)
                out['stat_%s_%d_%d_symval' % (sym, i, v)] = np.asarray(sv.symval)
            for key, fn in (('ext', exc.extinction), ('sca', exc.scattering),
                            ('abs', exc.absorption)):
                val = fn(sig)
                out['stat_%s_%d_%s' % (sym, i, key)] = np.asarray(val[0] if isinstance(val, tuple)
                                                                 else val)
            print('stat', sym, lam, 'ext', out['stat_%s_%d_ext' % (sym, i)], flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_mirror.npz'), **out)
    print('wrote golden_mirror.npz')


if __name__ == '__main__':
    main(reference_root())
