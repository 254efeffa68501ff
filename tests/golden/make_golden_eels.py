"""Golden electron-beam (EELS) excitations and loss probabilities, made by
running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_eels.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_eels.py

Geometry: trisphere(144, 20) (284 curved faces, the generator's default
interpolation), Drude gold in vacuum.
Electron beams along z, 200 keV (vel = EELSBase.ene2vel(2e5)), width 0.5 nm,
default cutoff, in three impact sets:

* ``A`` aloof: (15, 0) and (0, 12.5);
* ``B`` mixed: (15, 0) aloof and (3, 2) through the sphere;
* ``C`` penetrating: (3, 2) and (-4, 1.5).

For each set and 520 / 650 nm, ``golden_eels.npz`` holds ``EELSRet``
(mnpbem/simulation/eels_ret.py:24) potentials phi1, phi1p, a1, a1p, phi2,
phi2p, a2, a2p (eels_ret.py:149), the dense ``BEMRet`` solution sig1, sig2,
h1, h2, ``loss`` (psurf, pbulk; eels_ret.py:296), ``rad`` (prad;
eels_ret.py:468) and ``field(p, enei, inout=2)`` (e, h; eels_ret.py:506),
plus the beam set-up of ``EELSBase`` (eels_base.py:73): the adjusted impact
parameters, the z segments inside the particle with their impact and
medium indices, and the refinement mask.

The reference's crossing test uses matplotlib's ``Path``; fixtures are made
with the ray-casting stand-in under ``mplstub/`` (no impact parameter lies on
a face edge).  Only ``tests/`` read the output.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DRUDE = (10.0, 9.065, 0.0708)
LAMS = (520.0, 650.0)
SETS = {'A': [[15.0, 0.0], [0.0, 12.5]],
        'B': [[15.0, 0.0], [3.0, 2.0]],
        'C': [[3.0, 2.0], [-4.0, 1.5]]}


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
    from mnpbem.simulation.eels_ret import EELSRet
    from mnpbem.simulation.eels_base import EELSBase

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    cp = ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1)
    vel = EELSBase.ene2vel(200e3)
    out = {'n': cp.n, 'lams': np.array(LAMS), 'vel': vel, 'width': 0.5}
    bem = BEMRet(cp)
    for name, imp in SETS.items():
        exc = EELSRet(cp, np.array(imp), 0.5, vel)
        out[name + '_impact_in'] = np.array(imp)
        out[name + '_impact'] = np.asarray(exc.impact)
        out[name + '_z'] = np.asarray(exc._z).reshape(-1, 2)
        out[name + '_indimp'] = np.asarray(exc._indimp, dtype=np.int64)
        out[name + '_indmat'] = np.asarray(exc._indmat, dtype=np.int64)
        out[name + '_indquad'] = np.asarray(exc._indquad)
        out[name + '_path'] = np.asarray(exc.path())
        for i, lam in enumerate(LAMS):
            pre = '%s_%d_' % (name, i)
            pot = exc.potential(cp, lam)
            for key in ('phi1', 'phi1p', 'a1', 'a1p', 'phi2', 'phi2p', 'a2', 'a2p'):
                out[pre + key] = np.asarray(getattr(pot, key))
            sig, bem = bem.solve(pot)
            for key in ('sig1', 'sig2', 'h1', 'h2'):
                out[pre + key] = np.asarray(getattr(sig, key))
            psurf, pbulk = exc.loss(sig)
            out[pre + 'psurf'], out[pre + 'pbulk'] = np.asarray(psurf), np.asarray(pbulk)
            out[pre + 'prad'] = np.asarray(exc.rad(sig)[0])
            f = exc.field(cp, lam, inout=2)
            out[pre + 'e'], out[pre + 'h'] = np.asarray(f.e), np.asarray(f.h)
            print(name, lam, 'psurf', psurf, 'pbulk', pbulk, 'prad', out[pre + 'prad'],
                  flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_eels.npz'), **out)
    print('wrote golden_eels.npz')


if __name__ == '__main__':
    main(reference_root())
