"""Golden quasistatic electron-beam (EELS) excitations and loss
probabilities, made by running the reference (PyMNPBEM) on CPU.

    python tests/golden/make_golden_eels_stat.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_eels_stat.py

Geometry: trisphere(144, 20) (284 curved faces, the generator's default
interpolation), Drude gold in vacuum.  Electron beams along z, 200 keV
(vel = EELSBase.ene2vel(2e5)), width 0.5 nm, default cutoff, in three impact
sets:

* ``A`` aloof: (15, 0) and (0, 12.5);
* ``B`` mixed: (15, 0) aloof and (3, 2) through the sphere;
* ``C`` penetrating: (3, 2) and (-4, 1.5).

For each set and 520 / 650 nm, ``golden_eels_stat.npz`` holds ``EELSStat``
(mnpbem/simulation/eels_stat.py:23) potentials phi, phip
(eels_stat.py:107), the dense ``BEMStat`` solution sig, ``loss`` (psurf,
pbulk; eels_stat.py:163), and ``field(p, enei)`` (e; eels_stat.py:230).
Only ``tests/`` read the output.
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
    from mnpbem.bem.bem_stat import BEMStat
    from mnpbem.simulation.eels_stat import EELSStat
    from mnpbem.simulation.eels_base import EELSBase

    eps = [EpsConst(1.0), EpsDrude(*DRUDE)]
    cp = ComParticle(eps, [trisphere(144, 20.0)], [[2, 1]], 1)
    vel = EELSBase.ene2vel(200e3)
    out = {'n': cp.n, 'lams': np.array(LAMS), 'vel': vel, 'width': 0.5}
    bem = BEMStat(cp)
    for name, imp in SETS.items():
        exc = EELSStat(cp, np.array(imp), 0.5, vel)
        out[name + '_impact_in'] = np.array(imp)
        out[name + '_indimp'] = np.asarray(exc._indimp, dtype=np.int64)
        for i, lam in enumerate(LAMS):
            pre = '%s_%d_' % (name, i)
            pot = exc.potential(cp, lam)
            out[pre + 'phi'] = np.asarray(pot.phi)
            out[pre + 'phip'] = np.asarray(pot.phip)
            sig, bem = bem.solve(pot)
            out[pre + 'sig'] = np.asarray(sig.sig)
            psurf, pbulk = exc.loss(sig)
            out[pre + 'psurf'], out[pre + 'pbulk'] = np.asarray(psurf), np.asarray(pbulk)
            out[pre + 'e'] = np.asarray(exc.field(cp, lam).e)
            print(name, lam, 'psurf', psurf, 'pbulk', pbulk, flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_eels_stat.npz'), **out)
    print('wrote golden_eels_stat.npz')


if __name__ == '__main__':
    main(reference_root())
