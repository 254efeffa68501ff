"""Golden tabulated dielectric functions and a MATLAB-pinned spectrum that uses
one, made from the reference (PyMNPBEM) checkout.

    python tests/golden/make_golden_epstable.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_golden_epstable.py

``golden_epstable.npz`` holds, for the reference's gold.dat (Johnson &
Christy) and silverpalik.dat tables:

* the table rows (energy in eV, n, k) as its reader parses them;
* ``EpsTable(...)(enei)`` of the reference (mnpbem/materials/eps_table.py) on
  a 181-point wavelength grid 250-1600 nm (eps and k);

the 20 nm gold sphere spectrum of the reference's validation case
validation/03_bemret/sphere (trisphere(144, 20) curved, EpsTable('gold.dat')
in vacuum, plane wave pol x along z, 41 wavelengths 400-800 nm): extinction
and scattering from its data/bemret_matlab.csv (MATLAB MNPBEM) and
data/bemret_python.csv (the reference); the direct and iterative extinction
of validation/08_iterative/{sphere,rod} (data/ret_matlab.csv and
data/ret_python.csv; the rod is trirod(10, 40, [15, 15, 15]) made curved by
ComParticle(..., interp='curv')), the reference's face geometry of that
curved rod (pos, nvec, area), and extinction and scattering of both cases
from the reference's current code run here (``ref_*``).  Only ``tests/``
read the output.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = ('gold.dat', 'silverpalik.dat')


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


def parse(path):
    rows = []
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line[0] in '%#':
                continue
            try:
                vals = [float(v) for v in line.split()]
            except ValueError:
                continue
            if len(vals) >= 3:
                rows.append(vals[:3])
    return np.asarray(rows)


def main(ref_root):
    os.environ.setdefault('NUMBA_CACHE_DIR', '/tmp/numba_cache')
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.materials.eps_table import EpsTable
    out = {'enei': np.linspace(250.0, 1600.0, 181)}
    for name in TABLES:
        key = name.split('.')[0]
        out[key + '_table'] = parse(os.path.join(ref_root, 'mnpbem', 'materials', 'data', name))
        eps, k = EpsTable(name)(out['enei'])
        out[key + '_eps'] = np.asarray(eps)
        out[key + '_k'] = np.asarray(k)
    vd = os.path.join(ref_root, 'validation', '03_bemret', 'sphere', 'data')
    for src in ('matlab', 'python'):
        d = np.loadtxt(os.path.join(vd, 'bemret_%s.csv' % src), delimiter=',', skiprows=1)
        out['sphere_lams'] = d[:, 0]
        out['sphere_ext_' + src] = d[:, 1]
        out['sphere_sca_' + src] = d[:, 2]
    for case in ('sphere', 'rod'):
        vd = os.path.join(ref_root, 'validation', '08_iterative', case, 'data')
        for src in ('matlab', 'python'):
            d = np.loadtxt(os.path.join(vd, 'ret_%s.csv' % src), delimiter=',', skiprows=1)
            out['iter_%s_lams' % case] = d[:, 0]
            out['iter_%s_direct_%s' % (case, src)] = d[:, 1]
            out['iter_%s_iter_%s' % (case, src)] = d[:, 2]
    from mnpbem.geometry import ComParticle, trirod
    from mnpbem.materials.eps_const import EpsConst
    cp = ComParticle([EpsConst(1.0), EpsTable('gold.dat')], [trirod(10.0, 40.0, n=[15, 15, 15])],
                     [[2, 1]], 1, interp='curv')
    out['rod_pos'] = np.asarray(cp.pos)
    out['rod_nvec'] = np.asarray(cp.nvec)
    out['rod_area'] = np.asarray(cp.area)
    # the reference's current code on both cases (the data/*_python.csv files
    # of its validation folders predate it: they sit up to 1e-7 (sphere
    # scattering) and 6.7e-6 (rod extinction) from MATLAB, the current code
    # within 1e-10)
    from mnpbem.bem import BEMRet
    from mnpbem.geometry import trisphere
    from mnpbem.simulation import PlaneWaveRet
    exc = PlaneWaveRet(np.array([[1.0, 0.0, 0.0]]), np.array([[0.0, 0.0, 1.0]]))
    cases = {'sphere': ComParticle([EpsConst(1.0), EpsTable('gold.dat')], [trisphere(144, 20)],
                                   [[2, 1]], 1, interp='curv'), 'rod': cp}
    for case, part in cases.items():
        bem = BEMRet(part)
        ext, sca = [], []
        for lam in out['iter_%s_lams' % case]:
            sig, bem = bem.solve(exc.potential(part, float(lam)))
            ext.append(float(np.real(np.ravel(exc.extinction(sig))[0])))
            sv = exc.scattering(sig)
            sca.append(float(np.real(np.ravel(sv[0] if isinstance(sv, tuple) else sv)[0])))
        out['ref_%s_ext' % case] = np.asarray(ext)
        out['ref_%s_sca' % case] = np.asarray(sca)
        print(case, 'done', flush=True)
    np.savez_compressed(os.path.join(HERE, 'golden_epstable.npz'), **out)
    print('wrote golden_epstable.npz')


if __name__ == '__main__':
    main(reference_root())
