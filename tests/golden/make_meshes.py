"""Write the packaged meshes and far-field sphere used by the BEM path.

Run in a checkout that has the reference project (PyMNPBEM) available:

    python tests/golden/make_meshes.py /path/to/reference
    MNPBEM_REFERENCE=/path/to/reference python tests/golden/make_meshes.py

The meshes are the reference's own mesh-generator outputs (the BEM path takes
a ready surface mesh as input; mesh generation is not part of it):

* ``trisphere(n, d)`` -- mnpbem/geometry/mesh_generators.py:13, stored with its
  curved midpoint vertices (``verts2``/``faces2``, 9 face columns); also
  unit-diameter spheres of several n, which other diameters scale.  The
  underlying point sets are the reference's ``mnpbem/data/sphere*_tri.bin``.
* ``trirod(d, h, n)`` -- mnpbem/geometry/mesh_generators.py:592 (quads +
  triangles): the flat mesh (``verts``/``faces``) and, separately, its
  midpoint mesh on the rod surface (``verts2``/``faces2``, which carries its
  own copies of the corner vertices) that ``ComParticle(..., interp='curv')``
  uses.
* ``pinfty256`` -- the far-field integration sphere of
  mnpbem/spectrum/spectrum_ret.py:14 (``mnpbem/data/pinfty256.bin``): unit
  directions and their solid-angle weights.

Output: ``mnpbem_b200/data/meshes.npz``.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, '..', '..', 'mnpbem_b200', 'data')

SPHERES = [(32, 10.0), (60, 10.0), (144, 10.0), (144, 20.0), (256, 20.0), (1444, 40.0)]
# unit-diameter spheres: trisphere(n, D) for other diameters scales these
UNIT_SPHERES = (144, 256, 400, 576, 784, 1024, 1225)
RODS = [(20.0, 80.0, (31, 21, 41)), (20.0, 80.0, (61, 31, 101)), (20.0, 80.0, (97, 47, 171)),
        (10.0, 40.0, (15, 15, 15))]


def main(ref_root):
    sys.path.insert(0, ref_root)
    sys.path.insert(0, os.path.join(HERE, 'mplstub'))
    from mnpbem.geometry.mesh_generators import trisphere, trirod
    from mnpbem.spectrum.spectrum_ret import _load_pinfty_default

    out = {}
    for n, d in SPHERES:
        p = trisphere(n, d)
        key = 'trisphere_{}_{:g}'.format(n, d)
        out[key + '_verts'] = np.asarray(p.verts2, dtype=np.float64)
        out[key + '_faces'] = np.asarray(p.faces2, dtype=np.float64)
    for n in UNIT_SPHERES:
        p = trisphere(n, 1.0)
        key = 'trisphere_{}_1'.format(n)
        out[key + '_verts'] = np.asarray(p.verts2, dtype=np.float64)
        out[key + '_faces'] = np.asarray(p.faces2, dtype=np.float64)
    for d, h, n in RODS:
        p = trirod(d, h, list(n))
        key = 'trirod_{:g}_{:g}_{}_{}_{}'.format(d, h, *n)
        out[key + '_verts'] = np.asarray(p.verts, dtype=np.float64)
        out[key + '_faces'] = np.asarray(p.faces, dtype=np.float64)
        out[key + '_verts2'] = np.asarray(p.verts2, dtype=np.float64)
        out[key + '_faces2'] = np.asarray(p.faces2, dtype=np.float64)
    pin = _load_pinfty_default()
    out['pinfty256_nvec'] = np.asarray(pin.nvec, dtype=np.float64)
    out['pinfty256_area'] = np.asarray(pin.area, dtype=np.float64)
    np.savez_compressed(os.path.join(DATA, 'meshes.npz'), **out)
    print('wrote', sorted(out))


def reference_root():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get('MNPBEM_REFERENCE')
    if not root:
        raise SystemExit("give the reference checkout as the first argument or in "
                         "MNPBEM_REFERENCE")
    return root


if __name__ == '__main__':
    main(reference_root())
