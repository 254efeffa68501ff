"""Tabulated dielectric functions (EpsTable, mnpbem/materials/eps_table.py)
against the reference's values on a 250-1600 nm grid for its gold.dat and
silverpalik.dat tables (golden_epstable.npz, made by
tests/golden/make_golden_epstable.py): same cubic splines of n and k over the
wavelength, so eps and k agree to rounding."""
import os

import numpy as np
import pytest

from conftest import golden
from mnpbem_b200.materials import EpsTable, eps_k


def write_table(tmp_path, name, rows):
    path = os.path.join(str(tmp_path), name)
    with open(path, 'w') as f:
        f.write('% energy (eV)  n  k\n')
        for e, n, k in rows:
            f.write('%.17g\t%.17g\t%.17g\n' % (e, n, k))
    return path


@pytest.mark.parametrize('key', ['gold', 'silverpalik'])
def test_epstable_matches_reference(tmp_path, key):
    g = golden('golden_epstable')
    tab = EpsTable(write_table(tmp_path, key + '.dat', g[key + '_table']))
    eps, k = tab(g['enei'])
    assert np.abs(eps - g[key + '_eps']).max() <= 1e-12 * np.abs(g[key + '_eps']).max()
    assert np.abs(k - g[key + '_k']).max() <= 1e-12 * np.abs(g[key + '_k']).max()
    e1, k1 = eps_k(tab, 633.0)
    assert isinstance(e1, complex) and abs(e1 - tab(633.0)[0]) == 0


def test_epstable_lookup(tmp_path, monkeypatch):
    g = golden('golden_epstable')
    write_table(tmp_path, 'gold.dat', g['gold_table'])
    with pytest.raises(FileNotFoundError):
        EpsTable('no_such_table.dat')
    monkeypatch.setenv('MNPBEM_MATERIALS', str(tmp_path))
    eps, _ = EpsTable('gold.dat')(g['enei'])
    assert np.allclose(eps, g['gold_eps'], rtol=1e-12, atol=0)


def test_curved_rod_geometry():
    """ComParticle(..., interp='curv') on the packaged trirod(10, 40, [15, 15,
    15]) uses the reference's midpoint mesh on the rod surface: face
    centroids, normals and areas equal the reference's (validation/
    08_iterative/rod's particle), and the flat rod keeps its own geometry."""
    import mnpbem_b200 as M
    g = golden('golden_epstable')
    rod = M.trirod(10.0, 40.0, (15, 15, 15))
    flat_pos = rod.pos.copy()
    cp = M.ComParticle([M.EpsConst(1.0), M.EpsDrude(10.0, 9.065, 0.0708)], [rod], [[2, 1]], 1,
                       interp='curv')
    assert rod.interp == 'curv'
    assert np.abs(cp.pos - g['rod_pos']).max() <= 1e-12
    assert np.abs(cp.nvec - g['rod_nvec']).max() <= 1e-12
    assert np.abs(cp.area - g['rod_area']).max() <= 1e-12 * g['rod_area'].max()
    assert np.abs(rod.flat().pos - flat_pos).max() == 0
    with pytest.raises(TypeError):
        M.ComParticle([M.EpsConst(1.0)], [rod], [[1, 1]], 1, refun=True)


def test_flat_midpoints_keep_flat_geometry():
    """curved() on a particle without midpoint vertices adds straight-edge
    midpoints and quad centres (the reference's midpoints('flat')): planar
    faces keep their flat centroid, normal and area."""
    import mnpbem_b200 as M
    v = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [2, 0, 0]], dtype=float)
    f = np.array([[0, 1, 2, 3], [1, 4, 2, np.nan]])
    p = M.Particle(v, f)
    pos, nvec, area = p.pos.copy(), p.nvec.copy(), p.area.copy()
    p.curved()
    assert p.faces2.shape == (2, 9) and p.verts2.shape[0] == 5 + 6 + 1
    assert np.allclose(p.pos, pos, atol=1e-14) and np.allclose(p.area, area, rtol=1e-14)
    assert np.allclose(np.abs(p.nvec[:, 2]), 1.0)
