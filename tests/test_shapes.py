"""Particle meshes of the batched workload and the batching bookkeeping
(host only, no GPU): the rod generator against the reference's packaged
trirod, closed outward surfaces, the seeded particle set, and how entries of
a face-count group are cut into batches and per-particle runs."""
import pytest
import numpy as np

from mnpbem_b200.geometry import Particle, rod_mesh, trirod, trisphere
from mnpbem_b200.shapes import random_particles


def _closed_outward(p, h):
    c = p.pos.copy()
    c[:, 2] = np.where(np.abs(c[:, 2]) <= h, 0.0, c[:, 2] - np.sign(c[:, 2]) * h)
    assert np.all(np.sum(p.nvec * c, axis=1) > 0)                 # outward
    assert np.abs((p.nvec * p.area[:, None]).sum(axis=0)).max() < 1e-8 * p.area.sum()


def test_rod_mesh_matches_reference_trirod():
    """rod_mesh(20, 80, (31, 21, 41)) is the reference's trirod surface: the
    same vertices, and face for face the same centroid, normal and area."""
    v, f = rod_mesh(20.0, 80.0, (31, 21, 41))
    p = Particle(v, f, interp='flat')
    q = trirod(20.0, 80.0, (31, 21, 41))                          # packaged reference output
    assert p.n == q.n == 2400 and v.shape == q.verts.shape
    from scipy.spatial import cKDTree
    d, j = cKDTree(q.pos).query(p.pos)
    assert d.max() < 1e-7 and len(set(j)) == q.n
    assert np.abs(p.area - q.area[j]).max() < 1e-7
    assert np.abs(p.nvec - q.nvec[j]).max() < 1e-7
    _closed_outward(p, 30.0)


def test_rod_mesh_shapes():
    for d, h, n in ((12.0, 40.0, (17, 9, 13)), (25.0, 31.0, (21, 11, 17)), (10.0, 120.0, (31, 16, 25))):
        v, f = rod_mesh(d, h, n)
        p = Particle(v, f, interp='flat')
        assert p.n == (n[0] - 1) * (2 * (n[1] - 1) + n[2] - 1)
        assert np.isnan(f[:, 3]).sum() == 2 * (n[0] - 1)              # pole triangles
        _closed_outward(p, 0.5 * (h - d))


def test_scaled_sphere_is_reference_sphere():
    a = trisphere(144, 20.0)                                      # packaged at this diameter
    b = Particle(*_unit(144), interp='curv')
    assert np.abs(a.pos - 20.0 * b.pos).max() < 1e-12
    assert np.abs(a.area - 400.0 * b.area).max() < 1e-10


def _unit(n):
    from mnpbem_b200.geometry import load_mesh
    return load_mesh('trisphere_%d_1' % n)


def test_random_particle_set():
    a = random_particles(64, seed=0)
    b = random_particles(64, seed=0)
    assert [d for _, d in a] == [d for _, d in b]
    faces = [d['faces'] for _, d in a]
    assert min(faces) >= 256 and max(faces) <= 3000
    assert {d['kind'] for _, d in a} == {'sphere', 'rod', 'dimer'}
    # discrete resolutions: particles share face counts
    assert len(set(faces)) < 20


def test_batches_and_runs():
    from mnpbem_b200.batch import BatchedBEMRet
    eneis = [400.0, 500.0, 600.0]
    runs = BatchedBEMRet._runs([7, 9, 11], eneis, 2, 8)
    assert runs == [(7, 0, [600.0]), (9, 1, [400.0, 500.0, 600.0]), (11, 4, [400.0, 500.0])]
    bs = BatchedBEMRet.__new__(BatchedBEMRet)
    bs.max_batch, bs.mem_bytes = 256, 10 ** 15
    spans, size = bs._batches(284, 41 * 5, 3)
    assert spans == [(0, 205)] and size == 205
    bs.max_batch = 100                       # equal batches, none above the cap
    spans, size = bs._batches(284, 41 * 5, 3)
    assert spans == [(0, 69), (69, 138), (138, 205)] and size == 69
    bs.mem_bytes = 40 * BatchedBEMRet.entry_bytes(2000, 3)
    spans, size = bs._batches(2000, 100, 3)
    assert size <= 40 and spans[-1][1] == 100 and all(b - a <= size for a, b in spans)


def test_padding_buckets():
    from mnpbem_b200.batch import BatchedBEMRet
    sizes = [284, 300, 448, 284, 520, 700, 720, 2446]
    assert BatchedBEMRet.buckets(sizes) == {284: [0, 3], 300: [1], 448: [2], 520: [4],
                                            700: [5], 720: [6], 2446: [7]}
    g = BatchedBEMRet.buckets(sizes, 1.25)
    assert g == {300: [0, 3, 1], 520: [2, 4], 720: [5, 6], 2446: [7]}
    assert all(max(sizes[i] for i in v) == k for k, v in g.items())
    assert sorted(i for v in g.values() for i in v) == list(range(len(sizes)))
    with pytest.raises(ValueError):
        BatchedBEMRet.buckets(sizes, 0.9)
