"""Batched solves of particles of uneven size (BatchedBEMRet) against the
reference's dense BEMRet of each particle (golden_batch.npz): two spheres
that share a face count (one batch, different geometry and normals), two
rods likewise, and a dimer, three plane waves, three wavelengths, host
eps 1.77.  Mixed precision with FP64 refinement at 1e-8: extinction and
scattering within 1e-6, sigma within 1e-6."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _particles():
    from mnpbem_b200.geometry import ComParticle, trirod, trisphere
    from mnpbem_b200.materials import EpsConst, EpsDrude
    eps = [EpsConst(1.77), EpsDrude(10.0, 9.065, 0.0708)]
    ps = [ComParticle(eps, [trisphere(144, d)], [[2, 1]], 1) for d in (18.0, 31.5)]
    ps += [ComParticle(eps, [trirod(d, h, (17, 9, 13))], [[2, 1]], 1)
           for d, h in ((12.0, 40.0), (20.0, 70.0))]
    s = trisphere(144, 14.0)
    ps.append(ComParticle(eps, [s.shift([-8.0, 0, 0]), s.shift([8.0, 0, 0])],
                          [[2, 1], [2, 1]], 1, 2))
    return ps


def test_batched_uneven_particles(gpu_ok, tmp_path):
    from mnpbem_b200.autotune import GemmTuner
    from mnpbem_b200.batch import BatchedBEMRet
    from mnpbem_b200.excitation import PlaneWaveRet
    z = golden('golden_batch')
    ps = _particles()
    assert [p.n for p in ps] == list(z['faces'])
    exc = PlaneWaveRet([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]],
                       [[0, 0, 1.0], [0, 0, 1.0], [1.0, 0, 0]])
    tuner = GemmTuner(path=str(tmp_path / 'tune.json'))
    solver = BatchedBEMRet(ps, refine_tol=1e-8, tuner=tuner)
    res = solver.solve_spectrum(exc, list(z['lams']), keep_solutions=True)
    ext, sca = res['ext'], res['sca']
    err_e = np.abs(ext - z['ext']) / np.abs(z['ext'])
    err_s = np.abs(sca - z['sca']) / np.abs(z['sca'])
    print('batched: ext err %.2e, sca err %.2e, batches %s, tuned %s'
          % (err_e.max(), err_s.max(), solver.stats, tuner.table))
    assert err_e.max() < 1e-6 and err_s.max() < 1e-6
    for i in range(len(ps)):
        s2 = res['solutions'][i][1].sig2[:, 0]
        ref = z['sig2_%d' % i]
        assert np.abs(s2 - ref).max() / np.abs(ref).max() < 1e-6, i
    # equal face counts shared a batch: 3 groups (284, 448, 568 faces)
    assert sorted(st['n'] for st in solver.stats) == [284, 448, 568]
    assert [st['entries'] for st in sorted(solver.stats, key=lambda d: d['n'])] == [6, 6, 3]
    # the tuner chose a configuration per (faces, batch) and stored it
    assert len(tuner.table) == 3
    assert (tmp_path / 'tune.json').exists()
    # a second sweep reuses the stored choices and gives the same cross sections
    res2 = solver.solve_spectrum(exc, list(z['lams']))
    assert np.abs(res2['ext'] - ext).max() / np.abs(ext).max() < 1e-9


def test_batched_padded_to_one_size(gpu_ok):
    """Particles of 284, 448 and 568 faces in one group (pad_ratio 2): every
    entry padded to 568 faces with an identity block, one factorisation for
    all 15 (particle, wavelength) entries; the same cross sections and
    charges as the reference."""
    from mnpbem_b200.batch import BatchedBEMRet
    from mnpbem_b200.excitation import PlaneWaveRet
    z = golden('golden_batch')
    ps = _particles()
    exc = PlaneWaveRet([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]],
                       [[0, 0, 1.0], [0, 0, 1.0], [1.0, 0, 0]])
    solver = BatchedBEMRet(ps, refine_tol=1e-8, tuner=None, pad_ratio=2.0)
    assert list(solver.groups) == [568]
    res = solver.solve_spectrum(exc, list(z['lams']), keep_solutions=True)
    err_e = np.abs(res['ext'] - z['ext']) / np.abs(z['ext'])
    err_s = np.abs(res['sca'] - z['sca']) / np.abs(z['sca'])
    assert err_e.max() < 1e-6 and err_s.max() < 1e-6
    for i in range(len(ps)):
        s2 = res['solutions'][i][1].sig2[:, 0]
        ref = z['sig2_%d' % i]
        assert s2.shape == ref.shape
        assert np.abs(s2 - ref).max() / np.abs(ref).max() < 1e-6, i
    assert solver.stats[0]['entries'] == 15 and solver.stats[0]['faces'] == [284, 448, 568]
