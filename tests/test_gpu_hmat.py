"""H-matrix path on the GPU: ACA (mnpb_hmat_aca) against the reference's
ranks/factors and the ACA oracle, H-matrix products against the oracle and
the dense matrix, FP64 GMRES against a direct solve, and BEMRetIter against
the reference's BEMRetIter solutions (golden_hmat.npz) and the dense FP64
solver.

Tolerances: complex64 factor storage (2^-24 relative per entry) bounds the
product difference to the FP64 oracle at 1e-6; ACA at htol 1e-6 leaves
~2e-5 relative error against the dense matrix (the oracle shows 1.9e-5 on
this rod).  The reference's own dense-vs-H-matrix check allows 1e-3
(mnpbem/tests/test_hmatrix_iter.py:39-63)."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _rod():
    from mnpbem_b200.geometry import ComParticle, trirod
    from mnpbem_b200.materials import EpsConst, EpsDrude
    return ComParticle([EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)],
                       [trirod(20.0, 80.0, (31, 21, 41))], [[2, 1]], 1)


def _sphere():
    from mnpbem_b200.geometry import ComParticle, trisphere
    from mnpbem_b200.materials import EpsConst, EpsDrude
    return ComParticle([EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)],
                       [trisphere(144, 20.0)], [[2, 1]], 1)


@pytest.fixture(scope='module')
def rod_setup(gpu_ok):
    from mnpbem_b200.clustertree import BlockPartition, ClusterTree, make_kaware_fadmiss
    from mnpbem_b200.greenfun import CompGreenRet
    from mnpbem_b200.hmatrix import HMatrixGPU, HTopology
    cp = _rod()
    enei = 650.0
    t = CompGreenRet(cp, cp).tables
    n = t.n
    kblk, sblk = t.k_tables([enei])
    GG = torch.empty((2, 1, n, n), dtype=torch.complex128, device='cuda')
    HH = torch.empty((2, 1, n, n), dtype=torch.complex128, device='cuda')
    t.assemble(kblk, sblk, (GG[0], HH[0], GG[1], HH[1]), mode=0)
    tree = ClusterTree(cp.pos, 64)
    part = BlockPartition(tree, make_kaware_fadmiss(2 * np.pi / enei))
    topo = HTopology(part, 100, torch.device('cuda'))
    hms = [HMatrixGPU(topo, A, n, 1e-6) for A in (GG[0, 0], GG[1, 0], HH[0, 0], HH[1, 0])]
    torch.cuda.synchronize()
    dense = [A.cpu().numpy().T for A in (GG[0, 0], GG[1, 0], HH[0, 0], HH[1, 0])]
    return cp, tree, part, topo, hms, dense


def _explain(gpu_rank, orc, tol=1e-8):
    """Blocks whose GPU rank differs from the oracle's, each with the
    near-tie that explains it (None if nothing does)."""
    ranks = orc.ranks()
    return [(int(i), int(gpu_rank[i]), int(ranks[i]), orc.near_tie(i, gpu_rank[i], tol))
            for i in np.nonzero(gpu_rank != ranks)[0]]


def test_aca_ranks_and_factors(rod_setup):
    """GPU ACA ranks against the reference's (golden_hmat) and the oracle's.

    The GPU sums its norms and dot products in another order than NumPy's
    BLAS, so a block can only end at another rank where one of its decisions
    is a near-tie at rounding level (a stop test within 1e-8 of its threshold,
    or two pivot candidates within 1e-8); every differing block must be one of
    those, and the factors of equal-rank blocks must agree."""
    import torch
    from oracle import bem_oracle as bo
    from oracle.hmat_oracle import HMatrixOracle
    from mnpbem_b200.hmatrix import HMatrixGPU
    g = golden('golden_hmat')
    cp, tree, part, topo, hms, dense = rod_setup
    # 1. the reference's own input: the CPU-assembled G (the oracle on it
    #    reproduces every reference rank, tests/test_hmat_oracle.py)
    _, k_in = bo.eps_drude(10.0, 9.065, 0.0708, 650.0)
    Gc, _ = bo.RetGreen(cp).GF(k_in)
    orc_ref = HMatrixOracle(Gc, tree, part, htol=1e-6, kmax=100)
    assert np.array_equal(orc_ref.ranks(), g['aca_rank'])
    A = torch.from_numpy(np.ascontiguousarray(Gc.T)).cuda()
    hm_ref = HMatrixGPU(topo, A, cp.n, 1e-6)
    torch.cuda.synchronize()
    diff = _explain(hm_ref.rank_h, orc_ref)
    print('same input as the reference: %d of %d blocks differ: %s'
          % (len(diff), len(g['aca_rank']), diff))
    assert all(d[3] is not None for d in diff), diff
    # measured on B200: every rank equal on both inputs
    assert np.array_equal(hm_ref.rank_h, g['aca_rank'])
    # 2. the GPU-assembled G (what BEMRetIter uses) against the oracle on it
    gpu_rank = hms[0].rank_h
    orc = HMatrixOracle(dense[0], tree, part, htol=1e-6, kmax=100)
    diff = _explain(gpu_rank, orc)
    print('GPU-assembled input: %d blocks differ: %s' % (len(diff), diff))
    assert all(d[3] is not None for d in diff), diff
    assert np.array_equal(gpu_rank, g['aca_rank'])
    # 3. factors of the first 12 blocks against the reference's, where ranks agree
    ou = ov = 0
    for i in range(12):
        m, n, r = part.lowrank[i, 1], part.lowrank[i, 3], g['aca_rank'][i]
        Ur = g['aca_U'][ou:ou + m * r].reshape(m, r, order='F')
        Vr = g['aca_V'][ov:ov + n * r].reshape(n, r, order='F')
        ou += m * r
        ov += n * r
        if hm_ref.rank_h[i] != r:
            continue
        U, V = hm_ref.factors(i)
        assert np.abs(U - Ur).max() <= 1e-5 * np.abs(Ur).max()
        assert np.abs(V - Vr).max() <= 1e-5 * np.abs(Vr).max()


_ORC = {}


def _oracles(setup):
    from oracle.hmat_oracle import HMatrixOracle
    if 'h' not in _ORC:
        cp, tree, part, topo, hms, dense = setup
        _ORC['h'] = [HMatrixOracle(A, tree, part, htol=1e-6, kmax=100) for A in dense]
    return _ORC['h']


@pytest.mark.parametrize('nc', [1, 4, 12])
def test_hmat_matvec(rod_setup, nc):
    from mnpbem_b200.hmatrix import hmat_matvec
    from oracle.hmat_oracle import HMatrixOracle
    cp, tree, part, topo, hms, dense = rod_setup
    n = cp.n
    rng = np.random.default_rng(nc)
    X = rng.standard_normal((4, nc, n)) + 1j * rng.standard_normal((4, nc, n))
    xs = [torch.from_numpy(X[i]).cuda() for i in range(4)]
    ys = [torch.empty((nc, n), dtype=torch.complex128, device='cuda') for _ in range(4)]
    hmat_matvec(hms, xs, ys, nc)
    torch.cuda.synchronize()
    for i in range(4):
        y = ys[i].cpu().numpy().T
        ref = dense[i] @ X[i].T
        err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
        assert err < 1e-3, (i, err)
        orc = _oracles(rod_setup)[i]
        if np.array_equal(orc.ranks(), hms[i].rank_h):
            ref = orc.matvec(X[i].T)
            err = np.linalg.norm(y - ref) / np.linalg.norm(ref)
            assert err < 1e-6, (i, err)


def test_gmres_against_direct_solve(gpu_ok):
    from mnpbem_b200.bem_iter import gmres
    rng = np.random.default_rng(3)
    L = 600
    A = 2.0 * np.eye(L) + (rng.standard_normal((L, L)) + 1j * rng.standard_normal((L, L))) \
        * 0.3 / np.sqrt(L)
    b = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    xref = np.linalg.solve(A, b)
    dA = torch.from_numpy(A).cuda()
    db = torch.from_numpy(b).cuda()
    op = lambda v: dA @ v
    x, flag, relres, it = gmres(op, db, tol=1e-12, maxit=50, restart=8)
    assert flag == 0 and relres <= 1e-12 and it[0] > 1      # restarted at least once
    assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-10
    Ai = torch.from_numpy(np.linalg.inv(A)).cuda()
    x, flag, relres, it = gmres(op, db, tol=1e-10, maxit=10, apply_M=lambda v: Ai @ v)
    assert flag == 0 and it[1] <= 2
    assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-9


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def test_bemretiter_hmatrix_rod(gpu_ok):
    from mnpbem_b200 import BEMRet
    from mnpbem_b200.bem_iter import BEMRetIter
    from mnpbem_b200.excitation import PlaneWaveRet
    g = golden('golden_hmat')
    cp = _rod()
    exc = PlaneWaveRet([[1.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
    enei = 650.0
    bem = BEMRetIter(cp, hmatrix=True, cleaf=64, htol=1e-6, preconditioner='none', tol=1e-6,
                     maxit=200)
    sig, _ = bem.solve(exc.potential(cp, enei))
    flag, relres, it = bem.info()
    assert flag[-1] == 0 and relres[-1] <= 1e-6
    nmv = bem.matvec_counts()[-1]
    assert abs(nmv - int(g['iter_h_matvecs'])) <= 0.25 * int(g['iter_h_matvecs']), nmv
    dense, _ = BEMRet(cp).solve(exc.potential(cp, enei))
    ext = exc.extinction(sig)
    ext_d = exc.extinction(dense)
    print('hmatrix rod: matvecs %d (reference %d), ext %.12g (reference H-matrix %.12g, dense '
          '%.12g)' % (nmv, int(g['iter_h_matvecs']), ext, float(g['iter_h_ext']), ext_d))
    for name in ('sig1', 'sig2', 'h1', 'h2'):
        print('  %s: vs reference H-matrix %.3e, vs dense %.3e' % (
            name, _rel(getattr(sig, name), g['iter_h_' + name]),
            _rel(getattr(sig, name), getattr(dense, name))))
    # parity with the reference's H-matrix solve (same ACA, same GMRES tolerance)
    assert abs(ext - float(g['iter_h_ext'])) < 1e-5 * abs(float(g['iter_h_ext']))
    for name in ('sig1', 'sig2', 'h1', 'h2'):
        assert _rel(getattr(sig, name), g['iter_h_' + name]) < 2e-5, name
    # ACA at htol 1e-6 costs both implementations ~0.5 % of the dense extinction
    assert abs(ext - ext_d) / abs(ext_d) < 1e-2


def test_bemretiter_dense_sphere(gpu_ok):
    from mnpbem_b200.bem_iter import BEMRetIter
    from mnpbem_b200.excitation import PlaneWaveRet
    g = golden('golden_hmat')
    cp = _sphere()
    exc = PlaneWaveRet([[1.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
    bem = BEMRetIter(cp, tol=1e-6)
    sig, _ = bem.solve(exc.potential(cp, 550.0))
    flag, relres, it = bem.info()
    assert flag[-1] == 0 and it[-1][1] <= 3
    for name in ('sig1', 'sig2', 'h1', 'h2'):
        assert _rel(getattr(sig, name), g['iter_d_' + name]) < 1e-8, name
    assert abs(exc.extinction(sig) - float(g['iter_d_ext'])) < 1e-8 * abs(float(g['iter_d_ext']))


def test_bemretiter_hmatrix_rod9600(gpu_ok):
    """trirod(20, 80, [61, 31, 101]) (9600 flat faces, the largest rod of the
    iterative family the reference can hold in 62 GB of host memory) at 600 nm
    against the reference's BEMRetIter (cleaf 64, htol 1e-6, unpreconditioned
    GMRES tol 1e-6) and its dense BEMRet (golden_rod9600.npz).

    * The two GMRES runs walk the same Krylov process: operator applications
      within 3 % of the reference's, extinction within 1e-6 and sigma within
      1e-4 of the reference's iterative solution (measured 1.1e-7 / 4e-6).
    * The GPU dense FP64 solve gives the reference's dense extinction to 1e-9.
    * The H-matrix solve (both implementations) sits 21 % from the dense one
      on this rod at htol 1e-6 -- a property of the ACA operator, not of the
      GMRES tolerance (tol 1e-10 leaves it unchanged): the products of the
      compressed G1 and G2 differ from the dense ones by 1.7e-4 and 1.5e-3
      (random vectors), because the ACA stopping rule ends some blocks
      early; only htol 1e-12 brings the solve within 0.2 %.  The GPU path must
      reproduce the reference's deviation to 1e-5 of the dense value."""
    from mnpbem_b200 import BEMRet
    from mnpbem_b200.bem_iter import BEMRetIter
    from mnpbem_b200.excitation import PlaneWaveRet
    from mnpbem_b200.geometry import ComParticle, trirod
    from mnpbem_b200.materials import EpsConst, EpsDrude
    g = golden('golden_rod9600')
    cp = ComParticle([EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)],
                     [trirod(20.0, 80.0, (61, 31, 101))], [[2, 1]], 1)
    assert cp.n == int(g['n'])
    exc = PlaneWaveRet([[1.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
    enei = float(g['enei'])
    bem = BEMRetIter(cp, hmatrix=True, cleaf=64, htol=1e-6, preconditioner='none', tol=1e-6,
                     maxit=200)
    sig, _ = bem.solve(exc.potential(cp, enei))
    flag, relres, it = bem.info()
    nmv = bem.matvec_counts()[-1]
    ext = exc.extinction(sig)
    ref_it, ref_d = float(g['iter_ext']), float(g['dense_ext'])
    errs = {name: _rel(getattr(sig, name), g['iter_' + name]) for name in ('sig1', 'sig2')}
    del bem, sig
    torch.cuda.empty_cache()
    dense, _ = BEMRet(cp).solve(exc.potential(cp, enei))
    ext_d = exc.extinction(dense)
    print('rod 9600, tol 1e-6: matvecs %d (reference %d), ext %.10g (reference iterative '
          '%.10g), sigma vs reference iterative %s; dense ext %.10g (reference dense %.10g)'
          % (nmv, int(g['iter_matvecs']), ext, ref_it, errs, ext_d, ref_d))
    assert flag[-1] == 0 and relres[-1] <= 1e-6
    assert abs(nmv - int(g['iter_matvecs'])) <= 0.03 * int(g['iter_matvecs'])
    assert abs(ext - ref_it) / abs(ref_it) < 1e-6
    assert max(errs.values()) < 1e-4
    assert abs(ext_d - ref_d) / abs(ref_d) < 1e-9
    assert abs((ext - ext_d) - (ref_it - ref_d)) < 1e-5 * abs(ref_d)


def test_gmres_augmented(gpu_ok):
    """GCRO augmentation (gmres(augment=...)): with the solution direction in
    the augmentation space the solve needs no Krylov step; with nearly
    dependent vectors (dropped) and random ones it still converges on the
    true residual to the direct solution."""
    from mnpbem_b200.bem_iter import _Counter, gmres
    rng = np.random.default_rng(11)
    L = 500
    A = 2.0 * np.eye(L) + (rng.standard_normal((L, L)) + 1j * rng.standard_normal((L, L))) \
        * 0.3 / np.sqrt(L)
    b = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    xref = np.linalg.solve(A, b)
    dA, db = torch.from_numpy(A).cuda(), torch.from_numpy(b).cuda()
    op = lambda v: dA @ v
    rv = lambda: torch.from_numpy(rng.standard_normal(L) + 1j * rng.standard_normal(L)).cuda()
    cnt = _Counter()
    x, flag, relres, it = gmres(op, db, tol=1e-10, maxit=50,
                                augment=[3.0 * torch.from_numpy(xref).cuda(), rv()], counter=cnt)
    assert flag == 0 and relres <= 1e-10 and it[1] == 0
    assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-9
    u = rv()
    x, flag, relres, it = gmres(op, db, tol=1e-11, maxit=50, restart=10,
                                augment=[u, u * (1 + 1e-12), rv(), rv()])
    assert flag == 0 and relres <= 1e-11
    assert np.linalg.norm(x.cpu().numpy() - xref) / np.linalg.norm(xref) < 1e-9
