"""Mixed-precision path: TF32 tensor-core LU of planar FP32 matrices (relative
error of a cond ~ 3 solve below 1e-2: TF32 keeps 10 mantissa bits), and the
mixed BEMRet (TF32 factorisations + FP64 iterative refinement) against the
reference's golden fixtures.  Tolerances: the refined solution is held to the
FP64 operator's relative residual 1e-11, so sigma agrees with the reference
to 1e-9 and extinction / scattering to 1e-9 (1e-6)."""
import numpy as np
import pytest
import torch

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200 import _lib, bem, excitation
from mnpbem_b200._lib import call, ptr

pytestmark = pytest.mark.gpu
EPS = [M.EpsConst(1.0), M.EpsDrude(10.0, 9.065, 0.0708)]


def _cp(key):
    v, f = M.load_mesh(key)
    s = M.Particle(v, f, interp='curv' if f.shape[1] == 9 else 'flat')
    return M.ComParticle(EPS, [s], [[2, 1]]), s


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


@pytest.mark.parametrize('n,batch,nrhs', [(32, 1, 1), (100, 2, 3), (256, 3, 5), (300, 1, 40),
                                         (700, 2, 300), (130, 1, 130), (200, 150, 2)])
def test_getrf_getrs_c32p(gpu_ok, n, batch, nrhs):
    ld = (n + 3) // 4 * 4
    g = torch.Generator().manual_seed(7)
    # well conditioned (cond ~ 3): the TF32 updates bound the accuracy
    Ac = (torch.randn((batch, n, n), generator=g, dtype=torch.float64) +
          1j * torch.randn((batch, n, n), generator=g, dtype=torch.float64)) / (2 * n ** 0.5)
    Ac = Ac + 2 * torch.eye(n)
    X = (torch.randn((batch, n, nrhs), generator=g, dtype=torch.float64) +
         1j * torch.randn((batch, n, nrhs), generator=g, dtype=torch.float64))
    Bc = Ac @ X
    A = torch.zeros((batch, 2, n, ld), dtype=torch.float32)
    A[:, 0, :, :n] = Ac.real.transpose(1, 2).float()
    A[:, 1, :, :n] = Ac.imag.transpose(1, 2).float()
    B = torch.zeros((batch, 2, nrhs, ld), dtype=torch.float32)
    B[:, 0, :, :n] = Bc.real.transpose(1, 2).float()
    B[:, 1, :, :n] = Bc.imag.transpose(1, 2).float()
    A, B = A.cuda(), B.cuda()
    piv = torch.zeros((batch, n), dtype=torch.int32, device='cuda')
    info = torch.zeros(batch, dtype=torch.int32, device='cuda')
    wb = int(_lib.lib().mnpb_f32_workspace(n, batch))
    work = torch.empty(wb, dtype=torch.uint8, device='cuda')
    sh = _lib.stream_handle()
    call('mnpb_getrf_c32p', sh, n, batch, ptr(A), ld, n * ld, 2 * n * ld, ptr(piv), n, ptr(info),
         ptr(work), wb)
    call('mnpb_getrs_c32p', sh, n, batch, nrhs, ptr(A), ld, n * ld, 2 * n * ld, ptr(piv), n,
         ptr(B), ld, ld * nrhs, 2 * ld * nrhs, ptr(work), wb)
    torch.cuda.synchronize()
    assert info.sum().item() == 0
    Xg = (B[:, 0, :, :n].double() + 1j * B[:, 1, :, :n].double()).transpose(1, 2).cpu()
    err = ((Xg - X).abs().pow(2).sum() / X.abs().pow(2).sum()).sqrt().item()
    assert err < 1e-2, err


@pytest.mark.parametrize('n,batch', [(700, 2), (200, 150), (2884, 2)])
def test_getrf_c32p_pivoting(gpu_ok, n, batch):
    """Random complex matrices without a dominant diagonal, so partial
    pivoting moves rows at almost every step (the shared-memory slab leaves
    of 8 columns, of 4 columns for batches above the SM count, and the full
    2884-row leaf height): P A = L U to TF32 accuracy (relative to |L||U|),
    every multiplier |l_ij| <= sqrt(2) (pivots maximise |re| + |im|), and
    the pivot indices form a permutation."""
    ld = (n + 3) // 4 * 4
    g = torch.Generator().manual_seed(11 + n)
    Ac = (torch.randn((batch, n, n), generator=g, dtype=torch.float64) +
          1j * torch.randn((batch, n, n), generator=g, dtype=torch.float64))
    A = torch.zeros((batch, 2, n, ld), dtype=torch.float32)
    A[:, 0, :, :n] = Ac.real.transpose(1, 2).float()
    A[:, 1, :, :n] = Ac.imag.transpose(1, 2).float()
    A = A.cuda()
    piv = torch.zeros((batch, n), dtype=torch.int32, device='cuda')
    info = torch.zeros(batch, dtype=torch.int32, device='cuda')
    wb = int(_lib.lib().mnpb_f32_workspace(n, batch))
    work = torch.empty(wb, dtype=torch.uint8, device='cuda')
    call('mnpb_getrf_c32p', _lib.stream_handle(), n, batch, ptr(A), ld, n * ld, 2 * n * ld,
         ptr(piv), n, ptr(info), ptr(work), wb)
    torch.cuda.synchronize()
    assert info.sum().item() == 0
    F = (A[:, 0, :, :n].double() + 1j * A[:, 1, :, :n].double()).transpose(1, 2).cpu()
    pv = piv.cpu().numpy()
    for b in list(range(min(batch, 3))) + [batch - 1]:
        L = torch.tril(F[b], -1) + torch.eye(n, dtype=F.dtype)
        U = torch.triu(F[b])
        assert L.abs().max().item() <= 2 ** 0.5 * (1 + 1e-3)
        perm = np.arange(n)
        for c in range(n):
            p = int(pv[b, c])
            assert c <= p < n
            perm[[c, p]] = perm[[p, c]]
        assert sorted(perm.tolist()) == list(range(n))
        PA = Ac[b][torch.from_numpy(perm)]
        # backward error against |L||U| (TF32 storage of the factors alone
        # gives ~1e-5 here; a wrong interchange gives O(1))
        err = (torch.linalg.norm(PA - L @ U) / torch.linalg.norm(L.abs() @ U.abs())).item()
        assert err < 1e-3, (b, err)
        moved = int((pv[b] != np.arange(n)).sum())
        assert moved > n // 2, moved


@pytest.fixture(scope='module')
def tiny():
    cp, s = _cp('trisphere_32_10')
    return cp, bem.BEMRet(cp, precision='mixed'), golden('golden_tiny')


def test_mixed_bemret_tiny(gpu_ok, tiny):
    cp, b, z = tiny
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0], [0, 1, 0]], dir=[[0, 0, 1], [0, 0, 1]])
    for i, lam in enumerate(z['lams']):
        sig, _ = b.solve(exc.potential(cp, lam))
        assert rel(sig.sig1, z['sig1_%d' % i]) < 1e-9
        assert rel(sig.sig2, z['sig2_%d' % i]) < 1e-9
        assert rel(sig.h1, z['h1_%d' % i]) < 1e-7
        assert np.allclose(exc.extinction(sig), z['ext_%d' % i], rtol=1e-9)
        assert b._batch.relres.max() < 1e-11


def test_mixed_c0_spectrum(gpu_ok):
    cp, s = _cp('trisphere_144_20')
    z = golden('golden_c0')
    b = bem.BEMRet(cp, precision='mixed')
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=41)
    ext = np.array([exc.extinction(sg) for sg in sols])
    sca = np.array([exc.scattering(sg)[0] for sg in sols])
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-9
    assert np.max(np.abs(sca - z['sca']) / np.abs(z['sca'])) < 1e-9


def test_mixed_c1_2884_faces(gpu_ok):
    cp, s = _cp('trisphere_1444_40')
    z = golden('golden_c1')
    b = bem.BEMRet(cp, precision='mixed')
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=3)
    ext = np.array([exc.extinction(sg) for sg in sols])
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-6


def test_mixed_c1_sigma_five_wavelengths(gpu_ok):
    """trisphere(1444, 40) (2884 faces), the measured mixed path (TF32
    factorisations, FP64 refinement at the benchmark's refine_tol 1e-8)
    against the reference BEMRet at 400, 470 (resonance), 520, 600, 800 nm:
    extinction and scattering within 1e-6, sigma within
    1e-6 (max-norm relative)."""
    cp, s = _cp('trisphere_1444_40')
    z = golden('golden_c1_sig')
    b = bem.BEMRet(cp, precision='mixed', refine_tol=1e-8)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    sols = b.solve_spectrum(exc, list(z['lams']), batch=5)
    for i, sg in enumerate(sols):
        assert rel(sg.sig1, z['sig1_%d' % i]) < 1e-6, i
        assert rel(sg.sig2, z['sig2_%d' % i]) < 1e-6, i
    ext = np.array([exc.extinction(sg) for sg in sols]).ravel()
    sca = np.array([exc.scattering(sg)[0] for sg in sols]).ravel()
    assert np.max(np.abs(ext - z['ext']) / np.abs(z['ext'])) < 1e-6
    assert np.max(np.abs(sca - z['sca']) / np.abs(z['sca'])) < 1e-6


@pytest.mark.parametrize('n,batch', [(100, 2), (300, 3), (700, 2), (1000, 4)])
def test_getri_c32p(gpu_ok, n, batch):
    """Inverse from the TF32 LU (structured forward solve on the identity,
    diagonal-block inverses as leaves, column interchanges): A X = I to the
    TF32 bound of a cond ~ 3 matrix (relative Frobenius error < 1e-2)."""
    ld = (n + 3) // 4 * 4
    g = torch.Generator().manual_seed(n)
    Ac = (torch.randn((batch, n, n), generator=g, dtype=torch.float64) +
          1j * torch.randn((batch, n, n), generator=g, dtype=torch.float64)) / (2 * n ** 0.5)
    Ac = Ac + 2 * torch.eye(n)
    A = torch.zeros((batch, 2, n, ld), dtype=torch.float32)
    A[:, 0, :, :n] = Ac.real.transpose(1, 2).float()
    A[:, 1, :, :n] = Ac.imag.transpose(1, 2).float()
    A = A.cuda()
    X = torch.zeros_like(A)
    piv = torch.zeros((batch, n), dtype=torch.int32, device='cuda')
    info = torch.zeros(batch, dtype=torch.int32, device='cuda')
    wb = int(_lib.lib().mnpb_f32_workspace(n, batch))
    work = torch.empty(wb, dtype=torch.uint8, device='cuda')
    sh = _lib.stream_handle()
    call('mnpb_getrf_c32p', sh, n, batch, ptr(A), ld, n * ld, 2 * n * ld, ptr(piv), n, ptr(info),
         ptr(work), wb)
    call('mnpb_getri_c32p', sh, n, batch, ptr(A), ld, n * ld, 2 * n * ld, ptr(piv), n, ptr(X),
         ld, n * ld, 2 * n * ld, ptr(work), wb)
    torch.cuda.synchronize()
    Xc = (X[:, 0, :, :n].double() + 1j * X[:, 1, :, :n].double()).transpose(1, 2).cpu()
    E = Ac @ Xc - torch.eye(n)
    err = (E.abs().pow(2).sum() / n).sqrt().item()
    assert err < 1e-2, err
    ref = torch.linalg.inv(Ac)
    rel = ((Xc - ref).abs().pow(2).sum() / ref.abs().pow(2).sum()).sqrt().item()
    assert rel < 1e-2, rel
