"""Numerics of the dense FP64 kernels against torch float64/complex128
references on the same inputs (seeded), including ragged sizes and batches."""
import numpy as np
import pytest
import torch

from mnpbem_b200 import _lib
from mnpbem_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def _rand(shape, seed):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g, dtype=torch.float64) +
            1j * torch.randn(shape, generator=g, dtype=torch.float64)).cuda()


@pytest.mark.parametrize('m,n,k,batch', [(1, 1, 1, 1), (37, 53, 29, 2), (128, 64, 96, 3),
                                         (200, 13, 300, 1)])
def test_zgemm_vs_torch(gpu_ok, m, n, k, batch):
    # column-major C = alpha A B + beta C  <=>  row-major C^T = alpha B^T A^T + beta C^T
    A = _rand((batch, k, m), 1)   # A^T stored row-major == A column-major
    B = _rand((batch, n, k), 2)
    Cm = _rand((batch, n, m), 3)
    alpha, beta = (0.7 - 0.2j), (0.3 + 0.5j)
    ref = alpha * (B @ A) + beta * Cm
    C = Cm.clone()
    call('mnpb_zgemm', _lib.stream_handle(), m, n, k, batch, alpha.real, alpha.imag, ptr(A), m,
         m * k, ptr(B), k, k * n, beta.real, beta.imag, ptr(C), m, m * n)
    torch.cuda.synchronize()
    assert torch.allclose(C, ref, rtol=1e-12, atol=1e-12 * ref.abs().max().item())


@pytest.mark.parametrize('n,batch,nrhs', [(1, 1, 1), (31, 2, 3), (33, 1, 2), (97, 3, 5),
                                         (260, 2, 7)])
def test_getrf_getrs_vs_torch(gpu_ok, n, batch, nrhs):
    A = _rand((batch, n, n), 4) + 3 * torch.eye(n, dtype=torch.complex128, device='cuda')
    X = _rand((batch, nrhs, n), 5)
    # A_colmajor[b] = A[b].T ; B = A_colmajor X_colmajor
    Acm = A.transpose(1, 2)
    Bcm = (Acm @ X.transpose(1, 2)).transpose(1, 2).contiguous()   # (batch, nrhs, n)
    LU = A.clone()
    piv = torch.zeros((batch, n), dtype=torch.int32, device='cuda')
    info = torch.zeros(batch, dtype=torch.int32, device='cuda')
    call('mnpb_getrf_f64', _lib.stream_handle(), n, batch, ptr(LU), n, n * n, ptr(piv), n,
         ptr(info))
    call('mnpb_getrs_f64', _lib.stream_handle(), n, batch, nrhs, ptr(LU), n, n * n, ptr(piv), n,
         ptr(Bcm), n, n * nrhs)
    torch.cuda.synchronize()
    assert info.sum().item() == 0
    assert torch.allclose(Bcm, X, rtol=0, atol=1e-10 * X.abs().max().item())
    # pivots follow LAPACK's rule (first max of |re|+|im|): compare with scipy
    import scipy.linalg as sla
    a0 = Acm[0].cpu().numpy()
    lu_ref, piv_ref = sla.lu_factor(a0)
    assert np.array_equal(piv[0].cpu().numpy(), piv_ref)
    lu0 = LU[0].transpose(0, 1).cpu().numpy()
    assert np.allclose(lu0, lu_ref, rtol=0, atol=1e-10 * np.abs(lu_ref).max())


def test_getrf_reports_zero_pivot(gpu_ok):
    n = 40
    A = _rand((1, n, n), 6)
    A[0, 5, :] = 0          # column 5 (column-major) exactly zero -> singular
    piv = torch.zeros((1, n), dtype=torch.int32, device='cuda')
    info = torch.zeros(1, dtype=torch.int32, device='cuda')
    call('mnpb_getrf_f64', _lib.stream_handle(), n, 1, ptr(A), n, n * n, ptr(piv), n, ptr(info))
    torch.cuda.synchronize()
    assert info.item() == 6
