"""tcgen05 TF32 complex GEMM against a torch complex128 reference computed
from the same FP32 inputs.  Tolerance: TF32 (10-bit mantissa, inputs rounded
to nearest on A, truncated on B) -> relative Frobenius error below 2e-3."""
import numpy as np
import pytest
import torch

from mnpbem_b200 import _lib
from mnpbem_b200._lib import call, ptr

pytestmark = pytest.mark.gpu


def _planar(batch, rows, cols, ld, seed):
    g = torch.Generator().manual_seed(seed)
    x = torch.randn((batch, 2, cols, ld), generator=g, dtype=torch.float32)
    return x.cuda()


def _cplx(P, rows, cols):
    # planar column-major (batch, 2, cols, ld) -> complex (batch, rows, cols)
    return torch.complex(P[:, 0, :, :rows].double(), P[:, 1, :, :rows].double()).transpose(1, 2)


@pytest.mark.parametrize('m,n,k,batch,alpha,beta', [
    (128, 128, 32, 1, 1.0, 0.0), (256, 256, 256, 2, 1.0, 0.0), (200, 100, 50, 3, -1.0, 1.0),
    (37, 300, 130, 1, -1.0, 1.0), (384, 64, 1000, 2, 1.0, 1.0),
    # enough 128 x 128 tiles (>= 2 per SM) for the persistent kernel; ragged M, N
    (1000, 400, 300, 16, -1.0, 1.0), (777, 260, 96, 16, 1.0, 0.0),
    (2000, 32, 64, 24, -1.0, 1.0), (1500, 60, 200, 30, 1.0, 1.0)])
def test_cgemm_tf32(gpu_ok, m, n, k, batch, alpha, beta):
    lda, ldb, ldc = (m + 3) // 4 * 4, (k + 3) // 4 * 4, (m + 3) // 4 * 4
    A = _planar(batch, m, k, lda, 1)
    B = _planar(batch, k, n, ldb, 2)
    C = _planar(batch, m, n, ldc, 3)
    ref = alpha * (_cplx(A, m, k) @ _cplx(B, k, n)) + beta * _cplx(C, m, n)
    wb = int(_lib.lib().mnpb_cgemm_tf32_workspace(m, k, batch))
    work = torch.empty(wb, dtype=torch.uint8, device='cuda')
    call('mnpb_cgemm_tf32', _lib.stream_handle(), m, n, k, batch, alpha, ptr(A), lda, k * lda,
         2 * k * lda, ptr(B), ldb, n * ldb, 2 * n * ldb, beta, ptr(C), ldc, n * ldc, 2 * n * ldc,
         ptr(work), wb)
    torch.cuda.synchronize()
    code = np.zeros(1, dtype=np.int32)
    call('mnpb_tc_error', _lib.stream_handle(), ptr(code))
    assert code[0] == 0
    out = _cplx(C, m, n)
    err = (out - ref).abs().pow(2).sum().sqrt() / ref.abs().pow(2).sum().sqrt()
    assert err.item() < 2e-3, err.item()


def _round_tf32(x):
    """Round FP32 values to nearest TF32 (10 mantissa bits), ties away from
    zero -- the rounding of cvt.rna.tf32.f32."""
    u = x.contiguous().view(torch.int32)
    u = (u + 0x1000) & ~0x1FFF
    return u.view(torch.float32)


@pytest.mark.parametrize('m,n,k,batch,alpha,beta', [
    (128, 32, 32, 1, 1.0, 0.0),          # BN = 32 tiles
    (200, 60, 50, 3, -1.0, 1.0),         # BN = 64, ragged M, N, K
    (300, 130, 100, 2, 1.0, 1.0),        # BN = 128, grid kernel, ragged
    (1000, 400, 300, 16, -1.0, 1.0),     # 512 tiles >= 2 per SM: persistent kernel
    (2884, 1440, 1444, 2, -1.0, 1.0)])   # the largest trailing update of the 2884-face LU
def test_cgemm_tf32_a_in_place(gpu_ok, m, n, k, batch, alpha, beta):
    """A read in place (MN-major TMA tiles, 128B swizzle on 32-byte atoms):
    the path the mixed factorisation takes for its stored TF32 factors,
    compared with a complex128 product of the same (TF32-valued) A."""
    lda, ldb, ldc = (m + 3) // 4 * 4, (k + 3) // 4 * 4, (m + 3) // 4 * 4
    A = _round_tf32(_planar(batch, m, k, lda, 11))
    B = _planar(batch, k, n, ldb, 12)
    C = _planar(batch, m, n, ldc, 13)
    ref = alpha * (_cplx(A, m, k) @ _cplx(B, k, n)) + beta * _cplx(C, m, n)
    call('mnpb_cgemm_tf32_ex', _lib.stream_handle(), m, n, k, batch, alpha, ptr(A), lda, k * lda,
         2 * k * lda, ptr(B), ldb, n * ldb, 2 * n * ldb, beta, ptr(C), ldc, n * ldc, 2 * n * ldc,
         None, 0, 1)
    torch.cuda.synchronize()
    code = np.zeros(1, dtype=np.int32)
    call('mnpb_tc_error', _lib.stream_handle(), ptr(code))
    assert code[0] == 0
    out = _cplx(C, m, n)
    err = (out - ref).abs().pow(2).sum().sqrt() / ref.abs().pow(2).sum().sqrt()
    assert err.item() < 2e-3, err.item()


def test_cgemm_tf32_round_output(gpu_ok):
    """MNPB_GEMM_ROUND_C: every stored element of C is a TF32 value."""
    m, n, k, batch = 256, 100, 64, 2
    lda, ldb, ldc = m, k, m
    A = _round_tf32(_planar(batch, m, k, lda, 21))
    B = _planar(batch, k, n, ldb, 22)
    C = torch.zeros((batch, 2, n, ldc), dtype=torch.float32, device='cuda')
    ref = _cplx(A, m, k) @ _cplx(B, k, n)
    call('mnpb_cgemm_tf32_ex', _lib.stream_handle(), m, n, k, batch, 1.0, ptr(A), lda, k * lda,
         2 * k * lda, ptr(B), ldb, n * ldb, 2 * n * ldb, 0.0, ptr(C), ldc, n * ldc, 2 * n * ldc,
         None, 0, 3)
    torch.cuda.synchronize()
    assert int((C.view(torch.int32) & 0x1FFF).abs().sum().item()) == 0
    out = _cplx(C, m, n)
    err = (out - ref).abs().pow(2).sum().sqrt() / ref.abs().pow(2).sum().sqrt()
    assert err.item() < 2e-3, err.item()


def test_cgemm_tf32_ex_rejects_unaligned_in_place_a(gpu_ok):
    """An in-place A must be 16-byte aligned (TMA); refused on the host."""
    m = n = k = 64
    A = torch.zeros((2, k, 66), dtype=torch.float32, device='cuda')
    B = torch.zeros((2, n, k), dtype=torch.float32, device='cuda')
    C = torch.zeros((2, n, m), dtype=torch.float32, device='cuda')
    rc = _lib.lib().mnpb_cgemm_tf32_ex(_lib.stream_handle(), m, n, k, 1, 1.0, ptr(A), 66,
                                       k * 66, 2 * k * 66, ptr(B), k, n * k, 2 * n * k, 0.0,
                                       ptr(C), m, n * m, 2 * n * m, None, 0, 1)
    assert rc == 1     # MNPB_EINVAL: lda = 66 floats is not a multiple of 16 bytes
