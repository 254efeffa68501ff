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
