"""Allocation-free tensor-core GEMM (mnpb_cgemm_tf32_noalloc) against the
workspace-taking entry point (mnpb_cgemm_tf32) on the same inputs.

Calls of the allocation-free entry run back to back with different shapes,
so each reuses the static scratch the one before it wrote.  The last shape has
enough 128 x 128 tiles (384, at least two per SM) to run the persistent
kernel.  Each result must agree with mnpb_cgemm_tf32's and with a complex128
product of the same inputs within the TF32 GEMM tolerance (relative Frobenius
error below 2e-3).  The file name sorts last so that it also runs after every
other test."""
import ctypes

import numpy as np
import pytest
import torch

from mnpbem_b200 import _lib
from mnpbem_b200._lib import call, ptr

pytestmark = pytest.mark.gpu

STATIC_BYTES = 64 << 20


def _planar(batch, cols, ld, seed):
    g = torch.Generator().manual_seed(seed)
    return torch.randn((batch, 2, cols, ld), generator=g, dtype=torch.float32).cuda()


def _cplx(P, rows):
    return torch.complex(P[:, 0, :, :rows].double(), P[:, 1, :, :rows].double()).transpose(1, 2)


def _args(m, n, k, batch, alpha, beta, A, B, C):
    lda, ldb, ldc = A.shape[-1], B.shape[-1], C.shape[-1]
    return (m, n, k, batch, alpha, ptr(A), lda, k * lda, 2 * k * lda, ptr(B), ldb, n * ldb,
            2 * n * ldb, beta, ptr(C), ldc, n * ldc, 2 * n * ldc)


def _tc_error():
    code = np.zeros(1, dtype=np.int32)
    call('mnpb_tc_error', _lib.stream_handle(), ptr(code))
    return int(code[0])


def test_noalloc_matches_workspace_gemm_twice(gpu_ok):
    cases = [(200, 100, 50, 3, -1.0, 1.0, 11), (384, 64, 1000, 2, 1.0, 1.0, 21),
             (2048, 1024, 1024, 3, -1.0, 1.0, 31)]
    outs = []
    for m, n, k, batch, alpha, beta, seed in cases:
        lda, ldb, ldc = (m + 3) // 4 * 4, (k + 3) // 4 * 4, (m + 3) // 4 * 4
        A = _planar(batch, k, lda, seed)
        B = _planar(batch, n, ldb, seed + 1)
        C0 = _planar(batch, n, ldc, seed + 2)
        C_ws, C_na = C0.clone(), C0.clone()
        ref = alpha * (_cplx(A, m) @ _cplx(B, k)) + beta * _cplx(C0, m)
        wb = int(_lib.lib().mnpb_cgemm_tf32_workspace(m, k, batch))
        assert wb <= STATIC_BYTES
        work = torch.empty(wb, dtype=torch.uint8, device='cuda')
        call('mnpb_cgemm_tf32', _lib.stream_handle(),
             *_args(m, n, k, batch, alpha, beta, A, B, C_ws), ptr(work), wb)
        call('mnpb_cgemm_tf32_noalloc', _lib.stream_handle(),
             *_args(m, n, k, batch, alpha, beta, A, B, C_na))
        outs.append((m, C_ws, C_na, ref))
    torch.cuda.synchronize()
    assert _tc_error() == 0
    for m, C_ws, C_na, ref in outs:
        ws, na = _cplx(C_ws, m), _cplx(C_na, m)
        err = ((na - ws).abs().pow(2).sum().sqrt() / ws.abs().pow(2).sum().sqrt()).item()
        assert err < 2e-3, err
        err = ((na - ref).abs().pow(2).sum().sqrt() / ref.abs().pow(2).sum().sqrt()).item()
        assert err < 2e-3, err


def test_noalloc_rejects_oversize(gpu_ok):
    # 4096 x 4096 packed planar FP32 needs 128 MiB > 64 MiB: refused on the
    # host before anything is launched.
    m = n = k = 4096
    need = int(_lib.lib().mnpb_cgemm_tf32_workspace(m, k, 1))
    assert need > STATIC_BYTES
    f = _lib.lib().mnpb_cgemm_tf32_noalloc
    A = B = C = ctypes.c_void_p(16)    # never dereferenced: the size check comes first
    rc = f(_lib.stream_handle(), m, n, k, 1, 1.0, A, m, m * k, 2 * m * k, B, k, k * n,
           2 * k * n, 0.0, C, m, m * n, 2 * m * n)
    assert rc == 6                     # MNPB_ENOMEM
    msg = _lib.lib().mnpb_last_error().decode()
    assert 'static scratch' in msg and str(need) in msg
