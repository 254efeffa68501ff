"""Failure paths, made without faulting, trapping or hanging the GPU.

* Bounded device waits: ``mnpb_wait_probe`` runs the wait helper of the
  tensor-core GEMM (mbarrier), of the triangular solve (flag spin) and of the
  streamed triangular solve (mbarrier) against something nothing completes,
  with a 20 ms limit.  Each wait must give up, the call must return
  MNPB_ETIMEOUT (5) with a message, and the device must stay usable: a GEMM
  right after it runs and its error word reads 0.
* Non-convergence: the mixed solver's FP64 refinement with one correction
  allowed and an unreachable tolerance must raise MNPB_ENOCONV (4), never
  return an unrefined solution.
* Argument checks of the probe, on the host (no GPU needed).
"""
import numpy as np
import pytest
import torch

import mnpbem_b200 as M
from mnpbem_b200 import _lib
from mnpbem_b200._lib import call, ptr

EPS = [M.EpsConst(1.0), M.EpsDrude(10.0, 9.065, 0.0708)]


def test_wait_probe_rejects_bad_arguments():
    L = _lib.lib()
    assert L.mnpb_wait_probe(None, 3, 1000, None) == 1            # unknown kind
    assert L.mnpb_wait_probe(None, 0, 0, None) == 1               # limit must be > 0
    assert L.mnpb_wait_probe(None, 0, 3_000_000_000, None) == 1   # limit above 2 s
    assert L.mnpb_wait_probe(None, 1, 1000, None) == 1            # kind 1 needs a flag
    assert 'device int' in L.mnpb_last_error().decode()


@pytest.mark.gpu
@pytest.mark.parametrize('kind,what', [(0, 'tensor-core mbarrier'),
                                       (1, 'triangular-solve flag'),
                                       (2, 'triangular-solve mbarrier')])
def test_bounded_wait_gives_up(gpu_ok, kind, what):
    flag = torch.zeros(1, dtype=torch.int32, device='cuda')
    rc = _lib.lib().mnpb_wait_probe(_lib.stream_handle(), kind, 20_000_000, ptr(flag))
    assert rc == 5                                               # MNPB_ETIMEOUT
    assert what in _lib.lib().mnpb_last_error().decode()
    # the context is still usable and the error word was cleared
    m = n = k = 64
    A = torch.randn((1, 2, k, m), device='cuda')
    B = torch.randn((1, 2, n, k), device='cuda')
    C = torch.zeros((1, 2, n, m), device='cuda')
    wb = int(_lib.lib().mnpb_cgemm_tf32_workspace(m, k, 1))
    work = torch.empty(wb, dtype=torch.uint8, device='cuda')
    call('mnpb_cgemm_tf32', _lib.stream_handle(), m, n, k, 1, 1.0, ptr(A), m, k * m, 2 * k * m,
         ptr(B), k, n * k, 2 * n * k, 0.0, ptr(C), m, n * m, 2 * n * m, ptr(work), wb)
    code = np.zeros(1, dtype=np.int32)
    call('mnpb_tc_error', _lib.stream_handle(), ptr(code))
    assert code[0] == 0
    torch.cuda.synchronize()
    ref = torch.complex(A[0, 0].double(), A[0, 1].double()).T @ \
        torch.complex(B[0, 0].double(), B[0, 1].double()).T
    out = torch.complex(C[0, 0].double(), C[0, 1].double()).T
    assert ((out - ref).norm() / ref.norm()).item() < 2e-3


@pytest.mark.gpu
def test_refinement_reports_no_convergence(gpu_ok):
    from mnpbem_b200 import bem, excitation
    v, f = M.load_mesh('trisphere_32_10')
    cp = M.ComParticle(EPS, [M.Particle(v, f, interp='curv')], [[2, 1]])
    b = bem.BEMRet(cp, precision='mixed', refine_maxit=1, refine_tol=1e-30)
    exc = excitation.PlaneWaveRet(pol=[[1, 0, 0]], dir=[[0, 0, 1]])
    with pytest.raises(_lib.MNPBError) as ei:
        b.solve(exc.potential(cp, 550.0))
    assert ei.value.code == 4                                    # MNPB_ENOCONV
    assert 'tolerance' in str(ei.value)
    # the same solver converges with the default budget
    b.refine_maxit, b.refine_tol = 20, 1e-11
    sig, _ = b.solve(exc.potential(cp, 550.0))
    assert np.isfinite(sig.sig2).all()
