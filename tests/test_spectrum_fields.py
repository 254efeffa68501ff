"""Host-side layout of spectrum results: the batched reordering that
``BEMRet.solve_spectrum`` applies to a whole batch gives, for every
wavelength, exactly the fields ``BEMRet._to_compstruct`` builds from that
wavelength's solution vector (sig1, h1, sig2, h2 in the reference's
``CompStruct`` shapes), for one and for several excitations."""
import numpy as np
import pytest

from mnpbem_b200.bem import BEMRet, _fields_by_wavelength


class _Tables:
    n = 7


class _Stub(BEMRet):
    def __init__(self):          # only what _to_compstruct needs
        self.tables = _Tables()
        self.p = None


@pytest.mark.parametrize('K', [1, 3])
def test_batched_fields_match_per_wavelength(K):
    rng = np.random.default_rng(3)
    B, n = 5, _Tables.n
    x = rng.standard_normal((B, 8, K, n)) + 1j * rng.standard_normal((B, 8, K, n))
    sig1, sig2, h1, h2 = _fields_by_wavelength(x, K)
    stub = _Stub()
    for b in range(B):
        ref = stub._to_compstruct(x[b], K, 500.0 + b)
        for name, got in (('sig1', sig1[b]), ('sig2', sig2[b]), ('h1', h1[b]), ('h2', h2[b])):
            want = getattr(ref, name)
            assert got.shape == want.shape, name
            assert np.array_equal(got, want), name
            assert got.flags['C_CONTIGUOUS'], name


@pytest.mark.parametrize('K', [1, 3])
def test_device_reordering_matches_host(K):
    """``solve_spectrum`` reorders on the device (torch ops, here on CPU
    tensors) and only views the copied block on the host: the views equal
    the host reordering and are contiguous per wavelength."""
    import torch
    from mnpbem_b200.bem import _fields_device, _fields_host
    rng = np.random.default_rng(4)
    B, n = 5, _Tables.n
    x = rng.standard_normal((B, 8, K, n)) + 1j * rng.standard_normal((B, 8, K, n))
    want = _fields_by_wavelength(x, K)
    got = _fields_host(_fields_device(torch.from_numpy(x)).numpy(), x.shape)
    for w, g in zip(want, got):
        g = g[..., 0] if K == 1 else g
        assert g.shape == w.shape and np.array_equal(g, w)
        assert g[0].flags['C_CONTIGUOUS']
