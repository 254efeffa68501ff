"""C ABI: the library loads, exports every declared entry point, and the
host-side near-pair classifier is integer-exact against the reference.

No GPU is needed for these tests (no kernel is launched)."""
import hashlib
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden
from mnpbem_b200 import _lib
from mnpbem_b200.geometry import Particle, load_mesh


def _declared():
    names = []
    inc = os.path.join(ROOT, 'include')
    for fn in os.listdir(inc):
        if fn.endswith('.h'):
            src = open(os.path.join(inc, fn)).read()
            names += re.findall(r'^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(mnpb_[a-z_0-9]+)\s*\(',
                                src, flags=re.M)
    return sorted(set(names))


def test_library_exports_all_declared_symbols():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
        assert name in _lib.SIGNATURES, name


def test_version_and_error_text():
    L = _lib.lib()
    assert L.mnpb_version() >= 10000
    with pytest.raises(_lib.MNPBError) as ei:
        _lib.call('mnpb_zgemm', None, -1, 1, 1, 1, 1.0, 0.0, None, 1, 0, None, 1, 0, 0.0, 0.0,
                  None, 1, 0)
    assert 'zgemm' in str(ei.value)


def _digest(r, c, v):
    h = hashlib.sha256()
    for a in (r, c, v):
        h.update(np.ascontiguousarray(a, dtype=np.int64).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize('fn,key', [('golden_c0', 'trisphere_144_20'),
                                    ('golden_c1', 'trisphere_1444_40'),
                                    ('golden_rod', 'trirod_20_80_31_21_41')])
def test_refinematrix_c_bitexact(fn, key):
    from mnpbem_b200.greenfun import refinematrix_csr
    z = golden(fn)
    v, f = load_mesh(key)
    s = Particle(v, f, interp='curv' if f.shape[1] == 9 else 'flat')
    rp, c, k = refinematrix_csr(s.pos, s.pos, s.bradius(), s.bradius())
    r = np.repeat(np.arange(s.n), np.diff(rp))
    if 'near_digest' in z:
        assert len(c) == int(z['near_count'])
        assert _digest(r, c, k) == str(z['near_digest'])
    else:
        assert np.array_equal(r, z['near_rows'])
        assert np.array_equal(c, z['near_cols'])
        assert np.array_equal(k, z['near_vals'])


def test_refinematrix_empty_and_capacity():
    from mnpbem_b200.greenfun import refinematrix_csr
    # two far-apart points: no near pairs except the two self pairs
    pos = np.array([[0.0, 0, 0], [100.0, 0, 0]])
    rad = np.array([1.0, 1.0])
    rp, c, k = refinematrix_csr(pos, pos, rad, rad)
    assert list(rp) == [0, 1, 2] and list(c) == [0, 1] and list(k) == [2, 2]
    # capacity too small -> ENOMEM with the count reported
    import ctypes as C
    nnz = C.c_int64(0)
    row_ptr = np.zeros(3, dtype=np.int64)
    rc = _lib.lib().mnpb_refinematrix(2, 2, _lib.ptr(pos), _lib.ptr(pos), _lib.ptr(rad),
                                      _lib.ptr(rad), 0.0, 3.0, 1, C.byref(nnz),
                                      _lib.ptr(row_ptr), None, None)
    assert rc == 6 and nnz.value == 2
