"""Host logic of the mirror-symmetry dipoles (no GPU): the symmetry values
of the image combinations, and ``full`` taking the mean of the expanded
solutions and contracting it with the moments.  With image solutions
s_k for the unit dipoles at the points and their images, the combinations
c_v = sum_k coef[v, k] s_k expanded and averaged must give back s_0 on the
full particle's first block, for every symmetry."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200.compstruct import CompStruct
from mnpbem_b200.mirror import (ComParticleMirror, CompStructMirror, DipoleRetMirror,
                                DipoleStatMirror)


def _sphere_piece(sym):
    """The quarter (xy) or half sphere of golden_mirror.npz (the half one
    stands in for symmetry y as well: only the bookkeeping is tested)."""
    z = golden('golden_mirror')
    key = 'xy' if sym == 'xy' else 'x'
    return M.Particle(z[key + '_verts2'], z[key + '_faces2'], interp='flat')


@pytest.mark.parametrize('cls', [DipoleStatMirror, DipoleRetMirror])
@pytest.mark.parametrize('sym', ['x', 'y', 'xy'])
def test_full_recovers_the_unit_dipoles(cls, sym):
    cpm = ComParticleMirror([M.EpsConst(1.0), M.EpsDrude(10.0, 9.065, 0.0708)],
                            [_sphere_piece(sym)], [[2, 1]], sym, (1,))
    n, npt = cpm.n, 2
    rng = np.random.default_rng(7)
    combos = cls._COMBOS[sym]
    nk = len(cls._IMAGES[sym])
    assert len(combos) == nk
    # solutions of the images, on the irreducible part (unit moments: 3 columns per point)
    s = rng.standard_normal((nk, n, npt * 3)) + 1j * rng.standard_normal((nk, n, npt * 3))
    val = CompStructMirror(cpm, 500.0)
    for coef, key in combos:
        v = CompStruct(cpm, 500.0, sig=sum(c * s[k] for k, c in enumerate(coef)))
        v.symval = cpm.symvalue(key)
        val.val.append(v)
    dip = np.array([[1.0, 0.0, 0.0], [0.3, -0.5, 0.8]])        # two moments, shared
    exc = cls.__new__(cls)
    exc.dip = type('D', (), {'dip': np.tile(dip.T.reshape(1, 3, 2), (npt, 1, 1))})()
    out, pf = exc.full(val)
    assert pf is cpm.full()
    got = out.sig[:n].reshape(n, npt, 2)
    want = np.einsum('nic,jc->nij', s[0].reshape(n, npt, 3), dip)
    assert np.abs(got - want).max() < 1e-12 * np.abs(want).max()
