"""Mirror symmetry on the host (no GPU): the full particle built from the
irreducible part and its flipped images, the symmetry tables, and the
expansion of symmetry components to the full particle, against the
reference (golden_mirror.npz, made by running the reference)."""
import numpy as np
import pytest

from conftest import golden
import mnpbem_b200 as M
from mnpbem_b200.compstruct import CompStruct
from mnpbem_b200.mirror import ComParticleMirror, CompStructMirror, PlaneWaveRetMirror

DRUDE = M.EpsDrude(10.0, 9.065, 0.0708)


def mirror_particle(z, sym):
    p = M.Particle(z[sym + '_verts2'], z[sym + '_faces2'], interp='flat')
    return ComParticleMirror([M.EpsConst(1.0), DRUDE], [p], [[2, 1]], sym, (1,))


@pytest.mark.parametrize('sym', ['x', 'xy'])
def test_full_particle(sym):
    z = golden('golden_mirror')
    cpm = mirror_particle(z, sym)
    nk = 4 if sym == 'xy' else 2
    assert cpm.pfull.nfaces == nk * cpm.n
    assert np.allclose(cpm.pfull.pos, z[sym + '_full_pos'], rtol=0, atol=1e-13)
    assert np.allclose(cpm.pfull.nvec, z[sym + '_full_nvec'], rtol=0, atol=1e-13)
    assert cpm.pfull.closed == [list(range(1, nk + 1))] * nk
    # the stored symmetry values of every component are rows of the table
    for v in range(2):
        sv = z['%s_0_%d_symval' % (sym, v)]
        assert sv.shape == (3, nk)
        for r in range(3):
            cpm.symindex(sv[r])


def test_symmetry_keys():
    z = golden('golden_mirror')
    cpm = mirror_particle(z, 'xy')
    assert np.array_equal(cpm.symvalue(['++', '--']), [[1, 1, 1, 1], [1, -1, -1, 1]])
    assert cpm.symindex([1, -1, 1, -1]) == 2
    with pytest.raises(ValueError):
        cpm.symvalue('+')


def test_expand_and_combine():
    """Image k of a scalar takes symval[z, k], component l of a vector
    symval[l, k]; the full values combine the x and y components with the
    polarisation's weights."""
    z = golden('golden_mirror')
    cpm = mirror_particle(z, 'x')
    n = cpm.n
    rng = np.random.default_rng(0)
    exc = PlaneWaveRetMirror([[0.6, 0.8, 0.0]], [[0, 0, 1.0]])
    s = CompStructMirror(cpm, 550.0, lambda v: exc.full(v))
    vals = []
    for v, keys in enumerate((['+', '-', '-'], ['-', '+', '+'])):
        sig = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
        h = rng.standard_normal((n, 3, 2)) + 1j * rng.standard_normal((n, 3, 2))
        c = CompStruct(cpm, 550.0, sig1=sig, h1=h)
        c.symval = cpm.symvalue(keys)
        s.val.append(c)
        vals.append((sig, h, c.symval))
    full, pf = s.full()
    assert pf is cpm.pfull
    sig_full = 0.6 * np.concatenate([vals[0][0][:, 0], vals[0][2][2, 1] * vals[0][0][:, 0]]) + \
        0.8 * np.concatenate([vals[1][0][:, 0], vals[1][2][2, 1] * vals[1][0][:, 0]])
    assert np.allclose(full.sig1[:, 0], sig_full)
    hx = 0.6 * np.concatenate([vals[0][1][:, 0, 0], vals[0][2][0, 1] * vals[0][1][:, 0, 0]]) + \
        0.8 * np.concatenate([vals[1][1][:, 0, 0], vals[1][2][0, 1] * vals[1][1][:, 0, 0]])
    assert np.allclose(full.h1[:, 0, 0], hx)
