"""Two-particle parity against the reference (golden_dimer.npz, made by
tests/golden/make_golden_dimer.py): a 2 nm-gap dimer of gold Drude spheres
in a host of eps 1.77, three plane waves.  Exercises the cross-particle
terms of the Green-function assembly (both insides couple through the
connectivity table), the embedding-medium wavenumbers and three right-hand
sides at once.  FP64 path: sigma/h to 1e-10, cross sections to 1e-10; mixed
path (library default refinement): cross sections to 1e-9."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _dimer():
    from mnpbem_b200.geometry import ComParticle, trisphere
    from mnpbem_b200.materials import EpsConst, EpsDrude
    s = trisphere(144, 10.0)
    return ComParticle([EpsConst(1.77), EpsDrude(10.0, 9.065, 0.0708)],
                       [s.shift([-6.0, 0.0, 0.0]), s.shift([6.0, 0.0, 0.0])],
                       [[2, 1], [2, 1]], 1, 2)


def _exc():
    from mnpbem_b200.excitation import PlaneWaveRet
    return PlaneWaveRet([[1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]],
                        [[0, 0, 1.0], [0, 0, 1.0], [1.0, 0, 0]])


def _rel(a, b):
    return np.abs(np.asarray(a) - b).max() / np.abs(b).max()


@pytest.mark.parametrize('precision,tol', [('fp64', 1e-10), ('mixed', 1e-9)])
def test_dimer_against_reference(gpu_ok, precision, tol):
    from mnpbem_b200 import BEMRet
    g = golden('golden_dimer')
    cp = _dimer()
    exc = _exc()
    bem = BEMRet(cp, precision=precision)
    for i, enei in enumerate(g['lams']):
        sig, _ = bem.solve(exc.potential(cp, float(enei)))
        ext = np.asarray(exc.extinction(sig))
        sca = np.asarray(exc.scattering(sig)[0])
        assert _rel(ext, g['ext'][i]) < tol, (enei, ext, g['ext'][i])
        assert _rel(sca, g['sca'][i]) < tol, (enei, sca, g['sca'][i])
        if float(enei) == 600.0 and precision == 'fp64':
            for name in ('sig1', 'sig2', 'h1', 'h2'):
                assert _rel(getattr(sig, name), g[name]) < 1e-10, name
