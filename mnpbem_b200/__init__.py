"""mnpbem_b200 -- the boundary-element hot path of PyMNPBEM on NVIDIA B200.

Drop-in classes with the reference call surface (``BEMRet``, ``BEMStat``,
``BEMRetIter``,
``CompGreenRet``, ``CompGreenStat``, ``PlaneWaveRet``, ``PlaneWaveStat``,
``DipoleRet``, ``DipoleStat``, ``EELSRet``, ``EELSStat``, ``ComPoint``, ``CompStruct``, ``ComParticle``) backed by
hand-written sm_100a CUDA kernels
in ``libmnpbem_b200.so`` (C ABI: include/mnpbem_b200.h).  There is no CPU
fallback: importing the solvers requires the built library.
"""

from .compstruct import CompStruct
from .geometry import Particle, ComParticle, trisphere, trirod, load_mesh
from .clustertree import ClusterTree
from .materials import EpsConst, EpsDrude, EpsTable

__version__ = "1.0.0"


def __getattr__(name):
    # GPU-backed classes load the CUDA library on first use
    if name in ('BEMRet', 'BEMStat'):
        from . import bem
        return getattr(bem, name)
    if name in ('BEMRetIter',):
        from . import bem_iter
        return getattr(bem_iter, name)
    if name in ('CompGreenRet', 'CompGreenStat'):
        from . import greenfun
        return getattr(greenfun, name)
    if name in ('PlaneWaveRet', 'PlaneWaveStat'):
        from . import excitation
        return getattr(excitation, name)
    if name in ('DipoleRet', 'DipoleStat', 'ComPoint', 'Point', 'CompGreenStatPoints'):
        from . import points
        return getattr(points, name)
    if name in ('EELSRet', 'EELSStat'):
        from . import eels
        return getattr(eels, name)
    raise AttributeError(name)
