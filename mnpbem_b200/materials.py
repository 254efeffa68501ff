"""Dielectric functions used on the BEM path.

Each is a callable ``eps_func(enei) -> (eps, k)`` with the wavelength
``enei`` in nm, ``eps`` the (complex) dielectric constant and
``k = 2 pi / enei * sqrt(eps)`` the wavenumber in the medium, as in the
reference (mnpbem/materials/eps_const.py:48, eps_drude.py:73).
"""

import numpy as np

EV2NM = 1.0 / 8.0655477e-4   # photon energy (eV) <-> wavelength (nm), mnpbem/utils/constants.py:9


class EpsConst(object):
    """Constant dielectric function."""

    def __init__(self, eps):
        self.eps = eps

    def __call__(self, enei):
        enei = np.asarray(enei)
        eps = np.full_like(enei, self.eps, dtype=complex)
        return eps, 2 * np.pi / enei * np.sqrt(eps)


class EpsDrude(object):
    """Drude metal: eps = eps0 - wp^2 / (w (w + i gammad)), w = EV2NM / enei (eV)."""

    def __init__(self, eps0, wp, gammad, name=None):
        self.eps0, self.wp, self.gammad, self.name = eps0, wp, gammad, name

    def __call__(self, enei):
        enei = np.asarray(enei, dtype=float)
        w = EV2NM / enei
        eps = self.eps0 - self.wp ** 2 / (w * (w + 1j * self.gammad))
        return eps, 2 * np.pi / enei * np.sqrt(eps)


def eps_k(eps_func, enei):
    """(eps, k) of a dielectric function at one wavelength as Python complex."""
    e, k = eps_func(enei)
    return complex(np.asarray(e).flat[0]), complex(np.asarray(k).flat[0])
