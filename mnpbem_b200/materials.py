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


class EpsTable(object):
    """Tabulated dielectric function (mnpbem/materials/eps_table.py:18): a
    text table of lines "energy (eV)  n  k" ('%' or '#' lines are comments),
    interpolated over the vacuum wavelength by cubic splines (not-a-knot) of n
    and k separately; eps = (n + i k)^2.  ``filename`` is a path to such a
    table (for instance the reference's materials/data/gold.dat); a bare name
    is also looked up in the directories of the ``MNPBEM_MATERIALS``
    environment variable (os.pathsep-separated)."""

    def __init__(self, filename):
        import os
        from scipy.interpolate import CubicSpline
        path = filename
        if not os.path.exists(path):
            dirs = [d for d in os.environ.get('MNPBEM_MATERIALS', '').split(os.pathsep) if d]
            hits = [os.path.join(d, filename) for d in dirs
                    if os.path.exists(os.path.join(d, filename))]
            if not hits:
                raise FileNotFoundError("EpsTable: material table not found: {} (give a path, or "
                                        "set MNPBEM_MATERIALS)".format(filename))
            path = hits[0]
        rows = []
        with open(path) as f:
            for line in f:
                line = line.strip()
                if not line or line[0] in '%#':
                    continue
                try:
                    vals = [float(v) for v in line.split()]
                except ValueError:
                    continue
                if len(vals) >= 3:
                    rows.append(vals[:3])
        if not rows:
            raise ValueError("EpsTable: no data in {}".format(path))
        data = np.asarray(rows, dtype=float)
        enei = EV2NM / data[:, 0]
        order = np.argsort(enei)
        self.filename = filename
        self.enei = enei[order]
        self.ni = CubicSpline(self.enei, data[order, 1])
        self.ki = CubicSpline(self.enei, data[order, 2])

    def __call__(self, enei):
        enei = np.asarray(enei, dtype=float)
        eps = (self.ni(enei) + 1j * self.ki(enei)) ** 2
        return eps, 2 * np.pi / enei * np.sqrt(eps)

    def refractive_index(self, enei):
        enei = np.asarray(enei, dtype=float)
        return self.ni(enei) + 1j * self.ki(enei)

    def __repr__(self):
        return "EpsTable('{}')".format(self.filename)


def eps_k(eps_func, enei):
    """(eps, k) of a dielectric function at one wavelength as Python complex."""
    e, k = eps_func(enei)
    return complex(np.asarray(e).flat[0]), complex(np.asarray(k).flat[0])
