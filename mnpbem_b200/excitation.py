"""Plane-wave excitations and optical cross sections.

``PlaneWaveRet`` / ``PlaneWaveStat`` mirror the reference classes
(mnpbem/simulation/planewave_ret.py:81-504, planewave_stat.py:152-355):
``potential(p, enei)`` returns the excitation ``CompStruct`` for the BEM
solvers, ``extinction`` / ``scattering`` / ``absorption`` the cross sections
of a solution.  The retarded far fields (optical theorem and the
256-direction integration sphere of mnpbem/spectrum/spectrum_ret.py:14) are
evaluated by the CUDA library; ``potential_device`` produces the potentials
of a whole batch of wavelengths directly in GPU memory for spectrum sweeps.
"""

import os

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .materials import eps_k

__all__ = ["PlaneWaveRet", "PlaneWaveStat", "pinfty"]

_PINFTY = None


def pinfty():
    """Unit directions and solid-angle weights of the far-field sphere."""
    global _PINFTY
    if _PINFTY is None:
        path = os.path.join(os.path.dirname(__file__), 'data', 'meshes.npz')
        with np.load(path) as z:
            _PINFTY = (np.ascontiguousarray(z['pinfty256_nvec']),
                       np.ascontiguousarray(z['pinfty256_area']))
    return _PINFTY


def _inout_faces(p):
    io = getattr(p, 'inout_faces', None)
    if io is not None and not callable(io):
        return np.asarray(io)
    inout = np.atleast_2d(np.asarray(p.inout))
    sizes = [q.nfaces if hasattr(q, 'nfaces') else q.n for q in p.p]
    return np.repeat(inout, sizes, axis=0)


class _Sides(object):
    """Per-face flags 'inside / outside medium is the embedding medium' on the GPU."""

    def __init__(self, p, medium, device):
        io = _inout_faces(p)
        self.side_in = torch.from_numpy((io[:, 0] == medium).astype(np.int8)).to(device)
        self.side_out = torch.from_numpy((io[:, 1] == medium).astype(np.int8)).to(device)


class PlaneWaveRet(object):
    """Plane wave (retarded): pol (npol, 3), dir (npol, 3), embedding medium index."""

    def __init__(self, pol, dir, medium=1, **options):
        if pol is None or dir is None:
            raise ValueError("PlaneWaveRet: 'pol' and 'dir' are required")
        self.pol = np.atleast_2d(np.asarray(pol, dtype=float))
        self.dir = np.atleast_2d(np.asarray(dir, dtype=float))
        self.medium = medium
        if not np.allclose(np.sum(self.pol * self.dir, axis=1), 0):
            raise AssertionError("Polarization and propagation direction must be orthogonal")
        self._sides = {}

    # ---- potentials ------------------------------------------------------------
    def potential(self, p, enei):
        """a1, a1p, a2, a2p (mnpbem/simulation/planewave_ret.py:257-361)."""
        eps_med, _ = eps_k(p.eps[self.medium - 1], enei)
        k0 = 2 * np.pi / enei
        k = k0 * np.sqrt(eps_med)
        io = _inout_faces(p)
        n = io.shape[0]
        pos, nvec = np.asarray(p.pos), np.asarray(p.nvec)
        exc = CompStruct(p, enei)
        npol = self.pol.shape[0]
        for side in (0, 1):
            a = np.zeros((n, 3, npol), dtype=complex)
            ap = np.zeros((n, 3, npol), dtype=complex)
            ind = np.where(io[:, side] == self.medium)[0]
            for i in range(npol):
                phase = np.exp(1j * k * pos[ind, :] @ self.dir[i, :]) / (1j * k0)
                a[ind, :, i] = phase[:, None] * self.pol[i, :]
                nd = nvec[ind, :] @ self.dir[i, :]
                ap[ind, :, i] = (1j * k * nd)[:, None] * phase[:, None] * self.pol[i, :]
            if npol == 1:
                a, ap = a[:, :, 0], ap[:, :, 0]
            if side == 0:
                exc.set(a1=a, a1p=ap)
            else:
                exc.set(a2=a, a2p=ap)
        return exc

    __call__ = potential

    def _side_flags(self, p, device):
        key = (id(p), str(device))
        if key not in self._sides:
            self._sides[key] = _Sides(p, self.medium, device)
        return self._sides[key]

    def _wavenumbers(self, p, eneis):
        km = np.zeros((len(eneis), 2))
        k0 = np.zeros(len(eneis))
        for b, enei in enumerate(eneis):
            _, k = eps_k(p.eps[self.medium - 1], enei)
            km[b] = (k.real, k.imag)
            k0[b] = 2 * np.pi / enei
        return km, k0

    def potential_device(self, p, tables, eneis, stream=None):
        """Potentials of every wavelength of ``eneis`` on the GPU: ((B,16,K,n), K)."""
        dev = tables.device
        n, B, K = tables.n, len(eneis), self.pol.shape[0]
        sides = self._side_flags(p, dev)
        km, k0 = self._wavenumbers(p, eneis)
        pots = torch.empty((B, 16, K, n), dtype=torch.complex128, device=dev)
        d_pol = torch.from_numpy(np.ascontiguousarray(self.pol)).to(dev)
        d_dir = torch.from_numpy(np.ascontiguousarray(self.dir)).to(dev)
        call('mnpb_planewave_potential', _lib.stream_handle(stream), n, B, K, ptr(tables.pos),
             ptr(tables.nvec), ptr(sides.side_in), ptr(sides.side_out), ptr(d_pol), ptr(d_dir),
             ptr(torch.from_numpy(km).to(dev)), ptr(torch.from_numpy(k0).to(dev)), ptr(pots))
        return pots, K

    # ---- far fields and cross sections -------------------------------------------
    def farfield_device(self, p, tables, sol_dev, eneis, dirs, stream=None):
        """Far fields e, h (B, K, ndir, 3) for solutions sol_dev (B, 8, K, n)."""
        dev = tables.device
        n, B = tables.n, len(eneis)
        K = sol_dev.shape[2]
        sides = self._side_flags(p, dev)
        km, k0 = self._wavenumbers(p, eneis)
        d_dirs = torch.from_numpy(np.ascontiguousarray(dirs, dtype=np.float64)).to(dev)
        nd = d_dirs.shape[0]
        e = torch.empty((B, K, nd, 3), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        call('mnpb_farfield', _lib.stream_handle(stream), n, B, K, nd, ptr(tables.pos),
             ptr(tables.area), ptr(sides.side_in), ptr(sides.side_out), ptr(d_dirs),
             ptr(torch.from_numpy(km).to(dev)), ptr(torch.from_numpy(k0).to(dev)),
             ptr(sol_dev), ptr(e), ptr(h))
        return e, h

    @staticmethod
    def _sol_device(sig, device):
        def as3(x, K):
            x = np.asarray(x)
            return x.reshape(x.shape[0], -1, K) if x.ndim == 3 else x.reshape(x.shape[0], 3, 1)
        s1 = np.asarray(sig.sig1)
        K = 1 if s1.ndim == 1 else s1.shape[1]
        n = s1.shape[0]
        x = np.zeros((1, 8, K, n), dtype=complex)
        x[0, 0] = s1.reshape(n, K).T
        x[0, 1:4] = as3(sig.h1, K).transpose(1, 2, 0)
        x[0, 4] = np.asarray(sig.sig2).reshape(n, K).T
        x[0, 5:8] = as3(sig.h2, K).transpose(1, 2, 0)
        return torch.from_numpy(x).to(device), K

    def extinction(self, sig, tables=None):
        """4 pi / k Im(pol* . e_forward) (planewave_ret.py:437-504)."""
        p = sig.p
        dev = torch.device('cuda')
        x, K = self._sol_device(sig, dev)
        t = tables if tables is not None else _FaceTables(p, dev)
        e, _ = self.farfield_device(p, t, x, [sig.enei], self.dir)
        e = e[0].cpu().numpy()                      # (K, ndir, 3)
        _, k = eps_k(p.eps[self.medium - 1], sig.enei)
        npol = self.pol.shape[0]
        ext = np.array([np.imag(np.sum(np.conj(self.pol[i]) * e[i, i])) for i in range(npol)])
        ext = np.real(4 * np.pi / k * ext)
        return float(ext[0]) if npol == 1 else ext

    def scattering(self, sig, tables=None):
        """Radiated power over the far-field sphere / (0.5 n_b) (spectrum_ret.py:395-459)."""
        p = sig.p
        dev = torch.device('cuda')
        x, K = self._sol_device(sig, dev)
        t = tables if tables is not None else _FaceTables(p, dev)
        nvec_s, area_s = pinfty()
        e, h = self.farfield_device(p, t, x, [sig.enei], nvec_s)
        e = e[0].cpu().numpy()
        h = h[0].cpu().numpy()
        dsca = 0.5 * np.real(np.einsum('dc,kdc->kd', nvec_s, np.cross(e, np.conj(h))))
        sca = dsca @ area_s
        eps_med, _ = eps_k(p.eps[self.medium - 1], sig.enei)
        sca = sca / (0.5 * np.real(np.sqrt(eps_med)))
        return (float(sca[0]) if K == 1 else sca), CompStruct(p, sig.enei, dsca=dsca.T)

    def absorption(self, sig):
        return self.extinction(sig) - self.scattering(sig)[0]


class _FaceTables(object):
    """Minimal device face data (pos, area) for far-field evaluation."""

    def __init__(self, p, device):
        self.device = device
        self.pos = torch.from_numpy(np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))).to(device)
        self.area = torch.from_numpy(np.ascontiguousarray(np.asarray(p.area, dtype=np.float64))).to(device)
        self.n = self.pos.shape[0]


class PlaneWaveStat(object):
    """Plane wave in the quasistatic limit (mnpbem/simulation/planewave_stat.py)."""

    def __init__(self, pol, medium=1, **options):
        self.pol = np.atleast_2d(np.asarray(pol, dtype=float))
        self.medium = medium

    def potential(self, p, enei):
        phip = -np.asarray(p.nvec) @ self.pol.T
        if self.pol.shape[0] == 1:
            phip = phip[:, 0]
        return CompStruct(p, enei, phip=phip)

    __call__ = potential

    def _dip(self, sig):
        s = np.asarray(sig.sig)
        ap = np.asarray(sig.p.area)[:, None] * np.asarray(sig.p.pos)
        return (ap.T @ s).reshape(3, -1)

    def scattering(self, sig):
        dip = self._dip(sig)
        _, k = eps_k(sig.p.eps[self.medium - 1], sig.enei)
        sca = np.real(8 * np.pi / 3 * np.real(k) ** 4 * np.sum(np.abs(dip) ** 2, axis=0))
        return float(sca[0]) if sca.size == 1 else sca

    def absorption(self, sig):
        dip = self._dip(sig)
        _, k = eps_k(sig.p.eps[self.medium - 1], sig.enei)
        a = 4 * np.pi * np.real(k) * np.imag(np.sum(self.pol * dip.T, axis=1))
        return float(a[0]) if a.size == 1 else a

    def extinction(self, sig):
        return self.scattering(sig) + self.absorption(sig)
