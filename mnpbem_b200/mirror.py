"""Particles with mirror symmetry: the retarded BEM solver on the irreducible
part of a mirror-symmetric particle.

``ComParticleMirror``, ``CompStructMirror``, ``PlaneWaveRetMirror`` and
``BEMRetMirror`` mirror mnpbem/geometry/comparticle_mirror.py,
mnpbem/simulation/planewave_ret_mirror.py and mnpbem/bem/bem_ret_mirror.py:
the user gives the part of the particle with x >= 0 (sym 'x'), y >= 0
('y') or both ('xy'); the full particle is that part and its 1 or 3 mirror
images.  Every excitation is split into components with definite parity
under the mirror planes (symmetry values, rows of ``symtable``), and each
component is solved on the irreducible part alone: 2 or 4 BEM systems of
size n instead of one of size 2n or 4n.

GPU work (``libmnpbem_b200.so``): the full particle's Green functions
(``mnpb_assemble_ret``, rows of the irreducible part used), their
contraction to one n x n matrix per symmetry value (``mnpb_mirror_contract``),
the per-symmetry-value factorisations (``mnpb_bemret_init_mirror_f64``),
the Sigma matrix of every (x, y, z) symmetry-value combination
(``mnpb_bemret_sigma_mirror_f64``) and the solves
(``mnpb_bemret_solve_mirror_f64``), all in FP64.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .geometry import Particle, ComParticle
from .greenfun import SurfaceTables
from .excitation import PlaneWaveRet, PlaneWaveStat

__all__ = ["flip", "ComParticleMirror", "CompStructMirror", "PlaneWaveRetMirror",
           "BEMRetMirror", "PlaneWaveStatMirror", "BEMStatMirror", "DipoleStatMirror",
           "DipoleRetMirror", "CompGreenRetMirror"]


def flip(p, dirs):
    """The particle mirrored at the planes normal to ``dirs`` (0 x, 1 y, 2 z)
    with its faces' vertex order reversed so the normals point outwards
    again (mnpbem/geometry/particle.py:843-905, flip / flipfaces)."""
    dirs = [dirs] if np.isscalar(dirs) else list(dirs)
    if p.faces2 is not None:
        v = np.array(p.verts2, dtype=float)
        f = np.array(p.faces2, dtype=float)
        for d in dirs:
            v[:, d] = -v[:, d]
        tri = np.isnan(f[:, 3])
        g = f.copy()
        g[np.ix_(tri, [0, 1, 2, 4, 5, 6])] = f[np.ix_(tri, [2, 1, 0, 5, 4, 6])]
        g[np.ix_(~tri, [0, 1, 2, 3, 4, 5, 6, 7])] = f[np.ix_(~tri, [3, 2, 1, 0, 6, 5, 4, 7])]
        return Particle(v, g, interp=p.interp)
    v = np.array(p.verts, dtype=float)
    f = np.array(p.faces, dtype=float)
    for d in dirs:
        v[:, d] = -v[:, d]
    tri = np.isnan(f[:, 3])
    g = f.copy()
    g[np.ix_(tri, [0, 1, 2])] = f[np.ix_(tri, [2, 1, 0])]
    g[np.ix_(~tri, [0, 1, 2, 3])] = f[np.ix_(~tri, [3, 2, 1, 0])]
    return Particle(v, g, interp=p.interp)


_SYMVAL = {'+': [1, 1], '-': [1, -1],
           '++': [1, 1, 1, 1], '+-': [1, 1, -1, -1], '-+': [1, -1, 1, -1], '--': [1, -1, -1, 1]}


class ComParticleMirror(object):
    """Irreducible part of a mirror-symmetric particle
    (mnpbem/geometry/comparticle_mirror.py:110-404).

    ``ComParticleMirror(eps, particles, inout, sym='x', closed_args=None)``:
    ``closed_args`` (e.g. ``(1,)``) marks particles whose surface, together
    with its mirror images, is closed; without it every piece is taken as
    its own closed surface, as the reference does.  ``full()`` is the full particle: the given particles,
    then their x images, then (sym 'y' / 'xy') the y images of all of those.
    Face data (pos, nvec, area) are those of the irreducible part, the first
    n faces of the full particle.
    """

    def __init__(self, eps, particles, inout, sym='x', closed_args=None, **kwargs):
        if not isinstance(sym, str):
            if closed_args is not None:
                raise ValueError("ComParticleMirror: cannot pass both numeric sym and "
                                 "closed_args")
            closed_args = tuple(sym) if hasattr(sym, '__iter__') else (sym,)
            sym = kwargs.pop('sym', 'x')
        closed = tuple(closed_args) if closed_args is not None else ()
        if sym not in ('x', 'y', 'xy'):
            raise ValueError("ComParticleMirror: 'sym' must be one of 'x', 'y', 'xy'; got {!r}"
                             .format(sym))
        self.eps = list(eps)
        self.p = list(particles)
        self.inout = np.atleast_2d(np.asarray(inout, dtype=int))
        self.sym = sym
        if sym in ('x', 'y'):
            self.symtable = np.array([[1, 1], [1, -1]], dtype=np.float64)
        else:
            self.symtable = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, 1, -1],
                                      [1, -1, -1, 1]], dtype=np.float64)
        plist, io = list(self.p), [list(r) for r in self.inout]
        if sym in ('x', 'xy'):
            m = len(plist)
            plist += [flip(plist[i], 0) for i in range(m)]
            io += [io[i] for i in range(m)]
        if sym in ('y', 'xy'):
            m = len(plist)
            plist += [flip(plist[i], 1) for i in range(m)]
            io += [io[i] for i in range(m)]
        self.pfull = ComParticle(self.eps, plist, io)
        nk = self.symtable.shape[1]
        m = len(self.p)
        if closed:
            # particle c together with its mirror images forms a closed surface
            full_closed = [None] * (m * nk)
            for c in closed:
                for c1 in np.atleast_1d(c):
                    c1 = int(c1)
                    imgs = [c1 + k * m for k in range(nk)]
                    for j in imgs:
                        full_closed[j - 1] = imgs
            self.pfull.closed = [c if c is not None else [j + 1]
                                 for j, c in enumerate(full_closed)]
        self._n = sum(q.nfaces for q in self.p)

    @property
    def nk(self):
        return self.symtable.shape[1]

    def full(self):
        return self.pfull

    @property
    def n(self):
        return self._n

    nfaces = n

    @property
    def pos(self):
        return np.asarray(self.pfull.pos)[:self._n]

    @property
    def nvec(self):
        return np.asarray(self.pfull.nvec)[:self._n]

    @property
    def area(self):
        return np.asarray(self.pfull.area)[:self._n]

    def eps1(self, enei):
        return np.asarray(self.pfull.eps1(enei))[:self._n]

    def eps2(self, enei):
        return np.asarray(self.pfull.eps2(enei))[:self._n]

    def symvalue(self, key):
        """Symmetry values of ``key`` ('+', '-' for sym x / y; '++', '+-',
        '-+', '--' for xy), one row per key (comparticle_mirror.py:318-345)."""
        keys = [key] if isinstance(key, str) else list(key)
        for k in keys:
            if k not in _SYMVAL or len(_SYMVAL[k]) != self.nk:
                raise ValueError("Unknown symmetry key: {}".format(k))
        return np.array([_SYMVAL[k] for k in keys], dtype=np.float64)

    def symindex(self, tab):
        """Row of ``symtable`` equal to the symmetry values ``tab``."""
        tab = np.atleast_1d(tab)
        for i in range(self.symtable.shape[0]):
            if np.allclose(self.symtable[i], tab):
                return i
        raise ValueError("Symmetry values {} not found in table".format(tab))


_SCALARS = ('phi', 'phip', 'phi1', 'phi2', 'phi1p', 'phi2p', 'sig', 'sig1', 'sig2')
_VECTORS = ('a1', 'a1p', 'a2', 'a2p', 'e', 'h', 'h1', 'h2')


class CompStructMirror(object):
    """Values of the irreducible part, one ``CompStruct`` per symmetry
    combination in ``val`` (each with a 3 x nk ``symval``: rows x, y, z)
    (comparticle_mirror.py:9-106)."""

    def __init__(self, p, enei, fun=None):
        self.p = p
        self.enei = enei
        self.fun = fun
        self.val = []

    def full(self):
        return self.fun(self) if self.fun is not None else self

    def expand(self):
        """Every value on the full particle: image k of a scalar is
        symval[z, k] times the value, component l of a vector
        symval[l, k] times its component l."""
        out = []
        pf = self.p.full()
        for v in self.val:
            sv = v.symval
            nk = sv.shape[1]
            r = CompStruct(pf, self.enei)
            for name, a in v.val.items():
                if name == 'symval' or not isinstance(a, np.ndarray):
                    continue
                if name in _SCALARS:
                    r[name] = np.concatenate([a] + [sv[-1, k] * a for k in range(1, nk)])
                elif name in _VECTORS:
                    parts = [a]
                    for k in range(1, nk):
                        b = a.copy()
                        for l in range(3):
                            b[:, l] = sv[l, k] * a[:, l]
                        parts.append(b)
                    r[name] = np.concatenate(parts)
            out.append(r)
        return tuple(out)


class PlaneWaveRetMirror(object):
    """Plane waves along +-z on a mirror-symmetric particle
    (mnpbem/simulation/planewave_ret_mirror.py:8-198): pol in the xy plane."""

    def __init__(self, pol, dir, medium=1, **options):
        pol = np.atleast_2d(np.asarray(pol, dtype=float))
        dir = np.atleast_2d(np.asarray(dir, dtype=float))
        if not np.allclose(pol[:, 2], 0):
            raise AssertionError("pol[:, 2] must be 0 for mirror symmetry")
        self.pol, self.dir = pol, dir
        self.exc = PlaneWaveRet(pol, dir, medium=medium, **options)

    def potential(self, p, enei):
        """Two components: x- and y-polarised waves along +z and -z (2
        columns each), with the symmetry values of their x, y, z parts."""
        pot = CompStructMirror(p, enei, lambda s: self.full(s))
        for i in range(2):
            pb = np.zeros((2, 3))
            pb[:, i] = 1.0
            db = np.array([[0, 0, 1.0], [0, 0, -1.0]])
            pot.val.append(PlaneWaveRet(pb, db, medium=self.exc.medium).potential(p, enei))
        keys = {'x': (['+', '-', '-'], ['-', '+', '+']),
                'y': (['+', '-', '+'], ['-', '+', '-']),
                'xy': (['++', '--', '-+'], ['--', '++', '+-'])}[p.sym]
        pot.val[0].symval = p.symvalue(keys[0])
        pot.val[1].symval = p.symvalue(keys[1])
        return pot

    __call__ = potential

    def full(self, val):
        """Values on the full particle for the requested polarisations:
        pol_x times the x component plus pol_y times the y component, column
        of the matching propagation direction."""
        v1, v2 = val.expand()[:2]
        pf = v1.p
        out = CompStruct(pf, val.enei)
        npol = self.pol.shape[0]
        for name in v1.val:
            if name not in v2.val or not isinstance(v1.val[name], np.ndarray):
                continue
            a, b = v1.val[name], v2.val[name]
            shape = a.shape[:-1] + (npol,) if a.ndim > 1 else a.shape + (npol,)
            r = np.zeros(shape, dtype=complex)
            for ip in range(npol):
                j = 0 if self.dir[ip, 2] > 0 else 1
                r[..., ip] = self.pol[ip, 0] * a[..., j] + self.pol[ip, 1] * b[..., j]
            out[name] = r
        return out, pf

    def extinction(self, sig):
        return self.exc.extinction(self.full(sig)[0])

    def scattering(self, sig):
        return self.exc.scattering(self.full(sig)[0])

    def absorption(self, sig):
        return self.exc.absorption(self.full(sig)[0])


class BEMRetMirror(object):
    """Retarded BEM solver on the irreducible part of a mirror-symmetric
    particle, FP64 on the GPU (mnpbem/bem/bem_ret_mirror.py:147-815)."""

    def __init__(self, p, enei=None, **options):
        if not isinstance(p, ComParticleMirror):
            raise TypeError("BEMRetMirror: expected a ComParticleMirror")
        self.p = p
        self.device = torch.device('cuda')
        self.tables = SurfaceTables(p.pfull, rel_cutoff=options.get('RelCutoff', 3),
                                    abs_cutoff=options.get('AbsCutoff', 0))
        self.enei = None
        self.nvec = torch.from_numpy(np.ascontiguousarray(p.nvec, dtype=np.float64)).to(self.device)
        if enei is not None:
            self.init(enei)

    def init(self, enei):
        """Matrices of every symmetry value at ``enei`` (bem_ret_mirror.py:182-328)."""
        if self.enei is not None and self.enei == enei:
            return self
        from .bem import _scalar_eps
        p, t, dev = self.p, self.tables, self.device
        n, nf, nk = p.n, t.n, p.nk
        nsym = p.symtable.shape[0]
        sh = _lib.stream_handle()
        c128 = dict(dtype=torch.complex128, device=dev)
        kblk, sblk = t.k_tables([enei])
        full = [torch.empty((1, nf, nf), **c128) for _ in range(4)]   # G1, H1, G2, H2
        t.assemble(kblk, sblk, tuple(full), mode=0)
        G = torch.empty((2, nsym, n, n), **c128)
        H = torch.empty((2, nsym, n, n), **c128)
        tab = np.ascontiguousarray(p.symtable, dtype=np.float64)
        for src, dst in ((full[0], G[0]), (full[2], G[1]), (full[1], H[0]), (full[3], H[1])):
            call('mnpb_mirror_contract', sh, n, nk, nsym, 1, ptr(src), nf, nf * nf, ptr(tab),
                 ptr(dst), n, n * n)
        del full
        self.G, self.H = G, H
        self.Dinv = torch.empty((nsym, n, n), **c128)
        self.piv = torch.empty((3, nsym, n), dtype=torch.int32, device=dev)
        info = torch.zeros(3 * nsym, dtype=torch.int32, device=dev)
        wb = int(_lib.lib().mnpb_bemret_mirror_workspace(n, nsym))
        work = torch.empty(wb, dtype=torch.uint8, device=dev)
        call('mnpb_bemret_init_mirror_f64', sh, n, nsym, ptr(G[0]), ptr(G[1]), ptr(H[0]),
             ptr(H[1]), n, n * n, ptr(self.Dinv), ptr(self.piv), ptr(info), ptr(work), wb)
        if info.any():
            raise _lib.MNPBError('BEMRetMirror', 3, 'zero pivot in a symmetry block')
        e1, e2 = _scalar_eps(p, enei)
        self.eps = torch.tensor([[e1.real, e1.imag, e2.real, e2.imag]], dtype=torch.float64,
                                device=dev)
        self.kvac = torch.tensor([2 * np.pi / enei], dtype=torch.float64, device=dev)
        self._sigma = {}
        self.enei = enei
        return self

    def _sigma_lu(self, x, y, z):
        key = (x, y, z)
        if key not in self._sigma:
            n = self.p.n
            S = torch.empty((1, n, n), dtype=torch.complex128, device=self.device)
            piv = torch.empty((1, n), dtype=torch.int32, device=self.device)
            info = torch.zeros(1, dtype=torch.int32, device=self.device)
            nsym = self.p.symtable.shape[0]
            call('mnpb_bemret_sigma_mirror_f64', _lib.stream_handle(), n, nsym, 1,
                 ptr(self.H[0]), ptr(self.H[1]), ptr(self.Dinv), n, n * n, ptr(self.eps),
                 ptr(self.kvac), ptr(self.nvec), x, y, z, ptr(S), n * n, ptr(piv), ptr(info))
            if info.any():
                raise _lib.MNPBError('BEMRetMirror', 3, 'zero pivot in Sigma')
            self._sigma[key] = (S, piv)
        return self._sigma[key]

    def solve(self, exc):
        """Surface charges and currents of every symmetry component
        (bem_ret_mirror.py:654-760): a ``CompStructMirror``."""
        from .bem import BEMRet
        self.init(exc.enei)
        p = self.p
        n = p.n
        nsym = p.symtable.shape[0]
        sh = _lib.stream_handle()
        sig = CompStructMirror(p, exc.enei, exc.fun)
        for v in exc.val:
            sv = v.symval
            x, y, z = (p.symindex(sv[0]), p.symindex(sv[1]), p.symindex(sv[2]))
            S, pivS = self._sigma_lu(x, y, z)
            pots, K = BEMRet._pots(v, n)
            d_pots = torch.from_numpy(pots).to(self.device).unsqueeze(0)
            xin = torch.empty((1, 8, K, n), dtype=torch.complex128, device=self.device)
            xout = torch.empty_like(xin)
            call('mnpb_bemret_excitation', sh, n, 1, K, ptr(d_pots), ptr(self.eps),
                 ptr(self.kvac), ptr(self.nvec), 0, ptr(xin))
            wb = int(_lib.lib().mnpb_bemret_solve_mirror_workspace(n, 1, K))
            work = torch.empty(wb, dtype=torch.uint8, device=self.device)
            call('mnpb_bemret_solve_mirror_f64', sh, n, nsym, 1, K, ptr(self.G[0]),
                 ptr(self.G[1]), ptr(self.H[0]), ptr(self.Dinv), n, n * n, ptr(self.piv),
                 ptr(S), n * n, ptr(pivS), x, y, z, ptr(self.eps), ptr(self.kvac),
                 ptr(self.nvec), ptr(xin), ptr(xout), ptr(work), wb)
            X = xout[0].cpu().numpy()
            val = CompStruct(p, exc.enei, sig1=X[0].T.copy(), h1=X[1:4].transpose(2, 0, 1).copy(),
                             sig2=X[4].T.copy(), h2=X[5:8].transpose(2, 0, 1).copy())
            val.symval = sv
            sig.val.append(val)
        return sig, self

    def __truediv__(self, exc):
        return self.solve(exc)

    def __call__(self, enei):
        return self.init(enei)


class PlaneWaveStatMirror(object):
    """Quasistatic plane wave on a mirror-symmetric particle
    (mnpbem/simulation/planewave_stat_mirror.py:9-180): the x- and y-polarised
    potentials phip = -n . e with their symmetry values; ``full`` combines
    them on the full particle with the requested polarisations."""

    def __init__(self, pol, medium=1, **options):
        self.pol = np.atleast_2d(np.asarray(pol, dtype=float))
        self.exc = PlaneWaveStat(self.pol, medium=medium, **options)

    def potential(self, p, enei):
        pot = CompStructMirror(p, enei, lambda s: self.full(s))
        nvec = np.asarray(p.nvec)
        keys = {'x': (['+', '-', '-'], ['-', '+', '-']),
                'y': (['+', '-', '+'], ['-', '+', '-']),
                'xy': (['++', '--', '-+'], ['--', '++', '+-'])}
        if p.sym not in keys:
            raise ValueError("PlaneWaveStatMirror: unknown symmetry {!r}".format(p.sym))
        for i in range(2):
            v = CompStruct(p, enei, phip=-nvec[:, i].copy())
            v.symval = p.symvalue(keys[p.sym][i])
            pot.val.append(v)
        return pot

    __call__ = potential

    def full(self, val):
        """Values on the full particle: sum over the x and y parts weighted by
        each polarisation's x and y components (planewave_stat_mirror.py:92)."""
        parts = val.expand()
        pf = val.p.full()
        out = CompStruct(pf, val.enei)
        npol = self.pol.shape[0]
        for name in ('sig', 'phi', 'phip'):
            vecs = [e.val.get(name) for e in parts]
            if all(isinstance(v, np.ndarray) for v in vecs):
                r = np.zeros((vecs[0].shape[0], npol), dtype=complex)
                for ip in range(npol):
                    for ib, v in enumerate(vecs):
                        r[:, ip] += self.pol[ip, ib] * v
                out[name] = r
        return out, pf

    def extinction(self, sig):
        return self.exc.extinction(self.full(sig)[0])

    def scattering(self, sig):
        return self.exc.scattering(self.full(sig)[0])

    def absorption(self, sig):
        return self.exc.absorption(self.full(sig)[0])


class BEMStatMirror(object):
    """Quasistatic BEM solver on the irreducible part of a mirror-symmetric
    particle, FP64 on the GPU (mnpbem/bem/bem_stat_mirror.py:140-487): the
    full particle's refined, closure-corrected F contracted once per
    symmetry value (F_s = sum_k tab[s, k] F(:, image k), mnpb_mirror_contract),
    then per wavelength M_s = -(Lambda + F_s) factorised for every symmetry
    value in one batch, and each excitation value solved with the matrix of
    its symmetry."""

    def __init__(self, p, enei=None, **options):
        from .greenfun import CompGreenStat
        if not isinstance(p, ComParticleMirror):
            raise TypeError("BEMStatMirror: expected a ComParticleMirror")
        self.p = p
        self.device = torch.device('cuda')
        g = CompGreenStat(p.pfull, **options)
        n, nf, nk = p.n, g.tables.n, p.nk
        nsym = p.symtable.shape[0]
        tab = np.ascontiguousarray(p.symtable, dtype=np.float64)
        Fc = g.F_dev.to(torch.complex128)              # column-major, ld nf
        Fs = torch.empty((nsym, n, n), dtype=torch.complex128, device=self.device)
        call('mnpb_mirror_contract', _lib.stream_handle(), n, nk, nsym, 1, ptr(Fc), nf, nf * nf,
             ptr(tab), ptr(Fs), n, n * n)
        self.F = Fs.real.contiguous()                  # (nsym, n, n), column-major each
        del Fc, Fs, g
        self.enei = None
        if enei is not None:
            self.init(enei)

    def init(self, enei):
        if self.enei is not None and self.enei == enei:
            return self
        p, dev = self.p, self.device
        n, nsym = p.n, self.F.shape[0]
        e1, e2 = np.asarray(p.eps1(enei)), np.asarray(p.eps2(enei))
        eps = np.zeros((1, n, 4))
        eps[0, :, 0], eps[0, :, 1], eps[0, :, 2], eps[0, :, 3] = e1.real, e1.imag, e2.real, e2.imag
        d_eps = torch.from_numpy(eps).to(dev)
        sh = _lib.stream_handle()
        M = torch.empty((nsym, n, n), dtype=torch.complex128, device=dev)
        for s in range(nsym):
            call('mnpb_stat_matrix', sh, n, 1, ptr(self.F[s]), n, ptr(d_eps), ptr(M[s]), n, n * n)
        piv = torch.empty((nsym, n), dtype=torch.int32, device=dev)
        info = torch.zeros(nsym, dtype=torch.int32, device=dev)
        call('mnpb_getrf_f64', sh, n, nsym, ptr(M), n, n * n, ptr(piv), n, ptr(info))
        if info.cpu().numpy().any():
            raise _lib.MNPBError('BEMStatMirror', 3, 'zero pivot in a symmetry block')
        self._M, self._piv = M, piv
        self.enei = enei
        return self

    __call__ = init

    def solve(self, exc):
        """Surface charges of every excitation value (bem_stat_mirror.py:360)."""
        self.init(exc.enei)
        p, n = self.p, self.p.n
        sig = CompStructMirror(p, exc.enei, exc.fun)
        sh = _lib.stream_handle()
        for v in exc.val:
            ind = p.symindex(v.symval[-1, :])
            phip = np.asarray(v.phip)
            K = phip.size // n                  # trailing axes (npt, ndip, ...) as columns
            B = torch.from_numpy(np.ascontiguousarray(phip.reshape(n, K).T.astype(complex))) \
                .to(self.device).unsqueeze(0).contiguous()
            call('mnpb_getrs_f64', sh, n, 1, K, ptr(self._M[ind]), n, n * n, ptr(self._piv[ind]),
                 n, ptr(B), n, n * K)
            x = B[0].cpu().numpy().T.reshape(phip.shape)
            out = CompStruct(p, exc.enei, sig=x)
            out.symval = v.symval
            sig.val.append(out)
        return sig, self

    def __truediv__(self, exc):
        return self.solve(exc)


class _DipoleMirror(object):
    """Dipoles next to a mirror-symmetric particle
    (mnpbem/simulation/dipole_stat_mirror.py:15-274,
    dipole_ret_mirror.py:15-347).

    The unit dipoles at the points and at their mirror images (positions and
    moments flipped at the symmetry planes) give one excitation each;
    their sums and differences are the excitations of the symmetry values
    (x / y: image 0 +- image 1; xy: the four sign combinations of the
    images).  ``full`` takes the mean of the expanded solutions, the
    response to the unit dipoles at the points on the full particle, and
    contracts it with the requested moments; ``decayrate`` is the plain
    dipole class's decay rate of that.
    """

    # image k: (axes flipped, moment signs of the unit triple)
    _IMAGES = {'x': [((), (1, 1, 1)), ((0,), (-1, 1, 1))],
               'y': [((), (1, 1, 1)), ((1,), (1, -1, 1))],
               'xy': [((), (1, 1, 1)), ((0,), (-1, 1, 1)), ((1,), (1, -1, 1)),
                      ((0, 1), (-1, -1, 1))]}
    # symmetry values: (coefficients of the image excitations, symvalue keys)
    _COMBOS = {'x': [((1, 1), ['-', '+', '+']), ((1, -1), ['+', '-', '-'])],
               'y': [((1, 1), ['+', '-', '+']), ((1, -1), ['-', '+', '-'])],
               'xy': [((1, 1, 1, 1), ['-+', '+-', '++']), ((1, -1, 1, -1), ['++', '--', '-+']),
                      ((1, 1, -1, -1), ['--', '++', '+-']), ((1, -1, -1, 1), ['+-', '-+', '--'])]}

    def __init__(self, pt, dip=None, full=False, **options):
        self.dip = self._klass()(pt, dip, full=full, **options)
        self.sym = None
        self.mirror = []

    def _init_mirror(self, p):
        if self.sym == p.sym:
            return
        pt = self.dip.pt
        self.mirror = []
        for axes, signs in self._IMAGES[p.sym]:
            m = self._klass()(pt, np.diag(np.asarray(signs, dtype=float)))
            pos = m.h_pos.copy()
            for a in axes:
                pos[:, a] = -pos[:, a]
            m.h_pos = np.ascontiguousarray(pos)
            self.mirror.append(m)
        self.sym = p.sym

    def potential(self, p, enei):
        """Excitation of every symmetry value on the irreducible part."""
        self._init_mirror(p)
        vals = [m.potential(p, enei) for m in self.mirror]
        exc = CompStructMirror(p, enei, lambda x: self.full(x))
        for coef, key in self._COMBOS[p.sym]:
            v = CompStruct(p, enei)
            for name, a in vals[0].val.items():
                if isinstance(a, np.ndarray):
                    v[name] = sum(c * m.val[name] for c, m in zip(coef, vals))
            v.symval = p.symvalue(key)
            exc.val.append(v)
        return exc

    __call__ = potential

    def full(self, val):
        """Values on the full particle for the requested moments."""
        parts = val.expand()
        pf = val.p.full()
        out = CompStruct(pf, val.enei)
        dip = self.dip.dip                                          # (npt, 3, ndip)
        npt, ndip = dip.shape[0], dip.shape[2]
        for name in parts[0].val:
            vecs = [e.val.get(name) for e in parts]
            if not all(isinstance(v, np.ndarray) for v in vecs):
                continue
            mean = sum(vecs) / len(vecs)
            nf = mean.shape[0]
            if name in _VECTORS:
                r = np.einsum('nlic,icj->nlij', mean.reshape(nf, 3, npt, 3), dip)
                out[name] = r.reshape(nf, 3, npt * ndip) if self._flat else r
            else:
                r = np.einsum('nic,icj->nij', mean.reshape(nf, npt, 3), dip)
                out[name] = r.reshape(nf, npt * ndip) if self._flat else r
        return out, pf

    def field(self, p, enei, inout=1):
        return self.dip.field(p, enei)

    def decayrate(self, sig):
        return self.dip.decayrate(self.full(sig)[0])

    def farfield(self, spec=None, enei=None):
        return self.dip.farfield(spec, enei)


class DipoleStatMirror(_DipoleMirror):
    """Quasistatic dipoles next to a mirror-symmetric particle
    (mnpbem/simulation/dipole_stat_mirror.py:15-274): excitations phip
    (n, npt, 3) per symmetry value for ``BEMStatMirror``; ``full`` gives
    (n_full, npt, ndip)."""

    _flat = False

    @staticmethod
    def _klass():
        from .points import DipoleStat
        return DipoleStat


class DipoleRetMirror(_DipoleMirror):
    """Retarded dipoles next to a mirror-symmetric particle
    (mnpbem/simulation/dipole_ret_mirror.py:15-347): the eight potentials
    of ``DipoleRet`` per symmetry value for ``BEMRetMirror``; ``full`` gives
    the charges and currents on the full particle in ``DipoleRet``'s column
    layout (point q, moment j at column q ndip + j); ``scattering`` and
    ``decayrate`` are ``DipoleRet``'s of that."""

    _flat = True

    @staticmethod
    def _klass():
        from .points import DipoleRet
        return DipoleRet

    def scattering(self, sig):
        return self.dip.scattering(self.full(sig)[0])


class CompGreenRetMirror(object):
    """Retarded Green function of a mirror-symmetric particle with itself
    (mnpbem/greenfun/compgreen_ret_mirror.py:14-240): the full particle's
    matrices (assembled on the GPU by ``CompGreenRet``), rows of the
    irreducible part, contracted per symmetry value s as
    g_s = sum_k symtable[s, k] M(:, block k); ``field`` gives the fields of
    a mirror solution at the faces, per symmetry value."""

    def __init__(self, p, p2=None, **options):
        from .greenfun import CompGreenRet
        if not isinstance(p, ComParticleMirror):
            raise TypeError("CompGreenRetMirror: expected a ComParticleMirror")
        self.p = p
        self.g = CompGreenRet(p.pfull, **options)
        self.device = torch.device('cuda')

    def eval(self, i, j, key, enei):
        """Contracted matrices, one per symmetry value: (n, n), or (n, 3, n)
        for Gp / H1p / H2p; zeros where no block connects."""
        p = self.p
        n, nk = p.n, p.nk
        tab = torch.from_numpy(np.ascontiguousarray(p.symtable)).to(self.device,
                                                                    torch.complex128)
        m = self.g.eval(i, j, key, enei)
        if np.isscalar(m):
            return [0] * tab.shape[0]
        m = torch.as_tensor(np.asarray(m) if not torch.is_tensor(m) else m).to(self.device)
        m = m[:n].to(torch.complex128)
        if m.dim() == 2:
            b = m.reshape(n, nk, n)
            return [torch.einsum('k,rkc->rc', tab[s], b) for s in range(tab.shape[0])]
        b = m.reshape(n, 3, nk, n)
        return [torch.einsum('k,rlkc->rlc', tab[s], b) for s in range(tab.shape[0])]

    @staticmethod
    def _indmul(mats, v, ind):
        if not torch.is_tensor(mats[0]):
            return 0
        return torch.stack([mats[ind[l]] @ v[:, l] for l in range(3)], dim=1)

    @staticmethod
    def _mm3(a, x):
        if not torch.is_tensor(a):
            return 0
        return torch.stack([a[:, l] @ x for l in range(3)], dim=1)

    @staticmethod
    def _indcross(mats, v, ind):
        if not torch.is_tensor(mats[0]):
            return 0
        im = lambda k, c: mats[ind[k]][:, c]
        return torch.stack([im(2, 1) @ v[:, 2] - im(1, 2) @ v[:, 1],
                            im(0, 2) @ v[:, 0] - im(2, 0) @ v[:, 2],
                            im(1, 0) @ v[:, 1] - im(0, 1) @ v[:, 0]], dim=1)

    def field(self, sig, inout=1):
        """e = i k (G1 h1 + G2 h2) - H1p sig1 - H2p sig2 and
        h = H1p x h1 + H2p x h2 for every symmetry value
        (compgreen_ret_mirror.py:104-160): matrices of the symmetry value of
        each Cartesian component, the z one for the charges; e, h (n, 3[, K])."""
        p, enei = self.p, sig.enei
        k = 2 * np.pi / enei
        G1 = self.eval(inout - 1, 0, 'G', enei)
        G2 = self.eval(inout - 1, 1, 'G', enei)
        pk = 'H1p' if inout == 1 else 'H2p'
        H1p = self.eval(inout - 1, 0, pk, enei)
        H2p = self.eval(inout - 1, 1, pk, enei)
        out = CompStructMirror(p, enei, sig.fun)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=complex))) \
            .to(self.device)
        for s in sig.val:
            ind = [p.symindex(s.symval[l]) for l in range(3)]
            one = np.asarray(s.sig1).ndim == 1
            sig1, sig2 = T(s.sig1), T(s.sig2)
            h1, h2 = T(s.h1), T(s.h2)
            if one:
                sig1, sig2 = sig1[:, None], sig2[:, None]
                h1, h2 = h1[:, :, None], h2[:, :, None]
            e = 0
            for term in (1j * k * self._indmul(G1, h1, ind) if torch.is_tensor(G1[0]) else 0,
                         -self._mm3(H1p[ind[2]], sig1) if torch.is_tensor(H1p[0]) else 0,
                         1j * k * self._indmul(G2, h2, ind) if torch.is_tensor(G2[0]) else 0,
                         -self._mm3(H2p[ind[2]], sig2) if torch.is_tensor(H2p[0]) else 0):
                e = e + term
            h = 0
            for term in (self._indcross(H1p, h1, ind), self._indcross(H2p, h2, ind)):
                h = h + term
            cvt = lambda a: (a.cpu().numpy()[..., 0] if one else a.cpu().numpy()) \
                if torch.is_tensor(a) else a
            val = CompStruct(p, enei, e=cvt(e), h=cvt(h))
            val.symval = s.symval
            out.val.append(val)
        return out
