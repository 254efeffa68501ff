"""Points off the particle surface: point sets, dipole excitations and the
Green functions between points and faces.

``Point`` / ``ComPoint`` mirror mnpbem/geometry/compoint.py (points grouped by
the dielectric medium they sit in).  ``DipoleRet`` mirrors
mnpbem/simulation/dipole_ret.py: ``potential`` (the BEM excitation),
``field`` (the dipoles' own fields), ``farfield``, ``scattering`` and
``decayrate``.  ``CompGreenRetPoints`` is the reference's
``CompGreenRet(points, particle)`` (greenfun/compgreen_ret.py with a point
set as p1): entries, fields and potentials at the points, computed on the
GPU from on-the-fly entries (far formula, refined point-face pairs from
Taylor coefficients integrated over the faces' quadrature points).

All GPU work goes through ``libmnpbem_b200.so``; the host only classifies
points (once per point set) and reduces the 256-direction Poynting sums, as
``PlaneWaveRet.scattering`` does.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .excitation import _inout_faces, pinfty
from .greenfun import _nfaces, _points, refinematrix_csr
from .materials import eps_k

__all__ = ["Point", "ComPoint", "DipoleRet", "DipoleStat", "CompGreenRetPoints",
           "CompGreenStatPoints", "is_point_set"]


class Point(object):
    """Positions (n, 3) with zero normals and unit areas (compoint.py:11-100)."""

    def __init__(self, pos, nvec=None, area=None):
        self.pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
        n = self.pos.shape[0]
        self.nvec = (np.zeros((n, 3)) if nvec is None
                     else np.atleast_2d(np.asarray(nvec, dtype=np.float64)))
        self.area = np.ones(n) if area is None else np.asarray(area, dtype=np.float64).ravel()

    @property
    def n(self):
        return self.pos.shape[0]

    nfaces = n

    def __add__(self, other):
        return Point(np.vstack([self.pos, other.pos]), np.vstack([self.nvec, other.nvec]),
                     np.concatenate([self.area, other.area]))


class ComPoint(object):
    """Points grouped by the medium they sit in (compoint.py:102-480).

    ``ComPoint(p, pos, mindist=None, medium=None)`` classifies each position
    by the nearest face centroid of every particle of ``p``: the side of its
    normal gives the outside or inside medium; points closer than
    ``mindist`` are dropped.  Groups are ordered by medium index, so
    ``pos`` is the input reordered.  ``ComPoint(eps, [Point, ...], inout)``
    builds the groups directly.
    """

    def __init__(self, p_or_eps, pos_or_points, inout_or_medium=None, mindist=None,
                 medium=None):
        if isinstance(pos_or_points, list) and pos_or_points and \
                isinstance(pos_or_points[0], (Point, np.ndarray)):
            self.eps = p_or_eps
            self.p = [q if isinstance(q, Point) else Point(q) for q in pos_or_points]
            self.inout = np.atleast_1d(np.asarray(inout_or_medium, dtype=int))
            self._mask = list(range(len(self.p)))
            return
        cp = p_or_eps
        pos = np.atleast_2d(np.asarray(pos_or_points, dtype=np.float64)).copy()
        self.eps = cp.eps
        self._pin = cp
        med = self._classify(cp, pos, 0.0 if mindist is None else mindist)
        self.p, inout, self._ind = [], [], []
        for m in np.unique(med[med > 0]):
            idx = np.where(med == m)[0]
            self.p.append(Point(pos[idx]))
            inout.append(int(m))
            self._ind.append(idx)
        self.inout = np.array(inout, dtype=int)
        if medium is not None:
            medium = [medium] if np.isscalar(medium) else list(medium)
            self._mask = [i for i, io in enumerate(self.inout) if io in medium]
        else:
            self._mask = list(range(len(self.p)))

    @staticmethod
    def _classify(cp, pos, mindist):
        """Medium of every position (compoint.py:260-301): per particle, the
        nearest face centroid; the sign of (pos - centroid) . normal picks
        the outside (>= 0) or inside medium; 0 if closer than mindist.  Later
        particles overwrite earlier ones, as the reference's loop does."""
        med = np.ones(pos.shape[0], dtype=int)
        inout = np.atleast_2d(np.asarray(cp.inout))
        for ip, part in enumerate(cp.p):
            fpos = np.asarray(part.pos, dtype=np.float64)
            if fpos.shape[0] == 0:
                continue
            nvec = np.asarray(part.nvec, dtype=np.float64)
            md = abs(mindist if np.isscalar(mindist) else mindist[ip])
            for j in range(pos.shape[0]):
                d = np.sqrt(np.sum((fpos - pos[j]) ** 2, axis=1))
                imin = int(np.argmin(d))
                if d[imin] < md:
                    med[j] = 0
                    continue
                side = 1 if np.dot(pos[j] - fpos[imin], nvec[imin]) >= 0 else 0
                med[j] = int(inout[ip, side])
        return med

    def _active(self):
        return [self.p[i] for i in self._mask]

    @property
    def pos(self):
        act = self._active()
        return np.vstack([q.pos for q in act]) if act else np.zeros((0, 3))

    @property
    def n(self):
        return sum(q.n for q in self._active())

    nfaces = n

    @property
    def nvec(self):
        return np.zeros((self.n, 3))

    @property
    def area(self):
        return np.ones(self.n)

    @property
    def index(self):
        out, off = [], 0
        for q in self._active():
            out.append(np.arange(off, off + q.n))
            off += q.n
        return out

    @property
    def np(self):
        return len(self._mask)

    def eps1(self, enei):
        vals = np.zeros(self.n, dtype=complex)
        off = 0
        for i in self._mask:
            vals[off:off + self.p[i].n] = eps_k(self.eps[int(self.inout[i]) - 1], enei)[0]
            off += self.p[i].n
        return vals

    eps2 = eps1


def is_point_set(p):
    """True for this package's or the reference's ComPoint / Point (no faces)."""
    if isinstance(p, (ComPoint, Point)):
        return True
    return type(p).__name__ in ('ComPoint', 'Point') and not hasattr(p, 'bradius')


def point_media(pt):
    """Positions (npt, 3) and the medium of every point (npt,) of a point set
    (ours or the reference's ComPoint, whose active groups are ``_mask``)."""
    pos = np.ascontiguousarray(np.asarray(pt.pos, dtype=np.float64).reshape(-1, 3))
    groups = getattr(pt, 'p', None)
    if groups is None:
        return pos, np.ones(pos.shape[0], dtype=np.int32)
    mask = list(getattr(pt, '_mask', getattr(pt, 'mask', range(len(groups)))))
    inout = np.atleast_1d(np.asarray(pt.inout, dtype=int))
    med = np.concatenate([np.full(groups[i].n, inout[i], dtype=np.int32) for i in mask]) \
        if mask else np.zeros(0, dtype=np.int32)
    if med.shape[0] != pos.shape[0]:
        raise ValueError("point set: group sizes do not match the positions")
    return pos, med.astype(np.int32)


def _medium_tables(eps_funcs, eneis):
    """(B, nmed) complex eps, k and nb = sqrt(eps) as float64 (re, im) pairs."""
    B, M = len(eneis), len(eps_funcs)
    e = np.zeros((B, M), dtype=complex)
    k = np.zeros((B, M), dtype=complex)
    for b, enei in enumerate(eneis):
        for m, f in enumerate(eps_funcs):
            e[b, m], k[b, m] = eps_k(f, enei)
    return e, k, np.sqrt(e)


def _dev(a, dev, dtype=None):
    a = np.ascontiguousarray(a if dtype is None else np.asarray(a, dtype=dtype))
    if np.iscomplexobj(a):
        a = a.view(np.float64)
    return torch.from_numpy(a).to(dev)


class _FaceData(object):
    """Device positions, normals, areas and side media of a particle's faces."""

    def __init__(self, p, dev):
        self.n = _nfaces(p)
        self.pos = _dev(np.asarray(p.pos, dtype=np.float64), dev)
        self.nvec = _dev(np.asarray(p.nvec, dtype=np.float64), dev)
        self.area = _dev(np.asarray(p.area, dtype=np.float64), dev)
        self.h_med = np.ascontiguousarray(_inout_faces(p), dtype=np.int32)
        self.med = _dev(self.h_med, dev)


class CompGreenRetPoints(object):
    """Retarded Green function between a point set (p1) and a particle (p2).

    The reference's ``CompGreenRet(pt, p)`` (greenfun/compgreen_ret.py:14
    with a ComPoint as p1): a point in medium m is connected to side s of a
    face when the face's side-s medium is m; G and the Cartesian derivative
    Gp (= H1p = H2p, no self terms between points and faces) use that
    medium's wavenumber.  Point-face pairs closer than RelCutoff boundary
    radii of the face (refine_utils.py:29-150 with the face radius as the
    unit, the reference's fallback for sources without a radius) take
    order-5 refined entries (greenret_refined.py:287-442, the point as
    source).  F, H1 and H2 vanish: points carry zero normals.
    """

    def __init__(self, pt, p, **options):
        if options.get('order', 5) != 5 or not options.get('refine', True):
            raise NotImplementedError("CompGreenRetPoints: refinement order 5 only")
        if options.get('deriv', 'cart') != 'cart':
            raise NotImplementedError("CompGreenRetPoints: deriv='cart' (the default) only")
        self.p1, self.p2 = pt, p
        dev = torch.device('cuda')
        self.device = dev
        h_pos, h_med = point_media(pt)
        if h_pos.shape[0] == 0:
            raise ValueError("CompGreenRetPoints: empty point set")
        if h_med.max() > len(p.eps):
            raise ValueError("CompGreenRetPoints: point medium outside the dielectric table")
        self.npt, self.h_pos, self.h_med = h_pos.shape[0], h_pos, h_med
        self.faces = _FaceData(p, dev)
        self.eps_funcs = list(p.eps)
        rad2 = np.ascontiguousarray(np.asarray(p.bradius(), dtype=np.float64))
        fpos = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))
        rptr, cols, kinds = refinematrix_csr(h_pos, fpos, None, rad2,
                                             options.get('AbsCutoff', 0.0),
                                             options.get('RelCutoff', 3.0))
        if np.any(kinds == 2):
            raise ValueError("CompGreenRetPoints: a point coincides with a face centroid")
        rows = np.repeat(np.arange(self.npt, dtype=np.int32), np.diff(rptr)).astype(np.int32)
        self.nref = len(cols)
        self.ptpos = _dev(h_pos, dev)
        self.ptmed = _dev(h_med, dev)
        self.rptr = _dev(rptr, dev, np.int64)
        self.cols = _dev(cols if len(cols) else np.zeros(1, np.int32), dev, np.int32)
        f64 = dict(dtype=torch.float64, device=dev)
        self.g = torch.zeros((max(self.nref, 1), 6), **f64)
        self.f = torch.zeros((max(self.nref, 1), 3, 6), **f64)
        if self.nref:
            qpos, qw, qoff = _points(p, 'quad')
            keep = [_dev(a, dev) for a in (qpos, qw, qoff)]
            call('mnpb_refine_points', _lib.stream_handle(), self.npt, ptr(self.ptpos),
                 self.faces.n, ptr(self.faces.pos), self.nref, ptr(_dev(rows, dev)),
                 ptr(self.cols), ptr(keep[0]), ptr(keep[1]), ptr(keep[2]), ptr(self.g),
                 ptr(self.f))
            torch.cuda.current_stream().synchronize()

    def _args(self, kt):
        fd = self.faces
        return (self.npt, ptr(self.ptpos), ptr(self.ptmed), fd.n, ptr(fd.pos), ptr(fd.area),
                ptr(fd.med), len(self.eps_funcs), ptr(kt), ptr(self.rptr), ptr(self.cols),
                ptr(self.g), ptr(self.f))

    def connected(self, side):
        """True if any point borders side ``side`` (0 inside, 1 outside) of a face."""
        return bool(np.any(self.h_med[:, None] == self.faces.h_med[None, :, side]))

    def eval(self, i, j, key, enei):
        """(npt, n) for G, (npt, 3, n) for Gp / H1p / H2p of face side j
        (compgreen_ret.py:507-553); 0 where nothing connects, and for F,
        H1, H2 (zero point normals)."""
        if i != 0:
            raise IndexError("CompGreenRetPoints.eval: a point set has one region (0)")
        if key not in ('G', 'F', 'H1', 'H2', 'Gp', 'H1p', 'H2p'):
            raise ValueError("Unknown key: {}".format(key))
        if key in ('F', 'H1', 'H2') or not self.connected(j):
            return 0
        _, k, _ = _medium_tables(self.eps_funcs, [enei])
        kt = _dev(k, self.device)
        vec = key != 'G'
        n = self.faces.n
        out = torch.zeros((self.npt, 3, n) if vec else (self.npt, n), dtype=torch.complex128,
                          device=self.device)
        call('mnpb_point_green_eval', _lib.stream_handle(), *self._args(kt), j, int(vec), 0, n,
             ptr(out))
        return out.cpu().numpy()

    def apply_device(self, sol, eneis, mode=0, diag=0, stream=None):
        """Fields (mode 0: e, h (B, npt, 3, KC)) or potentials (mode 1: phi
        (B, npt, KC), a (B, npt, 3, KC)) at the points for device solutions
        sol (B, 8, K, n)."""
        B, _, K, n = sol.shape
        if n != self.faces.n:
            raise ValueError("CompGreenRetPoints: solution has %d faces, particle %d"
                             % (n, self.faces.n))
        _, k, _ = _medium_tables(self.eps_funcs, eneis)
        kt = _dev(k, self.device)
        k0 = torch.tensor([2 * np.pi / e for e in eneis], dtype=torch.float64,
                          device=self.device)
        KC = diag if diag > 0 else K
        c128 = dict(dtype=torch.complex128, device=self.device)
        if mode == 0:
            o1 = torch.empty((B, self.npt, 3, KC), **c128)
        else:
            o1 = torch.empty((B, self.npt, KC), **c128)
        o2 = torch.empty((B, self.npt, 3, KC), **c128)
        call('mnpb_point_green', _lib.stream_handle(stream), *self._args(kt), mode, B, K, diag,
             ptr(k0), ptr(sol.contiguous()), ptr(o1), ptr(o2))
        return o1, o2

    def field(self, sig, inout=1):
        """e = i k (G1 h1 + G2 h2) - Gp sig1 - Gp sig2, h = Gp x h1 + Gp x h2
        at the points (compgreen_ret.py:912-978); (npt, 3[, K])."""
        from .excitation import PlaneWaveRet
        x, K = PlaneWaveRet._sol_device(sig, self.device)
        e, h = self.apply_device(x, [sig.enei], mode=0)
        e, h = e[0].cpu().numpy(), h[0].cpu().numpy()
        if K == 1:
            e, h = e[..., 0], h[..., 0]
        return CompStruct(self.p1, sig.enei, e=e, h=h)

    def potential(self, sig, inout=1):
        """phi = G1 sig1 + G2 sig2, a = G1 h1 + G2 h2 at the points
        (compgreen_ret.py:980-1036); phip and ap vanish (zero normals)."""
        from .excitation import PlaneWaveRet
        x, K = PlaneWaveRet._sol_device(sig, self.device)
        phi, a = self.apply_device(x, [sig.enei], mode=1)
        phi, a = phi[0].cpu().numpy(), a[0].cpu().numpy()
        if K == 1:
            phi, a = phi[..., 0], a[..., 0]
        z1, z2 = np.zeros_like(phi), np.zeros_like(a)
        if inout == 1:
            return CompStruct(self.p1, sig.enei, phi1=phi, phi1p=z1, a1=a, a1p=z2)
        return CompStruct(self.p1, sig.enei, phi2=phi, phi2p=z1, a2=a, a2p=z2)


class DipoleRet(object):
    """Oscillating dipoles at the points of a ComPoint (retarded,
    mnpbem/simulation/dipole_ret.py:19-899).

    ``dip``: moments (ndip, 3) shared by all points (default: the unit
    triple), or (npt, 3[, ndip]) per point with ``full=True``.  The
    excitation has K = npt * ndip columns, column q * ndip + idip.
    ``medium`` is the embedding medium of the far-field sphere.
    """

    def __init__(self, pt, dip=None, full=False, medium=1, pinfty=None, **options):
        self.pt = pt
        self.varargin = options
        if dip is None:
            dip, full = np.eye(3), False
        dip = np.asarray(dip, dtype=float)
        h_pos, h_med = point_media(pt)
        npt = h_pos.shape[0]
        if full:
            self.dip = dip.reshape(dip.shape + (1,)) if dip.ndim == 2 else dip
        else:
            dip = np.atleast_2d(dip)
            self.dip = np.tile(dip.T.reshape(1, 3, dip.shape[0]), (npt, 1, 1))
        if self.dip.shape[:2] != (npt, 3):
            raise ValueError("DipoleRet: dipole moments must be (npt, 3, ndip)")
        self.medium = medium
        self._pinfty = pinfty
        if npt == 0:
            raise ValueError("DipoleRet: empty point set")
        if h_med.max() > len(pt.eps):
            raise ValueError("DipoleRet: point medium outside the dielectric table")
        self.h_pos, self.h_med = h_pos, h_med
        self._dev = None
        self._faces = {}
        self._greens = {}

    @property
    def ndip(self):
        return self.dip.shape[2]

    def _device(self):
        if self._dev is None:
            dev = torch.device('cuda')
            self._dev = (dev, _dev(self.h_pos, dev), _dev(self.h_med, dev),
                         _dev(np.ascontiguousarray(self.dip, dtype=np.float64), dev))
        return self._dev

    def _face_data(self, p):
        key = id(p)
        if key not in self._faces:
            self._faces[key] = (p, _FaceData(p, self._device()[0]))
        return self._faces[key][1]

    def _sphere(self):
        if self._pinfty is None:
            return pinfty()
        q = self._pinfty
        return (np.ascontiguousarray(np.asarray(q.nvec, dtype=np.float64)),
                np.ascontiguousarray(np.asarray(q.area, dtype=np.float64)))

    # ---- excitation ---------------------------------------------------------
    def potential_device(self, p, tables, eneis, stream=None):
        """Potentials of every wavelength of ``eneis`` on the GPU:
        ((B, 16, K, n), K), the layout the BEM solvers take."""
        dev, ptpos, ptmed, dip = self._device()
        fd = self._face_data(p)
        B, K, n = len(eneis), self.h_pos.shape[0] * self.ndip, fd.n
        e, k, _ = _medium_tables(list(p.eps), eneis)
        k0 = torch.tensor([2 * np.pi / x for x in eneis], dtype=torch.float64, device=dev)
        pots = torch.empty((B, 16, K, n), dtype=torch.complex128, device=dev)
        call('mnpb_dipole_potential', _lib.stream_handle(stream), n, B, self.h_pos.shape[0],
             self.ndip, ptr(fd.pos), ptr(fd.nvec), ptr(fd.med), ptr(ptpos), ptr(ptmed), ptr(dip),
             len(p.eps), ptr(_dev(e, dev)), ptr(_dev(k, dev)), ptr(k0), ptr(pots))
        return pots, K

    def potential(self, p, enei):
        """phi1, phi1p, a1, a1p, phi2, phi2p, a2, a2p at the faces, (n, K)
        and (n, 3, K) host arrays (dipole_ret.py:319-421)."""
        pots, K = self.potential_device(p, None, [enei])
        x = pots[0].cpu().numpy()                       # (16, K, n)
        out = {}
        comp = 0
        for name, w in (('phi1', 1), ('phi1p', 1), ('a1', 3), ('a1p', 3), ('phi2', 1),
                        ('phi2p', 1), ('a2', 3), ('a2p', 3)):
            v = x[comp:comp + w]
            out[name] = v[0].T.copy() if w == 1 else v.transpose(2, 0, 1).copy()
            comp += w
        return CompStruct(p, enei, **out)

    __call__ = potential

    def field(self, p, enei, inout=1):
        """The dipoles' own fields at the faces of ``p`` (side ``inout``) or
        at the points of a point set: e, h (n, 3, npt, ndip)
        (dipole_ret.py:163-317)."""
        dev, ptpos, ptmed, dip = self._device()
        if is_point_set(p):
            obs, omed = point_media(p)
        else:
            obs = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))
            omed = np.ascontiguousarray(_inout_faces(p)[:, inout - 1], dtype=np.int32)
        npt, ndip = self.h_pos.shape[0], self.ndip
        e, k, nb = _medium_tables(list(p.eps), [enei])
        c128 = dict(dtype=torch.complex128, device=dev)
        eo = torch.empty((1, obs.shape[0], 3, npt * ndip), **c128)
        ho = torch.empty_like(eo)
        call('mnpb_dipole_field', _lib.stream_handle(), obs.shape[0], 1, npt, ndip,
             ptr(_dev(obs, dev)), ptr(_dev(omed, dev, np.int32)), ptr(ptpos), ptr(ptmed),
             ptr(dip), len(p.eps), ptr(_dev(e, dev)), ptr(_dev(k, dev)), ptr(_dev(nb, dev)),
             ptr(eo), ptr(ho))
        shape = (obs.shape[0], 3, npt, ndip)
        return CompStruct(p, enei, e=eo[0].cpu().numpy().reshape(shape),
                          h=ho[0].cpu().numpy().reshape(shape))

    # ---- far fields, scattering, decay rates --------------------------------
    def _emb(self, eps_funcs, eneis):
        e, k, nb = _medium_tables(eps_funcs, eneis)
        m = self.medium - 1
        return np.stack([e[:, m], k[:, m], nb[:, m]], axis=1)          # (B, 3) complex

    def farfield_device(self, eps_funcs, eneis, dirs, e=None, h=None, stream=None):
        """Far fields of the dipoles in the embedding medium on directions
        ``dirs``, added onto e, h (B, K, ndir, 3) (zeros if not given)."""
        dev, ptpos, ptmed, dip = self._device()
        npt, ndip = self.h_pos.shape[0], self.ndip
        d_dirs = _dev(np.asarray(dirs, dtype=np.float64), dev)
        nd = d_dirs.shape[0]
        if e is None:
            e = torch.zeros((len(eneis), npt * ndip, nd, 3), dtype=torch.complex128, device=dev)
            h = torch.zeros_like(e)
        on = _dev((self.h_med == self.medium).astype(np.int8), dev)
        call('mnpb_dipole_farfield', _lib.stream_handle(stream), nd, len(eneis), npt, ndip,
             ptr(ptpos), ptr(on), ptr(dip), ptr(d_dirs), ptr(_dev(self._emb(eps_funcs, eneis), dev)),
             ptr(e), ptr(h))
        return e, h

    def farfield(self, spec=None, enei=None):
        """Far fields of the dipoles alone on the sphere at infinity
        (dipole_ret.py:602-672): e, h (ndir, 3, npt, ndip)."""
        if enei is None:
            raise ValueError("DipoleRet.farfield: enei is required")
        nvec = (np.asarray(spec.pinfty.nvec, dtype=np.float64) if spec is not None
                else self._sphere()[0])
        e, h = self.farfield_device(list(self.pt.eps), [enei], nvec)
        shape = (self.h_pos.shape[0], self.ndip, nvec.shape[0], 3)
        e = e[0].cpu().numpy().reshape(shape).transpose(2, 3, 0, 1)
        h = h[0].cpu().numpy().reshape(shape).transpose(2, 3, 0, 1)
        return CompStruct(None, enei, e=e, h=h)

    def _total_farfield(self, sig):
        """Far fields of the surface charges (spectrum_ret.py:331-376) plus the
        dipoles' own, on the sphere at infinity: e, h (K, ndir, 3) device."""
        from .excitation import PlaneWaveRet, _Sides
        p = sig.p
        dev = self._device()[0]
        x, K = PlaneWaveRet._sol_device(sig, dev)
        nvec, _ = self._sphere()
        fd = self._face_data(p)
        sides = _Sides(p, self.medium, dev)
        emb = self._emb(list(p.eps), [sig.enei])
        km = _dev(emb[:, 1], dev)
        k0 = torch.tensor([2 * np.pi / sig.enei], dtype=torch.float64, device=dev)
        d_dirs = _dev(nvec, dev)
        nd = d_dirs.shape[0]
        e = torch.empty((1, K, nd, 3), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        call('mnpb_farfield', _lib.stream_handle(), fd.n, 1, K, nd, ptr(fd.pos), ptr(fd.area),
             ptr(sides.side_in), ptr(sides.side_out), ptr(d_dirs), ptr(km), ptr(k0), ptr(x),
             ptr(e), ptr(h))
        e, h = self.farfield_device(list(p.eps), [sig.enei], nvec, e, h)
        return e[0], h[0]

    def scattering(self, sig):
        """Power radiated by the dipoles and the particle through the sphere at
        infinity, sum area 0.5 Re(n . (e x h*)) (dipole_ret.py:674-791):
        (npt, ndip), and the differential cross section."""
        e, h = self._total_farfield(sig)
        e, h = e.cpu().numpy(), h.cpu().numpy()
        nvec, area = self._sphere()
        dsca = 0.5 * np.real(np.einsum('dc,kdc->kd', nvec, np.cross(e, np.conj(h))))
        sca = dsca @ area
        npt, ndip = self.h_pos.shape[0], self.ndip
        return sca.reshape(npt, ndip), CompStruct(None, sig.enei,
                                                  dsca=dsca.T.reshape(-1, npt, ndip))

    def _green(self, p):
        key = id(p)
        if key not in self._greens:
            self._greens[key] = (p, CompGreenRetPoints(self.pt, p, **self.varargin))
        return self._greens[key][1]

    def decayrate(self, sig):
        """Total, radiative and free-space decay rates (npt, ndip)
        (dipole_ret.py:517-600): with gamma = 4/3 k0^3 and nb the refractive
        index at the dipole, tot = 1 + Im(e_ind . dip) / (0.5 nb gamma) from
        the induced field at the dipole's own position, rad = sca / (2 pi k0)
        / (0.5 nb gamma), rad0 = nb gamma."""
        from .excitation import PlaneWaveRet
        g = self._green(sig.p)
        npt, ndip = self.h_pos.shape[0], self.ndip
        x, K = PlaneWaveRet._sol_device(sig, g.device)
        if K != npt * ndip:
            raise ValueError("DipoleRet.decayrate: solution has %d columns, expected %d"
                             % (K, npt * ndip))
        e, _ = g.apply_device(x, [sig.enei], mode=0, diag=ndip)
        e = e[0].cpu().numpy()                                   # (npt, 3, ndip)
        k0 = 2 * np.pi / sig.enei
        gamma = 4.0 / 3.0 * k0 ** 3
        sca, _ = self.scattering(sig)
        nb = np.sqrt(np.asarray(self.pt.eps1(sig.enei)))         # (npt,)
        ed = np.einsum('qcd,qcd->qd', e, self.dip)
        tot = np.real(1 + np.imag(ed) / (0.5 * nb[:, None] * gamma))
        rad = np.real(sca / (2 * np.pi * k0) / (0.5 * nb[:, None] * gamma))
        rad0 = np.real(np.broadcast_to(nb[:, None] * gamma, (npt, ndip))).copy()
        return tot, rad, rad0


class CompGreenStatPoints(CompGreenRetPoints):
    """Quasistatic Green function between a point set (p1) and a particle
    (p2): the reference's ``CompGreenStat(pt, p)`` (greenfun/compgreen_stat.py:
    219-465 with a ComPoint as p1).  G = a_j / d and Gp = -a_j (pt - pos_j) /
    d^3 for every point and face (no media: the surface charge radiates in
    free space); pairs closer than RelCutoff boundary radii of the face
    (greenfun/utils.py:43-140, the same rule as the retarded one) integrate
    1/d and its gradient over the face's quadrature points.  These are the
    k = 0 entries of ``CompGreenRetPoints``, evaluated by the same kernels
    with every point connected to side 0 of every face."""

    def __init__(self, pt, p, **options):
        CompGreenRetPoints.__init__(self, pt, p, **options)
        dev = self.device
        self.ptmed_all = _dev(np.ones(self.npt, dtype=np.int32), dev)
        fmed = np.zeros((self.faces.n, 2), dtype=np.int32)
        fmed[:, 0] = 1
        self.fmed_all = _dev(fmed, dev)
        self.k_zero = torch.zeros(2, dtype=torch.float64, device=dev)

    def _args_stat(self):
        fd = self.faces
        return (self.npt, ptr(self.ptpos), ptr(self.ptmed_all), fd.n, ptr(fd.pos), ptr(fd.area),
                ptr(self.fmed_all), 1, ptr(self.k_zero), ptr(self.rptr), ptr(self.cols),
                ptr(self.g), ptr(self.f))

    def eval(self, *args):
        """(npt, n) for G, (npt, 3, n) for Gp / H1p / H2p
        (compgreen_stat.py:560-700); 0 for F, H1, H2 (points carry zero
        normals).  The key is the last argument."""
        key = args[-1]
        if key not in ('G', 'F', 'H1', 'H2', 'Gp', 'H1p', 'H2p'):
            raise ValueError("Unknown key: {}".format(key))
        if key in ('F', 'H1', 'H2'):
            return 0
        vec = key != 'G'
        n = self.faces.n
        out = torch.zeros((self.npt, 3, n) if vec else (self.npt, n), dtype=torch.complex128,
                          device=self.device)
        call('mnpb_point_green_eval', _lib.stream_handle(), *self._args_stat(), 0, int(vec), 0, n,
             ptr(out))
        return out.cpu().numpy()

    def apply_sig(self, sig, mode=0, diag=0):
        """e (mode 0, (npt, 3, KC)) or phi (mode 1, (npt, KC)) at the points
        for surface charges sig (n, K) on the device."""
        n, K = sig.shape
        sol = torch.zeros((1, 8, K, n), dtype=torch.complex128, device=self.device)
        sol[0, 0] = sig.T
        KC = diag if diag > 0 else K
        c128 = dict(dtype=torch.complex128, device=self.device)
        o1 = torch.empty((1, self.npt, 3, KC) if mode == 0 else (1, self.npt, KC), **c128)
        o2 = torch.empty((1, self.npt, 3, KC), **c128)
        k0 = torch.ones(1, dtype=torch.float64, device=self.device)
        call('mnpb_point_green', _lib.stream_handle(), *self._args_stat(), mode, 1, K, diag,
             ptr(k0), ptr(sol), ptr(o1), ptr(o2))
        return o1[0]

    def _sig(self, sig):
        s = np.asarray(sig.sig)
        n = self.faces.n
        return s.shape[1:], torch.from_numpy(np.ascontiguousarray(
            s.reshape(n, -1).astype(complex))).to(self.device)

    def field(self, sig, inout=1):
        """e = -Gp sig at the points (compgreen_stat.py:974-1009):
        (npt, 3) + the trailing shape of sig."""
        shape, s = self._sig(sig)
        e = self.apply_sig(s, mode=0).cpu().numpy()
        return CompStruct(self.p1, sig.enei, e=e.reshape((self.npt, 3) + shape))

    def potential(self, sig, inout=1):
        """phi = G sig at the points (compgreen_stat.py:1011-1060); the
        surface derivative vanishes (zero point normals)."""
        shape, s = self._sig(sig)
        phi = self.apply_sig(s, mode=1).cpu().numpy().reshape((self.npt,) + shape)
        if inout == 1:
            return CompStruct(self.p1, sig.enei, phi1=phi, phi1p=np.zeros_like(phi))
        return CompStruct(self.p1, sig.enei, phi2=phi, phi2p=np.zeros_like(phi))


class DipoleStat(object):
    """Oscillating dipoles at the points of a ComPoint, quasistatic
    (mnpbem/simulation/dipole_stat.py:24-543).

    ``dip``: moments (ndip, 3) shared by all points (default: the unit
    triple), or (npt, 3[, ndip]) per point with ``full=True``.  The
    excitation ``phip`` is (n, npt, ndip); ``BEMStat`` solves it column by
    column (K = npt * ndip).
    """

    name = 'dipole'
    needs = {'sim': 'stat'}

    def __init__(self, pt, dip=None, full=False, **options):
        self.pt = pt
        self.varargin = options
        if dip is None:
            dip, full = np.eye(3), False
        dip = np.asarray(dip, dtype=float)
        h_pos, h_med = point_media(pt)
        npt = h_pos.shape[0]
        if npt == 0:
            raise ValueError("DipoleStat: empty point set")
        if full:
            self.dip = dip.reshape(dip.shape + (1,)) if dip.ndim == 2 else dip
        else:
            dip = np.atleast_2d(dip)
            self.dip = np.tile(dip.T.reshape(1, 3, dip.shape[0]), (npt, 1, 1))
        if self.dip.shape[:2] != (npt, 3):
            raise ValueError("DipoleStat: dipole moments must be (npt, 3, ndip)")
        self.h_pos, self.h_med = h_pos, h_med
        self._dev = None
        self._greens = {}

    @property
    def ndip(self):
        return self.dip.shape[2]

    def _device(self):
        if self._dev is None:
            dev = torch.device('cuda')
            self._dev = (dev, _dev(self.h_pos, dev),
                         _dev(np.ascontiguousarray(self.dip, dtype=np.float64), dev))
        return self._dev

    def _run(self, obs, nvec, enei):
        dev, ptpos, dip = self._device()
        npt, ndip = self.h_pos.shape[0], self.ndip
        eps = np.asarray(self.pt.eps1(enei), dtype=complex)
        nobs = obs.shape[0]
        shape = (nobs, npt, ndip) if nvec is not None else (nobs, 3, npt, ndip)
        out = torch.empty(shape, dtype=torch.complex128, device=dev)
        call('mnpb_dipole_stat_field', _lib.stream_handle(), nobs, npt, ndip, ptr(_dev(obs, dev)),
             ptr(_dev(nvec, dev)) if nvec is not None else None, ptr(ptpos), ptr(dip),
             ptr(_dev(eps, dev)), ptr(out))
        return out.cpu().numpy()

    def field(self, p, enei, inout=1):
        """Electric field e (n, 3, npt, ndip) of the dipoles at the faces or
        points of ``p`` (dipole_stat.py:149-250), screened by the dielectric
        function at each dipole; ``inout`` is not used."""
        obs = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64).reshape(-1, 3))
        return CompStruct(p, enei, e=self._run(obs, None, enei))

    def potential(self, p, enei):
        """phip = -nvec . e at the faces (dipole_stat.py:252-289): (n, npt, ndip)."""
        obs = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))
        nvec = np.ascontiguousarray(np.asarray(p.nvec, dtype=np.float64))
        return CompStruct(p, enei, phip=self._run(obs, nvec, enei))

    __call__ = potential

    def _green(self, p):
        key = id(p)
        if key not in self._greens:
            self._greens[key] = (p, CompGreenStatPoints(self.pt, p, **self.varargin))
        return self._greens[key][1]

    def decayrate(self, sig):
        """Total, radiative and free-space decay rates (npt, ndip)
        (dipole_stat.py:291-413): gamma = 4/3 k0^3, nb the refractive index
        at the dipole, e_ind the field of sig at the dipole's own position,
        indip = sum area pos sig the induced dipole:
        tot = 1 + Im(e_ind . dip) / (0.5 nb gamma), rad = |nb^2 indip + dip|^2,
        rad0 = nb gamma (real parts)."""
        p = sig.p
        g = self._green(p)
        npt, ndip = self.h_pos.shape[0], self.ndip
        s = np.asarray(sig.sig).reshape(g.faces.n, -1).astype(complex)
        if s.shape[1] != npt * ndip:
            raise ValueError("DipoleStat.decayrate: solution has %d columns, expected %d"
                             % (s.shape[1], npt * ndip))
        e = g.apply_sig(torch.from_numpy(np.ascontiguousarray(s)).to(g.device), mode=0,
                        diag=ndip).cpu().numpy()                        # (npt, 3, ndip)
        gamma = 4.0 / 3.0 * (2 * np.pi / sig.enei) ** 3
        area_pos = np.asarray(p.pos, dtype=np.float64) * np.asarray(p.area)[:, None]
        indip = (area_pos.T @ s).reshape(3, npt, ndip)
        nb = np.sqrt(np.asarray(self.pt.eps1(sig.enei), dtype=complex))
        dip = self.dip
        rad = np.sum(np.abs(nb[None, :, None] ** 2 * indip + dip.transpose(1, 0, 2)) ** 2,
                     axis=0)
        ed = np.einsum('qcd,qcd->qd', e, dip)
        tot = np.real(1 + np.imag(ed) / (0.5 * nb[:, None] * gamma))
        rad0 = np.real(np.broadcast_to(nb[:, None] * gamma, (npt, ndip))).copy()
        return tot, rad, rad0

    def farfield(self, spec=None, enei=None):
        """Far fields of the dipoles on the sphere at infinity
        (dipole_stat.py:415-510): dipoles screened by eps_medium / eps at the
        dipole, h = k^2/nb (dir x d) g, e = k^2/eps ((dir x d) x dir) g with
        g = exp(-i k dir . pos); every dipole radiates when any point lies in
        the medium of the sphere.  e, h (ndir, 3, npt, ndip)."""
        if enei is None:
            raise ValueError("DipoleStat.farfield: enei is required")
        medium = getattr(spec, 'medium', 1) if spec is not None else 1
        nvec = (np.asarray(spec.pinfty.nvec, dtype=np.float64) if spec is not None
                else pinfty()[0])
        dev, ptpos, _ = self._device()
        npt, ndip = self.h_pos.shape[0], self.ndip
        epsm, km = eps_k(self.pt.eps[medium - 1], enei)
        scr = epsm / np.asarray(self.pt.eps1(enei), dtype=complex)
        dip = self.dip[:, :, :] * scr[:, None, None]
        on = np.full(npt, int(np.any(self.h_med == medium)), dtype=np.int8)
        emb = np.array([[epsm, km, np.sqrt(epsm)]], dtype=complex)
        nd = nvec.shape[0]
        e = torch.zeros((1, npt * ndip, nd, 3), dtype=torch.complex128, device=dev)
        h = torch.zeros_like(e)
        # the screened moments are complex: real and imaginary parts radiate
        # separately (the far field is linear in the moment)
        out = []
        for part in (np.real(dip), np.imag(dip)):
            ee, hh = torch.zeros_like(e), torch.zeros_like(h)
            call('mnpb_dipole_farfield', _lib.stream_handle(), nd, 1, npt, ndip, ptr(ptpos),
                 ptr(_dev(on, dev)), ptr(_dev(np.ascontiguousarray(part), dev)),
                 ptr(_dev(nvec, dev)), ptr(_dev(emb, dev)), ptr(ee), ptr(hh))
            out.append((ee, hh))
        e = out[0][0] + 1j * out[1][0]
        h = out[0][1] + 1j * out[1][1]
        shape = (npt, ndip, nd, 3)
        e = e[0].cpu().numpy().reshape(shape).transpose(2, 3, 0, 1)
        h = h[0].cpu().numpy().reshape(shape).transpose(2, 3, 0, 1)
        return CompStruct(None, enei, e=e, h=h)
