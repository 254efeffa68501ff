"""Electron-energy-loss excitation (retarded) on the GPU.

``EELSRet`` mirrors mnpbem/simulation/eels_ret.py (with eels_base.py): an
electron beam of velocity ``vel`` (units of c) and width ``width`` travels
along z through each impact parameter (x, y).  ``potential`` is the BEM
excitation, ``loss`` the surface and bulk loss probabilities of a solution,
``rad`` the photon loss probability, ``field`` the beams' own fields.

The beam set-up (crossing points with the faces, the beam segments inside
particles, the faces that need face quadrature) is host geometry done once
per beam set, as ``ComPoint``'s classification.  The potentials and fields
(modified Bessel functions K0/K1 of complex argument, wire integrals) are
evaluated by ``libmnpbem_b200.so``; the loss probabilities are area-weighted
sums of those potentials with the solution, done on the host as the far-field
Poynting sums are.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .excitation import _inout_faces, pinfty, _Sides
from .greenfun import _points
from .materials import eps_k

__all__ = ["EELSRet", "EELSStat", "ene2vel", "lgl_nodes"]

# units (mnpbem/misc/units.py)
EV2NM = 1.0 / 8.0655477e-4
BOHR = 0.05292
HARTREE = 27.211
FINE = 1.0 / 137.036


def ene2vel(ene):
    """Velocity (units of c) of an electron of kinetic energy ``ene`` eV."""
    return np.sqrt(1 - 1.0 / (1 + ene / 0.51e6) ** 2)


def lgl_nodes(n=10):
    """Legendre-Gauss-Lobatto nodes (descending from 1 to -1) and weights on
    [-1, 1] with n + 1 points: the end points and the roots of P_n', weights
    2 / (n (n + 1) P_n(x)^2)."""
    from numpy.polynomial import legendre as L
    dp = L.Legendre.basis(n).deriv()
    x = np.sort(np.real(dp.roots()))[::-1]
    ddp = dp.deriv()
    for _ in range(3):                         # Newton polish of the interior roots
        x = x - dp(x) / ddp(x)
    x = np.concatenate([[1.0], x, [-1.0]])
    w = 2.0 / (n * (n + 1) * L.Legendre.basis(n)(x) ** 2)
    return np.ascontiguousarray(x), np.ascontiguousarray(w)


def _in_polygon(x, y, xv, yv, tol=1e-10):
    """Points (x, y) inside or on the polygon (xv, yv), and those on its
    boundary: even-odd ray casting for the interior; a point within ``tol``
    of an edge that the ray test puts outside, or within ``tol`` of a vertex,
    is on the boundary (the reference's inpolygon, eels_base.py:655-711)."""
    m = len(xv)
    inside = np.zeros(len(x), dtype=bool)
    near_edge = np.zeros(len(x), dtype=bool)
    near_vert = np.zeros(len(x), dtype=bool)
    for a in range(m):
        x1, y1, x2, y2 = xv[a], yv[a], xv[(a + 1) % m], yv[(a + 1) % m]
        cross = (y1 > y) != (y2 > y)
        with np.errstate(divide='ignore', invalid='ignore'):
            xc = x1 + (y - y1) * (x2 - x1) / (y2 - y1)
        inside ^= cross & (x < xc)
        dx, dy = x2 - x1, y2 - y1
        t = np.clip(((x - x1) * dx + (y - y1) * dy) / max(dx * dx + dy * dy, 1e-300), 0, 1)
        near_edge |= np.hypot(x - x1 - t * dx, y - y1 - t * dy) <= tol
        near_vert |= np.hypot(x - x1, y - y1) < tol
    on = (near_edge & ~inside) | near_vert
    return inside | on, on


class _EELSBase(object):
    """Beam set-up shared by the retarded and quasistatic beams
    (mnpbem/simulation/eels_base.py:25-830): crossing points with the faces,
    segments inside particles, faces integrated with quadrature, path
    lengths, and the GPU evaluation of the infinite-beam and wire
    potentials."""

    def __init__(self, p, impact, width, vel, cutoff=None, phiout=1e-2, pinfty=None, medium=1,
                 **options):
        if options.get('refine', None) not in (None, 1) or \
                (isinstance(options.get('eels'), dict) and options['eels'].get('refine', 1) != 1):
            raise NotImplementedError("%s: refined face quadrature ('refine') is not supported"
                                      % type(self).__name__)
        self.p = p
        self.width = float(width)
        self.vel = float(vel)
        self.phiout = phiout
        self.medium = medium
        self._pinfty = pinfty
        self._init(p, np.array(impact, dtype=np.float64, ndmin=2),
                   10 * self.width if cutoff is None else cutoff)
        self._dev = None

    # ---- beam set-up (eels_base.py:73-240) ----------------------------------
    def _init(self, p, impact, cutoff):
        pos = np.asarray(p.pos, dtype=np.float64)
        nvec = np.asarray(p.nvec, dtype=np.float64)
        src = p if getattr(p, 'faces', None) is not None else p.pc
        faces = np.asarray(src.faces, dtype=np.float64)
        verts = np.asarray(src.verts, dtype=np.float64)
        n, nimp = pos.shape[0], impact.shape[0]
        corners = [f[~np.isnan(f)].astype(int) for f in faces[:, :4]]
        # enclosure radius: largest 2D centroid-corner distance
        rad = max(np.max(np.sqrt((pos[i, 0] - verts[c, 0]) ** 2 + (pos[i, 1] - verts[c, 1]) ** 2))
                  for i, c in enumerate(corners))
        eta = 1e-6
        d2 = (np.sum(pos[:, :2] ** 2, axis=1)[:, None] + np.sum(impact ** 2, axis=1)[None, :]
              - 2 * pos[:, :2] @ impact.T)
        d2[d2 < 1e-10] = 0
        dist = np.sqrt(d2)
        rows, cols = np.where(dist <= rad)
        cross = np.zeros((n, nimp), dtype=bool)
        for i in np.unique(rows):
            c = corners[i]
            sel = cols[rows == i]
            inn, on = _in_polygon(impact[sel, 0], impact[sel, 1], verts[c, 0], verts[c, 1])
            cross[i, sel[inn]] = True
            if np.any(on):
                j = sel[on]
                impact[j, 0] = (1 - eta) * impact[j, 0] + eta * pos[i, 0]
                impact[j, 1] = (1 - eta) * impact[j, 1] + eta * pos[i, 1]
        self.impact = impact
        io = _inout_faces(p)
        i1, j1 = np.where(cross)
        zc = pos[i1, 2] + (nvec[i1, 0] * (pos[i1, 0] - impact[j1, 0]) +
                           nvec[i1, 1] * (pos[i1, 1] - impact[j1, 1])) / nvec[i1, 2]
        z, imp, mat = [], [], []
        for j in range(nimp):
            k = np.where(j1 == j)[0]
            if len(k) < 2:
                continue
            order = np.argsort(zc[k])
            zz = zc[k[order]]
            fi = i1[k[order]]
            m = io[fi].copy()
            flip = nvec[fi, 2] < 0
            m[flip, 0], m[flip, 1] = m[flip, 1].copy(), m[flip, 0].copy()
            for a in range(len(zz) - 1):
                z.append([zz[a], zz[a + 1]])
                imp.append(j)
                mat.append(m[a + 1, 0])
        z = np.array(z, dtype=np.float64).reshape(-1, 2)
        imp = np.array(imp, dtype=np.int64)
        mat = np.array(mat, dtype=np.int64)
        keep = mat != 1
        self._z, self._indimp, self._indmat = z[keep], imp[keep], mat[keep]
        self._indquad = self._near_edges(verts, corners, impact, cutoff) | cross

    @staticmethod
    def _near_edges(verts, corners, impact, cutoff):
        """Faces with an edge closer than ``cutoff`` (in the xy plane) to an
        impact parameter (eels_base.py:592-653)."""
        n, nimp = len(corners), impact.shape[0]
        out = np.zeros((n, nimp), dtype=bool)
        x, y = impact[:, 0], impact[:, 1]
        for i, c in enumerate(corners):
            dmin = np.full(nimp, np.inf)
            for a in range(len(c)):
                v0, v1 = verts[c[a]], verts[c[(a + 1) % len(c)]]
                dx, dy = v1[0] - v0[0], v1[1] - v0[1]
                lam = (dx * (x - v0[0]) + dy * (y - v0[1])) / max(dx * dx + dy * dy,
                                                                   np.finfo(float).eps)
                lam = np.clip(lam, 0, 1)
                dmin = np.minimum(dmin, np.sqrt((x - v0[0] - lam * dx) ** 2 +
                                                (y - v0[1] - lam * dy) ** 2))
            out[i] = dmin < cutoff
        return out

    def path(self, medium=None):
        """Path lengths of the beams in every medium, (nmed, nimp) or (nimp,)
        for one medium (eels_base.py:242-276)."""
        res = np.zeros((len(self.p.eps), self.impact.shape[0]))
        for (z0, z1), j, m in zip(self._z, self._indimp, self._indmat):
            res[m - 1, j] += z1 - z0
        return res if medium is None else res[medium - 1]

    def full(self, a, ind=None):
        """Columns of beam segments summed into their impact parameters
        (eels_base.py:278-313)."""
        ind = np.arange(a.shape[1]) if ind is None else np.asarray(ind)
        out = np.zeros((a.shape[0], self.impact.shape[0]), dtype=a.dtype)
        for c in ind:
            out[:, self._indimp[c]] += a[:, c]
        return out

    def _full_segs(self, a, segs):
        """Columns of the segments ``segs`` summed into their impact parameters."""
        out = np.zeros((a.shape[0], self.impact.shape[0]), dtype=a.dtype)
        for col, c in enumerate(segs):
            out[:, self._indimp[c]] += a[:, col]
        return out

    def _beam_in(self, nmed):
        """(nmed, nimp) int8: beam j passes through medium m (all beams pass
        through the embedding medium 1)."""
        b = np.zeros((nmed, self.impact.shape[0]), dtype=np.int8)
        b[0] = 1
        for j, m in zip(self._indimp, self._indmat):
            b[m - 1, j] = 1
        return b

    # ---- device tables -------------------------------------------------------
    def _device(self):
        if self._dev is None:
            p = self.p
            dev = torch.device('cuda')
            T = lambda a, dt=None: torch.from_numpy(np.ascontiguousarray(
                a if dt is None else np.asarray(a, dtype=dt))).to(dev)
            qpos, qw, qoff = _points(p, 'quad')
            io = np.ascontiguousarray(_inout_faces(p), dtype=np.int32)
            nmed = len(p.eps)
            self._dev = dict(
                dev=dev, n=int(np.asarray(p.pos).shape[0]),
                pos=T(p.pos, np.float64), nvec=T(p.nvec, np.float64),
                area=T(p.area, np.float64), face_med=T(io), h_face_med=io,
                impact=T(self.impact, np.float64), indquad=T(self._indquad, np.int8),
                qpos=T(qpos), qw=T(qw), qoff=T(qoff),
                beam_in=T(self._beam_in(nmed)), nmed=nmed)
        return self._dev

    def _faces_args(self, d):
        return (d['n'], self.impact.shape[0], ptr(d['pos']), ptr(d['nvec']), ptr(d['area']))

    def _quad_args(self, d):
        return (ptr(d['impact']), ptr(d['indquad']), ptr(d['qpos']), ptr(d['qw']),
                ptr(d['qoff']), self.width, self.vel)


    # ---- beam potentials on the GPU ------------------------------------------
    def _infty(self, q, igam, face_on):
        d = self._device()
        K, n = self.impact.shape[0], d['n']
        phi = torch.empty((K, n), dtype=torch.complex128, device=d['dev'])
        phip = torch.empty_like(phi)
        fo = torch.from_numpy(np.ascontiguousarray(face_on, dtype=np.int8)).to(d['dev'])
        call('mnpb_eels_infty', _lib.stream_handle(), n, K, ptr(d['pos']), ptr(d['nvec']),
             ptr(d['area']), ptr(fo), *self._quad_args(d), float(q), float(igam.real),
             float(igam.imag), ptr(phi), ptr(phip))
        return phi.cpu().numpy().T, phip.cpu().numpy().T            # (n, nimp)

    def _inside(self, q, k, segs, face_on, deriv=False):
        """Wire potentials (n, nseg) of the segments ``segs`` (indices into
        the segment list), 0 columns if there are none; with ``deriv`` also
        their surface derivatives (phi, phip)."""
        d = self._device()
        n = d['n']
        if len(segs) == 0:
            z = np.zeros((n, 0), dtype=complex)
            return (z, z.copy()) if deriv else z
        return self._wire(d['n'], d['pos'], d['nvec'], d['area'], face_on, self._quad_args(d),
                          q, k, segs, deriv)

    def _wire(self, n, pos, nvec, area, face_on, quad_args, q, k, segs, deriv):
        d = self._device()
        dev = d['dev']
        seg = torch.from_numpy(np.ascontiguousarray(self._z[segs])).to(dev)
        simp = torch.from_numpy(np.ascontiguousarray(self._indimp[segs], dtype=np.int32)).to(dev)
        fo = torch.from_numpy(np.ascontiguousarray(face_on, dtype=np.int8)).to(dev)
        x, w = lgl_nodes(10)
        phi = torch.empty((len(segs), n), dtype=torch.complex128, device=dev)
        phip = torch.empty_like(phi) if deriv else None
        call('mnpb_eels_wire', _lib.stream_handle(), n, self.impact.shape[0], ptr(pos), ptr(nvec),
             ptr(area), ptr(fo), *quad_args, len(segs), ptr(seg), ptr(simp), float(q),
             float(np.real(k)), float(np.imag(k)), ptr(x), ptr(w), ptr(phi),
             ptr(phip) if deriv else None)
        if deriv:
            return phi.cpu().numpy().T, phip.cpu().numpy().T
        return phi.cpu().numpy().T

    def _face_sides(self, m):
        io = self._device()['h_face_med']
        return np.where(io[:, 0] == m)[0], np.where(io[:, 1] == m)[0]

class EELSRet(_EELSBase):
    """Electron beams along z (mnpbem/simulation/eels_ret.py:24-670).

    ``EELSRet(p, impact, width, vel, cutoff=None, phiout=1e-2, pinfty=None,
    medium=1)``: impact (nimp, 2) in nm, width of the beam, velocity in units
    of c (``ene2vel``), faces closer than ``cutoff`` (default 10 width) to a
    beam in the xy plane are integrated with their quadrature points.
    """

    def _media(self, enei):
        eps = np.array([eps_k(f, enei)[0] for f in self.p.eps], dtype=complex)
        gamma = 1.0 / np.sqrt(1 - eps * self.vel ** 2)
        if np.any(np.abs(np.angle(1.0 / gamma)) > 1.2):
            raise NotImplementedError(
                "EELSRet: |arg(1/gamma)| > 1.2 in some medium (Cherenkov regime or strongly "
                "absorbing medium); the Bessel evaluation covers |arg z| <= 1.2")
        return eps, gamma

    # ---- excitation ----------------------------------------------------------
    def _med_on(self, nmed):
        """Media whose beam potential enters the excitation: the embedding
        medium, and another medium only if every beam passes through it (the
        reference adds a medium's potential only when no impact column of it
        is zero, eels_ret.py:205-211)."""
        io = np.atleast_2d(np.asarray(self.p.inout))
        on = np.zeros(nmed, dtype=np.int8)
        on[0] = 1
        bi = self._beam_in(nmed)
        for m in np.unique(io.ravel()):
            if m != 1 and np.all(bi[m - 1]):
                on[m - 1] = 1
        return on

    def potential_device(self, p, tables, eneis, stream=None):
        """Potentials of every wavelength of ``eneis`` on the GPU:
        ((B, 16, nimp, n), nimp), the layout the BEM solvers take."""
        d = self._device()
        dev, nmed, B, K = d['dev'], d['nmed'], len(eneis), self.impact.shape[0]
        eps = np.zeros((B, nmed), dtype=complex)
        igam = np.zeros((B, nmed), dtype=complex)
        for b, enei in enumerate(eneis):
            e, g = self._media(enei)
            eps[b], igam[b] = e, 1.0 / g
        q = torch.tensor([2 * np.pi / (enei * self.vel) for enei in eneis], dtype=torch.float64,
                         device=dev)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.float64)).to(dev)
        pots = torch.empty((B, 16, K, d['n']), dtype=torch.complex128, device=dev)
        med_on = torch.from_numpy(self._med_on(nmed)).to(dev)
        call('mnpb_eels_potential', _lib.stream_handle(stream), d['n'], B, K, ptr(d['pos']),
             ptr(d['nvec']), ptr(d['area']), ptr(d['face_med']), nmed, ptr(med_on),
             ptr(d['beam_in']), *self._quad_args(d), ptr(q), ptr(T(eps)),
             ptr(T(igam)), ptr(pots))
        return pots, K

    def potential(self, p, enei):
        """phi1, phi1p, a1, a1p, phi2, phi2p, a2, a2p at the faces, (n, nimp)
        and (n, 3, nimp) host arrays (eels_ret.py:149-222)."""
        pots, K = self.potential_device(p, None, [enei])
        x = pots[0].cpu().numpy()
        out = {}
        comp = 0
        for name, w in (('phi1', 1), ('phi1p', 1), ('a1', 3), ('a1p', 3), ('phi2', 1),
                        ('phi2p', 1), ('a2', 3), ('a2p', 3)):
            v = x[comp:comp + w]
            out[name] = v[0].T.copy() if w == 1 else v.transpose(2, 0, 1).copy()
            comp += w
        return CompStruct(p, enei, **out)

    __call__ = potential

    # ---- loss probabilities ----------------------------------------------------
    def loss(self, sig):
        """Surface and bulk loss probabilities per impact parameter, in 1/eV
        (eels_ret.py:296-423): psurf = -Im sum_faces area phi* (sig - vel h_z)
        with phi the beam potential (infinite beam in the embedding medium
        minus its parts inside particles, plus the inside segments)."""
        p = self.p
        enei = sig.enei
        eps, gamma = self._media(enei)
        k = 2 * np.pi / enei * np.sqrt(eps)
        q = 2 * np.pi / (enei * self.vel)
        n, nimp = self._device()['n'], self.impact.shape[0]
        sig1 = np.asarray(sig.sig1).reshape(n, -1)
        sig2 = np.asarray(sig.sig2).reshape(n, -1)
        h1 = np.asarray(sig.h1).reshape(n, 3, -1)
        h2 = np.asarray(sig.h2).reshape(n, 3, -1)
        fun = (sig1 - self.vel * h1[:, 2], sig2 - self.vel * h2[:, 2])
        area = np.asarray(p.area, dtype=np.float64)
        allf = np.ones(n, dtype=np.int8)
        phi_inf, _ = self._infty(q, 1.0 / gamma[0], allf)
        phi_in = self._inside(-q, k[0], np.arange(len(self._z)), allf)
        phi = self.vel * (np.conj(phi_inf) - self.full(phi_in))
        psurf = np.zeros(nimp)
        for s, ind in enumerate(self._face_sides(1)):
            if len(ind):
                psurf -= np.imag(area[ind] @ (phi[ind] * fun[s][ind]))
        io = np.atleast_2d(np.asarray(p.inout))
        io_f = self._device()['h_face_med']
        for m in np.unique(io.ravel()):
            if m == 1:
                continue
            face_on = np.any(io_f == m, axis=1).astype(np.int8)
            segs = np.where(self._indmat == m)[0]
            phi_m = self.vel * self._full_segs(self._inside(-q, k[m - 1], segs, face_on), segs)
            for s, ind in enumerate(self._face_sides(m)):
                if len(ind):
                    psurf -= np.imag(area[ind] @ (phi_m[ind] * fun[s][ind]))
        psurf = FINE ** 2 / (BOHR * HARTREE * np.pi * self.vel) * psurf
        return psurf, self.bulkloss(enei)

    def bulkloss(self, enei):
        """Bulk loss probability per impact parameter in 1/eV (Garcia de
        Abajo, RMP 82, 209 (2010), Eq. 18; eels_ret.py:425-466)."""
        ene = EV2NM / enei
        mass = 0.51e6
        eps = np.array([eps_k(f, enei)[0] for f in self.p.eps], dtype=complex)
        q = 2 * np.pi / (enei * self.vel)
        qc = q * np.sqrt((mass / ene) ** 2 * self.vel ** 2 * self.phiout ** 2 + 1)
        k = 2 * np.pi / enei * np.sqrt(eps)
        ratio = (qc ** 2 - k ** 2) / (q ** 2 - k ** 2)
        ratio = np.where(ratio.imag == 0, ratio.real + 0.0j, ratio)   # log branch of -x: +i pi
        return (FINE ** 2 / (BOHR * HARTREE * np.pi * self.vel ** 2) *
                np.imag((self.vel ** 2 - 1.0 / eps) * np.log(ratio)) @ self.path())

    def _sphere(self):
        if self._pinfty is None:
            return pinfty()
        q = self._pinfty
        return (np.ascontiguousarray(np.asarray(q.nvec, dtype=np.float64)),
                np.ascontiguousarray(np.asarray(q.area, dtype=np.float64)))

    def rad(self, sig):
        """Photon loss probability FINE^2 / (2 pi^2 HARTREE BOHR k) sca with
        sca the radiated power through the sphere at infinity
        (eels_ret.py:468-504, spectrum_ret.py:395-459)."""
        from .excitation import PlaneWaveRet
        p = sig.p
        d = self._device()
        dev = d['dev']
        x, K = PlaneWaveRet._sol_device(sig, dev)
        nvec, area = self._sphere()
        _, km = eps_k(p.eps[self.medium - 1], sig.enei)
        sides = _Sides(p, self.medium, dev)
        d_dirs = torch.from_numpy(nvec).to(dev)
        nd = nvec.shape[0]
        e = torch.empty((1, K, nd, 3), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        kt = torch.tensor([km.real, km.imag], dtype=torch.float64, device=dev)
        k0 = torch.tensor([2 * np.pi / sig.enei], dtype=torch.float64, device=dev)
        call('mnpb_farfield', _lib.stream_handle(), d['n'], 1, K, nd, ptr(d['pos']),
             ptr(d['area']), ptr(sides.side_in), ptr(sides.side_out), ptr(d_dirs), ptr(kt),
             ptr(k0), ptr(x), ptr(e), ptr(h))
        e, h = e[0].cpu().numpy(), h[0].cpu().numpy()
        dsca = 0.5 * np.real(np.einsum('dc,kdc->kd', nvec, np.cross(e, np.conj(h))))
        sca = dsca @ area
        fac = FINE ** 2 / (2 * np.pi ** 2 * HARTREE * BOHR * km)
        prad = fac * sca
        return (prad[0] if K == 1 else prad), CompStruct(None, sig.enei, dprad=fac * dsca.T)

    # ---- fields ---------------------------------------------------------------
    def field(self, p, enei, inout=1):
        """The beams' own fields at the faces of ``p`` (side ``inout``):
        e, h (n, 3, nimp) (eels_ret.py:506-637)."""
        d = self._device()
        dev = d['dev']
        eps, gamma = self._media(enei)
        k = 2 * np.pi / enei * np.sqrt(eps)
        q = k / (self.vel * np.sqrt(eps))
        mtab = np.stack([eps, q, 1.0 / gamma], axis=1)              # (nmed, 3) complex
        obs = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))
        med = np.ascontiguousarray(_inout_faces(p)[:, inout - 1], dtype=np.int32)
        nimp = self.impact.shape[0]
        e = torch.empty((obs.shape[0], 3, nimp), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        call('mnpb_eels_field', _lib.stream_handle(), obs.shape[0], nimp, ptr(T(obs)),
             ptr(T(med)), d['nmed'], ptr(d['beam_in']), ptr(d['impact']), self.width, self.vel,
             ptr(T(mtab.view(np.float64))), ptr(e), ptr(h))
        return CompStruct(p, enei, e=e.cpu().numpy(), h=h.cpu().numpy())


class EELSStat(_EELSBase):
    """Electron beams along z, quasistatic (mnpbem/simulation/eels_stat.py:23-409).

    ``EELSStat(p, impact, width, vel, cutoff=None, phiout=1e-2)``: the beam
    set-up of ``EELSRet``; ``potential`` is the excitation of ``BEMStat``
    (phi, phip), ``loss`` the surface and bulk loss probabilities of its
    solution, ``field`` the beams' electric field.  The beam potentials are
    the retarded ones at gamma = 1 (infinite beam) and k = 0 (wire segments),
    evaluated by the same kernels.
    """

    name = 'eels'
    needs = {'sim': 'stat'}

    def _eps(self, p, enei):
        return np.array([eps_k(f, enei)[0] for f in p.eps], dtype=complex)

    def potential(self, p, enei):
        """phi, phip (n, nimp) (eels_stat.py:107-161): the infinite beam
        over eps of the embedding medium plus, for each segment inside
        medium m, its wire potential times 1/eps_m - 1/eps_1."""
        eps = self._eps(self.p, enei)
        q = 2 * np.pi / (enei * self.vel)
        n = self._device()['n']
        allf = np.ones(n, dtype=np.int8)
        phi, phip = self._infty(q, 1.0, allf)
        phi, phip = phi / eps[0], phip / eps[0]
        if len(self._z):
            pin, pinp = self._inside(q, 0.0, np.arange(len(self._z)), allf, deriv=True)
            f = (1.0 / eps - 1.0 / eps[0])[self._indmat - 1][None, :]
            phi = phi + self.full(pin * f)
            phip = phip + self.full(pinp * f)
        return CompStruct(p, enei, phi=phi, phip=phip)

    __call__ = potential

    def loss(self, sig):
        """Surface and bulk loss probabilities per impact parameter, in 1/eV
        (eels_stat.py:163-193): psurf = -FINE^2/(BOHR HARTREE pi)
        Im sum_faces area conj(phi) sig, phi the infinite beam (gamma = 1)."""
        q = 2 * np.pi / (sig.enei * self.vel)
        n = self._device()['n']
        phi, _ = self._infty(q, 1.0, np.ones(n, dtype=np.int8))
        s = np.asarray(sig.sig).reshape(n, -1)
        area = np.asarray(self.p.area, dtype=np.float64)
        psurf = -FINE ** 2 / (BOHR * HARTREE * np.pi) * np.imag(area @ (np.conj(phi) * s))
        return psurf, self.bulkloss(sig.enei)

    def bulkloss(self, enei):
        """Bulk loss probability per impact parameter in 1/eV (Garcia de
        Abajo, RMP 82, 209 (2010), Eq. 19; eels_stat.py:195-228)."""
        ene = EV2NM / enei
        mass = 0.51e6
        eps = self._eps(self.p, enei)
        fac = 2 * FINE ** 2 / (BOHR * HARTREE * np.pi * self.vel ** 2)
        return fac * (np.imag(-1.0 / eps) @ self.path()) * \
            np.log(np.sqrt((mass / ene) ** 2 * self.vel ** 2 * self.phiout ** 2 + 1))

    def field(self, p, enei, inout=1):
        """Electric field e (n, 3, nimp) of the beams at the positions of
        ``p`` (eels_stat.py:230-355): the infinite beam in the embedding
        medium (q = k_1 / (vel sqrt(eps_1)), gamma = 1), plus the segments
        inside media (gradients of their k = 0 wire potentials times
        1/eps_m - 1/eps_1), each segment taken with its own impact parameter
        and summed into it.  ``inout`` is not used."""
        d = self._device()
        dev = d['dev']
        eps = self._eps(p, enei)
        k1 = 2 * np.pi / enei * np.sqrt(eps[0])
        q = k1 / (self.vel * np.sqrt(eps[0]))
        obs = np.ascontiguousarray(np.asarray(p.pos, dtype=np.float64))
        nobs, nimp = obs.shape[0], self.impact.shape[0]
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        mtab = np.array([[eps[0], q, 1.0]], dtype=complex)
        e = torch.empty((nobs, 3, nimp), dtype=torch.complex128, device=dev)
        h = torch.empty_like(e)
        call('mnpb_eels_field', _lib.stream_handle(), nobs, nimp, ptr(T(obs)),
             ptr(T(np.ones(nobs, dtype=np.int32))), 1, ptr(T(np.ones((1, nimp), dtype=np.int8))),
             ptr(d['impact']), self.width, self.vel, ptr(T(mtab.view(np.float64))), ptr(e), ptr(h))
        e = e.cpu().numpy()
        if len(self._z):
            # the derivative along x^, y^, z^ of the wire potentials at every
            # position: the three copies of the positions carry those normals
            pos3 = np.concatenate([obs, obs, obs])
            nv3 = np.repeat(np.eye(3), nobs, axis=0)
            m = 3 * nobs
            quad = (d['impact'], T(np.zeros((m, nimp), dtype=np.int8)), T(np.zeros(3)),
                    T(np.zeros(1)), T(np.zeros(m + 1, dtype=np.int64)), self.width, self.vel)
            quad = tuple(ptr(a) if torch.is_tensor(a) else a for a in quad)
            segs = np.arange(len(self._z))
            _, dphi = self._wire(m, T(pos3), T(nv3), T(np.ones(m)), np.ones(m, dtype=np.int8),
                                 quad, np.real(q), 0.0, segs, True)
            f = (1.0 / eps - 1.0 / eps[0])[self._indmat - 1][None, :]
            # e_c = (1/eps_m - 1/eps_1) (Ir x_c / rr or Iz) / vel, which is
            # -(1/eps_m - 1/eps_1) phip with the normal c^
            ein = self.full(-dphi * f)                               # (3 nobs, nimp)
            e = e + ein.reshape(3, nobs, nimp).transpose(1, 0, 2)
        return CompStruct(p, enei, e=e)
