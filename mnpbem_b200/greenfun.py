"""Green functions of a particle surface on the GPU.

``SurfaceTables`` holds everything the assembly kernels need for one
particle surface, resident in HBM: face data (pos, nvec, tvec1/2, area),
the near/self pair list (CSR, from the host classifier) and the refined
Taylor coefficients of the retarded Green function (computed on the GPU in
FP64 from the face and polar quadrature points), closure-corrected.

``CompGreenRet`` / ``CompGreenStat`` mirror the reference classes
(mnpbem/greenfun/compgreen_ret.py:14, compgreen_stat.py:12): construction
builds the tables, ``eval(i, j, key, enei)`` returns the (n, n) matrix of a
region pair on the host, ``CompGreenStat.F`` the refined quasistatic F.

Particles may be this package's ``ComParticle`` or any object with the same
attributes (the reference's ``ComParticle`` included).
"""

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .materials import eps_k

__all__ = ["SurfaceTables", "CompGreenRet", "CompGreenStat", "region_tables"]

TWO_PI = 2.0 * np.pi


def _nfaces(p):
    for a in ('nfaces', 'n'):
        v = getattr(p, a, None)
        if v is not None and not callable(v):
            return int(v)
    return int(np.asarray(p.pos).shape[0])


def _face(p, name):
    v = getattr(p, name, None)
    if v is None and hasattr(p, 'pc'):
        v = getattr(p.pc, name)
    return np.ascontiguousarray(np.asarray(v, dtype=np.float64))


def _points(p, which):
    """Quadrature points of all faces sorted by face: pos (P,3), w (P,), off (n+1)."""
    n = _nfaces(p)
    ind = np.arange(n)
    if which == 'quad':
        fn = getattr(p, 'quad_integration', None)
        out = fn(ind) if fn is not None else p.quad(ind)
        pos, w = out[0], out[1]
        if hasattr(w, 'tocoo'):
            coo = w.tocoo()
            row = np.empty(coo.shape[1], dtype=np.int64)
            ww = np.empty(coo.shape[1])
            row[coo.col] = coo.row
            ww[coo.col] = coo.data
            w = ww
        else:
            row = np.asarray(out[2])
    else:
        pos, w, row = p.quadpol(ind)
    row = np.asarray(row, dtype=np.int64)
    order = np.argsort(row, kind='stable')
    counts = np.bincount(row, minlength=n)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    return (np.ascontiguousarray(np.asarray(pos, dtype=np.float64)[order]),
            np.ascontiguousarray(np.asarray(w, dtype=np.float64)[order]), off)


def refinematrix_csr(pos1, pos2, rad1, rad2, abs_cutoff=0.0, rel_cutoff=3.0):
    """Near/self pair list as CSR (row_ptr, cols, kinds) via the C classifier.
    ``rad1=None``: sources without a boundary radius (points), distances in
    units of the column face's radius."""
    L = _lib.lib()
    pos1 = np.ascontiguousarray(pos1, dtype=np.float64)
    pos2 = np.ascontiguousarray(pos2, dtype=np.float64)
    rad1 = None if rad1 is None else np.ascontiguousarray(rad1, dtype=np.float64)
    rad2 = np.ascontiguousarray(rad2, dtype=np.float64)
    n1, n2 = pos1.shape[0], pos2.shape[0]
    row_ptr = np.zeros(n1 + 1, dtype=np.int64)
    nnz = C.c_int64(0)
    rc = L.mnpb_refinematrix(n1, n2, ptr(pos1), ptr(pos2), ptr(rad1), ptr(rad2), abs_cutoff,
                             rel_cutoff, 0, C.byref(nnz), ptr(row_ptr), None, None)
    if rc not in (0, 6):
        raise _lib.MNPBError('mnpb_refinematrix', rc, L.mnpb_last_error().decode())
    cap = int(nnz.value)
    cols = np.zeros(max(cap, 1), dtype=np.int32)
    kinds = np.zeros(max(cap, 1), dtype=np.int8)
    call('mnpb_refinematrix', n1, n2, ptr(pos1), ptr(pos2), ptr(rad1), ptr(rad2), abs_cutoff,
         rel_cutoff, cap, C.byref(nnz), ptr(row_ptr), ptr(cols), ptr(kinds))
    return row_ptr, cols[:cap], kinds[:cap]


def closed_ranges(p):
    """Per face: [lo, hi) face range of its closed surface and the normal sign.

    Each particle is its own closed surface unless ``p.closed`` says
    otherwise (the reference's default, compgreen_ret.py:224-229).  Only
    closed surfaces made of consecutive particles of ``p`` are supported.
    """
    n = _nfaces(p)
    parts = list(getattr(p, 'p', [p]))
    off = np.cumsum([0] + [_nfaces(q) for q in parts]).astype(np.int64)
    closed = list(getattr(p, 'closed', [None] * len(parts)) or [None] * len(parts))
    if all(c is None for c in closed):
        closed = [[k + 1] for k in range(len(parts))]
    lo = np.zeros(n, dtype=np.int64)
    hi = np.zeros(n, dtype=np.int64)
    sign = np.zeros(n)
    for i, c in enumerate(closed):
        if c is None:
            continue
        c = [int(v) for v in np.atleast_1d(c)]
        if any(v <= 0 for v in c) or sorted(c) != list(range(min(c), max(c) + 1)):
            raise NotImplementedError("closed surfaces must be runs of this object's particles")
        a, b = off[min(c) - 1], off[max(c)]
        lo[off[i]:off[i + 1]] = a
        hi[off[i]:off[i + 1]] = b
        sign[off[i]:off[i + 1]] = 1.0
    return lo, hi, sign, off


class SurfaceTables(object):
    """Device-resident face data and refined coefficients for one surface."""

    def __init__(self, p, rel_cutoff=3.0, abs_cutoff=0.0, device=None):
        self.device = torch.device(device) if device is not None else torch.device('cuda')
        dev = self.device
        self.p = p
        n = _nfaces(p)
        self.n = n
        pos, nvec = _face(p, 'pos'), _face(p, 'nvec')
        tv1, tv2 = _face(p, 'tvec1'), _face(p, 'tvec2')
        area = np.ascontiguousarray(np.asarray(p.area, dtype=np.float64))
        rad = np.ascontiguousarray(np.asarray(p.bradius(), dtype=np.float64))
        self.h_pos, self.h_nvec, self.h_area = pos, nvec, area
        rptr, cols, kinds = refinematrix_csr(pos, pos, rad, rad, abs_cutoff, rel_cutoff)
        rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rptr)).astype(np.int32)
        if len(cols) > 1 and not np.all((np.diff(cols) > 0) | (np.diff(rows) != 0)):
            raise RuntimeError("refinematrix: columns not ascending within a row")
        self.h_rptr, self.h_rows, self.h_cols, self.h_kinds = rptr, rows, cols, kinds
        self.nref = len(cols)
        qpos, qw, qoff = _points(p, 'quad')
        ppos, pw, poff = _points(p, 'quadpol')

        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self.pos, self.nvec, self.tvec1, self.tvec2, self.area = map(T, (pos, nvec, tv1, tv2, area))
        self.rows, self.cols, self.kinds = T(rows), T(cols), T(kinds)
        self.rptr = T(rptr)
        d_qpos, d_qw, d_qoff, d_ppos, d_pw, d_poff = map(T, (qpos, qw, qoff, ppos, pw, poff))
        nref = self.nref
        f64 = dict(dtype=torch.float64, device=dev)
        self.g = torch.zeros((max(nref, 1), 6), **f64)
        self.f = torch.zeros((max(nref, 1), 3, 6), **f64)
        self.gstat = torch.zeros(max(nref, 1), **f64)
        self.fstat = torch.zeros(max(nref, 1), **f64)
        self.fn = torch.zeros((max(nref, 1), 6), **f64)
        sh = _lib.stream_handle()
        call('mnpb_refine_coefficients', sh, n, ptr(self.pos), ptr(self.nvec), ptr(self.tvec1),
             ptr(self.tvec2), nref, ptr(self.rows), ptr(self.cols), ptr(self.kinds), ptr(d_qpos),
             ptr(d_qw), ptr(d_qoff), ptr(d_ppos), ptr(d_pw), ptr(d_poff), ptr(self.g),
             ptr(self.f), ptr(self.gstat), ptr(self.fstat))
        # closed-surface correction: sums of the refined static F per column
        lo, hi, sign, self.part_off = closed_ranges(p)
        order = np.lexsort((rows, cols))
        cptr = np.concatenate([[0], np.cumsum(np.bincount(cols, minlength=n))]).astype(np.int64)
        d_order = torch.from_numpy(order).to(dev)
        crows = self.rows[d_order].contiguous()
        cfstat = self.fstat[d_order].contiguous()
        fsum = torch.zeros(n, **f64)
        call('mnpb_closure_sums', sh, n, ptr(self.pos), ptr(self.nvec), ptr(self.area),
             ptr(T(lo)), ptr(T(hi)), ptr(T(cptr)), ptr(crows), ptr(cfstat), ptr(fsum))
        self.fsum = fsum
        self.cdir = T(np.where(hi > lo, sign, 0.0))
        self.f_raw = self.f.clone()
        call('mnpb_refine_finalize', sh, n, nref, ptr(self.rows), ptr(self.cols), ptr(self.nvec),
             ptr(self.cdir), ptr(self.fsum), ptr(self.f), ptr(self.fn))
        self.parts = list(getattr(p, 'p', [p]))
        self.nparts = len(self.parts)
        self.inout = np.atleast_2d(np.asarray(getattr(p, 'inout', [[2, 1]]), dtype=int))
        self.eps_funcs = list(p.eps)

    # ---- per-wavelength tables --------------------------------------------
    def k_tables(self, eneis, sides=('G1', 'G2')):
        """Wavenumber/sign tables per particle block for a batch of wavelengths.

        Side 1 is G1 = G11 - G21 (region pairs (in,in) and (out,in)), side 2
        is G2 = G22 - G12 (compgreen_ret.py:435-505 connectivity, bem_ret.py:
        407-423).  Returns host arrays kblk (B,2,np,np,2), sblk (B,2,np,np).
        """
        npart = self.nparts
        io = self.inout
        B = len(eneis)
        kblk = np.zeros((B, 2, npart, npart, 2))
        sblk = np.zeros((B, 2, npart, npart))
        for b, enei in enumerate(eneis):
            ks = [eps_k(e, enei)[1] for e in self.eps_funcs]
            for p1 in range(npart):
                for p2 in range(npart):
                    # side 1: (in,in) direct, (out,in) subtracted
                    if io[p1, 0] == io[p2, 0]:
                        k, s = ks[io[p1, 0] - 1], 1.0
                    elif io[p1, 1] == io[p2, 0]:
                        k, s = ks[io[p1, 1] - 1], -1.0
                    else:
                        k, s = 0j, 0.0
                    kblk[b, 0, p1, p2] = (k.real, k.imag)
                    sblk[b, 0, p1, p2] = s
                    # side 2: (out,out) direct, (in,out) subtracted
                    if io[p1, 1] == io[p2, 1]:
                        k, s = ks[io[p1, 1] - 1], 1.0
                    elif io[p1, 0] == io[p2, 1]:
                        k, s = ks[io[p1, 0] - 1], -1.0
                    else:
                        k, s = 0j, 0.0
                    kblk[b, 1, p1, p2] = (k.real, k.imag)
                    sblk[b, 1, p1, p2] = s
        return kblk, sblk

    def assemble(self, kblk, sblk, out, mode=0, stream=None):
        """Launch the assembly into ``out`` = (G1, H1, G2, H2) device buffers."""
        B = kblk.shape[0]
        n = self.n
        d_k = torch.from_numpy(np.ascontiguousarray(kblk)).to(self.device)
        d_s = torch.from_numpy(np.ascontiguousarray(sblk)).to(self.device)
        poff = np.ascontiguousarray(self.part_off, dtype=np.int64)
        G1, H1, G2, H2 = out
        if mode == 0:
            ld, stride, plane = n, n * n, 0
        else:
            ld, stride, plane = n, 2 * n * n, n * n
        call('mnpb_assemble_ret', _lib.stream_handle(stream), n, B, ptr(self.pos),
             ptr(self.nvec), ptr(self.area), self.nparts, ptr(poff), ptr(d_k), ptr(d_s),
             self.nref, ptr(self.rows), ptr(self.cols), ptr(self.g), ptr(self.fn), mode,
             ptr(G1), ptr(H1), ptr(G2), ptr(H2), ld, stride, plane)
        return d_k, d_s


    # ---- entries and products of one region pair ---------------------------
    def _eval_args(self, kb, sb):
        dev = self.device
        d_k = torch.from_numpy(np.ascontiguousarray(kb, dtype=np.float64)).to(dev)
        d_s = torch.from_numpy(np.ascontiguousarray(sb, dtype=np.float64)).to(dev)
        poff = np.ascontiguousarray(self.part_off, dtype=np.int64)
        return (self.n, ptr(self.pos), ptr(self.nvec), ptr(self.area), self.nparts, ptr(poff),
                ptr(d_k), ptr(d_s), ptr(self.rptr), ptr(self.cols), ptr(self.g), ptr(self.fn),
                ptr(self.f)), (d_k, d_s)

    def green_eval(self, kb, sb, key, col_start=0, ncol=None, ind=None, stream=None):
        """Device entries of the region pair given by the block tables kb
        (np, np, 2), sb (np, np): columns [col_start, col_start + ncol) as
        (n, ncol) / (n, 3, ncol) complex, or the entries at row-major linear
        indices ``ind`` as (len(ind),) / (len(ind), 3)."""
        args, keep = self._eval_args(kb, sb)
        vec = key >= KEYS['Gp']
        c128 = dict(dtype=torch.complex128, device=self.device)
        if ind is not None:
            d_ind = torch.from_numpy(np.ascontiguousarray(ind, dtype=np.int64)).to(self.device)
            nind = d_ind.numel()
            out = torch.zeros((nind, 3) if vec else (nind,), **c128)
            call('mnpb_green_eval', _lib.stream_handle(stream), *args, key, 0, 0, ptr(d_ind),
                 nind, ptr(out))
            return out
        ncol = self.n - col_start if ncol is None else ncol
        out = torch.zeros((self.n, 3, ncol) if vec else (self.n, ncol), **c128)
        call('mnpb_green_eval', _lib.stream_handle(stream), *args, key, col_start, ncol, None,
             0, ptr(out))
        return out

    def green_apply(self, kb, sb, key, x, stream=None):
        """Product of the region-pair matrix with device vectors, entries on
        the fly: scalar key, x (n, m) -> (n, m); vector key, x (n, m) ->
        (n, 3, m); vector key, x (n, 3, m) -> cross products (n, 3, m)."""
        args, keep = self._eval_args(kb, sb)
        vec = key >= KEYS['Gp']
        x = x.to(torch.complex128).contiguous()
        n = self.n
        if not vec:
            outs = []
            for c0 in range(0, x.shape[1], 12):
                xx = x[:, c0:c0 + 12].contiguous()
                y = torch.empty_like(xx)
                call('mnpb_green_apply', _lib.stream_handle(stream), *args, key, 0,
                     xx.shape[1], ptr(xx), ptr(y))
                outs.append(y)
            return torch.cat(outs, dim=1)
        mode = 2 if x.dim() == 3 else 1
        m = x.shape[-1]
        outs = []
        for c0 in range(0, m, 4):
            xx = x[..., c0:c0 + 4].contiguous()
            y = torch.empty((n, 3, xx.shape[-1]), dtype=torch.complex128, device=self.device)
            call('mnpb_green_apply', _lib.stream_handle(stream), *args, key, mode,
                 xx.shape[-1], ptr(xx), ptr(y))
            outs.append(y)
        return torch.cat(outs, dim=2)


KEYS = {'G': 0, 'F': 1, 'H1': 2, 'H2': 3, 'Gp': 4, 'H1p': 5, 'H2p': 6}


def region_tables(tables, i, j, enei):
    """k/sign tables selecting region pair (i, j) on side 1 (compgreen_ret.py:739-858)."""
    npart = tables.nparts
    io = tables.inout
    ks = [eps_k(e, enei)[1] for e in tables.eps_funcs]
    kblk = np.zeros((1, 2, npart, npart, 2))
    sblk = np.zeros((1, 2, npart, npart))
    for p1 in range(npart):
        for p2 in range(npart):
            if io[p1, i] == io[p2, j]:
                k = ks[io[p1, i] - 1]
                for s in (0, 1):
                    kblk[0, s, p1, p2] = (k.real, k.imag)
                    sblk[0, s, p1, p2] = 1.0
    return kblk, sblk


class CompGreenRet(object):
    """Retarded Green function of a particle with itself (refined, closed).

    ``eval(i, j, key, enei[, ind])`` -> the (n, n) complex host matrix of
    region pair (i, j) (0 inside, 1 outside) for key G, F, H1, H2, or (n, 3, n)
    for the Cartesian derivatives Gp, H1p, H2p; 0 if no block connects
    (compgreen_ret.py:507-553, 739-858).  ``eval_block`` returns a column
    range, ``potential`` / ``field`` the potentials and fields at the faces
    of a solution (compgreen_ret.py:912-1036), computed with on-the-fly
    entries (no n x n matrix is stored for them).
    """

    def __new__(cls, p1, p2=None, **options):
        # a point set as p1 (the reference's CompGreenRet(ComPoint, particle))
        from .points import is_point_set, CompGreenRetPoints
        if is_point_set(p1) and p2 is not None:
            return CompGreenRetPoints(p1, p2, **options)
        return super(CompGreenRet, cls).__new__(cls)

    def __init__(self, p1, p2=None, **options):
        if p2 is not None and p2 is not p1:
            raise NotImplementedError("CompGreenRet: only p1 is p2 (the BEM matrices) is supported")
        self.p1 = self.p2 = p1
        self.deriv = options.get('deriv', 'cart')
        if self.deriv != 'cart':
            raise NotImplementedError("CompGreenRet: deriv='cart' (the default) only")
        if options.get('order', 5) != 5 or not options.get('refine', True):
            raise NotImplementedError("CompGreenRet: refinement order 5 only")
        self.tables = SurfaceTables(p1, rel_cutoff=options.get('RelCutoff', 3),
                                    abs_cutoff=options.get('AbsCutoff', 0))
        io = self.tables.inout
        self.con = [[np.where(io[:, a][:, None] == io[:, b][None, :], io[:, a][:, None], 0)
                     for b in range(2)] for a in range(2)]

    def _blocks(self, i, j, enei):
        kblk, sblk = region_tables(self.tables, i, j, enei)
        return kblk[0, 0], sblk[0, 0]

    @staticmethod
    def _key(key):
        if key not in KEYS:
            raise ValueError("Unknown key: {}".format(key))
        return KEYS[key]

    def eval(self, i, j, key, enei, ind=None):
        """Region-pair matrix (compgreen_ret.py:507-553).  With ``ind``
        (row-major linear indices i * n + j, as the reference's _eval2) the
        selected entries, (len(ind),) or (len(ind), 3); entries of blocks
        that are not connected are 0."""
        kk = self._key(key)
        kb, sb = self._blocks(i, j, enei)
        if ind is not None:
            ind = np.asarray(ind, dtype=np.int64).ravel()
            n = self.tables.n
            if ind.size and (ind.min() < 0 or ind.max() >= n * n):
                raise IndexError("CompGreenRet.eval: index out of range")
            out = self.tables.green_eval(kb, sb, kk, ind=ind)
            torch.cuda.synchronize()
            return out.cpu().numpy()
        if not np.any(self.con[i][j]):
            return 0
        out = self.tables.green_eval(kb, sb, kk).cpu().numpy()
        if not np.any(out):
            return 0
        return out

    def eval_block(self, i, j, key, enei, col_start, col_stop):
        """Columns [col_start, col_stop) of ``eval(i, j, key, enei)``
        (compgreen_ret.py:555-617): (n, ncol), or (n, 3, ncol) for Gp/H1p/H2p;
        zeros if no block connects."""
        kk = self._key(key)
        col_start, col_stop = int(col_start), int(col_stop)
        if not (0 <= col_start <= col_stop <= self.tables.n):
            raise ValueError("eval_block col range ({}, {}) out of bounds for p2.n={}"
                             .format(col_start, col_stop, self.tables.n))
        kb, sb = self._blocks(i, j, enei)
        out = self.tables.green_eval(kb, sb, kk, col_start=col_start,
                                     ncol=col_stop - col_start)
        return out.cpu().numpy()

    # ---- potentials and fields at the faces --------------------------------
    def _apply(self, region, col, key, x):
        """M(region, col; key) applied to device x, or None if no block of
        the region pair is connected (the reference's matmul with 0)."""
        if not np.any(self.con[region][col]):
            return None
        kb, sb = self._blocks(region, col, self._enei)
        return self.tables.green_apply(kb, sb, KEYS[key], x)

    @staticmethod
    def _as_cols(v, n, vec):
        """(n[, 3][, K]) host array -> device (n, K) or (n, 3, K), and K."""
        a = np.asarray(v, dtype=complex)
        if vec:
            a = a.reshape(n, 3, -1)
        else:
            a = a.reshape(n, -1)
        return torch.from_numpy(np.ascontiguousarray(a)).cuda(), a.shape[-1]

    def potential(self, sig, inout=1):
        """Potentials and surface derivatives inside (inout=1) or outside
        (inout=2) from sigma/h (compgreen_ret.py:980-1036): phi = G1 sig1 +
        G2 sig2, phip with H1/H2, a and ap with the currents."""
        n = self.tables.n
        self._enei = sig.enei
        r = min(inout - 1, 1)
        hk = 'H1' if inout == 1 else 'H2'
        s1, K = self._as_cols(sig.sig1, n, False)
        s2, _ = self._as_cols(sig.sig2, n, False)
        h1, _ = self._as_cols(sig.h1, n, True)
        h2, _ = self._as_cols(sig.h2, n, True)
        sh = s1.ndim

        def comb(key, x1, x2, vec):
            out = None
            for col, x in ((0, x1), (1, x2)):
                xx = x.reshape(n, -1) if vec else x
                y = self._apply(r, col, key, xx)
                if y is not None:
                    out = y if out is None else out + y
            if out is None:
                return 0
            out = out.cpu().numpy()
            out = out.reshape(n, 3, -1) if vec else out
            return out[..., 0] if K == 1 else out

        phi, phip = comb('G', s1, s2, False), comb(hk, s1, s2, False)
        a, ap = comb('G', h1, h2, True), comb(hk, h1, h2, True)
        del sh
        if inout == 1:
            return CompStruct(self.p1, sig.enei, phi1=phi, phi1p=phip, a1=a, a1p=ap)
        return CompStruct(self.p1, sig.enei, phi2=phi, phi2p=phip, a2=a, a2p=ap)

    def field(self, sig, inout=1):
        """Electric and magnetic fields inside (inout=1) or outside (inout=2)
        (compgreen_ret.py:912-978): e = i k (G1 h1 + G2 h2) - Hp1 sig1 -
        Hp2 sig2, h = Hp1 x h1 + Hp2 x h2 with Hp = H1p (inside) or H2p
        (outside) of both column regions, k = 2 pi / enei."""
        n = self.tables.n
        self._enei = sig.enei
        k = 2 * np.pi / sig.enei
        r = min(inout - 1, 1)
        pk = 'H1p' if inout == 1 else 'H2p'
        s1, K = self._as_cols(sig.sig1, n, False)
        s2, _ = self._as_cols(sig.sig2, n, False)
        h1, _ = self._as_cols(sig.h1, n, True)
        h2, _ = self._as_cols(sig.h2, n, True)
        e = torch.zeros((n, 3, K), dtype=torch.complex128, device='cuda')
        hh = torch.zeros_like(e)
        for col, s, h in ((0, s1, h1), (1, s2, h2)):
            g = self._apply(r, col, 'G', h.reshape(n, -1))
            if g is not None:
                e += 1j * k * g.reshape(n, 3, K)
            p = self._apply(r, col, pk, s)
            if p is not None:
                e -= p
            c = self._apply(r, col, pk, h)
            if c is not None:
                hh += c
        e, hh = e.cpu().numpy(), hh.cpu().numpy()
        if K == 1:
            e, hh = e[..., 0], hh[..., 0]
        return CompStruct(self.p1, sig.enei, e=e, h=hh)


class CompGreenStat(object):
    """Quasistatic Green function of a particle with itself: ``F`` (refined,
    closed-surface corrected), ``G``, and ``eval(*keys, ind=...)`` for G, F,
    H1, H2, Gp, H1p, H2p (mnpbem/greenfun/compgreen_stat.py:219-294, 466-528,
    678-990).  Entries come from the retarded entry kernel at k = 0, where the
    phase is 1 and only the order-0 refined coefficients remain."""

    def __new__(cls, p1, p2=None, **options):
        # a point set as p1 (the reference's CompGreenStat(ComPoint, particle))
        from .points import is_point_set, CompGreenStatPoints
        if is_point_set(p1) and p2 is not None:
            return CompGreenStatPoints(p1, p2, **options)
        return super(CompGreenStat, cls).__new__(cls)

    def __init__(self, p1, p2=None, **options):
        if p2 is not None and p2 is not p1:
            raise NotImplementedError("CompGreenStat: only p1 is p2 is supported")
        self.p1 = self.p2 = p1
        self.tables = SurfaceTables(p1, rel_cutoff=options.get('RelCutoff', 3),
                                    abs_cutoff=options.get('AbsCutoff', 0))
        t = self.tables
        n = t.n
        self.F_dev = torch.empty((n, n), dtype=torch.float64, device=t.device)
        call('mnpb_static_matrix', _lib.stream_handle(), n, ptr(t.pos), ptr(t.nvec), ptr(t.area),
             ptr(t.rptr), ptr(t.cols), ptr(t.fstat), ptr(t.cdir), ptr(t.fsum), ptr(self.F_dev), n)
        npart = t.nparts
        self._kb = np.zeros((npart, npart, 2))
        self._sb = np.ones((npart, npart))

    @property
    def F(self):
        torch.cuda.synchronize()
        return np.ascontiguousarray(self.F_dev.cpu().numpy().T)

    @property
    def G(self):
        return self._eval_key('G', None)

    def _eval_key(self, key, ind):
        if key not in KEYS:
            raise ValueError("Unknown key: {}".format(key))
        if key == 'F' and ind is None:
            return self.F
        if ind is not None:
            ind = np.asarray(ind, dtype=np.int64).ravel()
        out = self.tables.green_eval(self._kb, self._sb, KEYS[key], ind=ind).cpu().numpy()
        return out.real if key in ('G', 'F', 'H1', 'H2') else out.real.copy()

    def eval(self, *args, **kwargs):
        """``eval('G')``, ``eval('H1', 'H2')``, ``eval(ind, 'G')`` or
        ``eval('G', ind=ind)`` (compgreen_stat.py:678-750): one array per key,
        a tuple for several keys; ``ind`` are row-major linear indices."""
        if len(args) == 0:
            raise ValueError("At least one key must be provided")
        ind = kwargs.get('ind', None)
        if not isinstance(args[0], str):
            ind, keys = args[0], args[1:]
        else:
            keys = args
        res = [self._eval_key(k, ind) for k in keys]
        return res[0] if len(res) == 1 else tuple(res)

    def eval_block(self, key, enei, col_start, col_stop):
        """Columns [col_start, col_stop) of ``eval(key)`` (compgreen_stat.py:
        750-800; ``enei`` is accepted and unused, as in the reference)."""
        if key not in KEYS:
            raise ValueError("Unknown key: {}".format(key))
        col_start, col_stop = int(col_start), int(col_stop)
        if not (0 <= col_start <= col_stop <= self.tables.n):
            raise ValueError("eval_block col range out of bounds")
        if key == 'F':
            return np.ascontiguousarray(self.F[:, col_start:col_stop])
        out = self.tables.green_eval(self._kb, self._sb, KEYS[key], col_start=col_start,
                                     ncol=col_stop - col_start).cpu().numpy()
        return np.ascontiguousarray(out.real)
