"""Dense BEM solvers on the GPU: ``BEMRet`` (retarded) and ``BEMStat``
(quasistatic), with the reference call surface

    sig, bem = bem.solve(exc)          # exc = PlaneWaveRet(...).potential(p, enei)

(mnpbem/bem/bem_ret.py:138-1986, mnpbem/bem/bem_stat.py:101-807).  Every
wavelength's matrices are assembled, factorised and solved by the CUDA
library; results come back as host NumPy arrays in a ``CompStruct``.

``solve_spectrum`` runs a whole list of wavelengths through the same kernels
in batches (all wavelengths of a batch share every launch), which is how a
spectrum should be computed on the GPU.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .compstruct import CompStruct
from .greenfun import CompGreenRet, CompGreenStat
from .materials import eps_k

__all__ = ["BEMRet", "BEMStat"]


def _check_particle(p, name):
    if p is None:
        raise ValueError("{}: 'p' must be a ComParticle (or compatible particle object), "
                         "got None.".format(name))
    if not (hasattr(p, 'pos') and hasattr(p, 'nvec') and hasattr(p, 'eps')):
        raise TypeError("{}: 'p' must expose ComParticle-like attributes (pos, nvec, eps); "
                        "got {!r}.".format(name, type(p).__name__))


def _scalar_eps(p, enei):
    """Inside/outside dielectric constants; must be uniform over the faces."""
    e1 = np.asarray(p.eps1(enei))
    e2 = np.asarray(p.eps2(enei))
    if not (np.allclose(e1, e1[0]) and np.allclose(e2, e2[0])):
        raise NotImplementedError("BEMRet: face-dependent eps (several materials on one side) "
                                  "is not supported by the GPU solver")
    return complex(e1[0]), complex(e2[0])


def _fields_by_wavelength(x, K):
    """sig1, sig2 (B, n[, K]) and h1, h2 (B, n, 3[, K]) from a batch of
    solution vectors x (B, 8, K, n) (sig1, h1x..z, sig2, h2x..z): one
    reordering copy per field for the whole batch, so that each wavelength's
    fields are contiguous views; the trailing K axis is dropped for K = 1
    (the layout ``BEMRet._to_compstruct`` gives one wavelength)."""
    sig1 = np.ascontiguousarray(x[:, 0].transpose(0, 2, 1))
    sig2 = np.ascontiguousarray(x[:, 4].transpose(0, 2, 1))
    h1 = np.ascontiguousarray(x[:, 1:4].transpose(0, 3, 1, 2))
    h2 = np.ascontiguousarray(x[:, 5:8].transpose(0, 3, 1, 2))
    if K == 1:
        sig1, sig2, h1, h2 = sig1[..., 0], sig2[..., 0], h1[..., 0], h2[..., 0]
    return sig1, sig2, h1, h2


def _fields_device(x):
    """The reordering of ``_fields_by_wavelength`` done on the device: one
    flat tensor [sig1 (B, n, K) | sig2 | h1 (B, n, 3, K) | h2] from a batch of
    solution vectors x (B, 8, K, n)."""
    return torch.cat([x[:, 0].permute(0, 2, 1).reshape(-1),
                      x[:, 4].permute(0, 2, 1).reshape(-1),
                      x[:, 1:4].permute(0, 3, 1, 2).reshape(-1),
                      x[:, 5:8].permute(0, 3, 1, 2).reshape(-1)])


def _fields_host(flat, shape):
    """Views sig1, sig2 (B, n, K) and h1, h2 (B, n, 3, K) of the flat host
    array ``_fields_device`` made from solutions of shape (B, 8, K, n)."""
    B, _, K, n = shape
    s = B * n * K
    sig1 = flat[:s].reshape(B, n, K)
    sig2 = flat[s:2 * s].reshape(B, n, K)
    h1 = flat[2 * s:5 * s].reshape(B, n, 3, K)
    h2 = flat[5 * s:8 * s].reshape(B, n, 3, K)
    return sig1, sig2, h1, h2


class _RetBatch(object):
    """Device buffers of one factorised batch of wavelengths (FP64)."""

    mixed = False

    def __init__(self, tables, eneis):
        dev = tables.device
        n = tables.n
        B = len(eneis)
        self.n, self.B, self.eneis = n, B, list(eneis)
        c128 = dict(dtype=torch.complex128, device=dev)
        # G1/G2 and H1/H2 back to back: the solver factorises each pair as one batch
        self.GG = torch.empty((2, B, n, n), **c128)
        self.HH = torch.empty((2, B, n, n), **c128)
        self.G1, self.G2 = self.GG[0], self.GG[1]
        self.H1, self.H2 = self.HH[0], self.HH[1]
        self.D = torch.empty((B, n, n), **c128)
        self.piv = torch.empty((3, B, n), dtype=torch.int32, device=dev)
        self.info = torch.zeros((2, B), dtype=torch.int32, device=dev)
        wb = int(_lib.lib().mnpb_bemret_workspace_f64(n, B))
        self.work = torch.empty(wb, dtype=torch.uint8, device=dev)


class _MixedBatch(object):
    """Device buffers of a mixed-precision batch: FP64 G1, G2, H1, H2 (the
    exact operator for refinement) and their planar FP32 copies, factorised on
    the tensor cores.  Leading dimension ld = n rounded up to 4."""

    mixed = True

    def __init__(self, tables, eneis):
        dev = tables.device
        n = tables.n
        B = len(eneis)
        ld = (n + 3) // 4 * 4
        self.n, self.B, self.ld, self.eneis = n, B, ld, list(eneis)
        c128 = dict(dtype=torch.complex128, device=dev)
        f32 = dict(dtype=torch.float32, device=dev)
        self.G1, self.G2, self.H1, self.H2 = [torch.empty((B, n, ld), **c128) for _ in range(4)]
        # planar copies; G1p/G2p and H1p/H2p back to back (factorised as one batch)
        self.GGp = torch.empty((2, B, 2, n, ld), **f32)
        self.HHp = torch.empty((2, B, 2, n, ld), **f32)
        self.G1p, self.G2p = self.GGp[0], self.GGp[1]
        self.H1p, self.H2p = self.HHp[0], self.HHp[1]
        self.Dp = torch.empty((B, 2, n, ld), **f32)
        self.piv = torch.empty((3, B, n), dtype=torch.int32, device=dev)
        self.info = torch.zeros((2, B), dtype=torch.int32, device=dev)
        self.dinv = torch.empty(int(_lib.lib().mnpb_bemret_dinv_floats(n, B)), **f32)
        wb = int(_lib.lib().mnpb_bemret_workspace_mixed(n, B))
        self.work = torch.empty(wb, dtype=torch.uint8, device=dev)
        self.eps = torch.empty((B, 4), dtype=torch.float64, device=dev)
        self.kvac = torch.empty(B, dtype=torch.float64, device=dev)
        self.iters = None
        self.relres = None


class BEMRet(object):
    """Retarded BEM solver (full Maxwell equations), dense, on the GPU."""

    def __init__(self, p, enei=None, precision='fp64', refine_tol=1e-11, refine_maxit=20,
                 **options):
        """``precision``: 'fp64' (the reference's arithmetic) or 'mixed' (FP32
        storage, TF32 tensor-core factorisations, FP64 iterative refinement
        of every wavelength's solution until its last correction is below
        ``refine_tol`` relative to the solution)."""
        _check_particle(p, 'BEMRet')
        if precision not in ('fp64', 'mixed'):
            raise ValueError("BEMRet: precision must be 'fp64' or 'mixed'")
        self.precision = precision
        self.refine_tol = refine_tol
        self.refine_maxit = refine_maxit
        self.p = p
        self.enei = None
        self.options = dict(options)
        refun = self.options.pop('refun', None)
        schur = self.options.pop('schur', False)
        if refun is not None or schur:
            raise NotImplementedError("BEMRet: refun/schur are not supported by the GPU solver")
        self.g = CompGreenRet(p, p, **self.options)
        self.tables = self.g.tables
        self.nvec = np.asarray(p.nvec)
        self._batch = None
        self.k = None
        if enei is not None:
            self.init(enei)

    # ------------------------------------------------------------------ init
    def _eps_tables(self, eneis):
        B = len(eneis)
        eps = np.zeros((B, 4))
        kvac = np.zeros(B)
        for b, enei in enumerate(eneis):
            e1, e2 = _scalar_eps(self.p, enei)
            eps[b] = (e1.real, e1.imag, e2.real, e2.imag)
            kvac[b] = 2 * np.pi / enei
        return eps, kvac

    def _factor(self, eneis, stream=None, reuse=True):
        t = self.tables
        n, B = t.n, len(eneis)
        kblk, sblk = t.k_tables(eneis)
        eps, kvac = self._eps_tables(eneis)
        sh = _lib.stream_handle(stream)
        if self.precision == 'fp64':
            bt = _RetBatch(t, eneis)
            t.assemble(kblk, sblk, (bt.G1, bt.H1, bt.G2, bt.H2), mode=0, stream=stream)
            bt.eps = torch.from_numpy(eps).to(t.device)
            bt.kvac = torch.from_numpy(kvac).to(t.device)
            call('mnpb_bemret_init_f64', sh, n, B, ptr(bt.G1), ptr(bt.G2), ptr(bt.H1),
                 ptr(bt.H2), ptr(bt.D), n, n * n, ptr(bt.eps), ptr(bt.kvac), ptr(t.nvec), 0,
                 ptr(bt.piv), ptr(bt.info), ptr(bt.work), bt.work.numel())
            return bt
        bt = self._mixed_batch(eneis, stream) if reuse else _MixedBatch(t, eneis)
        ld = bt.ld
        d_k = torch.from_numpy(np.ascontiguousarray(kblk)).to(t.device)
        d_s = torch.from_numpy(np.ascontiguousarray(sblk)).to(t.device)
        poff = np.ascontiguousarray(t.part_off, dtype=np.int64)
        call('mnpb_assemble_ret2', sh, n, B, ptr(t.pos), ptr(t.nvec), ptr(t.area), t.nparts,
             ptr(poff), ptr(d_k), ptr(d_s), t.nref, ptr(t.rows), ptr(t.cols), ptr(t.g),
             ptr(t.fn), ptr(bt.G1), ptr(bt.H1), ptr(bt.G2), ptr(bt.H2), ld, ld * n,
             ptr(bt.G1p), ptr(bt.H1p), ptr(bt.G2p), ptr(bt.H2p), ld, 2 * ld * n, ld * n)
        bt.eps.copy_(torch.from_numpy(np.ascontiguousarray(eps)).view(B, 4))
        bt.kvac.copy_(torch.from_numpy(np.ascontiguousarray(kvac)).view(B))
        call('mnpb_bemret_init_mixed', sh, n, B, ptr(bt.G1p), ptr(bt.G2p), ptr(bt.H1p),
             ptr(bt.H2p), ptr(bt.Dp), ld, ptr(bt.eps), ptr(bt.kvac), ptr(t.nvec), 0, ptr(bt.piv),
             ptr(bt.info), ptr(bt.dinv), ptr(bt.work), bt.work.numel())
        return bt

    def _mixed_batch(self, eneis, stream):
        """Device buffers for a mixed batch.  The latest batch's buffers are
        kept and handed out again to the next batch of the same size on the
        same stream (stream order makes the reuse safe), so that the
        factorisation's launch sequence sees the same addresses and the
        library replays it as a CUDA graph."""
        key = (len(eneis), _lib.stream_handle(stream).value)
        cached = getattr(self, '_mixed_cache', None)
        if cached is not None and cached[0] == key:
            bt = cached[1]
            bt.eneis = list(eneis)
            bt.iters, bt.relres = None, None
            return bt
        self._mixed_cache = None       # release the old buffers before allocating
        bt = _MixedBatch(self.tables, eneis)
        self._mixed_cache = (key, bt)
        return bt

    def init(self, enei):
        """Matrices for wavelength ``enei``; no-op if already there (bem_ret.py:293-311)."""
        if self.enei is not None and np.isclose(self.enei, enei):
            return self
        self._batch = self._factor([enei], reuse=False)   # kept across solve() calls
        info = self._batch.info.cpu().numpy()
        if info.any():
            raise _lib.MNPBError('BEMRet.init', 3, "zero pivot at column {}".format(int(info.max())))
        self.enei = enei
        self.k = 2 * np.pi / enei
        return self

    __call__ = init

    def clear(self):
        self._batch = None
        self.enei = None
        return self

    # ----------------------------------------------------------------- solve
    @staticmethod
    def _pots(exc, n):
        """Potentials of an excitation as a (16, K, n) complex host array."""
        def get(name):
            v = exc.get(name, 0) if hasattr(exc, 'get') else getattr(exc, name, 0)
            return v if isinstance(v, np.ndarray) else None
        fields = [get(k) for k in ('phi1', 'phi1p', 'a1', 'a1p', 'phi2', 'phi2p', 'a2', 'a2p')]
        K = 1
        for f in fields:
            if f is not None:
                if f.ndim == 3:
                    K = max(K, f.shape[2])
                elif f.ndim == 2 and f.shape[1] != 3:
                    K = max(K, f.shape[1])
        out = np.zeros((16, K, n), dtype=complex)
        comp = 0
        for f, width in zip(fields, (1, 1, 3, 3, 1, 1, 3, 3)):
            if f is not None:
                if width == 1:
                    v = f.reshape(n, -1)
                    out[comp] = np.broadcast_to(v, (n, K)).T
                else:
                    v = f.reshape(n, 3, -1)
                    out[comp:comp + 3] = np.broadcast_to(v, (n, 3, K)).transpose(1, 2, 0)
            comp += width
        return out, K

    def _solve_batch(self, bt, pots_dev, K, stream=None):
        """x_out (B, 8, K, n) device for potentials (B, 16, K, n) device."""
        t = self.tables
        n, B = t.n, bt.B
        sh = _lib.stream_handle(stream)
        xin = torch.empty((B, 8, K, n), dtype=torch.complex128, device=t.device)
        xout = torch.empty_like(xin)
        call('mnpb_bemret_excitation', sh, n, B, K, ptr(pots_dev), ptr(bt.eps), ptr(bt.kvac),
             ptr(t.nvec), 0, ptr(xin))
        if not bt.mixed:
            wb = B * n * 15 * K * 16
            work = torch.empty(wb, dtype=torch.uint8, device=t.device)
            call('mnpb_bemret_solve_f64', sh, n, B, K, ptr(bt.G1), ptr(bt.G2), ptr(bt.H1),
                 ptr(bt.H2), ptr(bt.D), n, n * n, ptr(bt.piv), ptr(bt.eps), ptr(bt.kvac),
                 ptr(t.nvec), 0, ptr(xin), ptr(xout), ptr(work), wb)
            return xout
        out = []
        for k0 in range(0, K, 4):          # the refinement solves up to 4 excitations at once
            kk = min(4, K - k0)
            b_in = xin[:, :, k0:k0 + kk].contiguous()
            x = torch.empty_like(b_in)
            wb = int(_lib.lib().mnpb_bemret_refine_workspace(n, B, kk))
            work = torch.empty(wb, dtype=torch.uint8, device=t.device)
            iters = np.zeros(B, dtype=np.int32)
            relres = np.zeros(B)
            call('mnpb_bemret_solve_refine', sh, n, B, kk, ptr(bt.G1p), ptr(bt.G2p),
                 ptr(bt.H1p), ptr(bt.H2p), ptr(bt.Dp), bt.ld, ptr(bt.piv), ptr(bt.dinv), ptr(bt.G1),
                 ptr(bt.G2), ptr(bt.H1), ptr(bt.H2), ptr(bt.eps), ptr(bt.kvac), ptr(t.nvec), 0,
                 ptr(b_in), ptr(x), int(self.refine_maxit), float(self.refine_tol), ptr(iters),
                 ptr(relres), ptr(work), wb)
            bt.iters, bt.relres = iters, relres
            out.append(x)
        return out[0] if len(out) == 1 else torch.cat(out, dim=2).contiguous()

    def solve(self, exc):
        """Surface charges and currents for an excitation (bem_ret.py:1569-1831)."""
        enei = exc['enei']
        self.init(enei)
        n = self.tables.n
        pots, K = self._pots(exc, n)
        d_pots = torch.from_numpy(pots).to(self.tables.device).unsqueeze(0)
        xout = self._solve_batch(self._batch, d_pots, K)
        x = xout[0].cpu().numpy()
        sig = self._to_compstruct(x, K, enei)
        return sig, self

    def _to_compstruct(self, x, K, enei):
        n = self.tables.n
        sig1 = x[0].T.copy()
        h1 = x[1:4].transpose(2, 0, 1).copy()
        sig2 = x[4].T.copy()
        h2 = x[5:8].transpose(2, 0, 1).copy()
        if K == 1:
            sig1, sig2 = sig1[:, 0], sig2[:, 0]
            h1, h2 = h1[:, :, 0], h2[:, :, 0]
        return CompStruct(self.p, enei, sig1=sig1, sig2=sig2, h1=h1, h2=h2)

    def __truediv__(self, exc):
        return self.solve(exc)

    def potential(self, sig, inout=2):
        """Potentials and surface derivatives inside (1) or outside (2) of the
        particle for a solution (bem_ret.py:1833-1858, delegating to
        CompGreenRet.potential); the Green-function entries are evaluated on
        the fly on the GPU.  Unlike the reference this does not factorise the
        BEM matrices of ``sig.enei`` first: potentials need only G and H."""
        return self.g.potential(sig, inout)

    def field(self, sig, inout=2):
        """Electric and magnetic fields inside (1) or outside (2) of the
        particle for a solution (bem_ret.py:1860-1895, delegating to
        CompGreenRet.field: e = i k (G1 h1 + G2 h2) - H1p sig1 - H2p sig2,
        h = H1p x h1 + H2p x h2); no factorisation needed, as for potential."""
        return self.g.field(sig, inout)

    # ------------------------------------------------------- spectrum sweeps
    @staticmethod
    def pipeline(chunks, work, streams):
        """Run ``work(chunk, stream)`` for every chunk on ``streams`` CUDA
        streams, chunks dealt out round-robin, each stream driven by its own
        host thread; results in chunk order.  While one stream's refinement
        waits on the host between corrections, the other streams'
        factorisations keep the GPU busy.  The caller's current stream waits
        for all of them before returning."""
        import threading
        cur = torch.cuda.current_stream()
        if streams <= 1 or len(chunks) <= 1:
            return [work(c, cur) for c in chunks]
        streams = min(streams, len(chunks))
        sts = [torch.cuda.Stream() for _ in range(streams)]
        for st in sts:
            st.wait_stream(cur)
        results = [None] * len(chunks)
        errors = []

        def run(k):
            try:
                with torch.cuda.stream(sts[k]):
                    for i in range(k, len(chunks), streams):
                        results[i] = work(chunks[i], sts[k])
            except BaseException as e:       # re-raised in the caller's thread
                errors.append(e)

        threads = [threading.Thread(target=run, args=(k,)) for k in range(streams)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for st in sts:
            cur.wait_stream(st)
        if errors:
            raise errors[0]
        return results

    def solve_spectrum(self, exc, eneis, batch=16, stream=None, streams=1):
        """Solutions for every wavelength of ``eneis`` (host CompStructs).

        ``exc`` is a plane-wave excitation of this package (its potentials
        are generated on the GPU) or any object with ``potential(p, enei)``.
        Wavelengths are solved ``batch`` at a time; ``streams`` > 1 runs that
        many batches concurrently (see ``pipeline``).
        """
        chunks = [list(eneis[s:s + batch]) for s in range(0, len(eneis), batch)]

        def work(chunk, st):
            bt = self._factor(chunk, stream=st)
            pots, K = self._spectrum_pots(exc, chunk, st)
            xout = self._solve_batch(bt, pots, K, stream=st)
            with torch.cuda.stream(st):
                # fields reordered on the device (each wavelength's fields
                # contiguous), then one device -> pinned host copy
                # (page-locked: full PCIe rate) that the host only views
                dev = _fields_device(xout)
                host = torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
                host.copy_(dev, non_blocking=True)
            st.synchronize()
            return _fields_host(host.numpy(), xout.shape), K

        if streams > 1:
            res = self.pipeline(chunks, work, streams)
        else:
            cur = stream if stream is not None else torch.cuda.current_stream()
            res = [work(c, cur) for c in chunks]
        out = []
        for chunk, (fields, K) in zip(chunks, res):
            sig1, sig2, h1, h2 = fields
            if K == 1:
                sig1, sig2, h1, h2 = sig1[..., 0], sig2[..., 0], h1[..., 0], h2[..., 0]
            for b, enei in enumerate(chunk):
                out.append(CompStruct(self.p, enei, sig1=sig1[b], sig2=sig2[b], h1=h1[b],
                                      h2=h2[b]))
        return out

    def _spectrum_pots(self, exc, eneis, stream=None):
        if hasattr(exc, 'potential_device'):
            return exc.potential_device(self.p, self.tables, eneis, stream=stream)
        n = self.tables.n
        arrs = []
        K = 1
        for enei in eneis:
            pots, K = self._pots(exc.potential(self.p, enei), n)
            arrs.append(pots)
        return torch.from_numpy(np.stack(arrs)).to(self.tables.device), K


class BEMStat(object):
    """Quasistatic BEM solver, dense, on the GPU (mnpbem/bem/bem_stat.py:101-807)."""

    def __init__(self, p, enei=None, **options):
        _check_particle(p, 'BEMStat')
        self.p = p
        self.options = dict(options)
        if self.options.pop('schur', False):
            raise NotImplementedError("BEMStat: schur is not supported by the GPU solver")
        self.g = CompGreenStat(p, p, **self.options)
        self.tables = self.g.tables
        self.enei = None
        self._M = None
        if enei is not None:
            self(enei)

    @property
    def F(self):
        return self.g.F

    def _factor(self, eneis, stream=None):
        t = self.tables
        n, B = t.n, len(eneis)
        eps12 = np.zeros((B, n, 4))
        for b, enei in enumerate(eneis):
            e1 = np.asarray(self.p.eps1(enei))
            e2 = np.asarray(self.p.eps2(enei))
            eps12[b, :, 0], eps12[b, :, 1] = e1.real, e1.imag
            eps12[b, :, 2], eps12[b, :, 3] = e2.real, e2.imag
        d_eps = torch.from_numpy(eps12).to(t.device)
        M = torch.empty((B, n, n), dtype=torch.complex128, device=t.device)
        piv = torch.empty((B, n), dtype=torch.int32, device=t.device)
        info = torch.zeros(B, dtype=torch.int32, device=t.device)
        sh = _lib.stream_handle(stream)
        call('mnpb_stat_matrix', sh, n, B, ptr(self.g.F_dev), n, ptr(d_eps), ptr(M), n, n * n)
        call('mnpb_getrf_f64', sh, n, B, ptr(M), n, n * n, ptr(piv), n, ptr(info))
        return M, piv, info

    def __call__(self, enei):
        if self.enei is None or self.enei != enei:
            self._M, self._piv, info = self._factor([enei])
            if info.cpu().numpy().any():
                raise _lib.MNPBError('BEMStat', 3, "zero pivot")
            self.enei = enei
        return self

    init = __call__

    def solve(self, exc):
        return self.__truediv__(exc)

    def __truediv__(self, exc):
        self(exc.enei)
        phip = np.asarray(exc.phip)
        n = self.tables.n
        K = phip.size // n                      # trailing axes (npt, ndip, ...) as columns
        B = torch.from_numpy(np.ascontiguousarray(phip.reshape(n, K).T.astype(complex))) \
            .to(self.tables.device).unsqueeze(0).contiguous()
        call('mnpb_getrs_f64', _lib.stream_handle(), n, 1, K, ptr(self._M), n, n * n,
             ptr(self._piv), n, ptr(B), n, n * K)
        sig = B[0].cpu().numpy().T.reshape(phip.shape)
        return CompStruct(self.p, exc.enei, sig=sig), self

    def solve_spectrum(self, phip, eneis, batch=32, stream=None):
        """sigma (len(eneis), n, K) for a wavelength-independent phip (n, K)."""
        n = self.tables.n
        phip = np.asarray(phip).reshape(n, -1)
        K = phip.shape[1]
        out = []
        for s in range(0, len(eneis), batch):
            chunk = list(eneis[s:s + batch])
            M, piv, info = self._factor(chunk, stream)
            Bn = len(chunk)
            rhs = torch.from_numpy(np.ascontiguousarray(
                np.broadcast_to(phip.T.astype(complex), (Bn, K, n)))).to(self.tables.device)
            call('mnpb_getrs_f64', _lib.stream_handle(stream), n, Bn, K, ptr(M), n, n * n,
                 ptr(piv), n, ptr(rhs), n, n * K)
            out.append(rhs.cpu().numpy().transpose(0, 2, 1))
        return np.concatenate(out, axis=0)
