"""Spectra of many particles of uneven size, solved in shared launches.

The reference solves such a set one particle and one wavelength at a time
(``BEMRet(p).solve(exc.potential(p, enei))`` per pair, mnpbem/bem/bem_ret.py:
293-525, 1569-1831; one process per GPU over particles in
mnpbem/utils/multi_gpu.py:81).  Here every (particle, wavelength) pair is one
entry of a batched mixed-precision factorisation:

* particles are grouped by face count; a group's (particle, wavelength)
  entries are cut into launch batches sized to the device memory.  With
  ``pad_ratio`` particles whose face counts lie within that ratio share one
  group: every entry is padded to the group's largest face count with an
  identity block (``mnpb_pad_entries``; exact, the pad decouples), so
  particles of different size go through one factorisation;
* each particle's wavelengths are assembled into consecutive entries of the
  batch (one assembly launch per particle), with its own face normals
  (``nvec_stride`` of the C ABI) so one factorisation launch sequence serves
  particles of different shape;
* the factorisation of a batch is replayed as a CUDA graph when the same
  buffers come round again, and its GEMM launch configuration (tile width,
  persistent threshold, ring depth) is picked per (face count, batch size) by
  ``autotune.GemmTuner`` on the first batch of that shape;
* solutions are refined in FP64 against each entry's exact operator
  (``BEMRet(precision='mixed')``), then extinction and scattering of every
  excitation come from the far fields on the GPU.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .autotune import DEFAULT_CONFIG, GemmTuner, set_gemm_config
from .bem import _MixedBatch, _check_particle, _scalar_eps
from .compstruct import CompStruct
from .excitation import pinfty
from .greenfun import SurfaceTables
from .materials import eps_k

__all__ = ["BatchedBEMRet"]


class BatchedBEMRet(object):
    """Mixed-precision retarded BEM solver for a set of particles.

    ``particles``: ComParticle objects (any face counts; the same materials
    on each side of every face of one particle).  ``max_batch`` caps the
    entries per launch batch, ``mem_bytes`` the device memory the batch
    buffers may take (default: 70 % of the free memory at construction).
    ``tuner``: a ``GemmTuner`` (a new one by default; ``None`` keeps the
    library's default launch configuration).  ``pad_ratio`` (e.g. 1.25):
    particles whose face counts differ by at most that factor are padded to a
    common size and solved in the same launches (default: equal face counts
    only)."""

    def __init__(self, particles, refine_tol=1e-8, refine_maxit=20, max_batch=256,
                 mem_bytes=None, tuner='auto', pad_ratio=None):
        self.particles = list(particles)
        for p in self.particles:
            _check_particle(p, 'BatchedBEMRet')
        self.refine_tol = refine_tol
        self.refine_maxit = refine_maxit
        self.max_batch = int(max_batch)
        self.tables = [SurfaceTables(p) for p in self.particles]
        self.tuner = GemmTuner() if tuner == 'auto' else tuner
        if mem_bytes is None:
            free, _ = torch.cuda.mem_get_info()
            mem_bytes = int(0.7 * free)
        self.mem_bytes = int(mem_bytes)
        self.groups = self.buckets([t.n for t in self.tables], pad_ratio)
        self._bufs = None
        self.stats = []

    # ------------------------------------------------------------------ sizes
    @staticmethod
    def buckets(sizes, pad_ratio=None):
        """Groups of particle indices by face count: {size: [indices]}.  With
        ``pad_ratio``, consecutive face counts (ascending) join a group while
        they stay within pad_ratio of its smallest; the key is the group's
        largest face count, the size its entries are padded to."""
        groups = {}
        if pad_ratio is None:
            for i, n in enumerate(sizes):
                groups.setdefault(int(n), []).append(i)
            return groups
        if pad_ratio < 1.0:
            raise ValueError("BatchedBEMRet: pad_ratio must be >= 1")
        bucket, lo = [], None
        for i in sorted(range(len(sizes)), key=lambda i: sizes[i]):
            if bucket and sizes[i] > lo * pad_ratio:
                groups[int(max(sizes[j] for j in bucket))] = bucket
                bucket = []
            if not bucket:
                lo = sizes[i]
            bucket.append(i)
        if bucket:
            groups[int(max(sizes[j] for j in bucket))] = bucket
        return groups

    @staticmethod
    def entry_bytes(n, K):
        """Device bytes one (particle, wavelength) entry of a batch takes."""
        L = _lib.lib()
        ld = (n + 3) // 4 * 4
        mats = 4 * n * ld * 16 + 5 * 2 * n * ld * 4
        work = int(L.mnpb_bemret_workspace_mixed(n, 1)) + 4 * int(L.mnpb_bemret_dinv_floats(n, 1))
        refine = int(L.mnpb_bemret_refine_workspace(n, 1, K))
        vecs = (16 + 3 * 8) * K * n * 16 + n * 3 * 8
        return mats + work + refine + vecs

    def _batches(self, n, nentries, K):
        per = self.entry_bytes(n, K)
        bmax = max(1, min(self.max_batch, self.mem_bytes // per))
        nb = -(-nentries // bmax)
        size = -(-nentries // nb)
        return [(s, min(s + size, nentries)) for s in range(0, nentries, size)], size

    # --------------------------------------------------------------- buffers
    def _buffers(self, n, B, K):
        key = (n, B, K)
        if self._bufs is not None and self._bufs[0] == key:
            return self._bufs[1]
        self._bufs = None
        torch.cuda.empty_cache()
        dev = self.tables[self.groups[n][0]].device
        bt = _MixedBatch(type('Size', (), {'device': dev, 'n': n})(), [0.0] * B)
        bt.nv = torch.empty((B, n, 3), dtype=torch.float64, device=dev)
        bt.pots = torch.empty((B, 16, K, n), dtype=torch.complex128, device=dev)
        bt.xin = torch.empty((B, 8, K, n), dtype=torch.complex128, device=dev)
        bt.x = torch.empty_like(bt.xin)
        wb = int(_lib.lib().mnpb_bemret_refine_workspace(n, B, K))
        bt.rwork = torch.empty(wb, dtype=torch.uint8, device=dev)
        bt.n_of = torch.empty(B, dtype=torch.int32, device=dev)
        self._bufs = (key, bt)
        return bt

    # ------------------------------------------------------------------ steps
    @staticmethod
    def _runs(members, eneis, s0, s1):
        """Consecutive slots of one particle inside entries [s0, s1):
        (particle index, first slot, wavelengths)."""
        L = len(eneis)
        out = []
        e = s0
        while e < s1:
            m, li = divmod(e, L)
            stop = min(s1, (m + 1) * L)
            out.append((members[m], e - s0, [eneis[q] for q in range(li, li + stop - e)]))
            e = stop
        return out

    def _assemble(self, bt, runs, n):
        """Each particle's matrices (its own face count) into the top-left
        corner of the batch's n x n entries."""
        ld = bt.ld
        for m, off, lams in runs:
            t = self.tables[m]
            kblk, sblk = t.k_tables(lams)
            d_k = torch.from_numpy(np.ascontiguousarray(kblk)).to(t.device)
            d_s = torch.from_numpy(np.ascontiguousarray(sblk)).to(t.device)
            poff = np.ascontiguousarray(t.part_off, dtype=np.int64)
            nb = len(lams)
            sl = slice(off, off + nb)
            call('mnpb_assemble_ret2', _lib.stream_handle(), t.n, nb, ptr(t.pos), ptr(t.nvec),
                 ptr(t.area), t.nparts, ptr(poff), ptr(d_k), ptr(d_s), t.nref, ptr(t.rows),
                 ptr(t.cols), ptr(t.g), ptr(t.fn), ptr(bt.G1[sl]), ptr(bt.H1[sl]),
                 ptr(bt.G2[sl]), ptr(bt.H2[sl]), ld, ld * n, ptr(bt.G1p[sl]), ptr(bt.H1p[sl]),
                 ptr(bt.G2p[sl]), ptr(bt.H2p[sl]), ld, 2 * ld * n, ld * n)

    def _factor(self, bt, n, B):
        call('mnpb_bemret_init_mixed', _lib.stream_handle(), n, B, ptr(bt.G1p), ptr(bt.G2p),
             ptr(bt.H1p), ptr(bt.H2p), ptr(bt.Dp), bt.ld, ptr(bt.eps), ptr(bt.kvac), ptr(bt.nv),
             3 * n, ptr(bt.piv), ptr(bt.info), ptr(bt.dinv), ptr(bt.work), bt.work.numel())

    def solve_spectrum(self, exc, eneis, keep_solutions=False):
        """Extinction and scattering of every particle at every wavelength for
        the plane waves of ``exc`` (a ``PlaneWaveRet`` of this package with up
        to 4 polarisations): dict with ``ext`` and ``sca`` arrays of shape
        (particles, wavelengths, polarisations), ``iters`` (refinement
        corrections per entry) and, if ``keep_solutions``, ``solutions``:
        per particle a list of CompStructs."""
        eneis = [float(e) for e in eneis]
        P, L, K = len(self.particles), len(eneis), exc.pol.shape[0]
        if K > 4:
            raise ValueError("BatchedBEMRet: at most 4 excitations per solve")
        ext = np.zeros((P, L, K))
        sca = np.zeros((P, L, K))
        iters = np.zeros((P, L), dtype=np.int64)
        sols = [[None] * L for _ in range(P)] if keep_solutions else None
        nvec_s, area_s = pinfty()
        self.stats = []
        bt = None
        for n in sorted(self.groups):
            members = self.groups[n]
            spans, B = self._batches(n, len(members) * L, K)
            for s0, s1 in spans:
                nb = s1 - s0
                # drop this frame's reference first: a new buffer shape must be
                # able to free the previous set before it allocates its own
                bt = None
                bt = self._buffers(n, B, K)
                runs = self._runs(members, eneis, s0, s1)
                eps = np.zeros((B, 4))
                kvac = np.ones(B)
                n_of = np.zeros(B, dtype=np.int32)
                for m, off, lams in runs:
                    for q, lam in enumerate(lams):
                        e1, e2 = _scalar_eps(self.particles[m], lam)
                        eps[off + q] = (e1.real, e1.imag, e2.real, e2.imag)
                        kvac[off + q] = 2 * np.pi / lam
                    nm = self.tables[m].n
                    bt.nv[off:off + len(lams), :nm] = self.tables[m].nvec
                    bt.nv[off:off + len(lams), nm:] = 0.0
                    n_of[off:off + len(lams)] = nm
                if nb < B:
                    # unused tail slots of the last batch: copies of the first entry
                    eps[nb:] = eps[0]
                    kvac[nb:] = kvac[0]
                    n_of[nb:] = n_of[0]
                    bt.nv[nb:] = bt.nv[0]
                bt.eps.copy_(torch.from_numpy(eps))
                bt.kvac.copy_(torch.from_numpy(kvac))
                bt.n_of.copy_(torch.from_numpy(n_of))
                padded = bool((n_of[:nb] < n).any())

                def factor():
                    self._assemble(bt, runs, n)
                    if padded:
                        call('mnpb_pad_entries', _lib.stream_handle(), n, nb, ptr(bt.n_of),
                             ptr(bt.G1), ptr(bt.G2), ptr(bt.H1), ptr(bt.H2), bt.ld,
                             bt.ld * n, ptr(bt.G1p), ptr(bt.G2p), ptr(bt.H1p), ptr(bt.H2p),
                             bt.ld, bt.ld * n, 2 * bt.ld * n)
                    if nb < B:
                        for A in (bt.G1, bt.G2, bt.H1, bt.H2, bt.G1p, bt.G2p, bt.H1p, bt.H2p):
                            A[nb:] = A[0]
                    self._factor(bt, n, B)

                cfg = DEFAULT_CONFIG
                if self.tuner is not None:
                    cfg = self.tuner.choose((n, B), factor)
                factor()
                if self.tuner is not None:
                    set_gemm_config(DEFAULT_CONFIG)
                info = bt.info.cpu().numpy()
                if info[:, :nb].any():
                    raise _lib.MNPBError('BatchedBEMRet', 3, "zero pivot in a factorisation")
                # excitation of every entry
                bt.pots.zero_()
                for m, off, lams in runs:
                    pots, _ = exc.potential_device(self.particles[m], self.tables[m], lams)
                    bt.pots[off:off + len(lams), :, :, :self.tables[m].n] = pots
                call('mnpb_bemret_excitation', _lib.stream_handle(), n, B, K, ptr(bt.pots),
                     ptr(bt.eps), ptr(bt.kvac), ptr(bt.nv), 3 * n, ptr(bt.xin))
                it = np.zeros(B, dtype=np.int32)
                rr = np.zeros(B)
                call('mnpb_bemret_solve_refine', _lib.stream_handle(), n, B, K, ptr(bt.G1p),
                     ptr(bt.G2p), ptr(bt.H1p), ptr(bt.H2p), ptr(bt.Dp), bt.ld, ptr(bt.piv),
                     ptr(bt.dinv), ptr(bt.G1), ptr(bt.G2), ptr(bt.H1), ptr(bt.H2), ptr(bt.eps),
                     ptr(bt.kvac), ptr(bt.nv), 3 * n, ptr(bt.xin), ptr(bt.x),
                     int(self.refine_maxit), float(self.refine_tol), ptr(it), ptr(rr),
                     ptr(bt.rwork), bt.rwork.numel())
                # cross sections per particle
                for m, off, lams in runs:
                    p, t = self.particles[m], self.tables[m]
                    x = bt.x[off:off + len(lams), :, :, :t.n].contiguous()
                    e, _ = exc.farfield_device(p, t, x, lams, exc.dir)
                    ef, hf = exc.farfield_device(p, t, x, lams, nvec_s)
                    e, ef, hf = e.cpu().numpy(), ef.cpu().numpy(), hf.cpu().numpy()
                    mi = m
                    li0 = eneis.index(lams[0])
                    for q, lam in enumerate(lams):
                        eps_med, k = eps_k(p.eps[exc.medium - 1], lam)
                        for i in range(K):
                            ext[mi, li0 + q, i] = np.real(
                                4 * np.pi / k * np.imag(np.sum(np.conj(exc.pol[i]) * e[q, i, i])))
                        dsca = 0.5 * np.real(np.einsum('dc,kdc->kd', nvec_s,
                                                       np.cross(ef[q], np.conj(hf[q]))))
                        sca[mi, li0 + q] = dsca @ area_s / (0.5 * np.real(np.sqrt(eps_med)))
                        iters[mi, li0 + q] = it[off + q]
                    if keep_solutions:
                        xh = x.cpu().numpy()
                        for q, lam in enumerate(lams):
                            v = xh[q]
                            sols[mi][li0 + q] = CompStruct(
                                p, lam, sig1=v[0].T.copy(), h1=v[1:4].transpose(2, 0, 1).copy(),
                                sig2=v[4].T.copy(), h2=v[5:8].transpose(2, 0, 1).copy())
                self.stats.append({'n': n, 'entries': nb, 'batch': B, 'config': list(cfg),
                                   'faces': sorted(set(int(v) for v in n_of[:nb]))})
        out = {'ext': ext, 'sca': sca, 'iters': iters}
        if keep_solutions:
            out['solutions'] = sols
        return out
