"""H-matrices on the GPU: ACA compression of dense Green-function matrices and
H-matrix times vectors (mnpbem/greenfun/hmatrix.py, aca_compgreen_ret.py).

``HTopology`` holds what depends only on the cluster tree and block partition
(block rectangles, leaf contribution lists, scratch offsets) as device
arrays; ``HMatrixGPU`` holds one compressed matrix: dense leaf blocks and
low-rank factors U, V (A_block ~ U V^T) in complex64, ranks per block.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .clustertree import BlockPartition

__all__ = ["HTopology", "HMatrixGPU", "hmat_matvec"]


def _i32(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).to(dev)


def _i64(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int64)).to(dev)


class HTopology(object):
    """Device-side structure of one block partition of one cluster tree."""

    def __init__(self, part, kmax, device):
        if not isinstance(part, BlockPartition):
            raise TypeError("HTopology: expected a BlockPartition")
        tree = part.tree
        self.part = part
        self.n = tree.n
        self.kmax = int(kmax)
        self.device = device
        dn, lr = part.dense, part.lowrank
        self.ndense, self.nlr = dn.shape[0], lr.shape[0]
        self.c2p = _i32(tree.ind[:, 0], device)
        self.dense = _i32(dn.reshape(-1, 4), device)
        self.lowrank = _i32(lr.reshape(-1, 4), device)
        # dense storage offsets (complex entries)
        dsz = dn[:, 1].astype(np.int64) * dn[:, 3]
        self.offD_h = np.concatenate([[0], np.cumsum(dsz)[:-1]]).astype(np.int64) if dn.size else \
            np.zeros(0, np.int64)
        self.dense_entries = int(dsz.sum())
        self.offD = _i64(self.offD_h, device)
        # ACA scratch offsets (FP64 complex entries): U (m x cap), V (n x cap)
        m, k = lr[:, 1].astype(np.int64), lr[:, 3].astype(np.int64)
        cap = np.minimum(np.minimum(m, k), self.kmax)
        sizes = np.stack([m * cap, k * cap], axis=1).reshape(-1)
        offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64) if sizes.size else \
            np.zeros(0, np.int64)
        self.scr_offU = _i64(offs[0::2], device)
        self.scr_offV = _i64(offs[1::2], device)
        self.scratch_entries = int(sizes.sum())
        self.max_mn = int((m + k).max()) if lr.size else 0
        # leaves (cluster rows) and their contribution lists
        leaves = tree.leaves()
        order = np.argsort(tree.cind[leaves, 0])
        leaves = leaves[order]
        lstart = tree.cind[leaves, 0]
        lsize = tree.cind[leaves, 1] - lstart + 1
        self.nleaf = leaves.size
        self.leaf_rows = _i32(np.stack([lstart, lsize], axis=1), device)
        lists = [[] for _ in range(self.nleaf)]
        for kind, blocks in ((0, dn), (1, lr)):
            for b, (r0, rm, _, _) in enumerate(blocks):
                lo = np.searchsorted(lstart, r0)
                hi = np.searchsorted(lstart, r0 + rm)
                code = b if kind == 0 else -b - 1
                for L in range(lo, hi):
                    lists[L].append(code)
        lptr = np.zeros(self.nleaf + 1, dtype=np.int64)
        lptr[1:] = np.cumsum([len(x) for x in lists])
        ent = np.concatenate([np.asarray(x, dtype=np.int32) for x in lists]) if lptr[-1] else \
            np.zeros(1, np.int32)
        self.lent_h = ent
        self.lent_leaf = np.repeat(np.arange(self.nleaf), np.diff(lptr)).astype(np.int64)
        self.lstart_h = np.asarray(lstart, dtype=np.int64)
        # 32-row chunks of the leaves, and work items (chunk, segment of at
        # most SEG entries of the leaf's list, first row << 6 | rows): one
        # warp per item
        SEG = 6
        ch, items, cptr = [], [], [0]
        for L in range(self.nleaf):
            for r0 in range(0, int(lsize[L]), 32):
                k = len(ch)
                ch.append((L, r0))
                rows = (r0 << 6) | min(32, int(lsize[L]) - r0)
                for e in range(int(lptr[L]), int(lptr[L + 1]), SEG):
                    items.append((k, e, min(e + SEG, int(lptr[L + 1])), rows))
                if lptr[L + 1] == lptr[L]:
                    items.append((k, 0, 0, rows))
                cptr.append(len(items))
        self.nchunk = len(ch)
        self.chunks = _i32(np.asarray(ch, dtype=np.int64).reshape(-1, 2), device)
        # V^T x work items: (block, first column, end column, segment)
        VSEG = 64
        vit, vptr = [], [0]
        for b in range(self.nlr):
            ncol = int(lr[b, 3])
            for sg, j0 in enumerate(range(0, ncol, VSEG)):
                vit.append((b, j0, min(j0 + VSEG, ncol), sg))
            vptr.append(len(vit))
        self.vseg_count = np.diff(np.asarray(vptr, dtype=np.int64))
        self.nvitem = max(1, len(vit))
        self.vitems_h = np.asarray(vit if vit else [(0, 0, 0, 0)], dtype=np.int64).reshape(-1, 4)
        self.vptr = _i32(np.asarray(vptr, dtype=np.int64), device)
        self.nitem = len(items)
        assert max(it[2] - it[1] for it in items) <= 32    # records held one per lane
        self.items = _i32(np.asarray(items, dtype=np.int64).reshape(-1, 4), device)
        self.cptr = _i32(np.asarray(cptr, dtype=np.int64), device)


# work records of the product kernels (layouts of the C ABI's rent / vent)
ROW_ENT = np.dtype([('a', '<i8'), ('xo', '<i8'), ('lda', '<i4'), ('cnt', '<i4'),
                    ('kind', '<i4'), ('pad', '<i4')])
VTX_ENT = np.dtype([('v', '<i8'), ('out', '<i8'), ('xo', '<i4'), ('cnt', '<i4'),
                    ('r', '<i4'), ('pad', '<i4')])


def _records(rec, dev):
    return torch.from_numpy(np.frombuffer(rec.tobytes(), dtype=np.uint8).copy()).to(dev)


def row_records(topo, rank, offU, offT):
    """One ROW_ENT per entry of the leaves' contribution lists: where the
    leaf's rows of the entry's dense block (or low-rank factor U) start, its
    column stride and column count, and where its x (or t) columns are."""
    code = topo.lent_h[:len(topo.lent_leaf)].astype(np.int64)
    lst = topo.lstart_h[topo.lent_leaf]
    rec = np.zeros(max(1, code.size), dtype=ROW_ENT)
    dn, lr = topo.part.dense, topo.part.lowrank
    d = code >= 0
    if d.any():
        bk = dn[code[d]].astype(np.int64)
        rec['a'][:code.size][d] = topo.offD_h[code[d]] + lst[d] - bk[:, 0]
        rec['lda'][:code.size][d] = bk[:, 1]
        rec['cnt'][:code.size][d] = bk[:, 3]
        rec['xo'][:code.size][d] = bk[:, 2]
    q = ~d
    if q.any():
        b = -code[q] - 1
        bk = lr[b].astype(np.int64)
        rec['a'][:code.size][q] = offU[b] + lst[q] - bk[:, 0]
        rec['lda'][:code.size][q] = bk[:, 1]
        rec['cnt'][:code.size][q] = rank[b]
        rec['xo'][:code.size][q] = offT[b]
        rec['kind'][:code.size][q] = 1
    return rec


def vtx_records(topo, rank, offV, offTP):
    """One VTX_ENT per V^T x item (a segment of one low-rank block)."""
    vi = topo.vitems_h
    rec = np.zeros(vi.shape[0], dtype=VTX_ENT)
    if topo.nlr:
        b, j0, j1, sg = vi[:, 0], vi[:, 1], vi[:, 2], vi[:, 3]
        if (j1 - j0).max() > 64:
            raise ValueError("vtx_records: segments of at most 64 columns (kernel staging)")
        r = rank[b]
        rec['v'] = offV[b] + j0 * r
        rec['out'] = offTP[b] + sg * r
        rec['xo'] = topo.part.lowrank[b, 2].astype(np.int64) + j0
        rec['cnt'] = j1 - j0
        rec['r'] = r
    return rec


class HMatrixGPU(object):
    """One ACA-compressed matrix (complex64 factors, FP64 products)."""

    def __init__(self, topo, A, lda, htol, scratch=None, stream=None):
        """Compress the dense complex128 column-major matrix at ``A`` (a
        torch tensor whose storage holds A[i + j*lda]) with ACA tolerance
        ``htol``.  ``scratch``: optional FP64 tensor reused between matrices."""
        self.topo = topo
        dev = topo.device
        sh = _lib.stream_handle(stream)
        self.D = torch.empty(max(1, 2 * topo.dense_entries), dtype=torch.float32, device=dev)
        call('mnpb_hmat_gather_dense', sh, ptr(A), lda, ptr(topo.c2p), topo.ndense,
             ptr(topo.dense), ptr(topo.offD), ptr(self.D))
        self.rank = torch.zeros(max(1, topo.nlr), dtype=torch.int32, device=dev)
        if topo.nlr:
            need = 2 * topo.scratch_entries
            if scratch is None or scratch.numel() < need:
                scratch = torch.empty(need, dtype=torch.float64, device=dev)
            call('mnpb_hmat_aca', sh, topo.n, ptr(A), lda, ptr(topo.c2p), topo.nlr,
                 ptr(topo.lowrank), ptr(topo.scr_offU), ptr(topo.scr_offV), topo.max_mn,
                 topo.kmax, float(htol), ptr(scratch), ptr(self.rank))
            rank = self.rank.cpu().numpy()[:topo.nlr].astype(np.int64)
            lr = topo.part.lowrank
            su = lr[:, 1].astype(np.int64) * rank
            sv = lr[:, 3].astype(np.int64) * rank
            offU = np.concatenate([[0], np.cumsum(su)[:-1]]).astype(np.int64)
            offV = np.concatenate([[0], np.cumsum(sv)[:-1]]).astype(np.int64)
            offT = np.concatenate([[0], np.cumsum(rank)[:-1]]).astype(np.int64)
            tp = topo.vseg_count * rank
            offTP = np.concatenate([[0], np.cumsum(tp)[:-1]]).astype(np.int64)
            self.offTP = _i64(offTP, dev)
            self.tp_entries = int(tp.sum())
            self.rank_h = rank
            self.offU = _i64(offU, dev)
            self.offV = _i64(offV, dev)
            self.offT = _i64(offT, dev)
            self.U = torch.empty(max(1, 2 * int(su.sum())), dtype=torch.float32, device=dev)
            self.V = torch.empty(max(1, 2 * int(sv.sum())), dtype=torch.float32, device=dev)
            self.sum_rank = int(rank.sum())
            call('mnpb_hmat_compact', sh, topo.nlr, ptr(topo.lowrank), ptr(self.rank),
                 ptr(topo.scr_offU), ptr(topo.scr_offV), ptr(scratch), ptr(self.offU),
                 ptr(self.offV), ptr(self.U), ptr(self.V))
            self.rent = _records(row_records(topo, rank, offU, offT), dev)
            self.vent = _records(vtx_records(topo, rank, offV, offTP), dev)
        else:
            self.rank_h = np.zeros(0, np.int64)
            z = _i64(np.zeros(1), dev)
            self.offU = self.offV = self.offT = self.offTP = z
            self.tp_entries = 0
            self.U = self.V = torch.empty(2, dtype=torch.float32, device=dev)
            self.sum_rank = 0
            zr = np.zeros(0, np.int64)
            self.rent = _records(row_records(topo, zr, zr, zr), dev)
            self.vent = _records(vtx_records(topo, zr, zr, zr), dev)
        self.scratch = scratch

    def stored_bytes(self):
        """Bytes read by one product (complex64 dense blocks and factors)."""
        return 4 * (self.D.numel() + self.U.numel() + self.V.numel()) if self.topo.nlr else \
            4 * self.D.numel()

    def compression(self):
        n = self.topo.n
        return (self.topo.dense_entries + self.U.numel() // 2 + self.V.numel() // 2) / float(n * n)

    def factors(self, b):
        """(U, V) of low-rank block b as complex128 numpy arrays (for tests)."""
        r = int(self.rank_h[b])
        m, k = int(self.topo.part.lowrank[b, 1]), int(self.topo.part.lowrank[b, 3])
        ou = int(self.offU[b].item())
        ov = int(self.offV[b].item())
        U = self.U[2 * ou:2 * (ou + m * r)].double().cpu().numpy().view(complex)
        V = self.V[2 * ov:2 * (ov + k * r)].double().cpu().numpy().view(complex)
        return U.reshape(r, m).T, V.reshape(k, r)       # V is stored transposed


def hmat_matvec(hms, xs, ys, nc, stream=None):
    """ys[i] = hms[i] @ xs[i] for up to 4 H-matrices of one topology; x, y are
    complex128 (nc, n) tensors (column c contiguous) in face order."""
    if not 1 <= len(hms) <= 4:
        raise ValueError("hmat_matvec: 1 to 4 matrices per call")
    topo = hms[0].topo
    dev = topo.device
    n = topo.n
    # one V^T x scratch per matrix (the matrices run in the same launch)
    per = 2 * max(1, max(h.sum_rank for h in hms)) * min(nc, 4)
    T = torch.empty(per * len(hms), dtype=torch.float64, device=dev)
    pxc = 2 * n * min(nc, 4)
    Xc = torch.empty(pxc * len(hms), dtype=torch.float64, device=dev)
    partial = torch.empty(len(hms) * topo.nitem * 32 * 4 * 2, dtype=torch.float64, device=dev)
    ptp = 2 * 4 * max(1, max(h.tp_entries for h in hms))
    TP = torch.empty(ptp * len(hms), dtype=torch.float64, device=dev)
    desc = np.zeros((len(hms), 13), dtype=np.uint64)
    keep = []
    for i, (h, x, y) in enumerate(zip(hms, xs, ys)):
        if h.topo is not topo:
            raise ValueError("hmat_matvec: all matrices must share one topology")
        if x.dtype != torch.complex128 or y.dtype != torch.complex128 or not x.is_contiguous() \
                or not y.is_contiguous() or x.numel() < n * nc or y.numel() < n * nc:
            raise ValueError("hmat_matvec: x, y must be contiguous complex128 (nc, n)")
        desc[i] = [h.D.data_ptr(), h.U.data_ptr(), h.V.data_ptr(), h.rank.data_ptr(),
                   h.offT.data_ptr(), x.data_ptr(), y.data_ptr(), T[i * per:].data_ptr(),
                   Xc[i * pxc:].data_ptr(), h.offTP.data_ptr(), TP[i * ptp:].data_ptr(),
                   h.rent.data_ptr(), h.vent.data_ptr()]
        keep.append((x, y))
    call('mnpb_hmat_matvec', _lib.stream_handle(stream), n, nc, len(hms), ptr(desc),
         ptr(topo.c2p), topo.nlr, topo.nchunk, ptr(topo.chunks), ptr(topo.leaf_rows),
         topo.nitem, ptr(topo.items), ptr(topo.cptr), ptr(partial), topo.nvitem,
         ptr(topo.vptr))
    return ys
