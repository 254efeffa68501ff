"""Cluster tree and block partition of the H-matrix solver (host side).

Restates, with the same node numbering and index maps, the reference's
``ClusterTree`` (mnpbem/greenfun/clustertree.py:13-148): recursive bisection
of the face centroids along the longest bounding-box axis
(``pos[:, k] < mid`` goes to the first son), a particle split first when a
cluster holds faces of several particles, leaves of at most ``cleaf`` faces.
Node ``i`` covers cluster positions ``cind[i, 0]..cind[i, 1]``; ``ind[:, 0]``
maps cluster position -> face, ``ind[:, 1]`` face -> cluster position.

The block partition is ``ClusterTree.admissibility`` (clustertree.py:304-376):
a pair of nodes is a dense block (2) when both are leaves, a low-rank block (1)
when both lie in one particle and the admissibility predicate holds, and is
otherwise split into the sons' pairs.  The wavenumber-aware predicate is
mnpbem/greenfun/hmatrix.py:1284-1311.  Blocks come out in the reference's
depth-first order.

Tree and partition are integer-exact against the reference (the boxes use the
same NumPy min/max/norm operations on the same arrays).  They are built once
per geometry; everything per wavelength runs on the GPU.
"""

import numpy as np


class ClusterTree(object):
    """Bisection cluster tree over face centroids ``pos`` (n, 3)."""

    def __init__(self, pos, cleaf=32, ipart_arr=None):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.n = self.pos.shape[0]
        if ipart_arr is None:
            self._ipart_arr = np.zeros(self.n, dtype=np.int64)
        else:
            self._ipart_arr = np.asarray(ipart_arr, dtype=np.int64)
        self.cleaf = int(cleaf)
        self._build()

    # -- construction --------------------------------------------------------
    def _box(self, ind):
        p = self.pos[ind]
        lo = p.min(axis=0)
        hi = p.max(axis=0)
        return 0.5 * (lo + hi), 0.5 * np.linalg.norm(hi - lo)

    def _split(self, ind):
        ip = self._ipart_arr[ind]
        if np.unique(ip).size > 1:
            first = ip == ip[0]
            return ind[first], ind[~first], True
        p = self.pos[ind]
        lo = p.min(axis=0)
        hi = p.max(axis=0)
        ext = hi - lo
        k = int(np.argmax(ext))
        cut = lo[k] + 0.5 * ext[k]
        low = self.pos[ind, k] < cut
        a, b = ind[low], ind[~low]
        if a.size == 0:
            a, b = ind[:1], ind[1:]
        elif b.size == 0:
            a, b = ind[:-1], ind[-1:]
        return a, b, False

    def _build(self):
        n = self.n
        start, end, mids, rads, sons = [0], [n - 1], [], [], [[-1, -1]]
        m, r = self._box(np.arange(n))
        mids.append(m)
        rads.append(r)
        c2p = np.empty(n, dtype=np.int64)
        # explicit stack; the first son's subtree is numbered before the
        # second son's, as in the recursive reference
        stack = [(0, np.arange(n, dtype=np.int64), 0)]
        while stack:
            node, ind, c0 = stack.pop()
            s1 = len(start)
            sons[node] = [s1, s1 + 1]
            a, b, psplit = self._split(ind)
            todo = []
            for ix, (part, cs) in enumerate(((a, c0), (b, c0 + a.size))):
                start.append(cs)
                end.append(cs + part.size - 1)
                m, r = self._box(part)
                mids.append(m)
                rads.append(r)
                sons.append([-1, -1])
                if part.size > self.cleaf or psplit:
                    todo.append((s1 + ix, part, cs))
                else:
                    c2p[cs:cs + part.size] = part
            for t in reversed(todo):
                stack.append(t)
        self.son = np.asarray(sons, dtype=np.int64)
        self.cind = np.stack([np.asarray(start, dtype=np.int64),
                              np.asarray(end, dtype=np.int64)], axis=1)
        self.mid = np.asarray(mids, dtype=np.float64)
        self.rad = np.asarray(rads, dtype=np.float64)
        p2c = np.empty(n, dtype=np.int64)
        p2c[c2p] = np.arange(n, dtype=np.int64)
        self.ind = np.stack([c2p, p2c], axis=1)
        ip0 = self._ipart_arr[c2p[self.cind[:, 0]]]
        ip1 = self._ipart_arr[c2p[self.cind[:, 1]]]
        self.ipart = np.where(ip0 == ip1, ip0, -1).astype(np.int64)

    # -- queries ---------------------------------------------------------------
    @property
    def nnodes(self):
        return self.son.shape[0]

    def is_leaf(self, i):
        return self.son[i, 0] == -1

    def cluster_size(self, i):
        return int(self.cind[i, 1] - self.cind[i, 0] + 1)

    def leaves(self):
        return np.nonzero(self.son[:, 0] == -1)[0]

    def part2cluster(self, v):
        return v[self.ind[:, 0]]

    def cluster2part(self, v):
        return v[self.ind[:, 1]]

    # -- block partition -------------------------------------------------------
    def admissibility(self, fadmiss=None):
        """Ordered block partition: list of ((i1, i2), 1 | 2) as the reference's
        dictionary (clustertree.py:304-376)."""
        if fadmiss is None:
            fadmiss = make_kaware_fadmiss(None)
        out = []
        stack = [(0, 0)]
        while stack:
            i1, i2 = stack.pop()
            leaf1, leaf2 = self.son[i1, 0] == -1, self.son[i2, 0] == -1
            if leaf1 and leaf2:
                out.append(((i1, i2), 2))
                continue
            if self.ipart[i1] != -1 and self.ipart[i2] != -1:
                dist = np.linalg.norm(self.mid[i1] - self.mid[i2])
                if fadmiss(self.rad[i1], self.rad[i2], dist):
                    out.append(((i1, i2), 1))
                    continue
            kids1 = [i1] if leaf1 else [int(self.son[i1, 0]), int(self.son[i1, 1])]
            kids2 = [i2] if leaf2 else [int(self.son[i2, 0]), int(self.son[i2, 1])]
            pairs = [(a, b) for a in kids1 for b in kids2]
            for pr in reversed(pairs):
                stack.append(pr)
        return out


def make_kaware_fadmiss(k, eta0=2.5):
    """Admissibility predicate of mnpbem/greenfun/hmatrix.py:1284-1311:
    eta0 * min(rad) < dist, and, once k * min(rad) > 1, also dist >= 2 pi / k."""
    if k is None or not np.isfinite(k) or abs(k) < 1e-12:
        return lambda r1, r2, d: eta0 * min(r1, r2) < d
    k_abs = abs(complex(k))
    wavelength = 2.0 * np.pi / k_abs

    def fadmiss(r1, r2, d):
        rmin = min(r1, r2)
        if eta0 * rmin >= d:
            return False
        if k_abs * rmin > 1.0 and d < wavelength:
            return False
        return True
    return fadmiss


class BlockPartition(object):
    """Dense and low-rank blocks of a tree, as integer arrays.

    ``row1/col1`` (dense) and ``row2/col2`` (low-rank) are tree nodes in the
    reference's order; ``dense`` / ``lowrank`` are (nblk, 4) int32 arrays of
    (row start, rows, col start, cols) in cluster positions.
    """

    def __init__(self, tree, fadmiss=None):
        self.tree = tree
        blocks = tree.admissibility(fadmiss)
        self.row1 = np.array([b[0][0] for b in blocks if b[1] == 2], dtype=np.int64)
        self.col1 = np.array([b[0][1] for b in blocks if b[1] == 2], dtype=np.int64)
        self.row2 = np.array([b[0][0] for b in blocks if b[1] == 1], dtype=np.int64)
        self.col2 = np.array([b[0][1] for b in blocks if b[1] == 1], dtype=np.int64)
        self.dense = self._rect(self.row1, self.col1)
        self.lowrank = self._rect(self.row2, self.col2)

    def _rect(self, rows, cols):
        c = self.tree.cind
        out = np.zeros((rows.size, 4), dtype=np.int32)
        if rows.size:
            out[:, 0] = c[rows, 0]
            out[:, 1] = c[rows, 1] - c[rows, 0] + 1
            out[:, 2] = c[cols, 0]
            out[:, 3] = c[cols, 1] - c[cols, 0] + 1
        return out

    def key(self):
        """Hashable identity of the partition (equal partitions share device
        structures)."""
        return (self.row1.tobytes(), self.col1.tobytes(), self.row2.tobytes(),
                self.col2.tobytes())
