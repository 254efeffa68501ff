"""CPU oracle for the H-matrix / GMRES path -- TEST INFRASTRUCTURE ONLY.

NumPy/SciPy restatement of the reference's partially-pivoted ACA
(mnpbem/greenfun/hmatrix.py:195-336), H-matrix times vector
(hmatrix.py:450-541) and the BEMRetIter GMRES call
(mnpbem/bem/bem_iter.py:45-101, bem_ret_iter.py:1362-1501), in FP64.  Only
``tests/`` import it; the product (``mnpbem_b200``) never does.  Its ACA is
pinned against ranks, factors and block errors that
``tests/golden/make_golden_hmat.py`` recorded from the reference.
"""

import numpy as np
import scipy.sparse.linalg as spla


def _margin(a):
    """Relative gap between the largest and second-largest entry of a (the
    closeness of an argmax decision; 1 if there is no runner-up)."""
    if a.size < 2:
        return 1.0
    top = np.partition(a, -2)[-2:]
    return float((top[1] - top[0]) / top[1]) if top[1] > 0 else 1.0


def aca_block(fun_row, fun_col, m, n, htol, kmax, diag=None):
    """Partially-pivoted ACA of one m x n block (hmatrix.py:195-336).

    fun_row(i) -> row i (n,), fun_col(j) -> column j (m,) of the block.
    Returns U (m, r), V (n, r) with block ~ U V^T, and the pivots.  If
    ``diag`` is a list, one dict per step is appended to it: the stop-test
    ratio sqrt(new) / (htol sqrt(fro)) (the block stops once it is < 1) and
    the relative margins of the column and row pivot choices -- how close
    each decision was, for explaining a rank that differs under other
    rounding.
    """
    max_rank = min(m, n, kmax)
    U = np.empty((m, max_rank), dtype=complex)
    V = np.empty((n, max_rank), dtype=complex)
    used_r = np.zeros(m, dtype=bool)
    used_c = np.zeros(n, dtype=bool)
    rank, prow, fro = 0, 0, 0.0
    pivots = []
    for _ in range(max_rank):
        row = np.array(fun_row(prow), dtype=complex)
        for j in range(rank):                       # row -= U[prow, j] V[:, j]
            row -= U[prow, j] * V[:, j]
        a = np.abs(row)
        a[used_c] = 0.0
        pcol = int(np.argmax(a))
        step = {'col_margin': _margin(a)}
        if diag is not None:
            diag.append(step)
        piv = row[pcol]
        if np.abs(piv) < 1e-15:
            break
        col = np.array(fun_col(pcol), dtype=complex)
        for j in range(rank):                       # col -= V[pcol, j] U[:, j]
            col -= V[pcol, j] * U[:, j]
        u = col / piv
        U[:, rank] = u
        V[:, rank] = row
        rank += 1
        used_r[prow] = True
        used_c[pcol] = True
        pivots.append((prow, pcol))
        new = np.vdot(u, u).real * np.vdot(row, row).real
        cross = 0.0
        for j in range(rank - 1):
            cross += 2.0 * (np.vdot(U[:, j], u) * np.vdot(V[:, j], row)).real
        fro += new + cross
        step['stop_ratio'] = (np.sqrt(new) / (htol * np.sqrt(abs(fro)))) if fro > 0 else np.inf
        if fro > 0 and np.sqrt(new) < htol * np.sqrt(abs(fro)):
            break
        a = np.abs(u)
        a[used_r] = 0.0
        prow = int(np.argmax(a))
        step['row_margin'] = _margin(a)
    if rank == 0:
        return np.zeros((m, 1), complex), np.zeros((n, 1), complex), pivots
    return U[:, :rank].copy(), V[:, :rank].copy(), pivots


class HMatrixOracle(object):
    """H-matrix of a dense matrix A (particle order) over a cluster tree and
    block partition (mnpbem_b200.clustertree objects or equivalents)."""

    def __init__(self, A, tree, part, htol=1e-6, kmax=100):
        self.tree, self.part = tree, part
        c2p = tree.ind[:, 0]
        self.dense = []
        for r0, m, c0, k in part.dense:
            self.dense.append(A[np.ix_(c2p[r0:r0 + m], c2p[c0:c0 + k])])
        self.U, self.V, self.pivots, self.diag = [], [], [], []
        for r0, m, c0, k in part.lowrank:
            rows, cols = c2p[r0:r0 + m], c2p[c0:c0 + k]
            dg = []
            U, V, piv = aca_block(lambda i: A[rows[i], cols], lambda j: A[rows, cols[j]],
                                  m, k, htol, kmax, diag=dg)
            self.U.append(U)
            self.V.append(V)
            self.pivots.append(piv)
            self.diag.append(dg)

    def near_tie(self, i, rank_other, tol=1e-9):
        """Why block i could end at rank_other under other rounding: a stop
        test within tol of its threshold, or a pivot choice whose top two
        candidates are within tol, at or before the step where the two
        ranks part.  Returns a description, or None if nothing explains it."""
        dg = self.diag[i]
        upto = min(len(dg), max(rank_other, self.U[i].shape[1]))
        for s, st in enumerate(dg[:upto]):
            r = st.get('stop_ratio')
            if r is not None and np.isfinite(r) and abs(r - 1.0) < tol:
                return 'stop test at step %d within %.1e of its threshold' % (s + 1, abs(r - 1))
            for key in ('col_margin', 'row_margin'):
                if st.get(key, 1.0) < tol:
                    return '%s pivot at step %d: top two candidates %.1e apart' % (
                        key.split('_')[0], s + 1, st[key])
        return None

    def ranks(self):
        return np.array([u.shape[1] for u in self.U], dtype=np.int64)

    def matvec(self, x):
        """H x for x (n,) or (n, c) in particle order (hmatrix.py:450-541)."""
        c2p, p2c = self.tree.ind[:, 0], self.tree.ind[:, 1]
        xc = x[c2p]
        y = np.zeros_like(xc, dtype=complex)
        for (r0, m, c0, k), D in zip(self.part.dense, self.dense):
            y[r0:r0 + m] += D @ xc[c0:c0 + k]
        for (r0, m, c0, k), U, V in zip(self.part.lowrank, self.U, self.V):
            y[r0:r0 + m] += U @ (V.T @ xc[c0:c0 + k])
        return y[p2c]


def afun_packed(mv1, mv2, mh1, mh2, eps1, eps2, k, nvec, x):
    """The packed 8N operator (bem_ret_iter.py:1362-1501, scalar eps) for one
    polarisation: x = [sig1, h1 (n x 3, column-major), sig2, h2] ->
    [phi, a, De, alpha]; mv*/mh* apply G1, G2, H1, H2 to (n, c) blocks."""
    n = nvec.shape[0]
    v1 = x[:4 * n].reshape(n, 4, order='F')
    v2 = x[4 * n:].reshape(n, 4, order='F')
    g1, g2, q1, q2 = mv1(v1), mv2(v2), mh1(v1), mh2(v2)
    phi = g1[:, 0] - g2[:, 0]
    a = g1[:, 1:] - g2[:, 1:]
    gs = eps1 * g1[:, 0] - eps2 * g2[:, 0]
    gh = eps1 * g1[:, 1:] - eps2 * g2[:, 1:]
    alpha = q1[:, 1:] - q2[:, 1:] - 1j * k * nvec * gs[:, None]
    De = eps1 * q1[:, 0] - eps2 * q2[:, 0] - 1j * k * np.sum(nvec * gh, axis=1)
    return np.concatenate([phi, a.ravel(order='F'), De, alpha.ravel(order='F')])


def gmres_solve(op, b, tol, maxit, x0=None):
    """scipy GMRES as the reference calls it (bem_iter.py:79-89): restart =
    min(n, maxit), rtol = tol.  Returns x, relres = |A x - b| / |b| and the
    number of operator applications."""
    n = b.size
    count = [0]

    def mv(v):
        count[0] += 1
        return op(v)

    A = spla.LinearOperator((n, n), matvec=mv, dtype=complex)
    x, flag = spla.gmres(A, b, x0=x0, rtol=tol, maxiter=maxit, restart=min(n, maxit))
    r = op(x) - b
    return x, np.linalg.norm(r) / np.linalg.norm(b), count[0], flag
