"""CPU oracle for the BEM hot path -- TEST INFRASTRUCTURE ONLY.

A plain NumPy/SciPy restatement of the reference's (PyMNPBEM) retarded and
quasistatic boundary-element solve, used as the checker for the CUDA path:
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm import it.  The product (``mnpbem_b200``) never calls it.

Parity of this oracle with the reference itself is pinned by
``tests/test_oracle_golden.py`` against fixtures that
``tests/golden/make_golden.py`` wrote by running the reference.

Each function names the reference code it restates (file:line within the
reference project).  Face geometry comes from ``mnpbem_b200.geometry`` (or
any object with the same attributes); the geometry module is itself pinned
bit-exactly against the reference by the golden tests.
"""

import math

import numpy as np
import scipy.linalg as sla

EPS = np.finfo(float).eps
EV2NM = 1.0 / 8.0655477e-4          # mnpbem/utils/constants.py:9
ORDER = 5                            # refinement order, mnpbem/greenfun/compgreen_ret.py:184


# --------------------------------------------------------------------------
# materials (mnpbem/materials/eps_drude.py:73-107, eps_const.py:48-72)
# --------------------------------------------------------------------------

def eps_drude(eps0, wp, gammad, enei):
    w = EV2NM / np.asarray(enei, dtype=float)
    eps = eps0 - wp ** 2 / (w * (w + 1j * gammad))
    return eps, 2 * np.pi / enei * np.sqrt(eps)


def eps_const(val, enei):
    e = complex(val)
    return e, 2 * np.pi / enei * np.sqrt(e)


# --------------------------------------------------------------------------
# near-pair classification (mnpbem/greenfun/refine_utils.py:12-158)
# --------------------------------------------------------------------------

def pdist2_algebraic(p1, p2):
    """d = sqrt(|p1|^2 + |p2|^2 - 2 p1.p2) with d^2 < 1e-10 -> 0 (refine_utils.py:12-26)."""
    n1 = np.sum(p1 * p1, axis=1)
    n2 = np.sum(p2 * p2, axis=1)
    d2 = n1[:, None] + n2[None, :] - 2.0 * (p1 @ p2.T)
    d2[d2 < 1e-10] = 0.0
    return np.sqrt(d2)


def refinematrix(pos1, pos2, rad1, rad2, abs_cutoff=0.0, rel_cutoff=3.0):
    """Dense int matrix: 2 self (d == 0), 1 near, 0 far (refine_utils.py:29-158)."""
    d = pdist2_algebraic(pos1, pos2)
    d2 = d - rad2[None, :]
    idr = d2 / rad1[:, None]
    ir = np.zeros(d.shape, dtype=np.int8)
    ir[((d2 < abs_cutoff) | (idr < rel_cutoff)) & (d != 0)] = 1
    ir[d == 0] = 2
    return ir


# --------------------------------------------------------------------------
# refined retarded Green function coefficients
# (mnpbem/greenfun/greenret_refined.py:78-516)
# --------------------------------------------------------------------------

def refined_coefficients(p, ir, order=ORDER):
    """Taylor coefficients in (ik) for refined pairs, deriv='cart'.

    Returns rows, cols (CSR order), g (n_ref, order+1) c128,
    f (n_ref, 3, order+1) c128.  Self pairs use the polar quadrature
    (greenret_refined.py:122-285), near pairs the face quadrature with the
    centroid distance r0 subtracted (greenret_refined.py:287-516).  Faces are
    processed in batches of equal point count with the reference's operation
    order (incremental powers, einsum contractions, row sums).
    """
    rows, cols = np.nonzero(ir)
    nref = len(rows)
    g = np.zeros((nref, order + 1), dtype=complex)
    f = np.zeros((nref, 3, order + 1), dtype=complex)
    fact = [math.factorial(n) for n in range(order + 1)]
    kind = ir[rows, cols]

    # ---- self pairs: polar integration (greenret_refined.py:166-248)
    sel = np.where(kind == 2)[0]
    if len(sel):
        qpos, qw, qrow = p.quadpol(cols[sel])
        counts = np.bincount(qrow, minlength=len(sel))
        for cnt in np.unique(counts):
            grp = np.where(counts == cnt)[0]
            pts = np.concatenate([np.where(qrow == k)[0] for k in grp])
            pos2d = qpos[pts].reshape(len(grp), cnt, 3)
            w2d = qw[pts].reshape(len(grp), cnt)
            iref = sel[grp]
            fi = rows[iref]
            pos1, nvec1 = p.pos[fi], p.nvec[fi]
            vec = pos1[:, None, :] - pos2d
            r = np.sqrt((vec * vec).sum(axis=2))
            r = np.maximum(r, EPS)
            ndr = np.einsum('ij,ikj->ik', nvec1, vec)
            inv_r = 1.0 / r
            inv_r2 = inv_r * inv_r
            inv_r3 = inv_r * inv_r2
            rp1 = inv_r.copy()
            for n in range(order + 1):
                g[iref, n] = (w2d * rp1).sum(axis=1) / fact[n]
                rp1 = rp1 * r
            rr = np.maximum(r, 1e-4 * r.max(axis=1)[:, None])
            inv_rr3 = 1.0 / (rr * rr * rr)
            t1, t2 = p.tvec1[fi], p.tvec2[fi]
            in1 = np.einsum('ij,ikj->ik', t1, vec)
            in2 = np.einsum('ij,ikj->ik', t2, vec)
            rp3 = inv_r3.copy()
            rpn = np.ones_like(r)
            for n in range(order + 1):
                f1 = (w2d * (n - 1) * ndr * rp3).sum(axis=1) / fact[n]
                f2 = (w2d * (n - 1) * in1 * rpn * inv_rr3).sum(axis=1) / fact[n]
                f3 = (w2d * (n - 1) * in2 * rpn * inv_rr3).sum(axis=1) / fact[n]
                f[iref, :, n] = nvec1 * f1[:, None] + t1 * f2[:, None] + t2 * f3[:, None]
                rp3 = rp3 * r
                rpn = rpn * r

    # ---- near pairs: face quadrature of the column face (greenret_refined.py:336-442)
    sel = np.where(kind == 1)[0]
    if len(sel):
        ucols = np.unique(cols[sel])
        qpos, qw, qrow = p.quad(ucols)
        order_perm = np.argsort(qrow, kind='stable')
        qpos, qw, qrow = qpos[order_perm], qw[order_perm], qrow[order_perm]
        counts = np.bincount(qrow, minlength=len(ucols))
        starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
        colpos = np.full(p.pos.shape[0], -1)
        colpos[ucols] = np.arange(len(ucols))
        fc = colpos[cols[sel]]
        for cnt in np.unique(counts[fc]):
            m = counts[fc] == cnt
            iref = sel[m]
            fcm = fc[m]
            idx = starts[fcm][:, None] + np.arange(cnt)[None, :]
            pos_face = qpos[idx]
            w = qw[idx]
            src = rows[iref]
            rvec = p.pos[src][:, None, :] - pos_face
            x, y, zz = rvec[..., 0], rvec[..., 1], rvec[..., 2]
            r = np.sqrt((rvec * rvec).sum(axis=2))
            r = np.maximum(r, EPS)
            vec0 = p.pos[cols[iref]] - p.pos[src]
            r0 = np.sqrt((vec0 * vec0).sum(axis=1))
            dl = r - r0[:, None]
            inv_r = 1.0 / r
            inv_r2 = inv_r * inv_r
            inv_r3 = inv_r2 * inv_r
            dpn = np.ones_like(r)
            for n in range(order + 1):
                g[iref, n] = (dpn * inv_r / fact[n] * w).sum(axis=1)
                dpn = dpn * dl
            fs0 = -inv_r3
            f[iref, 0, 0] = (x * fs0 * w).sum(axis=1)
            f[iref, 1, 0] = (y * fs0 * w).sum(axis=1)
            f[iref, 2, 0] = (zz * fs0 * w).sum(axis=1)
            dpn = dl.copy()
            dpm = np.ones_like(r)
            for n in range(1, order + 1):
                fsc = -dpn * inv_r3 / fact[n] + dpm * inv_r2 / fact[n - 1]
                f[iref, 0, n] = (x * fsc * w).sum(axis=1)
                f[iref, 1, n] = (y * fsc * w).sum(axis=1)
                f[iref, 2, n] = (zz * fsc * w).sum(axis=1)
                dpm = dpn
                dpn = dpn * dl
    return rows, cols, g, f


# --------------------------------------------------------------------------
# quasistatic Green function with refinement
# (mnpbem/greenfun/compgreen_stat.py:219-464, _numba_kernels.py:32-68)
# --------------------------------------------------------------------------

def static_GF(p, ir):
    """Refined static G = a/d and F = -n.r a/d^3 (no closure correction).

    Far part as in _numba_kernels.py:32-68 (self pairs zeroed), self pairs by
    the polar rule and near pairs by the face rule as in
    compgreen_stat.py:340-416, with the same reductions (bincount, dot).
    """
    pos, nvec, area = p.pos, p.nvec, p.area
    rx = pos[:, 0:1] - pos[None, :, 0]
    ry = pos[:, 1:2] - pos[None, :, 1]
    rz = pos[:, 2:3] - pos[None, :, 2]
    d = np.sqrt(rx * rx + ry * ry + rz * rz)
    d = np.maximum(d, 2.220446049250313e-16)
    G = area[None, :] / d
    ndotr = nvec[:, 0:1] * rx + nvec[:, 1:2] * ry + nvec[:, 2:3] * rz
    F = -ndotr * area[None, :] / (d * d * d)
    np.fill_diagonal(G, 0.0)
    np.fill_diagonal(F, 0.0)
    drows, dcols = np.where(ir == 2)
    if len(drows):
        qpos, qw, qrow = p.quadpol(dcols)
        vec = pos[drows[qrow]] - qpos
        r = np.maximum(np.linalg.norm(vec, axis=1), EPS)
        nd = len(drows)
        G[drows, dcols] = np.bincount(qrow, weights=qw / r, minlength=nd)[:nd]
        ndv = np.sum(vec * nvec[drows[qrow]], axis=1)
        F[drows, dcols] = -np.bincount(qrow, weights=qw * ndv / (r ** 3), minlength=nd)[:nd]
    near = ir == 1
    ucols = np.unique(np.where(near)[1])
    if len(ucols):
        qpos, qw, qrow = p.quad(ucols)
        for k, face2 in enumerate(ucols):
            nb = np.where(near[:, face2])[0]
            m = qrow == k
            q, w = qpos[m], qw[m]
            vec = pos[nb, None, :] - q[None, :, :]
            r = np.maximum(np.linalg.norm(vec, axis=2), EPS)
            G[nb, face2] = (1.0 / r) @ w
            ndv = np.sum(nvec[nb, None, :] * vec, axis=2)
            F[nb, face2] = -(ndv / (r ** 3)) @ w
    return G, F


def closure_sums(area, F, groups):
    """f_j = sum_i a_i F_ij / a_j over each closed surface (compgreen_ret.py:302-356)."""
    f = np.zeros(len(area))
    for grp in groups:
        if grp is None:
            continue
        _, loc = grp
        sub = F[np.ix_(loc, loc)]
        f[loc] = np.sum(area[loc][:, None] * sub / area[loc][None, :], axis=0)
    return f


# --------------------------------------------------------------------------
# retarded Green function matrices (greenret_refined.py:654-810)
# --------------------------------------------------------------------------

class RetGreen(object):
    """Refinement tables + closure for one (single-region-pair) surface."""

    def __init__(self, p, rel_cutoff=3.0, abs_cutoff=0.0):
        self.p = p
        self.ir = refinematrix(p.pos, p.pos, p.bradius(), p.bradius(), abs_cutoff, rel_cutoff)
        self.rows, self.cols, self.g, self.f = refined_coefficients(p, self.ir)
        _, Fs = static_GF(p, self.ir)
        groups = p.closed_groups() if hasattr(p, 'closed_groups') else [(1.0, np.arange(p.n))]
        fsum = closure_sums(p.area, Fs, groups)
        self.Fstat = Fs
        self.fclosure = fsum
        # closure correction -2 pi dir - f on the self pairs (compgreen_ret.py:376-400)
        corr = np.zeros(p.n)
        for grp in groups:
            if grp is None:
                continue
            dirv, loc = grp
            corr[loc] = -2 * np.pi * dirv - fsum[loc]
        self.corr = corr
        diag = self.rows == self.cols
        self.f[diag, :, 0] += corr[self.rows[diag], None] * p.nvec[self.rows[diag]]
        x = p.pos[:, None, :] - p.pos[None, :, :]
        d = np.sqrt((x * x).sum(axis=2))
        d = np.maximum(d, EPS)
        np.fill_diagonal(d, EPS)
        self.x = x
        self.d = d

    def GF(self, k):
        """(G, F) at complex wavenumber k, with the refined overlay and phase."""
        p = self.p
        d, x = self.d, self.x
        inv_d = 1.0 / d
        area = p.area
        ikp = np.array([(1j * k) ** n for n in range(ORDER + 1)])
        G = inv_d * area[None, :] + 0j
        G[self.rows, self.cols] = self.g @ ikp
        faux = (1j * k - inv_d) * inv_d * inv_d
        xx = x                                   # x_ii = 0 on the diagonal
        F = (p.nvec[:, 0:1] * (faux * xx[:, :, 0]) + p.nvec[:, 1:2] * (faux * xx[:, :, 1]) +
             p.nvec[:, 2:3] * (faux * xx[:, :, 2])) * area[None, :]
        F[self.rows, self.cols] = np.einsum('ij,ijk,k->i', p.nvec[self.rows], self.f, ikp)
        ph = np.exp(1j * k * d)
        return G * ph, F * ph


# --------------------------------------------------------------------------
# BEMRet (mnpbem/bem/bem_ret.py:293-525, 1360-1831)
# --------------------------------------------------------------------------

def bemret_matrices(green, eps_in, eps_out, k_in, k_out, enei):
    """G1, G2, H1, H2 for one closed particle in a single host medium.

    Region pairs with con > 0 are (inside,inside)@k_in and
    (outside,outside)@k_out; cross terms vanish (compgreen_ret.py:739-858).
    """
    G1, F1 = green.GF(k_in)
    G2, F2 = green.GF(k_out)
    n = G1.shape[0]
    H1 = F1 + 2 * np.pi * np.eye(n)
    H2 = F2 - 2 * np.pi * np.eye(n)
    return G1, G2, H1, H2


class BEMRetOracle(object):
    """Dense FP64 retarded solve, same algebra as bem_ret.py:411-523."""

    def __init__(self, green, eps_funcs, inout):
        self.green = green
        self.eps_funcs = eps_funcs
        self.inout = inout

    def init(self, enei):
        p = self.green.p
        e_in, k_in = self.eps_funcs[self.inout[0] - 1](enei)
        e_out, k_out = self.eps_funcs[self.inout[1] - 1](enei)
        self.enei = enei
        self.k = 2 * np.pi / enei
        self.eps1, self.eps2 = e_in, e_out
        G1, G2, H1, H2 = bemret_matrices(self.green, e_in, e_out, k_in, k_out, enei)
        self.G1, self.G2, self.H1, self.H2 = G1, G2, H1, H2
        n = G1.shape[0]
        self.G1_lu = sla.lu_factor(G1, check_finite=False)
        self.G2_lu = sla.lu_factor(G2, check_finite=False)
        G1i = sla.lu_solve(self.G1_lu, np.eye(n), check_finite=False)
        G2i = sla.lu_solve(self.G2_lu, np.eye(n), check_finite=False)
        self.L1, self.L2 = e_in, e_out
        self.Sigma1 = H1 @ G1i
        Sigma2 = H2 @ G2i
        self.Delta_lu = sla.lu_factor(self.Sigma1 - Sigma2, check_finite=False)
        Deltai = sla.lu_solve(self.Delta_lu, np.eye(n), check_finite=False)
        L = self.L1 - self.L2
        nn = p.nvec @ p.nvec.T
        Sigma = self.Sigma1 * self.L1 - Sigma2 * self.L2 + self.k ** 2 * L * (Deltai * nn) * L
        self.Sigma_lu = sla.lu_factor(Sigma, check_finite=False)
        return self

    def excitation(self, a1, a1p, a2, a2p):
        """phi, a, alpha, De for a vector-potential excitation (bem_ret.py:1360-1429)."""
        k = self.k
        nvec = self.green.p.nvec
        phi = np.zeros(a1.shape[0], dtype=complex) if a1.ndim == 2 else \
            np.zeros((a1.shape[0], a1.shape[2]), dtype=complex)
        a = a2 - a1
        alpha = a2p - a1p                        # phi1 = phi2 = 0 for a plane wave
        if a1.ndim == 2:
            De = -1j * k * (np.sum(nvec * a2, axis=1) * self.eps2 - np.sum(nvec * a1, axis=1) * self.eps1)
        else:
            De = -1j * k * (np.einsum('ij,ijk->ik', nvec, a2) * self.eps2 -
                            np.einsum('ij,ijk->ik', nvec, a1) * self.eps1)
        return phi, a, alpha, De

    def solve_vars(self, phi, a, alpha, De):
        """sig1, h1, sig2, h2 from (phi, a, alpha, De) (bem_ret.py:1690-1752)."""
        k = self.k
        nvec = self.green.p.nvec
        ls = lambda lu, b: sla.lu_solve(lu, b.reshape(b.shape[0], -1),
                                        check_finite=False).reshape(b.shape)
        multi = a.ndim == 3
        L1, L2 = self.L1, self.L2
        S1 = self.Sigma1
        if not multi:
            alpha_m = alpha - S1 @ a + 1j * k * (nvec * (L1 * phi)[:, None])
            De_m = De - S1 @ (L1 * phi) + 1j * k * np.sum(nvec * (L1 * a), axis=1)
            Ld = L1 - L2
            inner = np.sum(nvec * (Ld * ls(self.Delta_lu, alpha_m)), axis=1)
            sig2 = ls(self.Sigma_lu, De_m + 1j * k * inner)
            h2 = ls(self.Delta_lu, 1j * k * (nvec * (Ld * sig2)[:, None]) + alpha_m)
        else:
            npol = a.shape[2]
            n = a.shape[0]
            S1a = (S1 @ a.reshape(n, -1)).reshape(n, 3, npol)
            alpha_m = alpha - S1a + 1j * k * (nvec[:, :, None] * (L1 * phi)[:, None, :])
            De_m = De - S1 @ (L1 * phi) + 1j * k * np.einsum('ij,ijk->ik', nvec, L1 * a)
            Ld = L1 - L2
            inner = np.einsum('ij,ijk->ik', nvec, Ld * ls(self.Delta_lu, alpha_m))
            sig2 = ls(self.Sigma_lu, De_m + 1j * k * inner)
            h2 = ls(self.Delta_lu, 1j * k * nvec[:, :, None] * (Ld * sig2)[:, None, :] + alpha_m)
        sig1 = ls(self.G1_lu, sig2 + phi)
        h1 = ls(self.G1_lu, h2 + a)
        return sig1, h1, ls(self.G2_lu, sig2), ls(self.G2_lu, h2)

    def afun(self, sig1, h1, sig2, h2):
        """The packed 8N operator of mnpbem/bem/bem_ret_iter.py:1362-1501 (scalar eps).

        Returns (phi, a, De, alpha) with the same meaning as the excitation.
        """
        k = self.k
        nvec = self.green.p.nvec
        G1, G2, H1, H2 = self.G1, self.G2, self.H1, self.H2
        e1, e2 = self.eps1, self.eps2
        n = G1.shape[0]
        mv = lambda M, v: (M @ v.reshape(n, -1)).reshape(v.shape)
        phi = mv(G1, sig1) - mv(G2, sig2)
        a = mv(G1, h1) - mv(G2, h2)
        Gs = e1 * mv(G1, sig1) - e2 * mv(G2, sig2)
        Gh = e1 * mv(G1, h1) - e2 * mv(G2, h2)
        if h1.ndim == 2:
            alpha = mv(H1, h1) - mv(H2, h2) - 1j * k * nvec * Gs[:, None]
            De = e1 * mv(H1, sig1) - e2 * mv(H2, sig2) - 1j * k * np.sum(nvec * Gh, axis=1)
        else:
            alpha = mv(H1, h1) - mv(H2, h2) - 1j * k * nvec[:, :, None] * Gs[:, None, :]
            De = e1 * mv(H1, sig1) - e2 * mv(H2, sig2) - 1j * k * np.einsum('ij,ijk->ik', nvec, Gh)
        return phi, a, De, alpha


# --------------------------------------------------------------------------
# plane wave excitation and cross sections
# (mnpbem/simulation/planewave_ret.py:257-504, spectrum/spectrum_ret.py:231-459)
# --------------------------------------------------------------------------

def planewave_ret_potential(p, inout_faces, medium, eps_med, enei, pol, dirs):
    """a1, a1p, a2, a2p of shape (n, 3, npol) (planewave_ret.py:257-361)."""
    nb = np.sqrt(eps_med)
    k0 = 2 * np.pi / enei
    k = k0 * nb
    n = p.pos.shape[0]
    npol = pol.shape[0]
    out = []
    for side in (0, 1):
        a = np.zeros((n, 3, npol), dtype=complex)
        ap = np.zeros((n, 3, npol), dtype=complex)
        ind = np.where(inout_faces[:, side] == medium)[0]
        for i in range(npol):
            phase = np.exp(1j * k * p.pos[ind, :] @ dirs[i, :]) / (1j * k0)
            a[ind, :, i] = phase[:, None] * pol[i, :]
            ndd = p.nvec[ind, :] @ dirs[i, :]
            ap[ind, :, i] = (1j * k * ndd)[:, None] * phase[:, None] * pol[i, :]
        out += [a, ap]
    return out  # a1, a1p, a2, a2p


def farfield(p, inout_faces, medium, k, enei, sig1, h1, sig2, h2, dirs):
    """Far-field e, h (ndir, 3, npol) (spectrum_ret.py:231-392)."""
    k0 = 2 * np.pi / enei
    phase = np.exp(-1j * k * dirs @ p.pos.T) * p.area
    npol = sig1.shape[1]
    e = np.zeros((len(dirs), 3, npol), dtype=complex)
    h = np.zeros_like(e)
    for side, s, hh in ((0, sig1, h1), (1, sig2, h2)):
        ind = np.where(inout_faces[:, side] == medium)[0]
        if len(ind) == 0:
            continue
        ph = phase[:, ind]
        for ip in range(npol):
            ph_h = ph @ hh[ind, :, ip]
            ph_s = ph @ s[ind, ip]
            e[:, :, ip] += 1j * k0 * ph_h - 1j * k * dirs * ph_s[:, None]
            h[:, :, ip] += 1j * k * np.cross(dirs, ph_h)
    return e, h


def extinction(p, inout_faces, medium, k, enei, sol, pol, dirs):
    """4 pi / k Im(pol* . e_forward) (planewave_ret.py:437-504)."""
    sig1, h1, sig2, h2 = sol
    e, _ = farfield(p, inout_faces, medium, k, enei, sig1, h1, sig2, h2, dirs)
    npol = pol.shape[0]
    ext = np.array([np.imag(np.sum(np.conj(pol[i]) * e[i, :, i])) for i in range(npol)])
    return np.real(4 * np.pi / k * ext)


def scattering(p, inout_faces, medium, k, enei, sol, sphere_nvec, sphere_area, eps_med):
    """Radiated power over the 256-direction sphere / (0.5 n_b) (spectrum_ret.py:395-459)."""
    sig1, h1, sig2, h2 = sol
    e, h = farfield(p, inout_faces, medium, k, enei, sig1, h1, sig2, h2, sphere_nvec)
    npol = e.shape[2]
    dsca = np.zeros((len(sphere_nvec), npol))
    for ip in range(npol):
        pv = np.cross(e[:, :, ip], np.conj(h[:, :, ip]))
        dsca[:, ip] = 0.5 * np.real(np.sum(sphere_nvec * pv, axis=1))
    return (sphere_area @ dsca) / (0.5 * np.real(np.sqrt(eps_med)))


# --------------------------------------------------------------------------
# BEMStat (mnpbem/bem/bem_stat.py:241-404, 752-807;
#          mnpbem/simulation/planewave_stat.py:152-355)
# --------------------------------------------------------------------------

class BEMStatOracle(object):
    def __init__(self, p, rel_cutoff=3.0):
        ir = refinematrix(p.pos, p.pos, p.bradius(), p.bradius(), 0.0, rel_cutoff)
        _, F = static_GF(p, ir)
        groups = p.closed_groups() if hasattr(p, 'closed_groups') else [(1.0, np.arange(p.n))]
        f = closure_sums(p.area, F, groups)
        for grp in groups:
            if grp is None:
                continue
            dirv, loc = grp
            F[loc, loc] += -2 * np.pi * dirv - f[loc]
        self.p = p
        self.F = F

    def solve(self, eps1, eps2, phip):
        lam = 2 * np.pi * (eps1 + eps2) / (eps1 - eps2)
        M = -(np.diag(lam) + self.F)
        return sla.lu_solve(sla.lu_factor(M, check_finite=False), phip, check_finite=False)


def stat_cross_sections(p, sig, pol, k_med):
    """sca, abs, ext for the quasistatic dipole (planewave_stat.py:279-355)."""
    dip = (p.area[:, None] * p.pos).T @ sig
    k = np.real(k_med)
    sca = 8 * np.pi / 3 * k ** 4 * np.sum(np.abs(dip) ** 2, axis=0)
    absc = 4 * np.pi * k * np.imag(np.sum(pol * dip.T, axis=1))
    return np.real(sca), absc, np.real(sca) + absc
