"""Learned warm start for wavelength sweeps of the iterative solver.

A small per-face network corrects the quadratic extrapolation of the packed
BEM solution over the wavelength sweep:

    x_i ~ q_i + s2 * MLP(features),   q_i = 3 x_{i-1} - 3 x_{i-2} + x_{i-3},
                                      s2 = rms(x_{i-1} - 2 x_{i-2} + x_{i-3})

Features per (face, polarisation): face geometry, lambda_i, the inside
dielectric function at lambda_i .. lambda_{i-3}, the outside one at
lambda_i, log ratios of the history's difference scales, and x_{i-1},
x_{i-1} - x_{i-2}, x_{i-1} - 2 x_{i-2} + x_{i-3} at that face (each scaled
by its own rms).  Scaling the target by s2 makes the network learn the
relative extrapolation error, so it helps equally where the spectrum is
flat and where it bends.

It supplies the GMRES start vector and, with ``deflate=m``, the first
direction of a GCRO augmentation space {prediction, x_{i-1}, ..., x_{i-m}}
(``bem_iter.gmres(augment=...)``, m + 1 extra operator applications): GMRES
minimises the residual over that span and runs its Krylov space on the
operator deflated by it.  GMRES still converges to the same tolerance, so
the network changes the cost of a solve, never its answer; the zero-start
GMRES (or the dense LU) result judges its error.

Network: 4 dense layers (67 -> 256 -> 256 -> 256 -> 16), SiLU, bf16 weights
with FP32 accumulation, trained with Adam on the GPU by the kernels of
csrc/mlp.cu (mnpb_mlp_*), on solutions of the FP64 dense solver.  The
reference has no learned component.
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr

__all__ = ["MLP", "LearnedWarmStart", "face_geometry"]

NFEAT = 67
NOUT = 16
HISTORY = 3


class MLP(object):
    """Dense network with bf16 weights (FP32 master copy) on the GPU."""

    def __init__(self, sizes, device='cuda', seed=0, out_scale=0.01):
        self.sizes = list(sizes)
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)
        self.W, self.b = [], []
        for l, (fi, fo) in enumerate(zip(self.sizes[:-1], self.sizes[1:])):
            std = np.sqrt(2.0 / fi) * (out_scale if l == len(self.sizes) - 2 else 1.0)
            self.W.append(torch.from_numpy((rng.standard_normal((fo, fi)) * std)
                                           .astype(np.float32)).to(self.device))
            self.b.append(torch.zeros(fo, dtype=torch.float32, device=self.device))
        self.Wb = [torch.empty(w.shape, dtype=torch.bfloat16, device=self.device) for w in self.W]
        self._sync_bf16()
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.step = 0
        self._acts = self._pre = None

    def _sync_bf16(self):
        sh = _lib.stream_handle()
        for w, wb in zip(self.W, self.Wb):
            call('mnpb_mlp_to_bf16', sh, w.numel(), ptr(w), ptr(wb))

    def set_weights(self, Ws, bs):
        """Load FP32 weights (list of (out, in) arrays) and biases."""
        for l, (w, b) in enumerate(zip(Ws, bs)):
            self.W[l].copy_(torch.as_tensor(np.asarray(w, dtype=np.float32)))
            self.b[l].copy_(torch.as_tensor(np.asarray(b, dtype=np.float32)))
        self._sync_bf16()

    def forward(self, X, keep=False):
        """Outputs for rows X (rows x sizes[0], FP32 contiguous device)."""
        sh = _lib.stream_handle()
        rows = X.shape[0]
        acts, pre = [X], []
        for l, (wb, b) in enumerate(zip(self.Wb, self.b)):
            fo, fi = wb.shape
            Y = torch.empty((rows, fo), dtype=torch.float32, device=self.device)
            Z = torch.empty_like(Y) if keep else None
            last = l == len(self.Wb) - 1
            call('mnpb_mlp_gemm', sh, rows, fo, fi, ptr(acts[-1]), fi, 1, ptr(wb), 1, fi, 1,
                 ptr(Y), fo, 1, ptr(b), 2 if last else 1, ptr(Z) if keep else None, 1, None)
            acts.append(Y)
            pre.append(Z)
        if keep:
            self._acts, self._pre = acts, pre
        return acts[-1]

    def backward(self, dY):
        """Weight/bias gradients of the last forward(keep=True) pass."""
        sh = _lib.stream_handle()
        acts, pre = self._acts, self._pre
        rows = dY.shape[0]
        gW, gb = [None] * len(self.W), [None] * len(self.W)
        d = dY
        for l in range(len(self.W) - 1, -1, -1):
            fo, fi = self.W[l].shape
            if l == len(self.W) - 1:
                dz = d
            else:
                dz = torch.empty_like(d)
                call('mnpb_mlp_silu_back', sh, d.numel(), ptr(d), ptr(pre[l]), ptr(dz))
            nsplit = max(1, min(256, rows // 2048))
            work = torch.empty(nsplit * fo * fi if nsplit > 1 else 1, dtype=torch.float32,
                               device=self.device)
            gW[l] = torch.empty((fo, fi), dtype=torch.float32, device=self.device)
            call('mnpb_mlp_gemm', sh, fo, fi, rows, ptr(dz), 1, fo, ptr(acts[l]), fi, 1, 0,
                 ptr(gW[l]), fi, 1, None, 0, None, nsplit, ptr(work) if nsplit > 1 else None)
            gb[l] = torch.empty(fo, dtype=torch.float32, device=self.device)
            call('mnpb_mlp_colsum', sh, rows, fo, ptr(dz), fo, ptr(gb[l]))
            if l > 0:
                dx = torch.empty((rows, fi), dtype=torch.float32, device=self.device)
                call('mnpb_mlp_gemm', sh, rows, fi, fo, ptr(dz), fo, 1, ptr(self.Wb[l]), fi, 1,
                     1, ptr(dx), fi, 1, None, 0, None, 1, None)
                d = dx
        return gW, gb

    def mse(self, Y, T):
        """(loss as a device scalar, dL/dY)."""
        sh = _lib.stream_handle()
        dY = torch.empty_like(Y)
        nb = (Y.numel() + 255) // 256
        part = torch.empty(nb, dtype=torch.float32, device=self.device)
        call('mnpb_mlp_mse', sh, Y.numel(), ptr(Y), ptr(T), ptr(dY), ptr(part))
        return part.sum() / Y.numel(), dY

    def adam(self, gW, gb, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        sh = _lib.stream_handle()
        for l in range(len(self.W)):
            call('mnpb_mlp_adam', sh, self.W[l].numel(), ptr(self.W[l]), ptr(self.Wb[l]),
                 ptr(gW[l]), ptr(self.mW[l]), ptr(self.vW[l]), lr, b1, b2, eps, self.step)
            call('mnpb_mlp_adam', sh, self.b[l].numel(), ptr(self.b[l]), None, ptr(gb[l]),
                 ptr(self.mb[l]), ptr(self.vb[l]), lr, b1, b2, eps, self.step)

    def train_step(self, X, T, lr=1e-3):
        Y = self.forward(X, keep=True)
        loss, dY = self.mse(Y, T)
        gW, gb = self.backward(dY)
        self.adam(gW, gb, lr=lr)
        return loss


def face_geometry(p, device):
    """Per-face geometry features (n, 7): centred position / R, normal,
    sqrt(area) / R, with R the largest centroid distance from the centre."""
    pos = np.asarray(p.pos, dtype=np.float64)
    c = 0.5 * (pos.min(axis=0) + pos.max(axis=0))
    rel = pos - c
    R = max(np.sqrt((rel ** 2).sum(axis=1)).max(), 1e-12)
    g = np.hstack([rel / R, np.asarray(p.nvec), np.sqrt(np.asarray(p.area))[:, None] / R])
    return torch.from_numpy(g.astype(np.float32)).to(device)


def _eps_in_out(p, enei):
    from .materials import eps_k
    io = np.atleast_2d(np.asarray(getattr(p, 'inout', [[2, 1]])))
    ein, _ = eps_k(p.eps[io[0][0] - 1], enei)
    eout, _ = eps_k(p.eps[io[0][1] - 1], enei)
    return ein, eout


def _rms(x):
    """rms over components and faces, per polarisation: x (8, K, n) -> (K,)."""
    return torch.sqrt(torch.mean(torch.abs(x) ** 2, dim=(0, 2))).clamp_min(1e-300)


def surface_modes(p, count, device='cuda'):
    """The ``count`` smoothest surface functions of a particle: eigenvectors
    of the smallest eigenvalues of a graph Laplacian over the face centroids
    (Gaussian weights exp(-d^2 / 2 h^2), h the median distance of a face to
    its six nearest neighbours; all pairs up to 4000 faces, the 32 nearest
    neighbours of each face above).  Returns an orthonormal (n, count) FP32
    device tensor."""
    from scipy.spatial import cKDTree
    pos = np.asarray(p.pos, dtype=np.float64)
    n = pos.shape[0]
    count = min(count, n - 1)
    d6, _ = cKDTree(pos).query(pos, k=min(7, n))
    h = float(np.median(d6[:, 1:]))
    if n <= 4000:
        d2 = ((pos[:, None, :] - pos[None, :, :]) ** 2).sum(axis=2)
        W = np.exp(-d2 / (2.0 * h * h))
        np.fill_diagonal(W, 0.0)
        ev, E = np.linalg.eigh(np.diag(W.sum(axis=1)) - W)
        E = E[:, :count]
    else:
        import scipy.sparse as sp
        from scipy.sparse.linalg import eigsh
        kk = min(33, n)
        dk, jk = cKDTree(pos).query(pos, k=kk)
        w = np.exp(-dk[:, 1:] ** 2 / (2.0 * h * h))
        W = sp.coo_matrix((w.ravel(), (np.repeat(np.arange(n), kk - 1), jk[:, 1:].ravel())),
                          shape=(n, n)).tocsr()
        W = 0.5 * (W + W.T)
        L = sp.diags(np.asarray(W.sum(axis=1)).ravel()) - W
        ev, E = eigsh(L, k=count, sigma=-1e-6, which='LM')
        E = E[:, np.argsort(ev)]
    return torch.from_numpy(np.ascontiguousarray(E, dtype=np.float32)).to(device)


class LearnedWarmStart(object):
    """Trainable corrector of the quadratic extrapolation of the solution.

    ``smooth_modes``: the network's correction is restricted to the span of
    that many smoothest surface functions of the particle (``surface_modes``;
    0 keeps it per face).  GMRES resolves the smooth part of a start-vector
    error quickly and the per-face part slowly; the network's per-face
    scatter would otherwise cost more iterations than its gain in accuracy
    saves."""

    def __init__(self, width=256, depth=4, device='cuda', seed=0, smooth_modes=30):
        sizes = [NFEAT] + [width] * (depth - 1) + [NOUT]
        self.mlp = MLP(sizes, device=device, seed=seed)
        self.device = self.mlp.device
        self.mu = torch.zeros(NFEAT, device=self.device)
        self.sd = torch.ones(NFEAT, device=self.device)
        self._X, self._T = [], []
        self.trained = False
        self.smooth_modes = int(smooth_modes)
        self._modes = {}

    def _smooth(self, p, Y, K, n):
        """Project every column of each polarisation's (n, 16) block of the
        network output onto the smooth surface modes: E (E^T Y), two FP32
        products by the network's own GEMM kernel."""
        key = id(p)
        if key not in self._modes:
            self._modes[key] = (p, surface_modes(p, self.smooth_modes, self.device))
        E = self._modes[key][1]
        m = E.shape[1]
        sh = _lib.stream_handle()
        out = torch.empty_like(Y)
        coef = torch.empty((m, 16), dtype=torch.float32, device=self.device)
        nsplit = max(1, min(64, n // 512))
        work = torch.empty(nsplit * m * 16, dtype=torch.float32, device=self.device)
        for k in range(K):
            Yk, Ok = Y[k * n:(k + 1) * n], out[k * n:(k + 1) * n]
            call('mnpb_mlp_gemm', sh, m, 16, n, ptr(E), 1, m, ptr(Yk), 16, 1, 0, ptr(coef), 16,
                 1, None, 0, None, nsplit, ptr(work) if nsplit > 1 else None)
            call('mnpb_mlp_gemm', sh, n, 16, m, ptr(E), m, 1, ptr(coef), 16, 1, 0, ptr(Ok), 16,
                 1, None, 0, None, 1, None)
        return out

    # ---------------------------------------------------------------- data
    @staticmethod
    def _rows(x, K, n):
        """(8, K, n) complex -> (K * n, 16) real rows (face-major per pol)."""
        xr = torch.view_as_real(x.reshape(8, K, n))          # (8, K, n, 2)
        return xr.permute(1, 2, 0, 3).reshape(K * n, 16).float()

    def features(self, p, geo, eneis3, hist, K):
        """Feature rows (K*n, NFEAT), quadratic extrapolation q (8, K, n) and
        the target scale s2 (K,).  eneis3 = (lambda_i, .., lambda_{i-3});
        hist = (x_{i-1}, x_{i-2}, x_{i-3}) packed device vectors."""
        n = geo.shape[0]
        x1, x2, x3 = [h.reshape(8, K, n) for h in hist]
        d1 = x1 - x2
        d2 = x1 - 2.0 * x2 + x3
        s0, s1, s2 = _rms(x1), _rms(d1), _rms(d2)
        q = x1 + d1 + d2
        eps = [_eps_in_out(p, e) for e in eneis3]
        spec = [eneis3[0] / 1000.0] + [v for ein, _ in eps for v in (ein.real / 10, ein.imag / 10)] \
            + [eps[0][1].real]
        spec = torch.tensor(spec, dtype=torch.float32, device=self.device)
        rows = []
        for k in range(K):
            lr = torch.stack([torch.log10(s1[k] / s0[k]), torch.log10(s2[k] / s1[k])]).float()
            rows.append(torch.cat([spec, lr])[None, :].expand(n, -1))
        per = torch.cat(rows, dim=0)
        rep = lambda s: s.repeat_interleave(n)[:, None].float()
        F = torch.cat([geo.repeat(K, 1), per, self._rows(x1, K, n) / rep(s0),
                       self._rows(d1, K, n) / rep(s1), self._rows(d2, K, n) / rep(s2)], dim=1)
        return F.contiguous(), q, s2

    def add_sweep(self, p, eneis, xs, K=1):
        """Training pairs from a solved sweep (xs: packed device solutions)."""
        geo = face_geometry(p, self.device)
        n = geo.shape[0]
        for i in range(HISTORY, len(eneis)):
            F, q, s2 = self.features(p, geo, [eneis[i - j] for j in range(4)],
                                     [xs[i - 1], xs[i - 2], xs[i - 3]], K)
            T = (self._rows(xs[i].reshape(8, K, n) - q, K, n)
                 / s2.repeat_interleave(n)[:, None].float())
            self._X.append(F)
            self._T.append(T.contiguous())

    def add_dense_sweep(self, p, exc, eneis, batch=16):
        """Solve a sweep with the FP64 dense solver (BEMRet) and add it."""
        from .bem import BEMRet
        bem = BEMRet(p)
        xs = []
        for s0 in range(0, len(eneis), batch):
            chunk = list(eneis[s0:s0 + batch])
            bt = bem._factor(chunk)
            pots, K = bem._spectrum_pots(exc, chunk)
            xout = bem._solve_batch(bt, pots, K)
            xs += [xout[b].reshape(-1).clone() for b in range(len(chunk))]
        self.add_sweep(p, list(eneis), xs, K)
        return xs

    # ------------------------------------------------------------- training
    def fit(self, epochs=150, batch=4096, lr=2e-3, seed=0, verbose=False):
        X = torch.cat(self._X)
        T = torch.cat(self._T)
        self.mu = X.mean(dim=0)
        self.sd = X.std(dim=0).clamp_min(1e-6)
        Xn = ((X - self.mu) / self.sd).contiguous()
        g = torch.Generator(device='cpu').manual_seed(seed)
        rows = Xn.shape[0]
        losses = []
        for ep in range(epochs):
            perm = torch.randperm(rows, generator=g).to(self.device)
            lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))
            tot = 0.0
            for s0 in range(0, rows, batch):
                idx = perm[s0:s0 + batch]
                loss = self.mlp.train_step(Xn[idx].contiguous(), T[idx].contiguous(), lr=lr_ep)
                tot = tot + loss
            losses.append(float(tot) / max(1, (rows + batch - 1) // batch))
            if verbose and ep % 20 == 0:
                print('epoch', ep, 'loss', losses[-1])
        self.trained = True
        return losses

    # ------------------------------------------------------------ inference
    def prepare(self, p):
        """Per-geometry setup of ``p`` (its smooth surface modes), done by the
        first prediction otherwise."""
        if self.smooth_modes > 0 and id(p) not in self._modes:
            self._modes[id(p)] = (p, surface_modes(p, self.smooth_modes, self.device))
        return self

    def predict(self, p, eneis3, hist, K=1, geo=None):
        """Predicted packed solution at eneis3[0] from hist = (x_{i-1},
        x_{i-2}, x_{i-3})."""
        geo = face_geometry(p, self.device) if geo is None else geo
        n = geo.shape[0]
        F, q, s2 = self.features(p, geo, eneis3, hist, K)
        Y = self.mlp.forward(((F - self.mu) / self.sd).contiguous())
        if self.smooth_modes > 0:
            Y = self._smooth(p, Y, K, n)
        d = (Y * s2.repeat_interleave(n)[:, None]).double()              # (K*n, 16)
        d = torch.view_as_complex(d.reshape(K, n, 8, 2)).permute(2, 0, 1)   # (8, K, n)
        return (q + d).reshape(-1).contiguous()
