"""Iterative retarded BEM solver on the GPU: ``BEMRetIter`` with the
reference call surface (mnpbem/bem/bem_ret_iter.py:461-1831,
mnpbem/bem/bem_iter.py:20-244)

    bem = BEMRetIter(p, hmatrix=True, htol=1e-6, cleaf=64, tol=1e-6)
    sig, bem = bem.solve(exc.potential(p, enei))

GMRES solves the packed 8N system of bem_ret_iter.py:1362-1501 for all
polarisations at once (one Krylov space over the stacked vector, as the
reference does).  The operator applies G1, G2, H1, H2 either as dense FP64
matrices or, with ``hmatrix=True``, as ACA-compressed H-matrices (complex64
factors, FP64 accumulation).  Arnoldi orthogonalisation and the Givens
rotations run in FP64 on the GPU.

Preconditioning (right-preconditioned GMRES, so the residual that is tested
is the true one): the reference's exact dense preconditioner
(bem_ret_iter.py:801-1086, 1503-1634) is this package's FP64 dense
``BEMRet`` factorisation of the same matrices; ``preconditioner='none'``
(H-matrix path) or ``precond=None`` (dense path) switch it off.

A warm start ``x0`` may be passed to ``solve``; ``warm_start`` /
``deflation`` hooks let a learned predictor supply it (see
``mnpbem_b200.learned``).
"""

import numpy as np
import torch

from . import _lib
from ._lib import call, ptr
from .bem import BEMRet, _check_particle, _scalar_eps
from .clustertree import BlockPartition, ClusterTree, make_kaware_fadmiss
from .compstruct import CompStruct
from .greenfun import CompGreenRet
from .hmatrix import HMatrixGPU, HTopology, hmat_matvec

__all__ = ["BEMRetIter", "gmres"]


class _Counter(object):
    def __init__(self):
        self.matvecs = 0


def _norm(v, stream=None):
    """Euclidean norm of a complex128 device vector (FP64, on the GPU)."""
    L = v.numel()
    nch = (L + 2047) // 2048
    part = torch.empty(nch, dtype=torch.float64, device=v.device)
    out = torch.empty(1, dtype=torch.float64, device=v.device)
    call('mnpb_vec_norms', _lib.stream_handle(stream), L, 1, ptr(v), L, ptr(part), ptr(out))
    return out


def gmres(apply_A, b, tol=1e-6, maxit=200, restart=None, x0=None, apply_M=None,
          stream=None, counter=None, r0=None, augment=None):
    """Restarted, right-preconditioned GMRES on complex128 device vectors.

    ``apply_A(v) -> A v`` and ``apply_M(v) -> M v`` take and return flat
    complex128 device tensors.  Stops when |b - A x| <= tol |b| (scipy
    semantics, bem_iter.py:79-89: restart = min(n, maxit), at most ``maxit``
    restart cycles).  ``r0``: b - A x0 when the caller already has it.

    ``augment``: optional list of flat device vectors U whose span is searched
    together with the Krylov space (GCRO augmentation, de Sturler 1999):
    C = A U is orthonormalised (U R^-1 alongside), the residual is projected
    off range(C) and Arnoldi runs on (I - C C^H) A M, so the solution
    minimises |b - A x| over x0 + range(U) + M K_m.  C occupies the first
    columns of the Arnoldi basis, so each CGS2 step projects against C and
    the Krylov vectors together.  Costs one operator application per vector
    of U; nearly dependent vectors are dropped.

    Returns (x, flag, relres, [cycles, iterations]).
    """
    dev = b.device
    L = b.numel()
    restart = min(L, maxit) if restart is None else int(restart)
    restart = max(1, restart)
    sh = _lib.stream_handle(stream)
    count = counter if counter is not None else _Counter()

    def A(v):
        count.matvecs += 1
        return apply_A(v)

    M = apply_M if apply_M is not None else (lambda v: v)
    bnorm = float(_norm(b, stream).item())
    if bnorm == 0.0:
        return torch.zeros_like(b), 0, 0.0, [0, 0]
    x = torch.zeros_like(b) if x0 is None else x0.reshape(-1).clone()
    if x0 is None:
        r = b.clone()
    else:
        r = r0.clone() if r0 is not None else b - A(x)
    kmax = len(augment) if augment else 0
    W = torch.empty((kmax + restart + 1, L), dtype=torch.complex128, device=dev)
    hcol = torch.zeros(kmax + restart + 2, dtype=torch.complex128, device=dev)
    nrm = torch.zeros(1, dtype=torch.float64, device=dev)
    wb = int(_lib.lib().mnpb_gmres_workspace(L, kmax + restart))
    work = torch.empty(wb, dtype=torch.uint8, device=dev)
    # augmentation: C = A U orthonormalised in W[0:kc], Uc = U R^-1
    Uc = []
    kc = 0
    for u in (augment or []):
        u = u.reshape(-1)
        c = A(u).reshape(-1).contiguous()
        cn = float(_norm(c, stream).item())
        if cn == 0.0:
            continue
        if kc == 0:
            W[0].copy_(c / cn)
            coef, diag = [], cn
        else:
            call('mnpb_gmres_arnoldi', sh, L, kc - 1, ptr(W), L, ptr(c), ptr(hcol), ptr(nrm),
                 ptr(work), wb)
            diag = float(nrm.item())
            if diag <= 1e-6 * cn:
                continue                               # (nearly) in the span already
            coef = hcol[:kc].clone()
        v = u.clone()
        for i in range(len(coef)):
            v -= coef[i] * Uc[i]
        Uc.append(v / diag)
        kc += 1
    C = W[:kc]

    def project(x, r):
        """x += Uc z, r -= C z with z = C^H r (r off range(C))."""
        if kc == 0:
            return x, r
        z = torch.mv(C.conj(), r)
        for i in range(kc):
            x = x + z[i] * Uc[i]
        return x, r - torch.mv(C.transpose(0, 1), z)

    V = W[kc:]
    H = torch.zeros((restart, restart + 1), dtype=torch.complex128, device=dev)
    Bm = torch.zeros((restart, max(kc, 1)), dtype=torch.complex128, device=dev)
    cs = torch.zeros(restart, dtype=torch.float64, device=dev)
    sn = torch.zeros(restart, dtype=torch.complex128, device=dev)
    g = torch.zeros(restart + 1, dtype=torch.complex128, device=dev)
    y = torch.zeros(restart, dtype=torch.complex128, device=dev)
    res = torch.zeros(1, dtype=torch.float64, device=dev)
    flag, cycles, iters = 1, 0, 0
    beta = float(_norm(r, stream).item())
    checked = False
    for cycle in range(maxit):
        # convergence is judged on the true residual b - A x; the projection
        # off range(C) only prepares the next cycle
        if beta <= tol * bnorm:
            flag = 0
            break
        if kc:
            x, r = project(x, r)
            beta = float(_norm(r, stream).item())
            if beta <= tol * bnorm and not checked:
                # the augmentation space alone solves the system: confirm it on
                # the true residual (once) instead of iterating on rounding noise
                checked = True
                r = b - A(x)
                beta = float(_norm(r, stream).item())
                continue
        cycles += 1
        V[0].copy_(r / beta)
        g.zero_()
        g[0] = beta
        H.zero_()
        m = 0
        for j in range(restart):
            w = A(M(V[j])).reshape(-1).contiguous()
            if kc == 0:
                call('mnpb_gmres_arnoldi', sh, L, j, ptr(V), L, ptr(w), ptr(H[j]), ptr(nrm),
                     ptr(work), wb)
            else:
                call('mnpb_gmres_arnoldi', sh, L, kc + j, ptr(W), L, ptr(w), ptr(hcol),
                     ptr(nrm), ptr(work), wb)
                Bm[j, :kc].copy_(hcol[:kc])
                H[j, :j + 2].copy_(hcol[kc:kc + j + 2])
            call('mnpb_gmres_givens', sh, j, ptr(H), restart + 1, ptr(cs), ptr(sn), ptr(g),
                 ptr(res))
            iters += 1
            m = j + 1
            if float(res.item()) <= tol * bnorm or float(nrm.item()) == 0.0:
                break
        z = torch.zeros_like(b)
        call('mnpb_gmres_update', sh, L, m, ptr(H), restart + 1, ptr(g), ptr(V), L, ptr(y),
             ptr(z))
        x = x + M(z)
        if kc:
            t = torch.mv(Bm[:m, :kc].transpose(0, 1), y[:m])
            for i in range(kc):
                x = x - t[i] * Uc[i]
        r = b - A(x)
        beta = float(_norm(r, stream).item())
    if beta <= tol * bnorm:
        flag = 0
    return x, flag, beta / bnorm, [cycles, iters]


class BEMRetIter(object):
    """Iterative retarded BEM solver (GMRES; dense or H-matrix operator)."""

    def __init__(self, p, enei=None, solver='gmres', tol=1e-4, maxit=200, restart=None,
                 precond='hmat', output=0, hmatrix=False, htol=1e-6, kmax=(4, 100), cleaf=200,
                 fadmiss=None, eta=2.5, preconditioner='auto', htol_precond=1e-4, **options):
        _check_particle(p, 'BEMRetIter')
        if solver != 'gmres':
            raise NotImplementedError("BEMRetIter: only solver='gmres' runs on the GPU")
        for key in ('refun', 'schur'):
            if options.pop(key, None):
                raise NotImplementedError("BEMRetIter: {} is not supported".format(key))
        self.p = p
        self.solver, self.tol, self.maxit, self.restart = solver, tol, maxit, restart
        self.output = output
        self.hmatrix = bool(hmatrix)
        self.htol = max(htol) if hasattr(htol, '__iter__') else htol
        self.kmax = int(max(kmax) if hasattr(kmax, '__iter__') else kmax)
        self.cleaf, self.eta, self.fadmiss = int(cleaf), eta, fadmiss
        if self.hmatrix and 'precond' not in options and precond == 'hmat':
            precond = None                  # bem_ret_iter.py: hmatrix path leaves it to
        self.precond = precond              # ``preconditioner``
        if preconditioner not in ('auto', 'none', 'hlu_dense', 'hlu_tree'):
            raise ValueError("BEMRetIter: unknown preconditioner {!r}".format(preconditioner))
        if preconditioner == 'hlu_tree':
            raise NotImplementedError("BEMRetIter: the hierarchical LU preconditioner "
                                      "('hlu_tree') is not built; use 'auto' or 'none'")
        self.preconditioner = preconditioner
        self.options = options
        self.g = CompGreenRet(p, p, **options)
        self.tables = self.g.tables
        self.device = self.tables.device
        self.nvec = torch.from_numpy(np.ascontiguousarray(p.nvec, dtype=np.float64)).to(self.device)
        self.enei = None
        self._flag, self._relres, self._iter = [], [], []
        self._matvecs = []
        self.tree = None
        self._topos = {}
        self._scratch = None
        if self.hmatrix:
            ipart = None
            parts = getattr(p, 'p', [p])
            if len(parts) > 1:
                ipart = np.concatenate([np.full(q.nfaces, i, dtype=np.int64)
                                        for i, q in enumerate(parts)])
            self.tree = ClusterTree(p.pos, cleaf=self.cleaf, ipart_arr=ipart)
        if enei is not None:
            self._init_matrices(enei)

    # ------------------------------------------------------------- matrices
    def _use_dense_precond(self):
        if self.hmatrix:
            return self.preconditioner in ('auto', 'hlu_dense')
        return self.precond is not None

    def _init_matrices(self, enei):
        """Operator (and preconditioner) at ``enei``; exact-equality cache as
        bem_ret_iter.py:585-600."""
        if self.enei is not None and self.enei == enei:
            return self
        t = self.tables
        n = t.n
        self.enei = enei
        self.k = 2 * np.pi / enei
        self.eps1, self.eps2 = _scalar_eps(self.p, enei)
        kblk, sblk = t.k_tables([enei])
        GG = torch.empty((2, 1, n, n), dtype=torch.complex128, device=self.device)
        HH = torch.empty((2, 1, n, n), dtype=torch.complex128, device=self.device)
        t.assemble(kblk, sblk, (GG[0], HH[0], GG[1], HH[1]), mode=0)
        self._pre = None
        if self._use_dense_precond():
            self._pre = self._dense_precond(GG, HH)
        if self.hmatrix:
            fad = self.fadmiss if self.fadmiss is not None else \
                make_kaware_fadmiss(2.0 * np.pi / enei, eta0=self.eta)
            part = BlockPartition(self.tree, fad)
            key = part.key()
            if key not in self._topos:
                self._topos = {key: HTopology(part, self.kmax, self.device)}
            topo = self._topos[key]
            self.topo = topo
            mats = []
            for A in (GG[0, 0], GG[1, 0], HH[0, 0], HH[1, 0]):
                h = HMatrixGPU(topo, A, n, self.htol, scratch=self._scratch)
                self._scratch = h.scratch
                mats.append(h)
            self.G1, self.G2, self.H1, self.H2 = mats
            del GG, HH
        else:
            self.G1, self.G2, self.H1, self.H2 = GG[0, 0], GG[1, 0], HH[0, 0], HH[1, 0]
            self._GG, self._HH = GG, HH
        return self

    def _dense_precond(self, GG, HH):
        """Exact preconditioner: FP64 dense BEMRet factorisation of G1, G2, H1,
        H2 (same algebra as bem_ret_iter.py:801-1086)."""
        t = self.tables
        n = t.n
        sh = _lib.stream_handle()
        pre = type('Pre', (), {})()
        pre.GG = GG.clone()
        pre.HH = HH.clone()
        pre.D = torch.empty((1, n, n), dtype=torch.complex128, device=self.device)
        pre.piv = torch.empty((3, 1, n), dtype=torch.int32, device=self.device)
        pre.info = torch.zeros((2, 1), dtype=torch.int32, device=self.device)
        wb = int(_lib.lib().mnpb_bemret_workspace_f64(n, 1))
        pre.work = torch.empty(wb, dtype=torch.uint8, device=self.device)
        e1, e2 = self.eps1, self.eps2
        pre.eps = torch.tensor([[e1.real, e1.imag, e2.real, e2.imag]], dtype=torch.float64,
                               device=self.device)
        pre.kvac = torch.tensor([self.k], dtype=torch.float64, device=self.device)
        call('mnpb_bemret_init_f64', sh, n, 1, ptr(pre.GG[0]), ptr(pre.GG[1]), ptr(pre.HH[0]),
             ptr(pre.HH[1]), ptr(pre.D), n, n * n, ptr(pre.eps), ptr(pre.kvac), ptr(t.nvec), 0,
             ptr(pre.piv), ptr(pre.info), ptr(pre.work), pre.work.numel())
        if pre.info.any():
            raise _lib.MNPBError('BEMRetIter precond', 3, 'zero pivot')
        return pre

    def _apply_precond(self, v, K):
        t = self.tables
        n = t.n
        xin = v.reshape(1, 8, K, n).contiguous()
        xout = torch.empty_like(xin)
        wb = n * 15 * K * 16
        work = torch.empty(wb, dtype=torch.uint8, device=self.device)
        pre = self._pre
        call('mnpb_bemret_solve_f64', _lib.stream_handle(), n, 1, K, ptr(pre.GG[0]),
             ptr(pre.GG[1]), ptr(pre.HH[0]), ptr(pre.HH[1]), ptr(pre.D), n, n * n, ptr(pre.piv),
             ptr(pre.eps), ptr(pre.kvac), ptr(t.nvec), 0, ptr(xin), ptr(xout), ptr(work), wb)
        return xout.reshape(-1)

    # -------------------------------------------------------------- operator
    def _afun(self, x, K):
        """y = A x for the packed vector (bem_ret_iter.py:1362-1501)."""
        n = self.tables.n
        X = x.reshape(8, K, n)
        v1 = X[0:4].reshape(4 * K, n).contiguous()
        v2 = X[4:8].reshape(4 * K, n).contiguous()
        P1, P2, Q1, Q2 = [torch.empty((4 * K, n), dtype=torch.complex128, device=self.device)
                          for _ in range(4)]
        if self.hmatrix:
            hmat_matvec([self.G1, self.G2, self.H1, self.H2], [v1, v2, v1, v2], [P1, P2, Q1, Q2],
                        4 * K)
        else:
            sh = _lib.stream_handle()
            for A, v, out in ((self.G1, v1, P1), (self.G2, v2, P2), (self.H1, v1, Q1),
                              (self.H2, v2, Q2)):
                call('mnpb_zgemm', sh, n, 4 * K, n, 1, 1.0, 0.0, ptr(A), n, n * n, ptr(v), n,
                     n * 4 * K, 0.0, 0.0, ptr(out), n, n * 4 * K)
        y = torch.empty(8 * K * n, dtype=torch.complex128, device=self.device)
        e1, e2 = self.eps1, self.eps2
        call('mnpb_bem_afun', _lib.stream_handle(), n, K, ptr(P1), ptr(P2), ptr(Q1), ptr(Q2),
             ptr(y), e1.real, e1.imag, e2.real, e2.imag, self.k, ptr(self.nvec))
        return y

    # ----------------------------------------------------------------- solve
    def _excitation(self, exc):
        t = self.tables
        n = t.n
        pots, K = BEMRet._pots(exc, n)
        d_pots = torch.from_numpy(pots).to(self.device).unsqueeze(0)
        e1, e2 = self.eps1, self.eps2
        eps = torch.tensor([[e1.real, e1.imag, e2.real, e2.imag]], dtype=torch.float64,
                           device=self.device)
        kvac = torch.tensor([self.k], dtype=torch.float64, device=self.device)
        b = torch.empty((1, 8, K, n), dtype=torch.complex128, device=self.device)
        call('mnpb_bemret_excitation', _lib.stream_handle(), n, 1, K, ptr(d_pots), ptr(eps),
             ptr(kvac), ptr(t.nvec), 0, ptr(b))
        return b.reshape(-1), K

    def solve(self, exc, x0=None):
        """Surface charges and currents (bem_ret_iter.py:1636-1746); ``x0``:
        optional warm start, a flat complex128 device vector in the packed
        layout (8, K, n) or a CompStruct with sig1, h1, sig2, h2."""
        self._init_matrices(exc['enei'])
        b, K = self._excitation(exc)
        if x0 is not None and not torch.is_tensor(x0):
            x0 = self._pack_solution(x0, K)
        x, flag, relres, it = self.solve_packed(b, K, x0=x0)
        xh = x.reshape(8, K, self.tables.n).cpu().numpy()
        return self._to_compstruct(xh, K, exc['enei']), self

    def solve_packed(self, b, K, x0=None):
        """GMRES on a packed right-hand side already on the device."""
        cnt = _Counter()
        M = (lambda v: self._apply_precond(v, K)) if self._pre is not None else None
        x, flag, relres, it = gmres(lambda v: self._afun(v, K), b, tol=self.tol,
                                    maxit=self.maxit, restart=self.restart, x0=x0, apply_M=M,
                                    counter=cnt)
        self._flag.append(flag)
        self._relres.append(relres)
        self._iter.append(np.array(it))
        self._matvecs.append(cnt.matvecs)
        if self.output:
            print('gmres: flag {}, relres {:.3e}, {} iterations, {} operator applications'.format(
                flag, relres, it[1], cnt.matvecs))
        return x, flag, relres, it

    def solve_spectrum(self, exc, eneis, warm=None, deflate=False):
        """Solve a wavelength sweep with GMRES warm starts.

        ``warm``: None (zero start, the reference's behaviour), 'previous'
        (x_{i-1}), 'extrapolate' (quadratic: 3 x_{i-1} - 3 x_{i-2} + x_{i-3})
        or a trained ``mnpbem_b200.learned.LearnedWarmStart`` (which corrects
        the quadratic extrapolation).  The first wavelengths fall back to the
        previous solution / linear extrapolation until the history is long
        enough.  ``deflate``: False, or the number m of previous solutions
        (True: 3) that, with the start vector, span the GCRO augmentation
        space of each solve (``gmres(augment=...)``): GMRES then minimises the
        residual over that span and the Krylov space of the operator
        deflated by it.  Returns (list of CompStruct, list of per-wavelength
        statistics dicts, list of packed device solutions).
        """
        from .learned import LearnedWarmStart, face_geometry
        n = self.tables.n
        learned = isinstance(warm, LearnedWarmStart)
        geo = face_geometry(self.p, self.device) if learned else None
        xs, sols, stats = [], [], []
        for i, enei in enumerate(eneis):
            self._init_matrices(enei)
            b, K = self._excitation(exc.potential(self.p, enei))
            cnt = _Counter()
            A = lambda v: self._afun(v, K)
            x0 = r0 = None
            if warm is not None and i >= 1:
                if warm == 'previous' or i < 2:
                    x0 = xs[i - 1]
                elif i < 3:
                    x0 = 2.0 * xs[i - 1] - xs[i - 2]
                elif warm == 'extrapolate':
                    x0 = 3.0 * xs[i - 1] - 3.0 * xs[i - 2] + xs[i - 3]
                elif learned:
                    x0 = warm.predict(self.p, [eneis[i - j] for j in range(4)],
                                      [xs[i - 1], xs[i - 2], xs[i - 3]], K, geo)
                else:
                    raise ValueError("solve_spectrum: unknown warm start {!r}".format(warm))
            aug = None
            if deflate and i >= 1:
                m = 3 if deflate is True else int(deflate)
                aug = ([x0] if x0 is not None else []) + xs[max(0, i - m):i]
                x0 = None
            M = (lambda v: self._apply_precond(v, K)) if self._pre is not None else None
            x, flag, relres, it = gmres(A, b, tol=self.tol, maxit=self.maxit,
                                        restart=self.restart, x0=x0, apply_M=M, counter=cnt,
                                        r0=r0, augment=aug)
            self._flag.append(flag)
            self._relres.append(relres)
            self._iter.append(np.array(it))
            self._matvecs.append(cnt.matvecs)
            stats.append(dict(enei=enei, flag=flag, relres=relres, iters=it[1],
                              matvecs=cnt.matvecs))
            xs.append(x)
            sols.append(self._to_compstruct(x.reshape(8, K, n).cpu().numpy(), K, enei))
        return sols, stats, xs

    def _pack_solution(self, sig, K):
        n = self.tables.n
        s1 = np.asarray(sig.sig1).reshape(n, -1)
        s2 = np.asarray(sig.sig2).reshape(n, -1)
        h1 = np.asarray(sig.h1).reshape(n, 3, -1)
        h2 = np.asarray(sig.h2).reshape(n, 3, -1)
        x = np.zeros((8, K, n), dtype=complex)
        x[0] = s1.T
        x[1:4] = h1.transpose(1, 2, 0)
        x[4] = s2.T
        x[5:8] = h2.transpose(1, 2, 0)
        return torch.from_numpy(x.reshape(-1)).to(self.device)

    def _to_compstruct(self, x, K, enei):
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

    def __call__(self, enei):
        return self._init_matrices(enei)

    def clear(self):
        self.enei = None
        self.G1 = self.G2 = self.H1 = self.H2 = None
        self._pre = None
        return self

    def info(self):
        """(flag, relres, iter) lists, one entry per solve (bem_iter.py);
        iter = [restart cycles, GMRES iterations]."""
        return self._flag, self._relres, self._iter

    def matvec_counts(self):
        return list(self._matvecs)

    def compression(self):
        """Stored fraction of the dense matrix per operator (G1, G2, H1, H2)."""
        if not self.hmatrix or self.G1 is None:
            return None
        return [h.compression() for h in (self.G1, self.G2, self.H1, self.H2)]
