"""Warm-start network on the GPU: forward/backward/Adam kernels against the
float64 CPU oracle (gradient check), and the ablation -- GMRES operator
applications over a held-out wavelength sweep with and without the trained
network, at the same converged answer.

Gradient-check tolerance: the GPU accumulates in FP32 over up to 10^4 rows
with identical bf16 weights, so relative Frobenius differences stay below
1e-4 (measured ~1e-6)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize('rows', [300, 10000])
def test_mlp_gradients_against_oracle(gpu_ok, rows):
    from mnpbem_b200.learned import MLP
    from oracle import mlp_oracle as mo
    sizes = [48, 256, 256, 256, 16]
    net = MLP(sizes, seed=1, out_scale=1.0)
    rng = np.random.default_rng(rows)
    X = rng.standard_normal((rows, 48)).astype(np.float32)
    T = rng.standard_normal((rows, 16)).astype(np.float32)
    dX, dT = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    Y = net.forward(dX, keep=True)
    loss, dY = net.mse(Y, dT)
    gW, gb = net.backward(dY)
    torch.cuda.synchronize()
    Ws = [mo.bf16_round(w.cpu().numpy()) for w in net.W]
    bs = [b.cpu().numpy().astype(np.float64) for b in net.b]
    rloss, rgW, rgb, ry = mo.loss_and_grads(Ws, bs, X.astype(np.float64), T.astype(np.float64))
    assert _rel(Y.cpu().numpy(), ry) < 1e-5
    assert abs(float(loss) - rloss) < 1e-5 * rloss
    for l in range(4):
        assert _rel(gW[l].cpu().numpy(), rgW[l]) < 1e-4, l
        assert _rel(gb[l].cpu().numpy(), rgb[l]) < 1e-4, l
    # one Adam step on the same gradients
    w0 = [w.cpu().numpy().astype(np.float64) for w in net.W]
    g = [x.cpu().numpy().astype(np.float64) for x in gW]
    net.adam(gW, gb, lr=1e-3)
    torch.cuda.synchronize()
    for l in range(4):
        ref, _, _ = mo.adam(w0[l], g[l], 0.0, 0.0, 1e-3, 0.9, 0.999, 1e-8, 1)
        assert _rel(net.W[l].cpu().numpy(), ref) < 1e-6
        assert np.array_equal(net.Wb[l].float().cpu().numpy(), mo.bf16_round(net.W[l].cpu().numpy()))


def _spheroid(a, nv=144, d=20.0):
    from mnpbem_b200.geometry import ComParticle, trisphere
    from mnpbem_b200.materials import EpsConst, EpsDrude
    s = trisphere(nv, d).scale([1.0, 1.0, a])
    return ComParticle([EpsConst(1.0), EpsDrude(10.0, 9.065, 0.0708)], [s], [[2, 1]], 1)


def test_learned_warm_start_saves_gmres_work(gpu_ok):
    """Train on four spheroid sweeps solved by the FP64 dense solver, then
    on a held-out spheroid (31 wavelengths, unpreconditioned dense operator,
    GMRES tol 1e-8):

    (1) the network's prediction must be at least 10x closer to the true
        solution than quadratic extrapolation (measured ~16x);
    (2) ablation of operator applications over the sweep -- zero start,
        quadratic extrapolation, extrapolation + GCRO augmentation with the
        last 3 solutions, the network's start, and the network's start + the
        same augmentation (measured 3118, 1390, 1208, 1328, 1292): the
        network's start must need fewer than 0.97x the applications of
        quadratic extrapolation and, with the augmentation, fewer than
        extrapolation and than 0.6x zero start.  Augmentation with the last
        solutions alone does better still; the network adds nothing on top
        of it (the error it removes lies mostly in directions GMRES resolves
        quickly anyway);
    (3) every variant gives the dense solver's extinction to 1e-4 (the
        operator's conditioning, ~1e4, times the GMRES tolerance)."""
    from mnpbem_b200 import BEMRet
    from mnpbem_b200.bem_iter import BEMRetIter
    from mnpbem_b200.excitation import PlaneWaveRet
    from mnpbem_b200.learned import LearnedWarmStart
    exc = PlaneWaveRet([[1.0, 0.0, 0.0]], [[0.0, 0.0, 1.0]])
    eneis = list(np.linspace(500.0, 800.0, 31))
    model = LearnedWarmStart(seed=0)
    for a in (1.0, 1.5, 2.0, 2.5):
        model.add_dense_sweep(_spheroid(a), exc, eneis)
    losses = model.fit(epochs=150, batch=4096, lr=2e-3)
    assert losses[-1] < 0.1 * losses[0]
    cp = _spheroid(1.75)                       # held out
    ext_dense = np.array([exc.extinction(s) for s in BEMRet(cp).solve_spectrum(exc, eneis)])
    xs = LearnedWarmStart(seed=1).add_dense_sweep(cp, exc, eneis)
    eq, el = [], []
    for i in range(3, len(eneis)):
        q = 3 * xs[i - 1] - 3 * xs[i - 2] + xs[i - 3]
        pr = model.predict(cp, [eneis[i - j] for j in range(4)], [xs[i - 1], xs[i - 2], xs[i - 3]])
        nx = torch.linalg.norm(xs[i])
        eq.append(float(torch.linalg.norm(q - xs[i]) / nx))
        el.append(float(torch.linalg.norm(pr - xs[i]) / nx))
    gq, gl = np.exp(np.mean(np.log(eq))), np.exp(np.mean(np.log(el)))
    print('\nheld-out prediction error: quadratic extrapolation %.2e, learned %.2e' % (gq, gl))
    assert gl < 0.1 * gq
    res = {}
    for name, warm, defl in (('zero', None, False), ('extrapolate', 'extrapolate', False),
                             ('extrapolate+deflation', 'extrapolate', 3),
                             ('learned', model, False), ('learned+deflation', model, 3)):
        bem = BEMRetIter(cp, tol=1e-8, precond=None)
        sols, stats, _ = bem.solve_spectrum(exc, eneis, warm=warm, deflate=defl)
        assert all(s['flag'] == 0 for s in stats), name
        ext = np.array([exc.extinction(s) for s in sols])
        res[name] = sum(s['matvecs'] for s in stats)
        # a relative residual of 1e-8 on the unpreconditioned operator (condition
        # number ~1e4) leaves ~1e-5 in the extinction, whatever the start
        assert np.max(np.abs(ext - ext_dense) / np.abs(ext_dense)) < 1e-4, name
    print('\noperator applications over 31 wavelengths (GMRES tol 1e-8):', res)
    assert res['learned'] < 0.97 * res['extrapolate']
    assert res['learned+deflation'] < res['extrapolate']
    assert res['learned+deflation'] < 0.6 * res['zero']
