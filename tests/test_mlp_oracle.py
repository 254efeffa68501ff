"""The float64 network oracle (oracle/mlp_oracle.py) pinned by central finite
differences, and its bf16 rounding against torch's."""
import numpy as np
import torch

from oracle import mlp_oracle as mo


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    sizes = [5, 7, 6, 3]
    Ws = [rng.standard_normal((o, i)) * 0.5 for i, o in zip(sizes[:-1], sizes[1:])]
    bs = [rng.standard_normal(o) * 0.1 for o in sizes[1:]]
    X = rng.standard_normal((11, 5))
    T = rng.standard_normal((11, 3))
    loss, gW, gb, _ = mo.loss_and_grads(Ws, bs, X, T)
    h = 1e-6
    for l in range(len(Ws)):
        for idx in [(0, 0), (Ws[l].shape[0] - 1, Ws[l].shape[1] - 1), (1, 2)]:
            Wp = [w.copy() for w in Ws]
            Wm = [w.copy() for w in Ws]
            Wp[l][idx] += h
            Wm[l][idx] -= h
            fd = (mo.loss_and_grads(Wp, bs, X, T)[0] - mo.loss_and_grads(Wm, bs, X, T)[0]) / (2 * h)
            assert abs(fd - gW[l][idx]) < 1e-7 * max(1.0, abs(fd))
        bp = [b.copy() for b in bs]
        bm = [b.copy() for b in bs]
        bp[l][0] += h
        bm[l][0] -= h
        fd = (mo.loss_and_grads(Ws, bp, X, T)[0] - mo.loss_and_grads(Ws, bm, X, T)[0]) / (2 * h)
        assert abs(fd - gb[l][0]) < 1e-7 * max(1.0, abs(fd))


def test_bf16_rounding_matches_torch():
    x = np.random.default_rng(1).standard_normal(10000).astype(np.float32) * 3
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy().astype(np.float64)
    assert np.array_equal(mo.bf16_round(x), ref)
