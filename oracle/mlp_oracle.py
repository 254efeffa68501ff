"""CPU float64 restatement of the warm-start network -- TEST INFRASTRUCTURE ONLY.

Same architecture and arithmetic definitions as the CUDA kernels of
``mnpbem_b200/csrc/mlp.cu`` (the network has no counterpart in the
reference): dense layers y = act(x W^T + b) with SiLU on hidden layers and a
linear output layer, mean-squared-error loss, Adam with the bias correction
folded into the step size (Kingma & Ba 2015, end of Sec. 2).  Weights enter
as the bf16-rounded values the GPU products read.  Only ``tests/`` import it.
"""

import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def bf16_round(w):
    """Round float32 values to bf16 (round to nearest even), as float64."""
    w = np.ascontiguousarray(w, dtype=np.float32)
    u = w.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(Ws, bs, X):
    """Activations and pre-activations of every layer (float64)."""
    acts, pre = [np.asarray(X, dtype=np.float64)], []
    for l, (W, b) in enumerate(zip(Ws, bs)):
        z = acts[-1] @ W.T + b
        pre.append(z)
        acts.append(z if l == len(Ws) - 1 else silu(z))
    return acts, pre


def loss_and_grads(Ws, bs, X, T):
    """MSE loss mean((y - t)^2) and its gradients w.r.t. weights and biases."""
    acts, pre = forward(Ws, bs, X)
    y = acts[-1]
    loss = np.mean((y - T) ** 2)
    d = 2.0 * (y - T) / y.size
    gW, gb = [None] * len(Ws), [None] * len(Ws)
    for l in range(len(Ws) - 1, -1, -1):
        dz = d if l == len(Ws) - 1 else d * silu_grad(pre[l])
        gW[l] = dz.T @ acts[l]
        gb[l] = dz.sum(axis=0)
        d = dz @ Ws[l]
    return loss, gW, gb, y


def adam(w, g, m, v, lr, b1, b2, eps, step):
    """One Adam step with lr_t = lr sqrt(1 - b2^t) / (1 - b1^t)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    lr_t = lr * np.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    return w - lr_t * m / (np.sqrt(v) + eps), m, v
