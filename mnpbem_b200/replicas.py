"""Multi-GPU spectrum sweeps: one process per GPU, wavelengths shared out.

Every (particle, wavelength) solve is independent, so the path shards without
any collective on the data path (the reference's multi-GPU worker pool,
mnpbem/utils/multi_gpu.py, does the same with processes).  Each rank solves
its own wavelengths with the full solver; the only collective is one
all-gather of the per-wavelength results (extinction, scattering, iteration
counts: a few numbers per wavelength) at the end, and a max over ranks of
the device time.

Wavelengths are dealt out interleaved (rank r takes i = r, r + N, ...), which
balances resonances whose iterative solves take longer across the ranks.
Works with any torch.distributed backend: NCCL on GPUs, gloo on CPU (tests).
"""

import numpy as np
import torch
import torch.distributed as dist

__all__ = ["shard", "gather_rows", "max_over_ranks", "sweep"]


def shard(n_items, rank, world, mode='interleaved'):
    """Indices of the items rank ``rank`` of ``world`` takes."""
    if not 0 <= rank < world:
        raise ValueError("shard: rank out of range")
    idx = np.arange(n_items)
    if mode == 'interleaved':
        return idx[rank::world]
    if mode == 'contiguous':
        return np.array_split(idx, world)[rank]
    raise ValueError("shard: mode must be 'interleaved' or 'contiguous'")


def _device_for_backend():
    if dist.get_backend() == 'nccl':
        return torch.device('cuda', torch.cuda.current_device())
    return torch.device('cpu')


def gather_rows(local, indices, n_items):
    """Reassemble per-item rows from all ranks: ``local`` (len(indices), m)
    float64 rows of this rank's items -> (n_items, m) on every rank.  One
    all-gather (rows padded to the largest shard)."""
    world = dist.get_world_size()
    dev = _device_for_backend()
    local = np.asarray(local, dtype=np.float64).reshape(len(indices), -1)
    m = local.shape[1]
    cap = (n_items + world - 1) // world
    buf = torch.full((cap, m + 1), -1.0, dtype=torch.float64, device=dev)
    if len(indices):
        buf[:len(indices), 0] = torch.as_tensor(np.asarray(indices, dtype=np.float64))
        buf[:len(indices), 1:] = torch.as_tensor(local)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = np.full((n_items, m), np.nan)
    for p in parts:
        p = p.cpu().numpy()
        for row in p:
            if row[0] >= 0:
                out[int(row[0])] = row[1:]
    return out


def max_over_ranks(value):
    """Largest value of a scalar over all ranks (device times of one step)."""
    t = torch.tensor([float(value)], dtype=torch.float64, device=_device_for_backend())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sweep(solve_one, eneis, mode='interleaved'):
    """Run ``solve_one(enei) -> sequence of floats`` over this rank's share of
    ``eneis`` and return the full (len(eneis), m) result table on every rank."""
    rank, world = dist.get_rank(), dist.get_world_size()
    idx = shard(len(eneis), rank, world, mode)
    rows = [np.atleast_1d(np.asarray(solve_one(eneis[i]), dtype=np.float64)) for i in idx]
    m = rows[0].size if rows else 0
    m = int(max_over_ranks(m))
    local = np.vstack(rows) if rows else np.zeros((0, m))
    return gather_rows(local, idx, len(eneis))
