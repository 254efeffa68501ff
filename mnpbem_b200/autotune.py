"""Launch-configuration autotuner for the tensor-core factorisation.

The tensor-core GEMMs of the mixed factorisation take three launch choices
(``mnpb_gemm_config``): the tile width used for N > 64 (64 or 128 columns),
the number of tiles per SM from which the persistent kernel replaces the
one-tile-per-CTA grid, and the depth of the TMA operand ring.  Which choice
is fastest depends on the matrix size and on how many matrices a launch
batches (small matrices in large batches want other tiles than a few large
ones).  ``GemmTuner.choose(key, run)`` times every candidate on the caller's
own workload once (``run()`` issues one representative launch sequence and
must be repeatable), keeps the fastest per key (typically the face count and
batch size) and applies it; later calls with the same key only apply the
stored choice.  The table can be kept in a JSON file between processes.

No reference counterpart: the reference calls cuBLAS/cuSOLVER with their
own heuristics (mnpbem/utils/gpu.py:145-251).
"""

import json
import os

import torch

from . import _lib

__all__ = ["GemmTuner", "set_gemm_config", "DEFAULT_CONFIG"]

# (tile width for N > 64, persistent from tiles per SM (0 = never), ring stages (0 = max))
DEFAULT_CONFIG = (128, 2, 0)
CANDIDATES = ((128, 2, 0), (128, 1, 0), (128, 4, 0), (128, 0, 0), (64, 2, 0), (128, 2, 2))


def set_gemm_config(cfg):
    """Apply a (bn_wide, persist_tiles_per_sm, stages) launch configuration."""
    _lib.call('mnpb_gemm_config', int(cfg[0]), int(cfg[1]), int(cfg[2]))


class GemmTuner(object):
    """Per-key choice of the GEMM launch configuration, measured on the
    caller's workload with CUDA events."""

    def __init__(self, path=None, candidates=CANDIDATES, repeats=1):
        self.path = path
        self.candidates = [tuple(c) for c in candidates]
        self.repeats = int(repeats)
        self.table = {}
        self.timings = {}
        if path and os.path.exists(path):
            with open(path) as f:
                self.table = {k: tuple(v) for k, v in json.load(f).items()}

    @staticmethod
    def _key(key):
        return key if isinstance(key, str) else '/'.join(str(k) for k in key)

    def _time(self, run):
        run()                                  # warm: graphs, attributes, caches
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(self.repeats):
            run()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / self.repeats

    def choose(self, key, run):
        """Apply the best configuration for ``key``, timing every candidate
        with ``run`` the first time the key is seen.  Returns the choice."""
        k = self._key(key)
        if k not in self.table:
            times = {}
            try:
                for cfg in self.candidates:
                    set_gemm_config(cfg)
                    times[cfg] = self._time(run)
            finally:
                set_gemm_config(DEFAULT_CONFIG)
            best = min(times, key=times.get)
            self.table[k] = best
            self.timings[k] = {'/'.join(map(str, c)): round(t, 4) for c, t in times.items()}
            self.save()
        set_gemm_config(self.table[k])
        return self.table[k]

    def save(self):
        if self.path:
            with open(self.path, 'w') as f:
                json.dump({k: list(v) for k, v in self.table.items()}, f, indent=1)
