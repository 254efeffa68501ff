"""Multi-rank sweep logic on CPU: two gloo ranks share out a wavelength list,
each "solves" its own (a host function standing in for the GPU solve), and
the all-gather rebuilds the full table in order on both ranks; the max over
ranks is the slowest rank's time."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from mnpbem_b200.replicas import shard


def test_shard_covers_each_item_once():
    for world in (1, 2, 3, 8):
        for mode in ('interleaved', 'contiguous'):
            got = np.sort(np.concatenate([shard(81, r, world, mode) for r in range(world)]))
            assert np.array_equal(got, np.arange(81))
    assert list(shard(10, 1, 4)) == [1, 5, 9]
    with pytest.raises(ValueError):
        shard(10, 4, 4)


def _fake_solve(enei):
    return [enei, np.sin(enei), enei ** 2]


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    from mnpbem_b200.replicas import max_over_ranks, sweep
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        eneis = list(np.linspace(400.0, 800.0, 13))
        table = sweep(_fake_solve, eneis)
        slowest = max_over_ranks(10.0 + rank)
        np.save(os.path.join(outdir, 'r%d.npy' % rank), np.append(table.ravel(), slowest))
    finally:
        dist.destroy_process_group()


def test_sweep_two_gloo_ranks():
    import socket
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_worker, args=(2, port, d), nprocs=2, join=True)
        eneis = np.linspace(400.0, 800.0, 13)
        ref = np.array([_fake_solve(e) for e in eneis])
        for r in range(2):
            got = np.load(os.path.join(d, 'r%d.npy' % r))
            assert np.allclose(got[:-1].reshape(13, 3), ref, rtol=0, atol=0)
            assert got[-1] == 11.0
