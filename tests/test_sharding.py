"""Multi-GPU path on the CPU: world size 2 over gloo.

Each rank integrates its own contiguous range of orbits (here with the CPU
oracle standing in for a GPU) with global orbit indices, so the union of the
shards equals one unsharded run bit for bit -- Euler-Maruyama included, whose
noise is keyed by the global orbit index -- and the job time is the max over
ranks."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sodecl_b200.sharding import max_over_ranks, shard


def test_shard_ranges_cover_all_orbits():
    for n in (0, 1, 7, 1000, 1 << 20):
        for world in (1, 2, 3, 8):
            ranges = [shard(n, r, world) for r in range(world)]
            assert sum(c for _, c in ranges) == n
            assert all(ranges[r][0] + ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
            assert max(c for _, c in ranges) - min(c for _, c in ranges) <= 1
    with pytest.raises(ValueError):
        shard(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from oracle.oracle import Oracle

    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    n_total, N = 37, 4
    rng = np.random.default_rng(5)
    p = np.concatenate([rng.uniform(0, 5, (n_total, 1)), rng.normal(size=(n_total, N)),
                        rng.uniform(0, 0.5, (n_total, N))], axis=1)
    y0 = rng.uniform(0, 2 * np.pi, (n_total, N))
    cnt = np.arange(n_total) * 64.0
    first, count = shard(n_total, rank, world)
    sl = slice(first, first + count)
    r = Oracle("kuramoto").run(0, np.zeros(count), y0[sl], p[sl], counters=cnt[sl], orbit_offset=first, neq=N,
                               npar=2 * N + 1, nnoi=N, dt=0.01, ksteps=10, nchunks=5)
    np.save(os.path.join(out_dir, "rank%d.npy" % rank), r.records)
    slowest = max_over_ranks(1.0 + rank, dist)
    np.save(os.path.join(out_dir, "max%d.npy" % rank), np.array([slowest]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharding_equals_single_run(tmp_path):
    from oracle.oracle import Oracle

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    parts = [np.load(tmp_path / ("rank%d.npy" % r)) for r in range(world)]
    n_total, N = 37, 4
    rng = np.random.default_rng(5)
    p = np.concatenate([rng.uniform(0, 5, (n_total, 1)), rng.normal(size=(n_total, N)),
                        rng.uniform(0, 0.5, (n_total, N))], axis=1)
    y0 = rng.uniform(0, 2 * np.pi, (n_total, N))
    whole = Oracle("kuramoto").run(0, np.zeros(n_total), y0, p, counters=np.arange(n_total) * 64.0, neq=N,
                                   npar=2 * N + 1, nnoi=N, dt=0.01, ksteps=10, nchunks=5).records
    np.testing.assert_array_equal(np.concatenate(parts, axis=2), whole)
    assert all(float(np.load(tmp_path / ("max%d.npy" % r))[0]) == 2.0 for r in range(world))
