"""Instance sharding across ranks: the balanced partition, and the gather of
per-instance results and the max over ranks with two gloo ranks on the CPU
(the collectives the multi-GPU path uses; the simulation itself runs per rank
with no exchange)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from diffcp_b200 import sharding


def test_partition_covers_every_instance_once_and_balances():
    rng = np.random.default_rng(0)
    sizes = rng.integers(100, 30000, 257)
    for world in (1, 2, 3, 8):
        parts = sharding.partition(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        assert all(p == sorted(p) for p in parts)
        loads = [sizes[p].sum() for p in parts]
        assert max(loads) - min(loads) <= sizes.max()


def test_partition_with_more_ranks_than_instances():
    parts = sharding.partition([5, 3], 4)
    assert sorted(i for p in parts for i in p) == [0, 1]
    assert sum(1 for p in parts if not p) == 2


def test_gather_rows_without_a_process_group():
    rows = np.arange(12.0).reshape(4, 3)
    out = sharding.gather_rows(rows[[2, 0, 3, 1]], [2, 0, 3, 1], 4)
    np.testing.assert_array_equal(out, rows)
    assert sharding.max_over_ranks(3.5) == 3.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, sizes, outdir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        idx = sharding.partition(sizes, world)[rank]
        local = np.stack([np.array([10.0 * i, i + 0.5]) for i in idx]) if idx else np.zeros((0, 2))
        full = sharding.gather_rows(local, idx, len(sizes))
        mx = sharding.max_over_ranks(1.0 + rank)
        np.save(os.path.join(outdir, "r%d.npy" % rank), np.concatenate([full.ravel(), [mx]]))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
    sizes = [400, 90, 3000, 25, 1200, 800, 64]
    world = 2
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank_main, args=(world, _free_port(), sizes, d), nprocs=world, join=True)
        want = np.concatenate([np.stack([[10.0 * i, i + 0.5] for i in range(len(sizes))]).ravel(), [2.0]])
        for r in range(world):
            np.testing.assert_array_equal(np.load(os.path.join(d, "r%d.npy" % r)), want)
