"""Shards of a batch simulated separately give the same per-instance losses
and gradients as the whole batch (the multi-GPU path runs one shard per GPU
with no exchange; here both shards run on one GPU, one after the other)."""
import numpy as np
import pytest
import torch

from diffcp_b200 import sharding
from tests.scenes import small_sheet

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def test_two_shards_equal_the_whole_batch():
    n = 12
    scenes = [small_sheet(n=5 + (k % 3), seed=20 + k, n_steps=n, E=3e3 + 1e3 * k) for k in range(5)]
    dt = scenes[0].meta["dt"]
    lo, gp = sharding.sharded_loss_and_grads(scenes, n, 0, 1, dt, ckpt_every=4)
    got_lo, got_gp = np.zeros_like(lo), np.zeros_like(gp)
    for r in range(2):
        idx, mine = sharding.my_shard(scenes, r, 2)
        l, g = sharding.sharded_loss_and_grads(mine, n, 0, 1, dt, ckpt_every=4)
        got_lo[idx], got_gp[idx] = l, g
    np.testing.assert_allclose(got_lo, lo, rtol=1e-6)
    np.testing.assert_allclose(got_gp[:, :6], gp[:, :6], rtol=1e-4, atol=1e-16)
