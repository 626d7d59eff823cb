"""The compiled CPU restatement of the substep and its adjoint
(oracle/cpu_port.cpp), which bench.py times as the CPU baseline: its float64
build against the FP64 torch oracle (loss, every parameter gradient, the
gripper-velocity gradient), and its parallel float32 runs.  CPU only."""
import numpy as np
import pytest
import torch

from oracle import cpu_port
from tests.scenes import oracle_loss, oracle_params, small_sheet

KEYS = ("E", "nu", "ks", "kc", "friction", "damping")


@pytest.mark.parametrize("seed,friction", [(3, 0.3), (5, 0.1)])
def test_float64_build_matches_oracle(seed, friction):
    n = 30
    sc = small_sheet(n_steps=n, seed=seed, friction=friction)
    loss, g, gv = cpu_port.rollout_grad(sc, n, double=True)
    p = oracle_params(sc, requires_grad=True)
    vel = torch.tensor(sc.velocities, dtype=torch.float64, requires_grad=True)
    lo, p, _, vel, _ = oracle_loss(sc, n, n, params=p, vel=vel)
    lo.backward()
    assert loss == pytest.approx(float(lo.detach()), rel=1e-12)
    for j, k in enumerate(KEYS):
        r = float(p[k].grad)
        assert g[j] == pytest.approx(r, rel=1e-9, abs=1e-30), (k, g[j], r)
    rv = vel.grad.numpy()
    assert np.abs(gv - rv).max() <= 1e-10 * np.abs(rv).max()


def test_parallel_float32_rollouts_run_every_cloth():
    n = 12
    scenes = [small_sheet(n=5 + i, n_steps=n, seed=i) for i in range(3)]
    losses, grads = cpu_port.rollouts(scenes, n, n_threads=2)
    for i, sc in enumerate(scenes):
        l64, g64, _ = cpu_port.rollout_grad(sc, n, double=True)
        assert losses[i] == pytest.approx(l64, rel=1e-4)
        assert np.all(np.isfinite(grads[i]))
