"""Host helpers of the trajectory optimisation against the library calls the
reference makes (scipy cdist / interp1d in
trajectory_generation_functions_and_variables.py:6-19), and the oracle's
kinematic-gripper gradients against central finite differences (the
kinematic gripper and ground friction have no reference counterpart, so FD
of the FP64 oracle pins them)."""
import numpy as np
import pytest
import scipy.spatial
import torch
from scipy.interpolate import interp1d

from diffcp_b200 import trajopt
from tests.scenes import oracle_loss, oracle_params, small_sheet


def test_chamfer_distance_matches_scipy():
    rng = np.random.default_rng(1)
    a, b = rng.random((300, 3)), rng.random((5000, 3))
    want = np.mean(np.min(scipy.spatial.distance.cdist(a, b), axis=1))
    assert trajopt.compute_chamfer_distance(a, b) == pytest.approx(want, rel=1e-12)


def test_interpolate_trajectory_matches_interp1d():
    rng = np.random.default_rng(2)
    tr = rng.random((7, 3))
    old = np.linspace(0, 6, 7)
    new = np.linspace(0, 6, 40)
    want = np.vstack([interp1d(old, tr[:, i], kind="linear")(new) for i in range(3)]).T
    np.testing.assert_allclose(trajopt.interpolate_trajectory(tr, 40), want, rtol=0, atol=1e-15)


def test_oracle_kinematic_gradients_match_finite_differences():
    n = 10
    sc = small_sheet(n=5, n_steps=n, seed=7)
    p = oracle_params(sc, requires_grad=True)
    vel = torch.tensor(sc.velocities, dtype=torch.float64, requires_grad=True)
    lo, p, _, vel, _ = oracle_loss(sc, n, n, params=p, vel=vel)
    lo.backward()
    rng = np.random.default_rng(0)
    coords = [tuple(int(rng.integers(0, s)) for s in sc.velocities.shape) for _ in range(8)]
    for c in coords:
        h = 1e-4     # h = 1e-3 makes some coordinates cross a stick/slip switch of the ground friction
        vals = []
        for sgn in (1, -1):
            v = sc.velocities.copy()
            v[c] += sgn * h
            vals.append(float(oracle_loss(sc, n, n, vel=torch.tensor(v, dtype=torch.float64))[0]))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert float(vel.grad[c]) == pytest.approx(fd, rel=1e-4, abs=1e-7 * abs(float(lo.detach()))), c
    for k in ("friction", "damping", "E"):
        base = float(p[k].detach())
        h = 1e-4 * max(abs(base), 1e-2)
        vals = []
        for sgn in (1, -1):
            q = oracle_params(sc)
            q[k] = torch.tensor(base + sgn * h, dtype=torch.float64)
            vals.append(float(oracle_loss(sc, n, n, params=q)[0]))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert float(p[k].grad) == pytest.approx(fd, rel=1e-4, abs=1e-9 * abs(float(lo.detach()))), k
