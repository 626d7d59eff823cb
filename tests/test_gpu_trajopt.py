"""Trajectory optimisation on the GPU: the batched trajectory gradient against
central finite differences of the FP64 oracle, and gradient descent on the
per-substep gripper velocities of several cloths at once."""
import numpy as np
import pytest
import torch

from tests.scenes import oracle_loss, small_sheet

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _sim(scenes, n):
    from diffcp_b200.batch import BatchSim, ClothBatch
    b = ClothBatch(scenes, dt=scenes[0].meta["dt"])
    return BatchSim(b, n_steps=n, loss_step=n, ckpt_every=4)


def test_trajectory_gradient_matches_oracle_finite_differences():
    n = 12
    scenes = [small_sheet(n=5, n_steps=n, seed=7), small_sheet(n=6, n_steps=n, seed=8, E=6e3)]
    sim = _sim(scenes, n)
    b = sim.batch
    traj = b.traj.clone().requires_grad_(True)
    sim.loss(b.params, traj).sum().backward()
    g = traj.grad.double().cpu().numpy()
    rng = np.random.default_rng(5)
    for i, sc in enumerate(scenes):
        off, _ = b.traj_slices(i)
        gv = g[off: off + sc.velocities.size].reshape(sc.velocities.shape)
        scale = np.abs(gv).max()
        for _ in range(16):
            c = tuple(int(rng.integers(0, s)) for s in sc.velocities.shape)
            h = 1e-4
            vals = []
            for sgn in (1, -1):
                v = sc.velocities.copy()
                v[c] += sgn * h
                vals.append(float(oracle_loss(sc, n, n, vel=torch.tensor(v, dtype=torch.float64))[0]))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(gv[c] - fd) <= 2e-4 * scale, (i, c, gv[c], fd, scale)


def test_gradient_descent_on_velocities_lowers_every_cloths_loss():
    from diffcp_b200 import trajopt
    n = 16
    scenes = []
    for k, seed in enumerate((11, 12, 13)):
        sc = small_sheet(n=6, n_steps=n, seed=seed)
        # targets: where the cloth ends up under a different grasp
        tgt = small_sheet(n=6, n_steps=n, seed=seed + 50)
        s0 = _sim([tgt], n)
        s0.loss(s0.batch.params, s0.batch.traj)
        sc.targets = s0.batch.vertex_x(s0.final_state, 0).double().cpu().numpy()
        scenes.append(sc)
    sim = _sim(scenes, n)
    b = sim.batch
    probe = b.traj.clone().requires_grad_(True)
    sim.loss(b.params, probe).sum().backward()
    lr = 0.02 * float(np.abs(scenes[0].velocities).max()) / float(probe.grad.abs().max())
    res = trajopt.traj_optimization(sim, 6, lr)
    assert res["loss"].shape == (6, 3) and res["chamfer"].shape == (6, 3)
    assert np.all(res["loss"][-1] < res["loss"][0]), res["loss"]
    # kinematic centres follow the updated velocities
    for i, sc in enumerate(scenes):
        off, ln = b.traj_slices(i)
        t = res["traj"][off: off + ln].double().cpu().numpy()
        vel = t[: ln // 2].reshape(sc.velocities.shape)
        cen = t[ln // 2:].reshape(sc.velocities.shape)
        np.testing.assert_allclose(cen[1:], cen[:-1] + sc.meta["dt"] * vel[:-1], rtol=0, atol=1e-6)
    out = trajopt.gradient_descent(sim, 2, lr0=lr * 10, rounds=2)
    assert out["GD_loss"].shape == (2, 2, 3) and out["GD_trajectories"].shape[0] == 2


def test_command_line_saves_the_scripts_arrays(tmp_path):
    import json
    import os

    from diffcp_b200 import trajopt
    from tests.golden import make_golden as mg
    from tests.ref_tree import write_tree
    src = write_tree(tmp_path)
    result = os.path.join(src, "..", "result")
    os.makedirs(result, exist_ok=True)
    with open(os.path.join(result, "fitting_result.json"), "w") as fh:
        json.dump(mg.PARAMS, fh)
    _, _, _, target, _ = mg.scene_arrays()
    np.save(os.path.join(src, "..", "data", "target_point_cloud.npy"), target[-1])
    res = trajopt.main(["--src", src, "--epochs", "2", "--rounds", "2", "--lr", "1e-3", "--seed", str(mg.SEED_OP),
                        "--scene-target", "--quiet"])
    for k in ("GD_loss", "GD_chamfer_distances", "GD_trajectories"):
        saved = np.load(os.path.join(result, k + ".npy"))
        np.testing.assert_array_equal(saved, res[k])
    assert res["GD_loss"].shape == (2, 2, 1) and np.isfinite(res["GD_loss"]).all()
