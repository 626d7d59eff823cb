"""Grasp-trajectory optimisation by gradient descent.

The reference's script (gradient_descent_for_traj_generation.py:1-71, with
trajectory_generation_functions_and_variables.py:6-22) intends to move the
grasp trajectory down the gradient of the Chamfer loss: per epoch one
tape-recorded window, ``grasp_tracking_seq -= learning_rate[action] * grad``
with NaN gradients mapped to 0, and five rounds with the learning rate cut by
10 each, saving the losses, Chamfer distances and trajectories.  As shipped it
does not run (it calls the parameter-fitting loop instead of its own, indexes
the trajectory field with the wrong rank, and reloads the original keyframes
at every epoch); this module is the working version, batched: every cloth of a :class:`~diffcp_b200.batch.BatchSim` has
its own trajectory and target, and one batched forward + adjoint per epoch
gives all their gradients.

Leaves: the keyframes of momentum-injecting grippers, or the per-substep
velocities of kinematic grippers (whose centres are re-integrated from the
velocities after every update).
"""
from __future__ import annotations

import argparse
import json
import os
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import native


def compute_chamfer_distance(array1: np.ndarray, array2: np.ndarray) -> float:
    """Mean over the points of ``array1`` of the Euclidean distance to the
    nearest point of ``array2`` (trajectory_generation_functions_and_variables.py:6-10)."""
    a = torch.as_tensor(np.asarray(array1, dtype=np.float64))
    b = torch.as_tensor(np.asarray(array2, dtype=np.float64))
    best = torch.full((a.shape[0],), float("inf"), dtype=torch.float64)
    for s in range(0, b.shape[0], 4096):
        best = torch.minimum(best, torch.cdist(a, b[s: s + 4096]).min(dim=1).values)
    return float(best.mean())


def interpolate_trajectory(trajectory: np.ndarray, total_length: int) -> np.ndarray:
    """Piecewise-linear resampling of an (n, 3) path to ``total_length``
    points with the same end points (trajectory_generation_functions_and_variables.py:12-19)."""
    tr = np.asarray(trajectory, dtype=np.float64)
    old = np.linspace(0, len(tr) - 1, len(tr))
    new = np.linspace(0, len(tr) - 1, total_length)
    return np.stack([np.interp(new, old, tr[:, i]) for i in range(3)], axis=1)


def _leaf_mask(batch) -> torch.Tensor:
    """1 on the trajectory-table entries that are optimised (keyframes or
    kinematic velocities), 0 on kinematic centres."""
    m = torch.zeros_like(batch.traj)
    for i, sc in enumerate(batch.scenes):
        off, ln = batch.traj_slices(i)
        if sc.gripper_mode == native.GRIP_KINEMATIC:
            m[off: off + ln // 2] = 1
        else:
            m[off: off + ln] = 1
    return m


def sync_centres(batch, traj: torch.Tensor) -> None:
    """Re-integrate each kinematic gripper's per-substep centres from its
    velocities: c[0] fixed, c[f+1] = c[f] + dt v[f]."""
    for i, sc in enumerate(batch.scenes):
        if sc.gripper_mode != native.GRIP_KINEMATIC:
            continue
        off, ln = batch.traj_slices(i)
        h = ln // 2
        vel = traj[off: off + h].view(sc.velocities.shape).double()
        c0 = torch.as_tensor(np.asarray(sc.centers)[0], dtype=torch.float64, device=traj.device)
        cen = torch.cat([c0[None], c0[None] + batch.dt * torch.cumsum(vel, 0)[:-1]], 0)
        traj[off + h: off + ln] = cen.reshape(-1).to(traj.dtype)


def traj_optimization(sim, epochs: int, lr: float, traj: Optional[torch.Tensor] = None,
                      params: Optional[torch.Tensor] = None, targets: Optional[Sequence[np.ndarray]] = None,
                      log=None) -> Dict[str, object]:
    """traj_optimization of gradient_descent_for_traj_generation.py:28-47 for
    every cloth of ``sim`` at once.  Returns {"loss": (epochs, n), "chamfer":
    (epochs, n) mean target-to-cloth distance at the rollout's last state,
    "traj": the updated trajectory table}."""
    b = sim.batch
    traj = (b.traj if traj is None else traj).detach().clone()
    params = b.params if params is None else params
    mask = _leaf_mask(b)
    tg = [np.asarray(t) for t in (targets if targets is not None else [sc.targets for sc in b.scenes])]
    losses, chamfers = [], []
    for e in range(epochs):
        leaf = traj.clone().requires_grad_(True)
        loss = sim.loss(params, leaf)
        loss.sum().backward()
        g = torch.nan_to_num(leaf.grad) * mask
        losses.append(loss.detach().cpu().numpy().astype(np.float64))
        fin = sim.final_state
        chamfers.append(np.array([compute_chamfer_distance(tg[i], b.vertex_x(fin, i).cpu().numpy())
                                  for i in range(b.n_inst)]))
        if log:
            log("epoch %d: mean loss %.6g, mean chamfer %.6g" % (e, losses[-1].mean(), chamfers[-1].mean()))
        with torch.no_grad():
            traj -= lr * g.to(traj.dtype)
            sync_centres(b, traj)
    return {"loss": np.array(losses), "chamfer": np.array(chamfers), "traj": traj}


def gradient_descent(sim, epochs: int, lr0: float = 1e-13, rounds: int = 5, log=None) -> Dict[str, np.ndarray]:
    """The script's outer loop (gradient_descent_for_traj_generation.py:58-71):
    ``rounds`` optimisations, the learning rate divided by 10 before each,
    each round continuing from the previous round's trajectory (in the
    reference every epoch's initialize_objects reloads the original keyframes,
    so no update would survive).  Returns the arrays the script saves
    (GD_loss, GD_chamfer_distances, GD_trajectories)."""
    lr = lr0
    traj = None
    out_l, out_c, out_t = [], [], []
    for _ in range(rounds):
        lr *= 0.1
        r = traj_optimization(sim, epochs, lr, traj=traj, log=log)
        traj = r["traj"]
        out_l.append(r["loss"])
        out_c.append(r["chamfer"])
        out_t.append(r["traj"].cpu().numpy())
    return {"GD_loss": np.array(out_l), "GD_chamfer_distances": np.array(out_c),
            "GD_trajectories": np.array(out_t)}


def main(argv: Optional[Sequence[str]] = None) -> Dict[str, np.ndarray]:
    """The script as a command: fitted parameters from
    ``<result dir>/fitting_result.json``, target cloud from
    ``<data dir>/target_point_cloud.npy``, results saved as .npy files in the
    result directory."""
    ap = argparse.ArgumentParser(prog="python -m diffcp_b200.trajopt")
    ap.add_argument("--src", required=True)
    ap.add_argument("--epochs", type=int, default=500)
    ap.add_argument("--rounds", type=int, default=5)
    ap.add_argument("--lr", type=float, default=1e-13)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--target", default=None)
    ap.add_argument("--params", default=None)
    ap.add_argument("--scene-target", action="store_true",
                    help="scale and re-centre the target cloud like the scene's data")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    from .batch import BatchSim, ClothBatch
    from .scene import load_reference_scene
    with open(os.path.join(a.src, "simulation_arguments.json")) as fh:
        args = json.load(fh)
    result_dir = a.src + args["result_dir"]
    with open(a.params or os.path.join(result_dir, "fitting_result.json")) as fh:
        fit = json.load(fh)
    sc = load_reference_scene(a.src, seed=a.seed, args=args)
    for k in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        sc.params[k] = fit[k]
    raw = np.asarray(np.load(a.target or os.path.join(a.src + args["data_dir"], "target_point_cloud.npy")),
                     dtype=np.float64).reshape(-1, 3)
    # the reference uploads the cloud as loaded; --scene-target applies the scene's scale and shift
    sc.targets = raw * sc.meta["scene_scaling"] + sc.meta["shift"] if a.scene_target else raw
    b = ClothBatch([sc], dt=sc.meta["dt"])
    n = int(sc.meta["max_steps"]) - 1
    sim = BatchSim(b, n_steps=n, loss_step=n - 2, ckpt_every=1)
    res = gradient_descent(sim, a.epochs, a.lr, a.rounds, log=None if a.quiet else print)
    for k, v in res.items():
        np.save(os.path.join(result_dir, k + ".npy"), v)
    return res


if __name__ == "__main__":
    main()
