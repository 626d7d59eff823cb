"""Shared test scenes: the small reference scene (the one the golden vectors
were generated on) as a product ClothScene, and small kinematic sheets, each
with the matching oracle set-up."""
from __future__ import annotations

import random

import numpy as np
import torch

from diffcp_b200 import scene as dscene
from oracle import sim64
from oracle.sim64 import Constants, KinematicGripper, OracleSim
from tests.golden import make_golden as mg


def reference_small_scene(variant="base"):
    """The synthetic scene of the golden vectors as a product ClothScene;
    variant "press" is the 300-substep scene whose grasp presses the sheet's
    corners down (ref_fd_press_f64.npz)."""
    verts, tris, traj, target, mark = mg.scene_arrays(variant)
    args = mg.ARGS_PRESS if variant == "press" else mg.ARGS
    random.seed(mg.SEED_OP)
    np.random.seed(mg.SEED_CUBE)
    n_c = args["rigid_cube_parameters"]["n_rigid_cube_particles"]
    cube_random = np.random.rand(n_c, 3)
    group = args["operator_parameters"]["n_operator_particles"] // traj.shape[1]
    op_random = np.array([[random.random(), random.random(), random.random()] for _ in range(group)])
    sc = dscene.reference_scene(args, verts, tris, traj, target, mark, op_random, cube_random)
    p = mg.PARAMS_PRESS if variant == "press" else mg.PARAMS
    sc.params.update({"E": p["E"], "nu": p["nu"], "shearing_stiffness": p["shearing_stiffness"],
                      "contact_stiffness": p["contact_stiffness"]})
    return sc


def oracle_for(sc: dscene.ClothScene, dtype=torch.float64, svd_grad="exact", device=None):
    """Oracle simulator + state 0 for a product scene."""
    const = Constants(
        n_grid=sc.n_grid, dt=float(sc.meta["dt"]), vertex_p_mass=sc.vertex_p_mass,
        quadrature_p_mass=sc.quadrature_p_mass, quadrature_p_vol=sc.quadrature_p_vol,
        operator_p_mass=sc.operator_p_mass, cube_p_mass=sc.cube_p_mass, gravity_dv=sc.gravity_dv, bound=sc.bound,
        operator_update_interval=sc.keyframe_interval, frames_per_window=sc.frames_per_window,
        grasper_group_size=max(sc.group_size, 1), n_actions=0 if sc.keyframes is None else sc.keyframes.shape[0])
    return OracleSim.initialize(const, sc.vertices, sc.triangles, sc.operator_x, sc.cube_x, dtype=dtype,
                                svd_grad=svd_grad, device=device)


def oracle_params(sc, dtype=torch.float64, requires_grad=False):
    p = sc.params
    out = {"E": p["E"], "nu": p["nu"], "ks": p["shearing_stiffness"], "kc": p["contact_stiffness"],
           "friction": p.get("friction", 0.0), "damping": p.get("damping", 0.95)}
    return {k: torch.tensor(float(v), dtype=dtype, requires_grad=requires_grad) for k, v in out.items()}


def oracle_loss(sc, n_steps, loss_step, window=0, dtype=torch.float64, svd_grad="exact", params=None, seq=None,
                vel=None, targets=None):
    """Loss of the oracle rollout; returns (loss, params, seq, vel, states)."""
    sim, st = oracle_for(sc, dtype, svd_grad)
    params = params or oracle_params(sc, dtype)
    grip = None
    if sc.gripper_mode == 2:
        vel = vel if vel is not None else torch.tensor(sc.velocities, dtype=dtype)
        grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=dtype), vel)
    if sc.gripper_mode == 1 and seq is None:
        seq = torch.tensor(sc.keyframes, dtype=dtype)
    fr = params["friction"] if sc.gripper_mode == 2 or float(params["friction"]) != 0.0 else None
    states = [st]
    for f in range(n_steps):
        st = sim.substep(st, f, window, params, seq=seq, friction=fr, damping=params["damping"], grip=grip)
        states.append(st)
    tg = torch.tensor(np.asarray(sc.targets if targets is None else targets), dtype=dtype)
    loss, arg = sim64.compute_loss(states[loss_step]["vx"], tg)
    return loss, params, seq, vel, states


def small_sheet(n=6, n_grid=24, n_steps=30, seed=3, friction=0.3, damping=0.95, E=3e3, nu=0.3, dt=2e-4,
                velocities=None, side=None, height=0.12):
    side = side if side is not None else (n - 1) * 0.2 / 31 * 3
    if velocities is None:
        rng = np.random.default_rng(seed + 100)
        velocities = np.repeat(rng.normal(0.0, 0.05, (1, 2, 3)), n_steps, 0) + rng.normal(0.0, 0.01, (n_steps, 2, 3))
    sc = dscene.sheet_scene(n=n, side=side, height=height, n_grid=n_grid, dt=dt, n_steps=n_steps, E=E, nu=nu,
                            friction=friction, damping=damping, seed=seed, n_targets=64, velocities=velocities)
    sc.targets = sc.targets + np.array([0.0, -0.01, 0.0])
    return sc
