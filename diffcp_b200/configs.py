"""The benchmark configurations as seeded synthetic scenes.

  single_sheet     a 32x32-vertex, 0.2 m sheet, 64^3 grid, dt 2e-4, 200 substeps,
                   E 5e3, nu 0.3, friction 0.3, two adjacent corners on cubic
                   splines (5 control points, +-5 cm); Chamfer to 2048 points of
                   the final state of the same run with E 8e3, nu 0.25
  large_sheet      a 128x128-vertex, 0.4 m sheet, 128^3 grid, dt 1e-4, 1000
                   substeps, checkpoints every 50
  parameter_sweep  256 sheets, side U{16..96} vertices at the single sheet's
                   spacing, E log-U[1e3, 1e5], nu U[0.1, 0.45], friction
                   U[0.1, 0.6], own splines, 64^3 grid each, 300 substeps
  trajectory_batch 64 sheets of 64x64 vertices, 96^3 grids, 400 substeps, per-
                   substep gripper velocities N(0, 0.01 m/s); targets from the
                   final state under another velocity draw
  stress_sheet     a 512x512-vertex sheet of 1 m side, 256^3 grid, dt 5e-5,
                   2000 substeps, checkpoints every 45; the domain is the unit
                   cube with 3-cell sticky walls (interior 0.977 m wide), so
                   the sheet's rest shape is a shallow bowl (radius 0.8 m:
                   0.936 m wide, edges still 1/511 m) and its grasped corners
                   move by up to 1 cm instead of 5

Targets that come from a simulated final state are computed with this
library on the GPU (``final_state_targets``).
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import scene

SPACING = 0.2 / 31    # vertex spacing of the single sheet


def final_state_targets(scenes: Sequence[scene.ClothScene], n_steps: int, n_targets: int, seed: int,
                        params: Dict[str, float] = None, velocities: Sequence[np.ndarray] = None,
                        device=None) -> List[np.ndarray]:
    """Area-uniform samples of each cloth's surface after ``n_steps`` forward
    substeps, run with ``params`` overriding the scenes' parameters and/or
    ``velocities`` replacing kinematic gripper velocities."""
    import copy

    from .batch import ClothBatch
    runs = []
    for i, sc in enumerate(scenes):
        s2 = copy.deepcopy(sc)
        if params:
            s2.params.update(params)
        if velocities is not None:
            v = np.asarray(velocities[i], dtype=np.float64)
            s2.velocities = v
            s2.centers = s2.centers[:1] + sc.meta["dt"] * np.concatenate(
                [np.zeros((1,) + v.shape[1:]), np.cumsum(v, 0)[:-1]], 0)
        runs.append(s2)
    b = ClothBatch(runs, dt=runs[0].meta["dt"], device=device)
    s = b.init_state()
    t = b.new_state()
    for f in range(n_steps):
        b.forward_step(s, f, out=t)
        s, t = t, s
    rng = np.random.default_rng(seed)
    out = []
    for i, sc in enumerate(scenes):
        v = b.vertex_x(s, i).double().cpu().numpy()
        out.append(scene.surface_samples(v, np.asarray(sc.triangles), n_targets, rng))
    b.close()
    return out


def single_sheet(seed: int = 0, with_targets: bool = True, device=None) -> Tuple[List[scene.ClothScene], dict]:
    sc = scene.sheet_scene(n=32, side=0.2, height=0.3, n_grid=64, dt=2e-4, n_steps=200, E=5e3, nu=0.3,
                           friction=0.3, seed=seed, n_targets=2048)
    if with_targets:
        sc.targets = final_state_targets([sc], 200, 2048, seed + 17, params={"E": 8e3, "nu": 0.25},
                                         device=device)[0]
    return [sc], dict(dt=2e-4, n_steps=200, ckpt_every=1,
                      desc="single cloth 32x32 vertices, 0.2 m, 64^3 grid, dt 2e-4, 200 substeps, targets from "
                           "the E 8e3 / nu 0.25 final state")


def large_sheet(seed: int = 0) -> Tuple[List[scene.ClothScene], dict]:
    return [scene.sheet_scene(n=128, side=0.4, height=0.3, n_grid=128, dt=1e-4, n_steps=1000, seed=seed,
                              n_targets=2048)], dict(
        dt=1e-4, n_steps=1000, ckpt_every=50,
        desc="single cloth 128x128 vertices, 0.4 m, 128^3 grid, dt 1e-4, 1000 substeps, checkpoints every 50")


def parameter_sweep(seed: int = 0, count: int = 256) -> Tuple[List[scene.ClothScene], dict]:
    """dt is not fixed by the configuration; 1e-4 keeps the stiffest draw
    (2 mu + lambda ~ 3.8e5 Pa) inside the explicit stability limit, which
    2e-4 does not."""
    rng = np.random.default_rng(seed)
    scenes = []
    for i in range(count):
        n = int(rng.integers(16, 97))
        E = float(10 ** rng.uniform(3, 5))
        nu = float(rng.uniform(0.1, 0.45))
        fr = float(rng.uniform(0.1, 0.6))
        scenes.append(scene.sheet_scene(n=n, side=(n - 1) * SPACING, height=0.3, n_grid=64, dt=1e-4, n_steps=300,
                                        E=E, nu=nu, friction=fr, seed=seed * 1000 + i, n_targets=2048))
    return scenes, dict(dt=1e-4, n_steps=300, ckpt_every=1,
                        desc="batched parameter sweep: %d cloths, side U{16..96} vertices, 64^3 grid each, dt 1e-4, "
                             "300 substeps, Chamfer to 2048 targets each" % count)


def trajectory_batch(seed: int = 0, count: int = 64, n: int = 64, n_steps: int = 400, dt: float = 1e-4,
                     with_targets: bool = True, device=None) -> Tuple[List[scene.ClothScene], dict]:
    rng = np.random.default_rng(seed)
    scenes, other = [], []
    for i in range(count):
        vel = rng.normal(0.0, 0.01, (n_steps, 2, 3))
        other.append(rng.normal(0.0, 0.01, (n_steps, 2, 3)))
        scenes.append(scene.sheet_scene(n=n, side=(n - 1) * SPACING, height=0.3, n_grid=96, dt=dt, n_steps=n_steps,
                                        seed=seed * 1000 + i, n_targets=2048, velocities=vel))
    if with_targets:
        tg = final_state_targets(scenes, n_steps, 2048, seed + 29, velocities=other, device=device)
        for sc, t in zip(scenes, tg):
            sc.targets = t
    return scenes, dict(dt=dt, n_steps=n_steps, ckpt_every=1,
                        desc="batched trajectory optimisation: %d cloths of %dx%d vertices, 96^3 grids, %d substeps, "
                             "per-substep gripper velocities" % (count, n, n, n_steps))


def stress_sheet(seed: int = 0) -> Tuple[List[scene.ClothScene], dict]:
    return [scene.sheet_scene(n=512, side=1.0, height=0.2, n_grid=256, dt=5e-5, n_steps=2000, seed=seed,
                              n_targets=2048, cap_radius=0.8, grasp_amplitude=0.01)], dict(
        dt=5e-5, n_steps=2000, ckpt_every=45, pool_blocks="auto",
        desc="stress: one cloth 512x512 vertices, 1 m side (bowl-shaped rest, 0.936 m wide), 256^3 grid paged "
             "through a pool of 4^3-node blocks, dt 5e-5, 2000 substeps, checkpoints every 45")
