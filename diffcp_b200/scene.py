"""Host-side construction of cloth scenes.

* :func:`reference_scene` -- the reference's scene normalisation and constants
  (src/initialization.py:26-193): scaling, recentring so the scene's bottom
  centre sits at (0.5, 2dx, 0.5), masses and volumes, operator and cube point
  clouds, ``max_steps``.
* :func:`load_reference_scene` -- the same from a reference-style
  ``simulation_arguments.json`` and data directory (PLY mesh, ``.npy`` arrays).
* :func:`sheet_scene` -- a regular square sheet with two kinematic corner
  grippers, the synthetic cloth of the benchmark configurations.
* :func:`morton_order` -- spatially coherent particle order (one-off, at set-up)
  so that a CTA's particles cover a compact grid region.
"""
from __future__ import annotations

import json
import os
import random as _pyrandom
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from . import io_ply
from .native import GRIP_KINEMATIC, GRIP_NONE, GRIP_OPERATOR

GRAVITY = -9.81  # initialization.py:23
BOUND = 3        # initialization.py:22

PARAM_NAMES = ("E", "nu", "shearing_stiffness", "contact_stiffness", "friction", "damping")
REFERENCE_DAMPING = 0.95  # simulation.py:383


@dataclass
class ClothScene:
    """One cloth instance: geometry, constants and gripper description."""
    vertices: np.ndarray                      # (Nv, 3) rest/initial positions in the unit domain
    triangles: np.ndarray                     # (Nt, 3) vertex ids
    n_grid: int
    vertex_p_mass: float
    quadrature_p_mass: float
    quadrature_p_vol: float
    gravity_dv: float
    bound: int = BOUND
    operator_x: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    operator_p_mass: float = 0.0
    cube_x: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    cube_p_mass: float = 0.0
    gripper_mode: int = GRIP_NONE
    n_grippers: int = 0
    group_size: int = 0
    keyframes: Optional[np.ndarray] = None    # mode 1: (n_actions, n_grippers, 3)
    keyframe_interval: float = 0.03
    frames_per_window: int = 0
    gripper_radius: float = 0.0
    velocities: Optional[np.ndarray] = None   # mode 2: (T, K, 3)
    centers: Optional[np.ndarray] = None      # mode 2: (T, K, 3)
    targets: Optional[np.ndarray] = None      # (Nq, 3)
    params: Dict[str, float] = field(default_factory=dict)
    meta: Dict[str, object] = field(default_factory=dict)

    @property
    def n_vertex(self):
        return int(self.vertices.shape[0])

    @property
    def n_tri(self):
        return int(self.triangles.shape[0])

    def param_row(self):
        p = self.params
        return [float(p.get("E", 100.0)), float(p.get("nu", 0.1)), float(p.get("shearing_stiffness", 100.0)),
                float(p.get("contact_stiffness", 100.0)), float(p.get("friction", 0.0)),
                float(p.get("damping", REFERENCE_DAMPING))]


def mesh_area(vertices, triangles) -> float:
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum())


def reference_scene(args: dict, mesh_vertices, mesh_triangles, grasp_seq, target_pcd, mark_pos, operator_random,
                    cube_random) -> ClothScene:
    """Scene of initialization.py:26-193 and initialize_objects
    (simulation.py:432-442).  ``operator_random`` (group, 3) and
    ``cube_random`` (n_cube, 3) are the raw uniform draws of
    initialization.py:166-168 and :85; ``target_pcd`` is (windows, Nq, 3)."""
    op = args["operator_parameters"]
    gp = args["garment_parameters"]
    cube = args["rigid_cube_parameters"]
    dt, n_grid, s = args["dt"], args["n_grid"], args["scene_scaling"]
    interval, gui = args["operator_update_interval"], args["grad_update_interval"]
    initial_frame, end_frame = args["initial_frame"], args["end_frame"]
    garment_mass = gp["garment_mass"] * s ** 3
    dx = 1 / n_grid
    side = cube["rigid_cube_side_length"]
    cube_model = np.asarray(cube_random, dtype=np.float64) * side - side / 2
    cube_model[:, 0] += mark_pos[0]
    cube_model[:, 1] += mark_pos[1] - side / 2
    cube_model[:, 2] += mark_pos[2]
    n_actions = grasp_seq.shape[0]
    if end_frame >= n_actions or end_frame == -1:
        end_frame = n_actions - 1
    if initial_frame > end_frame:
        initial_frame = end_frame - 1
    grasp_seq = np.asarray(grasp_seq, dtype=np.float64)[initial_frame:end_frame + 1] * s
    n_actions = end_frame - initial_frame + 1
    n_grip = grasp_seq.shape[1]
    verts = np.asarray(mesh_vertices, dtype=np.float64) * s
    tris = np.asarray(mesh_triangles, dtype=np.int64)
    cube_model = cube_model * s
    target = np.asarray(target_pcd, dtype=np.float64) * s
    area = mesh_area(verts, tris)
    n_v, n_t = verts.shape[0], tris.shape[0]
    n_op = int(op["n_operator_particles"] / n_grip) * n_grip
    group = n_op // n_grip
    garment_rho = garment_mass / (area * dx)
    edge = op["operator_edge_length"] * s
    op_model = (np.asarray(operator_random, dtype=np.float64) - 0.5) * edge
    scene = np.concatenate((verts, grasp_seq.reshape(-1, 3)))
    center = (scene.max(0) - scene.min(0)) / 2 + scene.min(0)
    shift = np.array([0.5, 2 * dx, 0.5]) - np.array([center[0], 0.0, center[2]])
    verts = verts + shift
    grasp = grasp_seq + shift
    cube_model = cube_model + shift
    target = target + shift
    operator_x = np.concatenate([op_model + grasp[0][g] for g in range(n_grip)])
    sc = ClothScene(
        vertices=verts, triangles=tris, n_grid=n_grid,
        vertex_p_mass=(area * dx / n_v) * garment_rho, quadrature_p_mass=garment_mass / n_v,
        quadrature_p_vol=3 * area * dx / n_t, gravity_dv=dt * s * GRAVITY, bound=BOUND,
        operator_x=operator_x, operator_p_mass=op["operator_mass"] / n_op,
        cube_x=cube_model, cube_p_mass=cube["cube_mass"] / cube_model.shape[0],
        gripper_mode=GRIP_OPERATOR, n_grippers=n_grip, group_size=group, keyframes=grasp,
        keyframe_interval=interval, frames_per_window=int(gui / interval),
        params={"E": gp["initial_constitutive_parameters"]["E"], "nu": gp["initial_constitutive_parameters"]["nu"],
                "shearing_stiffness": gp["initial_constitutive_parameters"]["shearing_stiffness"],
                "contact_stiffness": gp["initial_constitutive_parameters"]["contact_stiffness"],
                "friction": 0.0, "damping": REFERENCE_DAMPING},
        meta={"dt": dt, "max_steps": int(gui / dt) + 1, "targets_by_window": target, "area": area,
              "garment_mass": garment_mass, "n_actions": n_actions, "operator_model": op_model,
              "grad_update_interval": gui, "scene_scaling": s, "shift": shift,
              "bounds": {k: (gp["constitutive_parameter_lower_bounds"][k], gp["constitutive_parameter_upper_bounds"][k])
                         for k in ("E", "nu", "contact_stiffness", "shearing_stiffness")},
              "result_dir": args.get("result_dir", "/../result/")},
    )
    sc.targets = target[0] if target.ndim == 3 else target
    return sc


def load_reference_scene(src_dir: str, seed: Optional[int] = None, args: Optional[dict] = None,
                         seed_cube: Optional[int] = None) -> ClothScene:
    """Reads ``simulation_arguments.json`` in ``src_dir`` and the data files it
    names (initialization.py:26-77).  The reference draws its operator and cube
    clouds from unseeded generators; ``seed`` seeds them here (Python
    ``random`` for the operator cloud, ``numpy.random`` for the cube cloud,
    which ``seed_cube`` can seed separately)."""
    if args is None:
        with open(os.path.join(src_dir, "simulation_arguments.json")) as fh:
            args = json.load(fh)
    data = src_dir + args["data_dir"]
    target = np.load(os.path.join(data, "target_pcd_sample.npy"))
    mark = np.load(os.path.join(data, "rigid_cube_top_face_center_position.npy"))
    grasp = np.load(os.path.join(data, "grasp_traj_array.npy"))
    verts, tris = io_ply.read_ply(os.path.join(data, "cloth_mesh.ply"))
    n_c = args["rigid_cube_parameters"]["n_rigid_cube_particles"]
    rs = np.random.RandomState(seed if seed_cube is None else seed_cube)
    cube_random = rs.rand(n_c, 3)
    n_op = args["operator_parameters"]["n_operator_particles"]
    group = int(n_op / grasp.shape[1])
    pr = _pyrandom.Random(seed)
    op_random = np.array([[pr.random(), pr.random(), pr.random()] for _ in range(group)]).reshape(group, 3)
    return reference_scene(args, verts, tris, grasp, target, mark, op_random, cube_random)


# ------------------------------------------------------------------ sheets
def regular_sheet(n: int, side: float):
    """n x n vertices on a square of ``side`` metres in the xz plane, each
    quad split along the same diagonal: Nt = 2 (n-1)^2."""
    s = np.linspace(0.0, side, n)
    xx, zz = np.meshgrid(s, s, indexing="ij")
    verts = np.stack([xx, np.zeros_like(xx), zz], -1).reshape(-1, 3)
    ii, jj = np.meshgrid(np.arange(n - 1), np.arange(n - 1), indexing="ij")
    v0 = (ii * n + jj).ravel()
    v1 = v0 + n
    v2 = v0 + 1
    v3 = v0 + n + 1
    tris = np.concatenate([np.stack([v0, v1, v3], 1), np.stack([v0, v3, v2], 1)])
    return verts, tris


def cubic_spline_grasp(start: np.ndarray, n_steps: int, dt: float, rng: np.random.Generator, n_ctrl: int = 5,
                       amplitude: float = 0.05, duration: float = 1.0):
    """Smooth gripper path through ``n_ctrl`` control points spread over
    ``duration`` seconds: the first is the grasped corner, the others are
    offset by U(-amplitude, amplitude) per axis.  Returns per-substep
    velocities and centres, each (n_steps, 3)."""
    from scipy.interpolate import CubicSpline
    T = max(duration, n_steps * dt)
    tk = np.linspace(0.0, T, n_ctrl)
    pts = start[None, :] + np.concatenate([np.zeros((1, 3)), rng.uniform(-amplitude, amplitude, (n_ctrl - 1, 3))])
    cs = CubicSpline(tk, pts, axis=0, bc_type="clamped")
    t = np.arange(n_steps) * dt
    return cs(t, 1), cs(t)


def sheet_scene(n: int = 32, side: float = 0.2, height: float = 0.3, n_grid: int = 64, dt: float = 2e-4,
                n_steps: int = 200, E: float = 5e3, nu: float = 0.3, density: float = 0.2, friction: float = 0.3,
                damping: float = REFERENCE_DAMPING, seed: int = 0, n_targets: int = 2048,
                gripper_radius: Optional[float] = None, center=(0.5, 0.5), velocities=None,
                spline_duration: float = 1.0, cap_radius: Optional[float] = None,
                grasp_amplitude: float = 0.05) -> ClothScene:
    """Square cloth sheet held by two kinematic spheres at two adjacent
    corners, the cloth of the benchmark configurations.  Masses follow the
    reference's formulas (initialization.py:118-130) with the garment mass set
    from the areal ``density``; gravity is not scaled (scene_scaling = 1).
    ``velocities`` (n_steps, 2, 3) replaces the spline with per-substep
    gripper velocities (centres integrate them).

    ``cap_radius`` R: the sheet's rest shape is a shallow bowl instead of a
    plane: the point at in-plane offsets (u, v) from the centre sits at
    (R sin(u/R), R (2 - cos(u/R) - cos(v/R)), R sin(v/R)) relative to the
    centre at ``height``, so the mesh keeps its side length along both mesh
    directions (edges of side / (n - 1)) while its horizontal extent shrinks
    to 2 R sin(side / 2R).  A sheet as wide as the domain fits between the
    walls this way."""
    rng = np.random.default_rng(seed)
    verts, tris = regular_sheet(n, side)
    if cap_radius is None:
        verts = verts + np.array([center[0] - side / 2, height, center[1] - side / 2])
        area = side * side
    else:
        R = float(cap_radius)
        u, v = verts[:, 0] - side / 2, verts[:, 2] - side / 2
        verts = np.stack([center[0] + R * np.sin(u / R), height + R * (2.0 - np.cos(u / R) - np.cos(v / R)),
                          center[1] + R * np.sin(v / R)], -1)
        area = mesh_area(verts, tris)
    dx = 1.0 / n_grid
    M = density * area
    corners = np.stack([verts[0], verts[n - 1]])   # (0,0) and (0,n-1): adjacent corners
    if velocities is None:
        vel = np.zeros((n_steps, 2, 3))
        cen = np.zeros((n_steps, 2, 3))
        for k in range(2):
            vel[:, k], cen[:, k] = cubic_spline_grasp(corners[k], n_steps, dt, rng, amplitude=grasp_amplitude,
                                                      duration=spline_duration)
    else:
        vel = np.asarray(velocities, dtype=np.float64).reshape(n_steps, 2, 3)
        cen = corners[None] + dt * np.concatenate([np.zeros((1, 2, 3)), np.cumsum(vel, 0)[:-1]], 0)
    sc = ClothScene(
        vertices=verts, triangles=tris, n_grid=n_grid,
        vertex_p_mass=M / verts.shape[0], quadrature_p_mass=M / verts.shape[0],
        quadrature_p_vol=3 * area * dx / tris.shape[0], gravity_dv=dt * GRAVITY,
        gripper_mode=GRIP_KINEMATIC, n_grippers=2,
        gripper_radius=(1.25 * dx if gripper_radius is None else gripper_radius),
        velocities=vel, centers=cen,
        params={"E": E, "nu": nu, "shearing_stiffness": 100.0, "contact_stiffness": 100.0, "friction": friction,
                "damping": damping},
        meta={"dt": dt, "n_steps": n_steps, "side": side, "n": n, "seed": seed},
    )
    if n_targets:
        sc.targets = surface_samples(verts, tris, n_targets, rng)
    return sc


def surface_samples(verts, tris, n, rng):
    """Area-weighted uniform samples on the triangle mesh."""
    v = np.asarray(verts)
    a, b, c = v[tris[:, 0]], v[tris[:, 1]], v[tris[:, 2]]
    w = 0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1)
    t = rng.choice(len(tris), size=n, p=w / w.sum())
    r1, r2 = rng.random(n), rng.random(n)
    s1 = np.sqrt(r1)
    return (1 - s1)[:, None] * a[t] + (s1 * (1 - r2))[:, None] * b[t] + (s1 * r2)[:, None] * c[t]


# ------------------------------------------------------------------ order
def _part1by2(x):
    x = x.astype(np.uint64) & np.uint64(0x1FFFFF)
    x = (x | (x << np.uint64(32))) & np.uint64(0x1F00000000FFFF)
    x = (x | (x << np.uint64(16))) & np.uint64(0x1F0000FF0000FF)
    x = (x | (x << np.uint64(8))) & np.uint64(0x100F00F00F00F00F)
    x = (x | (x << np.uint64(4))) & np.uint64(0x10C30C30C30C30C3)
    x = (x | (x << np.uint64(2))) & np.uint64(0x1249249249249249)
    return x


def morton_order(points: np.ndarray, cell: float) -> np.ndarray:
    """Stable argsort of 3-D Morton codes of ``points`` quantised to ``cell``."""
    q = np.clip(np.floor(np.asarray(points) / cell), 0, 2 ** 21 - 1).astype(np.int64)
    code = _part1by2(q[:, 0]) | (_part1by2(q[:, 1]) << np.uint64(1)) | (_part1by2(q[:, 2]) << np.uint64(2))
    return np.argsort(code, kind="stable")
