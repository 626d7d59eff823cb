"""Generate the golden vectors in this folder by executing the reference's own
source files (``src/initialization.py``, ``src/taichi_variable_definition.py``,
``src/simulation.py``, ``src/parameter_fitting_functions.py``,
``src/simulation_without_grad.py`` of
denzelzheng/diffcp) unmodified, under the NumPy stand-ins for ``taichi`` and
``open3d`` in ``ti_standin.py`` / ``o3d_standin.py``.

The reference is copied (read-only sources) into a temporary tree together
with a small synthetic scene (mesh PLY, grasp trajectory, target clouds, cube
marker and a ``simulation_arguments.json`` with small sizes), because the
reference loads its data and configuration from paths relative to itself.

Outputs
  ref_forward_f32.npz   per-substep states, losses and scene constants of two
                        grasp windows, reference kernels in float32
  ref_svd_backward.npz  ``backward_inplane_svd`` (simulation.py:71-88) on
                        random and degenerate 2x2 inputs
  ref_fd_f64.npz        central finite differences of the window-0 loss with
                        respect to E, nu, contact/shearing stiffness and two
                        grasp-trajectory coordinates, reference kernels in
                        float64
  ref_fitting.npz       the parameter-fitting step-size heuristic on random
                        and edge inputs, and the epoch loop driven by the
                        compute_grad stand-in of fit_fake.py
  ref_replay_f32.npz    the forward-only replay of simulation_without_grad.py
                        (substep blocks with reset_quadrature_particles) and
                        the pose files animation() writes, float32
  ref_fd_press_f64.npz  central finite differences of the window-0 loss on the
                        "press" variant of the synthetic scene (the grasp
                        pushes the sheet's corners down for 300 substeps, so
                        that the contact term A22 of simulation.py:216-225
                        engages), reference kernels in float64
  ref_real_f32.npz      the reference's own scene (data/cloth_mesh.ply,
                        grasp_traj_array.npy, target_pcd_sample.npy,
                        rigid_cube_top_face_center_position.npy) with a short
                        horizon: compute_grad() itself run over 2 grasp
                        windows of 300 substeps (end-state carry-over of
                        parameter_fitting_functions.py:40-49), per-window
                        losses and vertex histories, float32; and the inputs
                        (PLY bytes, the 4 trajectory frames, the 2 target
                        windows, the arguments) so that tests rebuild the tree
  ref_real_fd_f64.npz   the same scene in float64: window 0, the carry-over,
                        and central finite differences of the window-1 loss
                        with respect to E, nu, contact/shearing stiffness and
                        three horizontal grasp-trajectory coordinates (two
                        step sizes each), the carried-in state held fixed (the
                        Tape of compute_grad covers one window)

Run:  python tests/golden/make_golden.py --ref PATH   (PATH: the reference's
source tree; or set DIFFCP_REFERENCE)
"""
from __future__ import annotations

import argparse
import json
import os
import random
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SEED_OP, SEED_CUBE, SEED_SCENE = 1234, 4321, 7

ARGS = {
    "dt": 0.0002,
    "n_grid": 15,
    "scene_scaling": 0.5,
    "initial_frame": 0,
    "end_frame": -1,
    "operator_update_interval": 0.00073,
    "clip_IFS": 0.8,
    "grad_update_interval": 0.0061,
    "operator_parameters": {"operator_edge_length": 0.03, "n_operator_particles": 8, "operator_mass": 99},
    "rigid_cube_parameters": {"rigid_cube_side_length": 0.14, "n_rigid_cube_particles": 6, "cube_mass": 999},
    "garment_parameters": {
        "number_of_triangles": 1500, "sim_number_of_triangles": 310,
        "constitutive_parameter_upper_bounds": {"E": 1000, "nu": 0.45, "contact_stiffness": 5000,
                                                "shearing_stiffness": 1000},
        "constitutive_parameter_lower_bounds": {"E": 10, "nu": 0.05, "contact_stiffness": 10,
                                                "shearing_stiffness": 1, "internal_friction_angle": 1,
                                                "damping": 0.1},
        "initial_constitutive_parameters": {"E": 100, "nu": 0.1, "contact_stiffness": 100,
                                            "shearing_stiffness": 100},
        "garment_mass": 0.5},
    "data_dir": "/../data/",
    "result_dir": "/../result/",
    "n_pose_estimation_output": 35,
}
PARAMS = {"E": 400.0, "nu": 0.3, "contact_stiffness": 300.0, "shearing_stiffness": 150.0}

# "press" variant: 300 substeps (0.0601 / 2e-4 -> max_steps 301) and a grasp
# that pushes the corners down, so the sheet is compressed along its normal
# (R22 < 1) and the contact stiffness matters to the loss.
ARGS_PRESS = dict(ARGS, grad_update_interval=0.0601)
PARAMS_PRESS = {"E": 400.0, "nu": 0.3, "contact_stiffness": 1000.0, "shearing_stiffness": 150.0}

# The reference's own scene with a short horizon: 300 substeps per grasp
# window (0.03001 / 1e-4 -> max_steps 301; one keyframe interval, so window g
# moves the grippers from frame g to g + 1), frames 0..3 of the grasp
# trajectory (end_frame 3) and the first REAL_WINDOWS target windows; the other
# keys are those of the reference's simulation_arguments.json.  Window 1's
# loss depends on keyframes 1 and 2 (REAL_SEQ_COORDS).  Frames 1-3 of the
# trajectory coincide, so the grippers rest through window 1 and the loss has
# a kink in every keyframe's height (y): a gripper velocity up or down moves
# the sheet against the floor differently.  The differences therefore run
# along horizontal coordinates (x: 0, z: 2), each with two steps
# (REAL_SEQ_STEPS); tests compare a gradient with them only where the two
# agree.
REAL_OVERRIDES = {"grad_update_interval": 0.03001, "end_frame": 3}
REAL_WINDOWS = 2
REAL_FRAMES = 4
REAL_SEQ_COORDS = ((1, 0, 2), (2, 1, 0), (2, 0, 0))
REAL_SEQ_STEPS = (1e-7, 1e-6)
REAL_HISTORY_STRIDE = 10   # vertex histories of ref_real_f32.npz: every 10th substep
REAL_WORKERS = 6


def write_ply(path, v, t):
    v = np.asarray(v, dtype="<f8")
    t = np.asarray(t, dtype="<u4")
    head = ("ply\nformat binary_little_endian 1.0\ncomment synthetic\nelement vertex %d\n"
            "property double x\nproperty double y\nproperty double z\nelement face %d\n"
            "property list uchar uint vertex_indices\nend_header\n" % (len(v), len(t)))
    rec = np.zeros(len(t), dtype=[("n", "u1"), ("idx", "<u4", (3,))])
    rec["n"] = 3
    rec["idx"] = t
    with open(path, "wb") as fh:
        fh.write(head.encode("ascii"))
        fh.write(v.tobytes())
        fh.write(rec.tobytes())


def scene_arrays(variant="base"):
    """Jittered 7x7 sheet (raw units), a 2-point grasp trajectory moving the two
    far corners, 2 windows x 12 target points, a cube marker.  variant "press":
    the same sheet, targets and marker, with a 100-frame trajectory that moves
    the corners down and inwards."""
    rng = np.random.default_rng(SEED_SCENE)
    n = 7
    ii, kk = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    verts = np.stack([0.55 + 0.1 * ii, 0.02 + 0.004 * rng.standard_normal((n, n)),
                      0.30 + 0.1 * kk], -1).reshape(-1, 3)
    verts[:, [0, 2]] += 0.01 * rng.standard_normal((n * n, 2))
    tris = []
    for a in range(n - 1):
        for b in range(n - 1):
            v0, v1, v2, v3 = a * n + b, (a + 1) * n + b, a * n + b + 1, (a + 1) * n + b + 1
            tris.append((v0, v1, v3) if (a + b) % 2 == 0 else (v0, v1, v2))
            tris.append((v0, v3, v2) if (a + b) % 2 == 0 else (v1, v3, v2))
    tris = np.array(tris)
    frames = 20
    t = np.arange(frames)[:, None]
    c0 = verts[(n - 1) * n + 0] + np.array([0.0, 0.02, 0.0])
    c1 = verts[(n - 1) * n + n - 1] + np.array([0.0, 0.02, 0.0])
    traj = np.stack([c0 + t * np.array([0.012, 0.010, -0.004]),
                     c1 + t * np.array([0.010, 0.012, 0.006])], 1)
    traj += 0.001 * rng.standard_normal(traj.shape)
    target = verts[None, rng.choice(n * n, 12, replace=False)] + 0.02 * rng.standard_normal((2, 12, 3))
    mark = np.array([0.85, 0.09, 0.55])
    if variant == "press":
        t = np.arange(100)[:, None]
        traj = np.stack([c0 + t * np.array([-0.003, -0.0015, -0.002]),
                         c1 + t * np.array([-0.003, -0.0015, 0.003])], 1)
    return verts, tris, traj, target, mark


def build_tree(ref, variant="base"):
    """A temporary copy of the reference's source files with a scene of its
    own: the synthetic sheet ("base", "press") or the reference's own data
    with a short horizon ("real")."""
    tmp = tempfile.mkdtemp(prefix="diffcp_ref_")
    os.makedirs(os.path.join(tmp, "src"))
    os.makedirs(os.path.join(tmp, "data"))
    os.makedirs(os.path.join(tmp, "result"))
    for name in os.listdir(os.path.join(ref, "src")):
        if name.endswith(".py"):
            shutil.copy(os.path.join(ref, "src", name), os.path.join(tmp, "src", name))
    open(os.path.join(tmp, "src", "__init__.py"), "w").close()
    if variant == "real":
        with open(os.path.join(ref, "src", "simulation_arguments.json")) as fh:
            args = json.load(fh)
        args.update(REAL_OVERRIDES)
        with open(os.path.join(tmp, "src", "simulation_arguments.json"), "w") as fh:
            json.dump(args, fh)
        data = os.path.join(ref, "data")
        shutil.copy(os.path.join(data, "cloth_mesh.ply"), os.path.join(tmp, "data", "cloth_mesh.ply"))
        shutil.copy(os.path.join(data, "rigid_cube_top_face_center_position.npy"),
                    os.path.join(tmp, "data", "rigid_cube_top_face_center_position.npy"))
        np.save(os.path.join(tmp, "data", "grasp_traj_array.npy"),
                np.load(os.path.join(data, "grasp_traj_array.npy"))[:REAL_FRAMES])
        np.save(os.path.join(tmp, "data", "target_pcd_sample.npy"),
                np.load(os.path.join(data, "target_pcd_sample.npy"))[:REAL_WINDOWS])
        return tmp
    with open(os.path.join(tmp, "src", "simulation_arguments.json"), "w") as fh:
        json.dump(ARGS_PRESS if variant == "press" else ARGS, fh)
    verts, tris, traj, target, mark = scene_arrays(variant)
    write_ply(os.path.join(tmp, "data", "cloth_mesh.ply"), verts, tris)
    np.save(os.path.join(tmp, "data", "grasp_traj_array.npy"), traj)
    np.save(os.path.join(tmp, "data", "target_pcd_sample.npy"), target)
    np.save(os.path.join(tmp, "data", "rigid_cube_top_face_center_position.npy"), mark)
    return tmp


def import_reference(tree, f64=False, forward_tape=False):
    sys.path.insert(0, HERE)
    import ti_standin
    import o3d_standin
    import types
    if f64:
        ti_standin.force_f64()
    if forward_tape:
        ti_standin.allow_forward_tape()
    sys.modules["taichi"] = ti_standin
    sys.modules["taichi_glsl"] = types.ModuleType("taichi_glsl")
    sys.modules["open3d"] = o3d_standin
    random.seed(SEED_OP)
    np.random.seed(SEED_CUBE)
    sys.path.insert(0, tree)
    import src.parameter_fitting_functions as pff   # noqa: E402  (executes the reference modules)
    return pff


def set_params(m, p):
    m.garment_E[None] = p["E"]
    m.garment_nu[None] = p["nu"]
    m.contact_stiffness[None] = p["contact_stiffness"]
    m.shearing_stiffness[None] = p["shearing_stiffness"]


def window_loss(m, g, keep=False):
    """The body of compute_grad (parameter_fitting_functions.py:21-29) without
    the tape: clear, set targets, substeps 0..max_steps-2, compute_loss."""
    m.initialize_objects()
    m.clear_distances()
    m.target_pos.from_numpy(m.target_pcd_array[g])
    m.loss[None] = 0
    for f in range(m.max_steps - 1):
        m.forward(f, g)
    m.compute_loss(f)
    return float(m.loss[None])


def run_forward32(tree, out):
    m = import_reference(tree)
    set_params(m, PARAMS)
    rec = {}
    keys = ["vertex_x", "vertex_v", "vertex_C", "quadrature_x", "quadrature_v", "quadrature_C",
            "quadrature_F", "quadrature_d", "operator_x", "operator_v", "operator_C", "cube_x", "cube_v",
            "cube_C"]
    for g in (0, 1):
        rec["loss_w%d" % g] = window_loss(m, g)
        for k in keys:
            rec["w%d_%s" % (g, k)] = getattr(m, k).to_numpy()
        rec["w%d_distances" % g] = m.distances.to_numpy()
    rec["initial_quadrature_d_inv"] = m.initial_quadrature_d_inv.to_numpy()
    rec["lagrangian_mesh_element"] = m.lagrangian_mesh_element.to_numpy()
    rec["grasp_point_pos"] = np.asarray(m.grasp_point_pos)
    rec["target_pcd_array"] = np.asarray(m.target_pcd_array)
    rec["soft_body_model_vertices"] = np.asarray(m.soft_body_model_vertices)
    rec["cube_model"] = np.asarray(m.cube_model)
    rec["operator_model_without_position"] = np.asarray(m.operator_model_without_position)
    for name in ("dt", "n_grid", "dx", "inv_dx", "vertex_p_mass", "quadrature_p_mass", "quadrature_p_vol",
                 "operator_p_mass", "cube_p_mass", "garment_surface_area", "max_steps", "n_actions",
                 "grasper_group_size", "operator_update_interval", "grad_update_interval", "scene_scaling"):
        rec["const_" + name] = np.asarray(getattr(m, name))
    rec["params"] = np.array([PARAMS["E"], PARAMS["nu"], PARAMS["contact_stiffness"],
                              PARAMS["shearing_stiffness"]])
    rec["seed_op"], rec["seed_cube"] = SEED_OP, SEED_CUBE
    np.savez_compressed(out, **rec)


def run_svd(tree, out):
    m = import_reference(tree)
    import ti_standin as ti
    rng = np.random.default_rng(11)
    mats = [np.eye(2), np.diag([1.3, 1.3]), np.array([[1.0, 1e-7], [0.0, 1.0 + 2e-7]]),
            np.array([[0.9, 0.2], [-0.1, 1.1]]), np.array([[-0.8, 0.1], [0.3, 1.2]])]
    mats += [np.eye(2) + 0.3 * rng.standard_normal((2, 2)) for _ in range(27)]
    rows = {k: [] for k in ("A", "U", "S", "V", "gU", "gS", "gV", "out")}
    for A in mats:
        A = A.astype(np.float32)
        U, S, V = ti.svd(A)
        gU = rng.standard_normal((2, 2)).astype(np.float32)
        gV = rng.standard_normal((2, 2)).astype(np.float32)
        gS = np.diag(rng.standard_normal(2)).astype(np.float32)
        res = m.backward_inplane_svd(gU.view(ti.TiArr), gS.view(ti.TiArr), gV.view(ti.TiArr), U, S, V)
        for k, v in zip(rows, (A, U, S, V, gU, gS, gV, res)):
            rows[k].append(np.asarray(v))
    np.savez_compressed(out, **{k: np.stack(v) for k, v in rows.items()})


def run_fd64(tree, out):
    m = import_reference(tree, f64=True)
    rec = {}
    base = dict(PARAMS)
    set_params(m, base)
    rec["loss"] = window_loss(m, 0)
    for name in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        h = 1e-5 * base[name]
        vals = []
        for sgn in (1, -1):
            p = dict(base)
            p[name] = base[name] + sgn * h
            set_params(m, p)
            vals.append(window_loss(m, 0))
        rec["fd_" + name] = (vals[0] - vals[1]) / (2 * h)
        set_params(m, base)
    coords = [(3, 0, 1), (5, 1, 0)]
    for (a, b, c) in coords:
        h = 1e-6
        vals = []
        for sgn in (1, -1):
            m.grasp_point_pos[a, b, c] += sgn * h
            vals.append(window_loss(m, 0))
            m.grasp_point_pos[a, b, c] -= sgn * h
        rec["fd_seq_%d_%d_%d" % (a, b, c)] = (vals[0] - vals[1]) / (2 * h)
    rec["params"] = np.array([base["E"], base["nu"], base["contact_stiffness"], base["shearing_stiffness"]])
    np.savez_compressed(out, **rec)


def _fd_params(m, base, loss_fn, rel_h=1e-5):
    """Central differences of loss_fn() in each of the four parameters."""
    rec = {}
    for name in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        h = rel_h * base[name]
        vals = []
        for sgn in (1, -1):
            p = dict(base)
            p[name] = base[name] + sgn * h
            set_params(m, p)
            vals.append(loss_fn())
        rec["fd_" + name] = (vals[0] - vals[1]) / (2 * h)
        set_params(m, base)
    return rec


# Keyframe coordinates of the press scene's trajectory finite differences.  The
# float64 run evaluates the reference's keyframe index int(f dt / interval) in
# float64, which at substeps 73, 146, 219 and 292 picks frames 20, 40, 60, 80
# where the reference's float32 arithmetic picks 19, 39, 59, 79; the trajectory
# is linear, so the states do not change, but the gradients of keyframes next
# to those boundaries (19-21, 39-41, 59-61, 79-81) do.  These are away from them.
PRESS_SEQ_COORDS = ((10, 1, 2), (50, 0, 2))


def press_seq_fd(m):
    rec = {}
    for (a, b, c) in PRESS_SEQ_COORDS:
        h = 1e-6
        vals = []
        for sgn in (1, -1):
            m.grasp_point_pos[a, b, c] += sgn * h
            vals.append(window_loss(m, 0))
            m.grasp_point_pos[a, b, c] -= sgn * h
        rec["fd_seq_%d_%d_%d" % (a, b, c)] = (vals[0] - vals[1]) / (2 * h)
    return rec


def run_press64(tree, out):
    m = import_reference(tree, f64=True)
    base = dict(PARAMS_PRESS)
    set_params(m, base)
    rec = {"loss": window_loss(m, 0)}
    rec.update(_fd_params(m, base, lambda: window_loss(m, 0), rel_h=1e-4))
    rec.update(press_seq_fd(m))
    rec["params"] = np.array([base["E"], base["nu"], base["contact_stiffness"], base["shearing_stiffness"]])
    rec["max_steps"] = np.array(m.max_steps)
    np.savez_compressed(out, **rec)


def _real_initial_params(m):
    """initial_constitutive_parameters of the arguments (what
    parameter_fitting_main.py:3-6 sets before fitting)."""
    return {"E": float(m.initial_garment_E), "nu": float(m.initial_garment_nu),
            "contact_stiffness": float(m.initial_contact_stiffness),
            "shearing_stiffness": float(m.initial_shearing_stiffness)}


def run_real32(tree, out):
    """compute_grad() of the reference over the short-horizon real scene; the
    window histories are read where compute_grad re-initialises the fields
    from the window's end state (parameter_fitting_functions.py:40-49)."""
    import contextlib
    import io
    m = import_reference(tree, forward_tape=True)
    base = _real_initial_params(m)
    set_params(m, base)
    m.initialize_objects()
    hist = []
    orig = m.initialize_ti_field

    def observed():
        hist.append({k: getattr(m, k).to_numpy() for k in ("vertex_x", "operator_x", "cube_x")})
        hist[-1]["loss"] = float(m.loss[None])
        orig()

    m.initialize_ti_field = observed
    with contextlib.redirect_stdout(io.StringIO()):
        loss_mean, _ = m.compute_grad()
    m.initialize_ti_field = orig
    rec = {"loss_mean": np.array(loss_mean), "n_windows": np.array(len(hist)), "params": np.array(
        [base["E"], base["nu"], base["contact_stiffness"], base["shearing_stiffness"]])}
    for g, h in enumerate(hist):
        rec["w%d_loss" % g] = np.array(h["loss"])
        rec["w%d_vertex_x" % g] = h["vertex_x"][::REAL_HISTORY_STRIDE]   # substeps 0, 10, ..., 300
        rec["w%d_operator_x_end" % g] = h["operator_x"][-1]
        rec["w%d_cube_x_end" % g] = h["cube_x"][-1]
    for name in ("dt", "n_grid", "vertex_p_mass", "quadrature_p_mass", "quadrature_p_vol", "operator_p_mass",
                 "cube_p_mass", "garment_surface_area", "max_steps", "n_actions", "grasper_group_size",
                 "n_grad_updates"):
        if hasattr(m, name):
            rec["const_" + name] = np.asarray(getattr(m, name))
    rec["soft_body_model_vertices"] = np.asarray(m.soft_body_model_vertices)
    rec["grasp_point_pos"] = np.asarray(m.grasp_point_pos)
    rec["target_pcd_array"] = np.asarray(m.target_pcd_array)
    rec["cube_model"] = np.asarray(m.cube_model)
    rec["operator_model_without_position"] = np.asarray(m.operator_model_without_position)
    # the inputs, so that tests rebuild the tree without the reference
    with open(os.path.join(tree, "data", "cloth_mesh.ply"), "rb") as fh:
        rec["in_ply_bytes"] = np.frombuffer(fh.read(), dtype=np.uint8)
    for name in ("grasp_traj_array", "target_pcd_sample", "rigid_cube_top_face_center_position"):
        rec["in_" + name] = np.load(os.path.join(tree, "data", name + ".npy"))
    with open(os.path.join(tree, "src", "simulation_arguments.json")) as fh:
        rec["in_arguments_json"] = np.array(fh.read())
    np.savez_compressed(out, **rec)


_REAL64 = {}


def _real64_worker(tree, carried_path):
    """Process initialiser: the reference in float64 and window 0's end state."""
    m = import_reference(tree, f64=True)
    m.initialize_objects()          # the keyframes (grasp_tracking_seq), as in the parent process
    c = np.load(carried_path)
    _REAL64.update(m=m, carried={k: c[k] for k in c.files})


def _window1_loss(m, carried, params, seq_delta=None):
    """compute_grad's window 1 (parameter_fitting_functions.py:21-29) from the
    carried-in state of window 0 (lines 40-49), with ``params`` and, when
    ``seq_delta`` = ((a, b, c), h), keyframe (a, b, c) moved by h."""
    set_params(m, params)
    m.initial_operator_x.from_numpy(carried["op"])
    m.initial_vertex_x.from_numpy(carried["vx"])
    m.lagrangian_mesh_element.from_numpy(carried["faces"])
    m.initial_cube_x.from_numpy(carried["cube"])
    m.initialize_ti_field()
    if seq_delta is not None:
        (a, b, c), h = seq_delta
        m.grasp_tracking_seq[a][b, c] += h
    try:
        return window_loss_carry(m, 1)
    finally:
        if seq_delta is not None:
            m.grasp_tracking_seq[a][b, c] -= h


def _real64_task(task):
    m, carried = _REAL64["m"], _REAL64["carried"]
    params, seq_delta = task
    return _window1_loss(m, carried, params, seq_delta)


def run_real64(tree, out):
    """Window 0, the carry-over of compute_grad (parameter_fitting_functions.py:
    40-49), and central differences of the window-1 loss with the carried-in
    state held fixed, in float64.  The window-1 evaluations run in parallel
    processes, each with its own copy of the reference's module state."""
    import concurrent.futures
    import multiprocessing
    m = import_reference(tree, f64=True)
    base = _real_initial_params(m)
    set_params(m, base)
    m.initialize_objects()
    rec = {"w0_loss": window_loss_carry(m, 0)}
    last = m.max_steps - 1
    carried = {"op": m.operator_x.to_numpy()[last], "vx": m.vertex_x.to_numpy()[last],
               "cube": m.cube_x.to_numpy()[last], "faces": np.asarray(m.soft_body_mesh.triangles)}
    rec["w0_vertex_x_end"] = carried["vx"]
    carried_path = out + ".carried.npz"
    np.savez(carried_path, **carried)
    tasks, keys = [(dict(base), None)], ["w1_loss"]
    rel_h = 1e-4
    for name in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        for sgn in (1, -1):
            p = dict(base)
            p[name] = base[name] + sgn * rel_h * base[name]
            tasks.append((p, None))
            keys.append(("param", name, sgn))
    for h_seq in REAL_SEQ_STEPS:
        for coord in REAL_SEQ_COORDS:
            for sgn in (1, -1):
                tasks.append((dict(base), (coord, sgn * h_seq)))
                keys.append(("seq", coord, sgn, h_seq))
    ctx = multiprocessing.get_context("spawn")
    with concurrent.futures.ProcessPoolExecutor(REAL_WORKERS, mp_context=ctx, initializer=_real64_worker,
                                                initargs=(tree, carried_path)) as ex:
        vals = list(ex.map(_real64_task, tasks))
    os.remove(carried_path)
    rec["w1_loss"] = vals[0]
    res = dict(zip(keys[1:], vals[1:]))
    for name in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        h = rel_h * base[name]
        rec["w1_fd_" + name] = (res[("param", name, 1)] - res[("param", name, -1)]) / (2 * h)
    # w1_fd_seq_*: step REAL_SEQ_STEPS[0]; w1_fd2_seq_*: step REAL_SEQ_STEPS[1]
    for prefix, h_seq in zip(("w1_fd_seq_", "w1_fd2_seq_"), REAL_SEQ_STEPS):
        for coord in REAL_SEQ_COORDS:
            rec[prefix + "%d_%d_%d" % coord] = (res[("seq", coord, 1, h_seq)] - res[("seq", coord, -1, h_seq)]) / (
                2 * h_seq)
    rec["params"] = np.array([base["E"], base["nu"], base["contact_stiffness"], base["shearing_stiffness"]])
    rec["max_steps"] = np.array(m.max_steps)
    np.savez_compressed(out, **rec)


def window_loss_carry(m, g):
    """The body of compute_grad for window g from the current fields (no
    re-initialisation): set targets, substeps 0..max_steps-2, compute_loss."""
    m.clear_distances()
    m.target_pos.from_numpy(m.target_pcd_array[g])
    m.loss[None] = 0
    for f in range(m.max_steps - 1):
        m.forward(f, g)
    m.compute_loss(f)
    return float(m.loss[None])


def run_fitting(tree, out):
    """``single_parameter_fitting`` (parameter_fitting_functions.py:65-92) on
    random and edge inputs, and ``parameters_learning`` (94-205) driven by the
    deterministic compute_grad stand-in of fit_fake.py."""
    import contextlib
    import io
    m = import_reference(tree)
    import fit_fake
    rng = np.random.default_rng(99)
    rows_in, rows_out = [], []
    for k in range(600):
        name = fit_fake.NAMES[k % 4]
        lo, hi = fit_fake.BOUNDS[name]
        p = float(rng.uniform(lo, hi))
        if k % 50 == 7:
            g = 0.0
        elif k % 50 == 13:
            g = float("nan")
        else:
            g = float((1 if rng.random() < 0.5 else -1) * 10.0 ** rng.uniform(-8, 8))
        lr = float(10.0 ** rng.uniform(-6, 3))
        epochs = int(rng.integers(2, 40))
        idx = 0 if k % 3 == 0 else int(rng.integers(0, epochs))
        res = m.single_parameter_fitting(p, g, 0, lo, hi, lr, epochs, idx)
        rows_in.append([p, g, lo, hi, lr, epochs, idx])
        rows_out.append([float(res[0]), float(res[1])])
    rec = {"spf_in": np.array(rows_in), "spf_out": np.array(rows_out)}
    for (name, init, tgt, w, epochs, nan_g, nan_l, flags) in fit_fake.scenarios():
        calls = fit_fake.install(m, init, tgt, w, nan_g, nan_l)
        with contextlib.redirect_stdout(io.StringIO()):
            m.parameters_learning(flags[0], flags[1], epochs)
        rec["calls_" + name] = np.array(calls)
        rec["final_" + name] = np.array([getattr(m, fit_fake.FIELD[n])[None] for n in fit_fake.NAMES])
        rec["loss_" + name] = np.array(m.loss[None])
    np.savez_compressed(out, **rec)


def run_replay(tree, out):
    """The forward-only replay of ``src/simulation_without_grad.py``: six
    blocks of int(IFS/dt) substeps, each followed by
    reset_quadrature_particles, recording the state after every reset; then
    ``animation()`` itself with the open3d stand-in recording which pose files
    it writes and their vertices."""
    sys.path.insert(0, HERE)
    import ti_standin
    import o3d_standin
    import types
    sys.modules["taichi"] = ti_standin
    sys.modules["taichi_glsl"] = types.ModuleType("taichi_glsl")
    sys.modules["open3d"] = o3d_standin
    random.seed(SEED_OP)
    np.random.seed(SEED_CUBE)
    sys.path.insert(0, tree)
    import src.simulation_without_grad as m   # noqa: E402
    m.garment_E[None] = PARAMS["E"]
    m.garment_nu[None] = PARAMS["nu"]
    m.contact_stiffness[None] = PARAMS["contact_stiffness"]
    m.shearing_stiffness[None] = PARAMS["shearing_stiffness"]
    m.initialize_objects()
    block = int(0.001 / m.dt)
    rec = {"block": np.array(block)}
    f = 0
    for count in range(6):
        for _ in range(block):
            m.forward(f)
            f += 1
        m.reset_quadrature_particles()
        for k in ("vertex_x", "vertex_v", "quadrature_d", "quadrature_F", "initial_quadrature_d_inv", "operator_x"):
            rec["c%d_%s" % (count, k)] = getattr(m, k).to_numpy()
    writes = []
    o3d_standin.io.write_triangle_mesh = lambda path, mesh, **kw: writes.append(
        (int(os.path.basename(path)[:-4]), np.asarray(mesh.vertices, dtype=np.float64).copy())) or True
    m.initialize_objects()
    anim = m.operator_update_interval * (m.n_actions - 1)
    m.animation(anim)
    rec["animation_time"] = np.array(anim)
    rec["n_pose_estimation_output"] = np.array(m.n_pose_estimation_output)
    rec["pose_index"] = np.array([w[0] for w in writes])
    rec["pose_vertices"] = np.stack([w[1] for w in writes]) if writes else np.zeros((0, 0, 3))
    np.savez_compressed(out, **rec)


MODES = ("forward32", "svd", "fd64", "fitting", "replay", "press64", "real32", "real64")
VARIANT = {"press64": "press", "real32": "real", "real64": "real"}
OUT = {"forward32": "ref_forward_f32.npz", "svd": "ref_svd_backward.npz", "fd64": "ref_fd_f64.npz",
       "fitting": "ref_fitting.npz", "replay": "ref_replay_f32.npz", "press64": "ref_fd_press_f64.npz",
       "real32": "ref_real_f32.npz", "real64": "ref_real_fd_f64.npz"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("DIFFCP_REFERENCE"),
                    help="the reference's source tree (default: $DIFFCP_REFERENCE)")
    ap.add_argument("--mode", default="all", choices=("all",) + MODES)
    ap.add_argument("--tree")
    ap.add_argument("--only", nargs="*", help="with --mode all: the modes to regenerate")
    a = ap.parse_args()
    if a.mode == "all":
        if not a.ref:
            ap.error("--ref (or DIFFCP_REFERENCE) is required")
        trees = {}
        try:
            for mode in a.only or MODES:
                variant = VARIANT.get(mode, "base")
                if variant not in trees:
                    trees[variant] = build_tree(a.ref, variant)
                t0 = time.time()
                subprocess.run([sys.executable, __file__, "--mode", mode, "--tree", trees[variant],
                                "--ref", a.ref], check=True)
                print("%s done in %.1f s" % (mode, time.time() - t0))
        finally:
            for tree in trees.values():
                shutil.rmtree(tree, ignore_errors=True)
        return
    out = os.path.join(HERE, OUT[a.mode])
    {"forward32": run_forward32, "svd": run_svd, "fd64": run_fd64, "fitting": run_fitting,
     "replay": run_replay, "press64": run_press64, "real32": run_real32, "real64": run_real64}[a.mode](a.tree, out)


if __name__ == "__main__":
    main()
