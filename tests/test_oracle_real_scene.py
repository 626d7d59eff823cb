"""The reference's own scene (data/cloth_mesh.ply: 427 vertices, 777
triangles, binary float64; the first grasp frames of grasp_traj_array.npy; the
first target windows of target_pcd_sample.npy) with a short horizon of 300
substeps per window, against golden vectors of the reference source run on it
(tests/golden/make_golden.py, modes real32 and real64):

  * the product's PLY reader on the reference's binary file;
  * the product's scene loader: the constants of src/initialization.py;
  * (tests/test_gpu_oracle_real_scene.py, the oracle run on the GPU) the
    FP64 oracle over two grasp windows with the end-state carry-over of
    compute_grad (parameter_fitting_functions.py:40-49), and its window-1
    gradients against central differences of the reference's window-1 loss.
Here, CPU only: the reference's binary PLY and the scene constants."""
import json
import os

import numpy as np
import pytest
import torch

from diffcp_b200 import io_ply, scene as dscene
from oracle import sim64
from oracle.scene_ref import reference_scene
from oracle.sim64 import OracleSim
from tests.golden import make_golden as mg
from tests.golden import o3d_standin
from tests.ref_tree import write_real_tree

GOLD = os.path.join(os.path.dirname(__file__), "golden")
# relative sensitivity |dL/dp| p / L below which a float64 central difference
# with h = 1e-4 p cannot pin a gradient to 2e-4 (the float64 loss carries
# rounding of about 1e-13 of itself, so the quotient errs by ~1e-9 / sensitivity;
# over one 300-substep window of the reference's soft cloth, E = 100 Pa, the
# Poisson ratio and the contact stiffness stay below it)
MIN_SENSITIVITY = 5e-6


# Two central differences of a keyframe coordinate (steps 1e-7 and 1e-6 of
# make_golden.REAL_SEQ_STEPS) that differ by more than this, relative, mark a
# coordinate where the loss is not smooth at the scale of the step; a
# gradient is compared with a difference only where the two agree.
SEQ_STEP_AGREEMENT = 2e-5


def resolved_seq_differences(fd):
    """(keyframe, grasp, axis, difference) of every trajectory coordinate of
    ref_real_fd_f64.npz whose two step sizes agree; asserts that the fixture
    holds at least two such coordinates."""
    out = []
    for name in fd.files:
        if not name.startswith("w1_fd_seq_"):
            continue
        key = name[len("w1_fd_seq_"):]
        a, b, c = (int(t) for t in key.split("_"))
        d1, d2 = float(fd[name]), float(fd["w1_fd2_seq_" + key])
        assert d1 != 0.0, name
        if abs(d1 - d2) <= SEQ_STEP_AGREEMENT * abs(d1):
            out.append((a, b, c, d1))
    assert len(out) >= 2, "fewer than two resolved keyframe differences"
    return out


def test_keyframe_differences_are_resolved():
    """The golden keyframe differences are taken where the window-1 loss is
    smooth: both step sizes give the same difference."""
    fd = _load("ref_real_fd_f64.npz")
    res = resolved_seq_differences(fd)
    assert len(res) == sum(1 for n in fd.files if n.startswith("w1_fd_seq_"))


def _load(name):
    path = os.path.join(GOLD, name)
    if not os.path.exists(path):
        pytest.skip("golden file %s missing" % name)
    return np.load(path)


@pytest.fixture(scope="module")
def gold():
    return _load("ref_real_f32.npz")


@pytest.fixture(scope="module")
def tree(tmp_path_factory, gold):
    return write_real_tree(tmp_path_factory.mktemp("real"), gold)


def oracle_scene(tree):
    """The oracle's own restatement of initialization.py on the tree, with the
    PLY parsed by the test stand-in for open3d (not the product's reader)."""
    with open(os.path.join(tree, "simulation_arguments.json")) as fh:
        args = json.load(fh)
    data = tree + args["data_dir"]
    verts, tris = o3d_standin.read_ply_mesh(os.path.join(data, "cloth_mesh.ply"))
    traj = np.load(os.path.join(data, "grasp_traj_array.npy"))
    target = np.load(os.path.join(data, "target_pcd_sample.npy"))
    mark = np.load(os.path.join(data, "rigid_cube_top_face_center_position.npy"))
    cube_random = np.random.RandomState(mg.SEED_CUBE).rand(args["rigid_cube_parameters"]["n_rigid_cube_particles"], 3)
    import random
    pr = random.Random(mg.SEED_OP)
    group = args["operator_parameters"]["n_operator_particles"] // traj.shape[1]
    op_random = np.array([[pr.random(), pr.random(), pr.random()] for _ in range(group)])
    return reference_scene(args, verts, tris, traj, target, mark, op_random, cube_random)


def _params(p, grad=False, device=None):
    names = (("E", 0), ("nu", 1), ("kc", 2), ("ks", 3))    # the golden's order: E, nu, contact, shearing
    return {k: torch.tensor(float(p[i]), dtype=torch.float64, requires_grad=grad, device=device) for k, i in names}


def _window(sc, g, init, params, seq, device=None):
    """Window g from initial positions init = (vertices, operator, cube):
    the rollout's states and the loss of compute_loss(max_steps - 2)."""
    sim, st = OracleSim.initialize(sc["const"], init[0], sc["triangles"], init[1], init[2], device=device)
    states = sim64.rollout(sim, st, sc["max_steps"] - 1, params, seq=seq, window=g, keep_states=True)
    loss, _ = sim64.compute_loss(states[sc["max_steps"] - 3]["vx"],
                                 torch.tensor(sc["targets"][g], dtype=torch.float64, device=device))
    return states, loss


def _end(states):
    return tuple(states[-1][k].detach().cpu().numpy() for k in ("vx", "ox", "cx"))


def test_product_ply_reader_reads_the_reference_binary_mesh(gold, tmp_path):
    raw = gold["in_ply_bytes"].tobytes()
    path = tmp_path / "cloth_mesh.ply"
    path.write_bytes(raw)
    v, t = io_ply.read_ply(str(path))
    # independent parse of the layout the header declares (double x y z;
    # list uchar uint vertex_indices)
    body = raw[raw.index(b"end_header\n") + len(b"end_header\n"):]
    assert b"element vertex 427" in raw and b"element face 777" in raw
    xyz = np.frombuffer(body, dtype="<f8", count=427 * 3).reshape(427, 3)
    faces = np.frombuffer(body, dtype=[("n", "u1"), ("i", "<u4", (3,))], count=777, offset=427 * 24)
    assert (faces["n"] == 3).all()
    np.testing.assert_array_equal(np.asarray(v), xyz)
    np.testing.assert_array_equal(np.asarray(t), faces["i"].astype(np.int64))


def test_product_scene_loader_matches_reference_constants(gold, tree):
    sc = dscene.load_reference_scene(tree, seed=mg.SEED_OP, seed_cube=mg.SEED_CUBE)
    for name, got in (("vertex_p_mass", sc.vertex_p_mass), ("quadrature_p_mass", sc.quadrature_p_mass),
                      ("quadrature_p_vol", sc.quadrature_p_vol), ("operator_p_mass", sc.operator_p_mass),
                      ("cube_p_mass", sc.cube_p_mass)):
        assert got == pytest.approx(float(gold["const_" + name]), rel=1e-14), name
    assert sc.meta["max_steps"] == int(gold["const_max_steps"])
    assert sc.keyframes.shape[0] == int(gold["const_n_actions"])
    assert sc.group_size == int(gold["const_grasper_group_size"])
    np.testing.assert_allclose(sc.vertices, gold["soft_body_model_vertices"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(sc.keyframes, gold["grasp_point_pos"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(sc.meta["targets_by_window"], gold["target_pcd_array"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(np.asarray(sc.cube_x), gold["cube_model"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(sc.meta["operator_model"], gold["operator_model_without_position"], rtol=0,
                               atol=1e-15)
