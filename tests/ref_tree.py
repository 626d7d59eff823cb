"""Writes the synthetic scenes of tests/golden/make_golden.py ("base", or the
contact-engaging "press" variant) as a reference-style source tree
(simulation_arguments.json + data directory)."""
import json
import os

import numpy as np

from tests.golden import make_golden as mg


def write_tree(root, variant="base"):
    src = os.path.join(str(root), "src")
    data = os.path.join(str(root), "data")
    os.makedirs(src, exist_ok=True)
    os.makedirs(data, exist_ok=True)
    with open(os.path.join(src, "simulation_arguments.json"), "w") as fh:
        json.dump(mg.ARGS_PRESS if variant == "press" else mg.ARGS, fh)
    verts, tris, traj, target, mark = mg.scene_arrays(variant)
    mg.write_ply(os.path.join(data, "cloth_mesh.ply"), verts, tris)
    np.save(os.path.join(data, "grasp_traj_array.npy"), traj)
    np.save(os.path.join(data, "target_pcd_sample.npy"), target)
    np.save(os.path.join(data, "rigid_cube_top_face_center_position.npy"), mark)
    return src


def write_real_tree(root, gold):
    """The reference's own scene, short horizon (tests/golden/ref_real_f32.npz
    holds its inputs: the PLY file's bytes, 4 grasp-trajectory frames, 3
    target windows, the cube marker and the arguments) as a reference-style
    source tree."""
    src = os.path.join(str(root), "src")
    data = os.path.join(str(root), "data")
    os.makedirs(src, exist_ok=True)
    os.makedirs(data, exist_ok=True)
    with open(os.path.join(src, "simulation_arguments.json"), "w") as fh:
        fh.write(str(gold["in_arguments_json"]))
    with open(os.path.join(data, "cloth_mesh.ply"), "wb") as fh:
        fh.write(gold["in_ply_bytes"].tobytes())
    for name in ("grasp_traj_array", "target_pcd_sample", "rigid_cube_top_face_center_position"):
        np.save(os.path.join(data, name + ".npy"), gold["in_" + name])
    return src
