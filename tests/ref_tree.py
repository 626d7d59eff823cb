"""Writes the small reference scene of tests/golden/make_golden.py as a
reference-style source tree (simulation_arguments.json + data directory)."""
import json
import os

import numpy as np

from tests.golden import make_golden as mg


def write_tree(root):
    src = os.path.join(str(root), "src")
    data = os.path.join(str(root), "data")
    os.makedirs(src, exist_ok=True)
    os.makedirs(data, exist_ok=True)
    with open(os.path.join(src, "simulation_arguments.json"), "w") as fh:
        json.dump(mg.ARGS, fh)
    verts, tris, traj, target, mark = mg.scene_arrays()
    mg.write_ply(os.path.join(data, "cloth_mesh.ply"), verts, tris)
    np.save(os.path.join(data, "grasp_traj_array.npy"), traj)
    np.save(os.path.join(data, "target_pcd_sample.npy"), target)
    np.save(os.path.join(data, "rigid_cube_top_face_center_position.npy"), mark)
    return src
