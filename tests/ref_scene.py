"""Rebuilds, for the oracle, the small reference scene that
``tests/golden/make_golden.py`` fed to the reference source, from the same
seeds and synthetic data."""
from __future__ import annotations

import os
import random
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden as mg  # noqa: E402

from oracle.scene_ref import reference_scene  # noqa: E402


def small_reference_scene(variant="base"):
    verts, tris, traj, target, mark = mg.scene_arrays(variant)
    args = mg.ARGS_PRESS if variant == "press" else mg.ARGS
    random.seed(mg.SEED_OP)
    np.random.seed(mg.SEED_CUBE)
    n_c = args["rigid_cube_parameters"]["n_rigid_cube_particles"]
    cube_random = np.random.rand(n_c, 3)
    n_op = args["operator_parameters"]["n_operator_particles"]
    group = n_op // traj.shape[1]
    op_random = np.array([[random.random(), random.random(), random.random()] for _ in range(group)])
    sc = reference_scene(args, verts, tris, traj, target, mark, op_random, cube_random)
    sc["params"] = dict(mg.PARAMS_PRESS if variant == "press" else mg.PARAMS)
    return sc
