"""Scene constants and normalisation of the reference (``src/initialization.py``).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  The reference draws the
operator and cube point clouds from unseeded ``random``/``np.random``; here the
raw draws are inputs so that a harness can reproduce them from a seed.
"""
from __future__ import annotations

import numpy as np

from .sim64 import Constants


def mesh_area(vertices, triangles) -> float:
    """``get_surface_area`` of the Open3D mesh (initialization.py:112)."""
    v = np.asarray(vertices, dtype=np.float64)
    t = np.asarray(triangles)
    a, b, c = v[t[:, 0]], v[t[:, 1]], v[t[:, 2]]
    return float(0.5 * np.linalg.norm(np.cross(b - a, c - a), axis=1).sum())


def reference_scene(args: dict, mesh_vertices, mesh_triangles, grasp_seq, target_pcd, mark_pos,
                    operator_random, cube_random):
    """Restates initialization.py:26-193.

    ``operator_random``: (group_size, 3) values of ``random.random()`` in draw
    order (initialization.py:165-168); ``cube_random``: (n_cube, 3) values of
    ``np.random.rand`` (initialization.py:85).
    """
    op = args["operator_parameters"]
    gp = args["garment_parameters"]
    cube = args["rigid_cube_parameters"]
    dt = args["dt"]
    n_grid = args["n_grid"]
    s = args["scene_scaling"]
    interval = args["operator_update_interval"]
    gui = args["grad_update_interval"]
    initial_frame, end_frame = args["initial_frame"], args["end_frame"]
    garment_mass = gp["garment_mass"] * (s ** 3)                         # :67-68
    dx = 1 / n_grid                                                       # :79
    L = cube["rigid_cube_side_length"]
    cube_model = np.asarray(cube_random) * L - L / 2                     # :85
    cube_model[:, 0] += mark_pos[0]
    cube_model[:, 1] += mark_pos[1] - L / 2
    cube_model[:, 2] += mark_pos[2]
    n_actions = grasp_seq.shape[0]                                        # :91-102
    if end_frame >= n_actions or end_frame == -1:
        end_frame = n_actions - 1
    if initial_frame > end_frame:
        initial_frame = end_frame - 1
    grasp_seq = np.asarray(grasp_seq)[initial_frame:end_frame + 1]
    n_actions = end_frame - initial_frame + 1
    grasp_point_num = grasp_seq[0].shape[0]
    verts = np.asarray(mesh_vertices, dtype=np.float64) * s               # :106
    tris = np.asarray(mesh_triangles)
    grasp_seq = grasp_seq * s                                             # :109-111
    cube_model = cube_model * s
    target = np.asarray(target_pcd) * s
    area = mesh_area(verts, tris)                                         # :112
    n_v, n_t = verts.shape[0], tris.shape[0]
    n_op = int(op["n_operator_particles"] / grasp_point_num) * grasp_point_num   # :115
    n_c = cube_model.shape[0]
    garment_rho = garment_mass / (area * dx)                              # :118
    edge = op["operator_edge_length"] * s                                 # :119
    L = L * s
    cube_p_mass = cube["cube_mass"] / n_c                                 # :123
    operator_p_mass = op["operator_mass"] / n_op                          # :125
    quadrature_p_vol = 3 * area * dx / n_t                                # :127
    vertex_p_vol = area * dx / n_v                                        # :128
    quadrature_p_mass = garment_mass / n_v                                # :129
    vertex_p_mass = vertex_p_vol * garment_rho                            # :130
    group = int(n_op / grasp_point_num)                                   # :164
    op_model = (np.asarray(operator_random) - 0.5) * edge                 # :165-169
    vmin, vmax = verts.min(0), verts.max(0)                               # :171-182
    scene = np.concatenate((verts, grasp_seq.reshape(-1, 3)))
    center = (scene.max(0) - scene.min(0)) / 2 + scene.min(0)
    bottom = np.array([center[0], 0, center[2]])
    new_center = np.array([0.5, 2 * dx, 0.5])
    verts = verts + new_center - bottom
    grasp_point_pos = grasp_seq + new_center - bottom
    cube_model = cube_model + new_center - bottom
    target = target + new_center - bottom
    max_steps = int(gui / dt) + 1                                         # :193
    operator_x = np.concatenate([op_model + grasp_point_pos[0][g] for g in range(grasp_point_num)])  # simulation.py:433-438
    const = Constants(
        n_grid=n_grid, dt=dt, vertex_p_mass=vertex_p_mass, quadrature_p_mass=quadrature_p_mass,
        quadrature_p_vol=quadrature_p_vol, operator_p_mass=operator_p_mass, cube_p_mass=cube_p_mass,
        gravity_dv=dt * s * -9.81, bound=3, operator_update_interval=interval,
        frames_per_window=int(gui / interval), grasper_group_size=group, n_actions=n_actions)
    return dict(const=const, vertices=verts, triangles=tris, operator_x=operator_x, cube_x=cube_model,
                grasp_point_pos=grasp_point_pos, targets=target, max_steps=max_steps, area=area,
                garment_mass=garment_mass, n_operator=n_op)
