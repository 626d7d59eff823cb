"""ctypes binding of ``libdiffcp_b200.so`` (declared in include/diffcp_b200.h).

The product path has no fallback: if the shared library is missing or fails to
load, :func:`lib` raises.  Build it with ``python -m diffcp_b200.build``.
"""
from __future__ import annotations

import ctypes
import os

from . import build as _build

c_int32 = ctypes.c_int32
c_int64 = ctypes.c_int64
c_float = ctypes.c_float
c_void_p = ctypes.c_void_p
_fp = ctypes.POINTER(ctypes.c_float)

DCP_OK = 0
DCP_ERR_INVALID = 1
DCP_ERR_CUDA = 2
GRIP_NONE, GRIP_OPERATOR, GRIP_KINEMATIC = 0, 1, 2
SVD_GRAD = {"exact": 0, "reference": 1}
STATUS_OUT_OF_DOMAIN, STATUS_NONFINITE, STATUS_POOL_FULL = 1, 2, 4

EXPORTED = (
    "dcp_plan", "dcp_create", "dcp_destroy", "dcp_sizes", "dcp_init_state", "dcp_substep_forward",
    "dcp_substep_backward", "dcp_chamfer_forward", "dcp_chamfer_backward", "dcp_rollout_floats", "dcp_tape_bytes", "dcp_reset_quadrature", "dcp_replay",
    "dcp_rollout_state_offset", "dcp_rollout_forward", "dcp_rollout_backward", "dcp_read_status", "dcp_last_error",
    "dcp_launch_count", "dcp_profile", "dcp_profile_read", "dcp_profile_launches", "dcp_kernel_count", "dcp_kernel_name",
    "dcp_chamfer_forward_static",
)
STATIC_MAX_TARGETS = 1 << 20


class DcpInstance(ctypes.Structure):
    _fields_ = [
        ("n_vertex", c_int32), ("n_tri", c_int32), ("n_operator", c_int32), ("n_cube", c_int32),
        ("n_target", c_int32), ("n_grid", c_int32), ("bound", c_int32),
        ("vertex_p_mass", c_float), ("quadrature_p_mass", c_float), ("quadrature_p_vol", c_float),
        ("operator_p_mass", c_float), ("cube_p_mass", c_float), ("gravity_dv", c_float),
        ("gripper_mode", c_int32), ("n_grippers", c_int32), ("group_size", c_int32), ("n_actions", c_int32),
        ("keyframe_interval", c_float), ("frames_per_window", c_int32), ("gripper_radius", c_float),
        ("n_traj_steps", c_int32),
    ]


class DcpOptions(ctypes.Structure):
    _fields_ = [("dt", c_float), ("chunk", c_int32), ("svd_grad", c_int32), ("grid_ctas", c_int32),
                ("scatter_mode", c_int32), ("min_blocks", c_int32 * 3),
                ("adj_scatter_mode", c_int32), ("pool_blocks", c_int32)]


class DcpSizes(ctypes.Structure):
    _fields_ = [(n, c_int64) for n in (
        "n_vertex", "n_tri", "n_operator", "n_cube", "n_target", "state_floats", "rest_floats", "traj_floats",
        "param_floats", "static_bytes", "workspace_bytes", "n_tri_chunks", "n_point_chunks", "total_nodes",
        "grid_blocks")]


_LIB = None


class DcpError(RuntimeError):
    pass


def lib_path() -> str:
    return _build.LIB


def lib():
    """Load (building first if stale or missing) the native library."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path) or _build._stale(path, [os.path.join(_build.CSRC, f) for f in
                                                         _build.SOURCES + _build.HEADERS]):
        _build.build()
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    L.dcp_plan.argtypes = [P(DcpInstance), c_int32, P(DcpOptions), P(DcpSizes)]
    L.dcp_create.argtypes = [P(DcpInstance), c_int32, P(DcpOptions), P(c_int32), P(c_int32), c_void_p, c_void_p,
                             c_void_p, P(c_void_p)]
    L.dcp_destroy.argtypes = [c_void_p]
    L.dcp_sizes.argtypes = [c_void_p, P(DcpSizes)]
    L.dcp_init_state.argtypes = [c_void_p] + [c_void_p] * 5 + [c_void_p]
    L.dcp_substep_forward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p,
                                      c_void_p]
    L.dcp_substep_backward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p,
                                       c_void_p, c_void_p, c_void_p, c_void_p]
    L.dcp_chamfer_forward.argtypes = [c_void_p] * 7
    L.dcp_chamfer_backward.argtypes = [c_void_p] * 8
    L.dcp_rollout_floats.argtypes = [c_void_p, c_int32, c_int32]
    L.dcp_rollout_floats.restype = c_int64
    L.dcp_rollout_state_offset.argtypes = [c_void_p, c_int32, c_int32, c_int32]
    L.dcp_rollout_state_offset.restype = c_int64
    L.dcp_reset_quadrature.argtypes = [c_void_p] * 5
    L.dcp_replay.argtypes = [c_void_p] * 7 + [c_int32] * 4 + [c_void_p]
    L.dcp_tape_bytes.argtypes = [c_void_p, c_int32, c_int64]
    L.dcp_tape_bytes.restype = c_int64
    L.dcp_rollout_forward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_void_p,
                                      c_void_p, c_int64, c_int32, c_void_p]
    L.dcp_rollout_backward.argtypes = [c_void_p, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_int32, c_int32,
                                       c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int64, c_int32, c_void_p]
    L.dcp_read_status.argtypes = [c_void_p, P(c_int32), c_int32, c_void_p]
    L.dcp_last_error.restype = ctypes.c_char_p
    L.dcp_launch_count.argtypes = [c_void_p]
    L.dcp_launch_count.restype = c_int64
    L.dcp_profile.argtypes = [c_void_p, c_int32]
    L.dcp_profile_read.argtypes = [c_void_p, P(ctypes.c_double), P(c_int64)]
    L.dcp_profile_launches.argtypes = [c_void_p, c_int32, P(ctypes.c_double), c_int64]
    L.dcp_profile_launches.restype = c_int64
    L.dcp_kernel_count.restype = c_int32
    L.dcp_kernel_name.argtypes = [c_int32]
    L.dcp_kernel_name.restype = ctypes.c_char_p
    L.dcp_chamfer_forward_static.argtypes = [c_void_p, c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_void_p,
                                             c_void_p]
    for name in EXPORTED:
        getattr(L, name)
    _LIB = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != DCP_OK:
        msg = lib().dcp_last_error().decode(errors="replace")
        raise DcpError("%s failed (code %d): %s" % (what or "diffcp_b200 call", rc, msg))
