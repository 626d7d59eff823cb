"""Build and ctypes binding of oracle/cpu_port.cpp, the compiled CPU
restatement of the substep and its adjoint (TEST INFRASTRUCTURE and the timed
CPU baseline of bench.py; the product never imports it).

    python -m oracle.cpu_port      # builds oracle/lib/libcpu_port.so
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_port.cpp")
LIB = os.path.join(HERE, "lib", "libcpu_port.so")
HEADER = os.path.join(os.path.dirname(HERE), "diffcp_b200", "csrc", "cloth_math.cuh")
# x86-64-v3 (AVX2, FMA): built once here, run on the GPU host's cores too
FLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-std=c++17", "-shared", "-fPIC"]


class CpuScene(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("nv", "nt", "nq", "n_grid", "bound", "n_grip", "n_steps")] + \
               [(n, ctypes.c_double) for n in ("dt", "m_v", "m_q", "vol_q", "gravity_dv", "grip_radius", "E", "nu",
                                              "ks", "kc", "friction", "damping")] + \
               [("x0", ctypes.c_void_p), ("tris", ctypes.c_void_p), ("vel", ctypes.c_void_p),
                ("centers", ctypes.c_void_p), ("targets", ctypes.c_void_p)]


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC),
                                                                           os.path.getmtime(HEADER)):
        return LIB
    tmp = LIB + ".tmp"
    res = subprocess.run(["g++", *FLAGS, SRC, "-o", tmp], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("g++ failed for cpu_port.cpp:\n" + res.stdout + res.stderr)
    os.replace(tmp, LIB)
    return LIB


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(build())
        L.cpu_rollout_grad.argtypes = [ctypes.POINTER(CpuScene), ctypes.c_int32, ctypes.c_int32,
                                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                       ctypes.c_void_p]
        L.cpu_rollouts.argtypes = [ctypes.POINTER(CpuScene), ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
        _LIB = L
    return _LIB


class Scenes:
    """CpuScene structs of kinematic-gripper ClothScenes; holds the arrays
    they point to."""

    def __init__(self, scenes):
        self.keep = []
        self.arr = (CpuScene * len(scenes))()
        for i, sc in enumerate(scenes):
            if sc.gripper_mode != 2 or len(sc.operator_x) or len(sc.cube_x):
                raise ValueError("cpu_port covers kinematic-gripper sheets only")
            a = {"x0": np.ascontiguousarray(sc.vertices, dtype=np.float64),
                 "tris": np.ascontiguousarray(sc.triangles, dtype=np.int32),
                 "vel": np.ascontiguousarray(sc.velocities, dtype=np.float64),
                 "centers": np.ascontiguousarray(sc.centers, dtype=np.float64),
                 "targets": np.ascontiguousarray(sc.targets, dtype=np.float64)}
            self.keep.append(a)
            s = self.arr[i]
            s.nv, s.nt, s.nq = sc.n_vertex, sc.n_tri, a["targets"].shape[0]
            s.n_grid, s.bound, s.n_grip, s.n_steps = sc.n_grid, sc.bound, sc.n_grippers, a["vel"].shape[0]
            s.dt = float(sc.meta["dt"])
            s.m_v, s.m_q, s.vol_q, s.gravity_dv = sc.vertex_p_mass, sc.quadrature_p_mass, sc.quadrature_p_vol, \
                sc.gravity_dv
            s.grip_radius = sc.gripper_radius
            p = sc.params
            s.E, s.nu, s.ks, s.kc = p["E"], p["nu"], p["shearing_stiffness"], p["contact_stiffness"]
            s.friction, s.damping = p.get("friction", 0.0), p.get("damping", 0.95)
            for k in ("x0", "tris", "vel", "centers", "targets"):
                setattr(s, k, a[k].ctypes.data)


def rollout_grad(sc, n_steps: int, double: bool = True):
    """(loss, dL/d(E, nu, k_s, k_c, friction, damping), dL/d velocities) of
    one cloth over n_steps substeps."""
    S = Scenes([sc])
    loss = ctypes.c_double()
    g = (ctypes.c_double * 6)()
    gv = np.zeros_like(S.keep[0]["vel"])
    rc = lib().cpu_rollout_grad(S.arr, n_steps, int(double), ctypes.byref(loss), g, gv.ctypes.data)
    if rc:
        raise RuntimeError("cpu_rollout_grad failed")
    return loss.value, np.array(g[:]), gv


def rollouts(scenes, n_steps: int, n_threads: int):
    """float32 rollouts of several cloths in parallel; (losses, grads[n][6])."""
    S = Scenes(scenes)
    n = len(scenes)
    losses = (ctypes.c_double * n)()
    grads = (ctypes.c_double * (6 * n))()
    rc = lib().cpu_rollouts(S.arr, n, n_steps, n_threads, losses, grads)
    if rc:
        raise RuntimeError("cpu_rollouts failed")
    return np.array(losses[:]), np.array(grads[:]).reshape(n, 6)


if __name__ == "__main__":
    print(build(force="--force" in sys.argv or True))
