"""FP64 oracle runs on the GPU for the parity checks of the benchmark
configurations at their full sizes, and the FP32-vs-FP64 error measures the
checks report.

The oracle (``oracle/sim64.py``) keeps an autograd graph per substep; over
hundreds of substeps of a large cloth that graph does not fit in memory, so
the rollout is split into segments recomputed in the backward pass
(``torch.utils.checkpoint``, non-reentrant, so the parameters and gripper
velocities that the substeps read from the enclosing scope get gradients).
"""
from __future__ import annotations

import json
from typing import Dict, Sequence

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from oracle import sim64
from oracle.sim64 import KinematicGripper
from tests.scenes import oracle_for, oracle_params

KEYS = ("vx", "vv", "vC", "qx", "qv", "qC", "qF", "qd", "ox", "ov", "oC", "cx", "cv", "cC")
COL = {"E": 0, "nu": 1, "ks": 2, "kc": 3, "friction": 4, "damping": 5}


def chamfer64(x: torch.Tensor, t: torch.Tensor) -> torch.Tensor:
    """One-sided Chamfer (sum_q min_p |x_p - t_q|^2 / 3 / Nq) with the argmin
    taken in chunks; the loss is piecewise smooth, so its gradient is that of
    the selected pairs."""
    with torch.no_grad():
        arg = torch.cat([torch.cdist(t[i: i + 256], x).argmin(1) for i in range(0, t.shape[0], 256)])
    return ((x[arg] - t) ** 2).sum() / 3 / t.shape[0]


def oracle_loss_and_grads(sc, n_steps: int, keys: Sequence[str] = ("E", "nu", "friction", "damping"),
                          device="cuda", seg: int = 10, want_vel: bool = True):
    """FP64 oracle rollout of ``n_steps`` substeps of a kinematic-gripper scene
    on ``device``: Chamfer loss of the final state, its gradients with respect
    to ``keys`` and (``want_vel``) the per-substep gripper velocities, and the
    final vertex positions."""
    dev = torch.device(device)
    sim, st = oracle_for(sc, device=dev)
    p = {k: v.to(dev).requires_grad_(k in keys) for k, v in oracle_params(sc).items()}
    vel = torch.tensor(sc.velocities, dtype=torch.float64, device=dev, requires_grad=want_vel)
    grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=torch.float64, device=dev), vel)

    def run(f0, f1, *flat):
        s = dict(zip(KEYS, flat))
        for f in range(f0, f1):
            s = sim.substep(s, f, 0, p, friction=p["friction"], damping=p["damping"], grip=grip)
        return tuple(s[k] for k in KEYS)

    flat = tuple(st[k] for k in KEYS)
    for f0 in range(0, n_steps, seg):
        flat = checkpoint(run, f0, min(f0 + seg, n_steps), *flat, use_reentrant=False)
    vx = flat[0]
    loss = chamfer64(vx, torch.tensor(np.asarray(sc.targets), dtype=torch.float64, device=dev))
    loss.backward()
    grads = {k: float(p[k].grad) for k in keys}
    gvel = vel.grad.detach().cpu().numpy() if want_vel else None
    return float(loss.detach()), grads, gvel, vx.detach()


def oracle_loss_only(sc, n_steps: int, velocities=None, device="cuda") -> float:
    """FP64 oracle loss of the final state, no gradients (for finite differences)."""
    dev = torch.device(device)
    sim, st = oracle_for(sc, device=dev)
    p = {k: v.to(dev) for k, v in oracle_params(sc).items()}
    vel = torch.tensor(sc.velocities if velocities is None else velocities, dtype=torch.float64, device=dev)
    grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=torch.float64, device=dev), vel)
    with torch.no_grad():
        for f in range(n_steps):
            st = sim.substep(st, f, 0, p, friction=p["friction"], damping=p["damping"], grip=grip)
        return float(chamfer64(st["vx"], torch.tensor(np.asarray(sc.targets), dtype=torch.float64, device=dev)))


def errors(name: str, loss32: float, loss64: float, g32: Dict[str, float], g64: Dict[str, float],
           vel32=None, vel64=None, x32=None, x64=None) -> dict:
    """FP32-vs-FP64 errors of one instance: loss and each parameter gradient
    relative to the FP64 value, the velocity gradient as max-abs error over
    max-abs FP64 value, positions as max-abs error in metres."""
    rec = {"case": name, "loss_rel": abs(loss32 - loss64) / abs(loss64)}
    for k, r in g64.items():
        rec["d" + k + "_rel"] = abs(g32[k] - r) / abs(r) if r != 0 else float(abs(g32[k]))
    if vel64 is not None:
        rec["dvel_rel_max"] = float(np.abs(vel32 - vel64).max() / np.abs(vel64).max())
    if x64 is not None:
        rec["x_abs_max_m"] = float((x32.double() - x64).abs().max())
    print("PARITY " + json.dumps(rec))
    return rec
