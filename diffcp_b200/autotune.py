"""Launch-configuration autotuner for a batch of cloths.

Chooses, by timing a few eager forward and adjoint substeps of the actual
workload on the device:
  * ``chunk``        particles per CTA (64, 128, 256),
  * ``scatter_mode`` warp-aggregated runs (0), one atomic per particle and
                     node (1), or lane pairs sharing a base cell (2),
  * ``min_blocks``   the register cap of each register-heavy kernel
                     (k_tri_forward, k_g2p_adj, k_tri_adj), chosen per kernel
                     from the per-kernel CUDA-event times of one run per level.
Results are cached per workload signature in ``tuned.json`` next to this
file (or a path given by the caller).
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Dict, Optional, Sequence

import numpy as np
import torch

from .batch import ClothBatch
from .scene import ClothScene

CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")
HEAVY = ("k_tri_forward", "k_g2p_adj", "k_tri_adj")
DEFAULT = {"chunk": 128, "scatter_mode": 0, "min_blocks": [2, 2, 1]}


def signature(scenes: Sequence[ClothScene], dt: float) -> str:
    h = hashlib.sha1()
    h.update(np.array([len(scenes), dt], dtype=np.float64).tobytes())
    for sc in scenes:
        h.update(np.array([sc.n_vertex, sc.n_tri, len(sc.operator_x), len(sc.cube_x), sc.n_grid,
                           sc.gripper_mode], dtype=np.int64).tobytes())
    return h.hexdigest()[:16]


def _time_substeps(batch: ClothBatch, substeps: int) -> Dict[str, float]:
    """Per-kernel milliseconds of ``substeps`` forward + adjoint substeps."""
    states = [batch.init_state()]
    for f in range(substeps):
        states.append(batch.forward_step(states[-1], f))
    gp, gt = batch.new_grads()
    adj = torch.zeros(batch.S, device=batch.device)
    torch.cuda.synchronize()
    batch.profile(True)
    for f in range(substeps):
        batch.forward_step(states[f], f, out=states[f + 1])
    a = adj
    for f in range(substeps - 1, -1, -1):
        a = batch.backward_step(states[f], a, f, gp, gt)
    torch.cuda.synchronize()
    prof = batch.profile_read()
    batch.profile(False)
    return {k: v[0] for k, v in prof.items()}


def tune(scenes: Sequence[ClothScene], dt: float, substeps: int = 3, device=None, cache: Optional[str] = CACHE,
         verbose: bool = False, force: bool = False) -> dict:
    key = signature(scenes, dt)
    table = {}
    if cache and os.path.exists(cache):
        with open(cache) as fh:
            table = json.load(fh)
        if key in table and not force:
            return table[key]["config"]
    runs = []
    for chunk in (64, 128, 256):
        for mode in (0, 1, 2):
            b = ClothBatch(scenes, dt=dt, chunk=chunk, scatter_mode=mode, min_blocks=DEFAULT["min_blocks"],
                           device=device)
            _time_substeps(b, 1)
            t = _time_substeps(b, substeps)
            runs.append((sum(t.values()), chunk, mode, t))
            if verbose:
                print("chunk %3d scatter %d: %.3f ms %s" % (chunk, mode, sum(t.values()),
                                                           {k: round(v, 3) for k, v in sorted(t.items())}))
            b.close()
            del b
    runs.sort(key=lambda r: r[0])
    _, chunk, mode, _ = runs[0]
    per_level = {}
    for level in (1, 2, 3, 4):
        b = ClothBatch(scenes, dt=dt, chunk=chunk, scatter_mode=mode, min_blocks=(level,) * 3, device=device)
        _time_substeps(b, 1)
        per_level[level] = _time_substeps(b, substeps)
        b.close()
        del b
    mb = [min((1, 2, 3, 4), key=lambda lv: per_level[lv].get(k, float("inf"))) for k in HEAVY]
    cfg = {"chunk": chunk, "scatter_mode": mode, "min_blocks": mb}
    if verbose:
        for lv, t in per_level.items():
            print("min_blocks %d: %s" % (lv, {k: round(t.get(k, 0.0), 3) for k in HEAVY}))
        print("chosen", cfg)
    if cache:
        table[key] = {"config": cfg, "instances": len(scenes), "dt": dt,
                      "particles": int(sum(s.n_vertex + s.n_tri for s in scenes)),
                      "device": torch.cuda.get_device_name(device)}
        with open(cache, "w") as fh:
            json.dump(table, fh, indent=1, sort_keys=True)
    return cfg


def cached(scenes: Sequence[ClothScene], dt: float, cache: str = CACHE) -> Optional[dict]:
    if not os.path.exists(cache):
        return None
    with open(cache) as fh:
        table = json.load(fh)
    ent = table.get(signature(scenes, dt))
    return ent["config"] if ent else None
