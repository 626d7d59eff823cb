"""Launch-configuration autotuner for a batch of cloths.

Chooses, by timing a few eager forward and adjoint substeps of the actual
workload on the device:
  * ``chunk``        particles per CTA (32, 64, 128, 256),
  * ``scatter_mode`` warp-aggregated runs (0), one atomic per particle and
                     node (1), or lane pairs sharing a base cell (2), for
                     the two P2G kernels, and ``adj_scatter_mode`` likewise
                     for the adjoint G2P kernel, each from its own kernels'
                     CUDA-event times,
  * ``min_blocks``   the register-cap level of each register-heavy kernel
                     (k_tri_forward, k_g2p_adj, k_tri_adj; 1 none, 2 128,
                     3 96, 4 80, 5 72, 6 64 registers), chosen per kernel
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
P2G = ("k_tri_forward", "k_point_p2g")
ADJ = ("k_g2p_adj",)
DEFAULT = {"chunk": 128, "scatter_mode": 0, "adj_scatter_mode": 0, "min_blocks": [2, 2, 1]}
LEVELS = (1, 2, 3, 4, 5, 6)   # register-cap levels (DcpOptions.min_blocks)


def batch_kwargs(cfg: dict) -> dict:
    """ClothBatch keyword arguments of a tuned configuration (entries tuned
    before the adjoint scatter had its own mode use the P2G mode for both)."""
    return {"chunk": cfg["chunk"], "scatter_mode": cfg["scatter_mode"], "min_blocks": cfg["min_blocks"],
            "adj_scatter_mode": cfg.get("adj_scatter_mode", cfg["scatter_mode"])}


def signature(scenes: Sequence[ClothScene], dt: float) -> str:
    h = hashlib.sha1()
    h.update(np.array([len(scenes), dt], dtype=np.float64).tobytes())
    for sc in scenes:
        h.update(np.array([sc.n_vertex, sc.n_tri, len(sc.operator_x), len(sc.cube_x), sc.n_grid,
                           sc.gripper_mode], dtype=np.int64).tobytes())
    return h.hexdigest()[:16]


def _time_substeps(batch: ClothBatch, substeps: int) -> Dict[str, float]:
    """Per-kernel milliseconds of ``substeps`` forward + adjoint substeps.

    The adjoint starts from a seeded random state adjoint: from a zero one
    every scatter contribution of the adjoint kernels is zero, the scatters
    that skip zero contributions issue no atomics, and their times say
    nothing about a rollout's adjoint."""
    states = [batch.init_state()]
    for f in range(substeps):
        states.append(batch.forward_step(states[-1], f))
    gp, gt = batch.new_grads()
    gen = torch.Generator(device=batch.device).manual_seed(0)
    adj = torch.randn(batch.S, device=batch.device, generator=gen) * 1e-3
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
    modes = (0, 1, 2)
    runs = []
    for chunk in (32, 64, 128, 256):
        per_mode = {}
        for mode in modes:
            # the same mode for P2G and the adjoint: the two scatters are timed
            # by their own kernels and combined below
            b = ClothBatch(scenes, dt=dt, chunk=chunk, scatter_mode=mode, adj_scatter_mode=mode,
                           min_blocks=DEFAULT["min_blocks"], device=device)
            _time_substeps(b, 1)
            t = _time_substeps(b, substeps)
            per_mode[mode] = t
            if verbose:
                print("chunk %3d scatter %d: %.3f ms %s" % (chunk, mode, sum(t.values()),
                                                           {k: round(v, 3) for k, v in sorted(t.items())}))
            b.close()
            del b
        part = lambda t, ks: sum(t.get(k, 0.0) for k in ks)
        pm = min(modes, key=lambda m: part(per_mode[m], P2G))
        am = min(modes, key=lambda m: part(per_mode[m], ADJ))
        total = sum(per_mode[pm].values()) - part(per_mode[pm], ADJ) + part(per_mode[am], ADJ)
        runs.append((total, chunk, pm, am))
    runs.sort(key=lambda r: r[0])
    _, chunk, mode, adj_mode = runs[0]
    per_level = {}
    for level in LEVELS:
        b = ClothBatch(scenes, dt=dt, chunk=chunk, scatter_mode=mode, adj_scatter_mode=adj_mode,
                       min_blocks=(level,) * 3, device=device)
        _time_substeps(b, 1)
        per_level[level] = _time_substeps(b, substeps)
        b.close()
        del b
    mb = [min(LEVELS, key=lambda lv: per_level[lv].get(k, float("inf"))) for k in HEAVY]
    cfg = {"chunk": chunk, "scatter_mode": mode, "adj_scatter_mode": adj_mode, "min_blocks": mb}
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
