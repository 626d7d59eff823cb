"""Instance sharding across GPUs (one process per GPU).

Cloth instances are independent: a batch shards by instance with no
exchange on the data path.  Each rank simulates its own shard on its own GPU;
the only collectives are the gather of per-instance results at the end and
the max over ranks of the device time.  Shards are balanced by particle count
(longest-first greedy assignment), and every rank keeps its instances in the
batch's original order.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def partition(sizes: Sequence[float], world: int) -> List[List[int]]:
    """Instance indices of each of ``world`` shards, balanced by ``sizes``
    (largest first onto the lightest shard), each shard in ascending order."""
    if world < 1:
        raise ValueError("world must be positive")
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-float(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(sizes[i])
    return [sorted(s) for s in out]


def my_shard(scenes: Sequence, rank: int, world: int,
             size: Callable[[object], float] = lambda s: s.n_vertex + s.n_tri) -> Tuple[List[int], list]:
    """(indices, scenes) of this rank's shard."""
    idx = partition([size(s) for s in scenes], world)[rank]
    return idx, [scenes[i] for i in idx]


def gather_rows(local: np.ndarray, indices: Sequence[int], n_total: int) -> np.ndarray:
    """Assemble per-instance rows computed on every rank into one array of
    ``n_total`` rows, available on every rank (all_gather of each rank's
    (indices, rows)); without an initialised process group the local rows are
    the whole result."""
    import torch.distributed as dist
    local = np.asarray(local)
    if not (dist.is_available() and dist.is_initialized()):
        if len(indices) != n_total:
            raise ValueError("without a process group the local shard must hold every instance")
        out = np.empty((n_total,) + local.shape[1:], dtype=local.dtype)
        out[np.asarray(indices, dtype=np.int64)] = local
        return out
    parts = [None] * dist.get_world_size()
    dist.all_gather_object(parts, (list(indices), local))
    out = np.empty((n_total,) + local.shape[1:], dtype=local.dtype)
    seen = np.zeros(n_total, dtype=bool)
    for idx, rows in parts:
        if len(idx):
            out[np.asarray(idx, dtype=np.int64)] = rows
            seen[np.asarray(idx, dtype=np.int64)] = True
    if not seen.all():
        raise RuntimeError("instances missing from every shard: %s" % np.nonzero(~seen)[0][:8].tolist())
    return out


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of ``value`` over all ranks (all_reduce MAX); ``value``
    itself without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sharded_loss_and_grads(scenes: Sequence, n_steps: int, rank: int, world: int, dt: float,
                           ckpt_every: int = 1, device=None, **batch_kw) -> Tuple[np.ndarray, np.ndarray]:
    """Per-instance Chamfer loss (n,) and parameter gradients (n, 8) of all
    ``scenes``, each rank simulating its shard on ``device``; results are
    gathered on every rank."""
    from .batch import BatchSim, ClothBatch
    idx, mine = my_shard(scenes, rank, world)
    if mine:
        b = ClothBatch(mine, dt=dt, device=device, **batch_kw)
        sim = BatchSim(b, n_steps=n_steps, ckpt_every=ckpt_every)
        params = b.params.clone().requires_grad_(True)
        loss = sim.loss(params, b.traj)
        loss.sum().backward()
        lo = loss.detach().double().cpu().numpy()
        gp = params.grad.double().cpu().numpy()
    else:
        lo, gp = np.zeros((0,)), np.zeros((0, 8))
    return gather_rows(lo, idx, len(scenes)), gather_rows(gp, idx, len(scenes))
