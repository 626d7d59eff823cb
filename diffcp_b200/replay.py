"""Forward-only state-estimation replay.

The reference replays a grasp with fitted material parameters and writes the
cloth's pose meshes (state_estimation_main.py:1-11, animation() of
simulation_without_grad.py:487-520): blocks of int(IFS / dt) substeps (IFS =
1 ms) of the same substep as the differentiable path, without the grasp-window
offset, each block followed by ``reset_quadrature_particles`` -- every
triangle's rest frame is rebuilt from its current vertices while its stored
deformation gradient is kept for the next substep's stress.  After the reset
of block ``count``, pose file ``i.ply`` is written for every
i in 0..n_pose_estimation_output with count == int(N * i / n - 2), N =
animation_time / IFS.

:class:`Replay` runs that loop on all cloths of a :class:`ClothBatch` at once
through the C ABI (``dcp_replay``: the block's substeps and the reset in one
call); :func:`animation` and :func:`main` reproduce the reference's files.
"""
from __future__ import annotations

import argparse
import json
import os
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import io_ply
from .batch import ClothBatch, _ptr, _stream
from .native import check

IFS = 0.001
POSE_COLOR = (30 / 255, 141 / 255, 255 / 255)


def pose_schedule(animation_time: float, n_out: int, ifs: float = IFS) -> Tuple[int, Dict[int, List[int]]]:
    """(number of blocks, {block: pose indices written after it}) of
    simulation_without_grad.py:508-516, truncating like Python's int()."""
    n_counts = int(animation_time / ifs)
    hits: Dict[int, List[int]] = {}
    for i in range(n_out + 1):
        c = int((animation_time / ifs) * i / n_out - 2)
        if 0 <= c < n_counts:
            hits.setdefault(c, []).append(i)
    return n_counts, hits


class Replay:
    """Forward-only replay of every cloth of ``batch`` from its rest state.

    ``block`` substeps per reset (default int(IFS / dt)).  The batch's rest
    buffer is re-based by every reset; the next differentiable rollout on the
    batch re-initialises it from the batch's rest positions.
    """

    def __init__(self, batch: ClothBatch, params: Optional[torch.Tensor] = None,
                 traj: Optional[torch.Tensor] = None, block: Optional[int] = None, ifs: float = IFS):
        self.batch = batch
        self.params = batch.params if params is None else params
        self.traj = batch.traj if traj is None else traj
        self.block = int(ifs / batch.dt) if block is None else int(block)
        if self.block < 1:
            raise ValueError("a replay block needs at least one substep")
        self.state = batch.init_state()
        self.work = batch.new_state()
        self.fdev = torch.zeros(max(9 * batch.nt, 1), dtype=torch.float32, device=batch.device)
        self.step = 0
        self.pending = False

    def run(self, n_blocks: int = 1) -> None:
        """``n_blocks`` blocks of substeps, each followed by the reset."""
        b = self.batch
        check(b.lib.dcp_replay(b.handle, _ptr(self.params), _ptr(self.traj), _ptr(b.rest), _ptr(self.state),
                               _ptr(self.work), _ptr(self.fdev), self.step, int(n_blocks), self.block,
                               int(self.pending), _stream()), "dcp_replay")
        if n_blocks > 0:
            self.step += n_blocks * self.block
            self.pending = True

    def vertices(self, i: int = 0) -> np.ndarray:
        """(Nv_i, 3) current vertex positions of cloth i (original order)."""
        return self.batch.vertex_x(self.state, i).double().cpu().numpy()


def animation(rep: Replay, animation_time: float, n_pose_estimation_output: int, out_dirs: Sequence[str],
              ifs: float = IFS, on_pose: Optional[Callable[[int, int, np.ndarray], None]] = None) -> List[int]:
    """animation() of simulation_without_grad.py:487-520 for every cloth of
    the replay: ``out_dirs[c]`` receives cloth c's pose meshes ``i.ply``
    (double xyz, vertex normals, uniform colour).  Returns the pose indices
    written, in order."""
    n_counts, hits = pose_schedule(animation_time, n_pose_estimation_output, ifs)
    written = []
    for d in out_dirs:
        os.makedirs(d, exist_ok=True)
    for count in range(n_counts):
        rep.run(1)
        for i in hits.get(count, []):
            for c, d in enumerate(out_dirs):
                v = rep.vertices(c)
                tris = np.asarray(rep.batch.scenes[c].triangles)
                io_ply.write_ply(os.path.join(d, "%d.ply" % i), v, tris, normals=io_ply.vertex_normals(v, tris),
                                 colors=POSE_COLOR)
                if on_pose is not None:
                    on_pose(c, i, v)
            written.append(i)
    return written


def main(argv: Optional[Sequence[str]] = None) -> List[int]:
    """state_estimation_main.py: read the fitted parameters (the reference
    reads ``fitting_result.json`` in its result directory), replay the whole
    grasp trajectory and write the pose meshes to
    ``<result dir>/pose_estimation_output``; also saves the rest vertices to
    ``<src>/../tmp/initial_vertices.npy`` as the reference does."""
    ap = argparse.ArgumentParser(prog="python -m diffcp_b200.replay")
    ap.add_argument("--src", required=True, help="directory holding simulation_arguments.json")
    ap.add_argument("--params", default=None, help="fitted-parameter JSON (default: <result dir>/fitting_result.json)")
    ap.add_argument("--seed", type=int, default=0, help="seed of the operator cloud")
    ap.add_argument("--seed-cube", type=int, default=None, help="seed of the cube cloud (default: --seed)")
    ap.add_argument("--out", default=None, help="pose directory (default: <result dir>/pose_estimation_output)")
    a = ap.parse_args(argv)
    from .scene import load_reference_scene
    with open(os.path.join(a.src, "simulation_arguments.json")) as fh:
        args = json.load(fh)
    result_dir = a.src + args["result_dir"]
    with open(a.params or os.path.join(result_dir, "fitting_result.json")) as fh:
        fit = json.load(fh)
    sc = load_reference_scene(a.src, seed=a.seed, args=args, seed_cube=a.seed_cube)
    for k in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        sc.params[k] = fit[k]
    tmp = os.path.join(a.src, "..", "tmp")
    os.makedirs(tmp, exist_ok=True)
    np.save(os.path.join(tmp, "initial_vertices.npy"), sc.vertices)
    batch = ClothBatch([sc], dt=sc.meta["dt"])
    rep = Replay(batch)
    anim = sc.keyframe_interval * (sc.keyframes.shape[0] - 1)
    out = a.out or os.path.join(result_dir, "pose_estimation_output")
    return animation(rep, anim, int(args["n_pose_estimation_output"]), [out])


if __name__ == "__main__":
    main()
