"""Batched cloth simulation on one GPU: device buffers, substeps, rollouts with
checkpointing, Chamfer loss, and the ``torch.autograd.Function`` that ties them
together.  All compute goes through the C ABI of ``libdiffcp_b200.so``;
PyTorch provides device memory and streams only.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import native
from .native import DcpInstance, DcpOptions, DcpSizes, check
from .scene import ClothScene, morton_order

PRM_STRIDE = 8
# Floats per particle in a state snapshot (vertex / operator / cube, triangle)
# and per triangle in the rest buffer (include/diffcp_b200.h).
POINT_STATE, TRI_STATE, TRI_REST = 15, 18, 21


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    if t is None:
        return None
    return t.data_ptr()


def _stream() -> int:
    return torch.cuda.current_stream().cuda_stream


def stencil_blocks(points: np.ndarray, n_grid: int) -> np.ndarray:
    """Block-major ids of the 4^3-node grid blocks that the quadratic stencils
    of ``points`` ([n, 3], metres) touch: base cell floor(x / dx - 0.5)
    (clamped as the kernels clamp it), nodes base .. base + 2 per axis."""
    pts = np.asarray(points, dtype=np.float64).reshape(-1, 3)
    base = np.clip(np.floor(pts * n_grid - 0.5), 0, n_grid - 3).astype(np.int64)
    nb = (n_grid + 3) // 4
    ids = [(((base + o) >> 2) * np.array([nb * nb, nb, 1])).sum(1)
           for o in np.array([[i, j, k] for i in (0, 2) for j in (0, 2) for k in (0, 2)])]
    return np.unique(np.concatenate(ids)) if len(pts) else np.zeros(0, dtype=np.int64)


def auto_pool_blocks(scenes: Sequence[ClothScene], margin: float = 4.0) -> int:
    """Pool size for paged grids: ``margin`` times the blocks that the rest
    configuration's particles (vertices, triangle centroids, operator and
    cube particles) touch, plus 256, at most every block of every grid."""
    touched = sum(len(stencil_blocks(np.concatenate([np.asarray(sc.vertices).reshape(-1, 3),
                                                     np.asarray(sc.vertices)[np.asarray(sc.triangles)].mean(1),
                                                     np.asarray(sc.operator_x).reshape(-1, 3),
                                                     np.asarray(sc.cube_x).reshape(-1, 3)]), sc.n_grid))
                  for sc in scenes)
    dense = sum(((sc.n_grid + 3) // 4) ** 3 for sc in scenes)
    return int(min(dense, int(np.ceil(margin * touched)) + 256))


class ClothBatch:
    """Instances of :class:`ClothScene` resident on one GPU.

    Particles of each instance are renumbered once into Morton order (a CTA's
    particles then cover a compact grid region); every public method takes and
    returns data in the scenes' original order.

    ``pool_blocks``: 0 keeps every instance's grid dense in memory; an int
    pages the grids through a pool of that many 4^3-node blocks shared by the
    batch; "auto" sizes the pool to ``pool_margin`` times the blocks the rest
    configuration touches (plus 256).  A substep that touches more blocks than
    the pool holds sets ``native.STATUS_POOL_FULL`` in :meth:`status`.
    """

    def __init__(self, scenes: Sequence[ClothScene], dt: float, chunk: int = 128, svd_grad: str = "exact",
                 grid_ctas: int = 0, device=None, reorder: bool = True, scatter_mode: int = 0,
                 min_blocks: Sequence[int] = (0, 0, 0), adj_scatter_mode: Optional[int] = None,
                 pool_blocks=0, pool_margin: float = 4.0):
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise ValueError("diffcp_b200 runs on CUDA devices only")
        if not torch.cuda.is_available():
            raise RuntimeError("diffcp_b200 needs a CUDA device")
        self.scenes = list(scenes)
        self.dt = float(dt)
        self.n_inst = len(self.scenes)
        self.lib = native.lib()
        n = self.n_inst
        insts = (DcpInstance * n)()
        tri_all, rank_all = [], []
        self.vperm, self.tperm = [], []
        xv, xo, xc = [], [], []
        for i, sc in enumerate(self.scenes):
            # Morton order of the stencil base cells (floor(x / dx - 0.5)): particles that
            # share a base cell, and so all 27 stencil nodes, sit next to each other
            dx = 1.0 / sc.n_grid
            vp = morton_order(sc.vertices - 0.5 * dx, dx) if reorder else np.arange(sc.n_vertex)
            inv = np.empty_like(vp)
            inv[vp] = np.arange(len(vp))
            tris = inv[np.asarray(sc.triangles)]
            cen = sc.vertices[vp][tris].mean(1)
            tp = morton_order(cen - 0.5 * dx, dx) if reorder else np.arange(sc.n_tri)
            tri_all.append(tris[tp])
            rank_all.append(vp)
            self.vperm.append(vp)
            self.tperm.append(tp)
            xv.append(sc.vertices[vp])
            xo.append(np.asarray(sc.operator_x).reshape(-1, 3))
            xc.append(np.asarray(sc.cube_x).reshape(-1, 3))
            I = insts[i]
            I.n_vertex, I.n_tri = sc.n_vertex, sc.n_tri
            I.n_operator, I.n_cube = len(xo[-1]), len(xc[-1])
            I.n_target = 0 if sc.targets is None else int(np.asarray(sc.targets).shape[0])
            I.n_grid, I.bound = sc.n_grid, sc.bound
            I.vertex_p_mass, I.quadrature_p_mass = sc.vertex_p_mass, sc.quadrature_p_mass
            I.quadrature_p_vol, I.operator_p_mass = sc.quadrature_p_vol, sc.operator_p_mass
            I.cube_p_mass, I.gravity_dv = sc.cube_p_mass, sc.gravity_dv
            I.gripper_mode, I.n_grippers, I.group_size = sc.gripper_mode, sc.n_grippers, sc.group_size
            I.n_actions = 0 if sc.keyframes is None else int(sc.keyframes.shape[0])
            I.keyframe_interval, I.frames_per_window = sc.keyframe_interval, sc.frames_per_window
            I.gripper_radius = sc.gripper_radius
            I.n_traj_steps = 0 if sc.velocities is None else int(sc.velocities.shape[0])
        self._insts = insts
        if pool_blocks == "auto":
            pool_blocks = auto_pool_blocks(self.scenes, pool_margin)
        self.pool_blocks = int(pool_blocks)
        opt = DcpOptions(dt=self.dt, chunk=chunk, svd_grad=native.SVD_GRAD[svd_grad], grid_ctas=grid_ctas,
                         scatter_mode=scatter_mode, min_blocks=(ctypes.c_int32 * 3)(*min_blocks),
                         adj_scatter_mode=scatter_mode if adj_scatter_mode is None else adj_scatter_mode,
                         pool_blocks=self.pool_blocks)
        self._opt = opt
        sizes = DcpSizes()
        check(self.lib.dcp_plan(insts, n, ctypes.byref(opt), ctypes.byref(sizes)), "dcp_plan")
        self.sizes = sizes
        self.static = torch.empty(max(int(sizes.static_bytes), 256), dtype=torch.uint8, device=self.device)
        self.workspace = torch.empty(max(int(sizes.workspace_bytes), 256), dtype=torch.uint8, device=self.device)
        tri_np = np.ascontiguousarray(np.concatenate(tri_all).astype(np.int32))
        rank_np = np.ascontiguousarray(np.concatenate(rank_all).astype(np.int32))
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(self.lib.dcp_create(insts, n, ctypes.byref(opt), tri_np.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                      rank_np.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), self.static.data_ptr(),
                                      self.workspace.data_ptr(), _stream(), ctypes.byref(handle)), "dcp_create")
        self.handle = handle
        f32 = dict(dtype=torch.float32, device=self.device)
        self.nv, self.nt = int(sizes.n_vertex), int(sizes.n_tri)
        self.no, self.nc, self.nq = int(sizes.n_operator), int(sizes.n_cube), int(sizes.n_target)
        self.S = int(sizes.state_floats)
        self.v_off = np.cumsum([0] + [sc.n_vertex for sc in self.scenes])
        self.t_off = np.cumsum([0] + [sc.n_tri for sc in self.scenes])
        self.q_off = np.cumsum([0] + [int(I.n_target) for I in insts])
        self.x0_vertex = torch.tensor(np.concatenate(xv).T.copy(), **f32).contiguous()
        self.x0_operator = torch.tensor(np.concatenate(xo).T.copy(), **f32).reshape(3, -1).contiguous()
        self.x0_cube = torch.tensor(np.concatenate(xc).T.copy(), **f32).reshape(3, -1).contiguous()
        self.params = torch.tensor(np.array([sc.param_row() + [0.0, 0.0] for sc in self.scenes]), **f32)
        self.traj = torch.tensor(self.pack_traj(), **f32) if sizes.traj_floats else torch.zeros(1, **f32)
        self.targets = self.pack_targets([sc.targets for sc in self.scenes]) if self.nq else torch.zeros(3, 1, **f32)
        self.rest = torch.empty(max(int(sizes.rest_floats), 1), **f32)

    # ------------------------------------------------------------- packing
    def pack_traj(self) -> np.ndarray:
        out = []
        for sc in self.scenes:
            if sc.gripper_mode == native.GRIP_OPERATOR:
                out.append(np.asarray(sc.keyframes, dtype=np.float64).reshape(-1))
            elif sc.gripper_mode == native.GRIP_KINEMATIC:
                out.append(np.asarray(sc.velocities, dtype=np.float64).reshape(-1))
                out.append(np.asarray(sc.centers, dtype=np.float64).reshape(-1))
        return np.concatenate(out) if out else np.zeros(0)

    def traj_slices(self, i: int):
        """(offset, length) of instance i's trajectory entries in the table."""
        off = 0
        for j, sc in enumerate(self.scenes):
            if sc.gripper_mode == native.GRIP_OPERATOR:
                ln = sc.keyframes.size
            elif sc.gripper_mode == native.GRIP_KINEMATIC:
                ln = 2 * sc.velocities.size
            else:
                ln = 0
            if j == i:
                return off, ln
            off += ln
        raise IndexError(i)

    def pack_targets(self, targets: List[np.ndarray]) -> torch.Tensor:
        arr = np.concatenate([np.asarray(t, dtype=np.float64).reshape(-1, 3) for t in targets])
        return torch.tensor(arr.T.copy(), dtype=torch.float32, device=self.device).contiguous()

    # ------------------------------------------------------------- views
    def vertex_x(self, state: torch.Tensor, i: int, absolute: bool = True) -> torch.Tensor:
        """(Nv_i, 3) positions (``absolute``) or displacements / adjoints of
        instance i in the scene's original order."""
        a, b = int(self.v_off[i]), int(self.v_off[i + 1])
        x = state[: 3 * self.nv].view(3, self.nv)[:, a:b]
        if absolute:
            x = x + self.rest_x0()[:, a:b]
        x = x.t()
        out = torch.empty_like(x)
        out[torch.as_tensor(self.vperm[i], device=x.device)] = x
        return out

    def rest_x0(self) -> torch.Tensor:
        """[3][Nv] rest vertex positions held in the rest buffer."""
        o = TRI_REST * self.nt
        return self.rest[o: o + 3 * self.nv].view(3, self.nv)

    def rest_n0(self) -> torch.Tensor:
        return self.rest[9 * self.nt: 12 * self.nt].view(3, self.nt)

    def absolute_fields(self, state: torch.Tensor):
        """Like :meth:`state_fields` with positions and d3 made absolute."""
        f = dict(self.state_fields(state))
        o = TRI_REST * self.nt + 3 * self.nv
        f["vx"] = f["vx"] + self.rest_x0()
        f["qd3"] = f["qd3"] + self.rest_n0()
        f["ox"] = f["ox"] + self.rest[o: o + 3 * self.no].view(3, self.no)
        o += 3 * self.no
        f["cx"] = f["cx"] + self.rest[o: o + 3 * self.nc].view(3, self.nc)
        return f

    def state_fields(self, state: torch.Tensor):
        """Dict of component-major views of one state snapshot (positions are
        displacements from the rest configuration, 'qd3' is d3 - n0; 'qx',
        'qv' the triangles' centroid position (absolute) and velocity)."""
        nv, nt, no, nc = self.nv, self.nt, self.no, self.nc
        P, T = POINT_STATE, TRI_STATE
        v = state[: P * nv].view(P, nv)
        t = state[P * nv: P * nv + T * nt].view(T, nt)
        o0 = P * nv + T * nt
        o = state[o0: o0 + P * no].view(P, no)
        c = state[o0 + P * no: o0 + P * no + P * nc].view(P, nc)
        return {"vx": v[0:3], "vv": v[3:6], "vC": v[6:15], "qC": t[0:9], "qd3": t[9:12], "qx": t[12:15],
                "qv": t[15:18], "ox": o[0:3], "ov": o[3:6], "oC": o[6:15], "cx": c[0:3], "cv": c[3:6],
                "cC": c[6:15]}

    def save_rest(self):
        """Copies of the rest positions (vertices, operator, cube)."""
        return self.x0_vertex.clone(), self.x0_operator.clone(), self.x0_cube.clone()

    def restore_rest(self, saved) -> None:
        self.x0_vertex.copy_(saved[0])
        self.x0_operator.copy_(saved[1])
        self.x0_cube.copy_(saved[2])

    def rebase_rest(self, state: torch.Tensor) -> None:
        """Make the positions of ``state`` the rest positions of the next
        :meth:`init_state` (the reference's window carry-over,
        parameter_fitting_functions.py:40-49: the end state's vertex, operator
        and cube positions become the initial positions and the triangles'
        rest shapes are rebuilt from them)."""
        f = self.absolute_fields(state)
        self.x0_vertex.copy_(f["vx"])
        if self.no:
            self.x0_operator.copy_(f["ox"])
        if self.nc:
            self.x0_cube.copy_(f["cx"])

    def new_state(self) -> torch.Tensor:
        return torch.zeros(self.S, dtype=torch.float32, device=self.device)

    # ------------------------------------------------------------- calls
    def init_state(self, out: Optional[torch.Tensor] = None, x0_vertex: Optional[torch.Tensor] = None):
        """State 0 and rest-shape inverses from the rest positions."""
        out = self.new_state() if out is None else out
        xv = self.x0_vertex if x0_vertex is None else x0_vertex
        check(self.lib.dcp_init_state(self.handle, _ptr(xv), _ptr(self.x0_operator), _ptr(self.x0_cube), _ptr(out),
                                      _ptr(self.rest), _stream()), "dcp_init_state")
        return out

    def forward_step(self, state_in, step: int, window: int = 0, out=None, params=None, traj=None):
        out = self.new_state() if out is None else out
        check(self.lib.dcp_substep_forward(self.handle, _ptr(self.params if params is None else params),
                                           _ptr(self.traj if traj is None else traj), _ptr(self.rest), step, window,
                                           _ptr(state_in), _ptr(out), _stream()), "dcp_substep_forward")
        return out

    def backward_step(self, state_in, adj_out, step: int, gparams, gtraj, window: int = 0, out=None, params=None,
                      traj=None):
        out = self.new_state() if out is None else out
        check(self.lib.dcp_substep_backward(self.handle, _ptr(self.params if params is None else params),
                                            _ptr(self.traj if traj is None else traj), _ptr(self.rest), step, window,
                                            _ptr(state_in), _ptr(adj_out), _ptr(out), _ptr(gparams), _ptr(gtraj),
                                            _stream()), "dcp_substep_backward")
        return out

    def chamfer(self, state, targets=None):
        targets = self.targets if targets is None else targets
        loss = torch.empty(self.n_inst, dtype=torch.float32, device=self.device)
        arg = torch.empty(max(self.nq, 1), dtype=torch.int32, device=self.device)
        check(self.lib.dcp_chamfer_forward(self.handle, _ptr(self.rest), _ptr(state), _ptr(targets), _ptr(arg),
                                           _ptr(loss), _stream()), "dcp_chamfer_forward")
        return loss, arg

    def chamfer_backward(self, state, argmin, gloss, adj, targets=None):
        targets = self.targets if targets is None else targets
        check(self.lib.dcp_chamfer_backward(self.handle, _ptr(self.rest), _ptr(state), _ptr(targets), _ptr(argmin),
                                            _ptr(gloss), _ptr(adj), _stream()), "dcp_chamfer_backward")
        return adj

    def rollout_buffer(self, n_steps: int, ckpt_every: int) -> torch.Tensor:
        nf = int(self.lib.dcp_rollout_floats(self.handle, n_steps, ckpt_every))
        return torch.empty(nf, dtype=torch.float32, device=self.device)

    def state_in_buffer(self, buf, n_steps, ckpt_every, step):
        off = int(self.lib.dcp_rollout_state_offset(self.handle, n_steps, ckpt_every, step))
        if off < 0:
            raise ValueError("state %d is not kept by a rollout with checkpoints every %d" % (step, ckpt_every))
        return buf[off: off + self.S]

    def tape_buffer(self, n_steps: int, blocks: int) -> torch.Tensor:
        """Grid tape for rollouts of n_steps substeps holding up to ``blocks``
        active 4^3 node blocks in total (1 KB each)."""
        nb = int(self.lib.dcp_tape_bytes(self.handle, n_steps, int(blocks)))
        if nb < 0:
            raise ValueError("bad tape size")
        return torch.empty(nb, dtype=torch.uint8, device=self.device)

    @staticmethod
    def tape_blocks(tape: torch.Tensor, n_steps: int) -> np.ndarray:
        """Per-substep (first slot or -1 when it did not fit, active blocks) of
        the last forward rollout recorded into ``tape``."""
        meta = tape[256: 256 + 8 * n_steps].view(torch.int32).reshape(n_steps, 2)
        return meta.cpu().numpy()

    def rollout_forward(self, buf, n_steps, ckpt_every, window=0, use_graph=True, params=None, traj=None, tape=None):
        check(self.lib.dcp_rollout_forward(self.handle, _ptr(self.params if params is None else params),
                                           _ptr(self.traj if traj is None else traj), _ptr(self.rest), window, n_steps,
                                           ckpt_every, _ptr(buf), _ptr(tape), 0 if tape is None else tape.numel(),
                                           int(use_graph), _stream()), "dcp_rollout_forward")

    def rollout_backward(self, buf, adj_work, n_steps, loss_step, ckpt_every, gparams, gtraj, window=0,
                         use_graph=True, params=None, traj=None, tape=None):
        check(self.lib.dcp_rollout_backward(self.handle, _ptr(self.params if params is None else params),
                                            _ptr(self.traj if traj is None else traj), _ptr(self.rest), window,
                                            n_steps, loss_step, ckpt_every, _ptr(buf), _ptr(adj_work),
                                            _ptr(gparams), _ptr(gtraj), _ptr(tape),
                                            0 if tape is None else tape.numel(), int(use_graph), _stream()),
              "dcp_rollout_backward")

    def launch_count(self) -> int:
        return int(self.lib.dcp_launch_count(self.handle))

    def profile(self, enable: bool) -> None:
        check(self.lib.dcp_profile(self.handle, int(enable)), "dcp_profile")

    def profile_read(self):
        """{kernel name: (total ms, launches)} of the launches since profile(True)."""
        k = int(self.lib.dcp_kernel_count())
        ms = (ctypes.c_double * k)()
        n = (ctypes.c_int64 * k)()
        check(self.lib.dcp_profile_read(self.handle, ms, n), "dcp_profile_read")
        return {self.lib.dcp_kernel_name(i).decode(): (ms[i], n[i]) for i in range(k) if n[i]}

    def profile_launches(self, name: str) -> np.ndarray:
        """Milliseconds of every profiled launch of kernel ``name``, in launch order."""
        names = [self.lib.dcp_kernel_name(i).decode() for i in range(int(self.lib.dcp_kernel_count()))]
        kid = names.index(name)
        n = int(self.lib.dcp_profile_launches(self.handle, kid, None, 0))
        out = (ctypes.c_double * max(n, 1))()
        got = int(self.lib.dcp_profile_launches(self.handle, kid, out, n))
        if got < 0:
            check(1, "dcp_profile_launches")
        return np.array(out[:n])

    def status(self, clear: bool = True) -> np.ndarray:
        out = (ctypes.c_int32 * self.n_inst)()
        check(self.lib.dcp_read_status(self.handle, out, int(clear), _stream()), "dcp_read_status")
        return np.array(out[:], dtype=np.int32)

    def new_grads(self):
        gp = torch.zeros(self.n_inst, PRM_STRIDE, dtype=torch.float64, device=self.device)
        gt = torch.zeros(max(int(self.sizes.traj_floats), 1), dtype=torch.float64, device=self.device)
        return gp, gt

    def close(self):
        if getattr(self, "handle", None):
            self.lib.dcp_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _RolloutLoss(torch.autograd.Function):
    """Chamfer loss of a rollout; gradients by the hand-written adjoint."""

    @staticmethod
    def forward(ctx, params, traj, sim, n_steps, loss_step, ckpt_every, window, use_graph):
        b = sim.batch
        L = loss_step
        buf = sim._buffer(L, ckpt_every)
        s0 = b.state_in_buffer(buf, L, ckpt_every, 0)
        b.init_state(out=s0, x0_vertex=sim.x0_vertex)
        tape = sim._tape_for(L)
        b.rollout_forward(buf, L, ckpt_every, window=window, use_graph=use_graph, params=params, traj=traj,
                          tape=tape)
        sim._tape_sized(tape, L)
        sL = b.state_in_buffer(buf, L, ckpt_every, L)
        loss, arg = b.chamfer(sL, sim.targets)
        # substeps after the loss state carry no gradient (the reference's loss
        # is taken two substeps before the end of the window)
        cur = sL
        for f in range(L, n_steps):
            nxt = sim._tail[(f - L) % 2]
            b.forward_step(cur, f, window, out=nxt, params=params, traj=traj)
            cur = nxt
        sim.final_state = cur.clone() if n_steps > L else sL.clone()
        ctx.sim, ctx.L, ctx.K, ctx.window, ctx.use_graph = sim, L, ckpt_every, window, use_graph
        ctx.buf, ctx.arg, ctx.tape = buf, arg, tape
        ctx.save_for_backward(params, traj)
        return loss

    @staticmethod
    def backward(ctx, gloss):
        params, traj = ctx.saved_tensors
        sim, L, K = ctx.sim, ctx.L, ctx.K
        b = sim.batch
        adj = sim._adj
        adj.zero_()
        sL = b.state_in_buffer(ctx.buf, L, K, L)
        b.chamfer_backward(sL, ctx.arg, gloss.contiguous().float(), adj[0], sim.targets)
        gp, gt = b.new_grads()
        b.rollout_backward(ctx.buf, adj, L, L, K, gp, gt, window=ctx.window, use_graph=ctx.use_graph, params=params,
                           traj=traj, tape=ctx.tape)
        sim.adj_state0 = adj[L % 2]
        return gp.to(params.dtype), gt[: traj.numel()].to(traj.dtype), None, None, None, None, None, None


class BatchSim:
    """Differentiable batched rollout + Chamfer loss.

    ``loss(params, traj)`` returns the per-instance loss (n_inst,), and
    ``backward()`` on it fills ``params.grad`` (n_inst, 8: dE, dnu,
    d shearing, d contact, d friction, d damping, 0, 0) and ``traj.grad``.

    ``tape``: "auto" records each forward substep's particle-to-grid result so
    that the adjoint restores it instead of recomputing P2G.  The first call
    only counts the active blocks per substep (and recomputes); the tape is
    then sized to ``tape_margin`` times that count.  Substeps that do not fit
    (the cloth spread over more blocks later) recompute.  None disables it; an
    int gives the capacity in blocks directly.
    """

    def __init__(self, batch: ClothBatch, n_steps: int, loss_step: Optional[int] = None, ckpt_every: int = 1,
                 use_graph: bool = True, tape="auto", tape_margin: float = 1.25):
        self.batch = batch
        self.n_steps = int(n_steps)
        self.loss_step = self.n_steps if loss_step is None else int(loss_step)
        self.ckpt_every = int(ckpt_every)
        self.use_graph = use_graph
        self.targets = batch.targets
        self.x0_vertex = batch.x0_vertex
        self._buf = None
        self._buf_key = None
        self._tail = [batch.new_state(), batch.new_state()]
        self._adj = torch.zeros(2, batch.S, dtype=torch.float32, device=batch.device)
        self.final_state = None
        self.adj_state0 = None
        self.tape_mode = tape
        self.tape_margin = float(tape_margin)
        self._tape = None
        self._tape_key = None

    def _tape_for(self, L):
        """The tape for a rollout of L substeps (None when disabled)."""
        if self.tape_mode is None:
            return None
        if self._tape_key != L:
            blocks = self.tape_mode if isinstance(self.tape_mode, int) else 0   # "auto": count first
            self._tape = self.batch.tape_buffer(L, blocks)
            self._tape_key = L
            self._tape_counted = isinstance(self.tape_mode, int)
        return self._tape

    def _tape_sized(self, tape, L):
        """After the counting rollout, replace the tape by one that fits."""
        if tape is None or self._tape_counted:
            return
        counts = ClothBatch.tape_blocks(tape, L)[:, 1].astype(np.int64)
        self._tape = self.batch.tape_buffer(L, int(np.ceil(counts.sum() * self.tape_margin)) + 64)
        self._tape_counted = True

    def _buffer(self, L, K):
        if self._buf_key != (L, K):
            self._buf = self.batch.rollout_buffer(L, K)
            self._buf_key = (L, K)
        return self._buf

    def loss(self, params: Optional[torch.Tensor] = None, traj: Optional[torch.Tensor] = None, window: int = 0):
        params = self.batch.params if params is None else params
        traj = self.batch.traj if traj is None else traj
        return _RolloutLoss.apply(params, traj, self, self.n_steps, self.loss_step, self.ckpt_every, window,
                                  self.use_graph)
