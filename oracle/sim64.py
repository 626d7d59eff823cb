"""Torch restatement of the DiffCP substep, Chamfer loss and clamped SVD adjoint.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Every function below restates one kernel or helper of the reference
(``denzelzheng/diffcp``) and cites it as ``file:line``.  The restatement keeps
the reference's state layout (full ``F`` and ``d`` stored per substep), its
floating-point formulas, and its quirks:

* dead return mapping in ``update_particle_state`` (simulation.py:406-428) --
  it writes only a local and is therefore omitted here;
* ``A[0,0]`` written twice, the first write dead (simulation.py:216-217);
* the mixed ``r1``/``r2`` vectors built from ``D0^-1`` and the current ``d``
  (simulation.py:247-248);
* triangle ("quadrature") particles carry mass ``M/Nv`` on top of the vertex
  mass (simulation.py:262-263 with initialization.py:129);
* gravity ``dt*scene_scaling*g`` on vertices only, inside P2G (simulation.py:182);
* cube particles scatter affine momentum only (simulation.py:150-152);
* the keyframe index evaluated in float32 (simulation.py:160-161);
* ``d <- F . inv(D0^-1)`` round trip (simulation.py:429);
* ``norm(eps) = sqrt(|v|^2 + eps)`` with eps 1e-9 in QR and 1e-6 at init;
* the clamped 2x2 SVD backward (simulation.py:44-50,71-94) as ``svd_grad="reference"``;
* sticky walls on x, z and the y-top, a slip floor, and the asymmetric
  ``i > n_grid - bound`` / ``i < bound`` tests (simulation.py:279-300).

Two build extensions are switched off by default so that the default
reproduces the reference: Coulomb ground friction (``friction``) and a
kinematic sphere gripper on the grid (``KinematicGripper``); ``damping`` is the
removed fraction of the symmetric part of the triangle ``C``, 0.95 in the
reference (simulation.py:381-383).

The forward-only replay of simulation_without_grad.py (same substep, frame
index without window offset) adds ``OracleSim.reset_quadrature_particles``,
which rebuilds the rest frames and leaves the stored ``F``, and ``replay``.

Gradients: ``torch.autograd`` through the restatement.  ``svd_grad="exact"``
differentiates the closed-form rotation factor of the 2x2 polar decomposition
(the ``U V^T`` that the reference uses, simulation.py:235);
``svd_grad="reference"`` routes the gradient of ``U`` and ``V`` through the
reference's clamped SVD backward, as Taichi's tape does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np
import torch

OFFSETS_NP = np.array([[i, j, k] for i in range(3) for j in range(3) for k in range(3)], dtype=np.int64)
_OFF = torch.from_numpy(OFFSETS_NP)

STATE_KEYS = ("vx", "vv", "vC", "qx", "qv", "qC", "qF", "qd", "ox", "ov", "oC", "cx", "cv", "cC")


@dataclass
class KinematicGripper:
    """Build extension (no reference counterpart): grid nodes within ``radius``
    of a gripper centre take the gripper velocity.  ``centers``/``velocities``
    have shape (T, K, 3): one entry per substep and gripper."""
    radius: float
    centers: torch.Tensor
    velocities: torch.Tensor


@dataclass
class Constants:
    """Per-scene constants of initialization.py:22-23,79,118-130 plus the
    operator keyframe settings used by p2g (simulation.py:160-165)."""
    n_grid: int
    dt: float
    vertex_p_mass: float
    quadrature_p_mass: float
    quadrature_p_vol: float
    operator_p_mass: float = 0.0
    cube_p_mass: float = 0.0
    gravity_dv: float = 0.0            # dt * scene_scaling * gravity (simulation.py:182)
    bound: int = 3                     # initialization.py:22
    operator_update_interval: float = 0.03
    frames_per_window: int = 100       # int(grad_update_interval / operator_update_interval)
    grasper_group_size: int = 1
    n_actions: int = 0

    @property
    def dx(self) -> float:
        return 1.0 / self.n_grid        # initialization.py:79

    @property
    def inv_dx(self) -> float:
        return float(self.n_grid)


def _dot(a, b):
    return (a * b).sum(-1, keepdim=True)


def _norm_eps(v, eps):
    """``x.norm(eps)`` of Taichi: sqrt(x.x + eps) (used at simulation.py:128-132,471-474)."""
    return torch.sqrt((v * v).sum(-1, keepdim=True) + eps)


def stencil(x: torch.Tensor, inv_dx: float):
    """Quadratic B-spline stencil (simulation.py:140-142, 155-157, 177-179, 194-196).

    ``base`` is ``ti.cast(x*inv_dx - 0.5, ti.i32)`` (truncation toward zero),
    ``fx = x*inv_dx - base``; ``w`` has shape (N, 3 stencil, 3 axes) and ``W``
    (N, 27) is the tensor-product weight in (i, j, k) order.
    """
    s = x.detach() * inv_dx - 0.5
    base = torch.trunc(s).to(torch.long)
    fx = x * inv_dx - base.to(x.dtype)
    w = torch.stack((0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1.0) ** 2, 0.5 * (fx - 0.5) ** 2), dim=1)
    off = _OFF.to(x.device)
    W = w[:, off[:, 0], 0] * w[:, off[:, 1], 1] * w[:, off[:, 2], 2]
    return base, fx, w, W


def stencil_nodes(base: torch.Tensor, n_grid: int) -> torch.Tensor:
    """Flat (i*G + j)*G + k index of the 27 nodes of each stencil, shape (N, 27)."""
    node = base[:, None, :] + _OFF.to(base.device)[None]
    if (node.min() < 0) or (node.max() >= n_grid):
        raise ValueError("particle stencil leaves the grid (reference would index out of bounds)")
    return (node[..., 0] * n_grid + node[..., 1]) * n_grid + node[..., 2]


def qr_decomposition_3d(F: torch.Tensor):
    """Classical Gram-Schmidt QR of simulation.py:123-135; ``R = Q^-1 F``."""
    c1, c2, c3 = F[..., 0], F[..., 1], F[..., 2]
    q1 = c1 / _norm_eps(c1, 1e-9)
    q2h = c2 - _dot(c2, q1) * q1
    q2 = q2h / _norm_eps(q2h, 1e-9)
    q3h = c3 - _dot(c3, q1) * q1 - _dot(c3, q2) * q2
    q3 = q3h / _norm_eps(q3h, 1e-9)
    Q = torch.stack((q1, q2, q3), dim=-1)
    R = torch.linalg.inv(Q) @ F
    return Q, R


def polar_rotation_2x2(A: torch.Tensor) -> torch.Tensor:
    """Rotation factor ``U V^T`` of the 2x2 SVD used at simulation.py:235.

    The reference's ``ti.svd`` on 2x2 matrices (third-party: Taichi, version
    unpinned) first extracts the rotation polar factor from
    ``(A00 + A11, A10 - A01)`` and builds ``U = R_polar V``, so ``U V^T`` is that
    rotation for every input, inverted ones included.
    """
    x = A[..., 0, 0] + A[..., 1, 1]
    y = A[..., 1, 0] - A[..., 0, 1]
    r = torch.sqrt(x * x + y * y)
    c, s = x / r, y / r
    return torch.stack((torch.stack((c, -s), -1), torch.stack((s, c), -1)), -2)


def svd2_taichi(A: torch.Tensor):
    """U, Sigma, V of a 2x2 matrix in the convention of Taichi's ``ti.svd`` (2-D).

    Restated algorithm (Taichi ``svd2d``, version unpinned): rotation polar
    factor ``Rp`` from ``(A00 + A11, A10 - A01)``; ``S = Rp^T A`` is symmetric
    and is diagonalised by one Jacobi rotation (identity when ``|S01| < 1e-5``);
    singular values sorted in descending signed order, swapping the columns of
    ``V`` with a sign so that ``V`` stays a rotation; ``U = Rp V``.
    Returned tensors carry no autograd history.
    """
    A = A.detach()
    x = A[..., 0, 0] + A[..., 1, 1]
    y = A[..., 1, 0] - A[..., 0, 1]
    sc = 1.0 / torch.sqrt(x * x + y * y)
    c0, s0 = x * sc, y * sc
    Rp = torch.stack((torch.stack((c0, -s0), -1), torch.stack((s0, c0), -1)), -2)
    S = Rp.transpose(-1, -2) @ A
    S00, S01, S11 = S[..., 0, 0], S[..., 0, 1], S[..., 1, 1]
    tau = 0.5 * (S00 - S11)
    w = torch.sqrt(tau * tau + S01 * S01)
    t = torch.where(tau > 0, S01 / (tau + w), S01 / (tau - w))
    c = 1.0 / torch.sqrt(t * t + 1.0)
    s = -t * c
    s1 = c * c * S00 - 2.0 * c * s * S01 + s * s * S11
    s2 = s * s * S00 + 2.0 * c * s * S01 + c * c * S11
    small = S01.abs() < 1e-5
    one = torch.ones_like(c)
    c = torch.where(small, one, c)
    s = torch.where(small, torch.zeros_like(s), s)
    s1 = torch.where(small, S00, s1)
    s2 = torch.where(small, S11, s2)
    swap = s1 < s2
    sig_a = torch.where(swap, s2, s1)
    sig_b = torch.where(swap, s1, s2)
    V_keep = torch.stack((torch.stack((c, s), -1), torch.stack((-s, c), -1)), -2)
    V_swap = torch.stack((torch.stack((-s, c), -1), torch.stack((-c, -s), -1)), -2)
    V = torch.where(swap[..., None, None], V_swap, V_keep)
    U = Rp @ V
    zero = torch.zeros_like(sig_a)
    Sig = torch.stack((torch.stack((sig_a, zero), -1), torch.stack((zero, sig_b), -1)), -2)
    return U, Sig, V


def _clamp_ref(a: torch.Tensor) -> torch.Tensor:
    """Sign-preserving magnitude floor of simulation.py:44-50 (0 maps to +1e-6)."""
    return torch.where(a >= 0, torch.clamp(a, min=1e-6), torch.clamp(a, max=-1e-6))


def svd_backward_clamped(gU, gS, gV, U, S, V):
    """backward_inplane_svd of simulation.py:71-88 (2x2), batched."""
    Vt = V.transpose(-1, -2)
    Ut = U.transpose(-1, -2)
    sigma_term = U @ gS @ Vt
    s0 = S[..., 0, 0] ** 2
    s1 = S[..., 1, 1] ** 2
    zero = torch.zeros_like(s0)
    Fm = torch.stack((torch.stack((zero, 1.0 / _clamp_ref(s1 - s0)), -1),
                      torch.stack((1.0 / _clamp_ref(s0 - s1), zero), -1)), -2)
    u_term = U @ ((Fm * (Ut @ gU - gU.transpose(-1, -2) @ U)) @ S) @ Vt
    v_term = U @ (S @ ((Fm * (Vt @ gV - gV.transpose(-1, -2) @ V)) @ Vt))
    return u_term + v_term + sigma_term


class TaichiSvd2(torch.autograd.Function):
    """``inplane_svd`` forward (simulation.py:39-42) with the reference's manual
    backward ``inplane_svd_grad`` (simulation.py:90-94) as its adjoint."""

    @staticmethod
    def forward(ctx, A):
        U, S, V = svd2_taichi(A)
        ctx.save_for_backward(U, S, V)
        return U, S, V

    @staticmethod
    def backward(ctx, gU, gS, gV):
        U, S, V = ctx.saved_tensors
        gU = torch.zeros_like(U) if gU is None else gU
        gS = torch.zeros_like(S) if gS is None else gS
        gV = torch.zeros_like(V) if gV is None else gV
        return svd_backward_clamped(gU, gS, gV, U, S, V)


def lame(E, nu):
    """simulation.py:230-232."""
    mu = E / (2 * (1 + nu))
    la = E * nu / ((1 + nu) * (1 - 2 * nu))
    return mu, la


def triangle_stress(F, E, nu, ks, kc, svd_grad="exact"):
    """First Piola stress ``quadrature_P`` of simulation.py:214-240 (with the
    in-plane QR of compute_inplane_F_tmp, simulation.py:24-28, on the same F)."""
    Q, R = qr_decomposition_3d(F)
    Fh = R[..., :2, :2]
    R02, R12, R22 = R[..., 0, 2], R[..., 1, 2], R[..., 2, 2]
    A00 = ks * R02 * R02                      # line 216 is overwritten by line 217
    A01 = ks * R02 * R12
    A02 = ks * R02 * R22
    A11 = ks * R12 * R12
    A12 = ks * R12 * R22
    A22 = (R22 <= 1).to(F.dtype) * (-kc) * (1 - R22) ** 2 * R22
    A = torch.stack((torch.stack((A00, A01, A02), -1),
                     torch.stack((A01, A11, A12), -1),
                     torch.stack((A02, A12, A22), -1)), -2)
    mu, la = lame(E, nu)
    J = Fh[..., 0, 0] * Fh[..., 1, 1] - Fh[..., 0, 1] * Fh[..., 1, 0]
    if svd_grad == "reference":
        U, S, V = TaichiSvd2.apply(Fh)
        Rp = U @ V.transpose(-1, -2)
    elif svd_grad == "exact":
        Rp = polar_rotation_2x2(Fh)
    else:
        raise ValueError(svd_grad)
    P_fc = 2 * mu * (Fh - Rp) + la * ((J - 1) * J)[..., None, None] * torch.linalg.inv(Fh).transpose(-1, -2)
    pad = torch.zeros_like(F)
    pad = torch.cat((torch.cat((P_fc, torch.zeros_like(P_fc[..., :1])), -1),
                     torch.zeros_like(F[..., :1, :])), -2)
    P = Q @ pad + Q @ A @ torch.linalg.inv(R).transpose(-1, -2)
    return P


def _kinematic_override(v, node_xyz, dx, grip: Optional[KinematicGripper], f: int):
    if grip is None:
        return v
    pos = node_xyz.to(v.dtype) * dx
    for k in range(grip.centers.shape[1]):
        c = grip.centers[f, k].to(v.dtype)
        inside = ((pos - c) ** 2).sum(-1) <= grip.radius ** 2
        v = torch.where(inside[:, None], grip.velocities[f, k].to(v.dtype)[None, :].expand_as(v), v)
    return v


def grid_op(p, m, node_xyz, n_grid, bound, friction=None, grip=None, f=0, dx=None):
    """Grid update of simulation.py:274-302 on the touched nodes only.

    ``friction`` (build extension) applies Coulomb friction to the tangential
    velocity where the reference zeroes only the normal component of the
    floor (line 295-296); ``friction=0`` reproduces the reference exactly.
    """
    inv_m = 1 / (m + 1e-9)
    v = inv_m[:, None] * p
    i, j, k = node_xyz[:, 0], node_xyz[:, 1], node_xyz[:, 2]
    zero3 = torch.zeros_like(v)

    def stick(cond):
        return torch.where(cond[:, None], zero3, v)

    v = stick((i < bound) & (v[:, 0] < 0))
    v = stick((i > n_grid - bound) & (v[:, 0] > 0))
    v = stick((k < bound) & (v[:, 2] < 0))
    v = stick((k > n_grid - bound) & (v[:, 2] > 0))
    floor = (j < bound) & (v[:, 1] < 0)
    if friction is not None:
        vn = v[:, 1]
        vt2 = v[:, 0] ** 2 + v[:, 2] ** 2
        moving = floor & (vt2 > 0)
        safe_vt = torch.sqrt(torch.where(moving, vt2, torch.ones_like(vt2)))
        scale = torch.clamp(1 - friction * (-vn) / safe_vt, min=0.0)
        scale = torch.where(moving, scale, torch.ones_like(scale))
        v = torch.stack((v[:, 0] * scale, v[:, 1], v[:, 2] * scale), -1)
    v = torch.stack((v[:, 0], torch.where(floor, torch.zeros_like(v[:, 1]), v[:, 1]), v[:, 2]), -1)
    v = stick((j > n_grid - bound) & (v[:, 1] > 0))
    if grip is not None:
        v = _kinematic_override(v, node_xyz, dx, grip, f)
    return v


def keyframe_index(f: int, dt: float, interval: float, frames_per_window: int, window: int) -> int:
    """``frame`` of simulation.py:160-161, evaluated in float32 like the reference kernel."""
    t = np.float32(f) * np.float32(dt)
    return int(np.float32(t) / np.float32(interval)) + frames_per_window * window


@dataclass
class OracleSim:
    """One cloth scene: constants, topology and rest-shape inverse."""
    const: Constants
    tris: torch.Tensor                  # (Nt, 3) long
    D0inv: torch.Tensor                 # (Nt, 3, 3)
    dtype: torch.dtype = torch.float64
    svd_grad: str = "exact"

    # ---------------------------------------------------------------- init
    @staticmethod
    def initialize(const: Constants, vertices, triangles, operator_x=None, cube_x=None,
                   dtype=torch.float64, svd_grad="exact", device=None):
        """initialize_ti_field of simulation.py:447-477; returns (sim, state0).
        ``device``: where the state lives (the CPU by default)."""
        vx = torch.as_tensor(np.asarray(vertices), dtype=dtype, device=device)
        tris = torch.as_tensor(np.asarray(triangles), dtype=torch.long, device=device)
        a, b, c = vx[tris[:, 0]], vx[tris[:, 1]], vx[tris[:, 2]]
        d1 = b - a
        d2 = c - a
        n1 = d1 / _norm_eps(d1, 1e-6)
        n2 = d2 / _norm_eps(d2, 1e-6)
        d3 = torch.cross(n1, n2, dim=-1)
        d3 = d3 / _norm_eps(d3, 1e-6)
        D0 = torch.stack((d1, d2, d3), dim=-1)
        D0inv = torch.linalg.inv(D0)
        Nv, Nt = vx.shape[0], tris.shape[0]
        kw = dict(dtype=dtype, device=device)
        ox = torch.as_tensor(np.zeros((0, 3)) if operator_x is None else np.asarray(operator_x), **kw)
        cx = torch.as_tensor(np.zeros((0, 3)) if cube_x is None else np.asarray(cube_x), **kw)
        eye = torch.eye(3, **kw)
        st = dict(
            vx=vx, vv=torch.zeros_like(vx), vC=torch.zeros(Nv, 3, 3, **kw),
            qx=(a + b + c) / 3, qv=torch.zeros(Nt, 3, **kw), qC=torch.zeros(Nt, 3, 3, **kw),
            qF=eye.expand(Nt, 3, 3).clone(), qd=D0,
            ox=ox, ov=torch.zeros_like(ox), oC=torch.zeros(ox.shape[0], 3, 3, **kw),
            cx=cx, cv=torch.zeros_like(cx), cC=torch.zeros(cx.shape[0], 3, 3, **kw),
        )
        return OracleSim(const, tris, D0inv, dtype, svd_grad), st

    # ---------------------------------------------------------------- step
    def substep(self, st: Dict[str, torch.Tensor], f: int, window: int, params: Dict[str, torch.Tensor],
                seq: Optional[torch.Tensor] = None, friction=None, damping=None,
                grip: Optional[KinematicGripper] = None) -> Dict[str, torch.Tensor]:
        """forward(s, grad_update) of simulation.py:480-488:
        clear_grid, compute_inplane_F_tmp, inplane_svd, p2g, grid_op, g2p,
        update_particle_state (one substep, state f -> f+1)."""
        k = self.const
        G, dx, inv_dx, dt = k.n_grid, k.dx, k.inv_dx, k.dt
        dtype = self.dtype
        dev = st["vx"].device
        off_f = _OFF.to(dtype=dtype, device=dev)
        E, nu, ks, kc = params["E"], params["nu"], params["ks"], params["kc"]

        idx_list, mom_list, mass_list = [], [], []

        def scatter(nodes, mom, mass=None):
            idx_list.append(nodes.reshape(-1))
            mom_list.append(mom.reshape(-1, 3))
            mass_list.append(torch.zeros_like(mom[..., 0]).reshape(-1) if mass is None else mass.reshape(-1))

        # --- p2g: cube particles (simulation.py:139-152), affine momentum only
        if st["cx"].shape[0]:
            base, fx, w, W = stencil(st["cx"], inv_dx)
            dpos = (off_f[None] - fx[:, None, :]) * dx
            affine = k.cube_p_mass * st["cC"]
            scatter(stencil_nodes(base, G), W[..., None] * torch.einsum("nij,nsj->nsi", affine, dpos),
                    W * k.cube_p_mass)
        # --- p2g: operator particles (simulation.py:154-174)
        if st["ox"].shape[0]:
            base, fx, w, W = stencil(st["ox"], inv_dx)
            dpos = (off_f[None] - fx[:, None, :]) * dx
            affine = k.operator_p_mass * st["oC"]
            frame = keyframe_index(f, dt, k.operator_update_interval, k.frames_per_window, window)
            No = st["ox"].shape[0]
            gid = torch.arange(No, device=dev) // k.grasper_group_size
            if frame + 1 < k.n_actions:
                vt = (seq[frame + 1, gid] - seq[frame, gid]) / k.operator_update_interval
            else:
                vt = torch.zeros(No, 3, dtype=dtype, device=dev)
            scatter(stencil_nodes(base, G),
                    W[..., None] * (k.operator_p_mass * vt[:, None, :]
                                    + torch.einsum("nij,nsj->nsi", affine, dpos)),
                    W * k.operator_p_mass)
        # --- p2g: vertex particles (simulation.py:176-191), gravity added here
        vbase, vfx, vw, vW = stencil(st["vx"], inv_dx)
        vnodes = stencil_nodes(vbase, G)
        dpos = (off_f[None] - vfx[:, None, :]) * dx
        temp_v = st["vv"] + torch.tensor([0.0, k.gravity_dv, 0.0], dtype=dtype, device=dev)
        affine = k.vertex_p_mass * st["vC"]
        scatter(vnodes, vW[..., None] * (k.vertex_p_mass * temp_v[:, None, :]
                                         + torch.einsum("nij,nsj->nsi", affine, dpos)),
                vW * k.vertex_p_mass)
        # --- p2g: triangle (quadrature) particles (simulation.py:193-271)
        qbase, qfx, qw, qW = stencil(st["qx"], inv_dx)
        qnodes = stencil_nodes(qbase, G)
        xj = torch.stack((qfx - 1.5, 2 * (1.0 - qfx), qfx - 0.5), dim=1) * inv_dx   # (N, 3, 3)
        o = _OFF.to(dev)
        gw = torch.stack((xj[:, o[:, 0], 0] * qw[:, o[:, 1], 1] * qw[:, o[:, 2], 2],
                          qw[:, o[:, 0], 0] * xj[:, o[:, 1], 1] * qw[:, o[:, 2], 2],
                          qw[:, o[:, 0], 0] * qw[:, o[:, 1], 1] * xj[:, o[:, 2], 2]), dim=-1)  # (N,27,3)
        qdpos = (off_f[None] - qfx[:, None, :]) * dx
        qaff = st["qC"] * k.quadrature_p_mass
        P = triangle_stress(st["qF"], E, nu, ks, kc, self.svd_grad)
        d = st["qd"]
        d3 = d[..., :, 2]
        r1 = torch.stack((self.D0inv[:, 0, 0], d[:, 0, 1], d[:, 0, 2]), -1)
        r2 = torch.stack((self.D0inv[:, 1, 0], d[:, 1, 1], d[:, 1, 2]), -1)
        vol = k.quadrature_p_vol
        mom = qW[..., None] * (k.quadrature_p_mass * st["qv"][:, None, :]
                               + torch.einsum("nij,nsj->nsi", qaff, qdpos))
        normal = -vol * P[:, None, :, 2] * (gw * d3[:, None, :]).sum(-1, keepdim=True) * dt
        scatter(qnodes, mom + normal, qW * k.quadrature_p_mass)
        t1, t2, t3 = self.tris[:, 0], self.tris[:, 1], self.tris[:, 2]
        f1 = vol * (P @ (r1 + r2)[..., None])[..., 0] * dt
        f2 = -vol * (P @ r1[..., None])[..., 0] * dt
        f3 = -vol * (P @ r2[..., None])[..., 0] * dt
        scatter(vnodes[t1], vW[t1][..., None] * f1[:, None, :])
        scatter(vnodes[t2], vW[t2][..., None] * f2[:, None, :])
        scatter(vnodes[t3], vW[t3][..., None] * f3[:, None, :])

        # --- grid (only touched nodes are materialised)
        flat = torch.cat(idx_list)
        uniq, inv = torch.unique(flat, return_inverse=True)
        gp = torch.zeros(uniq.shape[0], 3, dtype=dtype, device=dev).index_add(0, inv, torch.cat(mom_list))
        gm = torch.zeros(uniq.shape[0], dtype=dtype, device=dev).index_add(0, inv, torch.cat(mass_list))
        node_xyz = torch.stack((uniq // (G * G), (uniq // G) % G, uniq % G), -1)
        gv = grid_op(gp, gm, node_xyz, G, k.bound, friction=friction, grip=grip, f=f, dx=dx)
        lookup = {}
        pos = 0
        # position of each particle species' stencil inside ``inv``
        sizes = [t.numel() for t in idx_list]
        starts = np.cumsum([0] + sizes)

        def gathered(nodes):
            # map flat node ids to rows of gv via searchsorted on the sorted unique ids
            rows = torch.searchsorted(uniq, nodes.reshape(-1)).reshape(nodes.shape)
            return gv[rows]

        new = {}

        def g2p_point(x, nodes):
            """g2p for cube / operator / vertex particles (simulation.py:307-365)."""
            base, fx, w, W = stencil(x, inv_dx)
            dposc = off_f[None] - fx[:, None, :]
            g = gathered(nodes)
            v_new = (W[..., None] * g).sum(1)
            C_new = 4 * inv_dx * torch.einsum("ns,nsi,nsj->nij", W, g, dposc)
            return x + dt * v_new, v_new, C_new

        if st["cx"].shape[0]:
            new["cx"], new["cv"], new["cC"] = g2p_point(st["cx"], stencil_nodes(stencil(st["cx"], inv_dx)[0], G))
        else:
            new["cx"], new["cv"], new["cC"] = st["cx"], st["cv"], st["cC"]
        if st["ox"].shape[0]:
            new["ox"], new["ov"], new["oC"] = g2p_point(st["ox"], stencil_nodes(stencil(st["ox"], inv_dx)[0], G))
        else:
            new["ox"], new["ov"], new["oC"] = st["ox"], st["ov"], st["oC"]
        new["vx"], new["vv"], new["vC"] = g2p_point(st["vx"], vnodes)
        # triangles: C only, then 95 % of the symmetric part removed (simulation.py:367-383)
        g = gathered(qnodes)
        Ct = 4 * inv_dx * torch.einsum("ns,nsi,nsj->nij", qW, g, off_f[None] - qfx[:, None, :])
        damp = 0.95 if damping is None else damping
        skew = 0.5 * (Ct - Ct.transpose(-1, -2))
        sym = 0.5 * (Ct + Ct.transpose(-1, -2))
        qC_new = skew + (1 - damp) * sym
        # --- update_particle_state (simulation.py:386-430); the return mapping
        # (lines 406-428) only writes a local and has no effect.
        vxn, vvn = new["vx"], new["vv"]
        new["qv"] = (1 / 3) * (vvn[t1] + vvn[t2] + vvn[t3])
        new["qx"] = (1 / 3) * (vxn[t1] + vxn[t2] + vxn[t3])
        c1 = vxn[t2] - vxn[t1]
        c2 = vxn[t3] - vxn[t1]
        c3 = d3 + ((dt * qC_new + 0.5 * dt * dt * qC_new @ qC_new) @ d3[..., None])[..., 0]
        new_d = torch.stack((c1, c2, c3), dim=-1)
        new_F = new_d @ self.D0inv
        new["qd"] = new_F @ torch.linalg.inv(self.D0inv)
        new["qF"] = new_F
        new["qC"] = qC_new
        return new


    # ---------------------------------------------------------------- replay
    def reset_quadrature_particles(self, st: Dict[str, torch.Tensor]) -> Dict[str, torch.Tensor]:
        """reset_quadrature_particles of simulation_without_grad.py:471-485:
        triangle centroid, d = [e1, e2, n] of the current vertices (n from the
        eps-normalised edges, norm(1e-6)) and a new rest-shape inverse; the
        stored F (qF) is left as it is."""
        vx = st["vx"]
        a, b, c = vx[self.tris[:, 0]], vx[self.tris[:, 1]], vx[self.tris[:, 2]]
        d1 = b - a
        d2 = c - a
        n1 = d1 / _norm_eps(d1, 1e-6)
        n2 = d2 / _norm_eps(d2, 1e-6)
        d3 = torch.cross(n1, n2, dim=-1)
        d3 = d3 / _norm_eps(d3, 1e-6)
        D = torch.stack((d1, d2, d3), dim=-1)
        self.D0inv = torch.linalg.inv(D)
        new = dict(st)
        new["qx"] = (a + b + c) / 3
        new["qd"] = D
        return new


def replay(sim: OracleSim, st, n_counts: int, block: int, params, seq=None, first_step: int = 0,
           friction=None, damping=None, grip=None, on_count=None):
    """The substep loop of animation() (simulation_without_grad.py:487-511):
    ``n_counts`` times, ``block`` forward substeps (window 0) and a
    reset_quadrature_particles; ``on_count(count, state)`` sees the state after
    each reset.  Returns the final state."""
    f = first_step
    for count in range(n_counts):
        for _ in range(block):
            st = sim.substep(st, f, 0, params, seq=seq, friction=friction, damping=damping, grip=grip)
            f += 1
        st = sim.reset_quadrature_particles(st)
        if on_count is not None:
            on_count(count, st)
    return st


def compute_loss(vx: torch.Tensor, targets: torch.Tensor):
    """compute_loss of parameter_fitting_functions.py:3-15: one-sided Chamfer
    ``(1/Nq) sum_q min_p |x_p - t_q|^2 / 3``; ties go to the first vertex."""
    dist = ((vx[:, None, :] - targets[None, :, :]) ** 2)
    dist = (dist[..., 0] + dist[..., 1] + dist[..., 2]) / 3
    mins, arg = torch.min(dist, dim=0)
    return mins.sum() / targets.shape[0], arg


def rollout(sim: OracleSim, st0, n_steps: int, params, seq=None, window=0, friction=None, damping=None,
            grip=None, keep_states=False):
    """Run ``n_steps`` substeps (f = 0 .. n_steps-1) from ``st0``; returns the
    list of states (index = substep) if ``keep_states`` else the final state."""
    st = st0
    states = [st0] if keep_states else None
    for f in range(n_steps):
        st = sim.substep(st, f, window, params, seq=seq, friction=friction, damping=damping, grip=grip)
        if keep_states:
            states.append(st)
    return states if keep_states else st
