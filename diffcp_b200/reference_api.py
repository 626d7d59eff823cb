"""Drop-in replacement for the simulation path of the reference's scripts.

The reference's scripts reach the simulation with
``from src.parameter_fitting_functions import *`` (or ``src.simulation``) and
then use module-level names: ``initialize_objects``, ``forward``,
``backward``, ``compute_loss``, ``compute_grad``, ``clear_distances``, the
Taichi fields ``garment_E``, ``garment_nu``, ``contact_stiffness``,
``shearing_stiffness`` (``[None]``, ``.grad[None]``), ``loss``, the
per-substep particle fields ``vertex_x``/``operator_x``/``cube_x``,
``target_pos``, ``initial_*_x``, ``lagrangian_mesh_element``,
``grasp_tracking_seq`` and the Tape ``ti.ad.Tape(loss=loss)``
(src/simulation.py, src/parameter_fitting_functions.py,
src/taichi_variable_definition.py).  This module provides the same names with
the same meaning, computed by the CUDA kernels of ``libdiffcp_b200.so``:

    import diffcp_b200.reference_api as ref
    ref.configure("/path/to/src", seed=0)     # reads simulation_arguments.json + data
    from diffcp_b200.reference_api import *

Every substep's state is kept on the device, as the reference keeps its
time-indexed fields; ``vertex_x.to_numpy()`` returns the whole history.
Gradients: ``svd_grad="reference"`` reproduces the reference's clamped SVD
backward, ``"exact"`` (default) the exact derivative of the rotation factor.
"""
from __future__ import annotations

import types
from typing import List, Optional

import numpy as np
import torch

from . import scene as _scene
from .batch import ClothBatch

__all__ = ["configure", "initialize_objects", "initialize_ti_field", "clear_distances", "forward", "backward",
           "compute_loss", "compute_grad", "Tape", "ti"]

_st = None  # the configured simulation (module singleton, like the reference's Taichi fields)


class _Grad:
    def __init__(self, arr, idx):
        self._arr, self._idx = arr, idx

    def __getitem__(self, key):
        # gradients accumulate in float64; reads see the float32 of the reference's f32 .grad field
        return float(np.float32(self._arr[self._idx]))

    def __setitem__(self, key, value):
        self._arr[self._idx] = float(value)


class _ParamField:
    """0-D Taichi field stand-in over one entry of the device parameter table."""

    def __init__(self, col):
        self._col = col
        self.grad = _Grad(_st.grad_params, col)

    def __getitem__(self, key):
        return float(_st.batch.params[0, self._col].item())

    def __setitem__(self, key, value):
        _st.batch.params[0, self._col] = float(value)


class _Scalar:
    """Host-resident 0-D f32 field (the reference's learning_rate0..3,
    taichi_variable_definition.py:10-14): stores float32, reads Python floats."""

    def __init__(self, value=0.0):
        self._v = np.float32(value)

    def __getitem__(self, key):
        return float(self._v)

    def __setitem__(self, key, value):
        self._v = np.float32(value)


class _LossField:
    def __init__(self):
        self.value = 0.0
        self.grad = _Grad(np.ones(1), 0)

    def __getitem__(self, key):
        return float(self.value)

    def __setitem__(self, key, value):
        self.value = float(value)


class _HostField:
    """Vector field kept on the host (rest positions, mesh, targets)."""

    def __init__(self, arr, on_write=None):
        self.arr = np.array(arr)
        self._on_write = on_write

    @property
    def shape(self):
        return self.arr.shape[:-1]

    def from_numpy(self, a):
        a = np.asarray(a)
        if a.shape != self.arr.shape:
            raise ValueError("shape %s does not match field shape %s" % (a.shape, self.arr.shape))
        self.arr = a.astype(self.arr.dtype).copy()
        if self._on_write:
            self._on_write(self.arr)

    def to_numpy(self):
        return self.arr.copy()

    def __getitem__(self, key):
        return self.arr[key]


class _HistoryField:
    """Time-indexed particle field ``[max_steps, N, k]`` read from the device
    history (absolute positions, original particle order)."""

    def __init__(self, species, comp):
        self._species, self._comp = species, comp

    def _step(self, f):
        fields = _st.batch.absolute_fields(_st.history[f])
        key = {"vertex": "v", "operator": "o", "cube": "c"}[self._species] + self._comp
        a = fields[key].t().cpu().numpy()
        if self._species == "vertex":
            out = np.empty_like(a)
            out[_st.batch.vperm[0]] = a
            a = out
        if self._comp == "C":
            a = a.reshape(-1, 3, 3)
        return a

    def to_numpy(self):
        return np.stack([self._step(f) for f in range(_st.history.shape[0])])

    def __getitem__(self, key):
        if isinstance(key, tuple):
            return self._step(int(key[0]))[key[1:]]
        return self._step(int(key))


class _TrajRow:
    def __init__(self, j):
        self._j = j

    def __getitem__(self, k):
        return _traj_view()[self._j, k].cpu().numpy().astype(np.float64)

    def __setitem__(self, k, value):
        v = _traj_view()
        v[self._j, k] = torch.as_tensor(np.asarray(value, dtype=np.float32), device=v.device)


class _TrajField:
    """grasp_tracking_seq: keyframes [n_actions, n_grippers, 3] on the device."""

    def __init__(self):
        self.grad = None

    @property
    def shape(self):
        return tuple(_traj_view().shape[:2])

    def from_numpy(self, a):
        v = _traj_view()
        v.copy_(torch.as_tensor(np.asarray(a, dtype=np.float32).reshape(v.shape), device=v.device))

    def to_numpy(self):
        return _traj_view().cpu().numpy().astype(np.float64)

    def __getitem__(self, j):
        return _TrajRow(j)


def _traj_view():
    sc = _st.scene
    return _st.batch.traj[: sc.keyframes.size].view(*sc.keyframes.shape)


class _Mesh:
    def __init__(self, v, t):
        self.vertices, self.triangles = v, t


class _State:
    pass


# ----------------------------------------------------------------- set-up
def configure(src_dir: Optional[str] = None, seed: Optional[int] = 0, seed_cube: Optional[int] = None,
              scene: Optional[_scene.ClothScene] = None, args: Optional[dict] = None, svd_grad: str = "exact",
              device=None, chunk: int = 128):
    """Build the simulation of a reference configuration (``src_dir`` holding
    ``simulation_arguments.json``; or a ready :class:`ClothScene`) and bind the
    module-level names.  Returns the module's globals for convenience."""
    global _st
    sc = scene if scene is not None else _scene.load_reference_scene(src_dir, seed=seed, args=args,
                                                                      seed_cube=seed_cube)
    st = _State()
    st.scene = sc
    st.dt = float(sc.meta["dt"])
    st.batch = ClothBatch([sc], dt=st.dt, chunk=chunk, svd_grad=svd_grad, device=device)
    st.max_steps = int(sc.meta["max_steps"])
    st.history = torch.zeros(st.max_steps, st.batch.S, dtype=torch.float32, device=st.batch.device)
    st.adj = torch.zeros(2, st.batch.S, dtype=torch.float32, device=st.batch.device)
    st.grad_params = np.zeros(8)
    st.tape = None
    st.loss_state = None
    _st = st
    g = globals()
    targets = np.asarray(sc.meta.get("targets_by_window", sc.targets[None]))
    g.update(
        max_steps=st.max_steps, dt=st.dt, n_grid=sc.n_grid, dx=1.0 / sc.n_grid, inv_dx=float(sc.n_grid),
        bound=sc.bound, n_vertex_particles=sc.n_vertex, n_quadrature_particles=sc.n_tri,
        n_operator_particles=len(sc.operator_x), n_cube_particles=len(sc.cube_x), grasp_point_num=sc.n_grippers,
        grasper_group_size=sc.group_size, n_actions=sc.keyframes.shape[0], n_grad_updates=targets.shape[0],
        n_target_particles=targets.shape[1], target_pcd_array=targets, grasp_point_pos=sc.keyframes.copy(),
        soft_body_model_vertices=sc.vertices.copy(), soft_body_model_triangles=np.asarray(sc.triangles).copy(),
        cube_model=np.asarray(sc.cube_x).copy(), operator_model_without_position=sc.meta["operator_model"],
        operator_update_interval=sc.keyframe_interval, vertex_p_mass=sc.vertex_p_mass,
        quadrature_p_mass=sc.quadrature_p_mass, quadrature_p_vol=sc.quadrature_p_vol,
        operator_p_mass=sc.operator_p_mass, cube_p_mass=sc.cube_p_mass,
        soft_body_mesh=_Mesh(sc.vertices.copy(), np.asarray(sc.triangles).copy()),
        garment_E=_ParamField(0), garment_nu=_ParamField(1), shearing_stiffness=_ParamField(2),
        contact_stiffness=_ParamField(3), loss=_LossField(), grasp_tracking_seq=_TrajField(),
        initial_vertex_x=_HostField(sc.vertices), initial_operator_x=_HostField(sc.operator_x),
        initial_cube_x=_HostField(sc.cube_x), lagrangian_mesh_element=_HostField(np.asarray(sc.triangles)),
        target_pos=_HostField(targets[0], on_write=_upload_targets),
        vertex_x=_HistoryField("vertex", "x"), vertex_v=_HistoryField("vertex", "v"),
        vertex_C=_HistoryField("vertex", "C"), operator_x=_HistoryField("operator", "x"),
        operator_v=_HistoryField("operator", "v"), cube_x=_HistoryField("cube", "x"),
        cube_v=_HistoryField("cube", "v"),
        learning_rate0=_Scalar(), learning_rate1=_Scalar(), learning_rate2=_Scalar(), learning_rate3=_Scalar(),
    )
    bounds = sc.meta.get("bounds", {})
    for name in ("E", "nu", "contact_stiffness", "shearing_stiffness"):
        if name in bounds:
            g[name + "_lower_bound"], g[name + "_upper_bound"] = bounds[name]
    for name, key in (("initial_garment_E", "E"), ("initial_garment_nu", "nu"),
                      ("initial_contact_stiffness", "contact_stiffness"),
                      ("initial_shearing_stiffness", "shearing_stiffness")):
        g[name] = sc.params[key]
    if src_dir is not None:
        g["result_file_path"] = src_dir + sc.meta.get("result_dir", "/../result/") + "/fit_parameter.json"
    for name in ("garment_E", "garment_nu", "shearing_stiffness", "contact_stiffness", "loss", "grasp_tracking_seq",
                 "initial_vertex_x", "initial_operator_x", "initial_cube_x", "lagrangian_mesh_element",
                 "target_pos", "vertex_x", "vertex_v", "vertex_C", "operator_x", "operator_v", "cube_x",
                 "cube_v", "max_steps", "n_grad_updates", "target_pcd_array", "grasp_point_pos",
                 "soft_body_model_vertices", "soft_body_mesh", "n_actions", "dt", "learning_rate0",
                 "learning_rate1", "learning_rate2", "learning_rate3"):
        if name not in __all__:
            __all__.append(name)
    _upload_targets(targets[0])
    initialize_objects()
    return g


def _upload_targets(arr):
    b = _st.batch
    b.targets.copy_(torch.as_tensor(np.asarray(arr, dtype=np.float32).T.copy(), device=b.device))


# ------------------------------------------------------------ simulation
def initialize_objects():
    """simulation.py:432-442: keyframes, operator cloud around the first grasp
    points, rest vertices, cube; then initialize_ti_field."""
    g = globals()
    grasp = np.asarray(g["grasp_point_pos"])
    g["grasp_tracking_seq"].from_numpy(grasp)
    opm = np.asarray(g["operator_model_without_position"])
    g["initial_operator_x"].from_numpy(np.concatenate([opm + grasp[0][k] for k in range(grasp.shape[1])]))
    g["initial_vertex_x"].from_numpy(g["soft_body_model_vertices"])
    g["lagrangian_mesh_element"].from_numpy(g["soft_body_model_triangles"])
    g["initial_cube_x"].from_numpy(g["cube_model"])
    initialize_ti_field()


def initialize_ti_field():
    """simulation.py:447-477: state 0 and rest shape from the initial_* fields."""
    g = globals()
    b = _st.batch
    if not np.array_equal(g["lagrangian_mesh_element"].arr, np.asarray(_st.scene.triangles)):
        raise NotImplementedError("changing the mesh topology needs a new configure()")
    xv = np.asarray(g["initial_vertex_x"].arr)[b.vperm[0]]
    b.x0_vertex.copy_(torch.as_tensor(xv.T.astype(np.float32).copy(), device=b.device))
    if b.no:
        b.x0_operator.copy_(torch.as_tensor(np.asarray(g["initial_operator_x"].arr).T.astype(np.float32).copy(),
                                            device=b.device))
    if b.nc:
        b.x0_cube.copy_(torch.as_tensor(np.asarray(g["initial_cube_x"].arr).T.astype(np.float32).copy(),
                                        device=b.device))
    b.init_state(out=_st.history[0])


def clear_distances():
    """simulation.py:3-7; the Chamfer kernels keep no distance matrix."""


def forward(s: int, grad_update: int = 0):
    """One substep s -> s+1 (simulation.py:480-488)."""
    b = _st.batch
    b.forward_step(_st.history[s], int(s), int(grad_update), out=_st.history[s + 1])
    if _st.tape is not None:
        _st.tape.steps.append((int(s), int(grad_update)))


def backward(s: int, grad_update: int = 0):
    """Reverse of substep s (simulation.py:490-506): dL/d state(s+1), held by
    the running Tape, becomes dL/d state(s); parameter and keyframe gradients
    accumulate."""
    t = _st.tape
    if t is None:
        raise RuntimeError("backward() runs inside a Tape")
    b = _st.batch
    a_out = _st.adj[t.slot]
    a_in = _st.adj[1 - t.slot]
    b.backward_step(_st.history[s], a_out, int(s), t.gp, t.gt, window=int(grad_update), out=a_in)
    t.slot = 1 - t.slot


def compute_loss(f: int):
    """parameter_fitting_functions.py:3-15: Chamfer loss of vertex_x[f - 1]
    against target_pos, added to loss[None]."""
    state = f - 1
    lv, arg = _st.batch.chamfer(_st.history[state])
    g = globals()
    g["loss"].value += float(lv[0].item())
    _st.loss_state = (state, arg)
    if _st.tape is not None:
        _st.tape.loss_state = (state, arg)


class Tape:
    """``ti.ad.Tape(loss=loss)``: records forward() calls; on exit seeds
    dL/dloss = 1 and runs the recorded substeps' adjoints in reverse order,
    accumulating garment_E.grad, ..., grasp_tracking_seq.grad."""

    def __init__(self, loss=None, clear_gradients: bool = True):
        self.clear = clear_gradients
        self.steps: List[tuple] = []
        self.loss_state = None

    def __enter__(self):
        if self.clear:
            _st.grad_params[:] = 0.0
        self.gp, self.gt = _st.batch.new_grads()
        _st.tape = self
        return self

    def __exit__(self, exc_type, exc, tb):
        _st.tape = None
        if exc_type is not None:
            return False
        b = _st.batch
        g = globals()
        if self.loss_state is None:
            return False
        L, arg = self.loss_state
        _st.adj.zero_()
        gl = torch.full((1,), float(g["loss"].grad[None]), device=b.device)
        b.chamfer_backward(_st.history[L], arg, gl, _st.adj[0])
        self.slot = 0
        _st.tape = self
        for s, w in reversed(self.steps):
            if s < L:   # substeps at or after the loss state do not reach the loss
                backward(s, w)
        _st.tape = None
        gp = self.gp[0].cpu().numpy()
        _st.grad_params[:6] += gp[:6]
        sc = _st.scene
        g["grasp_tracking_seq"].grad = self.gt[: sc.keyframes.size].cpu().numpy().reshape(sc.keyframes.shape)
        return False


ti = types.SimpleNamespace(ad=types.SimpleNamespace(Tape=Tape))


def compute_grad():
    """parameter_fitting_functions.py:17-58: for every grasp window, a Tape
    over max_steps - 1 substeps and the Chamfer loss, then the window's end
    state becomes the next window's rest state.  Returns (mean loss, mean
    [dE, dnu, d contact, d shearing]) with NaN mapped to 0."""
    g = globals()
    losses, gE, gnu, gkc, gks = [], [], [], [], []
    for w in range(g["n_grad_updates"]):
        clear_distances()
        g["target_pos"].from_numpy(g["target_pcd_array"][w])
        with Tape(loss=g["loss"]):
            g["loss"][None] = 0
            for f in range(g["max_steps"] - 1):
                forward(f, w)
            compute_loss(f)
        gE.append(g["garment_E"].grad[None])
        gnu.append(g["garment_nu"].grad[None])
        gkc.append(g["contact_stiffness"].grad[None])
        gks.append(g["shearing_stiffness"].grad[None])
        losses.append(g["loss"][None])
        last = g["max_steps"] - 1
        g["initial_operator_x"].from_numpy(g["operator_x"][last])
        g["initial_vertex_x"].from_numpy(g["vertex_x"][last])
        g["initial_cube_x"].from_numpy(g["cube_x"][last])
        initialize_ti_field()
    n = g["n_grad_updates"]
    grads = [float(np.mean(np.nan_to_num(x))) for x in (gE, gnu, gkc, gks)]
    return sum(losses) / n, grads
