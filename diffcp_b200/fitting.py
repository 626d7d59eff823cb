"""Material-parameter fitting.

The reference's driver (parameter_fitting_functions.py:17-205,
parameter_fitting_main.py:1-23) estimates the garment's Young's modulus,
Poisson ratio and contact/shearing stiffness of one cloth by running the
windowed gradient (``compute_grad``) once per epoch and moving each parameter
with a step-size heuristic that rescales the learning rate to the decimal
magnitude of the distance left to the bound it heads for.  This module gives

* :func:`magnitude_level`, :func:`single_parameter_fitting` -- the heuristic;
* :func:`parameters_learning` -- the epoch loop over a drop-in namespace
  (:mod:`diffcp_b200.reference_api` by default), with the reference's
  bookkeeping of the best epoch;
* :class:`BatchFitter` -- the same loop for every cloth of a
  :class:`~diffcp_b200.batch.ClothBatch` at once: one batched windowed
  forward + adjoint per epoch on the GPU, then the heuristic per cloth;
* :func:`write_result` and :func:`main` -- the JSON result of
  parameter_fitting_main.py, runnable as ``python -m diffcp_b200.fitting``.

Parameters and learning rates live in float32, as the reference keeps them
in 0-D f32 Taichi fields (taichi_variable_definition.py:5-14) and reads them
back as Python floats.
"""
from __future__ import annotations

import argparse
import json
import math
import os
from typing import Callable, Dict, List, Optional, Sequence, Tuple

import numpy as np

#: order of the gradient list of compute_grad (parameter_fitting_functions.py:54-57)
NAMES = ("E", "nu", "contact_stiffness", "shearing_stiffness")
FIELDS = ("garment_E", "garment_nu", "contact_stiffness", "shearing_stiffness")
#: column of each name in the device parameter table (E, nu, shearing, contact, friction, damping)
PARAM_COL = {"E": 0, "nu": 1, "shearing_stiffness": 2, "contact_stiffness": 3}


def magnitude_level(a: float) -> int:
    """Decimal exponent floor(log10|a|) of ``a`` (1e-19 added before the
    absolute value, parameter_fitting_functions.py:60-63)."""
    return math.floor(math.log10(abs(a + 1e-19)))


def single_parameter_fitting(parameter: float, parameter_grad: float, grad_shock: int, lower_bound: float,
                             upper_bound: float, lr: float, epochs: int, epoch_index: int) -> Tuple[float, float]:
    """One update of one parameter (parameter_fitting_functions.py:65-92).
    Returns (new parameter, new learning rate).

    A zero or NaN gradient leaves both unchanged.  Otherwise the learning rate
    is rescaled so that the step has the magnitude of (bound - parameter) per
    remaining epoch, the bound being the one the step moves toward (in the
    first epoch before stepping as well).  A step that would leave the open
    interval is rescaled toward the opposite bound's magnitude and then halved
    until it lands inside.  ``grad_shock`` is accepted and unused, as in the
    reference.  Where the reference would halve forever (the parameter itself
    outside its bounds) this raises ValueError.
    """
    del grad_shock
    if not abs(parameter_grad) > 0:
        return parameter, lr
    period = epochs - epoch_index
    delta = lr * parameter_grad
    heading = upper_bound if parameter_grad < 0 else lower_bound
    level = magnitude_level((heading - parameter) / period)
    if epoch_index < 1:
        lr *= pow(10, level - magnitude_level(delta))
        delta = lr * parameter_grad
    trial = parameter - delta
    if lower_bound < trial < upper_bound:
        return trial, lr * pow(10, level - magnitude_level(delta))
    if trial < lower_bound:
        level = magnitude_level((upper_bound - parameter) / period)
    if trial > upper_bound:
        level = magnitude_level((lower_bound - parameter) / period)
    lr *= pow(10, level - magnitude_level(delta))
    trial = parameter - lr * parameter_grad
    while trial > upper_bound or trial < lower_bound:
        if lr == 0.0:
            raise ValueError("parameter %r lies outside its bounds [%r, %r]" % (parameter, lower_bound, upper_bound))
        lr *= 0.5
        trial = parameter - lr * parameter_grad
    return trial, lr


def _f32(x: float) -> float:
    return float(np.float32(x))


def parameters_learning(elasticity_parameter_learning: bool, contact_parameter_learning: bool, epoch: int,
                        sim=None, log: Optional[Callable[[str], None]] = None) -> Dict[str, object]:
    """The epoch loop of parameter_fitting_functions.py:94-205 over ``sim``, a
    namespace exposing the reference's names (``garment_E``, ``garment_nu``,
    ``contact_stiffness``, ``shearing_stiffness`` with ``[None]`` and
    ``.grad[None]``, ``loss``, ``learning_rate0..3``, the ``*_lower_bound`` /
    ``*_upper_bound`` constants, ``initialize_objects`` and
    ``compute_grad``); :mod:`diffcp_b200.reference_api` by default.

    Each epoch: re-initialise, run compute_grad, remember the parameters when
    the loss is not above the best so far or when it is epoch 1 (the
    reference's rule), stop when the E gradient is NaN, then update the
    elasticity pair (E, nu) and/or the contact pair (contact, shearing).
    Finally the best parameters and loss are written back.  The reference's
    previous-gradient variables stay 0, so its "grad shock" flags are always 0
    and unused; that is kept.  Returns {"E", "nu", "contact_stiffness",
    "shearing_stiffness", "loss", "epochs_run", "history"}.
    """
    if sim is None:
        from . import reference_api as sim
    say = log or (lambda *_: None)
    lrs = [getattr(sim, "learning_rate%d" % k) for k in range(4)]
    for f in lrs:
        f[None] = 1
    fields = [getattr(sim, n) for n in FIELDS]
    bounds = [(getattr(sim, n + "_lower_bound"), getattr(sim, n + "_upper_bound")) for n in NAMES]
    min_loss = 1e9
    best = None
    history: List[dict] = []
    epochs_run = 0
    for i in range(epoch):
        say("epoch: %d  E = %r  nu = %r  contact_stiffness = %r  shearing_stiffness = %r"
            % (i, fields[0][None], fields[1][None], fields[2][None], fields[3][None]))
        sim.initialize_objects()
        l, grads = sim.compute_grad()
        epochs_run = i + 1
        history.append({"epoch": i, "loss": l, "grads": list(grads),
                        "params": [f[None] for f in fields], "lr": [f[None] for f in lrs]})
        say(">>> loss = %r" % (l,))
        if min_loss >= l or i == 1:
            min_loss = l
            best = [f[None] for f in fields]
        if not abs(sim.garment_E.grad[None]) >= 0:
            say("Gradients disappear!")
            break
        pairs = []
        if elasticity_parameter_learning:
            pairs += [0, 1]
        if contact_parameter_learning:
            pairs += [2, 3]
        for j in pairs:
            p, lr = single_parameter_fitting(fields[j][None], grads[j], 0, bounds[j][0], bounds[j][1], lrs[j][None],
                                             epoch, i)
            fields[j][None] = p
            lrs[j][None] = lr
        if not abs(sim.loss[None]) > 0:
            say("loss is NaN!")
    if best is None:
        raise RuntimeError("no epoch produced a loss to keep (the reference fails here on an unset best value)")
    for f, v in zip(fields, best):
        f[None] = v
    sim.loss[None] = min_loss
    out = {n: fields[j][None] for j, n in enumerate(NAMES)}
    out.update(loss=sim.loss[None], epochs_run=epochs_run, history=history)
    return out


def write_result(path: str, values: Dict[str, float], create_missing: bool = False) -> dict:
    """parameter_fitting_main.py:16-23: merge E, nu, contact_stiffness and
    shearing_stiffness into the JSON file at ``path`` (indent 1).  The
    reference reads the file before writing it and fails when it does not
    exist; ``create_missing`` starts from an empty object instead."""
    if os.path.exists(path) or not create_missing:
        with open(path) as fh:
            result = json.load(fh)
    else:
        result = {}
    for n in NAMES:
        result[n] = values[n]
    with open(path, "w") as fh:
        json.dump(result, fh, indent=1)
    return result


class BatchFitter:
    """:func:`parameters_learning` for every cloth of a batch at once.

    Per epoch one batched ``compute_grad``: for each grasp window, the
    forward rollout and its Chamfer loss and adjoint of all cloths together
    (a :class:`~diffcp_b200.batch.BatchSim` call), after which each cloth's
    end state becomes its next window's rest state (the reference's carry-over,
    parameter_fitting_functions.py:40-49).  Window losses and gradients are
    averaged per cloth with NaN mapped to 0.  Then, on the host, each cloth
    runs the step-size heuristic on its own float32 parameters and learning
    rates and keeps its own best epoch.  A cloth whose E gradient is NaN
    stops updating (the reference's loop ends there) while the others go on.

    ``windows``: per window, the packed [3][Nq] target tensor of all cloths
    (same per-cloth target counts as the batch); None uses the batch's targets
    as one window.  ``bounds``: name -> (lower, upper), shared by all cloths,
    or name -> ((n,), (n,)) arrays.
    """

    def __init__(self, sim, bounds: Dict[str, Tuple], windows: Optional[Sequence] = None,
                 learn_elasticity: bool = True, learn_contact: bool = True):
        self.sim = sim
        self.batch = sim.batch
        n = self.batch.n_inst
        self.lower = np.array([np.broadcast_to(np.asarray(bounds[k][0], dtype=np.float64), (n,)) for k in NAMES])
        self.upper = np.array([np.broadcast_to(np.asarray(bounds[k][1], dtype=np.float64), (n,)) for k in NAMES])
        self.windows = list(windows) if windows is not None else [self.batch.targets.clone()]
        self.learn = [learn_elasticity, learn_elasticity, learn_contact, learn_contact]
        self._rest0 = self.batch.save_rest()

    def params(self) -> np.ndarray:
        """(4, n) current values in NAMES order (float32 values as float64)."""
        p = self.batch.params.detach().cpu().numpy().astype(np.float64)
        return np.array([p[:, PARAM_COL[k]] for k in NAMES])

    def _set_params(self, vals: np.ndarray) -> None:
        import torch
        p = self.batch.params
        for j, k in enumerate(NAMES):
            p[:, PARAM_COL[k]] = torch.as_tensor(vals[j], dtype=p.dtype, device=p.device)

    def compute_grad(self) -> Tuple[np.ndarray, np.ndarray]:
        """Per cloth (mean window loss, (4, n) mean gradients in NAMES order)."""
        b = self.batch
        losses, grads = [], []
        traj = b.traj
        for w, tgt in enumerate(self.windows):
            b.targets.copy_(tgt)
            params = b.params.clone().requires_grad_(True)
            loss = self.sim.loss(params, traj, window=w)
            loss.sum().backward()
            g = params.grad.detach().cpu().numpy().astype(np.float32).astype(np.float64)
            losses.append(loss.detach().cpu().numpy().astype(np.float64))
            grads.append(np.array([g[:, PARAM_COL[k]] for k in NAMES]))
            b.rebase_rest(self.sim.final_state)
        self.last_grad_E = grads[-1][0]     # the .grad field read by the NaN check holds the last window's
        nw = len(self.windows)
        return sum(losses) / nw, np.mean(np.nan_to_num(np.array(grads)), axis=0)

    def run(self, epochs: int, log: Optional[Callable[[str], None]] = None) -> Dict[str, np.ndarray]:
        """Fit for ``epochs`` epochs; the batch's parameters end at each
        cloth's best epoch.  Returns :func:`fit_many`'s result."""
        b = self.batch

        def grad_at(vals):
            b.restore_rest(self._rest0)          # initialize_objects
            self._set_params(vals)
            loss, g = self.compute_grad()
            return loss, g, self.last_grad_E

        learn = np.array(self.learn)[:, None].repeat(b.n_inst, 1)
        res = fit_many(self.params(), self.lower, self.upper, grad_at, epochs, learn, log=log)
        self._set_params(res["params"])
        b.restore_rest(self._rest0)
        return res


def fit_many(params0: np.ndarray, lower: np.ndarray, upper: np.ndarray,
             compute_grad: Callable[[np.ndarray], Tuple[np.ndarray, np.ndarray, np.ndarray]], epochs: int,
             learn: np.ndarray, log: Optional[Callable[[str], None]] = None) -> Dict[str, np.ndarray]:
    """:func:`parameters_learning` for n independent problems in lockstep.

    params0, lower, upper, learn: (4, n) in NAMES order.  ``compute_grad(p)``
    takes the (4, n) float32-valued parameters and returns the per-problem
    mean loss (n,), mean gradients (4, n) and the raw last-window E gradient
    (n,) that the NaN check reads.  A problem whose E gradient is NaN stops
    (no later update or best-epoch change), like the reference's loop.
    Returns {"params": best (4, n), "loss": best loss (n,), "best_set": (n,)
    whether an epoch qualified, "epochs_run": (n,), "history": per epoch
    {"loss", "params", "lr", "active"}}.
    """
    say = log or (lambda *_: None)
    n = params0.shape[1]
    cur = np.asarray(params0, dtype=np.float32).astype(np.float64)
    lr = np.ones((4, n), dtype=np.float32)
    min_loss = np.full(n, 1e9)
    best = np.full((4, n), np.nan)
    best_set = np.zeros(n, dtype=bool)
    active = np.ones(n, dtype=bool)
    epochs_run = np.zeros(n, dtype=np.int64)
    history = []
    for i in range(epochs):
        loss, g, g_e = compute_grad(cur.copy())
        loss = np.asarray(loss, dtype=np.float64)
        history.append({"loss": loss.copy(), "params": cur.copy(), "lr": lr.astype(np.float64), "active": active.copy()})
        epochs_run[active] += 1
        keep = active & ((min_loss >= loss) | (i == 1))
        min_loss[keep] = loss[keep]
        best[:, keep] = cur[:, keep]
        best_set |= keep
        active &= np.abs(np.asarray(g_e)) >= 0
        fin = loss[np.isfinite(loss)]
        say("epoch %d: mean loss %.6g, %d problems updating"
            % (i, float(fin.mean()) if fin.size else math.nan, int(active.sum())))
        for c in np.nonzero(active)[0]:
            for j in range(4):
                if learn[j, c]:
                    p, r = single_parameter_fitting(float(cur[j, c]), float(g[j, c]), 0, float(lower[j, c]),
                                                    float(upper[j, c]), float(lr[j, c]), epochs, i)
                    cur[j, c] = _f32(p)
                    lr[j, c] = np.float32(r)
        if not active.any():
            break
    best[:, ~best_set] = cur[:, ~best_set]
    return {"params": best, "loss": min_loss, "best_set": best_set, "epochs_run": epochs_run, "history": history}


def main(argv: Optional[Sequence[str]] = None) -> dict:
    """parameter_fitting_main.py: fit a reference configuration and write the
    result JSON.  ``--src`` is the directory holding
    simulation_arguments.json."""
    ap = argparse.ArgumentParser(prog="python -m diffcp_b200.fitting")
    ap.add_argument("--src", required=True)
    ap.add_argument("--epochs", type=int, default=35)
    ap.add_argument("--seed", type=int, default=0, help="seed of the operator and cube clouds")
    ap.add_argument("--result", default=None, help="result JSON (default: the reference's fit_parameter.json)")
    ap.add_argument("--create-missing", action="store_true", help="create the result file when it does not exist")
    ap.add_argument("--quiet", action="store_true")
    a = ap.parse_args(argv)
    from . import reference_api as ref
    g = ref.configure(a.src, seed=a.seed)
    for n, f in zip(NAMES, FIELDS):
        getattr(ref, f)[None] = g["initial_garment_" + n] if n in ("E", "nu") else g["initial_" + n]
    ref.initialize_objects()
    res = parameters_learning(True, True, a.epochs, sim=ref, log=None if a.quiet else print)
    path = a.result or g["result_file_path"]
    write_result(path, res, create_missing=a.create_missing)
    return res


if __name__ == "__main__":
    main()
