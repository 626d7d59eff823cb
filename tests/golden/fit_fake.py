"""A deterministic stand-in for ``compute_grad`` used to pin the parameter
fitting loop (parameter_fitting_functions.py:94-205) without a simulation.

The golden maker runs the reference's own ``parameters_learning`` against it,
and the tests run diffcp_b200.fitting.parameters_learning against the same
stand-in; both must visit the same parameters, learning rates and results.

Scalars behave like the reference's 0-D f32 Taichi fields read and written
from Python scope: values are stored as float32 and read back as Python
floats.
"""
import math

import numpy as np

NAMES = ("E", "nu", "contact_stiffness", "shearing_stiffness")
BOUNDS = {"E": (10.0, 1000.0), "nu": (0.05, 0.45), "contact_stiffness": (10.0, 5000.0),
          "shearing_stiffness": (1.0, 1000.0)}
FIELD = {"E": "garment_E", "nu": "garment_nu", "contact_stiffness": "contact_stiffness",
         "shearing_stiffness": "shearing_stiffness"}


class HostScalar:
    def __init__(self, value=0.0):
        self._v = np.float32(value)
        self._grad = None

    def __getitem__(self, key):
        return float(self._v)

    def __setitem__(self, key, value):
        self._v = np.float32(value)

    @property
    def grad(self):
        if self._grad is None:
            self._grad = HostScalar()
        return self._grad


def scenarios():
    """(name, initial params, targets, weights, epochs, nan_grad_at, nan_loss_at, learn flags)."""
    rng = np.random.default_rng(2024)
    out = []
    for k in range(6):
        init = {n: float(rng.uniform(*BOUNDS[n])) for n in NAMES}
        tgt = {n: float(rng.uniform(*BOUNDS[n])) for n in NAMES}
        w = {n: float(10.0 ** rng.uniform(-3, 3) / (BOUNDS[n][1] - BOUNDS[n][0]) ** 2) for n in NAMES}
        out.append(("random%d" % k, init, tgt, w, 12 if k % 2 else 35, None, None, (True, True)))
    init = {"E": 100.0, "nu": 0.1, "contact_stiffness": 100.0, "shearing_stiffness": 100.0}
    tgt = {"E": 400.0, "nu": 0.3, "contact_stiffness": 300.0, "shearing_stiffness": 150.0}
    w = {n: 1.0 / (BOUNDS[n][1] - BOUNDS[n][0]) ** 2 for n in NAMES}
    out.append(("elasticity_only", init, tgt, w, 10, None, None, (True, False)))
    out.append(("contact_only", init, tgt, w, 10, None, None, (False, True)))
    out.append(("nan_grad_epoch4", init, tgt, w, 10, 4, None, (True, True)))
    out.append(("nan_loss_epoch2", init, tgt, w, 6, None, 2, (True, True)))
    out.append(("near_bounds", {"E": 999.0, "nu": 0.0501, "contact_stiffness": 4999.0, "shearing_stiffness": 1.001},
                {"E": 10.0, "nu": 0.45, "contact_stiffness": 10.0, "shearing_stiffness": 1000.0}, w, 8, None, None,
                (True, True)))
    return out


def install(ns, init, tgt, w, nan_grad_at, nan_loss_at):
    """Binds f32 scalars and a quadratic-loss compute_grad into namespace
    ``ns`` (a module or object); returns the list that records, per call, the
    parameters and learning rates the loop passed in."""
    for n in NAMES:
        setattr(ns, FIELD[n], HostScalar(init[n]))
    setattr(ns, "loss", HostScalar())
    for k in range(4):
        setattr(ns, "learning_rate%d" % k, HostScalar())
    for n in NAMES:
        lo, hi = BOUNDS[n]
        setattr(ns, n + "_lower_bound", lo)
        setattr(ns, n + "_upper_bound", hi)
    calls = []

    def compute_grad():
        p = [getattr(ns, FIELD[n])[None] for n in NAMES]
        lr = [getattr(ns, "learning_rate%d" % k)[None] for k in range(4)]
        calls.append(p + lr)
        k = len(calls) - 1
        g = [float(np.float32(2.0 * w[n] * (p[j] - tgt[n]))) for j, n in enumerate(NAMES)]
        l = float(np.float32(sum(w[n] * (p[j] - tgt[n]) ** 2 for j, n in enumerate(NAMES))))
        if nan_grad_at == k:
            g[0] = math.nan
        if nan_loss_at == k:
            l = math.nan
        for j, n in enumerate(NAMES):
            getattr(ns, FIELD[n]).grad[None] = g[j]
        ns.loss[None] = l
        return l, g

    ns.compute_grad = compute_grad
    ns.initialize_objects = lambda: None
    return calls
