"""The parameter-fitting driver against the reference's own heuristic and epoch
loop (golden vectors from parameter_fitting_functions.py:60-205 executed
under the Taichi stand-in; see tests/golden/make_golden.py)."""
import json
import math
import os
import sys
import types

import numpy as np
import pytest

from diffcp_b200 import fitting

GOLD = os.path.join(os.path.dirname(__file__), "golden")
sys.path.insert(0, GOLD)
import fit_fake  # noqa: E402


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "ref_fitting.npz"))


def _same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


def test_single_parameter_fitting_matches_reference(gold):
    for row, want in zip(gold["spf_in"], gold["spf_out"]):
        p, g, lo, hi, lr, epochs, idx = row
        got = fitting.single_parameter_fitting(float(p), float(g), 0, float(lo), float(hi), float(lr), int(epochs),
                                               int(idx))
        assert _same(got[0], float(want[0])) and _same(got[1], float(want[1])), (row, got, want)


def test_magnitude_level():
    assert fitting.magnitude_level(0.0) == -19
    assert fitting.magnitude_level(999.0) == 2
    assert fitting.magnitude_level(-0.0123) == -2


def test_single_parameter_fitting_outside_bounds_raises():
    with pytest.raises(ValueError):
        fitting.single_parameter_fitting(2000.0, -1.0, 0, 10.0, 1000.0, 1.0, 10, 3)


@pytest.mark.parametrize("scenario", [s[0] for s in fit_fake.scenarios()])
def test_parameters_learning_matches_reference(gold, scenario):
    name, init, tgt, w, epochs, nan_g, nan_l, flags = [s for s in fit_fake.scenarios() if s[0] == scenario][0]
    ns = types.SimpleNamespace()
    calls = fit_fake.install(ns, init, tgt, w, nan_g, nan_l)
    res = fitting.parameters_learning(flags[0], flags[1], epochs, sim=ns)
    want = gold["calls_" + name]
    got = np.array(calls)
    assert got.shape == want.shape
    np.testing.assert_array_equal(got, want)
    final = np.array([getattr(ns, fit_fake.FIELD[n])[None] for n in fit_fake.NAMES])
    np.testing.assert_array_equal(final, gold["final_" + name])
    assert _same(ns.loss[None], float(gold["loss_" + name]))
    assert res["epochs_run"] == len(want)


def test_write_result_merges_and_reports_missing_file(tmp_path):
    vals = {"E": 1.5, "nu": 0.25, "contact_stiffness": 7.0, "shearing_stiffness": 3.0}
    path = str(tmp_path / "fit_parameter.json")
    with pytest.raises(FileNotFoundError):
        fitting.write_result(path, vals)
    fitting.write_result(path, vals, create_missing=True)
    with open(path) as fh:
        assert json.load(fh) == vals
    with open(path, "w") as fh:
        json.dump({"note": "kept", "E": 0.0}, fh)
    fitting.write_result(path, vals)
    with open(path) as fh:
        assert json.load(fh) == dict(vals, note="kept")


def _vector_fake(scen):
    """fit_fake's compute_grad for several scenarios at once, in the (4, n)
    layout of fitting.fit_many."""
    calls = [0]

    def compute_grad(p):
        i = calls[0]
        calls[0] += 1
        n = len(scen)
        loss, g = np.empty(n), np.empty((4, n))
        for c, (_, _, tgt, w, _, nan_g, nan_l, _) in enumerate(scen):
            gc = [float(np.float32(2.0 * w[nm] * (p[j, c] - tgt[nm]))) for j, nm in enumerate(fit_fake.NAMES)]
            lc = float(np.float32(sum(w[nm] * (p[j, c] - tgt[nm]) ** 2 for j, nm in enumerate(fit_fake.NAMES))))
            if nan_g == i:
                gc[0] = math.nan
            if nan_l == i:
                lc = math.nan
            loss[c], g[:, c] = lc, gc
        return loss, g, g[0].copy()

    return compute_grad


@pytest.mark.parametrize("epochs", sorted({s[4] for s in fit_fake.scenarios()}))
def test_lockstep_fitting_matches_reference_per_problem(gold, epochs):
    scen = [s for s in fit_fake.scenarios() if s[4] == epochs]
    names = fit_fake.NAMES
    p0 = np.array([[s[1][nm] for s in scen] for nm in names])
    lower = np.array([[fit_fake.BOUNDS[nm][0]] * len(scen) for nm in names])
    upper = np.array([[fit_fake.BOUNDS[nm][1]] * len(scen) for nm in names])
    learn = np.array([[s[7][0], s[7][0], s[7][1], s[7][1]] for s in scen]).T
    res = fitting.fit_many(p0, lower, upper, _vector_fake(scen), epochs, learn)
    for c, s in enumerate(scen):
        want = gold["calls_" + s[0]]
        assert res["epochs_run"][c] == len(want)
        for e in range(len(want)):
            np.testing.assert_array_equal(res["history"][e]["params"][:, c], want[e, :4])
            np.testing.assert_array_equal(res["history"][e]["lr"][:, c], want[e, 4:])
        np.testing.assert_array_equal(res["params"][:, c], gold["final_" + s[0]])
        assert _same(float(np.float32(res["loss"][c])), float(gold["loss_" + s[0]]))
