"""Parameter fitting on the GPU: the batched windowed gradient of BatchFitter
against the drop-in compute_grad (itself pinned to finite differences of the
reference source), and the parameter_fitting_main-style command line."""
import json
import os

import numpy as np
import pytest
import torch

from tests.golden import make_golden as mg
from tests.ref_tree import write_tree

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def tree(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return write_tree(tmp_path_factory.mktemp("ref"))


def _ref_grad(tree, p):
    import diffcp_b200.reference_api as ref
    ref.configure(tree, seed=mg.SEED_OP, seed_cube=mg.SEED_CUBE)
    ref.garment_E[None] = p["E"]
    ref.garment_nu[None] = p["nu"]
    ref.contact_stiffness[None] = p["contact_stiffness"]
    ref.shearing_stiffness[None] = p["shearing_stiffness"]
    ref.initialize_objects()
    return ref.compute_grad()


def test_batch_fitter_windows_match_drop_in_compute_grad(tree):
    from diffcp_b200.batch import BatchSim, ClothBatch
    from diffcp_b200.fitting import NAMES, PARAM_COL, BatchFitter
    from diffcp_b200.scene import load_reference_scene
    sets = [dict(mg.PARAMS), dict(mg.PARAMS, E=250.0, nu=0.2)]
    scenes = []
    for p in sets:
        sc = load_reference_scene(tree, seed=mg.SEED_OP, seed_cube=mg.SEED_CUBE)
        sc.params.update(p)
        scenes.append(sc)
    b = ClothBatch(scenes, dt=scenes[0].meta["dt"])
    n = scenes[0].meta["max_steps"] - 1
    sim = BatchSim(b, n_steps=n, loss_step=n - 2, ckpt_every=4)
    tw = [np.asarray(sc.meta["targets_by_window"]) for sc in scenes]
    windows = [b.pack_targets([t[w] for t in tw]) for w in range(tw[0].shape[0])]
    bounds = scenes[0].meta["bounds"]
    fit = BatchFitter(sim, bounds, windows=windows)
    loss, grads = fit.compute_grad()
    for c, p in enumerate(sets):
        want_loss, want = _ref_grad(tree, p)
        assert loss[c] == pytest.approx(want_loss, rel=1e-5)
        for j in range(4):
            assert grads[j, c] == pytest.approx(want[j], rel=1e-4, abs=1e-12), (c, NAMES[j], grads[j, c], want[j])
    # a short fit moves every cloth inside its bounds and leaves the batch at the best epoch
    res = fit.run(3)
    assert res["best_set"].all()
    vals = b.params.detach().cpu().numpy()
    for j, k in enumerate(NAMES):
        lo, hi = bounds[k]
        assert np.all((res["params"][j] >= lo) & (res["params"][j] <= hi))
        np.testing.assert_array_equal(vals[:, PARAM_COL[k]], res["params"][j].astype(np.float32))
    seen = np.array([h["loss"] for h in res["history"]])
    assert all(res["loss"][c] in seen[:, c] for c in range(len(sets)))


def test_fitting_command_line_writes_the_result_file(tree, tmp_path):
    from diffcp_b200 import fitting
    out = str(tmp_path / "fit_parameter.json")
    res = fitting.main(["--src", tree, "--epochs", "2", "--seed", str(mg.SEED_OP), "--result", out,
                        "--create-missing", "--quiet"])
    with open(out) as fh:
        written = json.load(fh)
    init = mg.ARGS["garment_parameters"]["initial_constitutive_parameters"]
    assert res["history"][0]["params"] == [float(np.float32(init[k])) for k in fitting.NAMES]
    for k in fitting.NAMES:
        lo = mg.ARGS["garment_parameters"]["constitutive_parameter_lower_bounds"][k]
        hi = mg.ARGS["garment_parameters"]["constitutive_parameter_upper_bounds"][k]
        assert lo <= written[k] <= hi
        assert written[k] == res[k]
    assert res["epochs_run"] == 2 and os.path.getsize(out) > 0
