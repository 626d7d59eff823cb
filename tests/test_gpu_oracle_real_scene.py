"""The FP64 oracle on the reference's own scene (data/cloth_mesh.ply, the
first grasp frames and target windows of its data/ files, windows of 300
substeps), run on the GPU, against golden vectors of the reference source run
on the same tree (tests/golden/make_golden.py, modes real32 and real64):

  * two grasp windows with the end-state carry-over of compute_grad
    (parameter_fitting_functions.py:40-49): vertex histories, the operator
    and cube end positions, per-window losses;
  * window 1's gradients against central differences of the reference's
    window-1 loss, the carried-in state held fixed (one Tape covers one
    window); only parameters whose relative sensitivity a float64 difference
    resolves are compared (MIN_SENSITIVITY)."""
import numpy as np
import pytest
import torch

from tests.golden import make_golden as mg
from tests.ref_tree import write_real_tree
from tests.test_oracle_real_scene import (MIN_SENSITIVITY, _end, _load, _params, _window, oracle_scene,
                                          resolved_seq_differences)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gold():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return _load("ref_real_f32.npz")


@pytest.fixture(scope="module")
def tree(tmp_path_factory, gold):
    return write_real_tree(tmp_path_factory.mktemp("real"), gold)


def test_oracle_windows_with_carry_over_match_reference_source(gold, tree):
    sc = oracle_scene(tree)
    dev = torch.device("cuda")
    n_win = int(gold["n_windows"])
    assert n_win == 2 and sc["max_steps"] == 301
    params = _params(gold["params"], device=dev)
    seq = torch.tensor(sc["grasp_point_pos"], dtype=torch.float64, device=dev)
    init = (sc["vertices"], sc["operator_x"], sc["cube_x"])
    losses = []
    for g in range(n_win):
        states, loss = _window(sc, g, init, params, seq, dev)
        ref = gold["w%d_vertex_x" % g]                 # every REAL_HISTORY_STRIDE-th substep
        got = np.stack([s["vx"].cpu().numpy() for s in states[::mg.REAL_HISTORY_STRIDE]])
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 2e-4, (g, err)
        np.testing.assert_allclose(states[-1]["ox"].cpu().numpy(), gold["w%d_operator_x_end" % g], rtol=0, atol=1e-5)
        np.testing.assert_allclose(states[-1]["cx"].cpu().numpy(), gold["w%d_cube_x_end" % g], rtol=0, atol=1e-5)
        assert float(loss) == pytest.approx(float(gold["w%d_loss" % g]), rel=1e-4, abs=0), g
        losses.append(float(loss))
        init = _end(states)                       # parameter_fitting_functions.py:40-49
    assert np.mean(losses) == pytest.approx(float(gold["loss_mean"]), rel=1e-4, abs=0)


def test_oracle_window1_gradients_match_reference_finite_differences(tree):
    g = _load("ref_real_fd_f64.npz")
    sc = oracle_scene(tree)
    dev = torch.device("cuda")
    seq0 = torch.tensor(sc["grasp_point_pos"], dtype=torch.float64, device=dev)
    states, loss0 = _window(sc, 0, (sc["vertices"], sc["operator_x"], sc["cube_x"]), _params(g["params"], device=dev),
                            seq0, dev)
    assert float(loss0) == pytest.approx(float(g["w0_loss"]), rel=1e-10, abs=0)
    np.testing.assert_allclose(states[-1]["vx"].cpu().numpy(), g["w0_vertex_x_end"], rtol=0, atol=1e-12)
    params = _params(g["params"], grad=True, device=dev)
    seq = seq0.clone().requires_grad_(True)
    _, loss = _window(sc, 1, _end(states), params, seq, dev)
    assert float(loss) == pytest.approx(float(g["w1_loss"]), rel=1e-10, abs=0)
    loss.backward()
    L = float(loss)
    checked = 0
    for k, key, pv in (("E", "w1_fd_E", 0), ("nu", "w1_fd_nu", 1), ("kc", "w1_fd_contact_stiffness", 2),
                       ("ks", "w1_fd_shearing_stiffness", 3)):
        fd = float(g[key])
        sens = abs(fd) * float(g["params"][pv]) / L
        if sens < MIN_SENSITIVITY:
            continue
        got = float(params[k].grad)
        assert got == pytest.approx(fd, rel=2e-4, abs=0), (k, got, fd)
        checked += 1
    for a, b, c, fd in resolved_seq_differences(g):
        assert float(seq.grad[a, b, c]) == pytest.approx(fd, rel=2e-4, abs=0), (a, b, c)
        checked += 1
    assert checked >= 2
