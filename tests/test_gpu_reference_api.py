"""The drop-in module (diffcp_b200.reference_api) driven exactly like the
reference's compute_grad, compared with finite differences of the reference's
own forward (golden vectors)."""
import os

import numpy as np
import pytest
import torch

from tests.golden import make_golden as mg
from tests.ref_tree import write_tree

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def ref(tmp_path_factory):
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    import diffcp_b200.reference_api as ref
    ref.configure(write_tree(tmp_path_factory.mktemp("ref")), seed=mg.SEED_OP, seed_cube=mg.SEED_CUBE)
    return ref


def _set_params(ref, p=None):
    p = p or mg.PARAMS
    ref.garment_E[None] = p["E"]
    ref.garment_nu[None] = p["nu"]
    ref.contact_stiffness[None] = p["contact_stiffness"]
    ref.shearing_stiffness[None] = p["shearing_stiffness"]


def _window_grads_vs_fd(ref, g, params, kc_material=True):
    _set_params(ref, params)
    ref.initialize_objects()
    ref.clear_distances()
    ref.target_pos.from_numpy(ref.target_pcd_array[0])
    with ref.ti.ad.Tape(loss=ref.loss):
        ref.loss[None] = 0
        for f in range(ref.max_steps - 1):
            ref.forward(f, 0)
        ref.compute_loss(f)
    assert ref.loss[None] == pytest.approx(float(g["loss"]), rel=2e-5, abs=0)
    for field, key in ((ref.garment_E, "fd_E"), (ref.garment_nu, "fd_nu"),
                       (ref.shearing_stiffness, "fd_shearing_stiffness"),
                       (ref.contact_stiffness, "fd_contact_stiffness")):
        fd = float(g[key])
        if key == "fd_contact_stiffness" and not kc_material:
            continue     # below float64 finite-difference resolution in this scene (see the press scene)
        assert fd != 0.0 and field.grad[None] == pytest.approx(fd, rel=1e-4, abs=0), (key, field.grad[None], fd)
    for name in g.files:
        if name.startswith("fd_seq_"):
            a, b, c = (int(t) for t in name[len("fd_seq_"):].split("_"))
            fd = float(g[name])
            # a single keyframe entry of a 300-substep window: float32 keeps it to
            # about 1.0e-4 (all keyframes together, max-norm: test_gpu_parity.py)
            assert fd != 0.0 and ref.grasp_tracking_seq.grad[a, b, c] == pytest.approx(fd, rel=1.5e-4, abs=0), name


def test_window_loss_and_gradients_match_reference_finite_differences(ref):
    _window_grads_vs_fd(ref, np.load(os.path.join(GOLD, "ref_fd_f64.npz")), mg.PARAMS, kc_material=False)


def test_forward_history_matches_reference_source(ref):
    gf = np.load(os.path.join(GOLD, "ref_forward_f32.npz"))
    _set_params(ref)
    ref.initialize_objects()
    for f in range(ref.max_steps - 1):
        ref.forward(f, 0)
    hist = ref.vertex_x.to_numpy()
    ref_hist = gf["w0_vertex_x"]
    assert hist.shape == ref_hist.shape
    assert np.abs(hist - ref_hist).max() < 2e-4 * np.abs(ref_hist).max()
    np.testing.assert_allclose(ref.operator_x[ref.max_steps - 1], gf["w0_operator_x"][-1], rtol=0, atol=1e-5)


def test_compute_grad_carries_state_across_windows(ref):
    _set_params(ref)
    ref.initialize_objects()
    loss, grads = ref.compute_grad()
    assert np.isfinite(loss) and loss > 0
    assert all(np.isfinite(x) for x in grads)
    # after the last window the rest shape is the end state of that window
    np.testing.assert_allclose(ref.initial_vertex_x.to_numpy(), ref.vertex_x[0], atol=1e-6)


def test_press_scene_gradients_match_reference_finite_differences(tmp_path):
    """The contact-engaging press scene (300 substeps): every gradient,
    contact stiffness included, against central differences of the
    reference's forward.  Reconfigures the module, so it runs last here."""
    import diffcp_b200.reference_api as ref
    ref.configure(write_tree(tmp_path, "press"), seed=mg.SEED_OP, seed_cube=mg.SEED_CUBE)
    _window_grads_vs_fd(ref, np.load(os.path.join(GOLD, "ref_fd_press_f64.npz")), mg.PARAMS_PRESS)
