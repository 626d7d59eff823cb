"""Host-side scene construction (CPU)."""
import numpy as np
import pytest

from diffcp_b200 import io_ply, scene
from tests.ref_scene import small_reference_scene
from tests.scenes import reference_small_scene


def test_product_reference_scene_matches_oracle_restatement():
    a = reference_small_scene()
    o = small_reference_scene()
    c = o["const"]
    assert a.n_grid == c.n_grid
    for k in ("vertex_p_mass", "quadrature_p_mass", "quadrature_p_vol", "operator_p_mass", "cube_p_mass",
              "gravity_dv"):
        assert getattr(a, k) == pytest.approx(getattr(c, k), rel=1e-14)
    assert a.group_size == c.grasper_group_size and a.frames_per_window == c.frames_per_window
    np.testing.assert_allclose(a.vertices, o["vertices"], atol=1e-15)
    np.testing.assert_allclose(a.operator_x, o["operator_x"], atol=1e-15)
    np.testing.assert_allclose(a.cube_x, o["cube_x"], atol=1e-15)
    np.testing.assert_allclose(a.keyframes, o["grasp_point_pos"], atol=1e-15)
    assert a.meta["max_steps"] == o["max_steps"]


def test_sheet_counts_of_the_single_cloth_configuration():
    sc = scene.sheet_scene(n=32, side=0.2, height=0.3, n_grid=64, dt=2e-4, n_steps=200)
    assert sc.n_vertex == 1024 and sc.n_tri == 1922
    assert sc.targets.shape == (2048, 3)
    assert sc.velocities.shape == (200, 2, 3) and sc.centers.shape == (200, 2, 3)
    np.testing.assert_allclose(sc.centers[0], sc.vertices[[0, 31]], atol=1e-12)
    assert sc.vertex_p_mass == pytest.approx(0.2 * 0.04 / 1024)
    big = scene.sheet_scene(n=128, side=0.4, n_grid=128, dt=1e-4, n_steps=10, n_targets=0)
    assert big.n_vertex == 16384 and big.n_tri == 32258


def test_ply_round_trip(tmp_path):
    v, t = scene.regular_sheet(5, 1.0)
    p = tmp_path / "m.ply"
    io_ply.write_ply(str(p), v, t)
    v2, t2 = io_ply.read_ply(str(p))
    np.testing.assert_array_equal(t2, t)
    np.testing.assert_allclose(v2, v)


def test_morton_order_is_a_permutation_and_local():
    v, _ = scene.regular_sheet(16, 0.3)
    order = scene.morton_order(v + 0.3, 1 / 64)
    assert sorted(order.tolist()) == list(range(len(v)))
    first = v[order[:16]]
    assert np.ptp(first[:, 0]) < 0.1 and np.ptp(first[:, 2]) < 0.1


def test_reference_api_fails_loudly_without_cuda(tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU error path")
    from tests.ref_tree import write_tree
    import diffcp_b200.reference_api as ref
    with pytest.raises(RuntimeError, match="CUDA"):
        ref.configure(write_tree(tmp_path), seed=0)
