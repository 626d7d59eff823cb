"""The benchmark workloads that are built on the host: their sizes (the bench
line's particle counts depend on them) and their determinism per seed.  The
workloads whose targets come from a simulated final state need the GPU and
are covered by the GPU configuration tests."""
import numpy as np

from diffcp_b200 import configs


def _counts(scenes):
    return len(scenes), sum(s.n_vertex for s in scenes), sum(s.n_tri for s in scenes)


def test_parameter_sweep_sizes_and_settings():
    scenes, info = configs.parameter_sweep(0)
    assert _counts(scenes) == (256, 1008650, 1957660)
    assert (info["dt"], info["n_steps"], info["ckpt_every"]) == (1e-4, 300, 1)
    for sc in scenes:
        side = int(round(np.sqrt(sc.n_vertex)))
        assert side * side == sc.n_vertex and 16 <= side <= 96
        assert sc.n_tri == 2 * (side - 1) ** 2
        assert sc.n_grid == 64 and sc.targets.shape == (2048, 3)
        assert np.all(sc.vertices > 0) and np.all(sc.vertices < 1)


def test_parameter_sweep_is_deterministic_per_seed():
    a, _ = configs.parameter_sweep(0)
    b, _ = configs.parameter_sweep(0)
    c, _ = configs.parameter_sweep(1)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.vertices, y.vertices)
        np.testing.assert_array_equal(x.targets, y.targets)
        np.testing.assert_array_equal(x.triangles, y.triangles)
    assert [s.n_vertex for s in a] != [s.n_vertex for s in c]


def test_single_cloth_workloads():
    scenes, info = configs.large_sheet(0)
    assert _counts(scenes) == (1, 16384, 32258)
    assert (info["dt"], info["n_steps"], info["ckpt_every"]) == (1e-4, 1000, 50)
    scenes, info = configs.stress_sheet(0)
    assert _counts(scenes) == (1, 262144, 522242)
    assert (info["dt"], info["n_steps"]) == (5e-5, 2000)
    assert 1 <= info["ckpt_every"] <= info["n_steps"]
