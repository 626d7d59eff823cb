"""Host side of the launch-configuration autotuner: workload signatures, the
cache file, and the ClothBatch arguments of a cached entry (no GPU)."""
import json

from diffcp_b200 import autotune, scene


def _sheet(n=6, n_grid=24, seed=1):
    return scene.sheet_scene(n=n, side=0.1, height=0.12, n_grid=n_grid, dt=2e-4, n_steps=4, E=3e3, nu=0.3,
                             friction=0.3, seed=seed, n_targets=32)


def test_signature_depends_on_shapes_and_dt_only():
    a, b = _sheet(seed=1), _sheet(seed=2)
    assert autotune.signature([a], 1e-4) == autotune.signature([b], 1e-4)   # same sizes, other draws
    assert autotune.signature([a], 1e-4) != autotune.signature([a], 2e-4)
    assert autotune.signature([a], 1e-4) != autotune.signature([a, a], 1e-4)
    assert autotune.signature([a], 1e-4) != autotune.signature([_sheet(n=7)], 1e-4)
    assert autotune.signature([a], 1e-4) != autotune.signature([_sheet(n_grid=32)], 1e-4)


def test_cached_reads_the_entry_of_the_workload(tmp_path):
    sc = _sheet()
    cfg = {"chunk": 64, "scatter_mode": 2, "adj_scatter_mode": 1, "min_blocks": [4, 3, 2]}
    path = tmp_path / "tuned.json"
    path.write_text(json.dumps({autotune.signature([sc], 1e-4): {"config": cfg}}))
    assert autotune.cached([sc], 1e-4, cache=str(path)) == cfg
    assert autotune.cached([sc, sc], 1e-4, cache=str(path)) is None
    assert autotune.cached([sc], 1e-4, cache=str(tmp_path / "absent.json")) is None


def test_batch_kwargs_of_new_and_older_entries():
    new = {"chunk": 64, "scatter_mode": 2, "adj_scatter_mode": 1, "min_blocks": [4, 3, 2]}
    assert autotune.batch_kwargs(new) == {"chunk": 64, "scatter_mode": 2, "adj_scatter_mode": 1,
                                          "min_blocks": [4, 3, 2]}
    # entries tuned before the adjoint scatter had its own mode use one mode for both
    old = {"chunk": 128, "scatter_mode": 0, "min_blocks": [2, 2, 1]}
    assert autotune.batch_kwargs(old)["adj_scatter_mode"] == 0
    assert autotune.batch_kwargs(autotune.DEFAULT)["chunk"] == autotune.DEFAULT["chunk"]


def test_committed_cache_entries_are_valid_launch_options():
    with open(autotune.CACHE) as fh:
        table = json.load(fh)
    assert table
    for ent in table.values():
        kw = autotune.batch_kwargs(ent["config"])
        assert kw["chunk"] % 32 == 0 and 32 <= kw["chunk"] <= 256
        assert kw["scatter_mode"] in (0, 1, 2) and kw["adj_scatter_mode"] in (0, 1, 2)
        assert len(kw["min_blocks"]) == 3 and all(1 <= v <= 6 for v in kw["min_blocks"])
