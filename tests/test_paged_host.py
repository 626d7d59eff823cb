"""Host side of the paged grids (CPU only): the stencil-block enumeration
that sizes the pool against a direct enumeration of every stencil node, and
the pool size chosen for the 512x512 stress sheet."""
import numpy as np

from diffcp_b200 import configs
from diffcp_b200.batch import auto_pool_blocks, stencil_blocks


def _brute(points, n_grid):
    nb = (n_grid + 3) // 4
    out = set()
    for p in points:
        base = np.clip(np.floor(p * n_grid - 0.5), 0, n_grid - 3).astype(int)
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    n = base + (i, j, k)
                    out.add(((n[0] // 4) * nb + n[1] // 4) * nb + n[2] // 4)
    return np.array(sorted(out))


def test_stencil_blocks_match_every_node_of_every_stencil():
    rng = np.random.default_rng(3)
    for n_grid in (16, 30, 64):
        pts = rng.uniform(-0.05, 1.05, (300, 3))     # some outside the domain: clamped like the kernels
        np.testing.assert_array_equal(stencil_blocks(pts, n_grid), _brute(pts, n_grid))


def test_stress_sheet_pool_is_a_small_part_of_the_dense_grid():
    scenes, info = configs.stress_sheet(0)
    assert info["pool_blocks"] == "auto"
    pool = auto_pool_blocks(scenes)
    touched = len(stencil_blocks(np.concatenate([scenes[0].vertices,
                                                 scenes[0].vertices[scenes[0].triangles].mean(1)]), 256))
    assert pool == 4 * touched + 256
    assert pool < 64 ** 3 // 6          # under a sixth of the dense 256^3 grid's blocks
