"""Paged grids (a pool of 4^3-node blocks shared by the batch and a page table
filled by k_alloc every substep) against dense grids on the same batches:
final vertex positions, losses and the gradients with respect to every
parameter and every gripper velocity or keyframe, through rollouts that
restore the grid from the tape and rollouts that recompute it, under each
scatter mode and register cap.  The two layouts add the same contributions
in different float-atomic orders, so they agree to that order's rounding.
Also: a pool too small for the batch flags STATUS_POOL_FULL and leaves the
CUDA context usable, and the stress configuration's pool holds every block
its first substeps touch."""
import numpy as np
import pytest
import torch

from diffcp_b200 import native
from tests.scenes import reference_small_scene, small_sheet

pytestmark = pytest.mark.gpu

ORDER_RTOL = 1e-4   # float-atomic summation order


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _sheets():
    # sheets of several sizes on grids of 24, 30 (not a multiple of 4) and 64
    # nodes, dragged by their grippers so the active blocks change every substep
    return [small_sheet(n=n, n_grid=g, n_steps=60, seed=s) for n, g, s in ((6, 24, 1), (12, 30, 2), (20, 64, 3))]


def _run(scenes, pool, tape, n_steps, ckpt, **launch):
    from diffcp_b200.batch import BatchSim, ClothBatch
    b = ClothBatch(scenes, dt=scenes[0].meta["dt"], pool_blocks=pool, **launch)
    sim = BatchSim(b, n_steps=n_steps, ckpt_every=ckpt, tape=tape)
    params = b.params.clone().requires_grad_(True)
    traj = b.traj.clone().requires_grad_(True)
    loss = sim.loss(params, traj)
    loss.sum().backward()
    torch.cuda.synchronize()
    x = [b.vertex_x(sim.final_state, i).double().cpu().numpy() for i in range(len(scenes))]
    return {"loss": loss.detach().double().cpu().numpy(), "gp": params.grad.double().cpu().numpy(),
            "gt": traj.grad.double().cpu().numpy(), "x": x, "status": b.status(), "batch": b}


def _agree(paged, dense):
    assert (paged["status"] == 0).all() and (dense["status"] == 0).all(), (paged["status"], dense["status"])
    np.testing.assert_allclose(paged["loss"], dense["loss"], rtol=1e-5, atol=0)
    for a, b in zip(paged["x"], dense["x"]):
        np.testing.assert_allclose(a, b, rtol=0, atol=1e-6)     # metres
    gp, gd = paged["gp"], dense["gp"]
    col = np.abs(gd).max(0, keepdims=True)
    assert (np.abs(gp - gd) <= ORDER_RTOL * col + 1e-30).all(), np.abs(gp - gd) / np.maximum(col, 1e-30)
    scale = np.abs(dense["gt"]).max()
    assert scale > 0 and np.abs(paged["gt"] - dense["gt"]).max() <= ORDER_RTOL * scale


@pytest.mark.parametrize("tape", ["auto", None])
@pytest.mark.parametrize("launch", [dict(scatter_mode=0, adj_scatter_mode=0),
                                    dict(scatter_mode=2, adj_scatter_mode=2, chunk=64, min_blocks=(6, 5, 3)),
                                    dict(scatter_mode=1, adj_scatter_mode=1, min_blocks=(3, 3, 3))])
def test_paged_sheets_match_dense_grids(tape, launch):
    scenes = _sheets()
    dense = _run(scenes, 0, "auto", 60, 7, **launch)
    paged = _run(scenes, "auto", tape, 60, 7, **launch)
    b = paged["batch"]
    assert 0 < b.pool_blocks < int(b.sizes.total_nodes) // 64
    assert int(b.sizes.grid_blocks) == b.pool_blocks + 1
    _agree(paged, dense)


def test_paged_operator_scene_matches_dense_grid():
    """The reference's kind of scene: operator particles driven by keyframes
    and a rigid cube, so the point chunks of every species claim blocks."""
    sc = reference_small_scene()
    dense = _run([sc], 0, "auto", 40, 5)
    paged = _run([sc], "auto", "auto", 40, 5)
    _agree(paged, dense)


def test_paged_single_substeps_match_dense_grid():
    """dcp_substep_forward / dcp_substep_backward one at a time (no tape)."""
    from diffcp_b200.batch import ClothBatch
    scenes = _sheets()
    out = {}
    for pool in (0, "auto"):
        b = ClothBatch(scenes, dt=scenes[0].meta["dt"], pool_blocks=pool)
        s = [b.init_state()]
        for f in range(5):
            s.append(b.forward_step(s[-1], f))
        gp, gt = b.new_grads()
        gen = torch.Generator(device=b.device).manual_seed(0)
        a = torch.randn(b.S, device=b.device, generator=gen) * 1e-3
        for f in range(4, -1, -1):
            a = b.backward_step(s[f], a, f, gp, gt)
        torch.cuda.synchronize()
        assert (b.status() == 0).all()
        out[pool] = (s[-1].double().cpu().numpy(), a.double().cpu().numpy(), gp.double().cpu().numpy())
    (sd, ad, gd), (sp, ap, gq) = out[0], out["auto"]
    # the state holds displacements (metres), velocities and affine matrices (order 1)
    np.testing.assert_allclose(sp, sd, rtol=0, atol=1e-5 * np.abs(sd).max())
    np.testing.assert_allclose(ap, ad, rtol=0, atol=ORDER_RTOL * np.abs(ad).max())
    np.testing.assert_allclose(gq, gd, rtol=0, atol=ORDER_RTOL * np.abs(gd).max())


def test_pool_too_small_flags_the_instances_and_the_context_stays_usable():
    """A pool of 4 blocks for sheets that touch dozens: the blocks without a
    slot are served by the spare block (wrong values, no access outside the
    arrays) and every instance reports STATUS_POOL_FULL.  A batch with a
    large enough pool then runs clean in the same context."""
    from diffcp_b200.batch import ClothBatch
    scenes = _sheets()
    b = ClothBatch(scenes, dt=scenes[0].meta["dt"], pool_blocks=4)
    s = b.init_state()
    for f in range(3):
        s = b.forward_step(s, f)
    gp, gt = b.new_grads()
    b.backward_step(s, torch.zeros(b.S, device=b.device), 2, gp, gt)
    torch.cuda.synchronize()
    st = b.status()
    assert (st & native.STATUS_POOL_FULL).all(), st
    ok = ClothBatch(scenes, dt=scenes[0].meta["dt"], pool_blocks="auto")
    s = ok.init_state()
    for f in range(3):
        s = ok.forward_step(s, f)
    torch.cuda.synchronize()
    assert (ok.status() == 0).all()


def test_stress_sheet_pool_holds_its_first_substeps():
    """The 512x512 sheet on its 256^3 grid, paged: 45 substeps (one
    checkpoint segment) forward and back with the tape; the pool never
    overflows, the grids take under a sixth of the dense grid's memory, and
    the state matches the dense layout's."""
    from diffcp_b200 import configs
    scenes, info = configs.stress_sheet(seed=0)
    paged = _run(scenes, info["pool_blocks"], "auto", 45, 45)
    dense = _run(scenes, 0, "auto", 45, 45)
    b = paged["batch"]
    assert int(b.sizes.grid_blocks) * 6 < int(b.sizes.total_nodes) // 64
    _agree(paged, dense)
