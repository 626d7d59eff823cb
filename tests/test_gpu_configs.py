"""The benchmark configurations at their own sizes: FP32 results against the
FP64 oracle where the oracle finishes in seconds, and size-independent
properties (checkpoint-interval invariance, finiteness, clean status) at the
full sizes."""
import numpy as np
import pytest
import torch

from diffcp_b200 import configs
from tests.scenes import oracle_loss, oracle_params

pytestmark = pytest.mark.gpu

ORDER_RTOL = 1e-4   # float-atomic summation order; the parity bar for gradients


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _grads(scenes, info, n_steps=None, ckpt=None):
    from diffcp_b200.batch import BatchSim, ClothBatch
    b = ClothBatch(scenes, dt=info["dt"], pool_blocks=info.get("pool_blocks", 0))
    n = n_steps or info["n_steps"]
    sim = BatchSim(b, n_steps=n, ckpt_every=ckpt or info["ckpt_every"])
    params = b.params.clone().requires_grad_(True)
    traj = b.traj.clone().requires_grad_(True)
    loss = sim.loss(params, traj)
    loss.sum().backward()
    return (loss.detach().double().cpu().numpy(), params.grad.double().cpu().numpy(),
            traj.grad.double().cpu().numpy(), b)


def _oracle(sc, n, keys=("E", "nu")):
    p = oracle_params(sc, requires_grad=True)
    lo, p, _, _, _ = oracle_loss(sc, n, n, params=p)
    lo.backward()
    return float(lo.detach()), {k: float(p[k].grad) for k in keys}


COL = {"E": 0, "nu": 1, "ks": 2, "kc": 3, "friction": 4, "damping": 5}


def test_single_sheet_config_loss_and_gradients_match_fp64_oracle():
    """32x32 sheet, 200 substeps, targets from the E 8e3 / nu 0.25 run:
    gradients w.r.t. E and nu within 1e-4 of the FP64 oracle."""
    scenes, info = configs.single_sheet(seed=0)
    loss, gp, _, b = _grads(scenes, info)
    assert b.status()[0] == 0
    lo, ref = _oracle(scenes[0], info["n_steps"])
    assert loss[0] == pytest.approx(lo, rel=1e-5)
    for k, r in ref.items():
        assert abs(gp[0, COL[k]] - r) <= 1e-4 * abs(r), (k, gp[0, COL[k]], r, abs(gp[0, COL[k]] - r) / abs(r))


def test_large_sheet_mesh_matches_oracle_on_a_short_horizon():
    """The 128x128 sheet on its 128^3 grid: 20 substeps against the FP64
    oracle, gradients w.r.t. E, nu, friction and damping."""
    scenes, info = configs.large_sheet(seed=0)
    n = 20
    loss, gp, _, _ = _grads(scenes, info, n_steps=n, ckpt=5)
    lo, ref = _oracle(scenes[0], n, keys=("E", "nu", "friction", "damping"))
    assert loss[0] == pytest.approx(lo, rel=1e-5)
    for k, r in ref.items():
        assert abs(gp[0, COL[k]] - r) <= 1e-4 * abs(r) + 1e-16, (k, gp[0, COL[k]], r)


def test_large_sheet_full_horizon_checkpoint_intervals_agree():
    """1000 substeps with checkpoints every 50 against every 20: the same
    loss and gradients (the recompute reproduces the forward)."""
    scenes, info = configs.large_sheet(seed=0)
    l50, g50, _, b = _grads(scenes, info)
    l20, g20, _, _ = _grads(scenes, info, ckpt=20)
    assert b.status()[0] == 0 and np.isfinite(g50).all()
    assert l50[0] == pytest.approx(l20[0], rel=1e-6)
    np.testing.assert_allclose(g50[0, :6], g20[0, :6], rtol=ORDER_RTOL, atol=1e-16)


def test_trajectory_config_gradients_match_oracle_finite_differences():
    """Two cloths shaped like the trajectory-optimisation batch (reduced mesh
    and horizon so the FP64 oracle stays fast): the velocity gradient on 32
    random coordinates per cloth against central differences of the oracle."""
    scenes, info = configs.trajectory_batch(seed=3, count=2, n=10, n_steps=30, dt=2e-4)
    _, _, gt, b = _grads(scenes, info)
    rng = np.random.default_rng(9)
    for i, sc in enumerate(scenes):
        off, _ = b.traj_slices(i)
        gv = gt[off: off + sc.velocities.size].reshape(sc.velocities.shape)
        scale = np.abs(gv).max()
        for _ in range(32):
            c = tuple(int(rng.integers(0, s)) for s in sc.velocities.shape)
            h = 1e-4
            vals = []
            for sgn in (1, -1):
                v = sc.velocities.copy()
                v[c] += sgn * h
                vals.append(float(oracle_loss(sc, info["n_steps"], info["n_steps"],
                                              vel=torch.tensor(v, dtype=torch.float64))[0]))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(gv[c] - fd) <= 2e-4 * scale, (i, c, gv[c], fd, scale)


def test_trajectory_config_full_size_runs_clean():
    scenes, info = configs.trajectory_batch(seed=0)
    loss, gp, gt, b = _grads(scenes, info)
    assert (b.status() == 0).all()
    assert np.isfinite(loss).all() and np.isfinite(gt).all() and np.abs(gt).max() > 0


def test_stress_config_full_size_memory_and_status():
    """512x512 sheet, 256^3 grid paged through a pool of 4^3-node blocks, 2000
    substeps with checkpoints every 45, loss and gradients: the run fits in a
    fraction of one GPU's memory, the grids hold under a sixth of the dense
    grid's blocks, the pool never overflows and every result is finite."""
    scenes, info = configs.stress_sheet(seed=0)
    torch.cuda.reset_peak_memory_stats()
    loss, gp, _, b = _grads(scenes, info)
    peak = torch.cuda.max_memory_allocated()
    assert peak < 60e9, peak
    assert int(b.sizes.grid_blocks) * 6 < int(b.sizes.total_nodes) // 64
    assert b.status()[0] == 0
    assert np.isfinite(loss).all() and np.isfinite(gp).all(), (loss, gp)


def test_stress_config_full_horizon_tracks_fp64_oracle():
    """The 512x512 sheet forward over all 2000 substeps, paged grid, against
    the FP64 oracle on the GPU: both stay finite, the float32 status stays
    clean, and the vertex positions stay within 1e-5 m of the oracle's (a
    compressed triangle column used to turn the float32 QR non-finite late in
    this horizon).  Prints the gap every 500 substeps."""
    from diffcp_b200.batch import ClothBatch
    from oracle.sim64 import KinematicGripper
    from tests.scenes import oracle_for
    scenes, info = configs.stress_sheet(seed=0)
    sc = scenes[0]
    dev = torch.device("cuda")
    b = ClothBatch(scenes, dt=info["dt"], reorder=False, pool_blocks=info["pool_blocks"])
    s, t = b.init_state(), b.new_state()
    sim, st = oracle_for(sc, device=dev)
    p = {k: v.to(dev) for k, v in oracle_params(sc).items()}
    grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=torch.float64, device=dev),
                            torch.tensor(sc.velocities, dtype=torch.float64, device=dev))
    worst = 0.0
    with torch.no_grad():
        for f in range(info["n_steps"]):
            b.forward_step(s, f, out=t)
            s, t = t, s
            st = sim.substep(st, f, 0, p, friction=p["friction"], damping=p["damping"], grip=grip)
            if f % 500 == 499:
                gap = float((b.vertex_x(s, 0).double() - st["vx"]).abs().max())
                assert np.isfinite(gap) and bool(torch.isfinite(st["vx"]).all()), f
                worst = max(worst, gap)
                print("STRESS-GAP substep %d: %.3e m" % (f + 1, gap))
    assert b.status()[0] == 0
    assert worst < 1e-5, worst


def test_stress_config_checkpoint_intervals_agree_on_200_substeps():
    scenes, info = configs.stress_sheet(seed=0)
    l45, g45, _, b = _grads(scenes, info, n_steps=200)
    l20, g20, _, _ = _grads(scenes, info, n_steps=200, ckpt=20)
    assert b.status()[0] == 0
    assert l45[0] == pytest.approx(l20[0], rel=1e-6)
    np.testing.assert_allclose(g45[0, :6], g20[0, :6], rtol=ORDER_RTOL, atol=1e-16)


def _chamfer64(x, t):
    """One-sided Chamfer (sum_q min_p |x_p - t_q|^2 / 3 / Nq) with the argmin
    taken in chunks (the loss is piecewise smooth, so its gradient is that of
    the selected pairs)."""
    with torch.no_grad():
        arg = torch.cat([torch.cdist(t[i: i + 256], x).argmin(1) for i in range(0, t.shape[0], 256)])
    return ((x[arg] - t) ** 2).sum() / 3 / t.shape[0]


def test_stress_config_matches_fp64_oracle_on_the_first_200_substeps():
    """The FP64 oracle (run on the GPU) against the FP32 kernels on the
    512x512 sheet: vertex positions over 200 substeps, and the loss and the
    E, nu, damping gradients of a 4-substep window."""
    from diffcp_b200.batch import ClothBatch
    from oracle.sim64 import KinematicGripper
    from tests.scenes import oracle_for
    scenes, info = configs.stress_sheet(seed=0)
    sc = scenes[0]
    dev = torch.device("cuda")
    b = ClothBatch(scenes, dt=info["dt"], reorder=False, pool_blocks=info["pool_blocks"])
    s, t = b.init_state(), b.new_state()
    sim, st = oracle_for(sc, device=dev)
    p = oracle_params(sc)
    p = {k: v.to(dev) for k, v in p.items()}
    grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=torch.float64, device=dev),
                            torch.tensor(sc.velocities, dtype=torch.float64, device=dev))
    worst = 0.0
    with torch.no_grad():
        for f in range(200):
            b.forward_step(s, f, out=t)
            s, t = t, s
            st = sim.substep(st, f, 0, p, friction=p["friction"], damping=p["damping"], grip=grip)
            if f % 50 == 49:
                got = b.vertex_x(s, 0).double()
                worst = max(worst, float((got - st["vx"]).abs().max()))
    assert worst < 1e-5, worst        # metres, in a unit domain
    # gradients of a 4-substep window
    from diffcp_b200.batch import BatchSim
    n = 4
    sim32 = BatchSim(b, n_steps=n, ckpt_every=2)
    params = b.params.clone().requires_grad_(True)
    loss = sim32.loss(params, b.traj)
    loss.sum().backward()
    sim64, st = oracle_for(sc, device=dev)
    q = {k: v.clone().requires_grad_(k in ("E", "nu", "damping")) for k, v in p.items()}
    for f in range(n):
        st = sim64.substep(st, f, 0, q, friction=q["friction"], damping=q["damping"], grip=grip)
    lo = _chamfer64(st["vx"], torch.tensor(sc.targets, dtype=torch.float64, device=dev))
    lo.backward()
    assert float(loss[0]) == pytest.approx(float(lo), rel=1e-5)
    for k in ("E", "nu", "damping"):
        r = float(q[k].grad)
        g = float(params.grad[0, COL[k]])
        assert abs(g - r) <= 1e-4 * abs(r) + 1e-18, (k, g, r)
