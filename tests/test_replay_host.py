"""Host logic of the forward-only replay: which pose files animation()
writes after which block (simulation_without_grad.py:508-516), against the
reference's own run (golden vectors), and the oracle's reset against the
reference source on the CPU."""
import os

import numpy as np
import torch

from diffcp_b200 import replay
from tests.scenes import oracle_for, oracle_params, reference_small_scene

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_pose_schedule_matches_reference_animation():
    g = np.load(os.path.join(GOLD, "ref_replay_f32.npz"))
    n_counts, hits = replay.pose_schedule(float(g["animation_time"]), int(g["n_pose_estimation_output"]))
    order = [i for c in range(n_counts) for i in hits.get(c, [])]
    assert order == [int(i) for i in g["pose_index"]]


def test_pose_schedule_truncates_toward_zero():
    n, hits = replay.pose_schedule(0.01387, 35)
    assert n == 13 and hits[0] == [3, 4, 5, 6, 7]   # 13.87 * 3 / 35 - 2 = -0.81 truncates to 0


def test_oracle_replay_matches_reference_source():
    """The oracle's replay (substeps + reset_quadrature_particles) in float64
    against the reference's float32 run of simulation_without_grad.py."""
    from oracle import sim64
    g = np.load(os.path.join(GOLD, "ref_replay_f32.npz"))
    sc = reference_small_scene()
    sim, st = oracle_for(sc)
    seq = torch.tensor(sc.keyframes, dtype=torch.float64)
    seen = {}
    sim64.replay(sim, st, 6, int(g["block"]), oracle_params(sc), seq=seq,
                 on_count=lambda c, s: seen.__setitem__(c, (s["vx"].numpy(), s["qd"].numpy(), s["qF"].numpy(),
                                                            sim.D0inv.numpy().copy())))
    for c in range(6):
        vx, qd, qF, dinv = seen[c]
        ref = g["c%d_vertex_x" % c]
        assert np.abs(vx - ref).max() <= 2e-4 * np.abs(ref).max()
        assert np.abs(qd - g["c%d_quadrature_d" % c]).max() <= 2e-4 * np.abs(qd).max()
        assert np.abs(qF - g["c%d_quadrature_F" % c]).max() <= 2e-4
        ref_inv = g["c%d_initial_quadrature_d_inv" % c]
        assert np.abs(dinv - ref_inv).max() <= 2e-3 * np.abs(ref_inv).max()
