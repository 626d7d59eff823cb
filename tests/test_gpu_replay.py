"""Forward-only replay on the GPU (dcp_replay: substep blocks with the
rest-frame reset of simulation_without_grad.py) against the reference's own
run (golden vectors) and the oracle, and the state-estimation command line's
pose files."""
import json
import os

import numpy as np
import pytest
import torch

from tests.golden import make_golden as mg
from tests.ref_tree import write_tree
from tests.scenes import oracle_for, oracle_params, reference_small_scene, small_sheet

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _rel(got, ref):
    return float(np.abs(got - ref).max()) / max(float(np.abs(ref).max()), 1e-12)


def _oracle_replay(sc, n_counts, block):
    from oracle import sim64
    from oracle.sim64 import KinematicGripper
    sim, st = oracle_for(sc)
    p = oracle_params(sc)
    seq = grip = None
    fr = None
    if sc.gripper_mode == 1:
        seq = torch.tensor(sc.keyframes, dtype=torch.float64)
    else:
        grip = KinematicGripper(sc.gripper_radius, torch.tensor(sc.centers, dtype=torch.float64),
                                torch.tensor(sc.velocities, dtype=torch.float64))
        fr = p["friction"]
    seen = []
    sim64.replay(sim, st, n_counts, block, p, seq=seq, friction=fr, damping=p["damping"], grip=grip,
                 on_count=lambda c, s: seen.append(s["vx"].numpy().copy()))
    return seen


def test_replay_matches_reference_source_golden():
    from diffcp_b200.batch import ClothBatch
    from diffcp_b200.replay import Replay
    g = np.load(os.path.join(GOLD, "ref_replay_f32.npz"))
    sc = reference_small_scene()
    b = ClothBatch([sc], dt=sc.meta["dt"])
    rep = Replay(b)
    assert rep.block == int(g["block"])
    for c in range(6):
        rep.run(1)
        assert _rel(rep.vertices(0), g["c%d_vertex_x" % c]) < 2e-4, c
    assert b.status()[0] & 3 == 0


def test_replay_matches_oracle_on_a_kinematic_sheet_and_in_a_batch():
    from diffcp_b200.batch import ClothBatch
    from diffcp_b200.replay import Replay
    scenes = [small_sheet(n=7, n_steps=40, seed=4), reference_small_scene(), small_sheet(n=5, n_steps=40, seed=9)]
    block = 4
    want = [_oracle_replay(sc, 8, block) for sc in scenes]
    b = ClothBatch(scenes, dt=scenes[0].meta["dt"])
    rep = Replay(b, block=block)
    for c in range(8):
        rep.run(1)
        for i in range(len(scenes)):
            assert _rel(rep.vertices(i), want[i][c]) < 2e-4, (c, i)


def test_replay_in_one_call_equals_block_by_block():
    from diffcp_b200.batch import ClothBatch
    from diffcp_b200.replay import Replay
    sc = small_sheet(n=7, n_steps=40, seed=4)
    r1 = Replay(ClothBatch([sc], dt=sc.meta["dt"]), block=3)
    r2 = Replay(ClothBatch([sc], dt=sc.meta["dt"]), block=3)
    r1.run(5)
    for _ in range(5):
        r2.run(1)
    assert _rel(r1.vertices(0), r2.vertices(0)) < 1e-6


def test_state_estimation_command_line_writes_reference_poses(tmp_path):
    from diffcp_b200 import io_ply, replay
    g = np.load(os.path.join(GOLD, "ref_replay_f32.npz"))
    src = write_tree(tmp_path)
    result = os.path.join(src, "..", "result")
    os.makedirs(result, exist_ok=True)
    with open(os.path.join(result, "fitting_result.json"), "w") as fh:
        json.dump(mg.PARAMS, fh)
    written = replay.main(["--src", src, "--seed", str(mg.SEED_OP), "--seed-cube", str(mg.SEED_CUBE)])
    assert written == [int(i) for i in g["pose_index"]]
    last = {int(i): v for i, v in zip(g["pose_index"], g["pose_vertices"])}
    for i, ref in last.items():
        v, t = io_ply.read_ply(os.path.join(result, "pose_estimation_output", "%d.ply" % i))
        assert t.shape[0] == len(reference_small_scene().triangles)
        assert _rel(v, ref) < 2e-4, i
    assert os.path.exists(os.path.join(src, "..", "tmp", "initial_vertices.npy"))
