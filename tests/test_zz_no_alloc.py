"""dcp_chamfer_forward_static: the Chamfer entry point for callers that cannot
allocate device memory (a plugin whose host application's allocator owns the
GPU, or a latency-bound loop where allocating is not allowed).  Its scratch is
a fixed device array inside the library; the caller passes only inputs and
outputs.  Two calls in a row, with different target counts, must each match
the batched entry point dcp_chamfer_forward on the same cloth state."""
import ctypes

import numpy as np
import pytest
import torch

from tests.scenes import small_sheet

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")


def _state_and_batch(n_targets, seed):
    from diffcp_b200.batch import ClothBatch
    sc = small_sheet(n=9, n_steps=6, seed=seed)
    rng = np.random.default_rng(seed)
    sc.targets = sc.vertices[rng.choice(sc.n_vertex, n_targets)] + rng.normal(0.0, 0.01, (n_targets, 3))
    b = ClothBatch([sc], dt=sc.meta["dt"], reorder=False)
    s = b.init_state()
    for f in range(5):
        s = b.forward_step(s, f)
    return b, s


def _static_call(lib, b, s, n_targets):
    loss = torch.full((1,), float("nan"), device=b.device)
    arg = torch.full((n_targets,), -7, dtype=torch.int32, device=b.device)
    x0 = b.rest_x0().contiguous()
    u = s[: 3 * b.nv].contiguous()
    rc = lib.dcp_chamfer_forward_static(x0.data_ptr(), u.data_ptr(), b.nv, b.targets.data_ptr(), n_targets,
                                        arg.data_ptr(), loss.data_ptr(), torch.cuda.current_stream().cuda_stream)
    return rc, loss, arg


def test_static_chamfer_matches_batched_entry_point_on_two_calls_in_a_row():
    from diffcp_b200 import native
    lib = native.lib()
    for n_targets, seed in ((300, 1), (100, 2)):       # the second call reads less scratch than the first wrote
        b, s = _state_and_batch(n_targets, seed)
        ref_loss, ref_arg = b.chamfer(s)
        rc, loss, arg = _static_call(lib, b, s, n_targets)
        assert rc == native.DCP_OK, lib.dcp_last_error()
        torch.cuda.synchronize()
        assert float(loss[0]) == pytest.approx(float(ref_loss[0]), rel=1e-6)
        np.testing.assert_array_equal(arg.cpu().numpy(), ref_arg[:n_targets].cpu().numpy())


def test_static_chamfer_rejects_more_targets_than_its_scratch_holds():
    from diffcp_b200 import native
    lib = native.lib()
    b, s = _state_and_batch(16, 3)
    rc, _, _ = _static_call(lib, b, s, 16)
    assert rc == native.DCP_OK
    x0 = b.rest_x0().contiguous()
    out = torch.zeros(1, device=b.device)
    rc = lib.dcp_chamfer_forward_static(x0.data_ptr(), None, b.nv, b.targets.data_ptr(),
                                        native.STATIC_MAX_TARGETS + 1, out.data_ptr(), out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    assert rc == native.DCP_ERR_INVALID if hasattr(native, "DCP_ERR_INVALID") else rc == 1
    assert b"DCP_STATIC_MAX_TARGETS" in lib.dcp_last_error()
