"""dcp_chamfer_forward_static: the Chamfer entry point for callers that cannot
allocate device memory (a plugin whose host application's allocator owns the
GPU, or a latency-bound loop where allocating is not allowed).  Its scratch is
a fixed device array inside the library; the caller passes only inputs and
outputs.

Checked here, always against the batched entry point dcp_chamfer_forward on
the same cloth state: two calls in a row with different target counts; the
NULL-displacement form; non-finite vertices; a call made from a second CUDA
context that the caller created with the driver API (the array has another
address there); and the rejection of target counts beyond the array."""
import ctypes
import math

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


def _static_call(lib, b, s, n_targets, with_u=True):
    loss = torch.full((1,), float("nan"), device=b.device)
    arg = torch.full((n_targets,), -7, dtype=torch.int32, device=b.device)
    x0 = b.rest_x0().contiguous()
    u = s[: 3 * b.nv].contiguous() if with_u else None
    rc = lib.dcp_chamfer_forward_static(x0.data_ptr(), None if u is None else u.data_ptr(), b.nv,
                                        b.targets.data_ptr(), n_targets, arg.data_ptr(), loss.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
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


def test_static_chamfer_without_displacements_matches_the_rest_state():
    """u = NULL means zero displacement: the batched loss of the initial state."""
    from diffcp_b200 import native
    lib = native.lib()
    b, _ = _state_and_batch(64, 4)
    s0 = b.init_state()
    ref_loss, ref_arg = b.chamfer(s0)
    rc, loss, arg = _static_call(lib, b, s0, 64, with_u=False)
    assert rc == native.DCP_OK, lib.dcp_last_error()
    torch.cuda.synchronize()
    assert float(loss[0]) == pytest.approx(float(ref_loss[0]), rel=1e-6)
    np.testing.assert_array_equal(arg.cpu().numpy(), ref_arg[:64].cpu().numpy())


def test_static_chamfer_skips_a_nan_vertex_and_gives_nan_when_all_are_nan():
    from diffcp_b200 import native
    lib = native.lib()
    b, s = _state_and_batch(80, 5)
    s = s.clone()
    s[7] = float("nan")                          # x displacement of vertex 7
    b.status()                                   # clear
    ref_loss, ref_arg = b.chamfer(s)
    st = b.status()
    rc, loss, arg = _static_call(lib, b, s, 80)
    assert rc == native.DCP_OK, lib.dcp_last_error()
    torch.cuda.synchronize()
    assert math.isfinite(float(ref_loss[0]))
    assert float(loss[0]) == pytest.approx(float(ref_loss[0]), rel=1e-6)
    np.testing.assert_array_equal(arg.cpu().numpy(), ref_arg[:80].cpu().numpy())
    assert not (arg.cpu().numpy() == 7).any()
    assert st[0] & native.STATUS_NONFINITE
    s[: 3 * b.nv] = float("nan")                 # every vertex
    ref_loss, ref_arg = b.chamfer(s)
    st = b.status()
    rc, loss, arg = _static_call(lib, b, s, 80)
    assert rc == native.DCP_OK, lib.dcp_last_error()
    torch.cuda.synchronize()
    assert math.isnan(float(ref_loss[0])) and math.isnan(float(loss[0]))
    assert (arg.cpu().numpy() == -1).all() and (ref_arg[:80].cpu().numpy() == -1).all()
    assert st[0] & native.STATUS_NONFINITE


class _Driver:
    """The few CUDA driver API calls the second-context test needs (libcuda)."""

    def __init__(self):
        self.cu = ctypes.CDLL("libcuda.so.1")
        for name in ("cuCtxCreate_v2", "cuMemAlloc_v2", "cuMemcpyHtoD_v2", "cuMemcpyDtoH_v2", "cuMemFree_v2",
                     "cuCtxDestroy_v2", "cuCtxSynchronize", "cuDeviceGet", "cuInit"):
            getattr(self.cu, name).restype = ctypes.c_int
        self.cu.cuMemcpyHtoD_v2.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_size_t]
        self.cu.cuMemcpyDtoH_v2.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_size_t]
        self.cu.cuMemFree_v2.argtypes = [ctypes.c_uint64]

    def ok(self, rc, what):
        assert rc == 0, "%s failed with CUresult %d" % (what, rc)

    def alloc_copy(self, arr):
        p = ctypes.c_uint64()
        self.ok(self.cu.cuMemAlloc_v2(ctypes.byref(p), ctypes.c_size_t(arr.nbytes)), "cuMemAlloc")
        self.ok(self.cu.cuMemcpyHtoD_v2(p.value, arr.ctypes.data, arr.nbytes), "cuMemcpyHtoD")
        return p.value


def test_static_chamfer_in_a_second_context_created_with_the_driver_api():
    """A host application may run the library in a context of its own (driver
    API, current on the calling thread) instead of the device's primary
    context: the scratch array has a different address there, and the entry
    point must look it up for that context.  Inputs live in that context."""
    from diffcp_b200 import native
    lib = native.lib()
    b, s = _state_and_batch(200, 6)
    ref_loss, ref_arg = b.chamfer(s)
    rc, loss_p, _ = _static_call(lib, b, s, 200)       # primary context first: its address is cached
    assert rc == native.DCP_OK, lib.dcp_last_error()
    torch.cuda.synchronize()
    x0 = np.ascontiguousarray(b.rest_x0().cpu().numpy(), dtype=np.float32)
    u = np.ascontiguousarray(s[: 3 * b.nv].cpu().numpy(), dtype=np.float32)
    tg = np.ascontiguousarray(b.targets.cpu().numpy(), dtype=np.float32)
    drv = _Driver()
    drv.ok(drv.cu.cuInit(0), "cuInit")
    dev = ctypes.c_int()
    drv.ok(drv.cu.cuDeviceGet(ctypes.byref(dev), torch.cuda.current_device()), "cuDeviceGet")
    ctx = ctypes.c_void_p()
    drv.ok(drv.cu.cuCtxCreate_v2(ctypes.byref(ctx), 0, dev), "cuCtxCreate")   # pushed: now current
    ptrs = []
    try:
        px0, pu, ptg = drv.alloc_copy(x0), drv.alloc_copy(u), drv.alloc_copy(tg)
        parg = drv.alloc_copy(np.full(200, -7, dtype=np.int32))
        ploss = drv.alloc_copy(np.full(1, np.nan, dtype=np.float32))
        ptrs = [px0, pu, ptg, parg, ploss]
        for _ in range(2):
            rc = lib.dcp_chamfer_forward_static(px0, pu, b.nv, ptg, 200, parg, ploss, None)
            assert rc == native.DCP_OK, lib.dcp_last_error()
        drv.ok(drv.cu.cuCtxSynchronize(), "cuCtxSynchronize")
        got_arg = np.empty(200, dtype=np.int32)
        got_loss = np.empty(1, dtype=np.float32)
        drv.ok(drv.cu.cuMemcpyDtoH_v2(got_arg.ctypes.data, parg, got_arg.nbytes), "cuMemcpyDtoH")
        drv.ok(drv.cu.cuMemcpyDtoH_v2(got_loss.ctypes.data, ploss, got_loss.nbytes), "cuMemcpyDtoH")
    finally:
        for p in ptrs:
            drv.cu.cuMemFree_v2(p)
        drv.ok(drv.cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")               # popped: primary current again
    assert float(got_loss[0]) == pytest.approx(float(ref_loss[0]), rel=1e-6)
    np.testing.assert_array_equal(got_arg, ref_arg[:200].cpu().numpy())
    rc, loss_p2, _ = _static_call(lib, b, s, 200)      # the primary context's cached address still serves
    assert rc == native.DCP_OK, lib.dcp_last_error()
    torch.cuda.synchronize()
    assert float(loss_p2[0]) == float(loss_p[0])


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
    assert rc == native.DCP_ERR_INVALID
    assert b"DCP_STATIC_MAX_TARGETS" in lib.dcp_last_error()
