"""CPU checks of the C-ABI boundary: the library loads without a GPU, exports
every entry point that include/diffcp_b200.h declares, its structs have the C
layout, and host-side validation rejects bad input (no CUDA call is made)."""
import ctypes
import os
import re
import subprocess

import pytest

from diffcp_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diffcp_b200.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|int32_t|int64_t|const char\*)\s+(dcp_\w+)\s*\(", txt, re.M)))


def test_library_loads_and_exports_every_declared_symbol():
    L = native.lib()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(native.EXPORTED)
    out = subprocess.run(["nm", "-D", native.lib_path()], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(r"\bT %s\b" % n, out), n


def test_struct_layout_matches_c_compiler(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "%s"\nint main(void){printf("%%zu %%zu %%zu %%zu %%zu\\n",'
                   ' sizeof(DcpInstance), sizeof(DcpOptions), sizeof(DcpSizes), offsetof(DcpInstance, gripper_radius),'
                   ' offsetof(DcpSizes, total_nodes)); printf("%%zu %%zu\\n", offsetof(DcpOptions, pool_blocks),'
                   ' offsetof(DcpSizes, grid_blocks)); return 0;}\n' % HEADER)
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    vals = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()]
    assert vals == [ctypes.sizeof(native.DcpInstance), ctypes.sizeof(native.DcpOptions),
                    ctypes.sizeof(native.DcpSizes), native.DcpInstance.gripper_radius.offset,
                    native.DcpSizes.total_nodes.offset, native.DcpOptions.pool_blocks.offset,
                    native.DcpSizes.grid_blocks.offset]


def _inst(**kw):
    I = native.DcpInstance()
    I.n_vertex, I.n_tri, I.n_grid, I.bound = 16, 18, 16, 3
    for k, v in kw.items():
        setattr(I, k, v)
    return I


def test_plan_sizes_and_validation():
    L = native.lib()
    insts = (native.DcpInstance * 2)(_inst(), _inst(n_grid=15, n_target=7))
    opt = native.DcpOptions(dt=1e-4, chunk=128, svd_grad=0, grid_ctas=0)
    s = native.DcpSizes()
    assert L.dcp_plan(insts, 2, ctypes.byref(opt), ctypes.byref(s)) == 0
    assert s.n_vertex == 32 and s.n_tri == 36 and s.n_target == 7
    assert s.state_floats == 15 * 32 + 18 * 36
    assert s.total_nodes == 4 ** 3 * 64 * 2      # 15 nodes per axis pad to 4 blocks of 4
    assert s.n_tri_chunks == 2 and s.n_point_chunks == 2
    bad = native.DcpOptions(dt=1e-4, chunk=100, svd_grad=0, grid_ctas=0)
    assert L.dcp_plan(insts, 2, ctypes.byref(bad), ctypes.byref(s)) == 1
    assert b"chunk" in L.dcp_last_error()
    bad = native.DcpOptions(dt=1e-4, chunk=128, svd_grad=0, grid_ctas=0, adj_scatter_mode=3)
    assert L.dcp_plan(insts, 2, ctypes.byref(bad), ctypes.byref(s)) == 1
    assert b"adj_scatter_mode" in L.dcp_last_error()
    insts2 = (native.DcpInstance * 1)(_inst(gripper_mode=1, n_grippers=2, group_size=3, n_operator=5, n_actions=4,
                                            keyframe_interval=0.03))
    assert L.dcp_plan(insts2, 1, ctypes.byref(opt), ctypes.byref(s)) == 1
    assert b"n_operator" in L.dcp_last_error()
    with pytest.raises(native.DcpError):
        native.check(L.dcp_plan(insts2, 1, ctypes.byref(opt), ctypes.byref(s)), "plan")


def test_paged_grid_plan_holds_only_the_pool():
    """pool_blocks > 0: each grid array holds the pool plus one spare block
    instead of every block of every instance; the dense plan reports all of
    them.  Out-of-range pool sizes are rejected."""
    L = native.lib()
    insts = (native.DcpInstance * 2)(_inst(n_grid=256), _inst(n_grid=64))
    dense = native.DcpOptions(dt=1e-4, chunk=128, svd_grad=0, grid_ctas=0)
    paged = native.DcpOptions(dt=1e-4, chunk=128, svd_grad=0, grid_ctas=0, pool_blocks=1000)
    sd, sp = native.DcpSizes(), native.DcpSizes()
    assert L.dcp_plan(insts, 2, ctypes.byref(dense), ctypes.byref(sd)) == 0
    assert L.dcp_plan(insts, 2, ctypes.byref(paged), ctypes.byref(sp)) == 0
    blocks = 64 ** 3 + 16 ** 3
    assert sd.total_nodes == sp.total_nodes == 64 * blocks
    assert sd.grid_blocks == blocks and sp.grid_blocks == 1001
    # three float4 grid arrays: dense minus paged is their size difference
    assert sd.workspace_bytes - sp.workspace_bytes >= 3 * 16 * 64 * (blocks - 1001)
    for bad in (-1, (1 << 24) + 1):
        opt = native.DcpOptions(dt=1e-4, chunk=128, svd_grad=0, grid_ctas=0, pool_blocks=bad)
        assert L.dcp_plan(insts, 2, ctypes.byref(opt), ctypes.byref(sp)) == 1
        assert b"pool_blocks" in L.dcp_last_error()
