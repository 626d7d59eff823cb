"""The committed ncu summaries that bench.py reads (profiles/<kernel>.md):
every summary of a kernel that bench.py's roofline can name carries the two
per-launch figures it reads (DRAM bytes for `roofline.traffic`, warp
instructions for `issue_roofline`), the command that made it, and no figure
that contradicts its own metric table.  CPU only."""
import os
import re
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

PROFILED = sorted(k for k in bench.KERNEL_BYTES if os.path.exists(os.path.join(ROOT, "profiles", k + ".md")))


def test_the_heavy_kernels_have_summaries():
    for k in ("k_tri_forward", "k_point_p2g", "k_g2p", "k_g2p_adj", "k_point_adj", "k_tri_adj"):
        assert k in PROFILED, k


@pytest.mark.parametrize("kernel", PROFILED)
def test_summary_carries_the_figures_bench_reads(kernel):
    text = open(os.path.join(ROOT, "profiles", kernel + ".md")).read()
    traffic = bench.ncu_figure(kernel, "dram_bytes_per_launch")
    inst = bench.ncu_figure(kernel, "warp_inst_per_launch")
    assert traffic and traffic > 0 and inst and inst > 0
    assert bench.ncu_traffic(kernel) == traffic
    # the capture command: one kernel, one to three launches, clocks left alone
    cmd = re.search(r"ncu --set full --clock-control none -k \S+ -s \d+ -c ([123]) ", text)
    assert cmd, kernel
    # the per-launch figures are the table's slice figures (of c launches)
    # scaled to the full sweep (about 2x) and divided by c
    c = int(cmd.group(1))
    m = re.search(r"\| DRAM read \+ write \| ([0-9.]+) MB", text)
    assert m and 1.9 / c < traffic / (float(m.group(1)) * 1e6) < 2.1 / c, kernel
    w = re.search(r"\| warp instructions \| ([0-9,]+)", text)
    assert w and 1.9 / c < inst / float(w.group(1).replace(",", "")) < 2.1 / c, kernel
