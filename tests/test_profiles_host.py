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


def test_step_issue_counts_full_launches_only(monkeypatch):
    """The whole-step issue figure: per-launch instruction counts times full
    launches (the P2G kernels' early-exit adjoint launches left out) over the
    step time, against 4 warp instructions per cycle per SM."""
    import torch

    class Props:
        multi_processor_count = 148

    monkeypatch.setattr(torch.cuda, "get_device_properties", lambda i: Props())
    prof = {"k_tri_forward": (78.4, 600), "k_g2p_adj": (99.6, 300), "k_unprofiled": (1.0, 300)}
    r = bench.step_issue(prof, 300, 400.0, 2000.0)
    inst = 300 * bench.ncu_figure("k_tri_forward", "warp_inst_per_launch") + \
        300 * bench.ncu_figure("k_g2p_adj", "warp_inst_per_launch")
    assert r["warp_inst_per_step"] == pytest.approx(inst)
    assert r["peak"] == pytest.approx(4 * 148 * 2000e6)
    assert r["frac"] == pytest.approx(inst / 0.4 / r["peak"])
    assert r["not_counted"] == ["k_unprofiled"] and r["profile_share_counted"] == pytest.approx(178.0 / 179.0)
    assert bench.step_issue(prof, 300, 400.0, None) is None
