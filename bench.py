"""Benchmark: fwd+bwd particle-steps/s of the batched differentiable cloth MPM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload sweep|single|small] [--impl ours|reference]

Workloads (synthetic data; seeded):
  sweep   256 square cloths, side U{16..96} vertices at the 0.2 m / 31 spacing of
          the single-cloth case, E log-U[1e3, 1e5], nu U[0.1, 0.45], ground
          friction U[0.1, 0.6], own 2-corner cubic-spline grasp each, separate
          64^3 grids, dt 1e-4, 300 substeps, Chamfer to 2048 targets each,
          gradients of every instance in one pass                   (default)
          (dt is not fixed by the configuration; 1e-4 keeps the stiffest draw,
          2mu + lambda ~ 3.8e5 Pa, inside the explicit stability limit, which
          2e-4 does not)
  single  one 128x128-vertex cloth, 0.4 m, 128^3 grid, dt 1e-4, 1000 substeps,
          checkpoints every 50 substeps
  small   one 32x32-vertex cloth, 0.2 m, 64^3 grid, dt 2e-4, 200 substeps

A step is one forward rollout + Chamfer loss + full adjoint rollout.  Targets are
area-uniform samples of each cloth's rest surface (no dataset is involved).
Under torchrun every rank runs its own, differently seeded copy of the workload
(instances are independent: no collective on the data path) and the line
reports the whole-job rate from the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+bwd particle-steps/s"
UNIT = "particle-steps/s"
# Algorithmic bytes per particle of one launch (float32 state, grid traffic
# excluded), for each kernel of the substep and its adjoint: the particle
# state, rest data and per-vertex sums the kernel must read or write once.
KERNEL_BYTES = {
    "k_tri_forward": {"tri": 228},
    "k_point_p2g": {"vertex": 88},
    "k_grid": {"node": 48},
    "k_g2p": {"vertex": 84, "tri": 204},
    # vertex_fold: the triangles' per-vertex adjoint sums of the previous
    # adjoint substep, read and cleared (two float4) in every adjoint substep
    # of a rollout but its first
    "k_g2p_adj": {"vertex": 96, "vertex_fold": 64, "tri": 144},
    "k_grid_adj": {"node": 64},
    "k_point_adj": {"vertex": 156},
    "k_tri_adj": {"tri": 372},
    "k_vertex_collect": {"vertex": 112},
}
# Whole fwd+bwd substep, per particle (float32): vertex 420 B, triangle 1068 B.
STEP_BYTES = {"vertex": 420, "tri": 1068}


def workload(name, seed):
    from diffcp_b200 import configs
    if name == "sweep":
        return configs.parameter_sweep(seed)
    if name == "single":
        return configs.large_sheet(seed)
    if name == "small":
        return configs.single_sheet(seed)
    if name == "traj":
        return configs.trajectory_batch(seed)
    if name == "stress":
        return configs.stress_sheet(seed)
    raise ValueError(name)


class ClockSampler:
    """nvidia-smi clock / throttle samples while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_figure(kernel, key):
    """A per-launch figure of ``kernel`` on this workload from its committed
    ncu summary (profiles/<kernel>.md, line '<key>: X'); None when absent."""
    path = os.path.join(ROOT, "profiles", kernel + ".md")
    if not os.path.exists(path):
        return None
    m = re.search(key + r":\s*([0-9.eE+-]+)", open(path).read())
    return float(m.group(1)) if m else None


def ncu_traffic(kernel):
    """DRAM read + write bytes of one launch of ``kernel``
    ('dram_bytes_per_launch')."""
    return ncu_figure(kernel, "dram_bytes_per_launch")


def step_issue(prof, restored, ms_per_step, sm_mhz):
    """Warp instructions of one step, from the per-launch counts of the ncu
    summaries and the eager profile's launch counts, against the SMs' issue
    ceiling over the step's time.  The P2G kernels' adjoint launches that
    return at once (the tape holds their substep, ``restored`` of them) are
    not counted; kernels without a summary are left out and named."""
    import torch
    if not sm_mhz:
        return None
    inst, counted, missing = 0.0, [], []
    for name, (ms, launches) in sorted(prof.items()):
        per = ncu_figure(name, "warp_inst_per_launch")
        if per is None:
            missing.append(name)
            continue
        full = launches - (restored if name in ("k_tri_forward", "k_point_p2g") else 0)
        inst += per * max(full, 0)
        counted.append(name)
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    peak = 4.0 * sms * sm_mhz * 1e6
    achieved = inst / (ms_per_step / 1e3)
    share = sum(prof[k][0] for k in counted) / max(sum(v[0] for v in prof.values()), 1e-12)
    return {"achieved": achieved, "peak": peak, "unit": "warp instructions/s", "frac": achieved / peak,
            "warp_inst_per_step": inst, "kernels": counted, "not_counted": missing,
            "profile_share_counted": share}


def issue_ceiling(kernel, avg_launch_s, sm_mhz):
    """The kernel's instruction-issue rate against the SMs' issue ceiling (one
    warp instruction per cycle on each of an SM's 4 schedulers) at the SM
    clock sampled under load: the stencil kernels are bound by issue and
    latency, not by HBM, and this says how far from that ceiling they run.
    Warp instructions per launch come from the ncu summary
    ('warp_inst_per_launch'); None when absent."""
    import torch
    inst = ncu_figure(kernel, "warp_inst_per_launch")
    if inst is None or not sm_mhz:
        return None
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    peak = 4.0 * sms * sm_mhz * 1e6
    achieved = inst / avg_launch_s
    return {"kernel": kernel, "achieved": achieved, "peak": peak, "unit": "warp instructions/s",
            "frac": achieved / peak, "warp_inst_per_launch": inst, "sms": sms, "sm_mhz": sm_mhz}


def counts(scenes):
    nv = sum(s.n_vertex for s in scenes)
    nt = sum(s.n_tri for s in scenes)
    return nv, nt


# ------------------------------------------------------------------ CPU
def median_instance(scenes):
    sizes = [s.n_vertex + s.n_tri for s in scenes]
    i = int(np.argsort(sizes)[len(sizes) // 2])
    return i, scenes[i]


def cpu_sample(scenes, k):
    """k instances spread evenly over the workload's sizes (sorted by particle
    count), so that the sample has the workload's mix of cloth sizes."""
    order = np.argsort([s.n_vertex + s.n_tri for s in scenes], kind="stable")
    idx = sorted({int(order[int(round(j * (len(scenes) - 1) / max(k - 1, 1)))]) for j in range(k)})
    return idx


def cpu_rate(scenes, info, seconds=15.0, steps=1, warmup=0, min_substeps=20):
    """The CPU baseline: oracle/cpu_port.cpp, the compiled float32 restatement
    of the substep and its adjoint (the reference's Taichi is not installed),
    on all host cores, one OpenMP thread per cloth.  A bounded sample of the
    workload: as many cloths as threads, spread over its sizes, each timed
    step the forward rollout, Chamfer loss and reverse pass of n >=
    ``min_substeps`` substeps of each, n sized so that the timed steps take
    about ``seconds``."""
    from oracle import cpu_port
    threads = os.cpu_count() or 1
    idx = cpu_sample(scenes, min(threads, len(scenes)))
    sample = [scenes[i] for i in idx]
    parts = sum(s.n_vertex + s.n_tri for s in sample)
    cpu_port.rollouts(sample, 2, threads)              # set-up, first touch, thread pool
    t0 = time.perf_counter()
    cpu_port.rollouts(sample, 2, threads)
    per = (time.perf_counter() - t0) / 2
    n = int(max(min_substeps, min(info["n_steps"], seconds / max(steps, 1) / max(per, 1e-4))))
    for _ in range(warmup):
        cpu_port.rollouts(sample, 2, threads)
    el = 0.0
    k = max(steps, 1)
    for _ in range(k):
        t0 = time.perf_counter()
        cpu_port.rollouts(sample, n, threads)
        el += time.perf_counter() - t0
    rate = parts * n * k / el
    return {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "ms_per_step": 1e3 * el / k,
            "instances": idx, "substeps_per_step": n,
            "sample": "compiled float32 CPU restatement of the substep and its adjoint (oracle/cpu_port.cpp; the "
                      "reference's Taichi is not installed), %d threads, one cloth each: %d cloths of the workload "
                      "spread over its sizes (%d particles), fwd+bwd of %d substeps per step, %d timed step(s) in "
                      "%.1f s" % (threads, len(sample), parts, n, k, el)}


def workload_config(scenes, info, world=1):
    """The `config` of the JSON line, the same for both arms: what the
    workload is, not how a run executed it."""
    from diffcp_b200.batch import POINT_STATE, TRI_STATE
    nv, nt = counts(scenes)
    state_floats = POINT_STATE * nv + TRI_STATE * nt
    return {"workload": info["desc"], "instances": len(scenes), "vertices": nv, "triangles": nt,
            "substeps": info["n_steps"], "checkpoint_every": info["ckpt_every"],
            "l2": "inputs larger than L2 (one state snapshot is %.0f MB; every substep reads its own)"
                  % (state_floats * 4 / 1e6),
            "parallelism": "independent instances per rank" if world > 1 else "one GPU"}


def profile_substeps(args):
    """Two eager rollouts of ``args.profile_substeps`` substeps of the workload
    (or of its first ``args.profile_instances`` instances) with forward,
    Chamfer and adjoint, through the same path as the bench: the first sizes
    the grid tape, the second records into it and the adjoint reads it.  A few
    GB on the device at most; for kernel profilers.  Launch order of the second
    rollout, per substep: forward k_tri_forward, k_point_p2g, k_tape_reserve,
    k_grid, k_g2p (points, then triangles); adjoint k_tri_forward and
    k_point_p2g (both return at once), k_grid, k_g2p_adj, k_grid_adj,
    k_point_adj, k_tri_adj (and k_vertex_collect after substep 0)."""
    import torch
    from diffcp_b200 import autotune
    from diffcp_b200.batch import BatchSim, ClothBatch
    scenes, info = workload(args.workload, 0)
    cache = args.tune_cache or autotune.CACHE
    # the launch configuration tuned for the whole workload, also on a slice of it
    launch = (autotune.cached(scenes, info["dt"], cache=cache) if os.path.exists(cache) else None) or autotune.DEFAULT
    if args.profile_instances:
        scenes = scenes[: args.profile_instances]
    b = ClothBatch(scenes, dt=info["dt"], **autotune.batch_kwargs(launch))
    n = args.profile_substeps
    sim = BatchSim(b, n_steps=n, ckpt_every=1, use_graph=False, tape="auto")
    for _ in range(2):
        params = b.params.clone().requires_grad_(True)
        traj = b.traj.clone().requires_grad_(True)
        sim.loss(params, traj).sum().backward()
    torch.cuda.synchronize()
    st = b.status()
    print(json.dumps({"profile_substeps": n, "instances": len(scenes), "finite": bool(torch.isfinite(params.grad).all()),
                      "status_nonzero": int((st != 0).sum())}))


# ------------------------------------------------------------------ main
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="sweep", choices=["sweep", "single", "small", "traj", "stress"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--profile-substeps", type=int, default=0,
                    help="run this many eager forward + adjoint substeps of the workload and exit (for ncu)")
    ap.add_argument("--profile-instances", type=int, default=0,
                    help="with --profile-substeps: only the first this many instances of the workload")
    ap.add_argument("--tune", action="store_true", help="autotune the launch configuration before timing")
    ap.add_argument("--tune-cache", default=None, help="autotuner cache file (default diffcp_b200/tuned.json)")
    ap.add_argument("--no-single", action="store_true", help="skip the single-instance plain-launch measurement")
    ap.add_argument("--no-tape", action="store_true",
                    help="recompute particle-to-grid in every adjoint substep instead of restoring it from the grid tape")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))

    if args.impl == "reference":
        if rank != 0:
            return
        scenes, info = workload(args.workload, 0)
        cb = cpu_rate(scenes, info, seconds=max(args.cpu_seconds, 5.0), steps=args.steps, warmup=args.warmup)
        line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
                "config": workload_config(scenes, info, args.gpus), "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    if args.profile_substeps:
        return profile_substeps(args)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    dev = torch.device("cuda", torch.cuda.current_device())
    from diffcp_b200.batch import BatchSim, ClothBatch

    from diffcp_b200 import autotune
    scenes, info = workload(args.workload, rank)
    nv, nt = counts(scenes)
    cache = args.tune_cache or autotune.CACHE
    if args.tune:
        launch = autotune.tune(scenes, info["dt"], device=dev, cache=cache, force=True)
    else:
        launch = autotune.cached(scenes, info["dt"], cache=cache) if os.path.exists(cache) else None
        launch = launch or dict(autotune.DEFAULT, source="default")
    batch = ClothBatch(scenes, dt=info["dt"], device=dev, pool_blocks=info.get("pool_blocks", 0),
                       **autotune.batch_kwargs(launch))
    tape = None if args.no_tape else "auto"
    sim = BatchSim(batch, n_steps=info["n_steps"], ckpt_every=info["ckpt_every"], use_graph=True, tape=tape)
    params = batch.params.clone().requires_grad_(True)
    traj = batch.traj.clone().requires_grad_(True)

    def step():
        params.grad = None
        traj.grad = None
        loss = sim.loss(params, traj)
        loss.sum().backward()
        return loss

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    for _ in range(max(args.warmup, 3) if args.warmup >= 0 else 3):
        step()
    torch.cuda.synchronize()
    status = batch.status()
    launches0 = batch.launch_count()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1) / args.steps
    launches = (batch.launch_count() - launches0) // max(args.steps, 1)
    from diffcp_b200 import sharding
    ms_max = sharding.max_over_ranks(ms, device=dev)
    psteps = (nv + nt) * info["n_steps"]
    # every rank simulates its own workload copy: the job's units are the sum over ranks
    units = torch.tensor([float(psteps)], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(units)
    job_psteps = float(units.item())
    value = job_psteps / (ms_max / 1e3)

    # ---- e2e: public API with host buffers (pinned H2D of the inputs, D2H of loss and gradients)
    h_params = params.detach().cpu().pin_memory()
    h_traj = traj.detach().cpu().pin_memory()
    h_targets = batch.targets.cpu().pin_memory()
    h_loss = torch.empty(batch.n_inst, dtype=torch.float32).pin_memory()
    h_gp = torch.empty_like(h_params).pin_memory()
    h_gt = torch.empty_like(h_traj).pin_memory()
    d_params = params.detach().clone().requires_grad_(True)
    d_traj = traj.detach().clone().requires_grad_(True)

    def e2e_step():
        with torch.no_grad():
            d_params.copy_(h_params, non_blocking=True)
            d_traj.copy_(h_traj, non_blocking=True)
            batch.targets.copy_(h_targets, non_blocking=True)
        d_params.grad = None
        d_traj.grad = None
        loss = sim.loss(d_params, d_traj)
        loss.sum().backward()
        h_loss.copy_(loss.detach(), non_blocking=True)
        h_gp.copy_(d_params.grad, non_blocking=True)
        h_gt.copy_(d_traj.grad, non_blocking=True)

    e2e_step()
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1) / args.steps
    ms_e2e_max = sharding.max_over_ranks(ms_e2e, device=dev)
    e2e_val = job_psteps / (ms_e2e_max / 1e3)
    h2d = (h_params.numel() + h_traj.numel() + h_targets.numel()) * 4
    d2h = (h_loss.numel() + h_gp.numel() + h_gt.numel()) * 4

    # ---- per-kernel device time of one eager step (CUDA events on the launch stream)
    batch.profile(True)
    sim.use_graph = False
    step()
    torch.cuda.synchronize()
    prof = batch.profile_read()
    # particle order kept from the start of the rollout: do the forward
    # scatters slow down as the cloth moves away from its initial Morton order?
    order_drift = {}
    for name in ("k_tri_forward", "k_point_p2g"):
        t = batch.profile_launches(name)[: info["n_steps"]]    # the forward rollout, substeps 0 .. n-1
        if len(t) >= 60:
            order_drift[name] = {"first30_ms": float(np.mean(t[:30])), "last30_ms": float(np.mean(t[-30:])),
                                 "last_over_first": float(np.mean(t[-30:]) / np.mean(t[:30]))}
    batch.profile(False)
    sim.use_graph = True
    n_nodes_active = None
    units = {"tri": nt, "vertex": nv, "corner": 3 * nt,
             "vertex_fold": nv * (info["n_steps"] - 1) / info["n_steps"]}
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dname, (dms, dn) = dom
    per_unit = KERNEL_BYTES.get(dname, {})
    alg = sum(units.get(u, 0) * b for u, b in per_unit.items())
    avg_s = dms / dn / 1e3
    peak, peak_kind = peaks()
    achieved = alg / avg_s / 1e9 if alg else None
    traffic = ncu_traffic(dname) if args.workload == "sweep" else None
    roof = {"bound": "hbm", "kernel": dname, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback", "traffic": traffic, "alg_bytes_per_launch": alg,
            "avg_launch_ms": dms / dn, "launches_in_profile_step": dn}
    total_prof_ms = sum(v[0] for v in prof.values())
    step_alg = (nv * STEP_BYTES["vertex"] + nt * STEP_BYTES["tri"]) * info["n_steps"]
    kernels = {k: {"ms": round(v[0], 3), "launches": v[1], "share": round(v[0] / total_prof_ms, 4)}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])}

    # ---- the same work as single instances with plain per-kernel launches (no CUDA graph)
    single = None
    if not args.no_single and len(scenes) > 1:
        _, sc1 = median_instance(scenes)
        b1 = ClothBatch([sc1], dt=info["dt"], device=dev, **autotune.batch_kwargs(launch))
        sim1 = BatchSim(b1, n_steps=info["n_steps"], ckpt_every=info["ckpt_every"], use_graph=False, tape=tape)
        p1 = b1.params.clone().requires_grad_(True)
        t1 = b1.traj.clone().requires_grad_(True)
        sim1.loss(p1, t1).sum().backward()
        torch.cuda.synchronize()
        e0.record(stream)
        sim1.loss(p1, t1).sum().backward()
        e1.record(stream)
        torch.cuda.synchronize()
        ms1 = e0.elapsed_time(e1)
        single = {"value": (sc1.n_vertex + sc1.n_tri) * info["n_steps"] / (ms1 / 1e3), "unit": UNIT,
                  "ms_per_step": ms1, "instance": "%d vertices + %d triangles (median instance)" % (
                      sc1.n_vertex, sc1.n_tri), "launches": "per-kernel launches, no CUDA graph"}
        del sim1, b1

    tape_info = None
    if sim._tape is not None:
        meta = ClothBatch.tape_blocks(sim._tape, info["n_steps"])
        tape_info = {"bytes": int(sim._tape.numel()), "substeps_restored": int((meta[:, 0] >= 0).sum()),
                     "active_blocks_per_substep": float(meta[:, 1].mean()),
                     "max_active_blocks": int(meta[:, 1].max())}
    grid_info = {"layout": "paged" if batch.pool_blocks else "dense", "pool_blocks": batch.pool_blocks,
                 "dense_blocks": int(batch.sizes.total_nodes) // 64,
                 "grid_bytes": 3 * 16 * 64 * int(batch.sizes.grid_blocks)}
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    cpu = None if args.no_cpu or world > 1 else cpu_rate(scenes, info, seconds=args.cpu_seconds)
    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(scenes, info, world),
        "run": {"launch": launch, "grid": grid_info, "grid_tape": tape_info,
                "rollout_buffer_gb": sim._buf.numel() * 4 / 1e9,
                "peak_device_bytes": int(torch.cuda.max_memory_allocated(dev))},
        "roofline": roof,
        "issue_roofline": issue_ceiling(dname, dms / dn / 1e3, clocks.get("sm_mhz")),
        "step_issue_roofline": step_issue(prof, tape_info["substeps_restored"] if tape_info else 0, ms_max,
                                          clocks.get("sm_mhz")),
        "step_roofline": {"achieved": step_alg / (ms_max / 1e3) / 1e9, "unit": "GB/s", "peak": peak,
                          "frac": step_alg / (ms_max / 1e3) / 1e9 / peak,
                          "bytes_per_particle": STEP_BYTES},
        "kernels": kernels,
        "order_drift": order_drift,
        "cpu_baseline": cpu,
        "single_instance": single,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": ms_e2e_max},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "status_nonzero_instances": int((status != 0).sum()),
        "nonfinite_instances": int(((status & 2) != 0).sum()),
    }
    print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
