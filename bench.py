#!/usr/bin/env python
"""bench.py — steps/s of the learned-theta Barnes-Hut walk against the plain
fixed-theta walk at equal RMS force error, N = 1,048,576 disk galaxy, 1 B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Workload: exponential disk (R_d 1, sech^2 z0 0.1, 80% of the mass) +
Hernquist bulge (a 0.2, 20%), N = 1,048,576, seed 1, eps 0.005, dt 5e-4,
21 Morton bits per axis, leaf 1, groups of 32.  A step is the whole
pipeline: bounding box, Morton keys, radix sort, reorder, octree + upward
pass, (learned criterion: group features + per-group budget choice), walk +
kick-drift.

Equal error: the RMS relative force error against the FP64 direct sum
(bh_direct_sum_f64 on 65,536 sampled bodies) is 1e-3 for both walks.  Before
timing, the learned walk's error target and the plain walk's theta are
calibrated on this workload (secant steps in log-log space) to the largest
value whose measured RMS error is at most 1e-3; the error is measured again
after the timed steps.

Engine arm: W untimed steps, then K steps timed one by one with CUDA events
on the simulation's stream, an L2 flush (a 512 MiB write, larger than the
126 MB L2) before each.  `value` = learned-walk steps/s over all ranks
(replicas: each GPU steps its own copy; no collective on the data path).
`plain_equal_error` = the fixed-theta walk timed the same way at its
calibrated theta, `speedup_vs_plain` their ratio.  `e2e` = the learned walk
through the C ABI's host-buffer step (bh_sim_step_host: pinned host arrays
copied in, one step, results copied back, every step).  `roofline`: the walk
kernel, the dominant one, against the measured FP32 FMA throughput (20 flops
per body-node interaction).  `cpu_baseline`: the C oracle (the reference
algorithm restated, OpenMP over the host cores) at the plain walk's
equal-error theta, two whole steps of the same workload (no sampling).

Reference arm (--impl reference): the reference's algorithm (fixed theta, at
the theta that gives RMS 1e-3 on this workload) on the host cores — the
reference ships no CPU implementation of the path, so the oracle port stands
for it — W + K whole steps of the same workload; plus, under
"reference_cuda", the reference's own CUDA build run on this GPU for W + K
steps at the same theta.  That process loads only the oracle's libraries.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORK = dict(n=1 << 20, seed=1, eps=0.005, dt=5e-4, bits=21, G=1.0, theta_cap=0.9, rms_target=1e-3)
# The fixed theta at which the plain walk's RMS relative force error on this
# workload is 1e-3 (the engine arm's calibration lands on 0.2386, RMS 9.8e-4;
# the engine arm recalibrates it on every run, the reference arm uses this
# value for the reference's method on the host cores and on this GPU).
PLAIN_THETA_EQUAL_ERROR = 0.2386
ERR_SAMPLE = 65536
METRIC = "steps/s @N=1M disk, learned-\u03b8 vs plain BH on 1 B200 at equal RMS force err"
WORKLOAD = ("learned-theta Barnes-Hut at RMS relative force error 1e-3 vs FP64 direct sum, "
            "disk galaxy N=1,048,576")
REF_WORKLOAD = ("fixed-theta Barnes-Hut (the reference's method) at RMS relative force error 1e-3 vs FP64 "
                "direct sum, disk galaxy N=1,048,576")
FLOPS_PER_INTERACTION = 20
CPU_BASELINE_STEPS = 2  # full CPU steps timed for the engine arm's cpu_baseline
# DRAM bytes of one k_walk launch per body, from an ncu capture of the learned
# walk on the 262,144-body disk (22.0 MB read, nothing written back within the
# launch); the walk's traffic grows in proportion to the bodies it processes.
WALK_DRAM_BYTES_PER_BODY = 22.021632e6 / 262144


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--n", "--bodies", dest="n", type=int, default=WORK["n"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-drift", action="store_true", help="skip the FP64 energy-drift check")
    ap.add_argument("--no-configs", action="store_true",
                    help="disk workload: skip the batch (256 systems) and merger (N=4M) sub-results")
    ap.add_argument("--sizes", default="1048576,4194304,16777216", help="body counts of --workload stages")
    ap.add_argument("--workload", choices=["disk", "batch", "merger", "stages"], default="disk",
                    help="disk: the headline (learned vs plain at equal error); batch: 256 uneven Plummer "
                         "systems in one simulation; merger: two-disk merger at N=4,194,304, learned walk; "
                         "stages: achieved bandwidth of the memory-bound stages at N = 1M, 4M, 16M")
    return ap.parse_args()


# ----------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self) -> dict:
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------ distributed
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist_mod.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        dist = dist_mod
    return world, rank, local, dist


def max_over_ranks(x: float, dist, device) -> float:
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------- baselines
def cpu_steps(pos, vel, theta: float, steps: int, warmup: int = 0) -> dict:
    """Whole reference steps of the oracle port on the host cores (bounding
    box, keys, sort, reorder, level-wise tree, the full group walk at fixed
    theta — every group, no sampling — and kick-drift, oracle/bh_oracle.c
    orc_step), advancing copies of (pos, vel); `warmup` untimed steps first.
    Returns the mean wall time per timed step."""
    from oracle import cpu
    p, v = pos.copy(), vel.copy()
    for _ in range(warmup):
        cpu.step(p, v, WORK["bits"], WORK["eps"], WORK["G"], theta, WORK["dt"])
    times, inter = [], 0
    for _ in range(steps):
        t0 = time.perf_counter()
        _, _, _, inter = cpu.step(p, v, WORK["bits"], WORK["eps"], WORK["G"], theta, WORK["dt"])
        times.append(time.perf_counter() - t0)
    return {"step_s": sum(times) / len(times), "times_s": times, "interactions_per_step": inter,
            "cores": cpu.num_threads(),
            "sample": f"{steps} whole steps (box, keys, sort, reorder, tree, walk of every group at fixed theta "
                      f"{theta}, kick-drift) of the N={pos.shape[0]} disk, after {warmup} untimed"}


# -------------------------------------------------------------- calibration
def rms_error(sim, pos, vel, steps: int = 2) -> float:
    """RMS relative force error of the walk after `steps` steps from the
    initial state (the first step bootstraps |a| for the relative walks)."""
    from cudagravitydemo_b200.accuracy import force_error
    sim.load(pos, vel)
    sim.step(steps)
    return force_error(sim, ERR_SAMPLE)["rms"]


def calibrate(sim, pos, vel, params_at, x0: float, target: float, iters: int = 7):
    """Largest x (error grows with x) whose RMS error is at most target:
    secant steps on log(rms) against log(x), kept inside the bracket."""
    lo = hi = None  # (x, rms) with rms <= target / > target
    pts = []
    x = x0
    for _ in range(iters):
        sim.set_params(params_at(x))
        e = rms_error(sim, pos, vel)
        pts.append((x, e))
        if e <= target:
            lo = (x, e) if lo is None or x > lo[0] else lo
            if e >= 0.97 * target:
                break
        else:
            hi = (x, e) if hi is None or x < hi[0] else hi
        if len(pts) >= 2 and pts[-1][1] != pts[-2][1] and pts[-1][0] != pts[-2][0]:
            (x1, e1), (x2, e2) = pts[-2], pts[-1]
            slope = math.log(e2 / e1) / math.log(x2 / x1)
            slope = min(max(slope, 0.3), 5.0)
        else:
            slope = 1.0
        nx = x * math.exp(math.log(0.985 * target / e) / slope)
        if lo and nx <= lo[0]:
            nx = lo[0] * 1.02 if hi is None else math.sqrt(lo[0] * hi[0])
        if hi and nx >= hi[0]:
            nx = hi[0] / 1.05 if lo is None else math.sqrt(lo[0] * hi[0])
        x = nx
    if lo is None:
        raise RuntimeError(f"calibration did not reach RMS {target}: {pts}")
    return lo[0], lo[1], pts


# ------------------------------------------------------------------ timing
def timed_steps(sim, stream, flush, steps: int, warmup: int, dist, clk=None, label: str | None = None):
    """ms of each of `steps` steps (one graph replay each), L2 flushed
    before each, after `warmup` untimed steps.  `label` names an NVTX range
    around the timed steps (a profiler can select them by it)."""
    import torch
    sim.step(warmup)
    stream.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clk:
        clk.__enter__()
    if label:
        torch.cuda.nvtx.range_push(label)
    with torch.cuda.stream(stream):
        for k in range(steps):
            flush.zero_()
            starts[k].record(stream)
            sim.step(1)
            ends[k].record(stream)
    stream.synchronize()
    if label:
        torch.cuda.nvtx.range_pop()
    if clk:
        clk.__exit__(None, None, None)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    return [a.elapsed_time(b) for a, b in zip(starts, ends)]


# ------------------------------------------------------------------ arms
def engine_arm(args, world, rank, local, dist):
    import torch

    import cudagravitydemo_b200 as bh
    from cudagravitydemo_b200.accuracy import force_error
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    n = args.n
    pos, vel = bh.disk_galaxy(n, seed=WORK["seed"])
    base = dict(bits_per_axis=WORK["bits"], eps=WORK["eps"], G=WORK["G"], dt=WORK["dt"])
    learned_at = lambda t: bh.Params(theta=WORK["theta_cap"], mac_mode=2, err_target=t, **base)  # noqa: E731
    plain_at = lambda th: bh.Params(theta=th, **base)  # noqa: E731
    sim = bh.Simulation(n, learned_at(1.2e-3))
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=device)

    # calibration to the equal-error point (untimed)
    tgt, rms_l, pts_l = calibrate(sim, pos, vel, learned_at, 1.2e-3, WORK["rms_target"])
    th, rms_p, pts_p = calibrate(sim, pos, vel, plain_at, PLAIN_THETA_EQUAL_ERROR, WORK["rms_target"])

    # learned walk: the headline
    sim.set_params(learned_at(tgt))
    sim.load(pos, vel)
    clk = ClockSampler(local)
    ms_l = timed_steps(sim, stream, flush, args.steps, args.warmup, dist, clk, label="bench_learned_timed")
    rms_l_end = force_error(sim, ERR_SAMPLE)["rms"]
    stats_l = sim.stats()
    total_l = max_over_ranks(sum(ms_l), dist, device)
    value = world * args.steps / (total_l * 1e-3)
    stages = sim.profile(3)
    stats_p3 = sim.stats()
    peak = bh.fma_peak_tflops(5)
    walk_s = stages["walk"] * 1e-3
    achieved = stats_p3["interactions"] * FLOPS_PER_INTERACTION / walk_s / 1e12
    launches = sim.kernels_per_step() * args.steps

    e2e = None
    e2e_id = None
    if not args.no_e2e:
        # end to end through the C ABI: pinned host arrays in, one step, the
        # state back in host memory, every step.  The headline call returns it
        # in the step's Morton order with body ids (the reference's frame
        # order; the walk writes the pinned arrays itself); the id-order call
        # (bh_sim_step_host) scatters back to body-id order and copies after
        # the walk.
        hp_t = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
        hv_t = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        hi_t = torch.empty((n,), dtype=torch.int32, pin_memory=True)
        hp, hv, hi = hp_t.numpy(), hv_t.numpy(), hi_t.numpy().view(np.uint32)

        def e2e_run(call):
            sim.load(pos, vel)
            hp[:] = pos
            hv[:] = vel
            hi[:] = np.arange(n, dtype=np.uint32)
            for _ in range(max(3, args.warmup)):  # the first also bootstraps |a|
                call()
            e_ms = []
            for _ in range(args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                call()
                e1.record(stream)
                e1.synchronize()
                e_ms.append(e0.elapsed_time(e1))
            return max_over_ranks(sum(e_ms), dist, device)

        e_total = e2e_run(lambda: sim.step_host_sorted(hp, hv, hi, 1))
        e2e = {"value": world * args.steps / (e_total * 1e-3), "unit": "steps/s",
               "h2d_bytes_per_step": n * (16 + 12 + 4), "d2h_bytes_per_step": n * (16 + 12 + 4),
               "ms_per_step": e_total / args.steps,
               "call": "bh_sim_step_host_sorted (learned walk; pinned pos/vel/ids in, state after the step out "
                       "in its Morton order with ids, written by the walk into the pinned arrays)"}
        i_total = e2e_run(lambda: sim.step_host(hp, hv, 1))
        e2e_id = {"value": world * args.steps / (i_total * 1e-3), "unit": "steps/s",
                  "h2d_bytes_per_step": n * (16 + 12), "d2h_bytes_per_step": n * (16 + 12),
                  "ms_per_step": i_total / args.steps,
                  "call": "bh_sim_step_host (learned walk; pinned pos/vel in and out in body-id order)"}

    # FP64 energy / momentum drift of the learned walk over 1000 steps (untimed)
    drift = None
    if not args.no_drift:
        sim.load(pos, vel)
        d0 = sim.diagnostics()
        sim.step(1000)
        d1 = sim.diagnostics()
        drift = {"steps": 1000, "walk": "learned", "energy_rel": (d1["total"] - d0["total"]) / abs(d0["total"]),
                 "momentum_abs": float(np.linalg.norm(np.array(d1["momentum"]) - np.array(d0["momentum"]))),
                 "E0": d0["total"], "note": "FP64 kinetic + exact pair-sum potential (bh_sim_diagnostics)"}

    # plain fixed-theta walk at the same RMS error, and at the reference's theta 0.5
    sim.set_params(plain_at(th))
    sim.load(pos, vel)
    ms_p = timed_steps(sim, stream, flush, args.steps, args.warmup, dist)
    rms_p_end = force_error(sim, ERR_SAMPLE)["rms"]
    stats_pe = sim.stats()
    total_p = max_over_ranks(sum(ms_p), dist, device)
    plain_value = world * args.steps / (total_p * 1e-3)
    sim.set_params(plain_at(0.5))
    sim.load(pos, vel)
    ms_5 = timed_steps(sim, stream, flush, args.steps, args.warmup, dist)
    rms_5 = force_error(sim, ERR_SAMPLE)["rms"]
    total_5 = max_over_ranks(sum(ms_5), dist, device)
    launches += sim.kernels_per_step() * 2 * args.steps  # plain kernels per step are the same at both thetas

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_steps(pos, vel, round(th, 4), CPU_BASELINE_STEPS)
        cpu = {"value": 1.0 / cb["step_s"], "unit": "steps/s", "cores": cb["cores"], "kind": "port",
               "sample": cb["sample"], "step_s": cb["step_s"]}

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_l / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded disk + bulge, seed 1)",
        "config": {"workload": WORKLOAD, "variant": "learned", "n_bodies": n, "rms_target": WORK["rms_target"],
                   "err_target": tgt, "theta_cap": WORK["theta_cap"], "eps": WORK["eps"], "dt": WORK["dt"],
                   "bits_per_axis": WORK["bits"], "group_width": 32, "leaf_size": 1, "compensated_sums": True,
                   "parallelism": f"replicas x{world}", "l2": "flushed before every timed step (512 MiB write)",
                   "error_sample": ERR_SAMPLE},
        "rms_error": {"calibrated": rms_l, "after_timed_steps": rms_l_end, "calibration": pts_l},
        "plain_equal_error": {"value": plain_value, "unit": "steps/s", "theta": th, "rms_calibrated": rms_p,
                              "rms_after_timed_steps": rms_p_end, "ms_per_step": total_p / args.steps,
                              "interactions_per_step": stats_pe["interactions"], "calibration": pts_p},
        "speedup_vs_plain": value / plain_value,
        "plain_theta_0_5": {"value": world * args.steps / (total_5 * 1e-3), "unit": "steps/s", "rms": rms_5,
                            "ms_per_step": total_5 / args.steps},
        "interactions_per_step": stats_l["interactions"],
        "interactions_per_s": stats_l["interactions"] * value,
        "nodes": stats_l["node_count"], "deepest_level": stats_l["deepest_level"],
        "stages_ms": stages,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": WALK_DRAM_BYTES_PER_BODY * n,
                     "traffic_note": "ncu dram read+write of k_walk at 262,144 bodies, scaled by body count",
                     "kernel": "k_walk (fused walk + kick-drift, learned criterion)",
                     "note": "20 flops per body-node interaction; peak = measured FMA-probe throughput"},
        "energy_drift": drift,
        "e2e": e2e, "e2e_id_order": e2e_id, "cpu_baseline": cpu, "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    line["stages_roofline"] = stage_roofline(stages, n, stats_l["node_count"], (3 * WORK["bits"] + 7) // 8)
    sim.close()
    if not args.no_configs:
        # the other measured configurations, each with its own timed region:
        # 256 uneven Plummer systems in one batched simulation, and the
        # N = 4,194,304 two-disk merger with the learned walk at RMS 1e-3
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup = min(args.steps, 10), max(3, min(args.warmup, 5))
        keep = ("metric", "value", "unit", "steps", "warmup", "ms_per_step", "config", "rms_error",
                "interactions_per_step", "interactions_per_s", "energy_drift", "gpu_launches", "clocks",
                "autotune_ms_per_step", "stages_ms")
        b = batch_arm(sub, world, rank, local, dist)
        line["config4_batch"] = {k: b[k] for k in keep if k in b}
        m = merger_arm(sub, world, rank, local, dist)
        line["config5_merger"] = {k: m[k] for k in keep if k in m}
    return line


def hbm_peak_gbs() -> tuple[float, str]:
    try:
        return float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"  # an earlier copy-bandwidth measurement on this pool


def stage_roofline(stages: dict, n: int, m: int, npass: int) -> dict:
    """Memory-bound stages of one step against the HBM copy bandwidth:
    algorithmic bytes (STAGE_BYTES) / event-timed stage time.  At N = 1M
    every array fits the 126 MB L2, so these stages are bound by latency, not
    by HBM; the fractions say how far from the HBM bound they are."""
    hbm, src = hbm_peak_gbs()
    out = {"peak_gbs": hbm, "peak": src}
    for k, fn in STAGE_BYTES.items():
        ms = stages[k]
        gb = fn(n, m, npass) / 1e9
        out[k] = {"ms": ms, "algorithmic_GB": gb, "GB_per_s": gb / (ms * 1e-3), "frac": gb / (ms * 1e-3) / hbm}
    return out


def batch_arm(args, world, rank, local, dist):
    """256 independent Plummer spheres (N log-uniform in [1024, 65536], seed 2;
    sphere k from seed 2000 + k), eps 0.01, dt 1e-3, theta 0.5, one batched
    simulation: bucket size autotuned, K graph-replayed steps timed with an
    L2 flush before each; per-system FP64 energy drift over 500 steps."""
    import torch

    import cudagravitydemo_b200 as bh
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    rng = np.random.default_rng(2)
    counts = np.exp(rng.uniform(np.log(1024), np.log(65536), 256)).astype(np.int32)
    ps, vs = zip(*[bh.plummer(int(c), seed=2000 + k) for k, c in enumerate(counts)])
    pos, vel = np.concatenate(ps), np.concatenate(vs)
    prm = bh.Params(theta=0.5, eps=0.01, G=1.0, dt=1e-3)
    sim = bh.Simulation(0, prm, counts=counts)
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=device)
    sim.load(pos, vel)
    sim.step(2)
    tune = sim.tune(5)
    sim.load(pos, vel)
    clk = ClockSampler(local)
    ms = timed_steps(sim, stream, flush, args.steps, args.warmup, dist, clk, label="bench_batch_timed")
    st = sim.stats()
    total = max_over_ranks(sum(ms), dist, device)
    value = world * args.steps / (total * 1e-3)
    stages = sim.profile(3)
    launches = sim.kernels_per_step() * args.steps
    drift = None
    if not args.no_drift:
        sim.load(pos, vel)
        d0 = sim.system_diagnostics()
        sim.step(500)
        d1 = sim.system_diagnostics()
        dr = np.array([abs(b["total"] - a["total"]) / abs(a["total"]) for a, b in zip(d0, d1)])
        big = counts >= np.median(counts)
        drift = {"steps": 500, "median": float(np.median(dr)), "p90": float(np.quantile(dr, 0.9)),
                 "max": float(dr.max()), "max_larger_half": float(dr[big].max()),
                 "max_smaller_half": float(dr[~big].max())}
    line = {
        "metric": "steps/s, 256 uneven Plummer systems in one batched simulation", "value": value,
        "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (256 seeded Plummer spheres)",
        "config": {"workload": "256 Plummer spheres, N log-uniform in [1024, 65536] (seed 2), theta 0.5, eps 0.01, "
                               "dt 1e-3", "n_bodies": int(counts.sum()), "systems": 256,
                   "leaf_size": tune["leaf_size"], "group_width": tune["group_width"],
                   "walk_stack_entries": tune["stack_entries"],
                   "l2": "flushed before every timed step (512 MiB write)"},
        "autotune_ms_per_step": {f"leaf{l}_width{w}_stack{d}": v for (l, w, d), v in tune["ms_per_step"].items()},
        "interactions_per_step": st["interactions"], "interactions_per_s": st["interactions"] * value,
        "stages_ms": stages, "energy_drift": drift, "gpu_launches": launches, "clocks": clk.summary(),
    }
    sim.close()
    return line


def merger_arm(args, world, rank, local, dist):
    """Two disk galaxies (N = 4,194,304, separation 20, pericentre 2, one disk
    inclined 30 degrees, seed 3), learned walk calibrated to RMS force error
    1e-3, eps 0.005, dt 5e-4; K timed steps; FP64 energy drift over 1000."""
    import torch

    import cudagravitydemo_b200 as bh
    from cudagravitydemo_b200.accuracy import force_error
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    n = 1 << 22
    pos, vel = bh.merger(n, seed=3)
    learned_at = lambda t: bh.Params(theta=WORK["theta_cap"], eps=0.005, G=1.0, dt=5e-4, mac_mode=2,  # noqa: E731
                                     err_target=t)
    sim = bh.Simulation(n, learned_at(1.2e-3))
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=device)
    tgt, rms, pts = calibrate(sim, pos, vel, learned_at, 1.2e-3, WORK["rms_target"])
    sim.set_params(learned_at(tgt))
    sim.load(pos, vel)
    clk = ClockSampler(local)
    ms = timed_steps(sim, stream, flush, args.steps, args.warmup, dist, clk, label="bench_merger_timed")
    rms_end = force_error(sim, ERR_SAMPLE)["rms"]
    st = sim.stats()
    total = max_over_ranks(sum(ms), dist, device)
    value = world * args.steps / (total * 1e-3)
    stages = sim.profile(3)
    launches = sim.kernels_per_step() * args.steps
    drift = None
    if not args.no_drift:
        sim.load(pos, vel)
        d0 = sim.diagnostics()
        sim.step(1000)
        d1 = sim.diagnostics()
        drift = {"steps": 1000, "energy_rel": (d1["total"] - d0["total"]) / abs(d0["total"]),
                 "momentum_abs": float(np.linalg.norm(np.array(d1["momentum"]) - np.array(d0["momentum"])))}
    line = {
        "metric": "steps/s, two-disk merger N=4,194,304, learned walk at RMS force error 1e-3", "value": value,
        "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded two-disk merger, seed 3)",
        "config": {"workload": "two-disk merger N=4,194,304, learned walk at RMS 1e-3", "err_target": tgt,
                   "theta_cap": WORK["theta_cap"], "eps": 0.005, "dt": 5e-4,
                   "l2": "flushed before every timed step (512 MiB write)"},
        "rms_error": {"calibrated": rms, "after_timed_steps": rms_end, "calibration": pts},
        "interactions_per_step": st["interactions"], "interactions_per_s": st["interactions"] * value,
        "stages_ms": stages, "energy_drift": drift, "gpu_launches": launches, "clocks": clk.summary(),
    }
    sim.close()
    return line


# Algorithmic bytes of the memory-bound stages (what each must move at least):
#   keys    bbox reads pos (16 B), Morton reads pos (16 B) and writes the key (8 B)
#   sort    per 8-bit pass: key + value read and written (24 B; the first pass
#           reads no values: 20 B)
#   reorder perm (4 B) + gathered pos, vel, id (32 B) + written pos, vel, id (32 B)
#   tree    per body: keys read by the count and node passes (16 B), the delta byte
#           written and read (2 B), pos and first-body index read by the leaves (20 B);
#           per node: child start and size, parent, first body, level/slot written
#           (20 B), and in the upward pass its child range read (8 B), its centre of
#           mass and count read by its parent (20 B), and mass, end, counts written (28 B)
STAGE_BYTES = {
    "keys": lambda n, m, npass: 40 * n,
    "sort": lambda n, m, npass: (24 * npass - 4) * n,
    "reorder": lambda n, m, npass: 68 * n,
    "tree": lambda n, m, npass: 38 * n + 76 * m,
}


def stages_arm(args, world, rank, local, dist):
    """Stage times (events between stages, plain theta 0.5 on the seeded disk)
    and the bandwidth they achieve on their algorithmic bytes, by default at
    N = 1M (every array fits the 126 MB L2), 4M and 16M (HBM-resident)."""
    import torch

    import cudagravitydemo_b200 as bh
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    hbm, _ = hbm_peak_gbs()
    out = []
    for n in [int(x) for x in args.sizes.split(",")]:
        pos, vel = bh.disk_galaxy(n, seed=WORK["seed"])
        sim = bh.Simulation(n, bh.Params(theta=0.5, eps=WORK["eps"], dt=WORK["dt"]))
        sim.load(pos, vel)
        sim.step(3)
        st = [sim.profile(5) for _ in range(3)]
        prof = {k: min(x[k] for x in st) for k in st[0]}
        m = sim.stats()["node_count"]
        npass = (3 * WORK["bits"] + 7) // 8
        row = {"n": n, "nodes": m}
        for k, fn in STAGE_BYTES.items():
            ms = prof[k]
            gb = fn(n, m, npass) / 1e9
            row[k] = {"ms": ms, "algorithmic_GB": gb, "GB_per_s": gb / (ms * 1e-3), "frac_of_hbm": gb / (ms * 1e-3) / hbm}
        row["walk_ms"] = prof["walk"]
        out.append(row)
        sim.close()
        del pos, vel
    return {"metric": "memory-bound stage bandwidth (algorithmic bytes / event-timed stage time)",
            "value": out[-1]["sort"]["GB_per_s"], "unit": "GB/s (sort at N=16M)", "n_gpus": world,
            "higher_is_better": True, "hbm_peak_gbs": hbm, "peak_note": "MEASURED_PEAKS.json hbm_gbs (copy read+write)",
            "data": "synthetic (seeded disk + bulge, seed 1)", "rows": out}


def reference_arm(args, world, rank, local, dist):
    """The reference's method — the fixed-theta group walk, at the theta where
    its RMS force error on this workload is 1e-3 — timed on the host cores:
    the reference ships no CPU implementation of the path, so the oracle port
    (its algorithm restated in C, OpenMP over the cores) stands for it.  W
    untimed and K timed whole steps, nothing sampled.  Beside it, under
    "reference_cuda", the reference's own CUDA build (oracle/_ref/libref.so)
    on this GPU, W + K steps at the same theta.  The inputs come from the
    oracle library's copy of the seeded generator: this process never loads
    the engine library."""
    if rank != 0:
        return None
    from oracle import cpu
    n = args.n
    th = PLAIN_THETA_EQUAL_ERROR
    pos, vel = cpu.disk_galaxy(n, seed=WORK["seed"])
    cb = cpu_steps(pos, vel, th, args.steps, args.warmup)
    value = 1.0 / cb["step_s"]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * cb["step_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded disk + bulge, seed 1)",
        "config": {"workload": REF_WORKLOAD, "variant": "plain", "n_bodies": n, "theta": th,
                   "rms_target": WORK["rms_target"], "eps": WORK["eps"], "dt": WORK["dt"],
                   "bits_per_axis": WORK["bits"], "group_width": 32, "leaf_size": 1},
        "comparison": "the metric compares the engine's learned walk with the reference's method, the fixed-theta "
                      "walk, at equal RMS force error 1e-3; this arm runs that fixed-theta method at theta "
                      f"{th}, where its RMS error on this workload is 1e-3",
        "interactions_per_step": cb["interactions_per_step"],
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        import torch
        if torch.cuda.is_available() and cpu.ref_available():
            if args.warmup:
                cpu.ref_run(pos, vel, WORK["eps"], WORK["G"], th, WORK["dt"], steps=args.warmup, want_nodes=False,
                            track_ids=False)
            r = cpu.ref_run(pos, vel, WORK["eps"], WORK["G"], th, WORK["dt"], steps=args.steps, want_nodes=False,
                            track_ids=False)
            line["reference_cuda"] = {"value": 1e3 / r["ms_per_step"], "unit": "steps/s",
                                      "ms_per_step": r["ms_per_step"], "steps": args.steps, "warmup": args.warmup,
                                      "theta": th, "timing": "cudaEvent around each step, mean over the timed steps",
                                      "what": "the reference's own CUDA build (sm_100a) on this GPU, same inputs"}
    except Exception as e:  # the CPU line stands on its own
        line["reference_cuda"] = {"unavailable": str(e)[:200]}
    return line


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            line = reference_arm(args, world, rank, local, dist)
        elif args.workload == "batch":
            line = batch_arm(args, world, rank, local, dist)
        elif args.workload == "merger":
            line = merger_arm(args, world, rank, local, dist)
        elif args.workload == "stages":
            line = stages_arm(args, world, rank, local, dist)
        else:
            line = engine_arm(args, world, rank, local, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
