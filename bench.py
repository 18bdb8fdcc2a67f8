#!/usr/bin/env python
"""bench.py — Barnes-Hut steps/s on the N=1,048,576 disk galaxy on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Workload (plain fixed-theta Barnes-Hut on the disk galaxy): exponential disk
(R_d 1, sech^2 z0 0.1, 80% of the mass) + Hernquist bulge (a 0.2, 20%),
N = 1,048,576, seed 1, eps 0.005, dt 5e-4, theta 0.5, 21 Morton bits per
axis, leaf 1, groups of 32 (the reference's semantics).  A step is the whole
pipeline: bounding box, Morton keys, radix sort, reorder, octree + upward
pass, walk + kick-drift.

Engine arm: W untimed steps, then K steps timed one by one with CUDA events
on the simulation's stream, an L2 flush (a 512 MiB write, larger than the
126 MB L2) before each.  `value` = steps/s over all ranks (replicas: each GPU
steps its own copy; no collective on the data path).  `e2e` = the same
metric through the C ABI's host-buffer step (bh_sim_step_host: pinned host
arrays copied in, one step, results copied back, every step).  `roofline`:
the walk kernel, the dominant one, against the measured FP32 FMA throughput
(20 flops per body-node interaction).  `cpu_baseline`: the C oracle (the
reference algorithm restated, OpenMP over the host cores) on a bounded sample
of the same workload.

Reference arm (--impl reference): the reference's algorithm on the host
cores (the reference ships no CPU implementation of the path; the oracle
port stands for it), timed on the same workload and a bounded sample per
step; plus, under "reference_cuda", the reference's own CUDA build run on
this GPU for a few steps.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORK = dict(n=1 << 20, seed=1, eps=0.005, dt=5e-4, theta=0.5, bits=21, G=1.0)
METRIC = "steps/s @N=1M disk, learned-θ vs plain BH on 1 B200 at equal RMS force err"
WORKLOAD = "plain fixed-theta Barnes-Hut (theta=0.5), disk galaxy N=1,048,576"
FLOPS_PER_INTERACTION = 20
WALK_SAMPLE_STRIDE = 16  # CPU baselines walk every 16th group of 32 bodies
# DRAM bytes of one k_walk launch per body, from an ncu capture of the walk on
# the 262,144-body disk (20.9 MB read, nothing written back within the launch);
# the walk's traffic grows in proportion to the bodies it processes.
WALK_DRAM_BYTES_PER_BODY = 20.893184e6 / 262144


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--n", type=int, default=WORK["n"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
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
def cpu_baseline(pos, vel, stride: int = WALK_SAMPLE_STRIDE) -> dict:
    """The oracle's reference step on the host cores: the full bbox / keys /
    sort / reorder / tree pipeline plus every stride-th group of the walk;
    the walk time is scaled by stride."""
    from oracle import cpu
    t0 = time.perf_counter()
    r = cpu.pipeline(pos, vel, WORK["bits"])
    t1 = time.perf_counter()
    _, inter = cpu.walk_sample(r["pos"], r["nodes"], r["ext_x"], WORK["eps"], WORK["G"], WORK["theta"], stride)
    t2 = time.perf_counter()
    step_s = (t1 - t0) + (t2 - t1) * stride
    return {"step_s": step_s, "build_s": t1 - t0, "walk_sample_s": t2 - t1, "interactions_sampled": inter,
            "cores": cpu.num_threads(),
            "sample": f"full box/keys/sort/reorder/tree at N={pos.shape[0]} + walk of every {stride}th "
                      f"32-body group, walk time x{stride}"}


# ------------------------------------------------------------------ arms
def engine_arm(args, world, rank, local, dist):
    import torch

    import cudagravitydemo_b200 as bh
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    n = args.n
    pos, vel = bh.disk_galaxy(n, seed=WORK["seed"])
    prm = bh.Params(bits_per_axis=WORK["bits"], theta=WORK["theta"], eps=WORK["eps"], G=WORK["G"], dt=WORK["dt"])
    sim = bh.Simulation(n, prm)
    sim.load(pos, vel)
    stream = torch.cuda.ExternalStream(sim.stream, device=device)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=device)

    sim.step(args.warmup)
    stream.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.zero_()
                starts[k].record(stream)
                sim.step(1)
                ends[k].record(stream)
        stream.synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(step_ms), dist, device)
    stats = sim.stats()
    value = world * args.steps / (total_ms * 1e-3)

    # per-stage breakdown (separate, stage-by-stage run) and walk roofline
    stages = sim.profile(3)
    stats_p = sim.stats()
    peak = bh.fma_peak_tflops(5)
    walk_s = stages["walk"] * 1e-3
    achieved = stats_p["interactions"] * FLOPS_PER_INTERACTION / walk_s / 1e12

    e2e = None
    if not args.no_e2e:
        hp_t = torch.empty((n, 4), dtype=torch.float32, pin_memory=True)
        hv_t = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
        hp, hv = hp_t.numpy(), hv_t.numpy()
        hp[:] = pos
        hv[:] = vel
        sim.step_host(hp, hv, 1)  # warm
        e_ms = []
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            sim.step_host(hp, hv, 1)
            e1.record(stream)
            e1.synchronize()
            e_ms.append(e0.elapsed_time(e1))
        e_total = max_over_ranks(sum(e_ms), dist, device)
        e2e = {"value": world * args.steps / (e_total * 1e-3), "unit": "steps/s",
               "h2d_bytes_per_step": n * (16 + 12), "d2h_bytes_per_step": n * (16 + 12),
               "ms_per_step": e_total / args.steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(pos, vel)
        cpu = {"value": 1.0 / cb["step_s"], "unit": "steps/s", "cores": cb["cores"], "kind": "port",
               "sample": cb["sample"], "step_s": cb["step_s"]}

    clocks = clk.summary()
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded disk + bulge, seed 1)",
        "config": {"workload": WORKLOAD, "variant": "plain", "n_bodies": n, "theta": WORK["theta"],
                   "eps": WORK["eps"], "dt": WORK["dt"], "bits_per_axis": WORK["bits"], "group_width": 32,
                   "leaf_size": 1, "compensated_sums": True, "parallelism": f"replicas x{world}",
                   "l2": "flushed before every timed step (512 MiB write)"},
        "interactions_per_step": stats["interactions"],
        "interactions_per_s": stats["interactions"] * value,
        "nodes": stats["node_count"], "deepest_level": stats["deepest_level"],
        "stages_ms": stages,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak if peak else None,
                     "traffic": WALK_DRAM_BYTES_PER_BODY * n,
                     "traffic_note": "ncu dram read+write of k_walk at 262,144 bodies, scaled by body count",
                     "kernel": "k_walk (fused walk + kick-drift)",
                     "note": "20 flops per body-node interaction; peak = measured FMA-probe throughput"},
        "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": sim.kernels_per_step() * args.steps,
        "clocks": clocks,
    }
    sim.close()
    return line


def reference_arm(args, world, rank, local, dist):
    if rank != 0:
        return None
    import cudagravitydemo_b200 as bh
    n = args.n
    pos, vel = bh.disk_galaxy(n, seed=WORK["seed"])
    # the walk sample shrinks as K grows so that the whole run stays within a
    # few minutes; the box/keys/sort/tree pipeline always runs at full size
    stride = max(WALK_SAMPLE_STRIDE, (args.steps + args.warmup + 3) // 4)
    for _ in range(args.warmup):
        cpu_baseline(pos, vel, stride)
    times = []
    for _ in range(args.steps):
        times.append(cpu_baseline(pos, vel, stride)["step_s"])
    cb = cpu_baseline(pos, vel, stride)
    value = args.steps / sum(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded disk + bulge, seed 1)",
        "config": {"workload": WORKLOAD, "variant": "plain", "n_bodies": n, "theta": WORK["theta"],
                   "eps": WORK["eps"], "dt": WORK["dt"], "bits_per_axis": WORK["bits"], "group_width": 32,
                   "leaf_size": 1},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": cb["cores"], "kind": "port",
                         "sample": cb["sample"]},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        import torch

        from oracle import cpu
        if torch.cuda.is_available() and cpu.ref_available():
            r = cpu.ref_run(pos, vel, WORK["eps"], WORK["G"], WORK["theta"], WORK["dt"], steps=3, want_nodes=False,
                            track_ids=False)
            line["reference_cuda"] = {"value": 1e3 / r["ms_per_step"], "unit": "steps/s",
                                      "ms_per_step": r["ms_per_step"], "steps": 3,
                                      "what": "the reference's own CUDA build (sm_100a) on this GPU"}
    except Exception as e:  # the CPU line stands on its own
        line["reference_cuda"] = {"unavailable": str(e)[:200]}
    return line


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    try:
        line = engine_arm(args, world, rank, local, dist) if args.impl == "engine" else \
            reference_arm(args, world, rank, local, dist)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
