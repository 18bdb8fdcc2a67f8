"""The CPU side of the measurement: the oracle library's copy of the seeded
generators, the sampled group walk the learned-walk parity test uses, and the
reference arm of bench.py, which must not load the engine library."""
from __future__ import annotations

import json
import subprocess
import sys

import numpy as np

from conftest import ROOT


def test_oracle_generators_equal_the_engine_generators(oracle, engine):
    for ours, theirs, n, seed in [(oracle.disk_galaxy, engine.disk_galaxy, 50_000, 1),
                                  (oracle.plummer, engine.plummer, 4096, 0),
                                  (oracle.merger, engine.merger, 60_000, 3)]:
        p1, v1 = ours(n, seed=seed)
        p2, v2 = theirs(n, seed=seed)
        assert np.array_equal(p1, p2) and np.array_equal(v1, v2)


def test_sampled_group_walk_equals_full_walk(oracle):
    p, v = oracle.disk_galaxy(20_000, seed=3)
    r = oracle.pipeline(p, v, 21)
    acc, lens, idx = oracle.walk_groups_sample(r["pos"], r["nodes"], r["ext_x"], 0.005, 1.0, 0.5, 7)
    full = oracle.list_lengths(r["pos"], r["nodes"], r["ext_x"], 0.5)
    assert np.array_equal(full[idx], lens)
    acc_full, _ = oracle.walk(r["pos"], r["nodes"], r["ext_x"], 0.005, 1.0, 0.5)
    body = (idx[:, None] * 32 + np.arange(32)[None, :]).ravel()
    body = body[body < 20_000]
    assert np.array_equal(acc[body], acc_full[body])
    # the relative criterion with per-group parameters, against the full relative walk
    amag = np.linalg.norm(acc_full, axis=1).astype(np.float32)
    gp = np.tile(np.array([[0.9, 1e-3]], np.float32), ((20_000 + 31) // 32, 1))
    gp[::3, 1] = 3e-4
    acc_s, lens_s, _ = oracle.walk_groups_sample(r["pos"], r["nodes"], r["ext_x"], 0.005, 1.0, 0.9, 5, amag=amag,
                                                 group_param=gp)
    acc_r, _ = oracle.walk_relative(r["pos"], r["nodes"], r["ext_x"], 0.005, 1.0, 0.9, 0.0, amag, group_param=gp)
    body = (np.arange(0, len(gp), 5)[:, None] * 32 + np.arange(32)[None, :]).ravel()
    body = body[body < 20_000]
    assert np.array_equal(acc_s[body], acc_r[body])


def test_reference_arm_runs_whole_steps_without_the_engine_library(tmp_path):
    """bench.py --impl reference on a small disk: one JSON line whose CPU
    value comes from whole steps, and the process never maps libbh_b200.so."""
    code = (
        "import sys, json; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '2', '--warmup', '1', "
        "'--n', '8192']; import bench; bench.main(); "
        "maps = open('/proc/self/maps').read(); print('ENGINE_MAPPED', 'libbh_b200' in maps)"
    )
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    line = json.loads(lines[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] == 2
    assert line["cpu_baseline"]["kind"] == "port" and "whole steps" in line["cpu_baseline"]["sample"]
    assert abs(line["ms_per_step"] * line["value"] - 1e3) < 1e-6 * 1e3
    assert "ENGINE_MAPPED False" in r.stdout
