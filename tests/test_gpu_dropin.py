"""The drop-in boundary as a reference caller uses it: tests/c/dropin.c is the
reference's host code written against include/main.h only, compiled by gcc
as plain C and linked with libbh_b200.so.

* levels: the reference's buildTree (basicGravity.cu:116-325) driven stage by
  stage through localMinMaxFinder / globalMinMaxReducer / createWorldBox,
  mortonEncode, sorterCreate / radixSortPairs, reorderParticles and, level by
  level, identifyNodesAtLevel / prefixSum / createNodes / updateTreeParticles,
  then updateTreeMass from the deepest level up.  Box, keys, permutation,
  level table, every node field and the sorted bodies equal the oracle's bit
  for bit (up to the 1M disk).
* loop: the reference's main loop (basicGravity.cu:709-783) as the
  integration guide shows it (initialiseTree, buildTree with its pointer
  swap, calculateAcceleration, positionUpdater, destroyTree); after several
  steps the state equals bh_sim's graph-replayed steps bit for bit.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT, dev_to_host, node_fields_equal

pytestmark = pytest.mark.gpu

SRC = ROOT / "tests" / "c" / "dropin.c"
PKG = ROOT / "cudagravitydemo_b200"


@pytest.fixture(scope="module")
def dropin(engine, tmp_path_factory):
    cc = shutil.which("gcc") or "cc"
    cuda = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
    exe = tmp_path_factory.mktemp("dropin") / "dropin"
    r = subprocess.run([cc, "-O2", "-Wall", "-Werror", "-std=c11", "-I", str(ROOT / "include"), "-I",
                        str(cuda / "include"), str(SRC), "-o", str(exe), "-L", str(PKG), "-lbh_b200", "-L",
                        str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{cuda / 'lib64'}"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _write_input(path: Path, p, v):
    with open(path, "wb") as f:
        np.array([p.shape[0]], np.int32).tofile(f)
        np.ascontiguousarray(p, np.float32).tofile(f)
        np.ascontiguousarray(v, np.float32).tofile(f)


def _run(exe, *args, timeout=300):
    r = subprocess.run([str(exe), *map(str, args)], capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stdout + r.stderr


class _Reader:
    def __init__(self, path: Path):
        self.buf = path.read_bytes()
        self.off = 0

    def take(self, dtype, count):
        dt = np.dtype(dtype)
        a = np.frombuffer(self.buf, dt, count, self.off).copy()
        self.off += dt.itemsize * count
        return a


def _case(engine, name):
    if name == "plummer16k":
        return engine.plummer(16384, seed=0)
    if name == "disk64k":
        return engine.disk_galaxy(65536, seed=1)
    if name == "disk1m":
        return engine.disk_galaxy(1 << 20, seed=1)
    if name == "coincident":
        p, v = engine.plummer(4096, seed=7)
        p[1::2, :3] = p[0::2, :3]
        return p, v
    raise KeyError(name)


@pytest.mark.parametrize("name", ["plummer16k", "disk64k", "coincident", "disk1m"])
def test_reference_level_loop_through_c_abi(engine, oracle, dropin, tmp_path, name):
    p, v = _case(engine, name)
    n = p.shape[0]
    _write_input(tmp_path / "in.bin", p, v)
    _run(dropin, "levels", tmp_path / "in.bin", tmp_path / "out.bin")
    o = oracle.pipeline(p, v, 21)
    r = _Reader(tmp_path / "out.bin")
    lo, hi = r.take(np.float32, 3), r.take(np.float32, 3)
    box = r.take(np.float32, 5)
    assert np.array_equal(lo, o["mn"]) and np.array_equal(hi, o["mx"])
    want_box = np.array([o["box"].minX, o["box"].minY, o["box"].minZ, o["box"].extent, o["box"].scale], np.float32)
    assert np.array_equal(box, want_box)
    assert np.array_equal(r.take(np.uint64, n), o["keys"])
    assert np.array_equal(r.take(np.uint64, n), o["skeys"])
    assert np.array_equal(r.take(np.uint32, n), o["perm"])
    deepest = int(r.take(np.int32, 1)[0])
    lo_tab, lc_tab = r.take(np.int32, 22), r.take(np.int32, 22)
    assert deepest == o["deepest"]
    assert np.array_equal(lo_tab[: deepest + 1], o["level_offsets"][: deepest + 1])
    assert np.array_equal(lc_tab[: deepest + 1], o["level_count"][: deepest + 1])
    count = int(r.take(np.int32, 1)[0])
    assert count == o["count"]
    nodes = r.take(engine.NODE_DTYPE, count)
    assert node_fields_equal(nodes, o["nodes"]) == []
    assert np.array_equal(r.take(np.float32, 4 * n).reshape(n, 4), o["pos"])
    assert np.array_equal(r.take(np.float32, 3 * n).reshape(n, 3), o["vel"])


@pytest.mark.parametrize("name,steps,prm", [
    ("plummer16k", 6, dict(eps=0.01, G=1.0, theta=0.5, dt=1e-3)),
    ("disk64k", 4, dict(eps=0.005, G=1.0, theta=0.5, dt=5e-4)),
])
def test_reference_main_loop_equals_sim_steps(torch_cuda, engine, dropin, tmp_path, name, steps, prm):
    p, v = _case(engine, name)
    n = p.shape[0]
    _write_input(tmp_path / "in.bin", p, v)
    _run(dropin, "loop", tmp_path / "in.bin", tmp_path / "out.bin", steps, prm["eps"], prm["G"], prm["theta"],
         prm["dt"])
    r = _Reader(tmp_path / "out.bin")
    got_p = r.take(np.float32, 4 * n).reshape(n, 4)
    got_v = r.take(np.float32, 3 * n).reshape(n, 3)
    got_perm = r.take(np.uint32, n)
    with engine.Simulation(n, engine.Params(theta=prm["theta"], eps=prm["eps"], G=prm["G"], dt=prm["dt"])) as sim:
        sim.load(p, v)
        sim.step(steps)
        pos_ptr, vel_ptr, _, _ = sim.device_state()
        sp = dev_to_host(pos_ptr, (n, 4), np.float32)
        sv = dev_to_host(vel_ptr, (n, 3), np.float32)
        perm = dev_to_host(sim.tree().indexOut, (n,), np.uint32)
    assert np.array_equal(got_perm, perm)
    assert np.array_equal(got_p, sp) and np.array_equal(got_v, sv)
