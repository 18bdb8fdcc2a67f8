"""Parity against the reference itself: its own kernels (compiled from its
sources into oracle/_ref/libref.so) run on the GPU on the same inputs.
Keys, permutation and tree bit-exact; the CPU oracle's walk reproduces the
reference's accelerations bit for bit; the engine's forces are within 1e-5
relative L2 of the reference's."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_to_host, node_fields_equal, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness oracle/_ref/libref.so not built")
    return oracle


def _inputs(engine, name):
    if name == "plummer16k":
        p, v = engine.plummer(16384, seed=0)
        return p, v, dict(eps=0.01, theta=0.5, dt=1e-3)
    if name == "disk32k":
        p, v = engine.disk_galaxy(32768, seed=1)
        return p, v, dict(eps=0.005, theta=0.5, dt=5e-4)
    if name == "coincident":
        p, v = engine.plummer(4096, seed=7)
        p[1::2, :3] = p[0::2, :3]
        return p, v, dict(eps=0.02, theta=0.7, dt=1e-3)
    if name == "line":
        # bodies on a line along x, a coincident pair: the tree reaches level 21
        rng = np.random.default_rng(13)
        p = np.zeros((2049, 4), np.float32)
        p[:, 0] = rng.normal(0, 1, 2049).astype(np.float32)
        p[:, 1], p[:, 2], p[:, 3] = -1.5, 2.0, 1.0 / 2049
        p[7, 0] = p[8, 0]
        return p, np.zeros((2049, 3), np.float32), dict(eps=0.01, theta=0.6, dt=1e-3)
    raise KeyError(name)


@pytest.mark.parametrize("name", ["plummer16k", "disk32k", "coincident", "line"])
def test_oracle_reproduces_reference(torch_cuda, engine, ref, name):
    p, v, prm = _inputs(engine, name)
    r = ref.ref_run(p, v, prm["eps"], 1.0, prm["theta"], prm["dt"], steps=1)
    o = ref.pipeline(p, v, 21)
    assert np.array_equal(r["keys"], o["keys"])
    assert np.array_equal(r["skeys"], o["skeys"])
    assert np.array_equal(r["perm"], o["perm"])
    assert r["deepest"] == o["deepest"]
    d = r["deepest"]
    assert np.array_equal(r["level_offsets"][: d + 1], o["level_offsets"][: d + 1])
    assert np.array_equal(r["level_count"][: d + 1], o["level_count"][: d + 1])
    assert node_fields_equal(r["nodes"], o["nodes"]) == []
    exact = {}
    for order in (ref.D2_REF, ref.D2_ALT, ref.D2_PLAIN):
        acc, _ = ref.walk(o["pos"], o["nodes"], o["ext_x"], prm["eps"], 1.0, prm["theta"], 32, order)
        exact[order] = bool(np.array_equal(acc.view(np.uint32), r["acc"].view(np.uint32)))
        print("d2 order", order, "bit-exact", exact[order], "rel", rel_l2(acc, r["acc"]))
    assert exact[ref.D2_REF], exact
    pos, vel = o["pos"].copy(), o["vel"].copy()
    acc, _ = ref.walk(o["pos"], o["nodes"], o["ext_x"], prm["eps"], 1.0, prm["theta"])
    ref.kick_drift(pos, vel, acc, prm["dt"])
    assert np.array_equal(pos, r["pos"]) and np.array_equal(vel, r["vel"])


@pytest.mark.parametrize("name", ["plummer16k", "disk32k", "coincident", "line"])
def test_engine_matches_reference(torch_cuda, engine, ref, name):
    p, v, prm = _inputs(engine, name)
    n = p.shape[0]
    r = ref.ref_run(p, v, prm["eps"], 1.0, prm["theta"], prm["dt"], steps=1)
    sim = engine.Simulation(n, engine.Params(theta=prm["theta"], eps=prm["eps"], dt=prm["dt"], export_nodes=True))
    sim.load(p, v)
    acc = sim.accelerations()
    st = sim.stats()
    ts = sim.tree()
    assert np.array_equal(dev_to_host(ts.mortonIn, (n,), np.uint64), r["keys"])
    assert np.array_equal(dev_to_host(ts.mortonOut, (n,), np.uint64), r["skeys"])
    perm = dev_to_host(ts.indexOut, (n,), np.uint32)
    assert np.array_equal(perm, r["perm"])
    nodes = dev_to_host(ts.nodes, (st["node_count"],), engine.NODE_DTYPE)
    assert node_fields_equal(nodes, r["nodes"]) == []
    acc_ref = np.empty_like(r["acc"])
    acc_ref[perm] = r["acc"]
    assert rel_l2(acc, acc_ref) < FORCE_TOL
    sim.close()


def test_multi_step_trajectory(torch_cuda, engine, ref):
    """Ten steps of the engine against ten reference steps: the trajectories
    stay within float32 rounding of each other."""
    p, v = engine.plummer(8192, seed=4)
    prm = dict(eps=0.01, theta=0.5, dt=1e-3)
    r = ref.ref_run(p, v, prm["eps"], 1.0, prm["theta"], prm["dt"], steps=10, want_nodes=False)
    sim = engine.Simulation(8192, engine.Params(theta=prm["theta"], eps=prm["eps"], dt=prm["dt"]))
    sim.load(p, v)
    sim.step(10)
    gp, gv = sim.store()
    rp = np.empty_like(r["pos"])
    rv = np.empty_like(r["vel"])
    rp[r["ids"]] = r["pos"]
    rv[r["ids"]] = r["vel"]
    assert np.array_equal(gp[:, 3], rp[:, 3])
    assert rel_l2(gp[:, :3] - p[:, :3], rp[:, :3] - p[:, :3]) < 1e-4  # displacement over 10 steps
    assert rel_l2(gv - v, rv - v) < 1e-3                              # velocity change over 10 steps
    sim.close()
