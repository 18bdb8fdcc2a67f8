"""Batches of independent systems (bh_sim_create_batch): every system of a
batch must evolve exactly as it does alone — same keys (below the system
index), same tree, same forces bit for bit — while one launch per stage
serves all systems."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(engine, counts, seed0=0):
    ps, vs = [], []
    for k, n in enumerate(counts):
        p, v = engine.plummer(int(n), seed=seed0 + k)
        p[:, :3] += np.float32(3.0 * k)  # far apart in space: a shared tree would notice
        ps.append(p)
        vs.append(v)
    return ps, vs


def _batch_bits(systems: int, bits: int = 21) -> int:
    sb = 0
    while (1 << sb) < systems:
        sb += 1
    return min(bits, (64 - sb) // 3)


@pytest.mark.parametrize("counts", [[1000, 33, 4096, 2, 5000, 1024], [64] * 40 + [20000], [70000]])
def test_batch_equals_systems_alone(torch_cuda, engine, counts):
    ps, vs = _systems(engine, counts)
    bits = _batch_bits(len(counts))
    prm = engine.Params(bits_per_axis=bits, theta=0.5, eps=0.01, dt=1e-3)
    with engine.Simulation(0, prm, counts=counts) as b:
        off = b.system_offsets()
        assert list(np.diff(off)) == list(counts)
        b.load(np.concatenate(ps), np.concatenate(vs))
        acc = b.accelerations()
        inter = b.stats()["interactions"]
        b.step(3)
        bp, bv = b.store()
    total = 0
    for k, n in enumerate(counts):
        with engine.Simulation(n, prm) as s:
            s.load(ps[k], vs[k])
            a = s.accelerations()
            total += s.stats()["interactions"]
            s.step(3)
            sp, sv = s.store()
        sl = slice(off[k], off[k + 1])
        assert np.array_equal(acc[sl], a), f"system {k}: forces differ"
        assert np.array_equal(bp[sl], sp) and np.array_equal(bv[sl], sv), f"system {k}: state differs"
    assert inter == total


def test_batch_system_diagnostics(torch_cuda, engine, oracle):
    counts = [3000, 1500, 777]
    ps, vs = _systems(engine, counts, seed0=20)
    with engine.Simulation(0, engine.Params(bits_per_axis=20, theta=0.5, eps=0.01, dt=1e-3), counts=counts) as b:
        b.load(np.concatenate(ps), np.concatenate(vs))
        b.step(2)
        d = b.system_diagnostics()
        bp, bv = b.store()
        off = b.system_offsets()
    assert len(d) == 3
    for k in range(3):
        want = oracle.diagnostics(bp[off[k]:off[k + 1]], bv[off[k]:off[k + 1]], float(np.float32(0.01)), 1.0)
        assert d[k]["total"] == pytest.approx(want["total"], rel=1e-12)
        assert d[k]["mass"] == pytest.approx(want["mass"], rel=1e-12)


def test_batch_rejects_unsupported_modes(torch_cuda, engine):
    with pytest.raises(engine.BHError):
        engine.Simulation(0, engine.Params(mac_mode=1), counts=[100, 200])
    with pytest.raises(engine.BHError):
        engine.Simulation(0, engine.Params(export_nodes=True), counts=[100, 200])
    with pytest.raises(engine.BHError):
        engine.Simulation(0, engine.Params(), counts=[100, 0])
    with engine.Simulation(0, engine.Params(eps=0.01), counts=[100, 200]) as b:
        p, v = engine.plummer(299, seed=1)
        with pytest.raises(engine.BHError):
            b.load(p, v)  # a batch loads all its bodies


def test_batch_of_256_uneven_plummer_spheres(torch_cuda, engine):
    """The batched workload: 256 Plummer spheres, N log-uniform in
    [1024, 65536] (seed 2); graph-replayed steps, no device errors, and the
    per-system FP64 energy drift over 20 steps: small for the typical system
    (measured median ~1e-6); the worst systems are the smallest ones, whose
    few heavy bodies meet in close encounters at eps 0.01 and dt 1e-3
    (measured max ~4e-5, the same when such a system runs alone)."""
    rng = np.random.default_rng(2)
    counts = np.exp(rng.uniform(np.log(1024), np.log(65536), 256)).astype(np.int32)
    ps, vs = _systems(engine, counts, seed0=1000)
    prm = engine.Params(bits_per_axis=21, theta=0.5, eps=0.01, dt=1e-3)
    with engine.Simulation(0, prm, counts=counts) as b:
        b.load(np.concatenate(ps), np.concatenate(vs))
        d0 = b.system_diagnostics()
        b.step(20)
        st = b.stats()
        d1 = b.system_diagnostics()
    assert st["error_bits"] == 0
    drift = np.array([abs(y["total"] - x["total"]) / abs(x["total"]) for x, y in zip(d0, d1)])
    assert np.all(np.isfinite(drift)) and np.median(drift) < 1e-5 and drift.max() < 1e-3


@pytest.mark.parametrize("leaf", [4, 16])
def test_batch_with_buckets_equals_systems_alone(torch_cuda, engine, leaf):
    counts = [2000, 777, 9000]
    ps, vs = _systems(engine, counts, seed0=40)
    prm = engine.Params(bits_per_axis=20, theta=0.5, eps=0.01, dt=1e-3, leaf_size=leaf)
    with engine.Simulation(0, prm, counts=counts) as b:
        off = b.system_offsets()
        b.load(np.concatenate(ps), np.concatenate(vs))
        b.step(2)
        bp, bv = b.store()
    for k, n in enumerate(counts):
        with engine.Simulation(n, prm) as s:
            s.load(ps[k], vs[k])
            s.step(2)
            sp, sv = s.store()
        assert np.array_equal(bp[off[k]:off[k + 1]], sp) and np.array_equal(bv[off[k]:off[k + 1]], sv)


def test_autotuner_keeps_state_and_choice(torch_cuda, engine):
    counts = [3000, 20000, 1500, 40000]
    ps, vs = _systems(engine, counts, seed0=60)
    prm = engine.Params(bits_per_axis=20, theta=0.5, eps=0.01, dt=1e-3)
    with engine.Simulation(0, prm, counts=counts) as b:
        b.load(np.concatenate(ps), np.concatenate(vs))
        b.step(2)
        before = b.store()
        r = b.tune(3)
        after = b.store()
        assert np.array_equal(before[0], after[0]) and np.array_equal(before[1], after[1])
        assert r["leaf_size"] in (1, 2, 4, 8, 16) and r["group_width"] in (32, 64)
        assert r["stack_entries"] in (384, 768, 1536) and b.walk_stack() == r["stack_entries"]
        shapes = {(l, w, 768) for l in (1, 2, 4, 8, 16) for w in (32, 64)}
        first = min(shapes, key=lambda k: r["ms_per_step"][k])  # the stack depths are tried at the best shape
        assert set(r["ms_per_step"]) == shapes | {(first[0], first[1], d) for d in (384, 1536)}
        chosen = (r["leaf_size"], r["group_width"], r["stack_entries"])
        assert r["ms_per_step"][chosen] == min(r["ms_per_step"].values())
        b.step(2)
        tuned = b.store()
    # the tuned simulation steps exactly like a fresh one with the chosen bucket size
    with engine.Simulation(0, engine.Params(**{**prm.__dict__, "leaf_size": r["leaf_size"],
                                               "group_width": r["group_width"]}), counts=counts) as c:
        c.load(*before)
        c.step(2)
        ref = c.store()
    assert np.array_equal(tuned[0], ref[0]) and np.array_equal(tuned[1], ref[1])


@pytest.mark.parametrize("entries", [128, 384, 1536, 2048])
def test_walk_stack_depth_changes_nothing_but_speed(torch_cuda, engine, entries):
    """Where the walk keeps its stack (shared memory up to `entries` per warp,
    a global spill area past it) does not change the traversal: states after
    steps are bit-identical to the default depth.  128 entries makes the 262K
    disk walk spill on most groups."""
    p, v = engine.disk_galaxy(262144, seed=5)
    out = []
    for e in (0, entries):
        with engine.Simulation(262144, engine.Params(theta=0.5, eps=0.005, dt=5e-4)) as s:
            s.set_walk_stack(e)
            assert s.walk_stack() == (e or 768)
            s.load(p, v)
            s.step(3)
            out.append(s.store())
            assert s.stats()["error_bits"] == 0
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_walk_stack_depth_is_validated(torch_cuda, engine):
    with engine.Simulation(1024, engine.Params()) as s:
        for bad in (96, 130, 4096, -32):
            with pytest.raises(engine.BHError):
                s.set_walk_stack(bad)
