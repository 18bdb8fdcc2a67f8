"""The CPU oracle checked against known answers and against golden fixtures
produced by the reference itself (tests/golden/ref_*.npz, written by
tests/golden/make_golden.py from the reference's own CUDA kernels)."""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from conftest import node_fields_equal, rel_l2

GOLDEN = sorted((Path(__file__).parent / "golden").glob("ref_*.npz"))


# ----------------------------------------------------------- Morton keys
def test_expand_bits_known_values(oracle):
    assert oracle.expand_bits(0) == 0
    assert oracle.expand_bits(1) == 1
    assert oracle.expand_bits(0b11) == 0b1001
    assert oracle.expand_bits(0b101) == 0b1000001
    assert oracle.expand_bits((1 << 21) - 1) == 0x1249249249249249
    assert oracle.expand_bits(1 << 21) == 0  # masked to 21 bits (tree.cu:333)
    assert oracle.expand_bits((1 << 10) - 1, 10) == int("001" * 10, 2)


def test_morton_corner_and_interior_points(oracle):
    pos = np.array([[0, 0, 0, 1], [1, 1, 1, 1], [0.5, 0, 0, 1], [0, 0.5, 0, 1], [0, 0, 0.5, 1], [1, 0, 0, 1]],
                   np.float32)
    mn, mx = oracle.bbox(pos)
    box = oracle.world_box(mn, mx, 21)
    assert box.extent == 1.0 and box.scale == np.float32(2097151.0)
    keys, idx = oracle.morton(pos, box, 21)
    assert keys[0] == 0
    assert keys[1] == 0x7FFFFFFFFFFFFFFF  # every bit of every axis set; bit 63 clear
    g = int(np.float32(0.5) * np.float32(2097151.0))  # 1048575
    assert keys[2] == oracle.expand_bits(g) << 2  # x is the most significant of each triple
    assert keys[3] == oracle.expand_bits(g) << 1
    assert keys[4] == oracle.expand_bits(g)
    assert keys[5] == oracle.expand_bits((1 << 21) - 1) << 2
    assert list(idx) == list(range(6))
    # 10 bits per axis: 30-bit keys, not a prefix of the 21-bit keys
    box10 = oracle.world_box(mn, mx, 10)
    k10, _ = oracle.morton(pos, box10, 10)
    assert k10[1] == (1 << 30) - 1
    assert k10[2] == oracle.expand_bits(int(np.float32(0.5) * np.float32(1023.0)), 10) << 2


def test_sort_is_stable(oracle):
    rng = np.random.default_rng(0)
    keys = rng.integers(0, 20, 5000).astype(np.uint64) << np.uint64(50)
    vals = np.arange(5000, dtype=np.uint32)
    ks, vs = oracle.sort_pairs(keys, vals)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(ks, keys[order]) and np.array_equal(vs, vals[order])


# ------------------------------------------------------------------- tree
def test_two_body_tree(oracle):
    pos = np.array([[0, 0, 0, 1], [1, 1, 1, 3]], np.float32)
    vel = np.zeros((2, 3), np.float32)
    r = oracle.pipeline(pos, vel, 21)
    nodes = r["nodes"]
    # root + one leaf per body at level 1 (octants 0 and 7)
    assert r["count"] == 3 and r["deepest"] == 1
    assert list(nodes["level"]) == [0, 1, 1]
    assert list(nodes[0]["child"]) == [1, -1, -1, -1, -1, -1, -1, 2]
    assert list(nodes["count"]) == [2, 1, 1]
    assert list(nodes["parent"][1:]) == [0, 0]
    np.testing.assert_array_equal(nodes[0]["mass"], np.float32([0.75, 0.75, 0.75, 4]))


def test_chain_and_multibody_leaf(oracle):
    """Two bodies in the same deepest cell: a chain of single-child nodes down
    to level 21 ending in one two-body leaf (no path compression)."""
    pos = np.array([[0, 0, 0, 1], [0, 0, 0, 1], [1, 1, 1, 1]], np.float32)
    vel = np.zeros((3, 3), np.float32)
    r = oracle.pipeline(pos, vel, 21)
    nodes = r["nodes"]
    assert r["deepest"] == 21 and r["count"] == 1 + 2 + 20
    leaf = nodes[-1]
    assert leaf["level"] == 21 and leaf["count"] == 2 and (leaf["child"] == -1).all()
    for L in range(2, 22):  # one node per level along the chain
        assert r["level_count"][L] == 1


def test_walk_theta_zero_is_direct_sum(oracle, engine):
    """With theta = 0 every internal node opens: the walk is the exact
    softened direct sum over single-body leaves."""
    p, v = engine.plummer(512, seed=3)
    r = oracle.pipeline(p, v, 21)
    acc, inter = oracle.walk(r["pos"], r["nodes"], r["ext_x"], 0.05, 1.0, 0.0)
    ds = oracle.direct_sum(r["pos"], 0.05, 1.0)
    assert rel_l2(acc, ds) < 1e-5
    assert inter == 512 * 512


def test_two_body_force_analytic(oracle):
    pos = np.array([[0, 0, 0, 2.0], [3, 4, 0, 5.0]], np.float32)
    vel = np.zeros((2, 3), np.float32)
    r = oracle.pipeline(pos, vel, 21)
    eps = 0.1
    acc, _ = oracle.walk(r["pos"], r["nodes"], r["ext_x"], eps, 1.0, 0.5)
    d = np.array([3, 4, 0], np.float64)
    s = (25 + eps * eps) ** 1.5
    want = {0: 5.0 * d / s, 1: -2.0 * d / s}
    for i in range(2):
        body = 0 if r["pos"][i, 3] == 2.0 else 1
        np.testing.assert_allclose(acc[i], want[body], rtol=2e-6)


def test_walk_error_vs_direct_sum(oracle, engine):
    p, v = engine.plummer(4096, seed=0)
    r = oracle.pipeline(p, v, 21)
    acc, _ = oracle.walk(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.5)
    ds = oracle.direct_sum(r["pos"], 0.01, 1.0)
    err = np.linalg.norm(acc - ds, axis=1) / np.linalg.norm(ds, axis=1)
    assert np.sqrt(np.mean(err ** 2)) < 2e-2  # monopole BH at theta 0.5 (about 8e-3 here)


def test_relative_walk_limits(oracle, engine):
    """The relative criterion: an infinite budget leaves the reference walk
    unchanged bit for bit; a zero budget opens every node down to the leaves
    (a direct sum over the leaves)."""
    p, v = engine.plummer(2048, seed=2)
    r = oracle.pipeline(p, v, 21)
    n = p.shape[0]
    acc0, inter0 = oracle.walk(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.6)
    amag = np.linalg.norm(acc0, axis=1).astype(np.float32)
    acc_inf, inter_inf = oracle.walk_relative(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.6, 1e30, amag)
    assert inter_inf == inter0 and np.array_equal(acc_inf, acc0)
    acc_z, inter_z = oracle.walk_relative(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.6, 0.0, amag)
    leaves = int(np.sum(r["nodes"]["count"] == 1)) if n == len(np.unique(r["skeys"])) else None
    assert leaves == n and inter_z == n * n
    ds = oracle.direct_sum(r["pos"], 0.01, 1.0)
    assert rel_l2(acc_z, ds) < 1e-5
    # per-group parameters override the global ones
    gp = np.tile(np.array([0.6, 1e30], np.float32), ((n + 31) // 32, 1))
    acc_g, inter_g = oracle.walk_relative(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.1, 0.0, amag, gp)
    assert inter_g == inter0 and np.array_equal(acc_g, acc0)
    # a budget in between: more accurate than the fixed test, fewer
    # interactions than the direct sum
    acc_m, inter_m = oracle.walk_relative(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.6, 1e-3, amag)
    e0, em = rel_l2(acc0, ds), rel_l2(acc_m, ds)
    assert inter0 < inter_m < inter_z and em < e0


def test_diagnostics_two_bodies(oracle):
    p = np.array([[0, 0, 0, 1], [3, 4, 0, 2]], np.float32)
    v = np.array([[0, 1, 0], [0, -0.5, 0]], np.float32)
    d = oracle.diagnostics(p, v, 0.0, 2.0)
    assert d["mass"] == 3.0 and d["kinetic"] == 0.75
    assert d["potential"] == pytest.approx(-2.0 * 1 * 2 / 5, rel=1e-15)
    assert np.allclose(d["com"], [2.0, 8.0 / 3.0, 0.0]) and np.allclose(d["momentum"], 0.0)
    assert np.allclose(d["angular_momentum"], [0.0, 0.0, -3.0])
    soft = oracle.diagnostics(p, v, 1.0, 1.0)
    assert soft["potential"] == pytest.approx(-2.0 / np.sqrt(26.0), rel=1e-15)


def test_bucket_walk_limits(oracle, engine):
    """Bucket leaves: size 1 is the reference walk bit for bit; with theta 0
    every bucket is opened, so every body meets every body (a direct sum);
    in between, buckets cost interactions and buy accuracy."""
    p, v = engine.plummer(3000, seed=4)
    r = oracle.pipeline(p, v, 21)
    n = p.shape[0]
    a0, i0 = oracle.walk(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.5)
    a1, i1 = oracle.walk_buckets(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.5, 1)
    assert i1 == i0 and np.array_equal(a1, a0)
    az, iz = oracle.walk_buckets(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.0, 16)
    assert iz == n * n
    ds = oracle.direct_sum(r["pos"], 0.01, 1.0)
    assert rel_l2(az, ds) < 1e-4  # FP32 sums of 3000 terms against FP64
    a8, i8 = oracle.walk_buckets(r["pos"], r["nodes"], r["ext_x"], 0.01, 1.0, 0.5, 8)
    assert i8 > i0 and rel_l2(a8, ds) < rel_l2(a0, ds)


def test_overflow_reported(oracle):
    p = np.zeros((64, 4), np.float32)
    p[:, 3] = 1
    p[0::2, :3] = np.random.default_rng(1).random((32, 3), dtype=np.float32)
    p[1::2, :3] = p[0::2, :3]  # coincident pairs: ~10 nodes per body
    p[0, :3] = [0, 0, 0]
    p[-1, :3] = [1, 1, 1]
    vel = np.zeros((64, 3), np.float32)
    mn, mx = oracle.bbox(p)
    keys, idx = oracle.morton(p, oracle.world_box(mn, mx), 21)
    ks, perm = oracle.sort_pairs(keys, idx)
    sp, _ = oracle.reorder(p, vel, perm)
    *_, count = oracle.build_tree(ks, sp, 21, max_nodes=8 * 64)
    assert count == -1


# ------------------------------------------------- golden fixtures (reference)
@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_oracle_matches_reference_fixture(oracle, path):
    g = np.load(path)
    pos, vel = g["pos"], g["vel"]
    eps, G, theta, dt = (float(g[k]) for k in ("eps", "G", "theta", "dt"))
    r = oracle.pipeline(pos, vel, 21)
    assert np.array_equal(r["keys"], g["keys"])
    assert np.array_equal(r["skeys"], g["skeys"])
    assert np.array_equal(r["perm"], g["perm"])
    d = int(g["deepest"])
    assert r["deepest"] == d
    assert np.array_equal(r["level_offsets"][: d + 1], g["level_offsets"][: d + 1])
    assert np.array_equal(r["level_count"][: d + 1], g["level_count"][: d + 1])
    ref_nodes = g["nodes"].view(oracle.NODE_DTYPE)
    assert node_fields_equal(r["nodes"], ref_nodes) == []
    acc, _ = oracle.walk(r["pos"], r["nodes"], r["ext_x"], eps, G, theta)
    assert np.array_equal(acc.view(np.uint32), g["acc"].view(np.uint32)), rel_l2(acc, g["acc"])
    p2, v2 = r["pos"].copy(), r["vel"].copy()
    oracle.kick_drift(p2, v2, acc, dt)
    assert np.array_equal(p2, g["pos_out"]) and np.array_equal(v2, g["vel_out"])


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 3, "golden fixtures from the reference are missing (tests/golden/make_golden.py)"
