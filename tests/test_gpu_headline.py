"""Parity at the configurations the headline numbers are quoted on.

* The N = 1,048,576 disk (seed 1, eps 0.005, 21 bits): Morton keys, sorted
  keys, permutation, level table and the whole reference-layout node array
  bit-exact against the reference's own build (oracle/_ref/libref.so run on
  this GPU) — the 256-tile look-back sort, the 17-level tree and the
  multi-block upward pass at full size; forces within 1e-5 relative L2 of
  the reference's over all bodies, at theta 0.5 and at the theta where the
  plain walk's RMS error against the FP64 direct sum is 1e-3 (0.2386, the
  denominator of the headline ratio).  At that theta the oracle's walk is
  also checked bit for bit against the reference's accelerations, and the
  engine's interaction count equals the oracle's.
* The N = 4,194,304 two-disk merger (seed 3): keys, permutation and tree
  bit-exact against the reference, forces within 1e-5; and, on the merger and
  on the 1M disk, the learned walk
  (the network's per-group budgets) against the oracle's relative walk with
  the engine's per-group parameters on a sample of whole groups: the
  interaction-list length of every sampled group equal, the sampled bodies'
  forces within 1e-5, and the per-group choice equal to the oracle's rule on
  the engine's features.
* The N = 16,777,216 disk: keys, permutation and tree bit-exact against the
  oracle, forces within 1e-5 and the interaction count equal at theta 0.5.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_to_host, node_fields_equal, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5
DISK = dict(n=1 << 20, seed=1, eps=0.005, dt=5e-4)
THETA_EQUAL_ERROR = 0.2386  # the plain walk's RMS relative force error is 1e-3 here
MERGER_ERR_TARGET = 9.1e-4  # the learned walk's target that gives RMS 1e-3 on the merger
DISK_ERR_TARGET = 9.5e-4    # ... and on the 1M disk


@pytest.fixture(scope="module")
def ref(oracle):
    if not oracle.ref_available():
        pytest.skip("reference harness oracle/_ref/libref.so not built")
    return oracle


@pytest.fixture(scope="module")
def disk(engine):
    return engine.disk_galaxy(DISK["n"], seed=DISK["seed"])


@pytest.fixture(scope="module")
def merger(engine):
    return engine.merger(1 << 22, seed=3)


def _engine_tree(engine, p, v, theta, eps, dt):
    n = p.shape[0]
    sim = engine.Simulation(n, engine.Params(theta=theta, eps=eps, dt=dt, export_nodes=True))
    sim.load(p, v)
    acc = sim.accelerations()
    st = sim.stats()
    ts = sim.tree()
    out = dict(acc=acc, stats=st, keys=dev_to_host(ts.mortonIn, (n,), np.uint64),
               skeys=dev_to_host(ts.mortonOut, (n,), np.uint64), perm=dev_to_host(ts.indexOut, (n,), np.uint32),
               nodes=dev_to_host(ts.nodes, (st["node_count"],), engine.NODE_DTYPE))
    sim.close()
    return out


def _check_against_reference(got, r):
    assert np.array_equal(got["keys"], r["keys"]), "Morton keys differ"
    assert np.array_equal(got["skeys"], r["skeys"]), "sorted keys differ"
    assert np.array_equal(got["perm"], r["perm"]), "sort permutation differs"
    d = r["deepest"]
    assert got["stats"]["deepest_level"] == d
    assert got["stats"]["level_offsets"][: d + 1] == list(r["level_offsets"][: d + 1])
    assert got["stats"]["level_count"][: d + 1] == list(r["level_count"][: d + 1])
    assert got["stats"]["node_count"] == r["count"]
    assert node_fields_equal(got["nodes"], r["nodes"]) == []
    acc_ref = np.empty_like(r["acc"])
    acc_ref[got["perm"]] = r["acc"]  # reference: sorted order -> input order
    assert rel_l2(got["acc"], acc_ref) < FORCE_TOL


def test_disk1m_keys_sort_tree_forces_match_reference(torch_cuda, engine, ref, disk):
    p, v = disk
    r = ref.ref_run(p, v, DISK["eps"], 1.0, 0.5, DISK["dt"], steps=1)
    assert r["count"] > 1_500_000 and r["deepest"] >= 16  # the full-size tree
    got = _engine_tree(engine, p, v, 0.5, DISK["eps"], DISK["dt"])
    _check_against_reference(got, r)


def test_disk1m_equal_error_theta(torch_cuda, engine, ref, disk):
    """The plain walk at the headline's equal-error theta: the oracle
    reproduces the reference's accelerations bit for bit, the engine opens
    the same nodes (interaction count equal) and its forces are within 1e-5
    of the reference's."""
    p, v = disk
    th = THETA_EQUAL_ERROR
    r = ref.ref_run(p, v, DISK["eps"], 1.0, th, DISK["dt"], steps=1, want_nodes=False, track_ids=False)
    o = ref.pipeline(p, v, 21)
    assert np.array_equal(o["perm"], r["perm"])
    acc_o, inter = ref.walk(o["pos"], o["nodes"], o["ext_x"], DISK["eps"], 1.0, th)
    assert np.array_equal(acc_o.view(np.uint32), r["acc"].view(np.uint32))
    sim = engine.Simulation(p.shape[0], engine.Params(theta=th, eps=DISK["eps"], dt=DISK["dt"]))
    sim.load(p, v)
    acc = sim.accelerations()
    st = sim.stats()
    lens = sim.group_lengths()
    sim.close()
    assert st["interactions"] == inter
    assert np.array_equal(lens, ref.list_lengths(o["pos"], o["nodes"], o["ext_x"], th))
    acc_ref = np.empty_like(r["acc"])
    acc_ref[r["perm"]] = r["acc"]
    assert rel_l2(acc, acc_ref) < FORCE_TOL


def test_merger4m_keys_sort_tree_forces_match_reference(torch_cuda, engine, ref, merger):
    p, v = merger
    r = ref.ref_run(p, v, 0.005, 1.0, 0.5, 5e-4, steps=1)
    got = _engine_tree(engine, p, v, 0.5, 0.005, 5e-4)
    _check_against_reference(got, r)


def _learned_walk_matches_oracle(engine, ref, p, v, err_target, stride):
    from cudagravitydemo_b200 import learned
    from oracle import mlp as M
    n = p.shape[0]
    prm = engine.Params(theta=0.9, eps=0.005, dt=5e-4, mac_mode=2, err_target=err_target)
    sim = engine.Simulation(n, prm)
    sim.load(p, v)
    sim.step(2)  # the first step bootstraps |a|
    feat, _ = sim.group_features()
    acc = sim.accelerations()
    st = sim.stats()
    gp = sim.group_params()
    lens = sim.group_lengths()
    pos_ptr, vel_ptr, idp, _ = sim.device_state()
    cur_p = dev_to_host(pos_ptr, (n, 4), np.float32)
    cur_v = dev_to_host(vel_ptr, (n, 3), np.float32)
    cur_ids = dev_to_host(idp, (n,), np.uint32)
    amag = sim.accel_magnitudes()
    mlp = learned.load_weights()
    sim.close()
    assert st["error_bits"] == 0 and np.all(np.isfinite(gp))
    assert len(lens) == (n + 31) // 32 and lens.sum() * 32 == st["interactions"]
    # the per-group choice: the oracle's rule on the engine's features.  The
    # tensor-core forward and the oracle's round hidden activations to BF16
    # at different sums, which moves a prediction by up to ~5e-3 (1 + |y|)
    # (the bound the forward test uses); a group whose predictions come
    # that close to the target may choose differently.  The budget is
    # interpolated between two ladder steps where the predicted curve crosses
    # the target, so where that curve is flat a small prediction difference
    # moves it within the interval: every group that is not close must choose
    # the same ladder interval, and nearly all the same budget to 1e-3.
    ladder = learned.mac_ladder()
    want, y = M.select(mlp, feat, ladder, err_target, 0.9)
    lt = np.float32(np.log10(np.float32(err_target)))
    close = np.any(np.abs(y - lt) < 5e-3 * (1 + np.abs(y)), axis=1)

    def interval(alpha):
        return np.floor(np.log2(np.asarray(alpha, np.float64) / float(ladder[0])) + 1e-6)

    same_interval = (gp[:, 0] == want[:, 0]) & (interval(gp[:, 1]) == interval(want[:, 1]))
    same = same_interval & np.isclose(gp[:, 1], want[:, 1], rtol=1e-3, atol=0)
    assert np.all(same_interval | close), np.sum(~(same_interval | close))
    assert same.mean() > 0.95, same.mean()
    # the walk with those parameters, on every stride-th group
    o = ref.pipeline(cur_p, cur_v, 21)
    acc_s, lens_o, idx = ref.walk_groups_sample(o["pos"], o["nodes"], o["ext_x"], 0.005, 1.0, 0.9, stride,
                                                amag=amag[o["perm"]], group_param=gp)
    assert np.array_equal(lens[idx], lens_o)
    body = (idx[:, None] * 32 + np.arange(32)[None, :]).ravel()
    body = body[body < n]
    # engine accelerations come in body-id order; sorted slot s holds body
    # cur_ids[perm[s]]
    assert rel_l2(acc[cur_ids[o["perm"][body]]], acc_s[body]) < FORCE_TOL


def test_merger4m_learned_walk_matches_oracle(torch_cuda, engine, ref, merger):
    _learned_walk_matches_oracle(engine, ref, *merger, MERGER_ERR_TARGET, 32)


def test_disk1m_learned_walk_matches_oracle(torch_cuda, engine, ref, disk):
    """The headline walk (config 3): the shipped network at the target that
    gives RMS 1e-3 on the 1M disk."""
    _learned_walk_matches_oracle(engine, ref, *disk, DISK_ERR_TARGET, 8)


def test_disk16m_pipeline_matches_oracle(torch_cuda, engine, oracle):
    """The largest size measured (the memory-bound stages' 16M case): keys,
    permutation, level table and node array bit-exact against the oracle,
    interaction count equal and forces within 1e-5 at theta 0.5."""
    n = 1 << 24
    p, v = engine.disk_galaxy(n, seed=1)
    got = _engine_tree(engine, p, v, 0.5, DISK["eps"], DISK["dt"])
    o = oracle.pipeline(p, v, 21)
    assert np.array_equal(got["keys"], o["keys"])
    assert np.array_equal(got["skeys"], o["skeys"])
    assert np.array_equal(got["perm"], o["perm"])
    d = o["deepest"]
    assert got["stats"]["deepest_level"] == d
    assert got["stats"]["level_offsets"][: d + 1] == list(o["level_offsets"][: d + 1])
    assert got["stats"]["level_count"][: d + 1] == list(o["level_count"][: d + 1])
    assert got["stats"]["node_count"] == o["count"]
    assert node_fields_equal(got["nodes"], o["nodes"]) == []
    del got["nodes"]
    acc_o, inter = oracle.walk(o["pos"], o["nodes"], o["ext_x"], DISK["eps"], 1.0, 0.5)
    assert got["stats"]["interactions"] == inter
    acc_ref = np.empty_like(acc_o)
    acc_ref[o["perm"]] = acc_o
    assert rel_l2(got["acc"], acc_ref) < FORCE_TOL
