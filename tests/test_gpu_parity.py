"""Parity of the CUDA engine with the CPU oracle (which restates the
reference's algorithm, tree.cu / sorting.cu / basicGravity.cu):
Morton keys, sort permutation and tree topology + masses bit-exact; forces
within 1e-5 relative L2 of the reference walk at the same theta (the engine
evaluates the same interaction set with rsqrt and compensated sums)."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_to_host, node_fields_equal, rel_l2, to_device

FORCE_TOL = 1e-5  # relative L2 vs the reference walk, at the same theta

pytestmark = pytest.mark.gpu


def _case(engine, name: str):
    if name == "plummer16k":
        p, v = engine.plummer(16384, seed=0)
        return p, v, dict(eps=0.01, theta=0.5, dt=1e-3)
    if name == "disk64k":
        p, v = engine.disk_galaxy(65536, seed=1)
        return p, v, dict(eps=0.005, theta=0.5, dt=5e-4)
    if name == "plummer_ragged1000":
        p, v = engine.plummer(1000, seed=5)
        return p, v, dict(eps=0.01, theta=0.7, dt=1e-3)
    if name == "tiny33":
        p, v = engine.plummer(33, seed=6)
        return p, v, dict(eps=0.05, theta=0.5, dt=1e-3)
    if name == "two_bodies":
        p = np.array([[0, 0, 0, 1], [1, 0.5, 0.25, 2]], np.float32)
        v = np.zeros((2, 3), np.float32)
        return p, v, dict(eps=0.01, theta=0.5, dt=1e-3)
    if name == "coincident":
        # pairs and a quadruple of bodies at identical positions: multi-body
        # leaves at the deepest level
        p, v = engine.plummer(4096, seed=7)
        p[1::2, :3] = p[0::2, :3]
        p[100:104, :3] = p[100, :3]
        return p, v, dict(eps=0.02, theta=0.5, dt=1e-3)
    if name == "one_octant":
        rng = np.random.default_rng(11)
        p = np.zeros((5000, 4), np.float32)
        p[:, :3] = rng.random((5000, 3), dtype=np.float32) * 0.01 + 5.0
        p[0, :3] = 0.0  # one far body: every other body lands in one root octant
        p[:, 3] = 1.0 / 5000
        v = np.zeros((5000, 3), np.float32)
        return p, v, dict(eps=0.001, theta=0.5, dt=1e-4)
    if name == "flat":
        # every body in the plane z = 0.3: the z bits of every key are equal
        p, v = engine.plummer(3000, seed=12)
        p[:, 2] = 0.3
        return p, v, dict(eps=0.01, theta=0.5, dt=1e-3)
    if name == "line":
        # bodies on a line along x (y, z constant), two of them coincident
        rng = np.random.default_rng(13)
        p = np.zeros((2049, 4), np.float32)
        p[:, 0] = rng.normal(0, 1, 2049).astype(np.float32)
        p[:, 1], p[:, 2], p[:, 3] = -1.5, 2.0, 1.0 / 2049
        p[7, 0] = p[8, 0]
        v = np.zeros((2049, 3), np.float32)
        return p, v, dict(eps=0.01, theta=0.6, dt=1e-3)
    raise KeyError(name)


CASES = ["plummer16k", "disk64k", "plummer_ragged1000", "tiny33", "two_bodies", "coincident", "one_octant", "flat",
         "line"]


def _sim_outputs(engine, p, v, bits, prm):
    n = p.shape[0]
    sim = engine.Simulation(n, engine.Params(bits_per_axis=bits, theta=prm["theta"], eps=prm["eps"], G=1.0,
                                             dt=prm["dt"], export_nodes=True))
    sim.load(p, v)
    acc = sim.accelerations()
    st = sim.stats()
    ts = sim.tree()
    out = dict(acc=acc, stats=st,
               keys=dev_to_host(ts.mortonIn, (n,), np.uint64),
               skeys=dev_to_host(ts.mortonOut, (n,), np.uint64),
               perm=dev_to_host(ts.indexOut, (n,), np.uint32))
    out["nodes"] = dev_to_host(ts.nodes, (st["node_count"],), engine.NODE_DTYPE)
    sim.close()
    return out


@pytest.mark.parametrize("bits", [21, 10])
@pytest.mark.parametrize("name", CASES)
def test_pipeline_bit_exact_and_forces(torch_cuda, engine, oracle, name, bits):
    p, v, prm = _case(engine, name)
    n = p.shape[0]
    got = _sim_outputs(engine, p, v, bits, prm)
    ref = oracle.pipeline(p, v, bits)
    assert np.array_equal(got["keys"], ref["keys"]), "Morton keys differ"
    assert np.array_equal(got["skeys"], ref["skeys"]), "sorted keys differ"
    assert np.array_equal(got["perm"], ref["perm"]), "sort permutation differs"
    assert got["stats"]["node_count"] == ref["count"]
    assert got["stats"]["deepest_level"] == ref["deepest"]
    d = ref["deepest"]
    assert got["stats"]["level_offsets"][: d + 1] == list(ref["level_offsets"][: d + 1])
    assert got["stats"]["level_count"][: d + 1] == list(ref["level_count"][: d + 1])
    assert node_fields_equal(got["nodes"], ref["nodes"]) == []
    acc_sorted, inter = oracle.walk(ref["pos"], ref["nodes"], ref["ext_x"], prm["eps"], 1.0, prm["theta"])
    acc_ref = np.empty_like(acc_sorted)
    acc_ref[ref["perm"]] = acc_sorted
    assert rel_l2(got["acc"], acc_ref) < FORCE_TOL
    assert got["stats"]["interactions"] == inter


@pytest.mark.parametrize("name", ["plummer16k", "disk64k", "coincident"])
def test_drop_in_tree_state(torch_cuda, engine, oracle, name):
    """initialiseTree / buildTree / calculateAcceleration / positionUpdater
    (the reference's entry points) on caller-owned torch buffers."""
    torch = torch_cuda
    p, v, prm = _case(engine, name)
    n = p.shape[0]
    padded = (n + 31) // 32 * 32
    pos = torch.zeros((padded, 4), dtype=torch.float32, device="cuda")
    vel = torch.zeros((padded, 3), dtype=torch.float32, device="cuda")
    pos[:n] = torch.from_numpy(p).cuda()
    vel[:n] = torch.from_numpy(v).cuda()
    ts = engine.TreeState(n, pos, vel)
    ts.build()
    ref = oracle.pipeline(p, v, 21)
    assert np.array_equal(ts.host_keys("in"), ref["keys"])
    assert np.array_equal(ts.host_keys("out"), ref["skeys"])
    assert np.array_equal(ts.host_index("out"), ref["perm"])
    deep, lo, lc = ts.levels()
    assert deep == ref["deepest"] and lo == list(ref["level_offsets"][: deep + 1])
    assert lc == list(ref["level_count"][: deep + 1])
    assert node_fields_equal(ts.host_nodes(), ref["nodes"]) == []
    assert np.array_equal(ts.host_pos(), ref["pos"]) and np.array_equal(ts.host_vel(), ref["vel"])
    acc = torch.zeros((padded, 3), dtype=torch.float32, device="cuda")
    ts.accelerations(acc, prm["eps"], 1.0, prm["theta"])
    acc_o, _ = oracle.walk(ref["pos"], ref["nodes"], ref["ext_x"], prm["eps"], 1.0, prm["theta"])
    torch.cuda.synchronize()
    acc_h = acc[:n].cpu().numpy()
    assert rel_l2(acc_h, acc_o) < FORCE_TOL
    # kick-drift with the engine's own accelerations: exact FMA semantics
    ts.kick_drift(acc, prm["dt"])
    pos_o, vel_o = ref["pos"].copy(), ref["vel"].copy()
    oracle.kick_drift(pos_o, vel_o, acc_h, prm["dt"])
    assert np.array_equal(ts.host_pos(), pos_o) and np.array_equal(ts.host_vel(), vel_o)
    ts.close()


@pytest.mark.parametrize("n", [1, 2, 31, 4095, 4096, 4097, 100_000, 1 << 20])
def test_radix_sort_stable(torch_cuda, engine, n):
    torch = torch_cuda
    rng = np.random.default_rng(n)
    # many duplicates, all 64 bits in play, some keys with the top bit set
    keys = (rng.integers(0, 50, n, dtype=np.uint64) << np.uint64(40)) | rng.integers(0, 1 << 20, n, dtype=np.uint64)
    keys[::7] |= np.uint64(1) << np.uint64(63)
    keys[::5] = keys[0]
    vals = rng.permutation(n).astype(np.uint32)
    kin = to_device(torch, keys.view(np.int64))
    vin = to_device(torch, vals.view(np.int32))
    kout = torch.empty_like(kin)
    vout = torch.empty_like(vin)
    engine.radix_sort_pairs(kin, vin, kout, vout, key_bits=64)
    torch.cuda.synchronize()
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(kout.cpu().numpy().view(np.uint64), keys[order])
    assert np.array_equal(vout.cpu().numpy().view(np.uint32), vals[order])
    # inputs untouched
    assert np.array_equal(kin.cpu().numpy().view(np.uint64), keys)


def test_sorted_and_reversed_inputs(torch_cuda, engine):
    torch = torch_cuda
    n = 300_000
    keys = np.arange(n, dtype=np.uint64) * np.uint64(977)
    for k in (keys, keys[::-1].copy()):
        vals = np.arange(n, dtype=np.uint32)
        kin, vin = to_device(torch, k.view(np.int64)), to_device(torch, vals.view(np.int32))
        kout, vout = torch.empty_like(kin), torch.empty_like(vin)
        engine.radix_sort_pairs(kin, vin, kout, vout, key_bits=64)
        order = np.argsort(k, kind="stable")
        assert np.array_equal(vout.cpu().numpy().view(np.uint32), vals[order])


def test_full_step_matches_oracle_step(torch_cuda, engine, oracle):
    """Device-resident steps (graph replay, fused walk + kick-drift) against the
    oracle's step, bodies matched by id."""
    p, v = engine.plummer(8192, seed=3)
    prm = dict(eps=0.01, theta=0.5, dt=1e-3)
    sim = engine.Simulation(8192, engine.Params(theta=prm["theta"], eps=prm["eps"], G=1.0, dt=prm["dt"]))
    sim.load(p, v)
    sim.step(1)
    gp, gv = sim.store()
    op, ov = p.copy(), v.copy()
    ids = np.arange(8192, dtype=np.uint32)
    perm, acc, m, _ = oracle.step(op, ov, 21, prm["eps"], 1.0, prm["theta"], prm["dt"])
    ids = ids[perm]
    back_p = np.empty_like(op)
    back_v = np.empty_like(ov)
    back_p[ids] = op
    back_v[ids] = ov
    # velocities and positions agree to a few float32 ulps (the forces agree
    # to FORCE_TOL; a*dt is ~1e-3 of v)
    assert rel_l2(gv, back_v) < 1e-6
    assert np.array_equal(gp[:, 3], p[:, 3])
    ulp = np.spacing(np.abs(back_p[:, :3]).astype(np.float32))
    assert np.all(np.abs(gp[:, :3] - back_p[:, :3]) <= 4 * ulp)
    sim.step(5)
    st = sim.stats()
    assert st["error_bits"] == 0 and st["node_count"] > 8192
    sim.close()


def test_step_host_round_trip(torch_cuda, engine):
    p, v = engine.disk_galaxy(50_000, seed=2)
    sim = engine.Simulation(50_000, engine.Params(theta=0.5, eps=0.005, dt=5e-4))
    hp, hv = p.copy(), v.copy()
    sim.step_host(hp, hv, 3)
    sim.load(p, v)
    sim.step(3)
    gp, gv = sim.store()
    assert np.array_equal(hp, gp) and np.array_equal(hv, gv)
    sim.close()


def test_errors_reported(torch_cuda, engine):
    p, v = engine.plummer(4096, seed=1)
    sim = engine.Simulation(4096, engine.Params())
    bad = p.copy()
    bad[17, 0] = np.nan
    sim.load(bad, v)
    with pytest.raises(engine.BHError) as e:
        sim.accelerations()
        sim.stats()
    assert e.value.name in ("BH_ERR_NONFINITE",)
    same = p.copy()
    same[:, :3] = 1.0
    sim.load(same, v)
    with pytest.raises(engine.BHError) as e:
        sim.accelerations()
        sim.stats()
    assert e.value.name == "BH_ERR_DEGENERATE_BOX"
    sim.close()


def test_bounded_wait_reports_timeout_and_context_survives(torch_cuda, engine):
    """Failure detection without a fault: a device wait whose partner never
    arrives gives up, reports BH_ERR_TIMEOUT, and the next work runs."""
    import time
    t0 = time.time()
    assert engine.lib().bh_selftest_bounded_wait(None) == 8  # BH_ERR_TIMEOUT
    assert time.time() - t0 < 60
    p, v = engine.plummer(2048, seed=2)
    with engine.Simulation(2048, engine.Params(eps=0.01)) as sim:
        sim.load(p, v)
        sim.step(2)
        assert sim.stats()["error_bits"] == 0


def test_sorter_reports_device_timeout(torch_cuda, engine):
    """A standalone sorter's device errors are reachable: a look-back wait on
    the sorter's own status words whose predecessor never publishes gives up,
    bh_sorter_errors() returns BH_ERR_TIMEOUT once (the word is cleared), and
    the sorter then sorts correctly."""
    import ctypes as C
    torch = torch_cuda
    lib = engine.lib()
    h = C.c_void_p()
    assert lib.bh_sorter_create(C.byref(h), 10000) == 0
    try:
        assert lib.bh_selftest_sorter_timeout(h, None) == 0
        bits = np.zeros(1, np.int32)
        assert lib.bh_sorter_errors(h, bits.ctypes.data, None) == 8  # BH_ERR_TIMEOUT
        assert bits[0] == 1 << 7
        assert lib.bh_sorter_errors(h, None, None) == 0
        rng = np.random.default_rng(5)
        keys = rng.integers(0, 1 << 40, 10000, dtype=np.uint64)
        vals = np.arange(10000, dtype=np.uint32)
        kin, vin = to_device(torch, keys.view(np.int64)), to_device(torch, vals.view(np.int32))
        kout, vout = torch.empty_like(kin), torch.empty_like(vin)
        assert lib.bh_radix_sort_pairs(h, kin.data_ptr(), kout.data_ptr(), vin.data_ptr(), vout.data_ptr(), 10000, 64,
                                       None) == 0
        assert lib.bh_sorter_errors(h, None, None) == 0
        assert np.array_equal(vout.cpu().numpy().view(np.uint32), np.argsort(keys, kind="stable"))
    finally:
        lib.bh_sorter_destroy(h)
