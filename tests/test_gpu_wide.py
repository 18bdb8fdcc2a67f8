"""Groups of 64 bodies (groupWidth 64, two bodies per lane): the engine opens
exactly the nodes the oracle's group walk of width 64 opens — with the
fixed-theta, relative, learned and bucket criteria — and its forces are
within the reference-walk tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_to_host, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _bodies(engine, name):
    if name == "plummer16k":
        p, v = engine.plummer(16384, seed=0)
        return p, v, 0.01
    if name == "disk64k":
        p, v = engine.disk_galaxy(65536, seed=1)
        return p, v, 0.005
    if name == "ragged1000":
        p, v = engine.plummer(1000, seed=5)
        return p, v, 0.01
    if name == "tiny33":
        p, v = engine.plummer(33, seed=6)
        return p, v, 0.05
    if name == "coincident":
        p, v = engine.plummer(4096, seed=7)
        p[1::2, :3] = p[0::2, :3]
        return p, v, 0.02
    raise KeyError(name)


@pytest.mark.parametrize("theta", [0.5, 0.3])
@pytest.mark.parametrize("name", ["plummer16k", "disk64k", "ragged1000", "tiny33", "coincident"])
def test_wide_plain_walk_matches_oracle(torch_cuda, engine, oracle, name, theta):
    p, v, eps = _bodies(engine, name)
    n = p.shape[0]
    with engine.Simulation(n, engine.Params(theta=theta, eps=eps, dt=1e-3, group_width=64)) as sim:
        sim.load(p, v)
        acc = sim.accelerations()
        st = sim.stats()
    ref = oracle.pipeline(p, v, 21)
    acc_s, inter = oracle.walk(ref["pos"], ref["nodes"], ref["ext_x"], eps, 1.0, theta, 64)
    acc_id = np.empty_like(acc_s)
    acc_id[ref["perm"]] = acc_s
    assert st["interactions"] == inter
    assert rel_l2(acc, acc_id) < FORCE_TOL


def test_wide_full_step_matches_oracle_step(torch_cuda, engine, oracle):
    """The fused walk + kick-drift of 64-body groups against the oracle's step."""
    p, v = engine.plummer(8192, seed=3)
    with engine.Simulation(8192, engine.Params(theta=0.5, eps=0.01, dt=1e-3, group_width=64)) as sim:
        sim.load(p, v)
        sim.step(1)
        gp, gv = sim.store()
    op, ov = p.copy(), v.copy()
    perm, _, _, _ = oracle.step(op, ov, 21, 0.01, 1.0, 0.5, 1e-3, group=64)
    back_p, back_v = np.empty_like(op), np.empty_like(ov)
    back_p[perm] = op
    back_v[perm] = ov
    assert rel_l2(gv, back_v) < 1e-6
    ulp = np.spacing(np.abs(back_p[:, :3]).astype(np.float32))
    assert np.all(np.abs(gp[:, :3] - back_p[:, :3]) <= 4 * ulp)


def _state(sim, n):
    pos_ptr, vel_ptr, ids_ptr, _ = sim.device_state()
    return (dev_to_host(pos_ptr, (n, 4), np.float32), dev_to_host(vel_ptr, (n, 3), np.float32),
            dev_to_host(ids_ptr, (n,), np.uint32), sim.accel_magnitudes())


@pytest.mark.parametrize("name", ["plummer16k", "disk64k", "ragged1000"])
def test_wide_relative_walk_matches_oracle(torch_cuda, engine, oracle, name):
    p, v, eps = _bodies(engine, name)
    n = p.shape[0]
    with engine.Simulation(n, engine.Params(theta=0.8, eps=eps, dt=1e-4, mac_mode=1, alpha=1e-3,
                                            group_width=64)) as sim:
        sim.load(p, v)
        sim.step(2)
        cur_p, cur_v, ids, amag = _state(sim, n)
        acc = sim.accelerations()
        st = sim.stats()
    ref = oracle.pipeline(cur_p, cur_v, 21)
    acc_s, inter = oracle.walk_relative(ref["pos"], ref["nodes"], ref["ext_x"], eps, 1.0, 0.8, 1e-3,
                                        amag[ref["perm"]], width=64)
    acc_c = np.empty_like(acc_s)
    acc_c[ref["perm"]] = acc_s
    acc_id = np.empty_like(acc_c)
    acc_id[ids] = acc_c
    assert st["interactions"] == inter
    assert rel_l2(acc, acc_id) < FORCE_TOL


def test_wide_learned_walk_matches_oracle(torch_cuda, engine, oracle):
    """The network's choices stay per 32-body group; a 64-body group takes the
    smaller theta and budget of its halves."""
    n = 65536 + 40  # a ragged last group
    p, v = engine.disk_galaxy(n, seed=2)
    prm = engine.Params(theta=0.9, eps=0.005, dt=5e-4, mac_mode=2, err_target=2e-3, group_width=64)
    with engine.Simulation(n, prm) as sim:
        sim.load(p, v)
        sim.step(2)
        cur_p, cur_v, ids, amag = _state(sim, n)
        acc = sim.accelerations()
        st = sim.stats()
        gp = sim.group_params()
    assert len(np.unique(gp[:, 1])) > 1
    ref = oracle.pipeline(cur_p, cur_v, 21)
    acc_s, inter = oracle.walk_relative(ref["pos"], ref["nodes"], ref["ext_x"], 0.005, 1.0, 0.9, 0.0,
                                        amag[ref["perm"]], group_param=gp, width=64)
    acc_c = np.empty_like(acc_s)
    acc_c[ref["perm"]] = acc_s
    acc_id = np.empty_like(acc_c)
    acc_id[ids] = acc_c
    assert st["interactions"] == inter
    assert rel_l2(acc, acc_id) < FORCE_TOL


@pytest.mark.parametrize("leaf", [4, 16])
def test_wide_bucket_walk_matches_oracle(torch_cuda, engine, oracle, leaf):
    p, v, eps = _bodies(engine, "disk64k")
    n = p.shape[0]
    with engine.Simulation(n, engine.Params(theta=0.5, eps=eps, dt=1e-3, leaf_size=leaf, group_width=64)) as sim:
        sim.load(p, v)
        acc = sim.accelerations()
        st = sim.stats()
    ref = oracle.pipeline(p, v, 21)
    acc_s, inter = oracle.walk_buckets(ref["pos"], ref["nodes"], ref["ext_x"], eps, 1.0, 0.5, leaf, 64)
    acc_id = np.empty_like(acc_s)
    acc_id[ref["perm"]] = acc_s
    assert st["interactions"] == inter
    assert rel_l2(acc, acc_id) < FORCE_TOL


def test_wide_batch_equals_systems_alone(torch_cuda, engine):
    counts = [1000, 33, 4096, 65, 5000]
    ps, vs = [], []
    for k, c in enumerate(counts):
        p, v = engine.plummer(c, seed=80 + k)
        ps.append(p)
        vs.append(v)
    prm = engine.Params(bits_per_axis=20, theta=0.5, eps=0.01, dt=1e-3, group_width=64)
    with engine.Simulation(0, prm, counts=counts) as b:
        off = b.system_offsets()
        b.load(np.concatenate(ps), np.concatenate(vs))
        b.step(2)
        bp, bv = b.store()
    for k, c in enumerate(counts):
        with engine.Simulation(c, prm) as s:
            s.load(ps[k], vs[k])
            s.step(2)
            sp, sv = s.store()
        assert np.array_equal(bp[off[k]:off[k + 1]], sp) and np.array_equal(bv[off[k]:off[k + 1]], sv)
