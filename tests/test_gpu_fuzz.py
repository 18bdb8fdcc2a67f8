"""Seeded random configurations against the oracle: clustered, uniform,
shell-like and heavy-tailed body sets of ragged sizes, uneven masses, at 21
and 10 Morton bits and several opening angles, with the plain and the
relative criterion.  Every case: keys, sorted keys, permutation and the whole
node array bit-exact, interaction count equal, forces within 1e-5 relative
L2 of the oracle's walk."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import dev_to_host, node_fields_equal, rel_l2

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-5


def _bodies(seed: int):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(500, 200_000))
    kind = seed % 4
    if kind == 0:  # clusters of different sizes
        k = int(rng.integers(2, 12))
        centres = rng.normal(0, 5, (k, 3))
        which = rng.integers(0, k, n)
        xyz = centres[which] + rng.normal(0, 1, (n, 3)) * rng.uniform(0.01, 1.0, k)[which, None]
    elif kind == 1:  # uniform cube, stretched
        xyz = rng.uniform(-1, 1, (n, 3)) * rng.uniform(0.1, 10, 3)
    elif kind == 2:  # thin shell
        d = rng.normal(0, 1, (n, 3))
        xyz = d / np.linalg.norm(d, axis=1, keepdims=True) * (1 + 0.01 * rng.normal(0, 1, (n, 1)))
    else:  # heavy-tailed radii
        d = rng.normal(0, 1, (n, 3))
        xyz = d / np.linalg.norm(d, axis=1, keepdims=True) * rng.pareto(1.5, (n, 1))
    p = np.zeros((n, 4), np.float32)
    p[:, :3] = xyz.astype(np.float32)
    p[:, 3] = (rng.lognormal(0, 1, n) / n).astype(np.float32)
    v = rng.normal(0, 0.1, (n, 3)).astype(np.float32)
    bits = 21 if seed % 3 else 10
    theta = float(rng.choice([0.3, 0.5, 0.7, 1.0]))
    eps = float(rng.choice([1e-3, 1e-2, 5e-2]))
    return p, v, bits, theta, eps


@pytest.mark.parametrize("seed", range(12))
def test_random_configuration_matches_oracle(torch_cuda, engine, oracle, seed):
    p, v, bits, theta, eps = _bodies(seed)
    n = p.shape[0]
    sim = engine.Simulation(n, engine.Params(bits_per_axis=bits, theta=theta, eps=eps, dt=1e-4, export_nodes=True))
    sim.load(p, v)
    acc = sim.accelerations()
    st = sim.stats()
    ts = sim.tree()
    keys = dev_to_host(ts.mortonIn, (n,), np.uint64)
    skeys = dev_to_host(ts.mortonOut, (n,), np.uint64)
    perm = dev_to_host(ts.indexOut, (n,), np.uint32)
    nodes = dev_to_host(ts.nodes, (st["node_count"],), engine.NODE_DTYPE)
    sim.close()
    o = oracle.pipeline(p, v, bits)
    assert np.array_equal(keys, o["keys"]) and np.array_equal(skeys, o["skeys"]) and np.array_equal(perm, o["perm"])
    assert st["node_count"] == o["count"] and node_fields_equal(nodes, o["nodes"]) == []
    acc_o, inter = oracle.walk(o["pos"], o["nodes"], o["ext_x"], eps, 1.0, theta)
    assert st["interactions"] == inter
    acc_ref = np.empty_like(acc_o)
    acc_ref[o["perm"]] = acc_o
    assert rel_l2(acc, acc_ref) < FORCE_TOL


@pytest.mark.parametrize("seed", range(4))
def test_random_configuration_relative_criterion_matches_oracle(torch_cuda, engine, oracle, seed):
    """The relative criterion (one budget alpha for every group) after a
    bootstrap step, against the oracle's relative walk with the engine's |a|."""
    p, v, bits, theta, eps = _bodies(100 + seed)
    n = p.shape[0]
    alpha = [3e-4, 1e-3, 3e-3, 1e-2][seed]
    prm = engine.Params(bits_per_axis=bits, theta=max(theta, 0.7), eps=eps, dt=1e-4, mac_mode=1, alpha=alpha)
    sim = engine.Simulation(n, prm)
    sim.load(p, v)
    sim.step(1)  # |a| for the relative test
    acc = sim.accelerations()
    st = sim.stats()
    pos_ptr, vel_ptr, idp, _ = sim.device_state()
    cur_p = dev_to_host(pos_ptr, (n, 4), np.float32)
    cur_v = dev_to_host(vel_ptr, (n, 3), np.float32)
    cur_ids = dev_to_host(idp, (n,), np.uint32)
    amag = sim.accel_magnitudes()
    sim.close()
    o = oracle.pipeline(cur_p, cur_v, bits)
    acc_s, inter = oracle.walk_relative(o["pos"], o["nodes"], o["ext_x"], eps, 1.0, max(theta, 0.7), alpha,
                                        amag[o["perm"]])
    assert st["interactions"] == inter
    acc_cur = np.empty_like(acc_s)
    acc_cur[o["perm"]] = acc_s
    acc_id = np.empty_like(acc_cur)
    acc_id[cur_ids] = acc_cur
    assert rel_l2(acc, acc_id) < FORCE_TOL
