"""bh_sim_step_host_sorted: end-to-end steps in the reference's frame order.

The reference leaves its device arrays in the Morton order of the last
step's sort and copies frames out with the body ids (indexOut,
basicGravity.cu:767-800).  The call takes host arrays in any order with their
ids and returns the state after the last step in that order; fed back in, it
continues the simulation exactly as device-resident steps do.  Page-locked
arrays are written by the walk itself, pageable ones are copied after it:
both give the same bits."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _arrays(torch, n: int, pinned: bool):
    if pinned:
        hp = torch.empty((n, 4), dtype=torch.float32, pin_memory=True).numpy()
        hv = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
        hi = torch.empty((n,), dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
        return hp, hv, hi
    return np.empty((n, 4), np.float32), np.empty((n, 3), np.float32), np.empty(n, np.uint32)


def _device_run(engine, n, prm, p, v, steps):
    """Reference run: load, device steps, then the state in simulation order
    (pos, vel, ids) and in body-id order."""
    from tests.conftest import dev_to_host
    with engine.Simulation(n, prm) as sim:
        sim.load(p, v)
        sim.step(steps)
        ptr_p, ptr_v, ptr_i, m = sim.device_state()
        sp = dev_to_host(ptr_p, (m, 4), np.float32)
        sv = dev_to_host(ptr_v, (m, 3), np.float32)
        si = dev_to_host(ptr_i, (m,), np.uint32)
        ip, iv = sim.store()
    return sp, sv, si, ip, iv


@pytest.mark.parametrize("pinned", [True, False], ids=["pinned", "pageable"])
@pytest.mark.parametrize("mode", ["plain", "learned"])
def test_sorted_host_steps_equal_device_steps(torch_cuda, engine, pinned, mode):
    """Calls of 1 + 1 + 2 + 4 steps, each fed the arrays the last one
    returned, against 8 device steps: the same bodies in the same order with
    the same ids, bit for bit; scattered by id they equal bh_sim_store's
    state."""
    n = 30000
    p, v = engine.disk_galaxy(n, seed=4)
    if mode == "learned":
        prm = engine.Params(theta=0.9, eps=0.005, dt=5e-4, mac_mode=2, err_target=2e-3)
    else:
        prm = engine.Params(theta=0.5, eps=0.005, dt=5e-4)
    sp, sv, si, ip, iv = _device_run(engine, n, prm, p, v, 8)
    hp, hv, hi = _arrays(torch_cuda, n, pinned)
    hp[:] = p
    hv[:] = v
    hi[:] = np.arange(n, dtype=np.uint32)
    with engine.Simulation(n, prm) as sim:
        # 1 + 1 + 2 + 4 steps: the four-step call runs its two middle steps
        # as graph replays between the eager first and last steps
        for k in (1, 1, 2, 4):
            sim.step_host_sorted(hp, hv, hi, k)
        assert sim.stats()["error_bits"] == 0
        # the device state the call leaves behind is the same state
        sp2, sv2 = sim.store()
    assert np.array_equal(hi, si)
    assert np.array_equal(hp, sp) and np.array_equal(hv, sv)
    assert np.array_equal(np.sort(hi), np.arange(n, dtype=np.uint32))
    by_id_p = np.empty_like(hp)
    by_id_v = np.empty_like(hv)
    by_id_p[hi] = hp
    by_id_v[hi] = hv
    assert np.array_equal(by_id_p, ip) and np.array_equal(by_id_v, iv)
    assert np.array_equal(sp2, ip) and np.array_equal(sv2, iv)


def test_sorted_host_batch_equals_device_steps(torch_cuda, engine):
    """A batch of uneven systems: calls of 1 + 2 steps fed back their own
    output equal 3 device steps bit for bit, and every system's bodies stay
    in that system's slots."""
    counts = [1000, 33, 4096, 2, 5000]
    ps, vs = [], []
    for k, n in enumerate(counts):
        p, v = engine.plummer(n, seed=20 + k)
        ps.append(p)
        vs.append(v)
    p, v = np.concatenate(ps), np.concatenate(vs)
    n = int(sum(counts))
    prm = engine.Params(bits_per_axis=19, theta=0.5, eps=0.01, dt=1e-3)
    with engine.Simulation(0, prm, counts=counts) as sim:
        off = sim.system_offsets()
        sim.load(p, v)
        sim.step(3)
        from tests.conftest import dev_to_host
        ptr_p, _, ptr_i, m = sim.device_state()
        sp = dev_to_host(ptr_p, (m, 4), np.float32)
        si = dev_to_host(ptr_i, (m,), np.uint32)
    hp, hv, hi = _arrays(torch_cuda, n, True)
    hp[:] = p
    hv[:] = v
    hi[:] = np.arange(n, dtype=np.uint32)
    with engine.Simulation(0, prm, counts=counts) as sim:
        sim.step_host_sorted(hp, hv, hi, 1)
        sim.step_host_sorted(hp, hv, hi, 2)
    assert np.array_equal(hi, si) and np.array_equal(hp, sp)
    for k in range(len(counts)):
        sl = slice(off[k], off[k + 1])
        assert np.array_equal(np.sort(hi[sl]), np.arange(off[k], off[k + 1], dtype=np.uint32))


def test_sorted_host_any_input_order(torch_cuda, engine):
    """Bodies handed over in a shuffled order with their ids: one step gives
    the same forces and new state by id as the step from body-id order, to
    within the reordering of equal Morton keys (none at this size: the result
    is bit-identical), and the output order is the step's Morton order."""
    n = 20000
    p, v = engine.plummer(n, seed=7)
    prm = engine.Params(theta=0.5, eps=0.01, dt=1e-3)
    sp, sv, si, ip, iv = _device_run(engine, n, prm, p, v, 1)
    rng = np.random.default_rng(3)
    order = rng.permutation(n).astype(np.uint32)
    hp, hv, hi = _arrays(torch_cuda, n, True)
    hp[:] = p[order]
    hv[:] = v[order]
    hi[:] = order
    with engine.Simulation(n, prm) as sim:
        sim.step_host_sorted(hp, hv, hi, 1)
    assert np.array_equal(hi, si)
    assert np.array_equal(hp, sp) and np.array_equal(hv, sv)


def test_sorted_host_zero_steps_uploads(torch_cuda, engine):
    """nsteps = 0 uploads the bodies and leaves the host arrays alone."""
    n = 5000
    p, v = engine.plummer(n, seed=2)
    hp, hv, hi = _arrays(torch_cuda, n, True)
    order = np.arange(n, dtype=np.uint32)[::-1].copy()
    hp[:] = p[order]
    hv[:] = v[order]
    hi[:] = order
    with engine.Simulation(n, engine.Params(theta=0.5, eps=0.01, dt=1e-3)) as sim:
        sim.step_host_sorted(hp, hv, hi, 0)
        assert np.array_equal(hp, p[order]) and np.array_equal(hi, order)
        gp, gv = sim.store()
    assert np.array_equal(gp, p) and np.array_equal(gv, v)


def test_sorted_host_rejects_bad_ids(torch_cuda, engine):
    """An id outside [0, n) is reported as BH_ERR_INVALID (the kernels never
    index through it); the next call with valid ids succeeds."""
    n = 4096
    p, v = engine.plummer(n, seed=5)
    prm = engine.Params(theta=0.9, eps=0.01, dt=1e-3, mac_mode=1, alpha=1e-3)
    hp, hv, hi = _arrays(torch_cuda, n, True)
    log = []
    with engine.Simulation(n, prm) as sim:
        for it, bad in enumerate((False, True, False)):
            hp[:] = p
            hv[:] = v
            hi[:] = np.arange(n, dtype=np.uint32)
            if bad:
                hi[17] = n + 5
            try:
                sim.step_host_sorted(hp, hv, hi, 2)
                log.append((it, bad, "ok"))
            except engine.BHError as e:
                log.append((it, bad, e.name, sim.stats(check=False)["error_bits"]))
            if not bad:
                assert np.array_equal(np.sort(hi), np.arange(n, dtype=np.uint32)), log
    assert [x[2] for x in log] == ["ok", "BH_ERR_INVALID", "ok"], log


def test_sorted_host_frames_from_c(torch_cuda, engine, tmp_path):
    """tests/c/frames.c, compiled by gcc against bh_api.h: three frames of
    two steps each through bh_sim_step_host_sorted with cudaHostAlloc'd
    mapped arrays; the arrays after the last frame equal six device steps
    bit for bit (same order, same ids)."""
    root = Path(__file__).resolve().parent.parent
    pkg = root / "cudagravitydemo_b200"
    cuda = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
    exe = tmp_path / "frames"
    cc = shutil.which("gcc") or "cc"
    r = subprocess.run([cc, "-O2", "-Wall", "-Werror", "-std=c11", "-I", str(root / "include"), "-I",
                        str(cuda / "include"), str(root / "tests" / "c" / "frames.c"), "-o", str(exe), "-L", str(pkg),
                        "-lbh_b200", "-L", str(cuda / "lib64"), "-lcudart", f"-Wl,-rpath,{pkg}",
                        f"-Wl,-rpath,{cuda / 'lib64'}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    n = 16384
    p, v = engine.plummer(n, seed=0)
    with open(tmp_path / "in.bin", "wb") as f:
        np.array([n], np.int32).tofile(f)
        p.astype(np.float32).tofile(f)
        v.astype(np.float32).tofile(f)
    r = subprocess.run([str(exe), str(tmp_path / "in.bin"), str(tmp_path / "out.bin"), "3", "2", "0.01", "1.0",
                        "0.5", "0.001"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    raw = (tmp_path / "out.bin").read_bytes()
    got_p = np.frombuffer(raw, np.float32, 4 * n, 0).reshape(n, 4)
    got_v = np.frombuffer(raw, np.float32, 3 * n, 16 * n).reshape(n, 3)
    got_i = np.frombuffer(raw, np.uint32, n, 28 * n)
    sp, sv, si, _, _ = _device_run(engine, n, engine.Params(theta=0.5, eps=0.01, G=1.0, dt=1e-3), p, v, 6)
    assert np.array_equal(got_i, si)
    assert np.array_equal(got_p, sp) and np.array_equal(got_v, sv)
