"""outputDump.bin (the reference's frame file) from the engine: the C ABI
writer and the C simulation program, frames in body-id order."""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "cudagravitydemo_b200" / "gravity_sim"


def read_dump(path):
    raw = Path(path).read_bytes()
    n, frames = np.frombuffer(raw[:8], np.int32)
    rgb = np.frombuffer(raw[8:8 + 3 * n], np.uint8).reshape(n, 3)
    body = np.frombuffer(raw[8 + 3 * n:], np.float32)
    assert body.size == frames * n * 3, "frame count does not match the header"
    return int(n), int(frames), rgb, body.reshape(frames, n, 3)


def _sim_frames(engine, n, steps, every, prm, pos, vel):
    """Frames the reference's loop would write: after step i for i % every == 0."""
    out = []
    with engine.Simulation(n, prm) as sim:
        sim.load(pos, vel)
        for i in range(steps):
            sim.step(1)
            if i % every == 0 and len(out) < steps // every:
                out.append(sim.store()[0][:, :3].copy())
    return np.stack(out)


def test_dump_writer_orders_frames_by_body_id(torch_cuda, engine, tmp_path):
    lib = engine.lib()
    n, steps, every = 3000, 23, 5
    p, v = engine.plummer(n, seed=4)
    prm = engine.Params(theta=0.5, eps=0.01, dt=1e-3)
    path = tmp_path / "outputDump.bin"
    h = C.c_void_p()
    frames = steps // every
    engine._check(lib.bh_dump_open(C.byref(h), str(path).encode(), n, frames, None), "bh_dump_open")
    with engine.Simulation(n, prm) as sim:
        sim.load(p, v)
        written = 0
        for i in range(steps):
            sim.step(1)
            if i % every == 0 and written < frames:
                engine._check(lib.bh_sim_dump_frame(h, sim.handle), "bh_sim_dump_frame")
                written += 1
        engine._check(lib.bh_dump_close(h), "bh_dump_close")
    n2, f2, rgb, body = read_dump(path)
    assert (n2, f2) == (n, frames) and np.all(rgb == 100)
    want = _sim_frames(engine, n, steps, every, prm, p, v)
    assert np.array_equal(body, want)


def test_dump_frame_count_is_checked(torch_cuda, engine, tmp_path):
    lib = engine.lib()
    h = C.c_void_p()
    p, v = engine.plummer(100, seed=1)
    engine._check(lib.bh_dump_open(C.byref(h), str(tmp_path / "d.bin").encode(), 100, 2, None), "bh_dump_open")
    with engine.Simulation(100, engine.Params(eps=0.01)) as sim:
        sim.load(p, v)
        engine._check(lib.bh_sim_dump_frame(h, sim.handle), "bh_sim_dump_frame")
        assert lib.bh_dump_close(h) != 0  # one frame of two


def test_c_driver_matches_python_simulation(torch_cuda, engine, tmp_path):
    out = tmp_path / "outputDump.bin"
    r = subprocess.run([str(DRIVER), "-n", "4096", "-steps", "20", "-ic", "plummer", "-seed", "0", "-theta", "0.5",
                        "-eps", "0.01", "-dt", "0.001", "-o", str(out), "-quiet"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    assert "relative energy drift" in r.stdout
    n, frames, rgb, body = read_dump(out)
    assert (n, frames) == (4096, 4)
    p, v = engine.plummer(4096, seed=0)
    want = _sim_frames(engine, 4096, 20, 5, engine.Params(theta=0.5, eps=0.01, dt=1e-3), p, v)
    assert np.array_equal(body, want)


def test_c_driver_learned_walk(torch_cuda, engine, tmp_path):
    w = ROOT / "cudagravitydemo_b200" / "data" / "mac_mlp.f32"
    r = subprocess.run([str(DRIVER), "-n", "65536", "-steps", "50", "-ic", "disk", "-seed", "1", "-theta", "0.9",
                        "-eps", "0.005", "-dt", "0.0005", "-mac", "2", "-target", "0.00118", "-mlp", str(w),
                        "-o", "none", "-quiet"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    drift = float(r.stdout.split("relative energy drift")[1].split(",")[0])
    assert abs(drift) < 1e-4


def test_c_driver_reference_demo(torch_cuda, engine, tmp_path):
    """The reference's own configuration end to end: its demo galaxy, theta 0.7,
    eps 0.02, dt 0.08, frames every 5 steps."""
    out = tmp_path / "outputDump.bin"
    r = subprocess.run([str(DRIVER), "-n", "20000", "-steps", "10", "-ic", "demo", "-seed", "4", "-theta", "0.7",
                        "-eps", "0.02", "-dt", "0.08", "-o", str(out), "-quiet"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    n, frames, _, body = read_dump(out)
    assert (n, frames) == (20000, 2)
    p, v = engine.demo_galaxy(20000, seed=4)
    want = _sim_frames(engine, 20000, 10, 5, engine.Params(theta=0.7, eps=0.02, dt=0.08), p, v)
    assert np.array_equal(body, want)
