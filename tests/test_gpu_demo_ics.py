"""The reference program's own demo galaxy (bh_ic_demo), seeded and built on
the device: the distribution the reference's initialConditions.c draws,
checked statistically and body by body where the construction is exact."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_demo_galaxy_is_seeded(torch_cuda, engine):
    a = engine.demo_galaxy(10000, seed=5)
    b = engine.demo_galaxy(10000, seed=5)
    c = engine.demo_galaxy(10000, seed=6)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])


def test_demo_galaxy_distribution(torch_cuda, engine):
    n = 200_000
    pos, vel = engine.demo_galaxy(n, seed=1)
    n_halo = int(n * np.float32(0.2))
    n_disk = n - n_halo
    assert np.all(pos[:, 3] == np.float32(5.0) / np.float32(n))
    disk, halo = pos[:n_disk], pos[n_disk:]
    # disk: radius below 5 R_d from P(R) ~ R exp(-R / 4), Laplace heights of scale 0.3
    R = np.hypot(disk[:, 0], disk[:, 1]).astype(np.float64)
    assert R.max() <= 20.0 + 1e-4
    r = np.linspace(0, 20, 200001)
    w = r * np.exp(-r / 4)
    mean_R = np.trapezoid(r * w, r) / np.trapezoid(w, r)
    assert abs(R.mean() / mean_R - 1) < 0.01
    assert abs(np.abs(disk[:, 2]).mean() / 0.3 - 1) < 0.02
    # disk speeds: the circular speed of the enclosed disk mass, tangential
    menc = 5.0 * (1 - (1 + R / 4) * np.exp(-R / 4))
    v = np.linalg.norm(vel[:n_disk].astype(np.float64), axis=1)
    # (the FP32 1 - (1 + x) e^-x, x = R / 4, cancels as x -> 0, in the reference
    # too: compare away from the centre, and only bound the speed near it)
    far = R > 1.0
    assert np.allclose(v[far], np.sqrt(menc[far] / R[far]), rtol=2e-5)
    assert np.all(np.isfinite(v)) and v.max() < 1.0
    assert np.all(vel[:n_disk, 2] == 0)
    radial = (disk[:, 0] * vel[:n_disk, 0] + disk[:, 1] * vel[:n_disk, 1]) / (R * np.maximum(v, 1e-30))
    assert np.abs(radial).max() < 1e-4
    # halo: radius uniform in [0, 20), cos(polar) uniform, at rest
    rh = np.linalg.norm(halo[:, :3].astype(np.float64), axis=1)
    assert abs(rh.mean() / 10.0 - 1) < 0.02 and rh.max() <= 20.0
    ch = halo[:, 2] / np.maximum(rh, 1e-30)
    assert abs(ch.mean()) < 0.02 and abs((ch ** 2).mean() - 1 / 3) < 0.01
    assert np.all(vel[n_disk:] == 0)


def test_demo_galaxy_rotation_and_offsets(torch_cuda, engine):
    base = engine.demo_galaxy(5000, seed=3)
    rot = engine.demo_galaxy(5000, seed=3, rotation=(0.3, -0.7, 1.1), centre=(1, 2, 3), velocity=(0.5, 0, -0.5))
    d0 = np.linalg.norm(base[0][:, :3], axis=1)
    d1 = np.linalg.norm(rot[0][:, :3] - np.array([1, 2, 3], np.float32), axis=1)
    assert np.allclose(d0, d1, rtol=1e-5, atol=1e-5)  # a rotation keeps distances
    v1 = rot[1] - np.array([0.5, 0, -0.5], np.float32)
    assert np.allclose(np.linalg.norm(base[1], axis=1), np.linalg.norm(v1, axis=1), rtol=1e-5, atol=1e-6)


def test_demo_galaxy_runs_with_reference_parameters(torch_cuda, engine):
    """The reference's own run: theta 0.7, eps 0.02, dt 0.08, G 1."""
    pos, vel = engine.demo_galaxy(100_000, seed=0, device=True)
    with engine.Simulation(100_000, engine.Params()) as sim:
        sim.load(pos, vel)
        sim.step(10)
        assert sim.stats()["error_bits"] == 0
