"""The C ABI without a GPU: the library loads, exports every function that
include/*.h declares, struct layouts match the reference's, argument checks
reject bad input before touching the device, and the seeded initial
conditions are reproducible."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> set[str]:
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        text = re.sub(r"//[^\n]*", "", text)
        for m in re.finditer(r"\b([A-Za-z_]\w*)\s*\(([^;{}()]*(?:\([^()]*\)[^;{}()]*)*)\)\s*;", text):
            name = m.group(1)
            if name in {"sizeof", "offsetof", "BH_STATIC_ASSERT", "_Static_assert", "static_assert"}:
                continue
            names.add(name)
    return names


def test_every_declared_function_is_exported(engine):
    lib = engine.lib()
    names = declared_functions()
    assert len(names) > 50
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert missing == []


def test_bindings_cover_the_headers(engine):
    from cudagravitydemo_b200 import _native
    assert declared_functions() == set(_native.SIGNATURES)


def test_struct_layouts(engine):
    from cudagravitydemo_b200 import _native as N
    assert C.sizeof(N.Node) == 80 and N.Node.massData.offset == 64 and N.Node.child.offset == 20
    assert N.Node.treeLevel.offset == 52 and N.Node.parentIndex.offset == 8
    assert C.sizeof(N.TreeState) == 304 and C.sizeof(N.WorldBox) == 20
    assert engine.NODE_DTYPE.itemsize == 80 and engine.NODE_DTYPE.fields["mass"][1] == 64


def test_params_defaults_are_the_reference_values(engine):
    from cudagravitydemo_b200 import _native as N
    p = N.Params()
    engine.lib().bh_params_default(C.byref(p))
    assert (p.bitsPerAxis, p.leafSize, p.groupWidth) == (21, 1, 32)
    assert np.float32(p.theta) == np.float32(0.7) and p.G == 1.0  # units.c:3-4
    assert np.float32(p.eps) == np.float32(0.02) and np.float32(p.dt) == np.float32(0.08)


def test_argument_checks_without_device(engine):
    lib = engine.lib()
    from cudagravitydemo_b200 import _native as N
    h = C.c_void_p()
    p = N.Params()
    lib.bh_params_default(C.byref(p))
    assert lib.bh_sim_create(C.byref(h), 0, C.byref(p), None) == 1
    assert lib.bh_sim_create(C.byref(h), -5, C.byref(p), None) == 1
    bad = N.Params.from_buffer_copy(p)
    bad.bitsPerAxis = 22
    assert lib.bh_sim_create(C.byref(h), 100, C.byref(bad), None) == 1
    bad.bitsPerAxis = 21
    bad.theta = -1.0
    assert lib.bh_sim_create(C.byref(h), 100, C.byref(bad), None) == 1
    assert lib.bh_sim_step(None, 1) == 1
    assert lib.bh_sim_step_host(None, None, None, 10, 1) == 1
    assert lib.bh_sim_step_host_sorted(None, None, None, None, 10, 1) == 1
    assert lib.bh_sorter_create(C.byref(h), 0) == 1
    assert lib.bh_initialise_tree(None, 10, 10, 1) == 1
    assert lib.bh_morton_encode(None, None, None, 10, N.WorldBox(), 21, None) == 1
    assert lib.roundNumberToMultiple(100, 32) == 128 and lib.roundNumberToMultiple(96, 32) == 96
    out = [C.c_int() for _ in range(6)]
    lib.blockNumCalculator(*[C.byref(o) for o in out], 100)
    acc_blocks, tree_blocks, int_blocks, padded, ithreads, tthreads = (o.value for o in out)
    assert (padded, acc_blocks, int_blocks, tree_blocks) == (128, 5, 1, 1)  # basicGravity.cu:374-427


def test_status_strings(engine):
    for code in range(10):
        assert engine.status_string(code)
    assert engine.status_string(6) == "tree node capacity exceeded"


def test_initial_conditions_seeded(engine):
    a = engine.plummer(4096, seed=9)
    b = engine.plummer(4096, seed=9)
    c = engine.plummer(4096, seed=10)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    p, v = a
    assert abs(p[:, 3].sum() - 1.0) < 1e-5
    assert np.abs((p[:, :3] * p[:, 3:]).sum(0)).max() < 1e-5  # centre of mass at the origin
    assert np.abs((v * p[:, 3:]).sum(0)).max() < 1e-5        # no bulk velocity
    # virial ratio of a Plummer sphere, 2K/|W| ~ 1 (K from the velocities,
    # W = -3 pi G M^2 / (32 a))
    K = 0.5 * (p[:, 3] * (v ** 2).sum(1)).sum()
    W = -3 * np.pi / 32
    assert 0.85 < 2 * K / abs(W) < 1.15


def test_disk_galaxy_shape(engine):
    p, v = engine.disk_galaxy(20000, seed=1)
    assert abs(p[:, 3].sum() - 1.0) < 1e-4
    R = np.hypot(p[:, 0], p[:, 1])
    disk = np.abs(p[:, 2]) < 0.5
    assert R.max() <= 5.0 + 1e-3 + 0.1  # disk truncated at 5 R_d (bulge within 20 a = 4)
    assert np.median(np.abs(p[disk, 2])) < 0.2  # thin sech^2 disk, z0 = 0.1
    # disk bodies rotate counter-clockwise about +z
    Lz = p[:, 0] * v[:, 1] - p[:, 1] * v[:, 0]
    assert (Lz[disk & (R > 1)] > 0).mean() > 0.9


def test_merger_two_galaxies(engine):
    p, v = engine.merger(8000, separation=20.0)
    left, right = p[:4000], p[4000:]
    assert abs(np.median(left[:, 0]) - np.median(right[:, 0]) + 20.0) < 1.0
    assert abs((p[:, :3] * p[:, 3:]).sum(0)).max() < 1e-3


def test_c_driver_built_and_rejects_bad_options():
    """The C simulation program links against the library; argument errors
    exit with status 2 before any device call."""
    import subprocess
    from pathlib import Path
    drv = Path(__file__).resolve().parent.parent / "cudagravitydemo_b200" / "gravity_sim"
    assert drv.exists(), "build the package: python -m cudagravitydemo_b200.build"
    r = subprocess.run([str(drv), "-bogus", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown option" in r.stderr
    r = subprocess.run([str(drv), "-ic", "nonsense", "-n", "16"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown initial conditions" in r.stderr
