"""B200-native Barnes-Hut gravity engine.

The engine is libbh_b200.so (hand-written sm_100a kernels behind a C ABI,
include/*.h).  This package is a thin Python mirror of that ABI:

* :class:`Simulation` — device-resident simulation (``bh_sim_*``): whole
  steps (box, keys, sort, reorder, octree, walk + kick-drift) replayed as one
  CUDA graph per step;
* :class:`TreeState` — the reference's drop-in entry points
  (``initialiseTree`` / ``buildTree`` / ``calculateAcceleration`` /
  ``positionUpdater``) on caller-owned device buffers;
* :func:`plummer`, :func:`disk_galaxy`, :func:`merger` — seeded initial
  conditions;
* :func:`radix_sort_pairs`, :func:`morton_encode`, :func:`world_box` — the
  individual stages.

Device arrays are torch CUDA tensors (PyTorch supplies device memory and
streams; all arithmetic runs in this library's kernels).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _native as N

__all__ = ["BHError", "Params", "Simulation", "TreeState", "plummer", "disk_galaxy", "merger",
           "radix_sort_pairs", "morton_encode", "world_box", "NODE_DTYPE", "lib", "status_string",
           "device_to_host"]

NODE_DTYPE = np.dtype([("path", "<u8"), ("parent", "<i4"), ("first", "<i4"), ("count", "<i4"),
                       ("child", "<i4", (8,)), ("level", "<i4"), ("pad", "<i4", (2,)), ("mass", "<f4", (4,))])
assert NODE_DTYPE.itemsize == 80

STATUS = {0: "BH_OK", 1: "BH_ERR_INVALID", 2: "BH_ERR_ALLOC", 3: "BH_ERR_CUDA", 4: "BH_ERR_DEGENERATE_BOX",
          5: "BH_ERR_NONFINITE", 6: "BH_ERR_TREE_OVERFLOW", 7: "BH_ERR_STACK_OVERFLOW", 8: "BH_ERR_TIMEOUT",
          9: "BH_ERR_INTERNAL"}


def lib() -> C.CDLL:
    return N.load()


def status_string(code: int) -> str:
    return lib().bh_status_string(code).decode()


class BHError(RuntimeError):
    def __init__(self, code: int, where: str = ""):
        self.code = code
        self.name = STATUS.get(code, str(code))
        detail = lib().bh_cuda_error_string().decode() if code == 3 else ""
        super().__init__(f"{where}: {self.name} ({status_string(code)}) {detail}".strip())


def _check(code: int, where: str) -> None:
    if code != 0:
        raise BHError(code, where)


def _ptr(t) -> int:
    """Device/host address of a torch tensor or numpy array (None -> 0)."""
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    return t.ctypes.data


def _stream(stream) -> int:
    if stream is None:
        return 0
    return getattr(stream, "cuda_stream", stream)


@dataclass
class Params:
    """bh_params.  Defaults are the reference's (units.c, basicGravity.cu)."""
    bits_per_axis: int = 21
    leaf_size: int = 1
    group_width: int = 32
    theta: float = 0.7
    eps: float = 0.02
    G: float = 1.0
    dt: float = 0.08
    compensated: bool = True
    export_nodes: bool = False
    mac_mode: int = 0          # 0 fixed theta, 1 relative (uniform alpha), 2 learned (MLP)
    alpha: float = 1e-3        # mode 1 budget
    err_target: float = 5e-3   # mode 2 target

    def to_c(self) -> N.Params:
        return N.Params(self.bits_per_axis, self.leaf_size, self.group_width, self.theta, self.eps, self.G,
                        self.dt, int(self.compensated), int(self.export_nodes), self.mac_mode, self.alpha,
                        self.err_target)


# ------------------------------------------------------------ initial conditions
def _host_bodies(n: int):
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 3), np.float32)
    return pos, vel


def plummer(n: int, M: float = 1.0, a: float = 1.0, G: float = 1.0, seed: int = 0):
    """Seeded Plummer sphere: (pos[n,4] with mass in w, vel[n,3]) float32."""
    pos, vel = _host_bodies(n)
    _check(lib().bh_ic_plummer(pos.ctypes.data, vel.ctypes.data, n, M, a, G, seed), "bh_ic_plummer")
    return pos, vel


def galaxy_params(**kw) -> N.GalaxyParams:
    g = N.GalaxyParams()
    lib().bh_galaxy_params_default(C.byref(g))
    for k, v in kw.items():
        setattr(g, k, v)
    return g


def disk_galaxy(n: int, seed: int = 1, **kw):
    """Seeded exponential disk + Hernquist bulge (defaults: the N=1M disk)."""
    pos, vel = _host_bodies(n)
    g = galaxy_params(**kw)
    _check(lib().bh_ic_disk_galaxy(pos.ctypes.data, vel.ctypes.data, n, C.byref(g), seed), "bh_ic_disk_galaxy")
    return pos, vel


def merger(n: int, separation: float = 20.0, pericentre: float = 2.0, inclination: float = 30.0, seed: int = 3,
           **kw):
    """Two disk galaxies on a parabolic orbit."""
    pos, vel = _host_bodies(n)
    g = galaxy_params(**kw)
    _check(lib().bh_ic_merger(pos.ctypes.data, vel.ctypes.data, n, C.byref(g), separation, pericentre,
                              inclination, seed), "bh_ic_merger")
    return pos, vel


def demo_galaxy(n: int, seed: int = 0, device: bool = False, **kw):
    """The reference program's own demo galaxy (bh_ic_demo), seeded, built on
    the device: 80% exponential disk, 20% uniform-radius halo, total mass 5.
    Returns torch CUDA tensors when device=True, else host numpy arrays."""
    import torch
    prm = N.DemoParams()
    lib().bh_demo_params_default(C.byref(prm))
    for k, v in kw.items():
        if k in ("rotation", "centre", "velocity"):
            getattr(prm, k)[:] = [float(x) for x in v]
        else:
            setattr(prm, k, v)
    pos = torch.empty((n, 4), dtype=torch.float32, device="cuda")
    vel = torch.empty((n, 3), dtype=torch.float32, device="cuda")
    _check(lib().bh_ic_demo(_ptr(pos), _ptr(vel), n, C.byref(prm), seed, None), "bh_ic_demo")
    if device:
        return pos, vel
    return pos.cpu().numpy(), vel.cpu().numpy()


# ------------------------------------------------------------------ stages
def world_box(pos, bits: int = 21, stream=None):
    """Bounding box + Morton grid mapping of device positions (float32 [n,4])."""
    box = N.WorldBox()
    mn, mx = N.Float3(), N.Float3()
    _check(lib().bh_world_box(_ptr(pos), pos.shape[0], bits, C.byref(box), C.byref(mn), C.byref(mx),
                              _stream(stream)), "bh_world_box")
    return box, (mn.x, mn.y, mn.z), (mx.x, mx.y, mx.z)


def morton_encode(pos, keys, idx, box: N.WorldBox, bits: int = 21, stream=None) -> None:
    """keys (int64 view of uint64) and idx (int32) for device positions."""
    _check(lib().bh_morton_encode(_ptr(pos), _ptr(keys), _ptr(idx), pos.shape[0], box, bits, _stream(stream)),
           "bh_morton_encode")


def radix_sort_pairs(keys_in, vals_in, keys_out, vals_out, key_bits: int = 64, stream=None) -> None:
    """Stable sort of device (uint64 key, uint32 value) pairs (int64/int32 tensors)."""
    n = keys_in.shape[0]
    sorter = C.c_void_p()
    _check(lib().bh_sorter_create(C.byref(sorter), n), "bh_sorter_create")
    try:
        _check(lib().bh_radix_sort_pairs(sorter, _ptr(keys_in), _ptr(keys_out), _ptr(vals_in), _ptr(vals_out), n,
                                         key_bits, _stream(stream)), "bh_radix_sort_pairs")
        # device-side errors of the passes (a look-back wait that gave up)
        _check(lib().bh_sorter_errors(sorter, None, _stream(stream)), "bh_sorter_errors")
    finally:
        lib().bh_sorter_destroy(sorter)


class _DeviceView:
    """Exposes a raw device address through __cuda_array_interface__."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3, "strides": None}


def device_to_host(ptr: int, nbytes: int) -> np.ndarray:
    """Copy nbytes of device memory at ptr into a new uint8 numpy array."""
    import torch
    if nbytes == 0:
        return np.zeros(0, np.uint8)
    t = torch.as_tensor(_DeviceView(ptr, nbytes), device="cuda")
    torch.cuda.synchronize()
    return t.cpu().numpy().copy()


def fma_peak_tflops(reps: int = 5, stream=None) -> float:
    """Measured FP32 FMA throughput of the current GPU (TFLOP/s)."""
    t = C.c_float()
    _check(lib().bh_fma_peak_tflops(reps, C.byref(t), _stream(stream)), "bh_fma_peak_tflops")
    return float(t.value)


# ------------------------------------------------------------- drop-in tree
class TreeState:
    """The reference's treeState driven through the drop-in entry points.

    ``pos``/``vel`` are caller device buffers (torch float32 [>=n,4] / [>=n,3]).
    ``build()`` swaps them with the state's second buffers like the reference's
    buildTree, so the current buffers are always ``self.pos`` / ``self.vel``.
    """

    def __init__(self, n: int, pos, vel):
        import torch
        self.n = n
        self.state = N.TreeState()
        padded = ((n + 31) // 32) * 32
        _check(lib().bh_initialise_tree(C.byref(self.state), n, padded, (padded + 255) // 256), "bh_initialise_tree")
        self._caller = (pos, vel)  # keep the caller's tensors alive while the state may hold them
        self._pos = C.c_void_p(_ptr(pos))
        self._vel = C.c_void_p(_ptr(vel))
        self._torch = torch

    @property
    def pos_ptr(self) -> int:
        return self._pos.value

    @property
    def vel_ptr(self) -> int:
        return self._vel.value

    def build(self, stream=None) -> None:
        _check(lib().bh_build_tree(C.byref(self.state), C.byref(self._pos), C.byref(self._vel), _stream(stream)),
               "bh_build_tree")

    def accelerations(self, acc, eps: float, G: float, theta: float, stream=None) -> None:
        _check(lib().bh_calculate_acceleration(self._pos, C.byref(self.state), _ptr(acc), eps * eps, G, theta,
                                               self.n, _stream(stream)), "bh_calculate_acceleration")

    def kick_drift(self, acc, dt: float, stream=None) -> None:
        _check(lib().bh_position_updater(self._pos, self._vel, _ptr(acc), self.n, dt, _stream(stream)),
               "bh_position_updater")

    def _copy(self, ptr: int, nbytes: int) -> np.ndarray:
        return device_to_host(ptr, nbytes)

    def host_pos(self) -> np.ndarray:
        return self._copy(self.pos_ptr, 16 * self.n).view(np.float32).reshape(self.n, 4)

    def host_vel(self) -> np.ndarray:
        return self._copy(self.vel_ptr, 12 * self.n).view(np.float32).reshape(self.n, 3)

    def host_nodes(self) -> np.ndarray:
        count = self.node_count()
        return self._copy(self.state.nodes, 80 * count).view(NODE_DTYPE)

    def host_keys(self, which: str = "out") -> np.ndarray:
        ptr = self.state.mortonOut if which == "out" else self.state.mortonIn
        return self._copy(ptr, 8 * self.n).view(np.uint64)

    def host_index(self, which: str = "out") -> np.ndarray:
        ptr = self.state.indexOut if which == "out" else self.state.indexIn
        return self._copy(ptr, 4 * self.n).view(np.uint32)

    def node_count(self) -> int:
        d = self.state.deepestLevel
        return self.state.levelOffsets[d] + self.state.levelCount[d]

    def levels(self):
        d = self.state.deepestLevel
        return d, list(self.state.levelOffsets)[: d + 1], list(self.state.levelCount)[: d + 1]

    def close(self) -> None:
        if self.state.builder:
            lib().bh_destroy_tree(C.byref(self.state))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def diagnostics_dict(d) -> dict:
    return {"mass": d.mass, "com": list(d.com), "com_vel": list(d.comVel), "momentum": list(d.momentum),
            "angular_momentum": list(d.angularMomentum), "kinetic": d.kinetic, "potential": d.potential,
            "total": d.total}


def diagnostics(pos, vel, eps: float, G: float = 1.0, potential: bool = True, stream=None) -> dict:
    """FP64 conserved quantities of device bodies (torch tensors pos [n,4], vel [n,3])."""
    d = N.Diagnostics()
    _check(lib().bh_diagnostics_f64(_ptr(pos), _ptr(vel), int(pos.shape[0]), float(eps), float(G), int(potential),
                                    C.byref(d), _stream(stream)), "bh_diagnostics_f64")
    return diagnostics_dict(d)


# ---------------------------------------------------------------- simulation
class Simulation:
    """Device-resident simulation (bh_sim_*)."""

    def __init__(self, capacity: int, params: Params | None = None, stream=None, counts=None):
        """counts: body counts of the independent systems of a batch
        (bh_sim_create_batch); capacity is then their sum."""
        self.params = params or Params()
        self._h = C.c_void_p()
        p = self.params.to_c()
        if counts is not None:
            cnt = np.ascontiguousarray(counts, np.int32)
            capacity = int(cnt.sum())
            _check(lib().bh_sim_create_batch(C.byref(self._h), len(cnt), cnt.ctypes.data, C.byref(p),
                                             _stream(stream)), "bh_sim_create_batch")
        else:
            _check(lib().bh_sim_create(C.byref(self._h), capacity, C.byref(p), _stream(stream)), "bh_sim_create")
        self.capacity = capacity
        self.n = 0
        self._mlp = False
        if self.params.mac_mode == 2:
            self.set_mac_mlp()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    @property
    def stream(self) -> int:
        return lib().bh_sim_stream(self._h) or 0

    def set_params(self, params: Params) -> None:
        p = params.to_c()
        _check(lib().bh_sim_set_params(self._h, C.byref(p)), "bh_sim_set_params")
        self.params = params
        if params.mac_mode == 2 and not self._mlp:
            self.set_mac_mlp()

    def set_mac_mlp(self, params: np.ndarray | None = None) -> None:
        """Loads the MLP of the learned criterion (default: the trained
        weights shipped in cudagravitydemo_b200/data)."""
        from .learned import load_weights
        w = load_weights() if params is None else np.ascontiguousarray(params, np.float32)
        assert w.size == N.MLP_PARAMS
        _check(lib().bh_sim_set_mac_mlp(self._h, w.ctypes.data), "bh_sim_set_mac_mlp")
        self._mlp = True

    def group_features(self):
        """(features [groups, 7], body ids in walk order [n]) of the current
        state, as the learned walk sees them."""
        g = (self.n + 31) // 32
        feat = np.zeros((g, N.GROUP_FEATURES), np.float32)
        ids = np.zeros(self.n, np.uint32)
        _check(lib().bh_sim_group_features(self._h, feat.ctypes.data, ids.ctypes.data, 1), "bh_sim_group_features")
        return feat, ids

    def group_params(self) -> np.ndarray:
        """(theta, alpha) per group chosen by the last learned walk."""
        gp = np.zeros(((self.n + 31) // 32, 2), np.float32)
        _check(lib().bh_sim_group_params(self._h, gp.ctypes.data, 1), "bh_sim_group_params")
        return gp

    def root_f64(self) -> dict:
        """The FP64 mass, centre of mass and bounding box of all bodies, from
        the last build (bh_sim_root_f64)."""
        out = np.zeros(10, np.float64)
        _check(lib().bh_sim_root_f64(self._h, out.ctypes.data), "bh_sim_root_f64")
        return {"mass": float(out[0]), "com": out[1:4].copy(), "min": out[4:7].copy(), "max": out[7:10].copy()}

    def group_lengths(self) -> np.ndarray:
        """Interaction-list length of every walk group of the last walk (walk order)."""
        g = C.c_int()
        probe = np.zeros(1, np.int32)
        lib().bh_sim_group_lengths(self._h, probe.ctypes.data, 0, C.byref(g), 1)  # the group count
        lens = np.zeros(max(g.value, 1), np.int32)
        _check(lib().bh_sim_group_lengths(self._h, lens.ctypes.data, len(lens), C.byref(g), 1),
               "bh_sim_group_lengths")
        return lens[: g.value].copy()

    def load(self, pos, vel) -> None:
        """Load bodies from host numpy arrays or device torch tensors."""
        host = isinstance(pos, np.ndarray)
        if host:
            pos = np.ascontiguousarray(pos, np.float32)
            vel = np.ascontiguousarray(vel, np.float32)
        n = pos.shape[0]
        _check(lib().bh_sim_load(self._h, _ptr(pos), _ptr(vel), n, int(host)), "bh_sim_load")
        self.n = n

    def store(self):
        """Current state in body-id order, as host arrays."""
        pos, vel = _host_bodies(self.n)
        _check(lib().bh_sim_store(self._h, pos.ctypes.data, vel.ctypes.data, 1), "bh_sim_store")
        return pos, vel

    def step(self, nsteps: int = 1) -> None:
        _check(lib().bh_sim_step(self._h, nsteps), "bh_sim_step")

    def step_host(self, pos: np.ndarray, vel: np.ndarray, nsteps: int = 1) -> None:
        """End to end: host arrays in, nsteps on the device, results back in place."""
        assert pos.dtype == np.float32 and vel.dtype == np.float32 and pos.flags.c_contiguous
        _check(lib().bh_sim_step_host(self._h, pos.ctypes.data, vel.ctypes.data, pos.shape[0], nsteps),
               "bh_sim_step_host")
        self.n = pos.shape[0]

    def step_host_sorted(self, pos: np.ndarray, vel: np.ndarray, ids: np.ndarray, nsteps: int = 1) -> None:
        """End to end in frame order: host arrays (any order, with their body
        ids) in, nsteps on the device, the state after the last step back in
        place in that step's Morton order with its ids (bh_sim_step_host_sorted).
        Page-locked arrays (e.g. numpy views of pinned torch tensors) are
        written by the walk itself."""
        n = pos.shape[0]
        assert pos.dtype == np.float32 and vel.dtype == np.float32 and ids.dtype == np.uint32
        assert pos.shape == (n, 4) and vel.shape == (n, 3) and ids.shape == (n,)
        assert pos.flags.c_contiguous and vel.flags.c_contiguous and ids.flags.c_contiguous
        _check(lib().bh_sim_step_host_sorted(self._h, pos.ctypes.data, vel.ctypes.data, ids.ctypes.data, n, nsteps),
               "bh_sim_step_host_sorted")
        self.n = n

    def accelerations(self) -> np.ndarray:
        acc = np.zeros((self.n, 3), np.float32)
        _check(lib().bh_sim_accelerations(self._h, acc.ctypes.data, 1), "bh_sim_accelerations")
        return acc

    def diagnostics(self, potential: bool = True) -> dict:
        """FP64 conserved quantities of the current state (bh_sim_diagnostics)."""
        d = N.Diagnostics()
        _check(lib().bh_sim_diagnostics(self._h, int(potential), C.byref(d)), "bh_sim_diagnostics")
        return diagnostics_dict(d)

    def tune(self, trial_steps: int = 5) -> dict:
        """Autotune the bucket size on the current state (bh_sim_tune); the
        choice is kept, the state is restored."""
        r = N.TuneResult()
        _check(lib().bh_sim_tune(self._h, trial_steps, C.byref(r)), "bh_sim_tune")
        self.params = Params(**{**self.params.__dict__, "leaf_size": r.leafSize, "group_width": r.groupWidth})
        return {"leaf_size": r.leafSize, "group_width": r.groupWidth, "stack_entries": r.stackEntries,
                "ms_per_step": {(int(r.leafSizes[k]), int(r.groupWidths[k]), int(r.stackEntriesTried[k])):
                                float(r.msPerStep[k]) for k in range(r.candidates)}}

    def set_walk_stack(self, entries: int) -> None:
        """Walk stack entries per warp in shared memory (0: the default)."""
        _check(lib().bh_sim_set_walk_stack(self._h, entries), "bh_sim_set_walk_stack")

    def walk_stack(self) -> int:
        return lib().bh_sim_walk_stack(self._h)

    def system_offsets(self) -> np.ndarray | None:
        """Body offsets of the systems of a batch (systems + 1), or None."""
        k = C.c_int()
        _check(lib().bh_sim_systems(self._h, C.byref(k), None), "bh_sim_systems")
        if k.value == 0:
            return None
        off = np.zeros(k.value + 1, np.int32)
        _check(lib().bh_sim_systems(self._h, C.byref(k), off.ctypes.data), "bh_sim_systems")
        return off

    def system_diagnostics(self, potential: bool = True) -> list[dict]:
        """FP64 conserved quantities of every system of a batch."""
        off = self.system_offsets()
        k = 1 if off is None else len(off) - 1
        arr = (N.Diagnostics * k)()
        _check(lib().bh_sim_system_diagnostics(self._h, int(potential), arr), "bh_sim_system_diagnostics")
        return [diagnostics_dict(d) for d in arr]

    def accel_magnitudes(self) -> np.ndarray:
        """|a| of every body from the last step, in the device (Morton) order
        of device_state(): the input of the relative opening criterion."""
        out = np.zeros(self.n, np.float32)
        _check(lib().bh_sim_accel_magnitudes(self._h, out.ctypes.data, 1), "bh_sim_accel_magnitudes")
        return out

    def stats(self, check: bool = True) -> dict:
        st = N.Stats()
        code = lib().bh_sim_stats(self._h, C.byref(st))
        if check:
            _check(code, "bh_sim_stats")
        d = st.deepestLevel
        return {"interactions": st.interactions, "nodes_tested": st.nodesTested, "node_count": st.nodeCount,
                "deepest_level": d, "level_offsets": list(st.levelOffsets)[: d + 2],
                "level_count": list(st.levelCount)[: d + 2], "error_bits": st.errorBits, "max_stack": st.maxStack,
                "group_votes": st.groupVotes, "status": code}

    def profile(self, nsteps: int = 3) -> dict:
        """Mean ms per stage over nsteps real steps (events between stages)."""
        names = ["keys", "sort", "reorder", "tree_count", "tree_scan", "tree_nodes", "tree_mass", "criterion", "walk"]
        ms = (C.c_float * len(names))()
        _check(lib().bh_sim_profile(self._h, nsteps, ms), "bh_sim_profile")
        out = dict(zip(names, [float(x) for x in ms]))
        out["tree"] = out["tree_count"] + out["tree_scan"] + out["tree_nodes"] + out["tree_mass"]
        return out

    def kernels_per_step(self) -> int:
        return lib().bh_sim_kernels_per_step(self._h)

    def device_state(self):
        pos, vel, ids, n = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_int()
        _check(lib().bh_sim_device_state(self._h, C.byref(pos), C.byref(vel), C.byref(ids), C.byref(n)),
               "bh_sim_device_state")
        return pos.value, vel.value, ids.value, n.value

    def tree(self) -> N.TreeState:
        ts = C.POINTER(N.TreeState)()
        _check(lib().bh_sim_tree(self._h, C.byref(ts)), "bh_sim_tree")
        return ts.contents

    def close(self) -> None:
        if self._h:
            lib().bh_sim_destroy(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
