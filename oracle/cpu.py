"""Python binding of the C oracle (liboracle.so) and the reference harness
(libref.so).  TEST INFRASTRUCTURE ONLY.

Arrays are numpy: positions float32 [n,4] (mass in column 3), velocities and
accelerations float32 [n,3], keys uint64, indices uint32, nodes NODE_DTYPE.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libref.so"

NODE_DTYPE = np.dtype([("path", "<u8"), ("parent", "<i4"), ("first", "<i4"), ("count", "<i4"),
                       ("child", "<i4", (8,)), ("level", "<i4"), ("pad", "<i4", (2,)), ("mass", "<f4", (4,))])

D2_REF, D2_ALT, D2_PLAIN = 0, 1, 2  # d^2 fusion orders; D2_REF is the reference's


class GalaxyParams(C.Structure):  # bh_galaxy_params (include/bh_api.h)
    _fields_ = [("diskMass", C.c_float), ("diskScale", C.c_float), ("diskHeight", C.c_float),
                ("diskTrunc", C.c_float), ("bulgeMass", C.c_float), ("bulgeScale", C.c_float),
                ("bulgeTrunc", C.c_float), ("dispersion", C.c_float), ("G", C.c_float)]


class WorldBox(C.Structure):
    _fields_ = [("minX", C.c_float), ("minY", C.c_float), ("minZ", C.c_float), ("extent", C.c_float),
                ("scale", C.c_float)]


_P = C.c_void_p
_I = C.c_int
_F = C.c_float
_lib = None
_ref = None


def _a(x) -> int:
    return x.ctypes.data


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            from . import build
            build.build_oracle()
        L = C.CDLL(str(ORACLE_LIB), mode=os.RTLD_LOCAL)
        sig = {
            "orc_bbox": (None, [_P, _I, _P, _P]),
            "orc_world_box": (None, [_P, _P, _I, C.POINTER(WorldBox)]),
            "orc_expand_bits": (C.c_uint64, [C.c_uint64, _I]),
            "orc_morton_encode": (None, [_P, _I, WorldBox, _I, _P, _P]),
            "orc_sort_pairs": (None, [_P, _P, _P, _P, _I]),
            "orc_reorder": (None, [_P, _P, _P, _P, _P, _I]),
            "orc_build_tree": (_I, [_P, _P, _I, _I, _P, _I, _P, _P, _P]),
            "orc_walk": (C.c_longlong, [_P, _I, _P, _F, _F, _F, _F, _I, _I, _P]),
            "orc_walk_list_lengths": (None, [_P, _I, _P, _F, _F, _I, _I, _P]),
            "orc_walk_relative": (C.c_longlong, [_P, _I, _P, _F, _F, _F, _F, _F, _P, _P, _I, _I, _P]),
            "orc_walk_buckets": (C.c_longlong, [_P, _I, _P, _F, _F, _F, _F, _I, _I, _P]),
            "orc_walk_sample": (C.c_longlong, [_P, _I, _P, _F, _F, _F, _F, _I, _I, _I, _P]),
            "orc_walk_groups_sample": (C.c_longlong, [_P, _I, _P, _F, _F, _F, _F, _F, _P, _P, _I, _I, _P, _P]),
            "orc_kick_drift": (None, [_P, _P, _P, _I, _F]),
            "orc_direct_sum_f64": (None, [_P, _I, _P, _I, C.c_double, C.c_double, _P]),
            "orc_step_scratch_bytes": (C.c_size_t, [_I]),
            "orc_step": (_I, [_P, _P, _I, _I, _F, _F, _F, _F, _I, _I, _P, _P, _P, C.POINTER(C.c_longlong)]),
            "orc_num_threads": (_I, []),
            "orc_diagnostics_f64": (None, [_P, _P, _I, C.c_double, _I, _P]),
            "bh_ic_plummer": (_I, [_P, _P, _I, _F, _F, _F, C.c_uint64]),
            "bh_galaxy_params_default": (None, [C.POINTER(GalaxyParams)]),
            "bh_ic_disk_galaxy": (_I, [_P, _P, _I, C.POINTER(GalaxyParams), C.c_uint64]),
            "bh_ic_merger": (_I, [_P, _P, _I, C.POINTER(GalaxyParams), _F, _F, _F, C.c_uint64]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def plummer(n: int, seed: int = 0, M: float = 1.0, a: float = 1.0, G: float = 1.0):
    """The seeded Plummer sphere of host/ics.c (the engine's generator, built
    into the oracle library)."""
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 3), np.float32)
    if lib().bh_ic_plummer(_a(pos), _a(vel), n, M, a, G, seed) != 0:
        raise ValueError("bh_ic_plummer")
    return pos, vel


def disk_galaxy(n: int, seed: int = 1):
    """The seeded disk + bulge of host/ics.c (default parameters)."""
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 3), np.float32)
    g = GalaxyParams()
    lib().bh_galaxy_params_default(C.byref(g))
    if lib().bh_ic_disk_galaxy(_a(pos), _a(vel), n, C.byref(g), seed) != 0:
        raise ValueError("bh_ic_disk_galaxy")
    return pos, vel


def merger(n: int, seed: int = 3, separation: float = 20.0, pericentre: float = 2.0, inclination: float = 30.0):
    """The seeded two-disk merger of host/ics.c."""
    pos = np.zeros((n, 4), np.float32)
    vel = np.zeros((n, 3), np.float32)
    g = GalaxyParams()
    lib().bh_galaxy_params_default(C.byref(g))
    if lib().bh_ic_merger(_a(pos), _a(vel), n, C.byref(g), separation, pericentre, inclination, seed) != 0:
        raise ValueError("bh_ic_merger")
    return pos, vel


def num_threads() -> int:
    return lib().orc_num_threads()


def bbox(pos: np.ndarray):
    mn = np.zeros(3, np.float32)
    mx = np.zeros(3, np.float32)
    lib().orc_bbox(_a(pos), pos.shape[0], _a(mn), _a(mx))
    return mn, mx


def world_box(mn: np.ndarray, mx: np.ndarray, bits: int = 21) -> WorldBox:
    box = WorldBox()
    lib().orc_world_box(_a(np.ascontiguousarray(mn, np.float32)), _a(np.ascontiguousarray(mx, np.float32)),
                        bits, C.byref(box))
    return box


def expand_bits(v: int, bits: int = 21) -> int:
    return lib().orc_expand_bits(v, bits)


def morton(pos: np.ndarray, box: WorldBox, bits: int = 21):
    n = pos.shape[0]
    keys = np.zeros(n, np.uint64)
    idx = np.zeros(n, np.uint32)
    lib().orc_morton_encode(_a(pos), n, box, bits, _a(keys), _a(idx))
    return keys, idx


def sort_pairs(keys: np.ndarray, vals: np.ndarray):
    n = keys.shape[0]
    ko = np.zeros(n, np.uint64)
    vo = np.zeros(n, np.uint32)
    lib().orc_sort_pairs(_a(np.ascontiguousarray(keys, np.uint64)), _a(np.ascontiguousarray(vals, np.uint32)),
                         _a(ko), _a(vo), n)
    return ko, vo


def reorder(pos, vel, idx):
    n = pos.shape[0]
    po = np.zeros_like(pos)
    vo = np.zeros_like(vel)
    lib().orc_reorder(_a(pos), _a(vel), _a(np.ascontiguousarray(idx, np.uint32)), _a(po), _a(vo), n)
    return po, vo


def build_tree(sorted_keys: np.ndarray, sorted_pos: np.ndarray, bits: int = 21, max_nodes: int | None = None):
    """Returns (nodes[count], level_offsets[23], level_count[23], deepest); count = -1 on overflow."""
    n = sorted_keys.shape[0]
    max_nodes = max_nodes if max_nodes is not None else 8 * n
    nodes = np.zeros(max_nodes, NODE_DTYPE)
    lo = np.zeros(23, np.int32)
    lc = np.zeros(23, np.int32)
    deep = C.c_int()
    count = lib().orc_build_tree(_a(sorted_keys), _a(sorted_pos), n, bits, _a(nodes), max_nodes, _a(lo), _a(lc),
                                 C.byref(deep))
    return (nodes[:count] if count >= 0 else nodes[:0]), lo, lc, deep.value, count


def walk(pos, nodes, ext_x: float, eps: float, G: float, theta: float, group: int = 32, d2order: int = 0):
    n = pos.shape[0]
    acc = np.zeros((n, 3), np.float32)
    nodes = np.ascontiguousarray(nodes)
    inter = lib().orc_walk(_a(pos), n, _a(nodes), np.float32(ext_x), np.float32(eps) * np.float32(eps), G, theta,
                           group, d2order, _a(acc))
    return acc, inter


def walk_buckets(pos, nodes, ext_x: float, eps: float, G: float, theta: float, leaf_size: int, width: int = 32):
    """The group walk with bucket leaves (at most leaf_size bodies)."""
    n = pos.shape[0]
    acc = np.zeros((n, 3), np.float32)
    inter = lib().orc_walk_buckets(_a(pos), n, _a(np.ascontiguousarray(nodes)), np.float32(ext_x),
                                   np.float32(eps) * np.float32(eps), G, theta, leaf_size, width, _a(acc))
    return acc, inter


def walk_relative(pos, nodes, ext_x: float, eps: float, G: float, theta: float, alpha: float, amag,
                  group_param=None, d2order: int = 0, width: int = 32):
    """The group walk with the relative opening criterion (sorted bodies,
    |a| of each from the previous step); returns (acc, interactions)."""
    n = pos.shape[0]
    acc = np.zeros((n, 3), np.float32)
    amag = np.ascontiguousarray(amag, np.float32)
    gp = None if group_param is None else np.ascontiguousarray(group_param, np.float32)
    inter = lib().orc_walk_relative(_a(pos), n, _a(np.ascontiguousarray(nodes)), np.float32(ext_x),
                                    np.float32(eps) * np.float32(eps), G, theta, alpha, _a(amag),
                                    None if gp is None else _a(gp), d2order, width, _a(acc))
    return acc, inter


def walk_sample(pos, nodes, ext_x: float, eps: float, G: float, theta: float, stride: int, group: int = 32):
    """The reference walk over every stride-th group; returns (acc, interactions)."""
    n = pos.shape[0]
    acc = np.zeros((n, 3), np.float32)
    inter = lib().orc_walk_sample(_a(pos), n, _a(np.ascontiguousarray(nodes)), np.float32(ext_x),
                                  np.float32(eps) * np.float32(eps), G, theta, group, 0, stride, _a(acc))
    return acc, inter


def walk_groups_sample(pos, nodes, ext_x: float, eps: float, G: float, theta: float, stride: int,
                       alpha: float = 0.0, amag=None, group_param=None, width: int = 32):
    """Every stride-th walk group (the relative criterion when amag is given,
    per-group (theta, alpha) from group_param): returns (acc [n,3] with only
    the sampled groups' bodies written, accepted-node count of each sampled
    group, sampled group indices)."""
    n = pos.shape[0]
    acc = np.zeros((n, 3), np.float32)
    groups = (n + width - 1) // width
    idx = np.arange(0, groups, stride)
    lens = np.zeros(len(idx), np.int32)
    am = None if amag is None else np.ascontiguousarray(amag, np.float32)
    gp = None if group_param is None else np.ascontiguousarray(group_param, np.float32)
    lib().orc_walk_groups_sample(_a(pos), n, _a(np.ascontiguousarray(nodes)), np.float32(ext_x),
                                 np.float32(eps) * np.float32(eps), G, theta, alpha,
                                 None if am is None else _a(am), None if gp is None else _a(gp), width, stride,
                                 _a(acc), _a(lens))
    return acc, lens, idx


def list_lengths(pos, nodes, ext_x: float, theta: float, group: int = 32, d2order: int = 0):
    n = pos.shape[0]
    out = np.zeros((n + group - 1) // group, np.int32)
    lib().orc_walk_list_lengths(_a(pos), n, _a(np.ascontiguousarray(nodes)), np.float32(ext_x), theta, group,
                                d2order, _a(out))
    return out


def kick_drift(pos, vel, acc, dt: float) -> None:
    lib().orc_kick_drift(_a(pos), _a(vel), _a(np.ascontiguousarray(acc, np.float32)), pos.shape[0], dt)


def direct_sum(pos, eps: float, G: float = 1.0, targets: np.ndarray | None = None) -> np.ndarray:
    n = pos.shape[0]
    nt = n if targets is None else len(targets)
    acc = np.zeros((nt, 3), np.float64)
    t = None if targets is None else np.ascontiguousarray(targets, np.int32)
    lib().orc_direct_sum_f64(_a(pos), n, None if t is None else _a(t), nt, float(eps) ** 2, G, _a(acc))
    return acc


def diagnostics(pos, vel, eps: float, G: float = 1.0, potential: bool = True) -> dict:
    """FP64 conserved quantities (the engine's definitions)."""
    out = np.zeros(12, np.float64)
    lib().orc_diagnostics_f64(_a(np.ascontiguousarray(pos, np.float32)), _a(np.ascontiguousarray(vel, np.float32)),
                              pos.shape[0], float(eps) ** 2, int(potential), _a(out))
    M = out[0]
    kin = 0.5 * out[10]
    pot = -0.5 * G * out[11] if potential else 0.0
    return {"mass": M, "com": list(out[1:4] / M), "com_vel": list(out[4:7] / M), "momentum": list(out[4:7]),
            "angular_momentum": list(out[7:10]), "kinetic": kin, "potential": pot, "total": kin + pot}


def step(pos, vel, bits=21, eps=0.01, G=1.0, theta=0.5, dt=1e-3, group=32, d2order=0):
    """One reference step in place on host arrays; returns (perm, acc, node_count, interactions)."""
    n = pos.shape[0]
    scratch = np.zeros(lib().orc_step_scratch_bytes(n), np.uint8)
    perm = np.zeros(n, np.uint32)
    acc = np.zeros((n, 3), np.float32)
    inter = C.c_longlong()
    m = lib().orc_step(_a(pos), _a(vel), n, bits, eps, G, theta, dt, group, d2order, _a(perm), _a(acc), _a(scratch),
                       C.byref(inter))
    return perm, acc, m, inter.value


def pipeline(pos, vel, bits=21):
    """bbox -> keys -> sort -> reorder -> tree on host arrays (no walk)."""
    mn, mx = bbox(pos)
    box = world_box(mn, mx, bits)
    keys, idx = morton(pos, box, bits)
    skeys, perm = sort_pairs(keys, idx)
    spos, svel = reorder(pos, vel, perm)
    nodes, lo, lc, deep, count = build_tree(skeys, spos, bits)
    return dict(mn=mn, mx=mx, box=box, keys=keys, skeys=skeys, perm=perm, pos=spos, vel=svel, nodes=nodes,
                level_offsets=lo, level_count=lc, deepest=deep, count=count, ext_x=np.float32(mx[0] - mn[0]))


# ------------------------------------------------------------ reference harness
def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        L = C.CDLL(str(REF_LIB), mode=os.RTLD_LOCAL)
        L.ref_run.restype = _I
        L.ref_run.argtypes = [_P, _P, _I, _F, _F, _F, _F, _I, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _P, _P, _P]
        _ref = L
    return _ref


def ref_run(pos, vel, eps, G=1.0, theta=0.5, dt=1e-3, steps=1, want_nodes=True, track_ids=True):
    """The reference's own step(s) on a B200 (needs a GPU).  Outputs describe the last step."""
    n = pos.shape[0]
    keys_in = np.zeros(n, np.uint64)
    keys_out = np.zeros(n, np.uint64)
    perm = np.zeros(n, np.uint32)
    cap = 8 * n if want_nodes else 0
    nodes = np.zeros(max(cap, 1), NODE_DTYPE)
    lo = np.zeros(22, np.int32)
    lc = np.zeros(22, np.int32)
    deep = C.c_int()
    acc = np.zeros((n, 3), np.float32)
    po = np.zeros((n, 4), np.float32)
    vo = np.zeros((n, 3), np.float32)
    ids = np.zeros(n, np.uint32)
    ms = C.c_float()
    pos = np.ascontiguousarray(pos, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    count = ref().ref_run(_a(pos), _a(vel), n, eps, G, theta, dt, steps, _a(keys_in), _a(keys_out), _a(perm),
                          _a(nodes) if want_nodes else None, cap, _a(lo), _a(lc), C.byref(deep), _a(acc), _a(po),
                          _a(vo), _a(ids) if track_ids else None, C.byref(ms))
    if count < 0:
        raise RuntimeError("reference harness failed")
    return dict(keys=keys_in, skeys=keys_out, perm=perm, nodes=nodes[:count] if want_nodes else None,
                level_offsets=lo, level_count=lc, deepest=deep.value, count=count, acc=acc, pos=po, vel=vo,
                ids=ids if track_ids else None, ms_per_step=ms.value)
