"""ctypes bindings of libbh_b200.so (the engine's C ABI, include/*.h).

The library is loaded from this package's directory; there is no fallback:
if it is missing or cannot be loaded, importing the engine fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libbh_b200.so"

c_float_p = C.POINTER(C.c_float)
c_void_pp = C.POINTER(C.c_void_p)

MLP_PARAMS = 1393       # bh_api.h BH_MLP_PARAMS
MLP_TRAINED = 1377      # bh_api.h BH_MLP_TRAINED
MAC_CANDIDATES = 8      # bh_api.h BH_MAC_CANDIDATES
GROUP_FEATURES = 7      # bh_api.h BH_GROUP_FEATURES


class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class Float4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class WorldBox(C.Structure):  # types.h worldBox
    _fields_ = [("minX", C.c_float), ("minY", C.c_float), ("minZ", C.c_float), ("extent", C.c_float),
                ("scale", C.c_float)]


class Node(C.Structure):  # types.h node (80 bytes)
    _fields_ = [("nodePathFromRoot", C.c_uint64), ("parentIndex", C.c_int), ("firstParticleIndex", C.c_int),
                ("particleCount", C.c_int), ("child", C.c_int * 8), ("treeLevel", C.c_int),
                ("_pad", C.c_int * 2), ("massData", C.c_float * 4)]


class TreeState(C.Structure):  # types.h treeState (304 bytes)
    _fields_ = [("nodes", C.c_void_p), ("maxNodes", C.c_int), ("mortonIn", C.c_void_p), ("mortonOut", C.c_void_p),
                ("indexIn", C.c_void_p), ("indexOut", C.c_void_p), ("boundingData", C.c_void_p * 4),
                ("sorter", C.c_void_p), ("builder", C.c_void_p), ("levelOffsets", C.c_int * 22),
                ("levelCount", C.c_int * 22), ("deepestLevel", C.c_int), ("treeBlocks", C.c_int),
                ("starCount", C.c_int), ("sortedPosMassVals", C.c_void_p), ("sortedVelVals", C.c_void_p)]


class Params(C.Structure):  # bh_api.h bh_params
    _fields_ = [("bitsPerAxis", C.c_int), ("leafSize", C.c_int), ("groupWidth", C.c_int), ("theta", C.c_float),
                ("eps", C.c_float), ("G", C.c_float), ("dt", C.c_float), ("compensated", C.c_int),
                ("exportNodes", C.c_int), ("macMode", C.c_int), ("alpha", C.c_float), ("errTarget", C.c_float)]


class Stats(C.Structure):  # bh_api.h bh_stats
    _fields_ = [("interactions", C.c_longlong), ("nodesTested", C.c_longlong), ("nodeCount", C.c_int),
                ("deepestLevel", C.c_int), ("levelOffsets", C.c_int * 23), ("levelCount", C.c_int * 23),
                ("errorBits", C.c_int), ("maxStack", C.c_int), ("groupVotes", C.c_longlong)]


class Diagnostics(C.Structure):  # bh_api.h bh_diagnostics
    _fields_ = [("mass", C.c_double), ("com", C.c_double * 3), ("comVel", C.c_double * 3),
                ("momentum", C.c_double * 3), ("angularMomentum", C.c_double * 3), ("kinetic", C.c_double),
                ("potential", C.c_double), ("total", C.c_double)]


class TuneResult(C.Structure):  # bh_api.h bh_tune_result
    _fields_ = [("leafSize", C.c_int), ("groupWidth", C.c_int), ("candidates", C.c_int),
                ("leafSizes", C.c_int * 16), ("groupWidths", C.c_int * 16), ("msPerStep", C.c_float * 16),
                ("stackEntries", C.c_int), ("stackEntriesTried", C.c_int * 16)]


class DemoParams(C.Structure):  # bh_api.h bh_demo_params
    _fields_ = [("totalMass", C.c_float), ("scaleLength", C.c_float), ("scaleThickness", C.c_float),
                ("haloFraction", C.c_float), ("G", C.c_float), ("rotation", C.c_float * 3),
                ("centre", C.c_float * 3), ("velocity", C.c_float * 3)]


class GalaxyParams(C.Structure):  # bh_api.h bh_galaxy_params
    _fields_ = [("diskMass", C.c_float), ("diskScale", C.c_float), ("diskHeight", C.c_float),
                ("diskTrunc", C.c_float), ("bulgeMass", C.c_float), ("bulgeScale", C.c_float),
                ("bulgeTrunc", C.c_float), ("dispersion", C.c_float), ("G", C.c_float)]


assert C.sizeof(Node) == 80 and C.sizeof(TreeState) == 304 and C.sizeof(WorldBox) == 20

P = C.c_void_p  # device or host pointer
I = C.c_int
F = C.c_float
S = C.c_void_p  # cudaStream_t

# name -> (restype, argtypes), one entry per function of include/*.h
SIGNATURES = {
    # sorting.h
    "sorterCreate": (P, [I]),
    "radixSortPairs": (None, [P, P, P, P, P, I]),
    "sorterDestroyer": (None, [P]),
    "reorderParticles": (None, [P, P, P, P, P, I, S]),
    "bh_sorter_create": (I, [c_void_pp, I]),
    "bh_radix_sort_pairs": (I, [P, P, P, P, P, I, I, S]),
    "bh_sorter_destroy": (I, [P]),
    "bh_radix_sort_pairs_noalloc": (I, [P, P, P, P, I, I, S]),
    "bh_radix_sort_noalloc_errors": (I, [P, S]),
    "bh_selftest_noalloc_timeout": (I, [S]),
    "bh_sorter_errors": (I, [P, P, S]),
    "bh_selftest_sorter_timeout": (I, [P, S]),
    # tree.h
    "mortonEncode": (None, [P, P, P, I, WorldBox, S]),
    "localMinMaxFinder": (None, [P, C.c_uint, P, P, S]),
    "globalMinMaxReducer": (None, [P, P, I, P, P, S]),
    "identifyNodesAtLevel": (None, [P, I, I, P, S]),
    "createNodes": (None, [P, P, P, P, P, P, I, I, I, I, I, S]),
    "updateTreeParticles": (None, [P, I, I, I, S]),
    "updateTreeMass": (None, [P, P, I, I, I, S]),
    "calculateAcceleration": (None, [P, TreeState, P, F, F, F, I, S]),
    "positionUpdater": (None, [P, P, P, I, F, S]),
    "sumCreate": (P, [I]),
    "prefixSum": (None, [P, P, P, I]),
    "sumDestroyer": (None, [P]),
    # main.h
    "initialiseTree": (None, [C.POINTER(TreeState), I, I, I]),
    "createWorldBox": (None, [P, I, P, P, P, P, C.POINTER(WorldBox)]),
    "buildTree": (None, [C.POINTER(TreeState), c_void_pp, c_void_pp]),
    "destroyTree": (None, [C.POINTER(TreeState)]),
    "blockNumCalculator": (None, [C.POINTER(I)] * 6 + [I]),
    "roundNumberToMultiple": (I, [I, I]),
    # bh_api.h
    "bh_status_string": (C.c_char_p, [I]),
    "bh_last_error": (I, []),
    "bh_cuda_error_string": (C.c_char_p, []),
    "bh_params_default": (None, [C.POINTER(Params)]),
    "bh_initialise_tree": (I, [C.POINTER(TreeState), I, I, I]),
    "bh_build_tree": (I, [C.POINTER(TreeState), c_void_pp, c_void_pp, S]),
    "bh_destroy_tree": (I, [C.POINTER(TreeState)]),
    "bh_calculate_acceleration": (I, [P, C.POINTER(TreeState), P, F, F, F, I, S]),
    "bh_position_updater": (I, [P, P, P, I, F, S]),
    "bh_world_box": (I, [P, I, I, C.POINTER(WorldBox), C.POINTER(Float3), C.POINTER(Float3), S]),
    "bh_morton_encode": (I, [P, P, P, I, WorldBox, I, S]),
    "bh_sim_create": (I, [c_void_pp, I, C.POINTER(Params), S]),
    "bh_sim_destroy": (I, [P]),
    "bh_sim_set_params": (I, [P, C.POINTER(Params)]),
    "bh_sim_get_params": (I, [P, C.POINTER(Params)]),
    "bh_sim_stream": (S, [P]),
    "bh_sim_load": (I, [P, P, P, I, I]),
    "bh_sim_store": (I, [P, P, P, I]),
    "bh_sim_device_state": (I, [P, c_void_pp, c_void_pp, c_void_pp, C.POINTER(I)]),
    "bh_sim_step": (I, [P, I]),
    "bh_sim_step_host": (I, [P, P, P, I, I]),
    "bh_sim_step_host_sorted": (I, [P, P, P, P, I, I]),
    "bh_sim_accelerations": (I, [P, P, I]),
    "bh_sim_accel_magnitudes": (I, [P, P, I]),
    "bh_sim_stats": (I, [P, C.POINTER(Stats)]),
    "bh_sim_tree": (I, [P, C.POINTER(C.POINTER(TreeState))]),
    "bh_sim_profile": (I, [P, I, C.POINTER(C.c_float)]),
    "bh_sim_kernels_per_step": (I, [P]),
    "bh_fma_peak_tflops": (I, [I, C.POINTER(C.c_float), S]),
    "bh_direct_sum_f64": (I, [P, I, P, I, C.c_double, C.c_double, P, S]),
    "bh_diagnostics_f64": (I, [P, P, I, C.c_double, C.c_double, I, C.POINTER(Diagnostics), S]),
    "bh_sim_synchronize": (I, [P]),
    "bh_selftest_bounded_wait": (I, [S]),
    "bh_sim_create_batch": (I, [c_void_pp, I, P, C.POINTER(Params), S]),
    "bh_sim_tune": (I, [P, I, C.POINTER(TuneResult)]),
    "bh_sim_set_walk_stack": (I, [P, I]),
    "bh_sim_walk_stack": (I, [P]),
    "bh_sim_systems": (I, [P, C.POINTER(I), P]),
    "bh_sim_system_diagnostics": (I, [P, I, P]),
    "bh_dump_open": (I, [c_void_pp, C.c_char_p, I, I, P]),
    "bh_dump_frame": (I, [P, P, P, I, S]),
    "bh_sim_dump_frame": (I, [P, P]),
    "bh_dump_close": (I, [P]),
    "bh_sim_diagnostics": (I, [P, I, C.POINTER(Diagnostics)]),
    "bh_mac_ladder": (I, [P]),
    "bh_demo_params_default": (None, [C.POINTER(DemoParams)]),
    "bh_ic_demo": (I, [P, P, I, C.POINTER(DemoParams), C.c_uint64, S]),
    "bh_sim_set_mac_mlp": (I, [P, P]),
    "bh_sim_group_features": (I, [P, P, P, I]),
    "bh_sim_group_params": (I, [P, P, I]),
    "bh_sim_group_lengths": (I, [P, P, I, C.POINTER(I), I]),
    "bh_sim_root_f64": (I, [P, P]),
    "bh_mlp_forward": (I, [P, P, I, P, S]),
    "bh_mlp_loss_grad": (I, [P, P, P, I, P, P, S]),
    "bh_mlp_train_epoch": (I, [P, P, P, I, P, P, P, I, C.POINTER(I), F, P, S]),
    "bh_ic_plummer": (I, [P, P, I, F, F, F, C.c_uint64]),
    "bh_galaxy_params_default": (None, [C.POINTER(GalaxyParams)]),
    "bh_ic_disk_galaxy": (I, [P, P, I, C.POINTER(GalaxyParams), C.c_uint64]),
    "bh_ic_merger": (I, [P, P, I, C.POINTER(GalaxyParams), F, F, F, C.c_uint64]),
}

_lib = None


def load() -> C.CDLL:
    """Load libbh_b200.so (once) and attach the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cudagravitydemo_b200.build`")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_LOCAL | getattr(os, "RTLD_NOW", 2))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib
