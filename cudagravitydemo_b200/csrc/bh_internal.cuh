// bh_internal.cuh — device-side types and helpers shared by the sm_100a
// kernels of the Barnes-Hut engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bh_api.h"
#include "types.h"

#define BH_MAX_BITS 21
#define BH_LEVEL_SLOTS 24  // levels 0..21, sentinel entries beyond the deepest level

// Device error word: bit (status - 1) is set when a kernel detects `status`.
#define BH_ERRBIT(s) (1u << ((s)-1))

// Bound on every device-side spin-wait (look-back in the sort, arrival flags):
// after this many polls a kernel records BH_ERR_TIMEOUT and stops waiting.
#define BH_SPIN_LIMIT (1u << 22)

// World box as the kernels use it.  Written by the bounding-box kernel.
struct DevBox {
    float mn[3];
    float mx[3];
    float extent;  // max(width, height, depth)
    float scale;   // (2^bits - 1) / extent
    float extX;    // x-extent: node sizes use it (the reference's tree.cu:506)
    int pad[3];
};

// The root's mass, centre of mass and bounding box reduced in FP64 (written
// by the bounding-box kernel; the FP32 tree keeps the reference's rounding).
struct DevRoot {
    double mass;
    double com[3];
    double mn[3];
    double mx[3];
};

// Device-resident tree summary.  levelOffset[L]/levelCount[L] for L <= bits;
// levelOffset[L] = nodeCount for every L past the deepest level.
struct DevTreeInfo {
    int levelOffset[BH_LEVEL_SLOTS];
    int levelCount[BH_LEVEL_SLOTS];
    float sizeSq[BH_LEVEL_SLOTS];  // (extX / 2^L)^2 rounded to float, per level
    int deepest;
    int nodeCount;
    int overflowLevel;  // first level that did not fit, or 0
    int pad;
};

// One node as the walk reads it: one 32-byte sector.
// com = centre of mass (xyz) and mass (w); children are the contiguous node
// range [childBegin, childEnd) (empty for a leaf); sizeSq of its level;
// count = bodies below it.
struct __align__(32) WalkNode {
    float4 com;
    int childBegin;
    int childEnd;
    float sizeSq;
    int count;
};

// Walk statistics accumulated on the device.
struct DevCounters {
    unsigned long long interactions;  // body-node interactions of valid bodies
    unsigned long long nodesTested;   // opening tests (per group)
    unsigned long long undecided;     // tests settled by a full group vote
    int maxStack;
    int groupCursor;                  // dynamic group scheduler of the walk
    int pad[2];
};

__device__ __forceinline__ void bh_set_error(int* err, int status) {
    atomicOr(err, (int)BH_ERRBIT(status));
}

__device__ __forceinline__ unsigned lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Level-L prefix of a key with 3*bits significant bits (the reference's
// extractBitsFromLevel, tree.cu:23-26, is the bits = 21 case).
__device__ __forceinline__ uint64_t level_prefix(uint64_t key, int bits, int level) {
    int shift = 3 * (bits - level);
    return shift >= 64 ? 0ull : (key >> shift);
}

// Host-side launch helpers -----------------------------------------------
#define BH_CUDA_TRY(call)                                        \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return bh_note_cuda_error(e_);    \
    } while (0)

int bh_note_cuda_error(cudaError_t e);  // records the text, returns BH_ERR_CUDA
int bh_record_status(int s);             // the calling thread's bh_last_error(); returns s
int bh_status_from_bits(int bits);      // lowest error bit of a device error word -> status
int bh_sm_count();                      // multiprocessors of the current device (cached)
