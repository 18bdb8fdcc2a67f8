// walk.cu — Barnes-Hut tree walk and kick-drift integrator (sm_100a).
//
// Semantics are the reference's calculateAcceleration (tree.cu:562-676):
// bodies are taken in groups of 32 Morton-consecutive bodies; starting from
// the root's children, a node is OPENED when it is not a leaf and at least one
// valid body of the group fails  size^2 < theta^2 * d^2  (size = x-extent /
// 2^level, d = distance from the body to the node's centre of mass,
// tree.cu:501-530, 610-634); otherwise every body of the group interacts with
// the node's monopole, Plummer-softened.  The set of interacting nodes is
// therefore a function of the group alone, and this kernel reproduces it
// exactly while changing how it is found:
//   - the 32 lanes test 64 different nodes per round, two each (the reference
//     tests one node per step with all 32 lanes);
//   - a node is accepted without a vote when the distance from its centre of
//     mass to the group's bounding box already satisfies the criterion with a
//     2^-16 relative margin (which dominates every rounding difference), and
//     opened without a vote when a representative body (the group's body
//     nearest the box corner on the node's side) already fails it;
//     only the rest take the exact group vote (same FP32 operations and
//     order as the reference, so the decision is bit-identical), two nodes
//     per pass with packed FP32x2 arithmetic on a compacted copy of them,
//     each lane collecting its body's verdicts in a bit mask that one warp OR
//     combines;
//   - accepted nodes' (centre of mass, mass) are appended to a per-warp list
//     in shared memory and evaluated in bulk, two list entries per
//     instruction with sm_100's packed FP32x2 arithmetic: per pair of
//     interactions 3 SUB2, 3 FMA2, two MUFU rsqrt, 3 MUL2 and 3 FMA2, fed by
//     two 16-byte shared loads (the list is stored as four component arrays
//     x[], y[], z[], m[]: a 16-byte load yields two ready packed operands, and
//     appending consecutive entries stores without bank conflicts);
//   - sums are compensated per block of list entries (Kahan on the block
//     partials) when requested;
//   - warps fetch groups from an atomic cursor (dynamic load balance).
// Leaves never open, as in the reference (count <= 1 or no children).
// Extensions (template switches, off for the reference's semantics): the
// relative opening criterion with per-group budgets (the learned criterion),
// bucket leaves (an opened node with at most leafSize bodies contributes its
// bodies), and a group table for batches of independent systems.
#include <math.h>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = kWarpsPerBlock * 32;
#ifndef BH_WALK_STACK_SMEM
#define BH_WALK_STACK_SMEM 768
#endif
#ifndef BH_WALK_LIST_CAP
#define BH_WALK_LIST_CAP 256
#endif
// stack entries per warp in shared memory when WalkArgs.stackSmem is 0; the
// size is a launch parameter (dynamic shared memory) that the autotuner sets
constexpr int kStackSmemDefault = BH_WALK_STACK_SMEM;
constexpr int kListCap = BH_WALK_LIST_CAP;      // interaction-list entries per warp (a multiple of 64)
#ifndef BH_WALK_MIN_BLOCKS_PLAIN
#define BH_WALK_MIN_BLOCKS_PLAIN 7
#endif
#ifndef BH_WALK_MIN_BLOCKS_RELATIVE
#define BH_WALK_MIN_BLOCKS_RELATIVE 6
#endif
#ifndef BH_WALK_MIN_BLOCKS_WIDE
#define BH_WALK_MIN_BLOCKS_WIDE 4
#endif
// Resident blocks per SM the register allocation must allow (64K registers /
// (128 threads x blocks)): fewer blocks, more registers per thread.  Measured
// on the 1M disk, the walk is faster with registers than with warps: 7 blocks
// (72 registers) for the fixed-theta walks, 6 (80) with the relative test.
// With the 256-entry list and the default 768-entry stack, shared memory
// (38 KB per block) binds first: 5 blocks per SM, which measured faster than
// 6 blocks with a 192-entry list.
constexpr int kMinBlocksPlain = BH_WALK_MIN_BLOCKS_PLAIN;
constexpr int kMinBlocksRelative = BH_WALK_MIN_BLOCKS_RELATIVE;
// 64-body groups (two bodies per lane), every criterion: 4 blocks (up to 128
// registers; 110 used) measured 7% faster than 6 blocks with spills
constexpr int kMinBlocksWide = BH_WALK_MIN_BLOCKS_WIDE;
__host__ __device__ constexpr int walk_min_blocks(bool relative, bool wide) {
    return wide ? kMinBlocksWide : (relative ? kMinBlocksRelative : kMinBlocksPlain);
}
constexpr int kBlocksPerSm = 8;  // persistent grid: blocks launched per SM (the excess waits)
constexpr int kSpillPerWarp = 4096;  // global stack entries per warp beyond shared memory
constexpr float kBoxMargin = 1.0f - 1.0f / 65536.0f;
#ifndef BH_WALK_PACKED
#define BH_WALK_PACKED 1
#endif
constexpr bool kWalkPacked = BH_WALK_PACKED != 0;
// Each lane's running force sums (and their Kahan compensations) live in
// shared memory between list flushes instead of in registers: they are only
// touched once per flushed list block, and the registers they free are what
// lets more warps be resident.
#ifndef BH_WALK_SUMS_SMEM
#define BH_WALK_SUMS_SMEM 1
#endif
constexpr bool kSumsSmem = BH_WALK_SUMS_SMEM != 0;
// Take groups in the order the caller gives (longest lists first).
#ifndef BH_WALK_GROUP_ORDER
#define BH_WALK_GROUP_ORDER 1
#endif
constexpr bool kGroupOrder = BH_WALK_GROUP_ORDER != 0;

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Two floats packed in one 64-bit register (low half = first), and the
// sm_100 packed FP32x2 operations on them (round to nearest).
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack2(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// The reference's d^2 (tree.cu:611) as its compiled walk evaluates it:
// fma(dz, dz, fma(dx, dx, dy * dy)).  The opening test must round exactly
// like the reference's for the interaction sets to be identical.
__device__ __forceinline__ float ref_dist_sq(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

}  // namespace

// One warp per group of 32 bodies (kWide: 64, two per lane).  kPacked selects
// the interaction loop: packed FP32x2 over a component-array list, or scalar
// FP32 over float4 entries (32-body groups only).
template <bool kFused, bool kCompensated, bool kPacked, bool kRelative, bool kBuckets, bool kWide>
__global__ void __launch_bounds__(kThreads, walk_min_blocks(kRelative, kWide))
k_walk(const WalkArgs a) {
    static_assert(kPacked || !kWide, "64-body groups use the packed interaction loop");
    constexpr int kW = kWide ? 64 : 32;
    const float4* __restrict__ pos = a.pos;
    const WalkNode* __restrict__ wn = a.wn;
    const int n = a.n;
    const float eps2 = a.eps2, G = a.G, dt = a.dt;
    int* err = a.err;
    const int spillPerWarp = kSpillPerWarp;
    // per-warp traversal stack: stackSmem entries per warp in dynamic shared
    // memory, entries past them spill to global memory
    extern __shared__ int sDynStack[];
    const int stackSmem = a.stackSmem;
    // per-warp interaction list: float4 (x, y, z, m) per entry, or, packed,
    // the same storage as four arrays of kListCap floats: x[], y[], z[], m[]
    __shared__ float4 sList[kWarpsPerBlock][kListCap];
    // the nodes a round votes on, compacted and pair-interleaved:
    // sVote[2j] = (x_2j, x_2j+1, y_2j, y_2j+1), sVote[2j+1] = (z.., z.., size^2.., size^2..)
    // (entries 64-65 take the writes of the nodes that are not staged, so that
    // staging needs no branch)
    __shared__ float4 sVote[kWarpsPerBlock][66];
    __shared__ __align__(8) float sVoteMs[kRelative ? kWarpsPerBlock : 1][66];  // mass * size^2 of those nodes
    // per warp: the group being walked and its interaction-list length so far
    // (kept here rather than in registers, which the walk is short of)
    __shared__ int sGroupLen[kWarpsPerBlock][2];
    // per warp: the group's representative body of each box octant, (x, y, z, |a|)
    __shared__ float4 sRep[kWarpsPerBlock][8];
    // per lane: sums x, y, z, compensations x, y, z (then the second body's)
    constexpr int kSums = kWide ? 12 : 6;
    __shared__ float sSum[kSumsSmem ? kWarpsPerBlock : 1][kSumsSmem ? kSums : 1][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    int* spill = a.spill + (size_t)(blockIdx.x * kWarpsPerBlock + w) * spillPerWarp;
    int* const sStk = sDynStack + w * stackSmem;  // this warp's stack
    const int stackCap = stackSmem + spillPerWarp;
    const int groups = a.groupTable ? a.groups : (n + kW - 1) / kW;
    const int leafSize = a.leafSize > 1 ? a.leafSize : 1;  // nodes with at most this many bodies are buckets
    unsigned nInteract = 0, nTested = 0, nVote = 0;
    // interactions of this warp so far; handed to the 64-bit total before the
    // 32-bit count could wrap (uniform across the warp)
    auto countInteractions = [&](int len, int nValid) {
        nInteract += (unsigned)len * (unsigned)nValid;
        if (nInteract >= 0x80000000u) {
            if (lane == 0) atomicAdd(&a.ctr->interactions, (unsigned long long)nInteract);
            nInteract = 0;
        }
    };
    int maxTop = 0;

    for (;;) {
        int g = 0;
        if (lane == 0) {
            g = atomicAdd(&a.ctr->groupCursor, 1);
            if (kGroupOrder && a.groupOrder && g < groups) g = a.groupOrder[g];  // longest lists first
        }
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= groups) break;
        // the group's bodies and the root of its tree (a batch: one per system)
        int first, cnt, root = 0;
        if (a.groupTable) {
            const int4 gt = a.groupTable[g];
            first = gt.x;
            cnt = gt.y;
            root = gt.z;
        } else {
            first = g * kW;
            cnt = n - first < kW ? n - first : kW;
        }
        const int b = first + lane;
        const bool valid = lane < cnt;
        const float4 p = valid ? pos[b] : make_float4(0.f, 0.f, 0.f, 0.f);
        // the second body of the lane (64-body groups)
        const int b1 = b + 32;
        const bool valid1 = kWide && lane + 32 < cnt;
        float3 p1 = make_float3(0.f, 0.f, 0.f);
        if (kWide && valid1) {
            const float4 q = pos[b1];
            p1 = make_float3(q.x, q.y, q.z);
        }
        int nValid = __popc(__ballot_sync(0xffffffffu, valid));
        if (kWide) nValid += __popc(__ballot_sync(0xffffffffu, valid1));
        // opening parameters of this group (per 32-body group; a 64-body group
        // takes the smaller theta and budget of its two halves)
        float theta = a.theta, kA = 0.f;
        if (a.groupParam) {
            float2 gp = a.groupParam[kWide ? 2 * g : g];
            if (kWide && 2 * g + 1 < a.groupParamCount) {
                const float2 q = a.groupParam[2 * g + 1];
                gp.x = fminf(gp.x, q.x);
                gp.y = fminf(gp.y, q.y);
            }
            theta = gp.x;
            kA = gp.y / G;
        } else {
            kA = a.alpha / G;
        }
        const float thetaSq = __fmul_rn(theta, theta);
        const float thetaSqBox = thetaSq * kBoxMargin;
        // relative criterion: open when M s^2 > kA |a_b| d^4 for some body
        float myA = 0.f, myA1 = 0.f, aMin = 0.f;
        if (kRelative) {
            myA = valid ? a.aMagIn[b] : INFINITY;
            aMin = myA;
            if (kWide) {
                myA1 = valid1 ? a.aMagIn[b1] : INFINITY;
                aMin = fminf(aMin, myA1);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) aMin = fminf(aMin, __shfl_xor_sync(0xffffffffu, aMin, o));
        }

        // group box as centre +- half extent; the half extent is rounded
        // outward so the box contains every body of the group exactly
        float bm[3], be[3];
        {
            float lo[3] = {valid ? p.x : INFINITY, valid ? p.y : INFINITY, valid ? p.z : INFINITY};
            float hi[3] = {valid ? p.x : -INFINITY, valid ? p.y : -INFINITY, valid ? p.z : -INFINITY};
            if (kWide && valid1) {
                lo[0] = fminf(lo[0], p1.x); lo[1] = fminf(lo[1], p1.y); lo[2] = fminf(lo[2], p1.z);
                hi[0] = fmaxf(hi[0], p1.x); hi[1] = fmaxf(hi[1], p1.y); hi[2] = fmaxf(hi[2], p1.z);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                    hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
                }
#pragma unroll
            for (int k = 0; k < 3; k++) {
                bm[k] = 0.5f * (lo[k] + hi[k]);
                const float mag = fmaxf(fabsf(lo[k]), fabsf(hi[k]));
                be[k] = __fmul_ru(0.5f, __fsub_ru(hi[k], lo[k])) + mag * 1.0e-6f;
            }
        }
        // representative bodies, one per octant of the group box: the valid
        // body nearest each corner of the box (among bodies whose squared
        // distances agree to 32 ulps, any).  A node is tested against the
        // representative of the octant its centre of mass lies in — a body on
        // the node's side of the group, so that a node some body fails is
        // mostly found without a vote (a third fewer votes than with the body
        // nearest the centre)
        {
#pragma unroll
            for (int o = 0; o < 8; o++) {
                const float cx = (o & 4) ? bm[0] + be[0] : bm[0] - be[0];
                const float cy = (o & 2) ? bm[1] + be[1] : bm[1] - be[1];
                const float cz = (o & 1) ? bm[2] + be[2] : bm[2] - be[2];
                float d = valid ? (p.x - cx) * (p.x - cx) + (p.y - cy) * (p.y - cy) + (p.z - cz) * (p.z - cz)
                                : INFINITY;
                bool second = false;
                if (kWide && valid1) {
                    const float d1 = (p1.x - cx) * (p1.x - cx) + (p1.y - cy) * (p1.y - cy) + (p1.z - cz) * (p1.z - cz);
                    if (d1 < d) { d = d1; second = true; }
                }
                const unsigned best = __reduce_min_sync(0xffffffffu, (__float_as_uint(d) & ~31u) | (unsigned)lane);
                if ((best & 31u) == (unsigned)lane)
                    sRep[w][o] = second ? make_float4(p1.x, p1.y, p1.z, myA1) : make_float4(p.x, p.y, p.z, myA);
            }
        }

        // root's children onto the stack
        int top;
        {
            const int rb = wn[root].childBegin, re = wn[root].childEnd;
            top = re - rb;
            if (lane < top) sStk[lane] = rb + lane;
        }
        __syncwarp();
        int listLen = 0;
        if (lane == 0) {
            sGroupLen[w][0] = g;
            sGroupLen[w][1] = 0;
        }
        float sx = 0.f, sy = 0.f, sz = 0.f;  // running sums
        float cx = 0.f, cy = 0.f, cz = 0.f;  // Kahan compensation
        float tx = 0.f, ty = 0.f, tz = 0.f;  // the second body's (64-body groups)
        float ux = 0.f, uy = 0.f, uz = 0.f;
        if (kSumsSmem)  // this lane's column only: no synchronisation needed
#pragma unroll
            for (int k = 0; k < kSums; k++) sSum[w][k][lane] = 0.f;

        // interactions with list entries [0, cnt); partial sums Kahan-added
        auto kahan = [&](float ax, float ay, float az, float& s0, float& s1, float& s2, float& c0, float& c1,
                         float& c2) {
            if (kCompensated) {
                float y, t;
                y = ax - c0; t = s0 + y; c0 = (t - s0) - y; s0 = t;
                y = ay - c1; t = s1 + y; c1 = (t - s1) - y; s1 = t;
                y = az - c2; t = s2 + y; c2 = (t - s2) - y; s2 = t;
            } else {
                s0 += ax; s1 += ay; s2 += az;
            }
        };
        auto flush = [&](int cnt) {
            float ax, ay, az;
            float bx = 0.f, by = 0.f, bz = 0.f;  // second body (64-body groups)
            if (kPacked) {
                // the list as four component arrays x[], y[], z[], m[]: one
                // 16-byte load gives four entries' x, i.e. two packed pairs
                const float* L = reinterpret_cast<const float*>(sList[w]);
                const ulonglong2* X = reinterpret_cast<const ulonglong2*>(L);
                const ulonglong2* Y = reinterpret_cast<const ulonglong2*>(L + kListCap);
                const ulonglong2* Z = reinterpret_cast<const ulonglong2*>(L + 2 * kListCap);
                const ulonglong2* Mq = reinterpret_cast<const ulonglong2*>(L + 3 * kListCap);
                const f32x2 px2 = pack2(p.x, p.x), py2 = pack2(p.y, p.y), pz2 = pack2(p.z, p.z);
                const f32x2 qx2 = pack2(p1.x, p1.x), qy2 = pack2(p1.y, p1.y), qz2 = pack2(p1.z, p1.z);
                const f32x2 e2 = pack2(eps2, eps2);
                const int quads = cnt >> 2;
                f32x2 ax2 = 0ull, ay2 = 0ull, az2 = 0ull;
                f32x2 bx2 = 0ull, by2 = 0ull, bz2 = 0ull;
                // one packed body-pair interaction: (bx, by, bz) against two entries
                auto pair = [&](f32x2 ex, f32x2 ey, f32x2 ez, f32x2 em, f32x2 ox, f32x2 oy, f32x2 oz, f32x2& sx2,
                                f32x2& sy2, f32x2& sz2) {
                    const f32x2 dx = sub2(ex, ox), dy = sub2(ey, oy), dz = sub2(ez, oz);
                    f32x2 r2 = fma2(dx, dx, e2);
                    r2 = fma2(dy, dy, r2);
                    r2 = fma2(dz, dz, r2);
                    float r2a, r2b;
                    unpack2(r2, r2a, r2b);
                    const f32x2 ri = pack2(rsqrt_approx(r2a), rsqrt_approx(r2b));
                    const f32x2 f = mul2(mul2(em, ri), mul2(ri, ri));
                    sx2 = fma2(f, dx, sx2);
                    sy2 = fma2(f, dy, sy2);
                    sz2 = fma2(f, dz, sz2);
                };
                if (kWide) {
#pragma unroll 1
                    for (int k = 0; k < quads; k++) {
                        const ulonglong2 x = X[k], y = Y[k], z = Z[k], m = Mq[k];
                        pair(x.x, y.x, z.x, m.x, px2, py2, pz2, ax2, ay2, az2);
                        pair(x.x, y.x, z.x, m.x, qx2, qy2, qz2, bx2, by2, bz2);
                        pair(x.y, y.y, z.y, m.y, px2, py2, pz2, ax2, ay2, az2);
                        pair(x.y, y.y, z.y, m.y, qx2, qy2, qz2, bx2, by2, bz2);
                    }
                } else {
#pragma unroll 8
                    for (int k = 0; k < quads; k++) {
                        const ulonglong2 x = X[k], y = Y[k], z = Z[k], m = Mq[k];
                        pair(x.x, y.x, z.x, m.x, px2, py2, pz2, ax2, ay2, az2);
                        pair(x.y, y.y, z.y, m.y, px2, py2, pz2, ax2, ay2, az2);
                    }
                }
                if (cnt & 2) {  // a pair left over
                    const int j = 4 * quads;
                    const f32x2 x = *reinterpret_cast<const f32x2*>(L + j);
                    const f32x2 y = *reinterpret_cast<const f32x2*>(L + kListCap + j);
                    const f32x2 z = *reinterpret_cast<const f32x2*>(L + 2 * kListCap + j);
                    const f32x2 m = *reinterpret_cast<const f32x2*>(L + 3 * kListCap + j);
                    pair(x, y, z, m, px2, py2, pz2, ax2, ay2, az2);
                    if (kWide) pair(x, y, z, m, qx2, qy2, qz2, bx2, by2, bz2);
                }
                float a0, a1;
                unpack2(ax2, a0, a1);
                ax = a0 + a1;
                unpack2(ay2, a0, a1);
                ay = a0 + a1;
                unpack2(az2, a0, a1);
                az = a0 + a1;
                if (kWide) {
                    unpack2(bx2, a0, a1);
                    bx = a0 + a1;
                    unpack2(by2, a0, a1);
                    by = a0 + a1;
                    unpack2(bz2, a0, a1);
                    bz = a0 + a1;
                }
                if (cnt & 1) {  // the last entry alone
                    const int j = cnt - 1;
                    const float ex = L[j], ey = L[kListCap + j], ez = L[2 * kListCap + j], em = L[3 * kListCap + j];
                    auto one = [&](float ox, float oy, float oz, float& rx, float& ry, float& rz) {
                        const float dx = ex - ox, dy = ey - oy, dz = ez - oz;
                        const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, eps2)));
                        const float ri = rsqrt_approx(r2);
                        const float f = (em * ri) * (ri * ri);
                        rx = __fmaf_rn(f, dx, rx);
                        ry = __fmaf_rn(f, dy, ry);
                        rz = __fmaf_rn(f, dz, rz);
                    };
                    one(p.x, p.y, p.z, ax, ay, az);
                    if (kWide) one(p1.x, p1.y, p1.z, bx, by, bz);
                }
            } else {
                float hx = 0.f, hy = 0.f, hz = 0.f;
                ax = ay = az = 0.f;
                int k = 0;
                for (; k + 1 < cnt; k += 2) {  // two independent chains
                    const float4 c0 = sList[w][k], c1 = sList[w][k + 1];
                    const float dx0 = c0.x - p.x, dy0 = c0.y - p.y, dz0 = c0.z - p.z;
                    const float dx1 = c1.x - p.x, dy1 = c1.y - p.y, dz1 = c1.z - p.z;
                    const float r0 = __fmaf_rn(dz0, dz0, __fmaf_rn(dy0, dy0, __fmaf_rn(dx0, dx0, eps2)));
                    const float r1 = __fmaf_rn(dz1, dz1, __fmaf_rn(dy1, dy1, __fmaf_rn(dx1, dx1, eps2)));
                    const float i0 = rsqrt_approx(r0), i1 = rsqrt_approx(r1);
                    const float f0 = (c0.w * i0) * (i0 * i0), f1 = (c1.w * i1) * (i1 * i1);
                    ax = __fmaf_rn(f0, dx0, ax);
                    hx = __fmaf_rn(f1, dx1, hx);
                    ay = __fmaf_rn(f0, dy0, ay);
                    hy = __fmaf_rn(f1, dy1, hy);
                    az = __fmaf_rn(f0, dz0, az);
                    hz = __fmaf_rn(f1, dz1, hz);
                }
                if (k < cnt) {
                    const float4 c = sList[w][k];
                    const float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
                    const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, eps2)));
                    const float ri = rsqrt_approx(r2);
                    const float f = (c.w * ri) * (ri * ri);
                    ax = __fmaf_rn(f, dx, ax);
                    ay = __fmaf_rn(f, dy, ay);
                    az = __fmaf_rn(f, dz, az);
                }
                ax += hx;
                ay += hy;
                az += hz;
            }
            if (kSumsSmem) {
                float (*S)[32] = sSum[w];
                float s0 = S[0][lane], s1 = S[1][lane], s2 = S[2][lane];
                float c0 = S[3][lane], c1 = S[4][lane], c2 = S[5][lane];
                kahan(ax, ay, az, s0, s1, s2, c0, c1, c2);
                S[0][lane] = s0; S[1][lane] = s1; S[2][lane] = s2;
                S[3][lane] = c0; S[4][lane] = c1; S[5][lane] = c2;
                if (kWide) {
                    float t0 = S[kSums - 6][lane], t1 = S[kSums - 5][lane], t2 = S[kSums - 4][lane];
                    float u0 = S[kSums - 3][lane], u1 = S[kSums - 2][lane], u2 = S[kSums - 1][lane];
                    kahan(bx, by, bz, t0, t1, t2, u0, u1, u2);
                    S[kSums - 6][lane] = t0; S[kSums - 5][lane] = t1; S[kSums - 4][lane] = t2;
                    S[kSums - 3][lane] = u0; S[kSums - 2][lane] = u1; S[kSums - 1][lane] = u2;
                }
            } else {
                kahan(ax, ay, az, sx, sy, sz, cx, cy, cz);
                if (kWide) kahan(bx, by, bz, tx, ty, tz, ux, uy, uz);
            }
        };

        // One round tests up to 64 nodes, two per lane (slot 0 from the top 32
        // stack entries, slot 1 from the next 32).
        // A stack entry is a node index (>= 0) or, below a bucket node that
        // was opened, a body b encoded as -(b + 2): a body is a leaf, always
        // accepted.  Slot index -1 is an idle slot.
        struct Slot {
            int idx;
            float4 com;
            int cb, ce;
            float sizeSq;
            int count;
            bool open, undecided;
        };
        auto load = [&](Slot& t, int stackPos, bool has) {
            t.idx = -1;
            if (has) t.idx = (stackPos < stackSmem) ? sStk[stackPos] : spill[stackPos - stackSmem];
            t.count = 0;
            if (!kBuckets) {
                // every lane loads a record (an idle slot the root's) and an
                // idle slot gets an empty child range: no branch
                const int li = t.idx >= 0 ? t.idx : 0;
                t.com = wn[li].com;
                const int4 meta = *reinterpret_cast<const int4*>(&wn[li].childBegin);
                t.cb = meta.x;
                t.ce = t.idx >= 0 ? meta.y : meta.x;
                t.sizeSq = __int_as_float(meta.z);
                return;
            }
            t.com = make_float4(0.f, 0.f, 0.f, 0.f);
            t.cb = t.ce = 0;
            t.sizeSq = 0.f;
            if (t.idx >= 0) {
                t.com = wn[t.idx].com;
                const int4 meta = *reinterpret_cast<const int4*>(&wn[t.idx].childBegin);
                t.cb = meta.x;
                t.ce = meta.y;
                t.sizeSq = __int_as_float(meta.z);
                t.count = meta.w;
            } else if (t.idx < -1) {
                t.com = pos[-t.idx - 2];
                t.count = 1;
            }
        };
        auto classify = [&](Slot& t) {
            // every test computed for every slot, combined without branches
            const bool internal = t.cb != t.ce;  // leaves and idle slots have cb == ce
            const float gx = fmaxf(fabsf(t.com.x - bm[0]) - be[0], 0.f);
            const float gy = fmaxf(fabsf(t.com.y - bm[1]) - be[1], 0.f);
            const float gz = fmaxf(fabsf(t.com.z - bm[2]) - be[2], 0.f);
            const float D2 = gx * gx + gy * gy + gz * gz;
            bool boxAccept = thetaSqBox * D2 > t.sizeSq;
            if (kRelative) boxAccept = boxAccept && (t.com.w * t.sizeSq < kA * aMin * (D2 * D2) * kBoxMargin);
            const int oc = (t.com.x > bm[0] ? 4 : 0) | (t.com.y > bm[1] ? 2 : 0) | (t.com.z > bm[2] ? 1 : 0);
            const float4 r = sRep[w][oc];  // (x, y, z, |a|) of the octant's representative
            const float d2 = ref_dist_sq(r.x - t.com.x, r.y - t.com.y, r.z - t.com.z);
            bool repOpen = !(t.sizeSq < __fmul_rn(thetaSq, d2));
            if (kRelative) repOpen = repOpen || (t.com.w * t.sizeSq > kA * r.w * (d2 * d2));
            t.open = internal && !boxAccept && repOpen;
            t.undecided = internal && !boxAccept && !repOpen;
        };
        auto append = [&](const Slot& t, bool accept, int k) {
            if (!accept) return;
            if (kPacked) {  // component arrays: consecutive entries, conflict-free stores
                float* L = reinterpret_cast<float*>(sList[w]);
                L[k] = t.com.x;
                L[kListCap + k] = t.com.y;
                L[2 * kListCap + k] = t.com.z;
                L[3 * kListCap + k] = t.com.w;
            } else {
                sList[w][k] = t.com;
            }
        };
        // entries an opened node puts on the stack: its children (next level,
        // at most 8; anything else is a broken tree, reported rather than
        // followed) or, for a bucket (at most leafSize bodies), its bodies.
        // first: the first pushed value; entries are first + c (children) or
        // first - c (bodies, encoded).
        auto children = [&](const Slot& t, int& first, int& stepSign) -> int {
            first = t.cb;
            stepSign = 1;
            if (!t.open) return 0;
            if (kBuckets && t.count <= leafSize) {
                first = -(a.nFirst[t.idx] + 2);
                stepSign = -1;
                return t.count;
            }
            const int c = t.ce - t.cb;
            if (t.cb <= t.idx || c > 8) {
                bh_set_error(err, BH_ERR_INTERNAL);
                return 0;
            }
            return c;
        };
        auto push = [&](int pos, int v) {
            if (pos < stackSmem) sStk[pos] = v;
            else spill[pos - stackSmem] = v;
        };

        bool overflow = false;
        while (top > 0) {
            const int take = top < 64 ? top : 64;
            top -= take;
            Slot s0, s1;
            load(s0, top + lane, lane < take);
            load(s1, top + 32 + lane, 32 + lane < take);
            __syncwarp();
            classify(s0);
            classify(s1);
            // exact group vote for the undecided nodes (tree.cu:629-640)
            unsigned und0 = __ballot_sync(0xffffffffu, s0.undecided);
            unsigned und1 = __ballot_sync(0xffffffffu, s1.undecided);
            if (und0 | und1) {
                // compact the undecided nodes (those of slot 0, then of slot 1)
                // pair-interleaved, so that one pass
                // tests two nodes with packed FP32x2 arithmetic; every packed
                // operation rounds exactly like the scalar one it replaces
                const int c0 = __popc(und0), u = c0 + __popc(und1);
                nVote += u;
                const int k0 = __popc(und0 & lt), k1 = c0 + __popc(und1 & lt);
                auto stage = [&](const Slot& t, int k) {
                    float* e = reinterpret_cast<float*>(&sVote[w][2 * (k >> 1)]) + (k & 1);
                    e[0] = t.com.x;
                    e[2] = t.com.y;
                    e[4] = t.com.z;
                    e[6] = t.sizeSq;
                    if (kRelative) sVoteMs[w][k] = t.com.w * t.sizeSq;
                };
                stage(s0, s0.undecided ? k0 : 64);
                stage(s1, s1.undecided ? k1 : 64);
                __syncwarp();
                const ulonglong2* V = reinterpret_cast<const ulonglong2*>(sVote[w]);
                const f32x2 th2 = pack2(thetaSq, thetaSq);
                const float kAa = kA * myA, kAa1 = kA * myA1;
                // which of the two staged nodes a body at (x, y, z) wants opened
                auto wants2 = [&](ulonglong2 xy, ulonglong2 zs, f32x2 ms, float bx, float by, float bz, float ka,
                                  bool& wa, bool& wb) {
                    const f32x2 dx = sub2(pack2(bx, bx), xy.x), dy = sub2(pack2(by, by), xy.y);
                    const f32x2 dz = sub2(pack2(bz, bz), zs.x);
                    const f32x2 d2 = fma2(dz, dz, fma2(dx, dx, mul2(dy, dy)));  // ref_dist_sq, packed
                    float ta, tb, sa, sb;
                    unpack2(mul2(th2, d2), ta, tb);
                    unpack2(zs.y, sa, sb);
                    wa = !(sa < ta);
                    wb = !(sb < tb);
                    if (kRelative) {
                        float ra, rb, ma, mb;
                        unpack2(mul2(pack2(ka, ka), mul2(d2, d2)), ra, rb);
                        unpack2(ms, ma, mb);
                        wa = wa || (ma > ra);
                        wb = wb || (mb > rb);
                    }
                };
                // each lane collects its own body's wishes, bit j for staged node
                // j; one warp OR per 32 staged nodes then gives the verdicts
                // (1% faster than an OR after every pass)
                unsigned long long mine = 0ull;
#pragma unroll 2
                for (int j = 0; j < u; j += 2) {
                    const ulonglong2 xy = V[j], zs = V[j + 1];
                    f32x2 ms = 0ull;
                    if (kRelative) ms = *reinterpret_cast<const f32x2*>(&sVoteMs[w][j]);
                    bool wa, wb;
                    wants2(xy, zs, ms, p.x, p.y, p.z, kAa, wa, wb);
                    wa = valid && wa;
                    wb = valid && wb;
                    if (kWide) {
                        bool va, vb;
                        wants2(xy, zs, ms, p1.x, p1.y, p1.z, kAa1, va, vb);
                        wa = wa || (valid1 && va);
                        wb = wb || (valid1 && vb);
                    }
                    mine |= (unsigned long long)((wa ? 1u : 0u) | (wb ? 2u : 0u)) << j;
                }
                // an odd count leaves the last pair's second half stale: masked
                const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)mine);
                const unsigned hi = u > 32 ? __reduce_or_sync(0xffffffffu, (unsigned)(mine >> 32)) : 0u;
                unsigned long long openedC = ((unsigned long long)hi << 32) | lo;
                if (u < 64) openedC &= (1ull << u) - 1ull;
                s0.open = s0.open || (s0.undecided && ((openedC >> k0) & 1ull));
                s1.open = s1.open || (s1.undecided && ((openedC >> k1) & 1ull));
                __syncwarp();
            }
            const bool acc0 = (kBuckets ? s0.idx != -1 : s0.idx >= 0) && !s0.open;
            const bool acc1 = (kBuckets ? s1.idx != -1 : s1.idx >= 0) && !s1.open;
            const unsigned am0 = __ballot_sync(0xffffffffu, acc0), am1 = __ballot_sync(0xffffffffu, acc1);
            nTested += take;
            append(s0, acc0, listLen + __popc(am0 & lt));
            append(s1, acc1, listLen + __popc(am0) + __popc(am1 & lt));
            listLen += __popc(am0) + __popc(am1);
            // opened nodes -> children (or a bucket's bodies) onto the stack
            int f0, f1, d0, d1;
            const int n0 = children(s0, f0, d0), n1 = children(s1, f1, d1);
            int incl = n0 + n1;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int pushed = __shfl_sync(0xffffffffu, incl, 31);
            if (pushed) {
                if (top + pushed > stackCap) {
                    overflow = true;
                    break;
                }
                const int base0 = top + incl - n0 - n1, base1 = base0 + n0;
                if (top + pushed <= stackSmem) {  // uniform: the usual case
                    // at most 8 entries per slot here (a bucket holds at most
                    // leafSize bodies; kBuckets walks take the loop below)
                    int* q0 = &sStk[base0];
                    int* q1 = &sStk[base1];
                    if (kBuckets && leafSize > 8) {
                        const int w0 = __reduce_max_sync(0xffffffffu, n0), w1 = __reduce_max_sync(0xffffffffu, n1);
                        for (int c = 0; c < w0; c++)
                            if (c < n0) q0[c] = f0 + d0 * c;
                        for (int c = 0; c < w1; c++)
                            if (c < n1) q1[c] = f1 + d1 * c;
                    } else {
#pragma unroll
                        for (int c = 0; c < 8; c++) {  // predicated, no loop
                            if (c < n0) q0[c] = f0 + d0 * c;
                            if (c < n1) q1[c] = f1 + d1 * c;
                        }
                    }
                } else {
                    for (int c = 0; c < n0; c++) push(base0 + c, f0 + d0 * c);
                    for (int c = 0; c < n1; c++) push(base1 + c, f1 + d1 * c);
                }
                top += pushed;
                maxTop = top > maxTop ? top : maxTop;
            }
            __syncwarp();
            if (listLen > kListCap - 64) {
                flush(listLen);
                countInteractions(listLen, nValid);
                if (lane == 0) sGroupLen[w][1] += listLen;
                listLen = 0;
                __syncwarp();
            }
        }
        if (overflow && lane == 0) bh_set_error(err, BH_ERR_STACK_OVERFLOW);
        if (listLen > 0) {
            flush(listLen);
            countInteractions(listLen, nValid);
            if (lane == 0) sGroupLen[w][1] += listLen;
        }
        if (a.groupLen && lane == 0) a.groupLen[sGroupLen[w][0]] = sGroupLen[w][1];
        __syncwarp();
        // results of one body: acceleration, |a|, and the fused kick-drift
        auto finish = [&](int bi, float bx, float by, float bz, float bm_, float s0, float s1, float s2, float c0,
                          float c1, float c2) {
            float gx = G * s0, gy = G * s1, gz = G * s2;
            if (kCompensated) { gx = G * (s0 - c0); gy = G * (s1 - c1); gz = G * (s2 - c2); }
            if (a.accOut) a.accOut[bi] = make_float3(gx, gy, gz);
            if (a.aMagOut) a.aMagOut[bi] = sqrtf(gx * gx + gy * gy + gz * gz);
            if (kFused) {
                // tree.cu:694-702: v = v + a dt, x = x + v dt (both fused)
                const float3 v = a.velIn[bi];
                const float vx = __fmaf_rn(gx, dt, v.x), vy = __fmaf_rn(gy, dt, v.y), vz = __fmaf_rn(gz, dt, v.z);
                a.velOut[bi] = make_float3(vx, vy, vz);
                const float4 np = make_float4(__fmaf_rn(vx, dt, bx), __fmaf_rn(vy, dt, by), __fmaf_rn(vz, dt, bz), bm_);
                a.posOut[bi] = np;
                if (a.idOut) a.idOut[bi] = a.idIn[bi];
                if (a.posHost) {  // the caller's host arrays, written over PCIe as groups finish
                    a.posHost[bi] = np;
                    a.velHost[bi] = make_float3(vx, vy, vz);
                    a.idHost[bi] = a.idIn[bi];
                }
            }
        };
        if (kSumsSmem) {
            const float (*S)[32] = sSum[w];
            sx = S[0][lane]; sy = S[1][lane]; sz = S[2][lane];
            cx = S[3][lane]; cy = S[4][lane]; cz = S[5][lane];
            if (kWide) {
                tx = S[kSums - 6][lane]; ty = S[kSums - 5][lane]; tz = S[kSums - 4][lane];
                ux = S[kSums - 3][lane]; uy = S[kSums - 2][lane]; uz = S[kSums - 1][lane];
            }
        }
        if (valid) finish(b, p.x, p.y, p.z, p.w, sx, sy, sz, cx, cy, cz);
        if (kWide && valid1) finish(b1, p1.x, p1.y, p1.z, pos[b1].w, tx, ty, tz, ux, uy, uz);
    }
    if (lane == 0) {
        atomicAdd(&a.ctr->interactions, (unsigned long long)nInteract);
        atomicAdd(&a.ctr->nodesTested, (unsigned long long)nTested);
        atomicAdd(&a.ctr->undecided, (unsigned long long)nVote);
        atomicMax(&a.ctr->maxStack, maxTop);
    }
}

// Walk order for the next walk: the groups by decreasing interaction-list
// length of the last walk (a group covers almost the same bodies from one
// step to the next), so that the persistent grid's warps finish together
// instead of waiting on a few long groups taken last.  A counting sort on 64
// logarithmic length bins in two launches of one thread per group: per-block
// bin counts, then each block finds where its groups of each bin start and
// scatters them.  The order inside a bin is arbitrary (it changes only which
// warp walks a group, never a result).
constexpr int kOrderThreads = 1024;
constexpr int kOrderBins = 64;

__device__ __forceinline__ int order_bin(int l) {
    l = l < 0 ? 0 : (l > (1 << 15) ? (1 << 15) : l);
    const int b = (int)(4.0f * __log2f((float)l + 1.0f));  // 4 bins per doubling
    return kOrderBins - 1 - (b < kOrderBins - 1 ? b : kOrderBins - 1);  // longest first
}

// blockHist[block][bin] = groups of this block's 1024 in each bin
__global__ void __launch_bounds__(kOrderThreads) k_group_order_count(const int* __restrict__ len, int groups,
                                                                     int* __restrict__ blockHist) {
    __shared__ int hist[kOrderBins];
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < kOrderBins) hist[threadIdx.x] = 0;
    __syncthreads();
    const int g = blockIdx.x * kOrderThreads + threadIdx.x;
    const int b = g < groups ? order_bin(len[g]) : -1;
    // neighbouring groups have similar lengths: one atomic per bin and warp
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    if (b >= 0 && lane == __ffs(peers) - 1) atomicAdd(&hist[b], __popc(peers));
    __syncthreads();
    if (threadIdx.x < kOrderBins) blockHist[blockIdx.x * kOrderBins + threadIdx.x] = hist[threadIdx.x];
}

// order[pos] = g, pos = (groups in longer bins) + (groups of this bin in
// earlier blocks) + rank in this block
__global__ void __launch_bounds__(kOrderThreads) k_group_order_scatter(const int* __restrict__ len, int groups,
                                                                       const int* __restrict__ blockHist,
                                                                       int* __restrict__ order) {
    __shared__ int base[kOrderBins];
    __shared__ int firstHalf;  // groups in bins 0..31 (all blocks)
    const int lane = threadIdx.x & 31;
    if (threadIdx.x < kOrderBins) {  // two warps, 32 bins each
        int total = 0, before = 0;
        for (int k = 0; k < (int)gridDim.x; k++) {
            const int c = blockHist[k * kOrderBins + threadIdx.x];
            total += c;
            if (k < (int)blockIdx.x) before += c;
        }
        int x = total;  // inclusive scan of the bin totals within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        base[threadIdx.x] = x - total + before;
        if (threadIdx.x == 31) firstHalf = x;
    }
    __syncthreads();
    if (threadIdx.x >= 32 && threadIdx.x < kOrderBins) base[threadIdx.x] += firstHalf;
    __syncthreads();
    const int g = blockIdx.x * kOrderThreads + threadIdx.x;
    const int b = g < groups ? order_bin(len[g]) : -1;
    const unsigned peers = __match_any_sync(0xffffffffu, b);
    const int leader = __ffs(peers) - 1;
    int at = 0;
    if (b >= 0 && lane == leader) at = atomicAdd(&base[b], __popc(peers));
    at = __shfl_sync(0xffffffffu, at, leader);
    if (b >= 0) order[at + __popc(peers & lanemask_lt())] = g;
}

int bh_group_order_hist_ints(int groups) { return ((groups + kOrderThreads - 1) / kOrderThreads) * kOrderBins; }

cudaError_t bh_launch_group_order(const int* len, int groups, int* order, int* blockHist, cudaStream_t s) {
    if (groups <= 0) return cudaSuccess;
    const int blocks = (groups + kOrderThreads - 1) / kOrderThreads;
    k_group_order_count<<<blocks, kOrderThreads, 0, s>>>(len, groups, blockHist);
    k_group_order_scatter<<<blocks, kOrderThreads, 0, s>>>(len, groups, blockHist, order);
    return cudaGetLastError();
}

// Reference positionUpdater (tree.cu:678-703).
__global__ void __launch_bounds__(256)
k_kick_drift(float4* __restrict__ pos, float3* __restrict__ vel, const float3* __restrict__ acc, int n, float dt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float3 a = acc[i];
        float3 v = vel[i];
        float4 p = pos[i];
        v.x = __fmaf_rn(a.x, dt, v.x);
        v.y = __fmaf_rn(a.y, dt, v.y);
        v.z = __fmaf_rn(a.z, dt, v.z);
        p.x = __fmaf_rn(v.x, dt, p.x);
        p.y = __fmaf_rn(v.y, dt, p.y);
        p.z = __fmaf_rn(v.z, dt, p.z);
        vel[i] = v;
        pos[i] = p;
    }
}

// ---------------------------------------------------------------- launchers

int bh_walk_grid() { return bh_sm_count() * kBlocksPerSm; }
static_assert(kMinBlocksPlain <= kBlocksPerSm && kMinBlocksRelative <= kBlocksPerSm && kMinBlocksWide <= kBlocksPerSm,
              "spill area sizing");

size_t bh_walk_spill_ints() { return (size_t)bh_walk_grid() * kWarpsPerBlock * kSpillPerWarp; }

// One walk variant: the persistent grid fills every SM with as many blocks as
// are resident at once for this stack size (registers or shared memory,
// whichever binds first, never more than the register budget the variant was
// compiled for).
template <typename Kernel>
static cudaError_t launch_walk_variant(Kernel kernel, const WalkArgs& a, int maxBlocks, cudaStream_t s) {
    const size_t dyn = (size_t)kWarpsPerBlock * (size_t)a.stackSmem * sizeof(int);
    // deep stacks take the block past 48 KB of shared memory, which needs
    // the kernel's opt-in (a function attribute; harmless below that)
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    if (e != cudaSuccess) return e;
    int resident = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kernel, kThreads, dyn);
    if (e != cudaSuccess) return e;
    resident = resident < maxBlocks ? resident : maxBlocks;
    if (resident < 1) return cudaErrorInvalidConfiguration;
    kernel<<<bh_sm_count() * resident, kThreads, dyn, s>>>(a);
    return cudaGetLastError();
}

int bh_walk_stack_default() { return kStackSmemDefault; }

cudaError_t bh_launch_walk(const WalkArgs& in, bool fused, bool compensated, cudaStream_t s) {
    WalkArgs a = in;
    if (a.stackSmem == 0) a.stackSmem = kStackSmemDefault;
    if (a.stackSmem < BH_WALK_STACK_MIN || a.stackSmem > BH_WALK_STACK_MAX || a.stackSmem % 32 != 0)
        return cudaErrorInvalidValue;
    if (a.relative && !a.aMagIn) return cudaErrorInvalidValue;
    const bool buckets = a.leafSize > 1;
    if (buckets && !a.nFirst) return cudaErrorInvalidValue;
    const int width = a.groupWidth ? a.groupWidth : 32;
    if (width != 32 && width != 64) return cudaErrorInvalidValue;
    const bool wide = width == 64 && kWalkPacked;
    // one block per resident slot (the spill area is sized for bh_walk_grid(), the largest)
    const int maxBlocks = walk_min_blocks(a.relative, wide);
#define BH_WALK_LAUNCH(F, C, R, B, W) \
    return launch_walk_variant(k_walk<F, C, kWalkPacked, R, B, W && kWalkPacked>, a, maxBlocks, s)
#define BH_WALK_BUCKETS(F, C, R)                                   \
    do {                                                           \
        if (wide) {                                                \
            if (buckets) BH_WALK_LAUNCH(F, C, R, true, true);      \
            else BH_WALK_LAUNCH(F, C, R, false, true);             \
        } else {                                                   \
            if (buckets) BH_WALK_LAUNCH(F, C, R, true, false);     \
            else BH_WALK_LAUNCH(F, C, R, false, false);            \
        }                                                          \
    } while (0)
    if (a.relative) {
        if (fused) {
            if (compensated) BH_WALK_BUCKETS(true, true, true);
            else BH_WALK_BUCKETS(true, false, true);
        } else {
            if (compensated) BH_WALK_BUCKETS(false, true, true);
            else BH_WALK_BUCKETS(false, false, true);
        }
    } else {
        if (fused) {
            if (compensated) BH_WALK_BUCKETS(true, true, false);
            else BH_WALK_BUCKETS(true, false, false);
        } else {
            if (compensated) BH_WALK_BUCKETS(false, true, false);
            else BH_WALK_BUCKETS(false, false, false);
        }
    }
#undef BH_WALK_BUCKETS
#undef BH_WALK_LAUNCH
}

cudaError_t bh_launch_kick_drift(float4* pos, float3* vel, const float3* acc, int n, float dt,
                                 cudaStream_t s) {
    int grid = (n + 255) / 256;
    const int cap = 8 * bh_sm_count();
    grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
    k_kick_drift<<<grid, 256, 0, s>>>(pos, vel, acc, n, dt);
    return cudaGetLastError();
}
