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
//   - the 32 lanes test 32 different nodes at once (the reference tests one
//     node per step with all 32 lanes);
//   - a node is accepted without a vote when the distance from its centre of
//     mass to the group's bounding box already satisfies the criterion with a
//     2^-16 relative margin (which dominates every rounding difference), and
//     opened without a vote when one representative body already fails it;
//     only the rest take the exact group vote (same FP32 operations and
//     order as the reference, so the decision is bit-identical);
//   - accepted nodes' (centre of mass, mass) are appended to a per-warp list
//     in shared memory and evaluated in bulk: per interaction 3 FADD, 3 FFMA,
//     one MUFU rsqrt, 3 FMUL and 3 FFMA;
//   - sums are compensated per block of list entries (Kahan on the block
//     partials) when requested;
//   - warps fetch groups from an atomic cursor (dynamic load balance).
// Leaves never open, as in the reference (count <= 1 or no children).
#include <math.h>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kThreads = kWarpsPerBlock * 32;
constexpr int kStackSmem = 1024;  // stack entries per warp in shared memory
constexpr int kListCap = 128;     // interaction-list entries per warp
constexpr float kBoxMargin = 1.0f - 1.0f / 65536.0f;

__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// The reference's d^2 (tree.cu:611) as its compiled walk evaluates it:
// fma(dz, dz, fma(dx, dx, dy * dy)).  The opening test must round exactly
// like the reference's for the interaction sets to be identical.
__device__ __forceinline__ float ref_dist_sq(float dx, float dy, float dz) {
    return __fmaf_rn(dz, dz, __fmaf_rn(dx, dx, __fmul_rn(dy, dy)));
}

// stack access: entries past kStackSmem live in this warp's global spill area
struct WarpStack {
    int* smem;
    int* spill;
    __device__ __forceinline__ int get(int s) const { return s < kStackSmem ? smem[s] : spill[s - kStackSmem]; }
    __device__ __forceinline__ void put(int s, int v) const {
        if (s < kStackSmem) smem[s] = v;
        else spill[s - kStackSmem] = v;
    }
};

}  // namespace

template <bool kFused, bool kCompensated>
__global__ void __launch_bounds__(kThreads, 8)
k_walk(const float4* __restrict__ pos, int n, const WalkNode* __restrict__ wn, float theta, float eps2,
       float G, float3* __restrict__ accOut, const float3* __restrict__ velIn, float4* __restrict__ posOut,
       float3* __restrict__ velOut, const uint32_t* __restrict__ idIn, uint32_t* __restrict__ idOut,
       float dt, DevCounters* ctr, int* err, int* spillBase, int spillPerWarp) {
    __shared__ int sStack[kWarpsPerBlock][kStackSmem];
    __shared__ float4 sList[kWarpsPerBlock][kListCap];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = lanemask_lt();
    const WarpStack stack{sStack[w], spillBase + (size_t)(blockIdx.x * kWarpsPerBlock + w) * spillPerWarp};
    const int stackCap = kStackSmem + spillPerWarp;
    float4* list = sList[w];
    const float thetaSq = __fmul_rn(theta, theta);
    const int groups = (n + 31) >> 5;
    unsigned long long nInteract = 0, nTested = 0, nVote = 0;
    int maxTop = 0;

    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(&ctr->groupCursor, 1);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= groups) break;
        const int b = g * 32 + lane;
        const bool valid = b < n;
        const float4 p = valid ? pos[b] : make_float4(0.f, 0.f, 0.f, 0.f);
        const unsigned validMask = __ballot_sync(0xffffffffu, valid);
        const int nValid = __popc(validMask);

        // group bounding box (valid bodies) and representative body
        float lo[3] = {valid ? p.x : INFINITY, valid ? p.y : INFINITY, valid ? p.z : INFINITY};
        float hi[3] = {valid ? p.x : -INFINITY, valid ? p.y : -INFINITY, valid ? p.z : -INFINITY};
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
#pragma unroll
            for (int k = 0; k < 3; k++) {
                lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
                hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
            }
        float repX, repY, repZ;
        {
            const float mx = 0.5f * (lo[0] + hi[0]), my = 0.5f * (lo[1] + hi[1]), mz = 0.5f * (lo[2] + hi[2]);
            float d = valid ? (p.x - mx) * (p.x - mx) + (p.y - my) * (p.y - my) + (p.z - mz) * (p.z - mz) : INFINITY;
            int who = lane;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float od = __shfl_xor_sync(0xffffffffu, d, o);
                const int ow = __shfl_xor_sync(0xffffffffu, who, o);
                if (od < d || (od == d && ow < who)) { d = od; who = ow; }
            }
            repX = __shfl_sync(0xffffffffu, p.x, who);
            repY = __shfl_sync(0xffffffffu, p.y, who);
            repZ = __shfl_sync(0xffffffffu, p.z, who);
        }

        // root's children onto the stack
        int top;
        {
            const int rb = wn[0].childBegin, re = wn[0].childEnd;
            top = re - rb;
            if (lane < top) stack.put(lane, rb + lane);
        }
        __syncwarp();
        int listLen = 0;
        float ax = 0.f, ay = 0.f, az = 0.f;   // partial sums of the current list block
        float sx = 0.f, sy = 0.f, sz = 0.f;   // running sums
        float cx = 0.f, cy = 0.f, cz = 0.f;   // Kahan compensation

        auto flush = [&](int cnt) {
            int k = 0;
#pragma unroll 4
            for (; k < cnt; k++) {
                const float4 c = list[k];
                const float dx = c.x - p.x, dy = c.y - p.y, dz = c.z - p.z;
                const float r2 = __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmaf_rn(dx, dx, eps2)));
                const float ri = rsqrt_approx(r2);
                const float f = (c.w * ri) * (ri * ri);
                ax = __fmaf_rn(f, dx, ax);
                ay = __fmaf_rn(f, dy, ay);
                az = __fmaf_rn(f, dz, az);
            }
            if (kCompensated) {
                float y, t;
                y = ax - cx; t = sx + y; cx = (t - sx) - y; sx = t;
                y = ay - cy; t = sy + y; cy = (t - sy) - y; sy = t;
                y = az - cz; t = sz + y; cz = (t - sz) - y; sz = t;
            } else {
                sx += ax; sy += ay; sz += az;
            }
            ax = ay = az = 0.f;
        };

        bool overflow = false;
        while (top > 0) {
            const int take = top < 32 ? top : 32;
            top -= take;
            const int nodeIdx = lane < take ? stack.get(top + lane) : -1;
            __syncwarp();
            const bool has = nodeIdx >= 0;
            float4 com = make_float4(0.f, 0.f, 0.f, 0.f);
            int cb = 0, ce = 0;
            float sizeSq = 0.f;
            if (has) {
                com = wn[nodeIdx].com;
                const int4 meta = *reinterpret_cast<const int4*>(&wn[nodeIdx].childBegin);
                cb = meta.x;
                ce = meta.y;
                sizeSq = __int_as_float(meta.z);
            }
            const bool leaf = cb == ce;
            bool open = false, undecided = false;
            if (has && !leaf) {
                const float gx = fmaxf(fmaxf(lo[0] - com.x, com.x - hi[0]), 0.f);
                const float gy = fmaxf(fmaxf(lo[1] - com.y, com.y - hi[1]), 0.f);
                const float gz = fmaxf(fmaxf(lo[2] - com.z, com.z - hi[2]), 0.f);
                const float boxD2 = gx * gx + gy * gy + gz * gz;
                if (!(thetaSq * boxD2 * kBoxMargin > sizeSq)) {
                    const float d2 = ref_dist_sq(repX - com.x, repY - com.y, repZ - com.z);
                    if (!(sizeSq < __fmul_rn(thetaSq, d2))) open = true;
                    else undecided = true;
                }
            }
            // exact group vote for the undecided nodes (tree.cu:629-640)
            unsigned und = __ballot_sync(0xffffffffu, undecided);
            nVote += __popc(und);
            while (und) {
                const int j = __ffs(und) - 1;
                und &= und - 1;
                const float qx = __shfl_sync(0xffffffffu, com.x, j);
                const float qy = __shfl_sync(0xffffffffu, com.y, j);
                const float qz = __shfl_sync(0xffffffffu, com.z, j);
                const float qs = __shfl_sync(0xffffffffu, sizeSq, j);
                const float d2 = ref_dist_sq(p.x - qx, p.y - qy, p.z - qz);
                const bool want = valid && !(qs < __fmul_rn(thetaSq, d2));
                if (__any_sync(0xffffffffu, want) && lane == j) open = true;
            }
            const bool accept = has && !open;
            const unsigned am = __ballot_sync(0xffffffffu, accept);
            nTested += take;
            // accepted nodes -> interaction list
            if (accept) list[listLen + __popc(am & lt)] = com;
            listLen += __popc(am);
            // opened nodes -> children onto the stack.  Children live on the
            // next level (higher indices), at most 8: a range that breaks
            // this is a broken tree, reported rather than followed.
            int nch = open ? ce - cb : 0;
            if (open && (cb <= nodeIdx || nch > 8)) {
                bh_set_error(err, BH_ERR_INTERNAL);
                nch = 0;
            }
            int incl = nch;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            const int pushed = __shfl_sync(0xffffffffu, incl, 31);
            if (top + pushed > stackCap) {
                overflow = true;
                break;
            }
            for (int c = 0; c < nch; c++) stack.put(top + incl - nch + c, cb + c);
            top += pushed;
            maxTop = top > maxTop ? top : maxTop;
            __syncwarp();
            if (listLen > kListCap - 32) {
                __syncwarp();
                flush(listLen);
                nInteract += (unsigned long long)listLen * nValid;
                listLen = 0;
                __syncwarp();
            }
        }
        if (overflow && lane == 0) bh_set_error(err, BH_ERR_STACK_OVERFLOW);
        __syncwarp();
        if (listLen > 0) {
            flush(listLen);
            nInteract += (unsigned long long)listLen * nValid;
        }
        __syncwarp();
        if (valid) {
            float gx = G * sx, gy = G * sy, gz = G * sz;
            if (kCompensated) { gx = G * (sx - cx); gy = G * (sy - cy); gz = G * (sz - cz); }
            if (accOut) accOut[b] = make_float3(gx, gy, gz);
            if (kFused) {
                // tree.cu:694-702: v = v + a dt, x = x + v dt (both fused)
                const float3 v = velIn[b];
                const float vx = __fmaf_rn(gx, dt, v.x), vy = __fmaf_rn(gy, dt, v.y), vz = __fmaf_rn(gz, dt, v.z);
                velOut[b] = make_float3(vx, vy, vz);
                posOut[b] = make_float4(__fmaf_rn(vx, dt, p.x), __fmaf_rn(vy, dt, p.y), __fmaf_rn(vz, dt, p.z), p.w);
                if (idOut) idOut[b] = idIn[b];
            }
        }
    }
    if (lane == 0) {
        atomicAdd(&ctr->interactions, nInteract);
        atomicAdd(&ctr->nodesTested, nTested);
        atomicAdd(&ctr->undecided, nVote);
        atomicMax(&ctr->maxStack, maxTop);
    }
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
namespace {
constexpr int kBlocksPerSm = 8;
constexpr int kSpillPerWarp = 4096;  // global stack entries per warp beyond shared memory
}  // namespace

int bh_walk_grid() { return bh_sm_count() * kBlocksPerSm; }

size_t bh_walk_spill_ints() { return (size_t)bh_walk_grid() * kWarpsPerBlock * kSpillPerWarp; }

cudaError_t bh_launch_walk(const WalkArgs& a, bool fused, bool compensated, cudaStream_t s) {
    const int grid = bh_walk_grid();
#define BH_WALK_LAUNCH(F, C)                                                                          \
    k_walk<F, C><<<grid, kThreads, 0, s>>>(a.pos, a.n, a.wn, a.theta, a.eps2, a.G, a.accOut, a.velIn, \
                                           a.posOut, a.velOut, a.idIn, a.idOut, a.dt, a.ctr, a.err,   \
                                           a.spill, kSpillPerWarp)
    if (fused) {
        if (compensated) BH_WALK_LAUNCH(true, true);
        else BH_WALK_LAUNCH(true, false);
    } else {
        if (compensated) BH_WALK_LAUNCH(false, true);
        else BH_WALK_LAUNCH(false, false);
    }
#undef BH_WALK_LAUNCH
    return cudaGetLastError();
}

cudaError_t bh_launch_kick_drift(float4* pos, float3* vel, const float3* acc, int n, float dt,
                                 cudaStream_t s) {
    int grid = (n + 255) / 256;
    const int cap = 8 * bh_sm_count();
    grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
    k_kick_drift<<<grid, 256, 0, s>>>(pos, vel, acc, n, dt);
    return cudaGetLastError();
}
