// bbox_morton.cu — bounding box and Morton keys (sm_100a).
//
// Reference: localMinMaxFinder / globalMinMaxReducer (tree.cu:385-490) reduce
// the box in two launches and the host turns it into a world box after two
// blocking copies (basicGravity.cu:79-113); mortonEncode (tree.cu:332-367)
// then reads that box by value.  Here one launch reduces the box and its last
// block derives the world box on the device, so the keys kernel reads it from
// device memory and no host round trip sits between the stages.  The keys
// kernel also produces the radix-sort digit histograms, so the sort does not
// read the keys an extra time.
#include <math.h>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"

namespace {

constexpr int kBoxThreads = 256;

__device__ __forceinline__ void warp_minmax(float v[6]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; k++) v[k] = fminf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
#pragma unroll
        for (int k = 3; k < 6; k++) v[k] = fmaxf(v[k], __shfl_xor_sync(0xffffffffu, v[k], o));
    }
}

// Block-wide min/max of v[0..2] and max of v[3..5]; result valid in thread 0.
__device__ __forceinline__ void block_minmax(float v[6]) {
    __shared__ float part[kBoxThreads / 32][6];
    warp_minmax(v);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0)
#pragma unroll
        for (int k = 0; k < 6; k++) part[w][k] = v[k];
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < 6; k++) v[k] = (lane_id() < (unsigned)nw) ? part[lane_id()][k] : (k < 3 ? INFINITY : -INFINITY);
        warp_minmax(v);
    }
    __syncthreads();
}

// Block-wide sums of v[0..3] in FP64, in a fixed order (deterministic);
// result valid in thread 0.
__device__ __forceinline__ void block_sum4(double v[4]) {
    __shared__ double part[kBoxThreads / 32][4];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int w = threadIdx.x >> 5;
    if (lane_id() == 0)
#pragma unroll
        for (int k = 0; k < 4; k++) part[w][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int j = 1; j < nw; j++)
#pragma unroll
            for (int k = 0; k < 4; k++) v[k] += part[j][k];
    }
    __syncthreads();
}

}  // namespace

// One launch: every block reduces a grid-stride slice; the last block to
// finish (ticket) reduces the block results and writes the world box
// (basicGravity.cu:90-112: extent = max(w, h, d), scale = (2^bits-1)/extent).
// It also zeroes `zeroWords` words at `zeroBuf` (the digit histograms the keys
// kernel accumulates next) and re-arms the ticket for the next call.
// With root != NULL the same pass sums mass and mass-weighted positions in
// FP64 (block partials in partials64, combined by the last block in block
// order) and writes the root's FP64 mass, centre of mass and box.
__global__ void __launch_bounds__(kBoxThreads)
k_bbox(const float4* __restrict__ pos, int n, float* __restrict__ partials, unsigned* ticket,
       DevBox* box, float3* outMin, float3* outMax, int bits, int* err, uint32_t* zeroBuf,
       int zeroWords, double* __restrict__ partials64, DevRoot* root) {
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    double m4[4] = {0.0, 0.0, 0.0, 0.0};  // sum m, sum m x, sum m y, sum m z
    const bool f64 = root != nullptr;
    bool bad = false;
    auto take = [&](const float4 p) {
        bad |= !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
        v[0] = fminf(v[0], p.x); v[3] = fmaxf(v[3], p.x);
        v[1] = fminf(v[1], p.y); v[4] = fmaxf(v[4], p.y);
        v[2] = fminf(v[2], p.z); v[5] = fmaxf(v[5], p.z);
        if (f64) {
            const double m = p.w;
            m4[0] += m;
            m4[1] = fma(m, (double)p.x, m4[1]);
            m4[2] = fma(m, (double)p.y, m4[2]);
            m4[3] = fma(m, (double)p.z, m4[3]);
        }
    };
    // four independent loads in flight per thread, then the remainder
    const int stride = gridDim.x * blockDim.x;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    for (; i + 3 * stride < n; i += 4 * stride) {
        const float4 a = __ldg(&pos[i]), b = __ldg(&pos[i + stride]);
        const float4 c = __ldg(&pos[i + 2 * stride]), d = __ldg(&pos[i + 3 * stride]);
        take(a); take(b); take(c); take(d);
    }
    for (; i < n; i += stride) take(__ldg(&pos[i]));
    if (bad) bh_set_error(err, BH_ERR_NONFINITE);
    block_minmax(v);
    if (f64) block_sum4(m4);
    __shared__ bool last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 6; k++) partials[blockIdx.x * 6 + k] = v[k];
        if (f64)
#pragma unroll
            for (int k = 0; k < 4; k++) partials64[blockIdx.x * 4 + k] = m4[k];
        __threadfence();
        last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    float r[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int k = 0; k < 3; k++) r[k] = fminf(r[k], __ldcg(&partials[b * 6 + k]));
#pragma unroll
        for (int k = 3; k < 6; k++) r[k] = fmaxf(r[k], __ldcg(&partials[b * 6 + k]));
    }
    block_minmax(r);
    if (f64) {
        double t[4] = {0.0, 0.0, 0.0, 0.0};
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
            for (int k = 0; k < 4; k++) t[k] += __ldcg(&partials64[b * 4 + k]);
        block_sum4(t);
        if (threadIdx.x == 0) {
            DevRoot rt;
            rt.mass = t[0];
            const double inv = t[0] > 0.0 ? 1.0 / t[0] : 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                rt.com[k] = t[k + 1] * inv;
                rt.mn[k] = (double)r[k];
                rt.mx[k] = (double)r[k + 3];
            }
            *root = rt;
        }
    }
    if (threadIdx.x == 0) {
        const float w = __fsub_rn(r[3], r[0]), h = __fsub_rn(r[4], r[1]), d = __fsub_rn(r[5], r[2]);
        const float extent = fmaxf(w, fmaxf(h, d));
        const float scale = __fdiv_rn((float)((1u << bits) - 1u), extent);
        DevBox bx;
        bx.mn[0] = r[0]; bx.mn[1] = r[1]; bx.mn[2] = r[2];
        bx.mx[0] = r[3]; bx.mx[1] = r[4]; bx.mx[2] = r[5];
        bx.extent = extent;
        bx.scale = scale;
        bx.extX = w;
        bx.pad[0] = bx.pad[1] = bx.pad[2] = 0;
        *box = bx;
        if (outMin) *outMin = make_float3(r[0], r[1], r[2]);
        if (outMax) *outMax = make_float3(r[3], r[4], r[5]);
        if (!(extent > 0.0f) || !isfinite(extent) || !(scale > 0.0f) || !isfinite(scale))
            bh_set_error(err, BH_ERR_DEGENERATE_BOX);
        *ticket = 0u;
    }
    for (int i = threadIdx.x; i < zeroWords; i += blockDim.x) zeroBuf[i] = 0u;
}

// Batch of independent systems: block s reduces the bodies of system s
// (segment [segOff[s], segOff[s+1])) and writes that system's world box, with
// the same arithmetic as k_bbox.  Block 0 also zeroes the digit histograms.
__global__ void __launch_bounds__(kBoxThreads)
k_bbox_segments(const float4* __restrict__ pos, const int* __restrict__ segOff, int systems, DevBox* boxes, int bits,
                int* err, uint32_t* zeroBuf, int zeroWords) {
    for (int sy = blockIdx.x; sy < systems; sy += gridDim.x) {
        const int lo = segOff[sy], hi = segOff[sy + 1];
        float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
        bool bad = false;
        auto take = [&](const float4 p) {
            bad |= !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z));
            v[0] = fminf(v[0], p.x); v[3] = fmaxf(v[3], p.x);
            v[1] = fminf(v[1], p.y); v[4] = fmaxf(v[4], p.y);
            v[2] = fminf(v[2], p.z); v[5] = fmaxf(v[5], p.z);
        };
        // eight independent loads in flight per thread: one block may have to
        // cover a system of tens of thousands of bodies
        constexpr int kIn = 8;
        int i = lo + threadIdx.x;
        for (; i + (kIn - 1) * (int)blockDim.x < hi; i += kIn * blockDim.x) {
            float4 q[kIn];
#pragma unroll
            for (int u = 0; u < kIn; u++) q[u] = __ldg(&pos[i + u * blockDim.x]);
#pragma unroll
            for (int u = 0; u < kIn; u++) take(q[u]);
        }
        for (; i < hi; i += blockDim.x) take(__ldg(&pos[i]));
        if (bad) bh_set_error(err, BH_ERR_NONFINITE);
        block_minmax(v);
        if (threadIdx.x == 0) {
            const float w = __fsub_rn(v[3], v[0]), h = __fsub_rn(v[4], v[1]), d = __fsub_rn(v[5], v[2]);
            const float extent = fmaxf(w, fmaxf(h, d));
            const float scale = __fdiv_rn((float)((1u << bits) - 1u), extent);
            DevBox bx;
            bx.mn[0] = v[0]; bx.mn[1] = v[1]; bx.mn[2] = v[2];
            bx.mx[0] = v[3]; bx.mx[1] = v[4]; bx.mx[2] = v[5];
            bx.extent = extent;
            bx.scale = scale;
            bx.extX = w;
            bx.pad[0] = bx.pad[1] = bx.pad[2] = 0;
            boxes[sy] = bx;
            if (!(extent > 0.0f) || !isfinite(extent) || !(scale > 0.0f) || !isfinite(scale))
                bh_set_error(err, BH_ERR_DEGENERATE_BOX);
        }
    }
    if (blockIdx.x == 0)
        for (int i = threadIdx.x; i < zeroWords; i += blockDim.x) zeroBuf[i] = 0u;
}

// Morton keys (tree.cu:343-367 generalised to `bits` bits per axis):
// grid coordinate = (uint32)((p - min) * scale) masked to `bits` bits; key =
// interleave with x highest (x<<2 | y<<1 | z per bit); idx[i] = i.
// Spreading uses a 256-entry table in shared memory: spread[b] moves bit k of
// byte b to bit 3k.
//
// In a batch (sysOf set) body i uses the world box of its system sysOf[i] and
// the system index goes above the Morton bits: key |= sys << 3*bits, so one
// sort orders the bodies by system, then along each system's curve.
//
// With `hist` set, the kernel also counts the radix-sort digits (8-bit digits
// 0..npass-1) of its keys.  Bodies arrive in nearly sorted order (last step's
// Morton order), so each thread counts runs of equal digits over 8
// consecutive keys and adds a run with one shared-memory atomic.
constexpr int kMortonThreads = 256;
constexpr int kMortonPerThread = 8;

__device__ __forceinline__ uint64_t spread_coord(const uint32_t* spread, uint32_t v) {
    return (uint64_t)spread[v & 255u] | ((uint64_t)spread[(v >> 8) & 255u] << 24) |
           ((uint64_t)spread[(v >> 16) & 255u] << 48);
}

__global__ void __launch_bounds__(kMortonThreads)
k_morton(const float4* __restrict__ pos, int n, const DevBox* __restrict__ box, worldBox boxVal,
         int bits, uint64_t* __restrict__ keys, uint32_t* __restrict__ idx,
         uint32_t* __restrict__ hist, int npass, const uint16_t* __restrict__ sysOf) {
    __shared__ uint32_t spread[256];
    __shared__ uint32_t shist[8][256];
    __shared__ __align__(16) uint64_t skeys[kMortonThreads * kMortonPerThread];
    {
        uint32_t b = threadIdx.x, s = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) s |= ((b >> k) & 1u) << (3 * k);
        spread[threadIdx.x] = s;
    }
    if (hist)
        for (int i = threadIdx.x; i < npass * 256; i += blockDim.x) (&shist[0][0])[i] = 0u;
    __syncthreads();

    const float minX = box ? box->mn[0] : boxVal.minX;
    const float minY = box ? box->mn[1] : boxVal.minY;
    const float minZ = box ? box->mn[2] : boxVal.minZ;
    const float scale = box ? box->scale : boxVal.scale;
    const uint32_t mask = (bits >= 32) ? 0xffffffffu : ((1u << bits) - 1u);
    const int tile = kMortonThreads * kMortonPerThread;
    for (int base = blockIdx.x * tile; base < n; base += gridDim.x * tile) {
#pragma unroll
        for (int j = 0; j < kMortonPerThread; j++) {
            const int i = base + j * kMortonThreads + threadIdx.x;
            uint64_t key = ~0ull;
            if (i < n) {
                const float4 p = __ldg(&pos[i]);
                float mx = minX, my = minY, mz = minZ, sc = scale;
                uint64_t sys = 0;
                if (sysOf) {
                    sys = sysOf[i];
                    const DevBox* bx = box + sys;
                    mx = bx->mn[0]; my = bx->mn[1]; mz = bx->mn[2]; sc = bx->scale;
                }
                const uint32_t x = __float2uint_rz(__fmul_rn(__fsub_rn(p.x, mx), sc)) & mask;
                const uint32_t y = __float2uint_rz(__fmul_rn(__fsub_rn(p.y, my), sc)) & mask;
                const uint32_t z = __float2uint_rz(__fmul_rn(__fsub_rn(p.z, mz), sc)) & mask;
                key = (spread_coord(spread, x) << 2) | (spread_coord(spread, y) << 1) | spread_coord(spread, z);
                if (sysOf) key |= sys << (3 * bits);
                keys[i] = key;
                if (idx) idx[i] = (uint32_t)i;
            }
            skeys[j * kMortonThreads + threadIdx.x] = key;
        }
        if (hist) {
            __syncthreads();
            const int first = threadIdx.x * kMortonPerThread;
            int valid = n - (base + first);
            valid = valid < 0 ? 0 : (valid > kMortonPerThread ? kMortonPerThread : valid);
            // this thread's run of consecutive keys, read once for all passes
            uint64_t kk[kMortonPerThread];
#pragma unroll
            for (int j = 0; j < kMortonPerThread; j += 2) {  // 16-byte loads
                const ulonglong2 two = *reinterpret_cast<const ulonglong2*>(&skeys[first + j]);
                kk[j] = two.x;
                kk[j + 1] = two.y;
            }
            for (int p = 0; p < npass; p++) {
                const int shift = 8 * p;
                uint32_t run = 0, cur = 0;
#pragma unroll
                for (int j = 0; j < kMortonPerThread; j++) {
                    if (j >= valid) break;
                    const uint32_t d = (uint32_t)(kk[j] >> shift) & 255u;
                    if (run && d != cur) { atomicAdd(&shist[p][cur], run); run = 0; }
                    cur = d;
                    run++;
                }
                if (run) atomicAdd(&shist[p][cur], run);
            }
            __syncthreads();
        }
    }
    if (hist) {
        __syncthreads();
        for (int i = threadIdx.x; i < npass * 256; i += blockDim.x) {
            const uint32_t c = (&shist[0][0])[i];
            if (c) atomicAdd(&hist[i], c);
        }
    }
}

// ---------------------------------------------------------------------------
// Reference-compatible two-stage box (tree.cu:414-490): per-block partial
// corners, then one block reduces `count` of them.
__global__ void __launch_bounds__(kBoxThreads)
k_local_minmax(const float4* __restrict__ pos, unsigned n, float3* minCorner, float3* maxCorner) {
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = __ldg(&pos[i]);
        v[0] = fminf(v[0], p.x); v[3] = fmaxf(v[3], p.x);
        v[1] = fminf(v[1], p.y); v[4] = fmaxf(v[4], p.y);
        v[2] = fminf(v[2], p.z); v[5] = fmaxf(v[5], p.z);
    }
    block_minmax(v);
    if (threadIdx.x == 0) {
        minCorner[blockIdx.x] = make_float3(v[0], v[1], v[2]);
        maxCorner[blockIdx.x] = make_float3(v[3], v[4], v[5]);
    }
}

__global__ void __launch_bounds__(kBoxThreads)
k_global_minmax(const float3* __restrict__ minCorner, const float3* __restrict__ maxCorner, int count,
                float3* outMin, float3* outMax) {
    float v[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const float3 a = minCorner[i], b = maxCorner[i];
        v[0] = fminf(v[0], a.x); v[1] = fminf(v[1], a.y); v[2] = fminf(v[2], a.z);
        v[3] = fmaxf(v[3], b.x); v[4] = fmaxf(v[4], b.y); v[5] = fmaxf(v[5], b.z);
    }
    block_minmax(v);
    if (threadIdx.x == 0) {
        *outMin = make_float3(v[0], v[1], v[2]);
        *outMax = make_float3(v[3], v[4], v[5]);
    }
}

// ---------------------------------------------------------------- launchers
cudaError_t bh_launch_bbox(const float4* pos, int n, float* partials, unsigned* ticket, DevBox* box,
                           float3* outMin, float3* outMax, int bits, int* err, uint32_t* zeroBuf,
                           int zeroWords, cudaStream_t s, double* partials64, DevRoot* root) {
    if ((root == nullptr) != (partials64 == nullptr)) return cudaErrorInvalidValue;
    int grid = (n + kBoxThreads * 8 - 1) / (kBoxThreads * 8);
    const int cap = 6 * bh_sm_count();
    grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
    grid = grid > kBboxMaxGrid ? kBboxMaxGrid : grid;
    k_bbox<<<grid, kBoxThreads, 0, s>>>(pos, n, partials, ticket, box, outMin, outMax, bits, err, zeroBuf,
                                        zeroWords, partials64, root);
    return cudaGetLastError();
}

cudaError_t bh_launch_morton(const float4* pos, int n, const DevBox* boxPtr, worldBox boxVal, int bits,
                             uint64_t* keys, uint32_t* idx, uint32_t* hist, int npass, cudaStream_t s,
                             const uint16_t* sysOf) {
    const int tile = kMortonThreads * kMortonPerThread;
    int grid = (n + tile - 1) / tile;
    grid = grid < 1 ? 1 : grid;
    k_morton<<<grid, kMortonThreads, 0, s>>>(pos, n, boxPtr, boxVal, bits, keys, idx, hist, npass, sysOf);
    return cudaGetLastError();
}

cudaError_t bh_launch_bbox_segments(const float4* pos, const int* segOff, int systems, DevBox* boxes, int bits,
                                    int* err, uint32_t* zeroBuf, int zeroWords, cudaStream_t s) {
    int grid = systems < 4 * bh_sm_count() ? systems : 4 * bh_sm_count();
    grid = grid < 1 ? 1 : grid;
    k_bbox_segments<<<grid, kBoxThreads, 0, s>>>(pos, segOff, systems, boxes, bits, err, zeroBuf, zeroWords);
    return cudaGetLastError();
}

cudaError_t bh_launch_local_minmax(const float4* pos, unsigned n, float3* minCorner, float3* maxCorner,
                                   int blocks, cudaStream_t s) {
    k_local_minmax<<<blocks, kBoxThreads, 0, s>>>(pos, n, minCorner, maxCorner);
    return cudaGetLastError();
}

cudaError_t bh_launch_global_minmax(const float3* minCorner, const float3* maxCorner, int count,
                                    float3* outMin, float3* outMax, cudaStream_t s) {
    k_global_minmax<<<1, kBoxThreads, 0, s>>>(minCorner, maxCorner, count, outMin, outMax);
    return cudaGetLastError();
}
