// radix_sort.cu — stable LSD radix sort of (uint64 key, uint32 value) pairs
// for sm_100a.
//
// Replaces the reference's CUB DeviceRadixSort::SortPairs call
// (sorting.cu:15-92).  Same contract: stable, ascending, inputs untouched,
// results in separate buffers.  Design: "onesweep" (Adinets & Merrill 2022):
//   - one histogram read of the keys gives every digit's global counts
//     (fused into the Morton kernel when the sort follows it);
//   - one kernel per 8-bit digit: each CTA takes the next tile from an atomic
//     counter, ranks its keys stably with warp ballots, publishes its
//     per-digit counts, and computes the count of each digit in all earlier
//     tiles by decoupled look-back; it then scatters through shared memory so
//     that each digit's run is written contiguously;
//   - each pass after the first is a programmatic dependent launch of the one
//     before: its tiles are scheduled while the previous pass drains and wait
//     for it only before loading their keys.
// Look-back waits are bounded (BH_SPIN_LIMIT polls): a wait that gives up sets
// BH_ERR_TIMEOUT in the error word instead of hanging.
#include "bh_internal.cuh"
#include "bh_kernels.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
#ifndef BH_SORT_ITEMS
#define BH_SORT_ITEMS 16
#endif
constexpr int kItems = BH_SORT_ITEMS;       // keys per thread
constexpr int kTile = kThreads * kItems;    // 4096 keys per tile
constexpr uint32_t kFlagAgg = 1u << 30;     // tile count published
constexpr uint32_t kFlagPrefix = 2u << 30;  // inclusive prefix published
constexpr uint32_t kValueMask = (1u << 30) - 1u;
#ifndef BH_SORT_LOOKBACK
#define BH_SORT_LOOKBACK 8
#endif
constexpr int kLookback = BH_SORT_LOOKBACK;  // predecessor tiles read per look-back round trip

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.volatile.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_volatile(uint32_t* p, uint32_t v) {
    asm volatile("st.volatile.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Decoupled look-back for one digit: the count of that digit in tiles
// 0..tile-1, read from status (one word per tile and digit, stride 256).  A
// window of kLookback predecessors is loaded per round trip (independent
// loads), then consumed in tile order until a published prefix (done) or an
// unpublished tile (wait on it).  The wait is bounded: after BH_SPIN_LIMIT
// round trips without progress it sets BH_ERR_TIMEOUT and returns what it
// has, so a tile that never publishes cannot hang the sort.
__device__ __forceinline__ uint32_t lookback_exclusive(const uint32_t* status, int tile, int d, int* err) {
    uint32_t excl = 0;
    int j = tile - 1;
    unsigned spins = 0;
    while (j >= 0) {
        uint32_t v[kLookback];
#pragma unroll
        for (int k = 0; k < kLookback; k++)
            v[k] = (j - k >= 0) ? ld_volatile(status + (size_t)(j - k) * 256 + d) : kFlagPrefix;
        bool done = false;
        int k = 0;
#pragma unroll
        for (; k < kLookback; k++) {
            const uint32_t flag = v[k] & ~kValueMask;
            if (flag == 0u) break;
            excl += v[k] & kValueMask;
            if (flag == kFlagPrefix) {
                done = true;
                break;
            }
        }
        if (done) break;
        j -= k;  // k < kLookback: tile j - k has published nothing yet
        if (k < kLookback && ++spins > BH_SPIN_LIMIT) {
            bh_set_error(err, BH_ERR_TIMEOUT);
            break;
        }
    }
    return excl;
}

}  // namespace

// Upfront digit histogram for a standalone sort: counts digits 0..npass-1 of
// every key into hist[npass][256] (must be zero on entry).
__global__ void __launch_bounds__(kThreads)
k_sort_histogram(const uint64_t* __restrict__ keys, int n, uint32_t* __restrict__ hist, int npass) {
    __shared__ uint32_t sh[8][256];
    for (int i = threadIdx.x; i < npass * 256; i += blockDim.x) (&sh[0][0])[i] = 0u;
    __syncthreads();
    const int per = 8;
    for (int base = (blockIdx.x * blockDim.x + threadIdx.x) * per; base < n;
         base += gridDim.x * blockDim.x * per) {
        const int cnt = (n - base < per) ? n - base : per;
        for (int p = 0; p < npass; p++) {
            uint32_t run = 0, cur = 0;
            for (int j = 0; j < cnt; j++) {
                const uint32_t d = (uint32_t)(__ldg(&keys[base + j]) >> (8 * p)) & 255u;
                if (run && d != cur) { atomicAdd(&sh[p][cur], run); run = 0; }
                cur = d;
                run++;
            }
            if (run) atomicAdd(&sh[p][cur], run);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < npass * 256; i += blockDim.x) {
        const uint32_t c = (&sh[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// One digit pass.  hist: the 256 global counts of this digit.  status:
// [numTiles][256] words, zero on entry.  tileCounter: zero on entry.
// identityVals: the values are the input positions (valsIn is not read).
__global__ void __launch_bounds__(kThreads)
k_sort_pass(const uint64_t* __restrict__ keysIn, const uint32_t* __restrict__ valsIn,
            uint64_t* __restrict__ keysOut, uint32_t* __restrict__ valsOut, int n, int shift,
            const uint32_t* __restrict__ hist, uint32_t* status, int* tileCounter, int* err,
            int identityVals) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint64_t* skeys = reinterpret_cast<uint64_t*>(smem);                        // kTile
    uint32_t* svals = reinterpret_cast<uint32_t*>(skeys + kTile);               // kTile
    uint32_t* warpHist = svals + kTile;                                         // [kWarps][256]
    uint32_t* localStart = warpHist + kWarps * 256;                             // [256]
    uint32_t* globalStart = localStart + 256;                                   // [256]
    uint32_t* digitBase = globalStart + 256;                                    // [256]
    __shared__ int sTile;

    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    // programmatic dependent launch: the next pass may be scheduled once every
    // tile of this one runs, and its prologue (tile id, digit bases from the
    // upfront histograms) overlaps this pass's tail
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tid == 0) sTile = atomicAdd(tileCounter, 1);
    for (int i = tid; i < kWarps * 256; i += kThreads) warpHist[i] = 0u;
    // exclusive scan of the global digit counts -> digit bases
    {
        const uint32_t c = hist[tid];
        uint32_t x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) localStart[w] = x;  // warp totals (temporary use)
        __syncthreads();
        uint32_t off = 0;
        for (int k = 0; k < w; k++) off += localStart[k];
        digitBase[tid] = off + x - c;
    }
    __syncthreads();
    const int tile = sTile;
    const int tileBase = tile * kTile;
    // the keys are the previous pass's output: wait for that grid to complete
    // (returns at once for a launch without a programmatic dependency)
    asm volatile("griddepcontrol.wait;" ::: "memory");

    // load: warp w owns keys [tileBase + w*32*kItems, +32*kItems), item k of
    // lane l at offset k*32 + l (coalesced, and in input order k-major).
    uint64_t key[kItems];
    uint32_t val[kItems];
    uint32_t rank[kItems];
    const int warpBase = tileBase + w * 32 * kItems;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const int i = warpBase + k * 32 + lane;
        if (i < n) {
            key[k] = keysIn[i];
            val[k] = identityVals ? (uint32_t)i : valsIn[i];
        } else {
            key[k] = ~0ull;
            val[k] = 0u;
        }
    }
    // stable ranks within the warp: items in order, peers by digit
    uint32_t* myHist = warpHist + w * 256;
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const int i = warpBase + k * 32 + lane;
        const uint32_t valid = __ballot_sync(0xffffffffu, i < n);
        const uint32_t d = (uint32_t)(key[k] >> shift) & 255u;
        // lanes with the same digit: AND over the 8 digit bits of the ballot
        // (or its complement) of that bit — 8 ballots, which measured 12-14%
        // faster per sort than one __match_any_sync
        uint32_t peers = valid;
#pragma unroll
        for (int bit = 0; bit < 8; bit++) {
            const uint32_t m = __ballot_sync(0xffffffffu, (d >> bit) & 1u);
            peers &= ((d >> bit) & 1u) ? m : ~m;
        }
        uint32_t before = 0;
        if (i < n) before = myHist[d];
        __syncwarp();
        if (i < n) {
            rank[k] = before + __popc(peers & lanemask_lt());
            if (lane == __ffs(peers) - 1) myHist[d] = before + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // per digit: exclusive over warps, tile total
    uint32_t tileCount;
    {
        const int d = tid;
        uint32_t s = 0;
#pragma unroll
        for (int k = 0; k < kWarps; k++) {
            const uint32_t c = warpHist[k * 256 + d];
            warpHist[k * 256 + d] = s;
            s += c;
        }
        tileCount = s;
        // publish, then look back over earlier tiles
        uint32_t* myStatus = status + (size_t)tile * 256 + d;
        if (tile == 0) {
            st_volatile(myStatus, kFlagPrefix | s);
            globalStart[d] = digitBase[d];
        } else {
            st_volatile(myStatus, kFlagAgg | s);
            const uint32_t excl = lookback_exclusive(status, tile, d, err);
            st_volatile(myStatus, kFlagPrefix | ((excl + s) & kValueMask));
            globalStart[d] = digitBase[d] + excl;
        }
    }
    // tile-local start of each digit (exclusive scan of tileCount over digits)
    {
        uint32_t x = tileCount;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        __shared__ uint32_t wsum[kWarps];
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        uint32_t off = 0;
        for (int k = 0; k < w; k++) off += wsum[k];
        localStart[tid] = off + x - tileCount;
    }
    __syncthreads();
    // scatter into shared memory in sorted-within-tile order
#pragma unroll
    for (int k = 0; k < kItems; k++) {
        const int i = warpBase + k * 32 + lane;
        if (i < n) {
            const uint32_t d = (uint32_t)(key[k] >> shift) & 255u;
            const uint32_t p = localStart[d] + warpHist[w * 256 + d] + rank[k];
            skeys[p] = key[k];
            svals[p] = val[k];
        }
    }
    __syncthreads();
    // write out: consecutive positions of a digit go to consecutive addresses
    const int tileValid = (n - tileBase < kTile) ? n - tileBase : kTile;
    for (int j = tid; j < tileValid; j += kThreads) {
        const uint64_t k = skeys[j];
        const uint32_t d = (uint32_t)(k >> shift) & 255u;
        const uint32_t dst = globalStart[d] + (uint32_t)j - localStart[d];
        keysOut[dst] = k;
        valsOut[dst] = svals[j];
    }
}

// ---------------------------------------------------------------- launchers
namespace {
size_t pass_smem() { return (size_t)kTile * (8 + 4) + (size_t)(kWarps * 256 + 3 * 256) * 4; }
}  // namespace

int bh_sort_tile() { return kTile; }

cudaError_t bh_sort_init() {
    return cudaFuncSetAttribute(k_sort_pass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem());
}

cudaError_t bh_launch_sort_histogram(const uint64_t* keys, int n, uint32_t* hist, int npass, cudaStream_t s) {
    int grid = (n + kThreads * 8 - 1) / (kThreads * 8);
    const int cap = 4 * bh_sm_count();
    grid = grid < 1 ? 1 : (grid > cap ? cap : grid);
    k_sort_histogram<<<grid, kThreads, 0, s>>>(keys, n, hist, npass);
    return cudaGetLastError();
}

cudaError_t bh_launch_sort_pass(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut,
                                uint32_t* valsOut, int n, int shift, const uint32_t* hist,
                                uint32_t* status, int* tileCounter, int* err, int identityVals,
                                cudaStream_t s) {
    const int tiles = (n + kTile - 1) / kTile;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tiles);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = pass_smem();
    cfg.stream = s;
    // passes after the first depend programmatically on their predecessor
    // (the first one follows the kernel that made its keys and histograms,
    // which its prologue reads)
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = shift > 0 ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k_sort_pass, keysIn, valsIn, keysOut, valsOut, n, shift, hist, status,
                              tileCounter, err, identityVals);
}

// Self-test of the bounded look-back wait: tile 1 looks back at a tile 0
// that never publishes; the wait gives up after BH_SPIN_LIMIT round trips,
// records BH_ERR_TIMEOUT and the kernel returns.
__global__ void k_lookback_selftest(const uint32_t* status, int* err) {
    if (threadIdx.x == 0) (void)lookback_exclusive(status, 1, 0, err);
}

cudaError_t bh_launch_lookback_selftest(const uint32_t* status, int* err, cudaStream_t s) {
    k_lookback_selftest<<<1, 32, 0, s>>>(status, err);
    return cudaGetLastError();
}

extern "C" int bh_selftest_bounded_wait(cudaStream_t s) {
    uint32_t* buf = nullptr;  // status words of two tiles (tile 0 left unpublished), then the error word
    const size_t words = 2 * 256 + 1;
    cudaError_t e = cudaMallocAsync(&buf, words * sizeof(uint32_t), s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    int* err = reinterpret_cast<int*>(buf + 2 * 256);
    e = cudaMemsetAsync(buf, 0, words * sizeof(uint32_t), s);
    if (e == cudaSuccess) {
        k_lookback_selftest<<<1, 32, 0, s>>>(buf, err);
        e = cudaGetLastError();
    }
    int h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaError_t f = cudaFreeAsync(buf, s);
    if (e == cudaSuccess) e = f;
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    return (h & BH_ERRBIT(BH_ERR_TIMEOUT)) ? BH_ERR_TIMEOUT : BH_OK;
}
