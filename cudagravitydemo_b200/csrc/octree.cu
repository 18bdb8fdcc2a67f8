// octree.cu — level-wise octree over Morton-sorted bodies, built for every
// level at once, plus the upward mass / centre-of-mass pass (sm_100a).
//
// The tree is the reference's (basicGravity.cu:232-319, tree.cu:50-235):
//   - a level-L node exists for each level-L cell whose parent cell holds at
//     least two bodies (identifyNodesAtLevel, tree.cu:50-78); chains of
//     single-child nodes are kept; cells at level `bits` may hold several
//     bodies with identical keys;
//   - nodes are stored level by level, each level in Morton order, so node
//     (L, first body i) has index levelOffset[L] + (number of level-L nodes
//     whose first body precedes i)  — the reference's exclusive scan.
// The reference discovers one level per host iteration (flags, scan, create,
// count: up to 21 host-synchronised rounds).  Here the levels at which body i
// starts a node form one contiguous range: with a = common levels of keys
// i-1 and i, b = common levels of keys i and i+1, body i starts nodes at
// levels a+1 .. min(max(a, b) + 1, bits).  So:
//   k_tree_count  one pass: a per body, per-block node counts per level
//   k_tree_scan   one block per level: per-level block offsets; the last
//                 block to finish writes the level table and sizes
//   k_tree_nodes  one pass: every node record, parent and child range
//   k_tree_mass   centre of mass level by level from the deepest, one
//                 cooperative launch with a grid barrier between levels
// Children of a node are contiguous in the next level, so a node stores the
// range [childBegin, childEnd) instead of child[8]; k_tree_export writes the
// reference's 80-byte records (child[slot]) when asked.
#include "bh_internal.cuh"
#include "bh_kernels.cuh"

namespace {
constexpr int kTreeThreads = 512;
constexpr int kTreeWarps = kTreeThreads / 32;
#ifndef BH_TREE_MASS_THREADS
#define BH_TREE_MASS_THREADS 256
#endif
#ifndef BH_TREE_MASS_BLOCKS_PER_SM
#define BH_TREE_MASS_BLOCKS_PER_SM 4
#endif
#ifndef BH_TREE_BARRIER_SLEEP_NS
#define BH_TREE_BARRIER_SLEEP_NS 64
#endif
// upward pass: threads per block, resident blocks per SM used, barrier poll pause
constexpr int kMassThreads = BH_TREE_MASS_THREADS;
constexpr int kMassBlocksPerSm = BH_TREE_MASS_BLOCKS_PER_SM;

// Number of levels below the root (0..bits) that two keys share; -1 when
// they belong to different systems of a batch (keys differ above the 3*bits
// Morton bits, where a batch keeps the system index).
__device__ __forceinline__ int common_levels(uint64_t a, uint64_t b, int bits) {
    const uint64_t x = a ^ b;
    if (x == 0ull) return bits;
    const int h = 63 - __clzll((long long)x);  // highest differing bit
    if (h >= 3 * bits) return -1;
    return bits - 1 - h / 3;
}

// delta[] stores common_levels with the left neighbour, 0xff for -1.
__device__ __forceinline__ int delta_levels(const uint8_t* delta, int i) {
    const int d = delta[i];
    return d == 0xff ? -1 : d;
}
}  // namespace

// Pass 1: delta[i] = common levels of keys i-1 and i (0xff for i = 0 and at
// the first body of every system of a batch) and, per block, how many nodes
// start at each level (blockLevel[L][block]); a root (level 0) starts at
// every body with no common level with its left neighbour.
__global__ void __launch_bounds__(kTreeThreads)
k_tree_count(const uint64_t* __restrict__ keys, int n, int bits, uint8_t* __restrict__ delta,
             int* __restrict__ blockLevel) {
    __shared__ int cnt[BH_LEVEL_SLOTS];
    const int tid = threadIdx.x, lane = tid & 31;
    if (tid < BH_LEVEL_SLOTS) cnt[tid] = 0;
    __syncthreads();
    const int i = blockIdx.x * kTreeThreads + tid;
    int lo = 1, hi = 0;
    bool root = false;
    if (i < n) {
        const uint64_t k = keys[i];
        const int a = (i > 0) ? common_levels(keys[i - 1], k, bits) : -1;
        const int b = (i + 1 < n) ? common_levels(k, keys[i + 1], bits) : -1;
        delta[i] = (uint8_t)(a < 0 ? 0xff : a);
        root = a < 0;
        lo = a + 1 < 1 ? 1 : a + 1;
        hi = (a > b ? a : b) + 1;
        hi = hi > bits ? bits : hi;
    }
    {
        const unsigned m = __ballot_sync(0xffffffffu, root);
        if (lane == 0 && m) atomicAdd(&cnt[0], __popc(m));
    }
    // only the levels where some body of the warp starts a node
    const int wlo = __reduce_min_sync(0xffffffffu, lo <= hi ? lo : bits + 1);
    const int whi = __reduce_max_sync(0xffffffffu, lo <= hi ? hi : 0);
    for (int L = wlo; L <= whi; L++) {
        const unsigned m = __ballot_sync(0xffffffffu, L >= lo && L <= hi);
        if (lane == 0 && m) atomicAdd(&cnt[L], __popc(m));
    }
    __syncthreads();
    if (tid < BH_LEVEL_SLOTS) blockLevel[tid * gridDim.x + blockIdx.x] = cnt[tid];
}

// Pass 2 (one block per level): blockLevel[L][b] (level-major) -> exclusive
// offset of block b within level L; then, in the last block to finish, the
// level table, per-level node size^2, the overflow check and the sentinel of
// the child ranges.
__global__ void __launch_bounds__(1024)
k_tree_scan(int* __restrict__ blockLevel, int nblocks, int n, int bits, int maxNodes,
            const DevBox* __restrict__ box, DevTreeInfo* info, int2* nCB, int* levelTotal, unsigned* ticket,
            int* err) {
    // block L scans level L's block counts (contiguous, level-major) in
    // chunks of 8192: each thread 8 consecutive counts, a block-wide scan of
    // the thread sums, a running carry between chunks
    __shared__ int warpSum[32];
    __shared__ bool last;
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int L = blockIdx.x;
    int* row = blockLevel + (size_t)L * nblocks;
    int carry = 0;
    for (int b0 = 0; b0 < nblocks; b0 += 8 * 1024) {
        int v[8];
        int sum = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int b = b0 + tid * 8 + k;
            v[k] = (b < nblocks) ? row[b] : 0;
            sum += v[k];
        }
        int x = sum;  // inclusive scan within the warp
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSum[w] = x;
        __syncthreads();
        if (w == 0) {  // scan of the 32 warp sums
            int y = warpSum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int z = __shfl_up_sync(0xffffffffu, y, o);
                if (lane >= o) y += z;
            }
            warpSum[lane] = y;  // inclusive
        }
        __syncthreads();
        int e = carry + (w > 0 ? warpSum[w - 1] : 0) + x - sum;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const int b = b0 + tid * 8 + k;
            if (b < nblocks) row[b] = e;
            e += v[k];
        }
        carry += warpSum[31];
        __syncthreads();  // warpSum is reused by the next chunk
    }
    // the last level block to finish builds the level table
    if (tid == 0) {
        levelTotal[L] = carry;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || tid != 0) return;
    __threadfence();
    DevTreeInfo t;
    int off = 0, deepest = 0, overflow = 0;
    for (int k = 0; k < BH_LEVEL_SLOTS; k++) {
        const int c = (k <= bits) ? __ldcg(&levelTotal[k]) : 0;
        t.levelOffset[k] = off;
        t.levelCount[k] = c;
        if (c > 0) deepest = k;
        if (!overflow && c > 0 && off + c > maxNodes) overflow = k;
        off += c;
    }
    t.deepest = deepest;
    t.nodeCount = off;
    t.overflowLevel = overflow;
    t.pad = 0;
    const float extX = box->extX;  // the first system's (the only one outside a batch)
    for (int k = 0; k < BH_LEVEL_SLOTS; k++) {
        const float sz = ldexpf(extX, -k);  // exact: extX / 2^k
        t.sizeSq[k] = __fmul_rn(sz, sz);
    }
    *info = t;
    if (overflow) bh_set_error(err, BH_ERR_TREE_OVERFLOW);
    else nCB[off].x = off;  // sentinel: end of the last child range
    *ticket = 0u;           // re-armed for the next build
}

// Pass 3: node records.  For body i with node range [lo, hi] and level-L
// exclusive rank r_L(i) (nodes at level L starting before i):
//   index(L, i)      = levelOffset[L] + r_L(i)
//   parent(L, i)     = levelOffset[L-1] + r_{L-1}(i) + f_{L-1}(i) - 1
//                      (the last level-(L-1) node starting at or before i,
//                       the reference's parent formula, tree.cu:224-231)
//   childBegin(L, i) = levelOffset[L+1] + r_{L+1}(i)
// A root (level 0) starts at body 0 and, in a batch, at the first body of
// every system; node sizes come from the box of the node's system (the key's
// bits above 3*bits), (extX / 2^L)^2.
__global__ void __launch_bounds__(kTreeThreads)
k_tree_nodes(const uint64_t* __restrict__ keys, const uint8_t* __restrict__ delta, int n, int bits,
             const int* __restrict__ blockLevel, const DevTreeInfo* __restrict__ info, int maxNodes,
             const DevBox* __restrict__ boxes, int2* __restrict__ nCB, int* __restrict__ nParent,
             int* __restrict__ nFirst, int* __restrict__ nMeta) {
    __shared__ int warpCnt[kTreeWarps][BH_LEVEL_SLOTS];
    __shared__ int levelOff[BH_LEVEL_SLOTS];
    __shared__ int blockOff[BH_LEVEL_SLOTS];
    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    const int nodeCount = info->nodeCount;
    if (info->overflowLevel) return;
    if (tid < BH_LEVEL_SLOTS) {
        levelOff[tid] = info->levelOffset[tid];
        blockOff[tid] = blockLevel[tid * gridDim.x + blockIdx.x];
    }
    const int i = blockIdx.x * kTreeThreads + tid;
    const bool valid = i < n;
    int lo = 1, hi = 0;  // node levels of body i (empty range when lo > hi)
    bool root = false;   // body i starts a root
    uint64_t key = 0;
    float extX = 0.f;
    if (valid) {
        key = keys[i];
        const int a = (i > 0) ? delta_levels(delta, i) : -1;
        const int b = (i + 1 < n) ? delta_levels(delta, i + 1) : -1;
        root = a < 0;
        lo = a + 1 < 1 ? 1 : a + 1;
        hi = (a > b ? a : b) + 1;
        hi = hi > bits ? bits : hi;
        const int shift = 3 * bits;
        extX = boxes[shift >= 64 ? 0 : (int)(key >> shift)].extX;
    }
    // flag of level L for this body (level 0: a root)
    auto flag = [&](int L) -> bool { return valid && (L == 0 ? root : (L >= lo && L <= hi)); };
    // the levels where some body of the warp starts a node: [wlo, whi]
    // (empty when wlo > whi); every other level has no flag in this warp
    const bool anyRoot = __any_sync(0xffffffffu, valid && root);
    int wlo = __reduce_min_sync(0xffffffffu, valid && lo <= hi ? lo : bits + 1);
    const int whi = __reduce_max_sync(0xffffffffu, valid && lo <= hi ? hi : 0);
    if (anyRoot) wlo = 0;
    // warp totals per level
    if (lane <= bits + 1) warpCnt[w][lane] = 0;
    __syncwarp();
    for (int L = wlo; L <= whi; L++) {
        const unsigned m = __ballot_sync(0xffffffffu, flag(L));
        if (lane == 0) warpCnt[w][L] = __popc(m);
    }
    __syncthreads();
    if (tid <= bits + 1) {  // exclusive scan over warps, per level
        int s = 0;
        for (int k = 0; k < kTreeWarps; k++) {
            const int c = warpCnt[k][tid];
            warpCnt[k][tid] = s;
            s += c;
        }
    }
    __syncthreads();
    // walk the levels keeping r_{L-2}, r_{L-1}, r_L; node L-1 is complete at
    // L.  Below wlo no body of the warp has a flag, so its ranks there are the
    // warp's offsets alone; the walk starts at wlo and ends at whi + 1 (the
    // child ranges of the level-whi nodes).
    if (wlo > whi) return;  // uniform: this warp starts no node
    int r2 = 0, r1 = 0, f2 = 0, f1 = 0;
    if (wlo >= 2) r2 = blockOff[wlo - 2] + warpCnt[w][wlo - 2];
    if (wlo >= 1) r1 = blockOff[wlo - 1] + warpCnt[w][wlo - 1];
    const unsigned lt = lanemask_lt();
    for (int L = wlo; L <= whi + 1; L++) {
        const bool f = flag(L);
        const unsigned m = (L <= whi) ? __ballot_sync(0xffffffffu, f) : 0u;
        const int r = blockOff[L] + warpCnt[w][L] + __popc(m & lt);
        const int Ln = L - 1;  // node level completed in this iteration
        if (Ln >= 0 && f1) {
            const int idx = levelOff[Ln] + r1;
            const int parent = (Ln == 0) ? -1 : levelOff[Ln - 1] + r2 + f2 - 1;
            const int childBegin = levelOff[L] + r;
            if (idx < maxNodes && idx < nodeCount) {
                const float sz = ldexpf(extX, -Ln);  // exact: extX / 2^L
                nCB[idx] = make_int2(childBegin, __float_as_int(__fmul_rn(sz, sz)));
                nParent[idx] = parent;
                nFirst[idx] = i;
                nMeta[idx] = Ln | ((int)(level_prefix(key, bits, Ln) & 7ull) << 8);
            }
        }
        r2 = r1; f2 = f1;
        r1 = r; f1 = f;
    }
}

// Pass 4: upward pass, level by level from the deepest, in one cooperative
// launch (every block resident; a grid barrier separates levels).  A node
// whose child range is empty is a leaf: its centre of mass comes from its
// bodies (tree.cu:105-135: sum of x*w fused, then divide) — one body, or a
// run of identical keys at the deepest possible level, or every body when the
// root is the only node.  An internal node sums its children in slot order
// (tree.cu:139-176: mass first, then x*w, then divide).  Zero-mass nodes get
// (0,0,0,0), like the reference.  Barrier waits are bounded: a wait that
// gives up records BH_ERR_TIMEOUT and the kernel runs to its end.
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void grid_barrier(unsigned* bar, unsigned target, int* err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
        atomicAdd(bar, 1u);
        unsigned spins = 0;
        while (ld_acquire_u32(bar) < target) {
            if (++spins > BH_SPIN_LIMIT) {
                bh_set_error(err, BH_ERR_TIMEOUT);
                break;
            }
            if (BH_TREE_BARRIER_SLEEP_NS > 0) __nanosleep(BH_TREE_BARRIER_SLEEP_NS);
        }
    }
    __syncthreads();
}


__global__ void __launch_bounds__(kMassThreads)
k_tree_mass(const float4* __restrict__ pos, const uint8_t* __restrict__ delta, int n, int bits,
            const DevTreeInfo* __restrict__ info, const int2* __restrict__ nCB, float4* nCom, WalkNode* __restrict__ wn,
            const int* __restrict__ nFirst, int* nCount, unsigned* bar, int* err) {
    if (info->overflowLevel) return;  // uniform: every block returns
    const int nodeCount = info->nodeCount;
    const int deepest = info->deepest;
    // A level with at most blockDim.x nodes (the few deepest and the top
    // ones) is done by block 0 alone, one node per thread; two such levels in
    // a row need only block 0's __syncthreads between them, not a grid barrier.
    auto small = [&](int L) { return info->levelCount[L] <= (int)blockDim.x; };
    unsigned target = 0;
    for (int L = deepest; L >= 0; L--) {
        const int begin = info->levelOffset[L], end = begin + info->levelCount[L];
        const bool alone = small(L);  // uniform; the other blocks skip the level
        const int first = alone ? (blockIdx.x == 0 ? begin + (int)threadIdx.x : end)
                                : begin + blockIdx.x * blockDim.x + threadIdx.x;
        const int stride = alone ? (int)blockDim.x : gridDim.x * blockDim.x;
        for (int k = first; k < end; k += stride) {
            const int2 me = nCB[k];
            const int cb = me.x;
            const int ce = nCB[k + 1].x;
            float4 com = make_float4(0.f, 0.f, 0.f, 0.f);
            int count;
            if (cb == ce) {  // leaf
                const int first = (k == 0) ? 0 : nFirst[k];
                if (nodeCount == 1) {
                    count = n;
                } else if (L == bits) {
                    int j = first + 1;
                    while (j < n && (int)delta[j] == bits) j++;
                    count = j - first;
                } else {
                    count = 1;
                }
                float wx = 0.f, wy = 0.f, wz = 0.f, m = 0.f;
                for (int t = 0; t < count; t++) {
                    const float4 p = pos[first + t];
                    wx = __fmaf_rn(p.x, p.w, wx);
                    wy = __fmaf_rn(p.y, p.w, wy);
                    wz = __fmaf_rn(p.z, p.w, wz);
                    m = __fadd_rn(m, p.w);
                }
                if (m > 0.0f) com = make_float4(__fdiv_rn(wx, m), __fdiv_rn(wy, m), __fdiv_rn(wz, m), m);
            } else {
                const int nch = ce - cb;
                if (nch > 8 || cb <= k) {  // broken links: report, do not follow
                    bh_set_error(err, BH_ERR_INTERNAL);
                    continue;
                }
                float4 cm[8];
                int cc[8];
#pragma unroll
                for (int t = 0; t < 8; t++) {  // all children in one round trip
                    if (t < nch) {
                        cm[t] = __ldcg(&nCom[cb + t]);
                        cc[t] = __ldcg(&nCount[cb + t]);
                    }
                }
                float m = 0.f, x = 0.f, y = 0.f, z = 0.f;
                count = 0;
#pragma unroll
                for (int t = 0; t < 8; t++)
                    if (t < nch) {
                        m = __fadd_rn(m, cm[t].w);
                        count += cc[t];
                    }
#pragma unroll
                for (int t = 0; t < 8; t++)
                    if (t < nch) {
                        x = __fmaf_rn(cm[t].x, cm[t].w, x);
                        y = __fmaf_rn(cm[t].y, cm[t].w, y);
                        z = __fmaf_rn(cm[t].z, cm[t].w, z);
                    }
                if (m > 0.0f) com = make_float4(__fdiv_rn(x, m), __fdiv_rn(y, m), __fdiv_rn(z, m), m);
            }
            // the walk's record in one 32-byte store pair; the compact copies
            // serve the parent level
            float4* rec = reinterpret_cast<float4*>(&wn[k]);
            rec[0] = com;
            rec[1] = make_float4(__int_as_float(cb), __int_as_float(ce), __int_as_float(me.y), __int_as_float(count));
            nCom[k] = com;
            nCount[k] = count;
        }
        if (L > 0) {
            if (alone && small(L - 1)) {
                __syncthreads();  // block 0 only has work on both levels
            } else {
                target += gridDim.x;
                grid_barrier(bar, target, err);
            }
        }
    }
}

// Reference layout (types.h:52-62): one thread per node writes the 80-byte
// record, child[slot] from the contiguous child range.
__global__ void __launch_bounds__(256)
k_tree_export(const uint64_t* __restrict__ keys, int bits, const DevTreeInfo* __restrict__ info,
              const WalkNode* __restrict__ wn, const int* __restrict__ nParent,
              const int* __restrict__ nFirst, const int* __restrict__ nCount,
              const int* __restrict__ nMeta, node* __restrict__ out, int n) {
    if (info->overflowLevel) return;
    const int nodeCount = info->nodeCount;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nodeCount; k += gridDim.x * blockDim.x) {
        const WalkNode w = wn[k];
        node r;
        const int first = (k == 0) ? 0 : nFirst[k];
        const int level = (k == 0) ? 0 : (nMeta[k] & 0xff);
        r.nodePathFromRoot = (k == 0) ? 0ull : level_prefix(keys[first], bits, level);
        r.parentIndex = (k == 0) ? -1 : nParent[k];
        r.firstParticleIndex = first;
        r.particleCount = (k == 0) ? n : nCount[k];
#pragma unroll
        for (int s = 0; s < 8; s++) r.child[s] = -1;
        const int ce = w.childEnd < w.childBegin + 8 ? w.childEnd : w.childBegin + 8;
        for (int c = w.childBegin; c < ce; c++) r.child[(nMeta[c] >> 8) & 7] = c;
        r.treeLevel = level;
        r.massData = w.com;
        out[k] = r;
    }
}

// Gather bodies into sorted order (sorting.cu:99-107), carrying body ids.
__global__ void __launch_bounds__(256)
k_reorder(const float4* __restrict__ posIn, const float3* __restrict__ velIn,
          const uint32_t* __restrict__ idIn, const uint32_t* __restrict__ perm,
          float4* __restrict__ posOut, float3* __restrict__ velOut, uint32_t* __restrict__ idOut,
          const float* __restrict__ auxIn, float* __restrict__ auxOut, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = perm[i];
        if (posOut) posOut[i] = __ldg(&posIn[s]);
        if (velOut) velOut[i] = velIn[s];
        if (idOut) idOut[i] = idIn ? idIn[s] : s;
        if (auxOut) auxOut[i] = auxIn[s];
    }
}

// Scatter state from simulation order back to body-id order.
__global__ void __launch_bounds__(256)
k_scatter_by_id(const float4* __restrict__ pos, const float3* __restrict__ vel,
                const float3* __restrict__ acc, const uint32_t* __restrict__ ids,
                float4* __restrict__ posOut, float3* __restrict__ velOut,
                float3* __restrict__ accOut, const float* __restrict__ aux, float* __restrict__ auxOut, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t d = ids[i];
        if (d >= (uint32_t)n) continue;  // ids a caller supplied may be out of range: never written through
        if (posOut) posOut[d] = pos[i];
        if (velOut) velOut[d] = vel[i];
        if (accOut) accOut[d] = acc[i];
        if (auxOut) auxOut[d] = aux[i];
    }
}

// out[i] = in[ids[i]]: a per-body value kept by body id, brought into the
// order of ids.  The ids are a caller's: one outside [0, n) reads nothing,
// gets +inf and sets BH_ERR_INVALID in the error word.  in/out NULL: the ids
// are only checked.
__global__ void __launch_bounds__(256)
k_gather_by_id(const float* __restrict__ in, const uint32_t* __restrict__ ids, float* __restrict__ out, int n,
               int* err) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t d = ids[i];
        const bool ok = d < (uint32_t)n;
        if (!ok) bh_set_error(err, BH_ERR_INVALID);
        if (out) out[i] = ok ? in[d] : INFINITY;
    }
}

// Holds its stream for about ns nanoseconds of the global timer, so that the
// host has queued the launches behind it before they start (events between
// those launches then time the device, not the host's launch rate).  Bounded
// by time and by an iteration count.
__global__ void k_hold(unsigned long long ns) {
    unsigned long long t0, t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (int i = 0; i < 200000; i++) {
        __nanosleep(1000);
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        if (t - t0 >= ns) break;
    }
}

__global__ void k_iota(uint32_t* ids, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) ids[i] = (uint32_t)i;
}

// ---------------------------------------------------------------- launchers
namespace {
int stream_grid(int n, int threads) {
    int g = (n + threads - 1) / threads;
    const int cap = 8 * bh_sm_count();
    return g < 1 ? 1 : (g > cap ? cap : g);
}
}  // namespace

int bh_tree_threads() { return kTreeThreads; }

cudaError_t bh_launch_tree_count(const uint64_t* keys, int n, int bits, uint8_t* delta, int* blockLevel,
                                 cudaStream_t s) {
    const int blocks = (n + kTreeThreads - 1) / kTreeThreads;
    k_tree_count<<<blocks, kTreeThreads, 0, s>>>(keys, n, bits, delta, blockLevel);
    return cudaGetLastError();
}

cudaError_t bh_launch_tree_scan(int* blockLevel, int nblocks, int n, int bits, int maxNodes,
                                const DevBox* box, DevTreeInfo* info, int2* nCB, int* levelTotal, unsigned* ticket,
                                int* err, cudaStream_t s) {
    k_tree_scan<<<bits + 1, 1024, 0, s>>>(blockLevel, nblocks, n, bits, maxNodes, box, info, nCB, levelTotal, ticket,
                                          err);
    return cudaGetLastError();
}

cudaError_t bh_launch_tree_nodes(const uint64_t* keys, const uint8_t* delta, int n, int bits,
                                 const int* blockLevel, const DevTreeInfo* info, int maxNodes, const DevBox* boxes,
                                 int2* nCB, int* nParent, int* nFirst, int* nMeta, cudaStream_t s) {
    const int blocks = (n + kTreeThreads - 1) / kTreeThreads;
    k_tree_nodes<<<blocks, kTreeThreads, 0, s>>>(keys, delta, n, bits, blockLevel, info, maxNodes, boxes, nCB,
                                                  nParent, nFirst, nMeta);
    return cudaGetLastError();
}

// Blocks of the cooperative upward pass: every block must be resident.
int bh_tree_mass_grid() {
    static int grid = 0;
    if (!grid) {
        int per = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tree_mass, kMassThreads, 0) != cudaSuccess || per < 1)
            per = 1;
        per = per > kMassBlocksPerSm ? kMassBlocksPerSm : per;
        grid = per * bh_sm_count();
    }
    return grid;
}

cudaError_t bh_launch_tree_mass(const float4* pos, const uint8_t* delta, int n, int bits, const DevTreeInfo* info,
                                const int2* nCB, float4* nCom, WalkNode* wn, const int* nFirst, int* nCount,
                                unsigned* bar, int* err, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(bar, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(bh_tree_mass_grid());
    cfg.blockDim = dim3(kMassThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_tree_mass, pos, delta, n, bits, info, nCB, nCom, wn, nFirst, nCount, bar, err);
}

cudaError_t bh_launch_tree_export(const uint64_t* keys, int bits, const DevTreeInfo* info,
                                  const WalkNode* wn, const int* nParent, const int* nFirst,
                                  const int* nCount, const int* nMeta, node* out, int n, int maxNodes,
                                  cudaStream_t s) {
    k_tree_export<<<stream_grid(maxNodes, 256), 256, 0, s>>>(keys, bits, info, wn, nParent, nFirst, nCount, nMeta,
                                                               out, n);
    return cudaGetLastError();
}

cudaError_t bh_launch_reorder(const float4* posIn, const float3* velIn, const uint32_t* idIn,
                              const uint32_t* perm, float4* posOut, float3* velOut, uint32_t* idOut,
                              int n, cudaStream_t s, const float* auxIn, float* auxOut) {
    k_reorder<<<stream_grid(n, 256), 256, 0, s>>>(posIn, velIn, idIn, perm, posOut, velOut, idOut, auxIn, auxOut,
                                                   n);
    return cudaGetLastError();
}

cudaError_t bh_launch_scatter_by_id(const float4* pos, const float3* vel, const float3* acc,
                                    const uint32_t* ids, float4* posOut, float3* velOut,
                                    float3* accOut, int n, cudaStream_t s, const float* aux, float* auxOut) {
    k_scatter_by_id<<<stream_grid(n, 256), 256, 0, s>>>(pos, vel, acc, ids, posOut, velOut, accOut, aux, auxOut, n);
    return cudaGetLastError();
}

cudaError_t bh_launch_gather_by_id(const float* in, const uint32_t* ids, float* out, int n, int* err,
                                   cudaStream_t s) {
    k_gather_by_id<<<stream_grid(n, 256), 256, 0, s>>>(in, ids, out, n, err);
    return cudaGetLastError();
}

cudaError_t bh_launch_hold(unsigned long long ns, cudaStream_t s) {
    k_hold<<<1, 32, 0, s>>>(ns);
    return cudaGetLastError();
}

cudaError_t bh_launch_iota(uint32_t* ids, int n, cudaStream_t s) {
    k_iota<<<stream_grid(n, 256), 256, 0, s>>>(ids, n);
    return cudaGetLastError();
}
