// compat.cu — the reference's level-at-a-time tree entry points and its
// prefix-sum object, for callers that drive the per-level build themselves
// (tree.h:26-32, 38-46; tree.cu:50-318).  buildTree() does not use them: it
// builds all levels in one pass (octree.cu).  Semantics follow the reference
// kernel by kernel; the exclusive scan is this library's own (reduce, scan of
// block sums, downsweep) instead of CUB's DeviceScan.
#include <stdio.h>
#include <stdlib.h>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"
#include "tree.h"

namespace {
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warpSums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warpSums[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t s = lane < nw ? warpSums[lane] : 0u;
        uint32_t t = s;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) warpSums[lane] = t - s;
        if (lane == nw - 1) *total = t;
    }
    __syncthreads();
    const uint32_t r = warpSums[w] + x - v;
    __syncthreads();
    return r;
}
}  // namespace

__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(const uint32_t* in, int n, uint32_t* blockSums) {
    __shared__ uint32_t total;
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) s += (base + k < n) ? in[base + k] : 0u;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(uint32_t* blockSums, int nblocks) {
    __shared__ uint32_t total;
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += kScanThreads) {
        const int b = b0 + threadIdx.x;
        const uint32_t v = b < nblocks ? blockSums[b] : 0u;
        const uint32_t e = block_exclusive_scan(v, &total);
        if (b < nblocks) blockSums[b] = carry + e;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kScanThreads)
k_scan_down(const uint32_t* in, uint32_t* out, int n, const uint32_t* blockOffsets) {
    __shared__ uint32_t total;
    const int base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t run = blockOffsets[blockIdx.x] + block_exclusive_scan(s, &total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

// tree.cu:50-78
__global__ void k_identify_nodes(const uint64_t* codes, int level, int n, uint32_t* flags) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t k = codes[i];
    const uint64_t cur = level_prefix(k, BH_MAX_BITS, level), par = level_prefix(k, BH_MAX_BITS, level - 1);
    const bool parentLeft = i > 0 && par == level_prefix(codes[i - 1], BH_MAX_BITS, level - 1);
    const bool parentRight = i < n - 1 && par == level_prefix(codes[i + 1], BH_MAX_BITS, level - 1);
    const bool sameLeft = i > 0 && cur == level_prefix(codes[i - 1], BH_MAX_BITS, level);
    flags[i] = (parentLeft || parentRight) && !sameLeft ? 1u : 0u;
}

// tree.cu:205-235
__global__ void k_create_nodes(const uint64_t* codes, const uint32_t* flags, const uint32_t* prevFlags,
                               const uint32_t* offsets, const uint32_t* prevOffsets, node* nodes, int level,
                               int levelOffset, int prevLevelOffset, int n, int maxNodes) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || flags[i] == 0u) return;
    const uint64_t path = level_prefix(codes[i], BH_MAX_BITS, level);
    const int idx = (int)offsets[i] + levelOffset;
    if (idx >= maxNodes) return;
    node* nd = &nodes[idx];
    nd->nodePathFromRoot = path;
    nd->treeLevel = level;
    nd->firstParticleIndex = i;
#pragma unroll
    for (int c = 0; c < 8; c++) nd->child[c] = -1;
    const int parent = (level == 1) ? 0 : prevLevelOffset + (int)prevOffsets[i] + (int)prevFlags[i] - 1;
    nodes[parent].child[path & 7] = idx;
    nd->parentIndex = parent;
}

// tree.cu:181-203
__global__ void k_update_particles(node* nodes, int levelStart, int levelCount) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= levelCount) return;
    const int k = levelStart + t;
    const int parent = nodes[k].parentIndex;
    const bool sibling = t + 1 < levelCount && nodes[k + 1].parentIndex == parent;
    const int end = sibling ? nodes[k + 1].firstParticleIndex
                            : nodes[parent].firstParticleIndex + nodes[parent].particleCount;
    nodes[k].particleCount = end - nodes[k].firstParticleIndex;
}

// tree.cu:89-179
__global__ void k_update_mass(node* nodes, const float4* pos, int levelCount, int levelStart) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= levelCount) return;
    node* nd = &nodes[levelStart + t];
    bool leaf = true;
#pragma unroll
    for (int c = 0; c < 8; c++) leaf = leaf && nd->child[c] == -1;
    float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
    if (leaf) {
        float wx = 0.f, wy = 0.f, wz = 0.f, m = 0.f;
        for (int k = 0; k < nd->particleCount; k++) {
            const float4 p = pos[nd->firstParticleIndex + k];
            wx = __fmaf_rn(p.x, p.w, wx);
            wy = __fmaf_rn(p.y, p.w, wy);
            wz = __fmaf_rn(p.z, p.w, wz);
            m = __fadd_rn(m, p.w);
        }
        if (m > 0.f) r = make_float4(__fdiv_rn(wx, m), __fdiv_rn(wy, m), __fdiv_rn(wz, m), m);
    } else {
        float m = 0.f, x = 0.f, y = 0.f, z = 0.f;
        for (int c = 0; c < 8; c++)
            if (nd->child[c] != -1) m = __fadd_rn(m, nodes[nd->child[c]].massData.w);
        for (int c = 0; c < 8; c++) {
            if (nd->child[c] == -1) continue;
            const float4 cm = nodes[nd->child[c]].massData;
            x = __fmaf_rn(cm.x, cm.w, x);
            y = __fmaf_rn(cm.y, cm.w, y);
            z = __fmaf_rn(cm.z, cm.w, z);
        }
        if (m > 0.f) r = make_float4(__fdiv_rn(x, m), __fdiv_rn(y, m), __fdiv_rn(z, m), m);
    }
    nd->massData = r;
}

// ------------------------------------------------------------------ C ABI
static int grid_for(int n) { return n <= 0 ? 1 : (n + 255) / 256; }

extern "C" void identifyNodesAtLevel(uint64_t* mortonCodes, int nodeLevel, int starCount, uint32_t* nodeFlags,
                                     cudaStream_t stream) {
    k_identify_nodes<<<grid_for(starCount), 256, 0, stream>>>(mortonCodes, nodeLevel, starCount, nodeFlags);
}

extern "C" void createNodes(const uint64_t* mortonCodes, const uint32_t* flags, const uint32_t* previousFlags,
                            const uint32_t* offsets, const uint32_t* offsetsPrev, node* nodes, int level,
                            int arrayLevelOffset, int prevArrayLevelOffset, int starCount, int maxNodes,
                            cudaStream_t stream) {
    k_create_nodes<<<grid_for(starCount), 256, 0, stream>>>(mortonCodes, flags, previousFlags, offsets, offsetsPrev,
                                                             nodes, level, arrayLevelOffset, prevArrayLevelOffset,
                                                             starCount, maxNodes);
}

extern "C" void updateTreeParticles(node* nodes, int levelStartIndex, int levelNodeCount, int starCount,
                                    cudaStream_t stream) {
    (void)starCount;
    k_update_particles<<<grid_for(levelNodeCount), 256, 0, stream>>>(nodes, levelStartIndex, levelNodeCount);
}

extern "C" void updateTreeMass(node* nodes, const float4* positionMassVals, int level, int levelNodes,
                               int levelStartIndex, cudaStream_t stream) {
    (void)level;
    k_update_mass<<<grid_for(levelNodes), 256, 0, stream>>>(nodes, positionMassVals, levelNodes, levelStartIndex);
}

static void scan_die(const char* msg) {
    printf("%s", msg);
    fflush(stdout);
    exit(-1);
}

extern "C" treeBuilder* sumCreate(int maxCount) {
    if (maxCount <= 0) scan_die("ERROR: Attempted to initialise a prefix sum over an array of <= 0 elements.\n");
    treeBuilder* b = (treeBuilder*)calloc(1, sizeof(treeBuilder));
    if (!b) scan_die("ERROR: Prefix sum could not be initialised.\n");
    const int blocks = (maxCount + kScanTile - 1) / kScanTile;
    b->tempStorageBytes = sizeof(uint32_t) * (size_t)blocks;
    const size_t bytes = sizeof(uint32_t) * (size_t)maxCount;
    if (cudaMalloc(&b->tempStorage, b->tempStorageBytes) != cudaSuccess ||
        cudaMalloc((void**)&b->flagsPing, bytes) != cudaSuccess || cudaMalloc((void**)&b->flagsPong, bytes) != cudaSuccess ||
        cudaMalloc((void**)&b->offsetsPing, bytes) != cudaSuccess ||
        cudaMalloc((void**)&b->offsetsPong, bytes) != cudaSuccess)
        scan_die("ERROR: Failed to malloc data for the exclusive sum");
    b->capacity = maxCount;
    return b;
}

extern "C" void prefixSum(treeBuilder* builder, uint32_t* flags, uint32_t* offsets, int maxCount) {
    if (!builder) scan_die("ERROR: treeBuilder struct passed to prefixSum() was uninitialised.\n");
    if (maxCount <= 0 || maxCount > builder->capacity)
        scan_die("ERROR: Length of array to sum conflicts with capacity of treeBuilder struct.\n");
    const int blocks = (maxCount + kScanTile - 1) / kScanTile;
    uint32_t* sums = (uint32_t*)builder->tempStorage;
    k_scan_reduce<<<blocks, kScanThreads>>>(flags, maxCount, sums);
    k_scan_blocks<<<1, kScanThreads>>>(sums, blocks);
    k_scan_down<<<blocks, kScanThreads>>>(flags, offsets, maxCount, sums);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        printf("ERROR: Error occured while performing prefix sum: %s\n", cudaGetErrorString(e));
        exit(-1);
    }
}

extern "C" void sumDestroyer(treeBuilder* sum) {
    if (!sum) scan_die("ERROR: Attempted to delete non-existant prefix sum object.\n");
    cudaFree(sum->flagsPing);
    cudaFree(sum->flagsPong);
    cudaFree(sum->offsetsPing);
    cudaFree(sum->offsetsPong);
    cudaFree(sum->tempStorage);
    free(sum);
}

// scratch for a prefix sum of up to maxCount elements (bytes)
size_t bh_scan_temp_bytes(int maxCount) { return sizeof(uint32_t) * (size_t)((maxCount + kScanTile - 1) / kScanTile); }
