/*
 * dropin.c — the reference's host code, written against this library's
 * drop-in headers only (main.h: types.h, tree.h, sorting.h) and compiled by
 * gcc as plain C.  Test program: tests/test_gpu_dropin.py builds and runs it.
 *
 *   dropin levels <in.bin> <out.bin>
 *       The reference's buildTree (basicGravity.cu:116-325) step by step
 *       through the reference-named entry points: localMinMaxFinder +
 *       globalMinMaxReducer and createWorldBox, mortonEncode, sorterCreate +
 *       radixSortPairs, reorderParticles, then per level identifyNodesAtLevel,
 *       prefixSum, createNodes (with the host reads of the last flag and
 *       offset), updateTreeParticles, and the upward updateTreeMass loop.
 *       Writes: box corners (6 floats), keys in, keys out, permutation, level
 *       count, offsets and counts, node count, nodes, sorted pos and vel.
 *
 *   dropin loop <in.bin> <out.bin> <steps> <eps> <G> <theta> <dt>
 *       The reference's main loop (basicGravity.cu:709-783) as INTEGRATION.md
 *       shows it: initialiseTree once, then per step buildTree (pointer swap),
 *       calculateAcceleration, positionUpdater; destroyTree.  Writes the final
 *       pos (n float4) and vel (n float3) in the order the last build left
 *       them, and that build's permutation.
 *
 * Input: int32 n, then n float4 positions (mass in w), n float3 velocities.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "main.h"

#define CK(x)                                                                         \
    do {                                                                              \
        cudaError_t e_ = (x);                                                         \
        if (e_ != cudaSuccess) {                                                      \
            fprintf(stderr, "dropin: %s at line %d\n", cudaGetErrorString(e_), __LINE__); \
            exit(2);                                                                  \
        }                                                                             \
    } while (0)

static void* xmalloc(size_t b) {
    void* p = calloc(1, b ? b : 1);
    if (!p) {
        fprintf(stderr, "dropin: out of host memory\n");
        exit(2);
    }
    return p;
}

static int read_input(const char* path, float4** pos, float3** vel) {
    FILE* f = fopen(path, "rb");
    int n = 0;
    if (!f || fread(&n, sizeof n, 1, f) != 1 || n <= 0) {
        fprintf(stderr, "dropin: cannot read %s\n", path);
        exit(2);
    }
    *pos = (float4*)xmalloc(sizeof(float4) * (size_t)n);
    *vel = (float3*)xmalloc(sizeof(float3) * (size_t)n);
    if (fread(*pos, sizeof(float4), (size_t)n, f) != (size_t)n || fread(*vel, sizeof(float3), (size_t)n, f) != (size_t)n) {
        fprintf(stderr, "dropin: short input %s\n", path);
        exit(2);
    }
    fclose(f);
    return n;
}

static void put(FILE* f, const void* p, size_t bytes) {
    if (fwrite(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "dropin: write failed\n");
        exit(2);
    }
}

static void put_device(FILE* f, const void* dev, size_t bytes) {
    void* h = xmalloc(bytes);
    CK(cudaMemcpy(h, dev, bytes, cudaMemcpyDeviceToHost));
    put(f, h, bytes);
    free(h);
}

static int levels(const char* in, const char* out) {
    float4* hPos;
    float3* hVel;
    const int n = read_input(in, &hPos, &hVel);
    const int maxNodes = 8 * n;
    float4 *pos, *sortedPos;
    float3 *vel, *sortedVel, *corners;
    uint64_t *keysIn, *keysOut;
    uint32_t *idxIn, *idxOut;
    node* nodes;
    CK(cudaMalloc((void**)&pos, sizeof(float4) * n));
    CK(cudaMalloc((void**)&vel, sizeof(float3) * n));
    CK(cudaMalloc((void**)&sortedPos, sizeof(float4) * n));
    CK(cudaMalloc((void**)&sortedVel, sizeof(float3) * n));
    CK(cudaMalloc((void**)&corners, sizeof(float3) * (2 * BOXBLOCKS + 4)));
    CK(cudaMalloc((void**)&keysIn, sizeof(uint64_t) * n));
    CK(cudaMalloc((void**)&keysOut, sizeof(uint64_t) * n));
    CK(cudaMalloc((void**)&idxIn, sizeof(uint32_t) * n));
    CK(cudaMalloc((void**)&idxOut, sizeof(uint32_t) * n));
    CK(cudaMalloc((void**)&nodes, sizeof(node) * (size_t)maxNodes));
    CK(cudaMemcpy(pos, hPos, sizeof(float4) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(vel, hVel, sizeof(float3) * n, cudaMemcpyHostToDevice));

    /* stage 1: bounding box, both ways (tree.cu:414-490; basicGravity.cu:79-113) */
    float3* blockMin = corners;
    float3* blockMax = corners + BOXBLOCKS;
    float3* gMin = corners + 2 * BOXBLOCKS;
    float3* gMax = gMin + 1;
    localMinMaxFinder(pos, (unsigned)n, blockMin, blockMax, 0);
    globalMinMaxReducer(blockMin, blockMax, BOXBLOCKS, gMin, gMax, 0);
    CK(cudaDeviceSynchronize());
    float3 lo, hi;
    CK(cudaMemcpy(&lo, gMin, sizeof lo, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&hi, gMax, sizeof hi, cudaMemcpyDeviceToHost));
    worldBox box;
    memset(&box, 0, sizeof box);
    createWorldBox(pos, n, blockMin, blockMax, gMin + 2, gMin + 3, &box);
    if (box.scale == 0.0f) {
        fprintf(stderr, "dropin: world box failed\n");
        return 3;
    }
    /* root node (basicGravity.cu:158-169) */
    node root;
    memset(&root, 0, sizeof root);
    root.particleCount = n;
    for (int c = 0; c < 8; c++) root.child[c] = -1;
    CK(cudaMemcpy(nodes, &root, sizeof root, cudaMemcpyHostToDevice));

    /* stages 2-3: keys, sort, reorder */
    mortonEncode(pos, keysIn, idxIn, n, box, 0);
    radixSorter* sorter = sorterCreate(n);
    radixSortPairs(sorter, keysIn, keysOut, idxIn, idxOut, n);
    reorderParticles(pos, vel, sortedPos, sortedVel, idxOut, n, 0);
    CK(cudaDeviceSynchronize());

    /* stage 4: the level loop (basicGravity.cu:232-310) */
    treeBuilder* sum = sumCreate(n);
    uint32_t* offsets = sum->offsetsPing;
    uint32_t* prevOffsets = sum->offsetsPong;
    uint32_t* flags = sum->flagsPing;
    uint32_t* prevFlags = sum->flagsPong;
    int levelOffsets[22] = {0}, levelCount[22] = {0}, deepest = 0;
    int arrayLevelOffset = 1, prevArrayLevelOffset = 0;
    levelCount[0] = 1;
    for (int level = 1; level <= 21; level++) {
        identifyNodesAtLevel(keysOut, level, n, flags, 0);
        CK(cudaDeviceSynchronize());
        prefixSum(sum, flags, offsets, n);
        CK(cudaDeviceSynchronize());
        createNodes(keysOut, flags, prevFlags, offsets, prevOffsets, nodes, level, arrayLevelOffset,
                    prevArrayLevelOffset, n, maxNodes, 0);
        CK(cudaDeviceSynchronize());
        uint32_t lastFlag = 0, lastOffset = 0;
        CK(cudaMemcpy(&lastFlag, flags + (n - 1), sizeof lastFlag, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(&lastOffset, offsets + (n - 1), sizeof lastOffset, cudaMemcpyDeviceToHost));
        const int nodeCount = (int)(lastFlag + lastOffset);
        if (nodeCount == 0) {
            levelCount[level] = 0;
            levelOffsets[level] = arrayLevelOffset;
            break;
        }
        if (nodeCount + arrayLevelOffset > maxNodes) {
            fprintf(stderr, "dropin: node array overflow at level %d\n", level);
            return 3;
        }
        updateTreeParticles(nodes, arrayLevelOffset, nodeCount, n, 0);
        prevArrayLevelOffset = arrayLevelOffset;
        levelOffsets[level] = arrayLevelOffset;
        arrayLevelOffset += nodeCount;
        levelCount[level] = nodeCount;
        uint32_t* t = prevOffsets;
        prevOffsets = offsets;
        offsets = t;
        t = prevFlags;
        prevFlags = flags;
        flags = t;
        deepest++;
    }
    CK(cudaDeviceSynchronize());
    /* stage 5: upward mass pass (basicGravity.cu:317-319) */
    for (int j = deepest; j >= 0; j--) updateTreeMass(nodes, sortedPos, j, levelCount[j], levelOffsets[j], 0);
    CK(cudaDeviceSynchronize());
    const int count = levelOffsets[deepest] + levelCount[deepest];

    FILE* f = fopen(out, "wb");
    if (!f) return 2;
    put(f, &lo, sizeof lo);
    put(f, &hi, sizeof hi);
    put(f, &box, sizeof box);
    put_device(f, keysIn, sizeof(uint64_t) * n);
    put_device(f, keysOut, sizeof(uint64_t) * n);
    put_device(f, idxOut, sizeof(uint32_t) * n);
    put(f, &deepest, sizeof deepest);
    put(f, levelOffsets, sizeof levelOffsets);
    put(f, levelCount, sizeof levelCount);
    put(f, &count, sizeof count);
    put_device(f, nodes, sizeof(node) * (size_t)count);
    put_device(f, sortedPos, sizeof(float4) * n);
    put_device(f, sortedVel, sizeof(float3) * n);
    fclose(f);

    sumDestroyer(sum);
    sorterDestroyer(sorter);
    cudaFree(pos);
    cudaFree(vel);
    cudaFree(sortedPos);
    cudaFree(sortedVel);
    cudaFree(corners);
    cudaFree(keysIn);
    cudaFree(keysOut);
    cudaFree(idxIn);
    cudaFree(idxOut);
    cudaFree(nodes);
    free(hPos);
    free(hVel);
    return 0;
}

static int loop(const char* in, const char* out, int steps, float eps, float G, float theta, float dt) {
    float4* hPos;
    float3* hVel;
    const int n = read_input(in, &hPos, &hVel);
    int accelerationBlocks, treeBuilderBlocks, integrateBlocks, padded, integrationThreads, treeThreads;
    blockNumCalculator(&accelerationBlocks, &treeBuilderBlocks, &integrateBlocks, &padded, &integrationThreads,
                       &treeThreads, n);
    float4* pos;
    float3 *vel, *acc;
    CK(cudaMalloc((void**)&pos, sizeof(float4) * padded));
    CK(cudaMalloc((void**)&vel, sizeof(float3) * padded));
    CK(cudaMalloc((void**)&acc, sizeof(float3) * padded));
    CK(cudaMemset(pos, 0, sizeof(float4) * padded));
    CK(cudaMemset(vel, 0, sizeof(float3) * padded));
    CK(cudaMemset(acc, 0, sizeof(float3) * padded));
    CK(cudaMemcpy(pos, hPos, sizeof(float4) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(vel, hVel, sizeof(float3) * n, cudaMemcpyHostToDevice));
    float4* ownedPos = pos;
    float3* ownedVel = vel;

    treeState* state = (treeState*)xmalloc(sizeof(treeState));
    initialiseTree(state, n, padded, integrateBlocks);
    for (int i = 0; i < steps; i++) {
        buildTree(state, &pos, &vel);
        calculateAcceleration(pos, *state, acc, eps * eps, G, theta, n, 0);
        positionUpdater(pos, vel, acc, n, dt, 0);
    }
    CK(cudaDeviceSynchronize());
    FILE* f = fopen(out, "wb");
    if (!f) return 2;
    put_device(f, pos, sizeof(float4) * n);
    put_device(f, vel, sizeof(float3) * n);
    put_device(f, state->indexOut, sizeof(uint32_t) * n);
    fclose(f);
    /* destroyTree frees the pos/vel pair initialiseTree allocated, whichever
     * side of the swap it is on now; the caller frees the pair it allocated */
    destroyTree(state);
    cudaFree(ownedPos);
    cudaFree(ownedVel);
    cudaFree(acc);
    free(state);
    free(hPos);
    free(hVel);
    return 0;
}

int main(int argc, char** argv) {
    if (argc == 4 && !strcmp(argv[1], "levels")) return levels(argv[2], argv[3]);
    if (argc == 9 && !strcmp(argv[1], "loop"))
        return loop(argv[2], argv[3], atoi(argv[4]), (float)atof(argv[5]), (float)atof(argv[6]),
                    (float)atof(argv[7]), (float)atof(argv[8]));
    fprintf(stderr, "usage: dropin levels <in> <out> | dropin loop <in> <out> <steps> <eps> <G> <theta> <dt>\n");
    return 1;
}
