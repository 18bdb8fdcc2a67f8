// ref_harness.cu — drives the reference's own step on given inputs.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's sources
// (basicGravity.cu with -Dmain=ref_main, tree.cu, sorting.cu, units.c,
// inputOutput.c, initialConditions.c) by oracle/build.py into
// oracle/_ref/libref.so.  It calls the reference's initialiseTree, buildTree,
// calculateAcceleration and positionUpdater exactly as its main() loop does
// (basicGravity.cu:481-486, 709, 767-792), with two deliberate differences:
// the inputs are given instead of time-seeded, and buildTree always gets the
// velocity buffer (main() passes the acceleration buffer at its first call,
// basicGravity.cu:715).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "main.h"

void initialiseTree(treeState* state, int starCount, int paddedStarCount, int integrateBlocks);
void buildTree(treeState* tree, float4** cudaPosMasVals, float3** cudaVelVals);
void blockNumCalculator(int* accelerationBlocks, int* treeBuilderBlocks, int* integrateBlocks, int* paddedStarCount,
                        int* integrationThreadsPerBlock, int* treeBuilderThreadsPerBlock, int starCount);
void sumDestroyer(treeBuilder* sum);

#define H_CHECK(x)                                                                \
    do {                                                                          \
        cudaError_t e_ = (x);                                                     \
        if (e_ != cudaSuccess) {                                                  \
            fprintf(stderr, "ref harness: %s at %d\n", cudaGetErrorString(e_), __LINE__); \
            return -1;                                                            \
        }                                                                         \
    } while (0)

extern "C" {

// Runs `steps` reference steps from (pos, vel).  Outputs describe the LAST
// step: keysIn = its Morton keys before sorting, keysOut/perm = after,
// nodes = its tree (first nodeCap nodes), levelOffsets/levelCount (22 each),
// acc = accelerations (sorted order), posOut/velOut = state after the step
// (sorted order), ids = input index of each output body (the composition of
// every step's permutation; the reference itself does not track it).  Any
// output pointer may be NULL.  msPerStep = mean cudaEvent time of the steps
// (with ids requested, each step also copies its permutation to the host
// outside the timed region).  Returns the node count, or -1.
int ref_run(const float* pos4, const float* vel3, int n, float eps, float G, float theta, float dt, int steps,
            uint64_t* keysIn, uint64_t* keysOut, uint32_t* perm, void* nodes, int nodeCap, int* levelOffsets,
            int* levelCount, int* deepest, float* acc3, float* posOut4, float* velOut3, uint32_t* ids,
            float* msPerStep) {
    uint32_t* stepPerm = nullptr;
    uint32_t* idTmp = nullptr;
    if (ids) {
        stepPerm = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
        idTmp = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
        for (int i = 0; i < n; i++) ids[i] = (uint32_t)i;
    }
    int accelerationBlocks, treeBuilderBlocks, integrateBlocks, integrationThreads, treeThreads, padded;
    blockNumCalculator(&accelerationBlocks, &treeBuilderBlocks, &integrateBlocks, &padded, &integrationThreads,
                       &treeThreads, n);
    float4* dPos = nullptr;
    float3* dVel = nullptr;
    float3* dAcc = nullptr;
    H_CHECK(cudaMalloc(&dPos, sizeof(float4) * padded));
    H_CHECK(cudaMalloc(&dVel, sizeof(float3) * padded));
    H_CHECK(cudaMalloc(&dAcc, sizeof(float3) * padded));
    H_CHECK(cudaMemset(dPos, 0, sizeof(float4) * padded));
    H_CHECK(cudaMemset(dVel, 0, sizeof(float3) * padded));
    H_CHECK(cudaMemset(dAcc, 0, sizeof(float3) * padded));
    H_CHECK(cudaMemcpy(dPos, pos4, sizeof(float4) * n, cudaMemcpyHostToDevice));
    H_CHECK(cudaMemcpy(dVel, vel3, sizeof(float3) * n, cudaMemcpyHostToDevice));
    float4* ownedPos = dPos;
    float3* ownedVel = dVel;

    treeState* state = (treeState*)calloc(1, sizeof(treeState));
    initialiseTree(state, n, padded, integrateBlocks);
    float4* statePos = state->sortedPosMassVals;
    float3* stateVel = state->sortedVelVals;

    cudaEvent_t t0, t1;
    H_CHECK(cudaEventCreate(&t0));
    H_CHECK(cudaEventCreate(&t1));
    float total = 0.f;
    for (int s = 0; s < steps; s++) {
        const bool last = (s == steps - 1);
        H_CHECK(cudaEventRecord(t0, 0));
        buildTree(state, &dPos, &dVel);
        if (last && keysIn) H_CHECK(cudaMemcpy(keysIn, state->mortonIn, 8 * (size_t)n, cudaMemcpyDeviceToHost));
        calculateAcceleration<<<accelerationBlocks, WARPTHREADS>>>(dPos, *state, dAcc, eps * eps, G, theta, n);
        if (last && (nodes || acc3)) {
            H_CHECK(cudaDeviceSynchronize());
            if (acc3) H_CHECK(cudaMemcpy(acc3, dAcc, 12 * (size_t)n, cudaMemcpyDeviceToHost));
        }
        positionUpdater<<<integrateBlocks, integrationThreads>>>(dPos, dVel, dAcc, n, dt);
        H_CHECK(cudaEventRecord(t1, 0));
        H_CHECK(cudaDeviceSynchronize());
        H_CHECK(cudaGetLastError());
        float ms = 0.f;
        H_CHECK(cudaEventElapsedTime(&ms, t0, t1));
        total += ms;
        if (ids) {
            H_CHECK(cudaMemcpy(stepPerm, state->indexOut, 4 * (size_t)n, cudaMemcpyDeviceToHost));
            for (int i = 0; i < n; i++) idTmp[i] = ids[stepPerm[i]];
            memcpy(ids, idTmp, 4 * (size_t)n);
        }
    }
    free(stepPerm);
    free(idTmp);
    if (msPerStep) *msPerStep = total / (steps > 0 ? steps : 1);
    int count = state->levelOffsets[state->deepestLevel] + state->levelCount[state->deepestLevel];
    if (keysOut) H_CHECK(cudaMemcpy(keysOut, state->mortonOut, 8 * (size_t)n, cudaMemcpyDeviceToHost));
    if (perm) H_CHECK(cudaMemcpy(perm, state->indexOut, 4 * (size_t)n, cudaMemcpyDeviceToHost));
    if (nodes) {
        const int c = count < nodeCap ? count : nodeCap;
        H_CHECK(cudaMemcpy(nodes, state->nodes, sizeof(node) * (size_t)c, cudaMemcpyDeviceToHost));
    }
    if (levelOffsets) memcpy(levelOffsets, state->levelOffsets, sizeof(int) * 22);
    if (levelCount) memcpy(levelCount, state->levelCount, sizeof(int) * 22);
    if (deepest) *deepest = state->deepestLevel;
    if (posOut4) H_CHECK(cudaMemcpy(posOut4, dPos, 16 * (size_t)n, cudaMemcpyDeviceToHost));
    if (velOut3) H_CHECK(cudaMemcpy(velOut3, dVel, 12 * (size_t)n, cudaMemcpyDeviceToHost));

    // release everything the reference allocated (it has no destroy)
    sorterDestroyer(state->sorter);
    sumDestroyer(state->builder);
    cudaFree(state->nodes);
    cudaFree(state->mortonIn);
    cudaFree(state->mortonOut);
    cudaFree(state->indexIn);
    cudaFree(state->indexOut);
    for (int k = 0; k < 4; k++) cudaFree(state->boundingData[k]);
    cudaFree(ownedPos);
    cudaFree(ownedVel);
    cudaFree(statePos);
    cudaFree(stateVel);
    cudaFree(dAcc);
    free(state);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return count;
}

}  // extern "C"
