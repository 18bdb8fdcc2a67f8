/*
 * frames.c — the reference's frame loop (steps, then a frame of positions
 * with their body ids, basicGravity.cu:767-800) through the status-returning
 * API, with the host arrays page-locked and mapped so that the last step of
 * each call writes them from the walk.  Plain C, compiled by gcc.  Test
 * program: tests/test_gpu_frames.py builds and runs it.
 *
 *   frames <in.bin> <out.bin> <frames> <stepsPerFrame> <eps> <G> <theta> <dt>
 *
 * Input: int32 n, then n float4 positions (mass in w), n float3 velocities.
 * Output: the arrays after the last frame: n float4 positions, n float3
 * velocities and n uint32 body ids, in that step's Morton order.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime_api.h>

#include "bh_api.h"

#define CK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            fprintf(stderr, "frames: %s at line %d\n", cudaGetErrorString(e_), __LINE__); \
            exit(2);                                                                   \
        }                                                                              \
    } while (0)

#define BK(x)                                                                         \
    do {                                                                              \
        int s_ = (x);                                                                 \
        if (s_ != BH_OK) {                                                            \
            fprintf(stderr, "frames: %s at line %d\n", bh_status_string(s_), __LINE__); \
            exit(3);                                                                  \
        }                                                                             \
    } while (0)

static void put(FILE* f, const void* p, size_t bytes) {
    if (fwrite(p, 1, bytes, f) != bytes) {
        fprintf(stderr, "frames: write failed\n");
        exit(2);
    }
}

int main(int argc, char** argv) {
    if (argc != 9) {
        fprintf(stderr, "usage: frames <in> <out> <frames> <stepsPerFrame> <eps> <G> <theta> <dt>\n");
        return 1;
    }
    const int frames = atoi(argv[3]), per = atoi(argv[4]);
    FILE* f = fopen(argv[1], "rb");
    int n = 0;
    if (!f || fread(&n, sizeof n, 1, f) != 1 || n <= 0) {
        fprintf(stderr, "frames: cannot read %s\n", argv[1]);
        return 2;
    }
    float4* pos;
    float3* vel;
    uint32_t* ids;
    CK(cudaHostAlloc((void**)&pos, sizeof(float4) * (size_t)n, cudaHostAllocMapped));
    CK(cudaHostAlloc((void**)&vel, sizeof(float3) * (size_t)n, cudaHostAllocMapped));
    CK(cudaHostAlloc((void**)&ids, sizeof(uint32_t) * (size_t)n, cudaHostAllocMapped));
    if (fread(pos, sizeof(float4), (size_t)n, f) != (size_t)n || fread(vel, sizeof(float3), (size_t)n, f) != (size_t)n) {
        fprintf(stderr, "frames: short input %s\n", argv[1]);
        return 2;
    }
    fclose(f);
    for (int k = 0; k < n; k++) ids[k] = (uint32_t)k;

    bh_params p;
    bh_params_default(&p);
    p.eps = (float)atof(argv[5]);
    p.G = (float)atof(argv[6]);
    p.theta = (float)atof(argv[7]);
    p.dt = (float)atof(argv[8]);
    bh_sim* sim;
    BK(bh_sim_create(&sim, n, &p, 0));
    for (int fr = 0; fr < frames; fr++) {
        BK(bh_sim_step_host_sorted(sim, pos, vel, ids, n, per));
        /* a frame: body ids[k] is at pos[k]; a writer would store it here */
    }
    BK(bh_sim_destroy(sim));

    FILE* o = fopen(argv[2], "wb");
    if (!o) return 2;
    put(o, pos, sizeof(float4) * (size_t)n);
    put(o, vel, sizeof(float3) * (size_t)n);
    put(o, ids, sizeof(uint32_t) * (size_t)n);
    fclose(o);
    CK(cudaFreeHost(pos));
    CK(cudaFreeHost(vel));
    CK(cudaFreeHost(ids));
    return 0;
}
