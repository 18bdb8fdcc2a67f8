// peak.cu — FP32 FMA-pipe throughput probe.
//
// The walk is bound by the FP32 pipe (about 12 FP32 instructions per
// body-node interaction), so its roofline denominator is the FMA throughput
// this GPU sustains, measured here rather than taken from a data sheet: each
// thread runs 8 independent FMA chains for `iters` iterations; FLOPs =
// 2 * 8 * iters * threads.
#include "bh_internal.cuh"

__global__ void __launch_bounds__(256) k_fma_probe(float* out, int iters, float a, float b) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            x0 = __fmaf_rn(x0, a, b); x1 = __fmaf_rn(x1, a, b); x2 = __fmaf_rn(x2, a, b); x3 = __fmaf_rn(x3, a, b);
            x4 = __fmaf_rn(x4, a, b); x5 = __fmaf_rn(x5, a, b); x6 = __fmaf_rn(x6, a, b); x7 = __fmaf_rn(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 12345.678f) out[0] = s;  // keeps the chains alive
}

// Runs the probe `reps` times on `stream`; returns the best TFLOP/s.
extern "C" int bh_fma_peak_tflops(int reps, float* tflops, cudaStream_t stream) {
    if (!tflops || reps <= 0) return BH_ERR_INVALID;
    float* out = nullptr;
    cudaEvent_t e0, e1;
    BH_CUDA_TRY(cudaMalloc(&out, sizeof(float)));
    BH_CUDA_TRY(cudaEventCreate(&e0));
    BH_CUDA_TRY(cudaEventCreate(&e1));
    const int blocks = bh_sm_count() * 8, threads = 256, iters = 2048;
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    float best = 0.f;
    k_fma_probe<<<blocks, threads, 0, stream>>>(out, iters / 4, 0.999f, 1e-3f);  // warm-up
    for (int r = 0; r < reps; r++) {
        BH_CUDA_TRY(cudaEventRecord(e0, stream));
        k_fma_probe<<<blocks, threads, 0, stream>>>(out, iters, 0.999f, 1e-3f);
        BH_CUDA_TRY(cudaEventRecord(e1, stream));
        BH_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        BH_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        const float t = (float)(flops / (ms * 1e-3) / 1e12);
        best = t > best ? t : best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = best;
    return BH_OK;
}
