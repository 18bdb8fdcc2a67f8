// direct.cu — FP64 direct-sum accelerations of selected target bodies.
//
// The error of every Barnes-Hut walk is stated against this sum:
// a_t = sum_j G m_j (x_j - x_t) / (|x_j - x_t|^2 + eps^2)^{3/2} in double
// precision over all n source bodies.  One thread per target; sources stream
// through shared memory in tiles.  It is an evaluation tool (labels for the
// learned opening criterion, RMS force errors), not part of a step.
#include "bh_internal.cuh"

namespace {
constexpr int kThreads = 256;
}

__global__ void __launch_bounds__(kThreads)
k_direct_f64(const float4* __restrict__ pos, int n, const int* __restrict__ targets, int nt, double eps2,
             double G, double* __restrict__ acc) {
    __shared__ float4 tile[kThreads];
    const int t = blockIdx.x * kThreads + threadIdx.x;
    const bool active = t < nt;
    double xt = 0, yt = 0, zt = 0;
    if (active) {
        const float4 p = pos[targets ? targets[t] : t];
        xt = p.x; yt = p.y; zt = p.z;
    }
    double ax = 0, ay = 0, az = 0;
    for (int base = 0; base < n; base += kThreads) {
        const int j = base + threadIdx.x;
        tile[threadIdx.x] = (j < n) ? pos[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int cnt = (n - base < kThreads) ? n - base : kThreads;
        if (active) {
#pragma unroll 4
            for (int k = 0; k < cnt; k++) {
                const float4 s = tile[k];
                const double dx = (double)s.x - xt, dy = (double)s.y - yt, dz = (double)s.z - zt;
                const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
                const double ri = rsqrt(r2);
                const double f = (double)s.w * ri * ri * ri;
                ax = fma(f, dx, ax);
                ay = fma(f, dy, ay);
                az = fma(f, dz, az);
            }
        }
        __syncthreads();
    }
    if (active) {
        acc[3 * t] = G * ax;
        acc[3 * t + 1] = G * ay;
        acc[3 * t + 2] = G * az;
    }
}

extern "C" int bh_direct_sum_f64(const float4* pos, int n, const int* targets, int ntargets, double eps, double G,
                                 double* acc, cudaStream_t s) {
    if (!pos || !acc || n <= 0 || ntargets <= 0) return BH_ERR_INVALID;
    const int blocks = (ntargets + kThreads - 1) / kThreads;
    k_direct_f64<<<blocks, kThreads, 0, s>>>(pos, n, targets, ntargets, eps * eps, G, acc);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BH_OK : bh_note_cuda_error(e);
}
