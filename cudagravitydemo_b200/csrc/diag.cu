// diag.cu — FP64 conserved-quantity diagnostics of a body set.
//
// The reference has none; the engine states its energy drift against these:
//   M = sum m, centre of mass and its velocity, P = sum m v,
//   L = sum m (x cross v) about the origin, T = sum m v^2 / 2,
//   W = -(G/2) sum_{i != j} m_i m_j / sqrt(|x_i - x_j|^2 + eps^2)
// (the Plummer-softened potential whose gradient is the walk's force law).
// Every sum is in double precision; W is the exact O(N^2) pair sum.  Block
// partials are reduced by one block in a fixed order, so results are
// deterministic for a given launch geometry.
#include "bh_internal.cuh"

namespace {
constexpr int kThreads = 256;
constexpr int kMoments = 11;  // M, Mx, My, Mz, Px, Py, Pz, Lx, Ly, Lz, 2T
constexpr int kMomentBlocksMax = 1184;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block sum of v[0..K); result in thread 0.
template <int K>
__device__ void block_sum(double v[K]) {
    __shared__ double part[kThreads / 32][K];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < K; k++) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; k++) part[w][k] = v[k];
    __syncthreads();
    if (w == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = warp_sum(lane < kThreads / 32 ? part[lane][k] : 0.0);
    }
    __syncthreads();
}
}  // namespace

__global__ void __launch_bounds__(kThreads)
k_diag_moments(const float4* __restrict__ pos, const float3* __restrict__ vel, int n, double* __restrict__ partial) {
    double v[kMoments] = {0};
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
        const float4 p = pos[i];
        const float3 u = vel[i];
        const double m = p.w, x = p.x, y = p.y, z = p.z, vx = u.x, vy = u.y, vz = u.z;
        v[0] += m;
        v[1] += m * x;
        v[2] += m * y;
        v[3] += m * z;
        v[4] += m * vx;
        v[5] += m * vy;
        v[6] += m * vz;
        v[7] += m * (y * vz - z * vy);
        v[8] += m * (z * vx - x * vz);
        v[9] += m * (x * vy - y * vx);
        v[10] += m * (vx * vx + vy * vy + vz * vz);
    }
    block_sum<kMoments>(v);
    if (threadIdx.x == 0)
        for (int k = 0; k < kMoments; k++) partial[(size_t)blockIdx.x * kMoments + k] = v[k];
}

// Per block: sum over its targets i of m_i * sum_{j != i} m_j / r_ij (softened).
__global__ void __launch_bounds__(kThreads)
k_diag_potential(const float4* __restrict__ pos, int n, double eps2, double* __restrict__ partial) {
    __shared__ double4 tile[kThreads];
    const int i = blockIdx.x * kThreads + threadIdx.x;
    const bool active = i < n;
    double xi = 0, yi = 0, zi = 0, mi = 0;
    if (active) {
        const float4 p = pos[i];
        xi = p.x; yi = p.y; zi = p.z; mi = p.w;
    }
    double phi = 0.0;
    for (int base = 0; base < n; base += kThreads) {
        const int j = base + threadIdx.x;
        if (j < n) {
            const float4 q = pos[j];
            tile[threadIdx.x] = make_double4(q.x, q.y, q.z, q.w);
        }
        __syncthreads();
        const int cnt = (n - base < kThreads) ? n - base : kThreads;
        if (active) {
            for (int k = 0; k < cnt; k++) {
                const double4 q = tile[k];
                const double dx = q.x - xi, dy = q.y - yi, dz = q.z - zi;
                const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, eps2)));
                const double t = q.w * rsqrt(r2);
                phi += (base + k == i) ? 0.0 : t;
            }
        }
        __syncthreads();
    }
    double v[1] = {mi * phi};
    block_sum<1>(v);
    if (threadIdx.x == 0) partial[blockIdx.x] = v[0];
}

// One block: fixed-order reduction of the partials into the result
// (kMoments moment sums, then sum m_i phi_i).
__global__ void __launch_bounds__(kThreads)
k_diag_finalize(const double* __restrict__ moments, int nMomentBlocks, const double* __restrict__ pot, int nPotBlocks,
                double* __restrict__ out) {
    double v[kMoments + 1] = {0};
    for (int b = threadIdx.x; b < nMomentBlocks; b += kThreads)
        for (int k = 0; k < kMoments; k++) v[k] += moments[(size_t)b * kMoments + k];
    for (int b = threadIdx.x; b < nPotBlocks; b += kThreads) v[kMoments] += pot[b];
    block_sum<kMoments + 1>(v);
    if (threadIdx.x == 0)
        for (int k = 0; k <= kMoments; k++) out[k] = v[k];
}

extern "C" int bh_diagnostics_f64(const float4* pos, const float3* vel, int n, double eps, double G, int withPotential,
                                  bh_diagnostics* out, cudaStream_t s) {
    if (!pos || !vel || !out || n <= 0) return BH_ERR_INVALID;
    int mBlocks = (n + kThreads - 1) / kThreads;
    mBlocks = mBlocks > kMomentBlocksMax ? kMomentBlocksMax : mBlocks;
    const int pBlocks = withPotential ? (n + kThreads - 1) / kThreads : 0;
    double* scratch = nullptr;
    const size_t words = (size_t)mBlocks * kMoments + pBlocks + kMoments + 1;
    cudaError_t e = cudaMallocAsync(&scratch, words * sizeof(double), s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    double* mPart = scratch;
    double* pPart = mPart + (size_t)mBlocks * kMoments;
    double* res = pPart + pBlocks;
    double h[kMoments + 1];
    k_diag_moments<<<mBlocks, kThreads, 0, s>>>(pos, vel, n, mPart);
    if (withPotential) k_diag_potential<<<pBlocks, kThreads, 0, s>>>(pos, n, eps * eps, pPart);
    k_diag_finalize<<<1, kThreads, 0, s>>>(mPart, mBlocks, pPart, pBlocks, res);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, res, sizeof h, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaFreeAsync(scratch, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    bh_diagnostics d;
    d.mass = h[0];
    const double inv = h[0] != 0.0 ? 1.0 / h[0] : 0.0;
    for (int k = 0; k < 3; k++) {
        d.com[k] = h[1 + k] * inv;
        d.momentum[k] = h[4 + k];
        d.comVel[k] = h[4 + k] * inv;
        d.angularMomentum[k] = h[7 + k];
    }
    d.kinetic = 0.5 * h[10];
    d.potential = withPotential ? -0.5 * G * h[11] : 0.0;
    d.total = d.kinetic + d.potential;
    *out = d;
    return BH_OK;
}
