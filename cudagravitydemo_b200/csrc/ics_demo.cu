// ics_demo.cu — the reference program's own initial conditions, seeded and
// generated on the device.
//
// The reference's main() (basicGravity.cu:491-507, 694-697) builds its demo
// galaxy on the host with rand() seeded by the clock: N stars of equal mass
// (total 5), 80% in an exponential disk (initialConditions.c:246-297:
// radius by rejection sampling of P(R) ~ R exp(-R/R_d) below 5 R_d, uniform
// angle, Laplace-distributed height, the circular speed of the enclosed
// disk mass, a yaw-pitch-roll rotation and an offset) and 20% in a "halo"
// (initialConditions.c:306-382: radius uniform in [0, 5 R_d), direction with
// cos(polar) uniform, at the galaxy's net velocity).  Here one thread builds
// one body from a counter-based generator keyed by (seed, body, draw), so the
// result depends only on the seed, not on the launch.
#include <math.h>

#include "bh_internal.cuh"

namespace {

// SplitMix64 finaliser: a bijective 64-bit mix (Steele, Lea, Flood 2014).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Uniform float in (0, 1] for draw k of body i (never 0, like the reference's
// randDecimal, initialConditions.c:33-37, so logs and divisions stay finite).
__device__ __forceinline__ float uniform(uint64_t seed, uint32_t i, uint32_t k) {
    const uint64_t h = mix64(seed ^ mix64(((uint64_t)i << 32) | k));
    return (float)((h >> 40) + 1) * (1.0f / 16777216.0f);
}

constexpr int kMaxAttempts = 200;  // initialConditions.c:24
constexpr float kTruncation = 5.0f;  // scale lengths (initialConditions.c:20)

}  // namespace

__global__ void k_ic_demo(float4* __restrict__ pos, float3* __restrict__ vel, int n, int nDisk, bh_demo_params p,
                          uint64_t seed, int* err) {
    // rotation (initialConditions.c:208-240): the product yaw * pitch * roll
    // of the matrices as written there, each initialiser read the way cglm
    // reads it (column by column), i.e. Y^T P^T R^T of the row-wise reading
    const float cy = cosf(p.rotation[0]), sy = sinf(p.rotation[0]);
    const float cp = cosf(p.rotation[1]), sp = sinf(p.rotation[1]);
    const float cr = cosf(p.rotation[2]), sr = sinf(p.rotation[2]);
    const float R[3][3] = {{cy * cp, sy * cr + cy * sp * sr, sy * sr - cy * sp * cr},
                           {-sy * cp, cy * cr - sy * sp * sr, cy * sr + sy * sp * cr},
                           {sp, -cp * sr, cp * cr}};
    const float m = p.totalMass / (float)n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float x, y, z, vx = 0.f, vy = 0.f, vz = 0.f;
        if (i < nDisk) {
            const float alpha = 1.0f / p.scaleLength;
            const float yMax = p.scaleLength * 0.367879441171f;  // max of R exp(-alpha R), at R = 1/alpha
            const float rMax = kTruncation * p.scaleLength;
            float r = -1.f;
            for (int a = 0; a < kMaxAttempts; a++) {
                const float rr = rMax * uniform(seed, i, 2 * a);
                const float yy = yMax * uniform(seed, i, 2 * a + 1);
                if (yy < rr * expf(-alpha * rr)) {
                    r = rr;
                    break;
                }
            }
            if (r < 0.f) {  // the reference exits here (initialConditions.c:64-67)
                bh_set_error(err, BH_ERR_INTERNAL);
                r = p.scaleLength;
            }
            const float ang = 6.28318530717958647692f * uniform(seed, i, 1000);
            const float ca = cosf(ang), sa = sinf(ang);
            const float u = uniform(seed, i, 1001);  // Laplace height (initialConditions.c:150-161)
            const float h = (u >= 0.5f) ? -logf(2.0f - 2.0f * u) * p.scaleThickness : logf(2.0f * u) * p.scaleThickness;
            // circular speed of the enclosed exponential-disk mass (initialConditions.c:163-175)
            const float menc = p.totalMass * (1.0f - (1.0f + r / p.scaleLength) * expf(-r / p.scaleLength));
            const float v = r > 0.f ? sqrtf(p.G * menc / r) : 0.f;
            const float lx = r * ca, ly = r * sa, lvx = -v * sa, lvy = v * ca;
            x = R[0][0] * lx + R[0][1] * ly + R[0][2] * h;
            y = R[1][0] * lx + R[1][1] * ly + R[1][2] * h;
            z = R[2][0] * lx + R[2][1] * ly + R[2][2] * h;
            vx = R[0][0] * lvx + R[0][1] * lvy;
            vy = R[1][0] * lvx + R[1][1] * lvy;
            vz = R[2][0] * lvx + R[2][1] * lvy;
        } else {  // halo (initialConditions.c:327-353)
            const float u1 = uniform(seed, i, 0), u2 = uniform(seed, i, 1), u3 = uniform(seed, i, 2);
            const float phi = 6.28318530717958647692f * u1;
            const float c = 2.0f * u2 - 1.0f;
            const float s = sqrtf(fmaxf(1.0f - c * c, 0.0f));
            const float r = p.scaleLength * kTruncation * u3;
            x = r * s * cosf(phi);
            y = r * s * sinf(phi);
            z = r * c;
        }
        pos[i] = make_float4(x + p.centre[0], y + p.centre[1], z + p.centre[2], m);
        vel[i] = make_float3(vx + p.velocity[0], vy + p.velocity[1], vz + p.velocity[2]);
    }
}

extern "C" void bh_demo_params_default(bh_demo_params* p) {
    if (!p) return;
    p->totalMass = 5.0f;       // basicGravity.cu:500
    p->scaleLength = 4.0f;     // basicGravity.cu:541
    p->scaleThickness = 0.3f;  // basicGravity.cu:542
    p->haloFraction = 0.2f;    // basicGravity.cu:694
    p->G = 1.0f;               // units.c:3
    for (int k = 0; k < 3; k++) p->rotation[k] = p->centre[k] = p->velocity[k] = 0.0f;
}

extern "C" int bh_ic_demo(float4* pos, float3* vel, int n, const bh_demo_params* params, uint64_t seed,
                          cudaStream_t s) {
    if (!pos || !vel || n <= 0) return BH_ERR_INVALID;
    bh_demo_params p;
    if (params) p = *params;
    else bh_demo_params_default(&p);
    if (!(p.scaleLength > 0.f) || !(p.scaleThickness > 0.f) || !(p.haloFraction >= 0.f && p.haloFraction <= 1.f))
        return BH_ERR_INVALID;
    const int nHalo = (int)(n * p.haloFraction);  // calculateHaloNum, initialConditions.c:302-305
    int* err = nullptr;
    cudaError_t e = cudaMallocAsync(&err, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    const int blocks = (n + 255) / 256 < 8 * bh_sm_count() ? (n + 255) / 256 : 8 * bh_sm_count();
    k_ic_demo<<<blocks, 256, 0, s>>>(pos, vel, n, n - nHalo, p, seed, err);
    int h = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaFreeAsync(err, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    return h ? BH_ERR_INTERNAL : BH_OK;
}
