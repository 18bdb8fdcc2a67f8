// mlp.cu — the learned opening criterion: group features, a BF16 MLP
// (8 -> 32 -> 32 -> 1, ReLU, FP32 accumulation) on the tensor cores, its
// training (forward + backward + Adam) and the per-group choice of the
// relative-criterion budget.
//
// For a 32-body group and a candidate budget alpha, the MLP predicts
// log10 of the group's RMS relative force error under the relative opening
// criterion (walk.cu).  Per group, c = the largest candidate whose prediction
// meets the target; the budget is interpolated between candidates c and c+1
// where the predicted curve crosses the target (linear in log alpha), so a
// group's error sits at the target rather than up to a ladder step below it.
// A group whose predictions are not finite falls back to the reference's
// fixed-theta test (theta 0.5).
//
// Inputs (8): log10 alpha, then seven group features computed from the
// sorted bodies and the last step's accelerations (k_group_features).
// Matrix products use mma.sync m16n8k16 (BF16 in, FP32 accumulate): the
// network is 1.4k parameters, its GEMMs are 16 x 16 x 32 tiles, and a single
// warp-level MMA per tile is the right size for them.  The accumulator layout
// of one layer is the A-operand layout of the next, so layers chain in
// registers.
#include <cuda_bf16.h>

#include "bh_internal.cuh"
#include "bh_kernels.cuh"

// ------------------------------------------------------------- parameters
// Packed FP32 parameter block (row-major W[in][out]):
//   W1[8][32] b1[32] W2[32][32] b2[32] W3[32] b3  + feature mean[8], scale[8]
#define MLP_W1 0
#define MLP_B1 256
#define MLP_W2 288
#define MLP_B2 1312
#define MLP_W3 1344
#define MLP_B3 1376
#define MLP_TRAINED 1377  // trained parameters
#define MLP_MU 1377
#define MLP_SIG 1385
#define MLP_TOTAL 1393

static_assert(MLP_TOTAL == BH_MLP_PARAMS, "parameter block size");
static_assert(MLP_TRAINED == BH_MLP_TRAINED, "trained parameter count");

// The budget ladder: alpha_c = kMacAlpha0 * 2^c, c = 0..BH_MAC_CANDIDATES-1
// (about 5e-4 to 1e-2 RMS relative force error on a disk galaxy).
constexpr float kMacAlpha0 = 2e-4f;
static_assert(BH_MAC_CANDIDATES == 8, "the selection kernel evaluates 8 candidates per group");

namespace {

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// D = A * B + C, m16n8k16, A/B bf16, C/D f32
__device__ __forceinline__ void mma_bf16(float d[4], const uint32_t a[4], const uint32_t b[2], const float c[4]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%10,%11,%12,%13};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "f"(c[0]), "f"(c[1]), "f"(c[2]),
          "f"(c[3]));
}

// B fragment of a row-major weight W[in][out] (stride `out`) for the n-tile
// starting at column n0 and the k-step starting at row k0; rows >= kmax and
// columns >= nmax are zero.
__device__ __forceinline__ void load_b(uint32_t b[2], const float* W, int out, int k0, int n0, int kmax, int nmax) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int n = n0 + g;
    auto w = [&](int k) { return (k < kmax && n < nmax) ? W[k * out + n] : 0.f; };
    b[0] = pack_bf16(w(k0 + 2 * t), w(k0 + 2 * t + 1));
    b[1] = pack_bf16(w(k0 + 2 * t + 8), w(k0 + 2 * t + 9));
}

// Warp-resident weights: B fragments of W1 (1 k-step x 4 n-tiles), W2 (2 x 4),
// W3 (2 x 1, 1 output) and the biases of this thread's columns.
struct MlpRegs {
    uint32_t w1[4][2], w2[2][4][2], w3[2][2];
    float b1[4][2], b2[4][2], b3;
    float mu[2], sig[2];  // normalisation of this thread's inputs 2t, 2t+1
};

__device__ void load_mlp(MlpRegs& r, const float* P) {
    const int t = threadIdx.x & 3;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        load_b(r.w1[j], P + MLP_W1, 32, 0, 8 * j, 8, 32);
        load_b(r.w2[0][j], P + MLP_W2, 32, 0, 8 * j, 32, 32);
        load_b(r.w2[1][j], P + MLP_W2, 32, 16, 8 * j, 32, 32);
        r.b1[j][0] = P[MLP_B1 + 8 * j + 2 * t];
        r.b1[j][1] = P[MLP_B1 + 8 * j + 2 * t + 1];
        r.b2[j][0] = P[MLP_B2 + 8 * j + 2 * t];
        r.b2[j][1] = P[MLP_B2 + 8 * j + 2 * t + 1];
    }
    load_b(r.w3[0], P + MLP_W3, 1, 0, 0, 32, 1);
    load_b(r.w3[1], P + MLP_W3, 1, 16, 0, 32, 1);
    r.b3 = P[MLP_B3];
#pragma unroll
    for (int f = 0; f < 2; f++) {
        r.mu[f] = P[MLP_MU + 2 * t + f];
        r.sig[f] = P[MLP_SIG + 2 * t + f];
    }
}

// Forward pass of a 16-row tile.  x0/x1: this thread's raw features 2t, 2t+1
// of rows g and g+8 (x0 = row g, x1 = row g+8).  Returns pre-activations z1,
// z2 (accumulator layout) and the output of rows g and g+8 (valid in threads
// with t == 0).
struct Acts {
    float z1[4][4], z2[4][4];
    float y[2];
};

__device__ void forward(const MlpRegs& r, const float x0[2], const float x1[2], Acts& a) {
    const int t = threadIdx.x & 3;
    uint32_t ax[4];
    ax[0] = pack_bf16((x0[0] - r.mu[0]) * r.sig[0], (x0[1] - r.mu[1]) * r.sig[1]);
    ax[1] = pack_bf16((x1[0] - r.mu[0]) * r.sig[0], (x1[1] - r.mu[1]) * r.sig[1]);
    ax[2] = ax[3] = 0u;  // features 8..15: padding
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const float c[4] = {r.b1[j][0], r.b1[j][1], r.b1[j][0], r.b1[j][1]};
        mma_bf16(a.z1[j], ax, r.w1[j], c);
    }
    uint32_t ah[2][4];  // relu(z1) as the A operand of layer 2 (k-steps 0, 1)
#pragma unroll
    for (int s = 0; s < 2; s++) {
        ah[s][0] = pack_bf16(fmaxf(a.z1[2 * s][0], 0.f), fmaxf(a.z1[2 * s][1], 0.f));
        ah[s][1] = pack_bf16(fmaxf(a.z1[2 * s][2], 0.f), fmaxf(a.z1[2 * s][3], 0.f));
        ah[s][2] = pack_bf16(fmaxf(a.z1[2 * s + 1][0], 0.f), fmaxf(a.z1[2 * s + 1][1], 0.f));
        ah[s][3] = pack_bf16(fmaxf(a.z1[2 * s + 1][2], 0.f), fmaxf(a.z1[2 * s + 1][3], 0.f));
    }
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float c[4] = {r.b2[j][0], r.b2[j][1], r.b2[j][0], r.b2[j][1]};
        mma_bf16(a.z2[j], ah[0], r.w2[0][j], c);
        mma_bf16(a.z2[j], ah[1], r.w2[1][j], a.z2[j]);
    }
    uint32_t ah2[2][4];
#pragma unroll
    for (int s = 0; s < 2; s++) {
        ah2[s][0] = pack_bf16(fmaxf(a.z2[2 * s][0], 0.f), fmaxf(a.z2[2 * s][1], 0.f));
        ah2[s][1] = pack_bf16(fmaxf(a.z2[2 * s][2], 0.f), fmaxf(a.z2[2 * s][3], 0.f));
        ah2[s][2] = pack_bf16(fmaxf(a.z2[2 * s + 1][0], 0.f), fmaxf(a.z2[2 * s + 1][1], 0.f));
        ah2[s][3] = pack_bf16(fmaxf(a.z2[2 * s + 1][2], 0.f), fmaxf(a.z2[2 * s + 1][3], 0.f));
    }
    float o[4] = {r.b3, 0.f, r.b3, 0.f};
    mma_bf16(o, ah2[0], r.w3[0], o);
    mma_bf16(o, ah2[1], r.w3[1], o);
    a.y[0] = o[0];  // row g, column 0 (threads with t == 0)
    a.y[1] = o[2];  // row g + 8
}

}  // namespace

// ---------------------------------------------------------------- features
// Seven features of each 32-body group (sorted order), from the bodies, the
// last step's |a| and the tree: see bh_group_features() in bh_api.h.
__global__ void __launch_bounds__(256)
k_group_features(const float4* __restrict__ pos, const float* __restrict__ aMag, const uint64_t* __restrict__ keys,
                 int n, int bits, const DevBox* __restrict__ box, const DevRoot* __restrict__ root, float G,
                 float* __restrict__ feat) {
    const int lane = threadIdx.x & 31;
    const int g = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int groups = (n + 31) >> 5;
    if (g >= groups) return;
    const int b = g * 32 + lane;
    const bool valid = b < n;
    const float4 p = valid ? pos[b] : make_float4(0.f, 0.f, 0.f, 0.f);
    const float am = valid ? aMag[b] : 0.f;
    float lo[3] = {valid ? p.x : INFINITY, valid ? p.y : INFINITY, valid ? p.z : INFINITY};
    float hi[3] = {valid ? p.x : -INFINITY, valid ? p.y : -INFINITY, valid ? p.z : -INFINITY};
    float aMin = valid ? am : INFINITY, aMax = valid ? am : 0.f, aSum = am, mSum = valid ? p.w : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; k++) {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
        aMin = fminf(aMin, __shfl_xor_sync(0xffffffffu, aMin, o));
        aMax = fmaxf(aMax, __shfl_xor_sync(0xffffffffu, aMax, o));
        aSum += __shfl_xor_sync(0xffffffffu, aSum, o);
        mSum += __shfl_xor_sync(0xffffffffu, mSum, o);
    }
    if (lane != 0) return;
    const int cnt = (n - g * 32 < 32) ? n - g * 32 : 32;
    const float ext = fmaxf(box->extent, 1e-30f);
    // the system's centre of mass and total mass from the FP64 root reduction
    const float mTot = (float)root->mass;
    const float hx = 0.5f * (hi[0] - lo[0]), hy = 0.5f * (hi[1] - lo[1]), hz = 0.5f * (hi[2] - lo[2]);
    const float R = sqrtf(hx * hx + hy * hy + hz * hz);
    const float cx = (float)((double)(0.5f * (lo[0] + hi[0])) - root->com[0]),
                cy = (float)((double)(0.5f * (lo[1] + hi[1])) - root->com[1]),
                cz = (float)((double)(0.5f * (lo[2] + hi[2])) - root->com[2]);
    const float D = sqrtf(cx * cx + cy * cy + cz * cz);
    const float aMean = aSum / cnt;
    const float aScale = G * fmaxf(mTot, 1e-30f) / (ext * ext);
    const uint64_t x = keys[g * 32] ^ keys[g * 32 + cnt - 1];
    const int depth = (x == 0ull) ? bits : bits - 1 - (63 - __clzll((long long)x)) / 3;
    const float vol = fmaxf(8.f * hx * hy * hz, 1e-30f * ext * ext * ext);
    const float hmin = fminf(hx, fminf(hy, hz)), hmax = fmaxf(hx, fmaxf(hy, hz));
    float* f = feat + (size_t)g * 7;
    f[0] = log10f(R / ext + 1e-7f);                                       // group radius
    f[1] = log10f(aMean / aScale + 1e-12f);                               // force scale
    f[2] = log10f((aMax + 1e-30f) / (aMin + 1e-30f));                     // force spread in the group
    f[3] = log10f(D / ext + 1e-4f);                                       // distance from the centre
    f[4] = (float)depth / (float)bits;                                    // tree depth of the group
    f[5] = log10f(mSum / fmaxf(mTot, 1e-30f) * ext * ext * ext / vol);   // local density
    f[6] = log10f((hmin + 1e-7f * ext) / (hmax + 1e-7f * ext));           // flatness
}

// --------------------------------------------------------------- inference
// Per group, evaluate the MLP at the kMacCandidates budgets and choose.
__global__ void __launch_bounds__(128)
k_mac_select(const float* __restrict__ P, const float* __restrict__ feat, int groups, float logTarget, float thetaCap,
             float2* __restrict__ groupParam) {
    MlpRegs r;
    load_mlp(r, P);
    const int lane = threadIdx.x & 31, g8 = lane >> 2, t = lane & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    // a 16-row tile = 2 groups x 8 candidates: row = 8 * (group in tile) + candidate
    for (int tile = warp; tile * 2 < groups; tile += nwarps) {
        const int gA = tile * 2, gB = gA + 1;
        // row g8 -> group gA, candidate g8; row g8 + 8 -> group gB, candidate g8
        float x0[2], x1[2];
        auto feature = [&](int grp, int cand, int f) -> float {
            if (grp >= groups) return 0.f;
            return f == 0 ? log10f(ldexpf(kMacAlpha0, cand)) : feat[(size_t)grp * 7 + f - 1];
        };
        x0[0] = feature(gA, g8, 2 * t);
        x0[1] = feature(gA, g8, 2 * t + 1);
        x1[0] = feature(gB, g8, 2 * t);
        x1[1] = feature(gB, g8, 2 * t + 1);
        Acts a;
        forward(r, x0, x1, a);
        // lanes with t == 0 hold rows g8 (group A) and g8 + 8 (group B)
        const float yA = __shfl_sync(0xffffffffu, a.y[0], (lane & ~3));
        const float yB = __shfl_sync(0xffffffffu, a.y[1], (lane & ~3));
        // lane (4c + t), t == 0 carries candidate c: ballots over candidates
        const bool finiteA = isfinite(yA), finiteB = isfinite(yB);
        const unsigned okA = __ballot_sync(0xffffffffu, t == 0 && finiteA && yA <= logTarget);
        const unsigned okB = __ballot_sync(0xffffffffu, t == 0 && finiteB && yB <= logTarget);
        const unsigned badA = __ballot_sync(0xffffffffu, t == 0 && !finiteA);
        const unsigned badB = __ballot_sync(0xffffffffu, t == 0 && !finiteB);
        // largest budget that meets the target (uniform), its prediction and the next one's
        const int cA = okA ? (31 - __clz(okA)) >> 2 : 0, cB = okB ? (31 - __clz(okB)) >> 2 : 0;
        const float ycA = __shfl_sync(0xffffffffu, yA, 4 * cA), ycB = __shfl_sync(0xffffffffu, yB, 4 * cB);
        const float ynA = __shfl_sync(0xffffffffu, yA, cA < 7 ? 4 * cA + 4 : 28);
        const float ynB = __shfl_sync(0xffffffffu, yB, cB < 7 ? 4 * cB + 4 : 28);
        if (lane == 0) {
            auto pick = [&](unsigned ok, unsigned bad, int c, float yc, float yn) -> float2 {
                if (bad) return make_float2(0.5f, 1e30f);  // fallback: the fixed-theta test alone
                float alpha = ldexpf(kMacAlpha0, c);
                // c meets the target and c+1 does not: interpolate in log alpha
                if (ok && c < BH_MAC_CANDIDATES - 1 && yn > logTarget && yn > yc) {
                    const float frac = __fdiv_rn(__fsub_rn(logTarget, yc), __fsub_rn(yn, yc));
                    alpha = __fmul_rn(alpha, exp2f(frac));
                }
                return make_float2(thetaCap, alpha);
            };
            groupParam[gA] = pick(okA, badA, cA, ycA, ynA);
            if (gB < groups) groupParam[gB] = pick(okB, badB, cB, ycB, ynB);
        }
    }
}

// ---------------------------------------------------------------- training
// One pass over `rows` training rows (8 inputs, 1 target each): loss =
// mean squared error; gradients of the trained parameters are accumulated
// into grad (FP32, zeroed by the caller); lossOut += sum of squared errors.
// Forward and the backward product through W2 use the tensor cores (BF16 in,
// FP32 out); weight gradients are FP32 sums over the rows.
__global__ void __launch_bounds__(128)
k_mlp_train(const float* __restrict__ P, const float* __restrict__ X, const float* __restrict__ Y, int rows,
            float* __restrict__ grad, float* __restrict__ lossOut) {
    __shared__ float sG[MLP_TRAINED];
    __shared__ float sAct[4][16][32 * 3 + 8 + 1];  // per warp: bf16-rounded x, h1, h2; dh1; dy
    for (int i = threadIdx.x; i < MLP_TRAINED; i += blockDim.x) sG[i] = 0.f;
    __syncthreads();
    MlpRegs r;
    load_mlp(r, P);
    const int lane = threadIdx.x & 31, g8 = lane >> 2, t = lane & 3, w = threadIdx.x >> 5;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    float (*S)[32 * 3 + 8 + 1] = sAct[w];  // S[row][...]: x 0..7 | h1 8..39 | h2 40..71 | dh1 72..103 | dy 104
    const int XH1 = 8, XH2 = 40, XDH1 = 72, XDY = 104;
    float lossAcc = 0.f;
    for (int tile = warp; tile * 16 < rows; tile += nwarps) {
        const int r0 = tile * 16;
        float x0[2], x1[2];
        auto in = [&](int row, int f) { return row < rows ? X[(size_t)row * 8 + f] : 0.f; };
        x0[0] = in(r0 + g8, 2 * t);
        x0[1] = in(r0 + g8, 2 * t + 1);
        x1[0] = in(r0 + g8 + 8, 2 * t);
        x1[1] = in(r0 + g8 + 8, 2 * t + 1);
        Acts a;
        forward(r, x0, x1, a);
        // normalised, bf16-rounded inputs and activations (what the MMAs saw)
        S[g8][2 * t] = bf16_round((x0[0] - r.mu[0]) * r.sig[0]);
        S[g8][2 * t + 1] = bf16_round((x0[1] - r.mu[1]) * r.sig[1]);
        S[g8 + 8][2 * t] = bf16_round((x1[0] - r.mu[0]) * r.sig[0]);
        S[g8 + 8][2 * t + 1] = bf16_round((x1[1] - r.mu[1]) * r.sig[1]);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = 8 * j + 2 * t;
            S[g8][XH1 + c] = bf16_round(fmaxf(a.z1[j][0], 0.f));
            S[g8][XH1 + c + 1] = bf16_round(fmaxf(a.z1[j][1], 0.f));
            S[g8 + 8][XH1 + c] = bf16_round(fmaxf(a.z1[j][2], 0.f));
            S[g8 + 8][XH1 + c + 1] = bf16_round(fmaxf(a.z1[j][3], 0.f));
            S[g8][XH2 + c] = bf16_round(fmaxf(a.z2[j][0], 0.f));
            S[g8][XH2 + c + 1] = bf16_round(fmaxf(a.z2[j][1], 0.f));
            S[g8 + 8][XH2 + c] = bf16_round(fmaxf(a.z2[j][2], 0.f));
            S[g8 + 8][XH2 + c + 1] = bf16_round(fmaxf(a.z2[j][3], 0.f));
        }
        // dL/dy = 2 (y - target) / rows (rows past the end contribute nothing)
        if (t == 0) {
            const int ra = r0 + g8, rb = r0 + g8 + 8;
            const float da = ra < rows ? a.y[0] - Y[ra] : 0.f;
            const float db = rb < rows ? a.y[1] - Y[rb] : 0.f;
            lossAcc += da * da + db * db;
            S[g8][XDY] = 2.f * da / rows;
            S[g8 + 8][XDY] = 2.f * db / rows;
        }
        __syncwarp();
        // dh2 = dy * W3 * relu'(z2), as the A operand (bf16) of dh1 = dh2 W2^T
        float dyA = S[g8][XDY], dyB = S[g8 + 8][XDY];
        uint32_t ad[2][4];
        float dh2[4][4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int c = 8 * j + 2 * t;
            const float w0 = bf16_round(P[MLP_W3 + c]), w1 = bf16_round(P[MLP_W3 + c + 1]);
            dh2[j][0] = a.z2[j][0] > 0.f ? dyA * w0 : 0.f;
            dh2[j][1] = a.z2[j][1] > 0.f ? dyA * w1 : 0.f;
            dh2[j][2] = a.z2[j][2] > 0.f ? dyB * w0 : 0.f;
            dh2[j][3] = a.z2[j][3] > 0.f ? dyB * w1 : 0.f;
        }
#pragma unroll
        for (int s2 = 0; s2 < 2; s2++) {
            ad[s2][0] = pack_bf16(dh2[2 * s2][0], dh2[2 * s2][1]);
            ad[s2][1] = pack_bf16(dh2[2 * s2][2], dh2[2 * s2][3]);
            ad[s2][2] = pack_bf16(dh2[2 * s2 + 1][0], dh2[2 * s2 + 1][1]);
            ad[s2][3] = pack_bf16(dh2[2 * s2 + 1][2], dh2[2 * s2 + 1][3]);
        }
        // dh1[r][i] = sum_j dh2[r][j] W2[i][j] * relu'(z1[r][i]); B[k=j][n=i] = W2[i][j]
#pragma unroll
        for (int j = 0; j < 4; j++) {  // n-tile over i
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int s2 = 0; s2 < 2; s2++) {  // k-step over j
                uint32_t bw[2];
                const int i = 8 * j + g8;
                const int k0 = 16 * s2 + 2 * t;
                bw[0] = pack_bf16(P[MLP_W2 + i * 32 + k0], P[MLP_W2 + i * 32 + k0 + 1]);
                bw[1] = pack_bf16(P[MLP_W2 + i * 32 + k0 + 8], P[MLP_W2 + i * 32 + k0 + 9]);
                mma_bf16(acc, ad[s2], bw, acc);
            }
            const int c = 8 * j + 2 * t;
            S[g8][XDH1 + c] = a.z1[j][0] > 0.f ? acc[0] : 0.f;
            S[g8][XDH1 + c + 1] = a.z1[j][1] > 0.f ? acc[1] : 0.f;
            S[g8 + 8][XDH1 + c] = a.z1[j][2] > 0.f ? acc[2] : 0.f;
            S[g8 + 8][XDH1 + c + 1] = a.z1[j][3] > 0.f ? acc[3] : 0.f;
        }
        __syncwarp();
        // weight and bias gradients, FP32 sums over the 16 rows; each lane owns
        // a slice of the parameters
        for (int idx = lane; idx < MLP_TRAINED; idx += 32) {
            float gsum = 0.f;
            if (idx < MLP_B1) {  // W1[f][i]: x[r][f] * dh1[r][i]
                const int f = idx / 32, i = idx % 32;
                for (int rr = 0; rr < 16; rr++) gsum += S[rr][f] * S[rr][XDH1 + i];
            } else if (idx < MLP_W2) {  // b1[i]
                const int i = idx - MLP_B1;
                for (int rr = 0; rr < 16; rr++) gsum += S[rr][XDH1 + i];
            } else if (idx < MLP_B2) {  // W2[i][j]: h1[r][i] * dh2[r][j]
                const int i = (idx - MLP_W2) / 32, j = (idx - MLP_W2) % 32;
                const float w3 = bf16_round(P[MLP_W3 + j]);
                for (int rr = 0; rr < 16; rr++) {
                    const float h2 = S[rr][XH2 + j];
                    const float d2 = h2 > 0.f ? S[rr][XDY] * w3 : 0.f;
                    gsum += S[rr][XH1 + i] * d2;
                }
            } else if (idx < MLP_W3) {  // b2[j]
                const int j = idx - MLP_B2;
                const float w3 = bf16_round(P[MLP_W3 + j]);
                for (int rr = 0; rr < 16; rr++) gsum += S[rr][XH2 + j] > 0.f ? S[rr][XDY] * w3 : 0.f;
            } else if (idx < MLP_B3) {  // W3[j]: h2[r][j] * dy[r]
                const int j = idx - MLP_W3;
                for (int rr = 0; rr < 16; rr++) gsum += S[rr][XH2 + j] * S[rr][XDY];
            } else {  // b3
                for (int rr = 0; rr < 16; rr++) gsum += S[rr][XDY];
            }
            atomicAdd(&sG[idx], gsum);
        }
        __syncwarp();
    }
    // loss: reduce over lanes, one atomic per warp
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, o);
    if (lane == 0) atomicAdd(lossOut, lossAcc);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_TRAINED; i += blockDim.x)
        if (sG[i] != 0.f) atomicAdd(&grad[i], sG[i]);
}

// Adam on the trained parameters (FP32 master weights).
__global__ void k_adam(float* P, const float* grad, float* m, float* v, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_TRAINED) return;
    const float g = grad[i];
    m[i] = b1 * m[i] + (1.f - b1) * g;
    v[i] = b2 * v[i] + (1.f - b2) * g * g;
    P[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
}

// ------------------------------------------------------------------ C ABI
extern "C" int bh_mlp_train_epoch(float* params, const float* X, const float* Y, int rows, float* grad, float* adamM,
                                  float* adamV, int batch, int* step, float lr, float* lossOut, cudaStream_t s) {
    if (!params || !X || !Y || rows <= 0 || !grad || !adamM || !adamV || batch <= 0 || !step || !lossOut)
        return BH_ERR_INVALID;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int r0 = 0; r0 < rows; r0 += batch) {
        const int nb = (rows - r0 < batch) ? rows - r0 : batch;
        BH_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(float) * MLP_TRAINED, s));
        const int tiles = (nb + 15) / 16;
        int blocks = (tiles + 3) / 4;
        blocks = blocks > 4 * bh_sm_count() ? 4 * bh_sm_count() : blocks;
        k_mlp_train<<<blocks, 128, 0, s>>>(params, X + (size_t)r0 * 8, Y + r0, nb, grad, lossOut);
        BH_CUDA_TRY(cudaGetLastError());
        const int t = ++(*step);
        const float c1 = 1.f - powf(b1, (float)t), c2 = 1.f - powf(b2, (float)t);
        k_adam<<<(MLP_TRAINED + 255) / 256, 256, 0, s>>>(params, grad, adamM, adamV, lr, b1, b2, eps, c1, c2);
        BH_CUDA_TRY(cudaGetLastError());
    }
    return BH_OK;
}

extern "C" int bh_mlp_loss_grad(const float* params, const float* X, const float* Y, int rows, float* grad,
                                float* lossOut, cudaStream_t s) {
    if (!params || !X || !Y || rows <= 0 || !grad || !lossOut) return BH_ERR_INVALID;
    BH_CUDA_TRY(cudaMemsetAsync(grad, 0, sizeof(float) * MLP_TRAINED, s));
    BH_CUDA_TRY(cudaMemsetAsync(lossOut, 0, sizeof(float), s));
    const int tiles = (rows + 15) / 16;
    int blocks = (tiles + 3) / 4;
    blocks = blocks > 4 * bh_sm_count() ? 4 * bh_sm_count() : blocks;
    k_mlp_train<<<blocks, 128, 0, s>>>(params, X, Y, rows, grad, lossOut);
    BH_CUDA_TRY(cudaGetLastError());
    return BH_OK;
}

// Raw forward pass: Y[r] = MLP(X[r]) for `rows` rows of 8 inputs (a test and
// tooling entry; the selection kernel uses the same forward()).
__global__ void __launch_bounds__(128) k_mlp_forward(const float* P, const float* X, int rows, float* Y) {
    MlpRegs r;
    load_mlp(r, P);
    const int lane = threadIdx.x & 31, g8 = lane >> 2, t = lane & 3;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int tile = warp; tile * 16 < rows; tile += nwarps) {
        const int r0 = tile * 16;
        auto in = [&](int row, int f) { return row < rows ? X[(size_t)row * 8 + f] : 0.f; };
        const float x0[2] = {in(r0 + g8, 2 * t), in(r0 + g8, 2 * t + 1)};
        const float x1[2] = {in(r0 + g8 + 8, 2 * t), in(r0 + g8 + 8, 2 * t + 1)};
        Acts a;
        forward(r, x0, x1, a);
        if (t == 0) {
            if (r0 + g8 < rows) Y[r0 + g8] = a.y[0];
            if (r0 + g8 + 8 < rows) Y[r0 + g8 + 8] = a.y[1];
        }
    }
}

extern "C" int bh_mlp_forward(const float* params, const float* X, int rows, float* Y, cudaStream_t s) {
    if (!params || !X || !Y || rows <= 0) return BH_ERR_INVALID;
    const int tiles = (rows + 15) / 16;
    int blocks = (tiles + 3) / 4;
    blocks = blocks > 4 * bh_sm_count() ? 4 * bh_sm_count() : blocks;
    k_mlp_forward<<<blocks, 128, 0, s>>>(params, X, rows, Y);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? BH_OK : bh_note_cuda_error(e);
}

// ---------------------------------------------------------- engine hooks
cudaError_t bh_launch_group_features(const float4* pos, const float* aMag, const uint64_t* keys, int n, int bits,
                                     const DevBox* box, const DevRoot* root, float G, float* feat, cudaStream_t s) {
    const int groups = (n + 31) / 32;
    k_group_features<<<(groups + 7) / 8, 256, 0, s>>>(pos, aMag, keys, n, bits, box, root, G, feat);
    return cudaGetLastError();
}

cudaError_t bh_launch_mac_select(const float* params, const float* feat, int groups, float logTarget, float thetaCap,
                                 float2* groupParam, cudaStream_t s) {
    const int tiles = (groups + 1) / 2;
    int blocks = (tiles + 3) / 4;
    blocks = blocks > 8 * bh_sm_count() ? 8 * bh_sm_count() : blocks;
    blocks = blocks < 1 ? 1 : blocks;
    k_mac_select<<<blocks, 128, 0, s>>>(params, feat, groups, logTarget, thetaCap, groupParam);
    return cudaGetLastError();
}

extern "C" int bh_mac_ladder(float alphas[BH_MAC_CANDIDATES]) {
    if (!alphas) return BH_ERR_INVALID;
    for (int c = 0; c < BH_MAC_CANDIDATES; c++) alphas[c] = ldexpf(kMacAlpha0, c);
    return BH_OK;
}
