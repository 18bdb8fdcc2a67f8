/*
 * bh_oracle.c — CPU oracle for the Barnes-Hut step pipeline.
 *
 * TEST INFRASTRUCTURE ONLY (see bh_oracle.h).  A restatement of the
 * reference's algorithm in plain C; every function names the reference lines
 * it follows.  Build with -ffp-contract=off (no implicit multiply-add
 * fusion): fmaf() appears exactly where nvcc fuses in the reference's device
 * code, everything else is a separately rounded FP32 operation.
 */
#include "bh_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ bbox */
/* tree.cu:414-490: min/max of x, y, z over all bodies.  fminf/fmaxf are
 * exact, so the reduction order does not matter. */
void orc_bbox(const float4* pos, int n, float mn[3], float mx[3]) {
    mn[0] = mn[1] = mn[2] = INFINITY;
    mx[0] = mx[1] = mx[2] = -INFINITY;
    for (int i = 0; i < n; i++) {
        mn[0] = fminf(mn[0], pos[i].x); mx[0] = fmaxf(mx[0], pos[i].x);
        mn[1] = fminf(mn[1], pos[i].y); mx[1] = fmaxf(mx[1], pos[i].y);
        mn[2] = fminf(mn[2], pos[i].z); mx[2] = fmaxf(mx[2], pos[i].z);
    }
}

/* basicGravity.cu:90-112 (bits = 21 there: scale = 2097151 / extent). */
void orc_world_box(const float mn[3], const float mx[3], int bits, worldBox* out) {
    float width = mx[0] - mn[0];
    float height = mx[1] - mn[1];
    float depth = mx[2] - mn[2];
    float extent = fmaxf(width, fmaxf(height, depth));
    uint32_t biggest = (1u << bits) - 1u;
    out->minX = mn[0];
    out->minY = mn[1];
    out->minZ = mn[2];
    out->extent = extent;
    out->scale = (float)biggest / extent;
}

/* --------------------------------------------------------------- Morton */
/* tree.cu:332-340 spreads 21 bits with magic masks; for any bit count the
 * result is: bit k of v moves to bit 3k.  Written as a loop so the oracle
 * does not depend on the mask constants being right. */
uint64_t orc_expand_bits(uint64_t v, int bits) {
    uint64_t out = 0;
    v &= (bits >= 64) ? ~0ull : ((1ull << bits) - 1ull); /* tree.cu:333 masks to 21 bits */
    for (int k = 0; k < bits; k++) out |= ((v >> k) & 1ull) << (3 * k);
    return out;
}

/* tree.cu:343-367: grid coordinate = (uint32)((p - min) * scale), key =
 * E(x) << 2 | E(y) << 1 | E(z); originalIndex[i] = i. */
void orc_morton_encode(const float4* pos, int n, worldBox box, int bits, uint64_t* keys,
                       uint32_t* idx) {
    for (int i = 0; i < n; i++) {
        uint32_t x = (uint32_t)((pos[i].x - box.minX) * box.scale);
        uint32_t y = (uint32_t)((pos[i].y - box.minY) * box.scale);
        uint32_t z = (uint32_t)((pos[i].z - box.minZ) * box.scale);
        keys[i] = (orc_expand_bits(x, bits) << 2) | (orc_expand_bits(y, bits) << 1) |
                  orc_expand_bits(z, bits);
        idx[i] = (uint32_t)i;
    }
}

/* ----------------------------------------------------------------- sort */
/* sorting.cu:65-79 calls a stable radix sort over all 64 key bits.  Any
 * stable ascending sort gives the same permutation; this is an LSD counting
 * sort with 16-bit digits. */
void orc_sort_pairs(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut,
                    uint32_t* valsOut, int n) {
    uint64_t* ka = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    uint32_t* va = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    size_t* count = (size_t*)malloc(sizeof(size_t) * 65536);
    memcpy(keysOut, keysIn, sizeof(uint64_t) * (size_t)n);
    memcpy(valsOut, valsIn, sizeof(uint32_t) * (size_t)n);
    for (int shift = 0; shift < 64; shift += 16) {
        memset(count, 0, sizeof(size_t) * 65536);
        for (int i = 0; i < n; i++) count[(keysOut[i] >> shift) & 0xffff]++;
        size_t run = 0;
        for (int d = 0; d < 65536; d++) { size_t c = count[d]; count[d] = run; run += c; }
        for (int i = 0; i < n; i++) {
            size_t dst = count[(keysOut[i] >> shift) & 0xffff]++;
            ka[dst] = keysOut[i];
            va[dst] = valsOut[i];
        }
        memcpy(keysOut, ka, sizeof(uint64_t) * (size_t)n);
        memcpy(valsOut, va, sizeof(uint32_t) * (size_t)n);
    }
    free(ka); free(va); free(count);
}

/* sorting.cu:99-107. */
void orc_reorder(const float4* posIn, const float3* velIn, const uint32_t* idx, float4* posOut,
                 float3* velOut, int n) {
    for (int i = 0; i < n; i++) {
        posOut[i] = posIn[idx[i]];
        velOut[i] = velIn[idx[i]];
    }
}

/* ----------------------------------------------------------------- tree */
/* tree.cu:23-26: level-L path prefix.  With 3*bits key bits the reference's
 * shift 63 - 3L becomes 3*(bits - L). */
static inline uint64_t level_prefix(uint64_t key, int bits, int level) {
    int shift = 3 * (bits - level);
    return shift >= 64 ? 0 : (key >> shift);
}

/* basicGravity.cu:116-325 (levels 1..21, host loop) with the kernels
 * identifyNodesAtLevel tree.cu:50-78, prefixSum tree.cu:286-302,
 * createNodes tree.cu:205-235, updateTreeParticles tree.cu:181-203 and
 * updateTreeMass tree.cu:89-179, each restated as a sequential loop. */
int orc_build_tree(const uint64_t* keys, const float4* pos, int n, int bits, node* nodes,
                   int maxNodes, int* levelOffsets, int* levelCount, int* deepestLevel) {
    uint32_t* flags = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
    uint32_t* prevFlags = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
    uint32_t* offsets = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
    uint32_t* prevOffsets = (uint32_t*)calloc((size_t)n, sizeof(uint32_t));
    int status = 0;

    for (int l = 0; l < 23; l++) { levelOffsets[l] = 0; levelCount[l] = 0; }

    /* root node (basicGravity.cu:158-169); its parentIndex is never set by
     * the reference, -1 here. */
    memset(&nodes[0], 0, sizeof(node));
    nodes[0].nodePathFromRoot = 0;
    nodes[0].parentIndex = -1;
    nodes[0].treeLevel = 0;
    nodes[0].firstParticleIndex = 0;
    nodes[0].particleCount = n;
    for (int c = 0; c < 8; c++) nodes[0].child[c] = -1;

    int arrayLevelOffset = 1, prevArrayLevelOffset = 0, deepest = 0;
    levelOffsets[0] = 0;
    levelCount[0] = 1;

    for (int level = 1; level <= bits; level++) {
        /* identifyNodesAtLevel (tree.cu:50-78) */
        for (int i = 0; i < n; i++) {
            uint64_t cur = level_prefix(keys[i], bits, level);
            uint64_t par = level_prefix(keys[i], bits, level - 1);
            int sameParentLeft = (i > 0) && (par == level_prefix(keys[i - 1], bits, level - 1));
            int sameParentRight = (i < n - 1) && (par == level_prefix(keys[i + 1], bits, level - 1));
            int sameNodeLeft = (i > 0) && (cur == level_prefix(keys[i - 1], bits, level));
            if (!sameParentLeft && !sameParentRight) flags[i] = 0;
            else if (!sameNodeLeft) flags[i] = 1;
            else flags[i] = 0;
        }
        /* exclusive prefix sum (tree.cu:286-302) */
        uint32_t run = 0;
        for (int i = 0; i < n; i++) { offsets[i] = run; run += flags[i]; }
        /* createNodes (tree.cu:205-235) */
        for (int i = 0; i < n; i++) {
            if (!flags[i]) continue;
            uint64_t path = level_prefix(keys[i], bits, level);
            int idx = (int)offsets[i] + arrayLevelOffset;
            if (idx >= maxNodes) continue;
            node* nd = &nodes[idx];
            memset(nd, 0, sizeof(node));
            nd->nodePathFromRoot = path;
            nd->treeLevel = level;
            nd->firstParticleIndex = i;
            for (int c = 0; c < 8; c++) nd->child[c] = -1;
            int parent = (level == 1) ? 0
                                      : prevArrayLevelOffset + (int)prevOffsets[i] + (int)prevFlags[i] - 1;
            nodes[parent].child[path & 7] = idx;
            nd->parentIndex = parent;
        }
        int nodeCount = (int)(flags[n - 1] + offsets[n - 1]);
        if (nodeCount == 0) { /* basicGravity.cu:276-279 */
            levelCount[level] = 0;
            levelOffsets[level] = arrayLevelOffset;
            break;
        }
        if (nodeCount + arrayLevelOffset > maxNodes) { status = -1; break; } /* :282 */
        /* updateTreeParticles (tree.cu:181-203) */
        for (int t = 0; t < nodeCount; t++) {
            int ni = arrayLevelOffset + t;
            int parent = nodes[ni].parentIndex;
            int nextIsSibling = (t + 1 < nodeCount) && (nodes[ni + 1].parentIndex == parent);
            int end = nextIsSibling ? nodes[ni + 1].firstParticleIndex
                                    : nodes[parent].firstParticleIndex + nodes[parent].particleCount;
            nodes[ni].particleCount = end - nodes[ni].firstParticleIndex;
        }
        prevArrayLevelOffset = arrayLevelOffset;
        levelOffsets[level] = arrayLevelOffset;
        arrayLevelOffset += nodeCount;
        levelCount[level] = nodeCount;
        uint32_t* t;
        t = prevOffsets; prevOffsets = offsets; offsets = t;
        t = prevFlags; prevFlags = flags; flags = t;
        deepest++;
    }
    /* a full-depth tree never meets an empty level: entry deepest+1 then
     * marks the end of the array */
    if (status == 0 && deepest == bits) levelOffsets[bits + 1] = arrayLevelOffset;

    if (status == 0) {
        /* updateTreeMass, deepest level first (basicGravity.cu:317-319,
         * tree.cu:89-179) */
        for (int level = deepest; level >= 0; level--) {
            for (int t = 0; t < levelCount[level]; t++) {
                node* nd = &nodes[levelOffsets[level] + t];
                int leaf = 1;
                for (int c = 0; c < 8; c++) if (nd->child[c] != -1) { leaf = 0; break; }
                float4 m = {0.f, 0.f, 0.f, 0.f};
                if (leaf) {
                    float wx = 0.f, wy = 0.f, wz = 0.f, total = 0.f;
                    for (int k = 0; k < nd->particleCount; k++) {
                        const float4 p = pos[nd->firstParticleIndex + k];
                        wx = fmaf(p.x, p.w, wx); /* x*w + acc, fused by nvcc */
                        wy = fmaf(p.y, p.w, wy);
                        wz = fmaf(p.z, p.w, wz);
                        total = total + p.w;
                    }
                    if (total > 0.0f) { m.x = wx / total; m.y = wy / total; m.z = wz / total; m.w = total; }
                } else {
                    float4 acc = {0.f, 0.f, 0.f, 0.f};
                    for (int c = 0; c < 8; c++)
                        if (nd->child[c] != -1) acc.w = acc.w + nodes[nd->child[c]].massData.w;
                    for (int c = 0; c < 8; c++) {
                        if (nd->child[c] == -1) continue;
                        float4 cm = nodes[nd->child[c]].massData;
                        acc.x = fmaf(cm.x, cm.w, acc.x);
                        acc.y = fmaf(cm.y, cm.w, acc.y);
                        acc.z = fmaf(cm.z, cm.w, acc.z);
                    }
                    if (acc.w > 0.0f) { m.x = acc.x / acc.w; m.y = acc.y / acc.w; m.z = acc.z / acc.w; m.w = acc.w; }
                }
                nd->massData = m;
            }
        }
    }
    *deepestLevel = deepest;
    free(flags); free(prevFlags); free(offsets); free(prevOffsets);
    return status == 0 ? arrayLevelOffset : -1;
}

/* ----------------------------------------------------------------- walk */
/* tree.cu:501-530: size = (x-extent) / pow(2, level), evaluated in double
 * (pow returns double) and rounded to float on return. */
static inline float node_size(float extX, int level) {
    return (float)((double)extX / ldexp(1.0, level));
}

static inline float dist_sq(float dx, float dy, float dz, int order) {
    switch (order) {
    case ORC_D2_REF: return fmaf(dz, dz, fmaf(dx, dx, dy * dy));
    case ORC_D2_ALT: return fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    default: return (dx * dx + dy * dy) + dz * dz;
    }
}

static inline int is_leaf(const node* nd) { /* tree.cu:532-545 + :627 */
    if (nd->particleCount <= 1) return 1;
    for (int c = 0; c < 8; c++) if (nd->child[c] != -1) return 0;
    return 1;
}

#define ORC_STACK 256

/* The walk runs on the host cores for the tests and for the CPU baselines.
 * Its per-lane loops are written without branches so that the compiler
 * vectorises them (every operation is an IEEE-rounded FP32 operation, the
 * same per lane whether it runs in a SIMD register or not: the results are
 * bit-identical to a scalar evaluation); an AVX2+FMA clone is picked at run
 * time where the host has it (fmaf then inlines to one instruction). */
#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__)
#define ORC_SIMD_CLONES __attribute__((target_clones("arch=x86-64-v3", "default")))
#else
#define ORC_SIMD_CLONES
#endif

/* Lanes l < width of the group: does any valid lane want node (c, sizeSq)
 * opened (tree.cu:610-634), with the relative criterion when aMag is given. */
static inline int lanes_open(const float* px, const float* py, const float* pz, const float* am, const int* valid,
                             int width, float4 c, float sizeSq, float thetaSq, float kA, int relative, int d2Order) {
    int any = 0;
    for (int l = 0; l < width; l++) {
        float dx = px[l] - c.x, dy = py[l] - c.y, dz = pz[l] - c.z;
        float d2 = dist_sq(dx, dy, dz, d2Order);
        int o = !(sizeSq < thetaSq * d2);
        /* relative criterion: also open when M s^2 > (alpha / G) |a_b| d^4 */
        if (relative) o |= c.w * sizeSq > kA * am[l] * (d2 * d2);
        any |= o & valid[l];
    }
    return any;
}

/* tree.cu:660-668: every lane accumulates the monopole of (c, m). */
static inline void lanes_accumulate(const float* px, const float* py, const float* pz, float* ax, float* ay,
                                    float* az, int width, float4 c, float eps2, float G, int d2Order) {
    for (int l = 0; l < width; l++) {
        float dx = px[l] - c.x, dy = py[l] - c.y, dz = pz[l] - c.z;
        float d2 = dist_sq(dx, dy, dz, d2Order);
        float accelMag = -(G * c.w) / (d2 + eps2);
        float dist = sqrtf(d2 + eps2);
        ax[l] = fmaf(accelMag, dx / dist, ax[l]);
        ay[l] = fmaf(accelMag, dy / dist, ay[l]);
        az[l] = fmaf(accelMag, dz / dist, az[l]);
    }
}

/* One group of the reference walk (tree.cu:562-676).  If acc is NULL only
 * the accepted-node count is returned (interaction-list length).  Lanes past
 * the last body compute on zeros and are never stored. */
/* leafSize > 1 (an extension, not in the reference): an opened node with at
 * most leafSize bodies contributes its bodies as single-body leaves instead
 * of its children. */
ORC_SIMD_CLONES
static long long walk_group(const float4* pos, int n, const node* nodes, float extX, float eps2,
                            float G, float theta, int first, int width, int d2Order, float3* acc,
                            const float* aMag, float kA, int leafSize) {
    int stack[ORC_STACK];
    int top = -1;
    float px[64], py[64], pz[64], ax[64], ay[64], az[64], am[64];
    int valid[64];
    for (int l = 0; l < width; l++) {
        int b = first + l;
        valid[l] = b < n;
        px[l] = valid[l] ? pos[b].x : 0.f;
        py[l] = valid[l] ? pos[b].y : 0.f;
        pz[l] = valid[l] ? pos[b].z : 0.f;
        am[l] = (valid[l] && aMag) ? aMag[b] : 0.f;
        ax[l] = ay[l] = az[l] = 0.f;
    }
    int nvalid = 0;
    for (int l = 0; l < width; l++) nvalid += valid[l];
    const float thetaSq = theta * theta;
    const int relative = aMag != NULL;
    long long accepted = 0;

    for (int c = 0; c < 8; c++) /* tree.cu:595-601 */
        if (nodes[0].child[c] != -1) stack[++top] = nodes[0].child[c];

    while (top >= 0) { /* tree.cu:603-670 */
        const int entry = stack[top];
        top--;
        if (entry < -1) { /* a body below an opened bucket: a one-body leaf */
            accepted++;
            if (acc) lanes_accumulate(px, py, pz, ax, ay, az, width, pos[-entry - 2], eps2, G, d2Order);
            continue;
        }
        const node* nd = &nodes[entry];
        const float size = node_size(extX, nd->treeLevel);
        const float sizeSq = size * size;
        const int descend = !is_leaf(nd) && lanes_open(px, py, pz, am, valid, width, nd->massData, sizeSq,
                                                       thetaSq, kA, relative, d2Order);
        if (descend && nd->particleCount <= leafSize) { /* bucket: its bodies */
            for (int b = 0; b < nd->particleCount && top + 1 < ORC_STACK; b++)
                stack[++top] = -(nd->firstParticleIndex + b + 2);
            continue;
        }
        if (descend) { /* tree.cu:640-651: push every non-empty child */
            for (int c = 0; c < 8; c++)
                if (nd->child[c] != -1 && top + 1 < ORC_STACK) stack[++top] = nd->child[c];
            continue;
        }
        accepted++;
        if (acc) lanes_accumulate(px, py, pz, ax, ay, az, width, nd->massData, eps2, G, d2Order);
    }
    if (acc)
        for (int l = 0; l < width; l++)
            if (valid[l]) { acc[first + l].x = ax[l]; acc[first + l].y = ay[l]; acc[first + l].z = az[l]; }
    return accepted * nvalid;
}

long long orc_walk(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                   float theta, int groupWidth, int d2Order, float3* acc) {
    int groups = (n + groupWidth - 1) / groupWidth;
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
    for (int g = 0; g < groups; g++)
        total += walk_group(pos, n, nodes, extX, eps2, G, theta, g * groupWidth, groupWidth, d2Order, acc, NULL, 0.f, 1);
    return total;
}

long long orc_walk_sample(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                          float theta, int groupWidth, int d2Order, int stride, float3* acc) {
    int groups = (n + groupWidth - 1) / groupWidth;
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
    for (int g = 0; g < groups; g += stride)
        total += walk_group(pos, n, nodes, extX, eps2, G, theta, g * groupWidth, groupWidth, d2Order, acc, NULL, 0.f, 1);
    return total;
}

/* The group walk (width 32 or 64) with bucket leaves of at most leafSize bodies. */
long long orc_walk_buckets(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                           float theta, int leafSize, int width, float3* acc) {
    int groups = (n + width - 1) / width;
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
    for (int g = 0; g < groups; g++)
        total += walk_group(pos, n, nodes, extX, eps2, G, theta, g * width, width, 0, acc, NULL, 0.f, leafSize);
    return total;
}

/* The relative opening criterion of the engine's walk (an extension, not in
 * the reference): besides the reference's test, a node opens when
 * M s^2 > (alpha / G) |a_b| d^4 for a valid body b of the group, |a_b| being
 * that body's acceleration magnitude from the previous step (aMag, sorted
 * order).  groupParam (optional, one (theta, alpha) per 32-body group)
 * overrides theta and alpha per group; a group of width 64 takes the smaller
 * theta and alpha of its two 32-body halves. */
long long orc_walk_relative(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                            float theta, float alpha, const float* aMag, const float* groupParam,
                            int d2Order, int width, float3* acc) {
    int groups = (n + width - 1) / width;
    int groups32 = (n + 31) / 32;
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 8) reduction(+ : total)
    for (int g = 0; g < groups; g++) {
        float th = theta, al = alpha;
        if (groupParam) {
            int h = g * (width / 32);
            th = groupParam[2 * h];
            al = groupParam[2 * h + 1];
            if (width == 64 && h + 1 < groups32) {
                th = fminf(th, groupParam[2 * h + 2]);
                al = fminf(al, groupParam[2 * h + 3]);
            }
        }
        total += walk_group(pos, n, nodes, extX, eps2, G, th, g * width, width, d2Order, acc, aMag, al / G, 1);
    }
    return total;
}

/* Every stride-th group (width 32 or 64) of the walk, with the relative
 * criterion when aMag is given (per-group parameters as in
 * orc_walk_relative), else the reference's fixed-theta walk: accelerations of
 * those groups' bodies into acc (the rest untouched) and the accepted-node
 * count of group stride*k into listLen[k]. */
long long orc_walk_groups_sample(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                                 float theta, float alpha, const float* aMag, const float* groupParam,
                                 int width, int stride, float3* acc, int* listLen) {
    int groups = (n + width - 1) / width;
    int groups32 = (n + 31) / 32;
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
    for (int g = 0; g < groups; g += stride) {
        float th = theta, al = alpha;
        if (groupParam) {
            int h = g * (width / 32);
            th = groupParam[2 * h];
            al = groupParam[2 * h + 1];
            if (width == 64 && h + 1 < groups32) {
                th = fminf(th, groupParam[2 * h + 2]);
                al = fminf(al, groupParam[2 * h + 3]);
            }
        }
        int first = g * width;
        int nvalid = (n - first < width) ? n - first : width;
        long long a = walk_group(pos, n, nodes, extX, eps2, G, th, first, width, 0, acc, aMag, al / G, 1);
        if (listLen) listLen[g / stride] = (int)(a / nvalid);
        total += a;
    }
    return total;
}

void orc_walk_list_lengths(const float4* pos, int n, const node* nodes, float extX, float theta,
                           int groupWidth, int d2Order, int* listLen) {
    int groups = (n + groupWidth - 1) / groupWidth;
#pragma omp parallel for schedule(dynamic, 8)
    for (int g = 0; g < groups; g++) {
        int first = g * groupWidth;
        int nvalid = (n - first < groupWidth) ? n - first : groupWidth;
        long long a = walk_group(pos, n, nodes, extX, 0.f, 0.f, theta, first, groupWidth, d2Order, NULL, NULL, 0.f, 1);
        listLen[g] = (int)(a / nvalid);
    }
}

/* ----------------------------------------------------- FP64 diagnostics */
/* out[0..11]: M, sum m x (3), sum m v (3), sum m (x cross v) (3), sum m v^2,
 * sum_i m_i sum_{j != i} m_j / sqrt(r_ij^2 + eps2) (0 when !withPotential).
 * No reference counterpart: the engine's conserved-quantity definitions. */
void orc_diagnostics_f64(const float4* pos, const float3* vel, int n, double eps2, int withPotential, double* out) {
    double v[12] = {0};
    for (int i = 0; i < n; i++) {
        double m = pos[i].w, x = pos[i].x, y = pos[i].y, z = pos[i].z;
        double vx = vel[i].x, vy = vel[i].y, vz = vel[i].z;
        v[0] += m;
        v[1] += m * x; v[2] += m * y; v[3] += m * z;
        v[4] += m * vx; v[5] += m * vy; v[6] += m * vz;
        v[7] += m * (y * vz - z * vy);
        v[8] += m * (z * vx - x * vz);
        v[9] += m * (x * vy - y * vx);
        v[10] += m * (vx * vx + vy * vy + vz * vz);
    }
    double w = 0.0;
    if (withPotential) {
#pragma omp parallel for schedule(static) reduction(+ : w)
        for (int i = 0; i < n; i++) {
            double phi = 0.0;
            for (int j = 0; j < n; j++) {
                if (j == i) continue;
                double dx = (double)pos[j].x - pos[i].x, dy = (double)pos[j].y - pos[i].y,
                       dz = (double)pos[j].z - pos[i].z;
                phi += (double)pos[j].w / sqrt(dx * dx + dy * dy + dz * dz + eps2);
            }
            w += (double)pos[i].w * phi;
        }
    }
    v[11] = w;
    for (int k = 0; k < 12; k++) out[k] = v[k];
}

/* ------------------------------------------------------------ integrate */
/* tree.cu:678-703: v = v + a*dt (fused), then x = x + v_new*dt (fused). */
void orc_kick_drift(float4* pos, float3* vel, const float3* acc, int n, float dt) {
    for (int i = 0; i < n; i++) {
        vel[i].x = fmaf(acc[i].x, dt, vel[i].x);
        vel[i].y = fmaf(acc[i].y, dt, vel[i].y);
        vel[i].z = fmaf(acc[i].z, dt, vel[i].z);
        pos[i].x = fmaf(vel[i].x, dt, pos[i].x);
        pos[i].y = fmaf(vel[i].y, dt, pos[i].y);
        pos[i].z = fmaf(vel[i].z, dt, pos[i].z);
    }
}

/* ----------------------------------------------------- FP64 direct sum */
void orc_direct_sum_f64(const float4* pos, int n, const int* targets, int ntargets, double eps2,
                        double G, double* acc) {
    int nt = targets ? ntargets : n;
#pragma omp parallel for schedule(static)
    for (int k = 0; k < nt; k++) {
        int t = targets ? targets[k] : k;
        double x = pos[t].x, y = pos[t].y, z = pos[t].z;
        double sx = 0, sy = 0, sz = 0;
        for (int j = 0; j < n; j++) {
            double dx = (double)pos[j].x - x, dy = (double)pos[j].y - y, dz = (double)pos[j].z - z;
            double r2 = dx * dx + dy * dy + dz * dz + eps2;
            double inv = 1.0 / (r2 * sqrt(r2));
            double f = G * (double)pos[j].w * inv;
            sx += f * dx; sy += f * dy; sz += f * dz;
        }
        acc[3 * k] = sx; acc[3 * k + 1] = sy; acc[3 * k + 2] = sz;
    }
}

/* ---------------------------------------------------------------- step */
size_t orc_step_scratch_bytes(int n) {
    size_t nn = (size_t)n;
    return nn * (8 + 8 + 4 + 16 + 12) + nn * 8 * sizeof(node) + 256;
}

/* basicGravity.cu:767-783 with the reference's correct pointer use: build,
 * walk, kick-drift. */
int orc_step(float4* pos, float3* vel, int n, int bits, float eps, float G, float theta, float dt,
             int groupWidth, int d2Order, uint32_t* perm, float3* acc, void* scratch,
             long long* interactions) {
    char* s = (char*)scratch;
    size_t nn = (size_t)n;
    uint64_t* kin = (uint64_t*)s; s += nn * 8;
    uint64_t* kout = (uint64_t*)s; s += nn * 8;
    uint32_t* iin = (uint32_t*)s; s += nn * 4;
    float4* ptmp = (float4*)s; s += nn * 16;
    float3* vtmp = (float3*)s; s += nn * 12;
    s = (char*)(((uintptr_t)s + 63) & ~(uintptr_t)63);
    node* nodes = (node*)s;
    float mn[3], mx[3];
    worldBox box;
    int lo[23], lc[23], deepest;
    orc_bbox(pos, n, mn, mx);
    orc_world_box(mn, mx, bits, &box);
    orc_morton_encode(pos, n, box, bits, kin, iin);
    orc_sort_pairs(kin, iin, kout, perm, n);
    orc_reorder(pos, vel, perm, ptmp, vtmp, n);
    memcpy(pos, ptmp, nn * 16);
    memcpy(vel, vtmp, nn * 12);
    int m = orc_build_tree(kout, pos, n, bits, nodes, 8 * n, lo, lc, &deepest);
    if (m < 0) return -1;
    long long it = orc_walk(pos, n, nodes, mx[0] - mn[0], eps * eps, G, theta, groupWidth, d2Order, acc);
    if (interactions) *interactions = it;
    orc_kick_drift(pos, vel, acc, n, dt);
    return m;
}
