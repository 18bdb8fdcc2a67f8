/*
 * bh_oracle.h — CPU oracle for the Barnes-Hut step pipeline.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * algorithm (internet-cabbage/CUDAGravityDemo: tree.cu, sorting.cu,
 * basicGravity.cu) used to check the CUDA engine.  Only the tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
 * product never calls it.
 *
 * Arithmetic follows the reference operation by operation in FP32: the file
 * is compiled with -ffp-contract=off and uses fmaf() exactly where nvcc
 * contracts a multiply-add in the reference's device code.  Parity is pinned
 * against the reference itself: the reference's own kernels, compiled from
 * its sources into oracle/_ref/ and run on a B200, produce the fixtures under
 * tests/golden/ that this oracle must reproduce bit for bit.
 */
#ifndef BH_ORACLE_H
#define BH_ORACLE_H

#include <stdint.h>
#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Bounding box of n float4 bodies (tree.cu:414-490). */
void orc_bbox(const float4* pos, int n, float mn[3], float mx[3]);

/* World box for `bits` bits per axis (basicGravity.cu:79-113):
 * extent = fmaxf(w, fmaxf(h, d)), scale = (float)(2^bits - 1) / extent. */
void orc_world_box(const float mn[3], const float mx[3], int bits, worldBox* out);

/* Spread the low `bits` bits of v with two zero bits between them
 * (tree.cu:332-340 for bits = 21). */
uint64_t orc_expand_bits(uint64_t v, int bits);

/* Morton keys + identity indices (tree.cu:343-367). */
void orc_morton_encode(const float4* pos, int n, worldBox box, int bits, uint64_t* keys,
                       uint32_t* idx);

/* Stable ascending sort of (key, value) pairs (sorting.cu:65-79 semantics). */
void orc_sort_pairs(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut,
                    uint32_t* valsOut, int n);

/* Gather by permutation (sorting.cu:99-107). */
void orc_reorder(const float4* posIn, const float3* velIn, const uint32_t* idx, float4* posOut,
                 float3* velOut, int n);

/* Level-wise octree build + particle counts + upward mass pass
 * (basicGravity.cu:116-325 with tree.cu:50-235 and tree.cu:89-179).
 * levelOffsets/levelCount have 23 entries.  Returns the node count, or -1 if
 * the tree needs more than maxNodes nodes (basicGravity.cu:282). */
int orc_build_tree(const uint64_t* sortedKeys, const float4* sortedPos, int n, int bits,
                   node* nodes, int maxNodes, int* levelOffsets, int* levelCount,
                   int* deepestLevel);

/* d^2 evaluation orders for the walk, i.e. which multiply-adds nvcc fuses in
 * (dx*dx + dy*dy) + dz*dz (tree.cu:611).  ORC_D2_REF = fma(dz, dz, fma(dx,
 * dx, dy*dy)) is the one the reference's compiled walk uses: with it the
 * oracle reproduces the reference's accelerations bit for bit (pinned by the
 * golden fixtures); the others exist to show that the choice matters. */
enum { ORC_D2_REF = 0, ORC_D2_ALT = 1, ORC_D2_PLAIN = 2 };

/* Reference tree walk (tree.cu:501-676): groups of `groupWidth` consecutive
 * bodies, shared depth-first stack, open when any valid member fails
 * size^2 < theta^2 d^2 (size from the x-extent, tree.cu:501-530), leaves
 * (count <= 1 or no children) never opened, monopole with Plummer softening.
 * Writes acc[3*i]; returns the number of body-node interactions of valid
 * bodies. OpenMP over groups. */
long long orc_walk(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                   float theta, int groupWidth, int d2Order, float3* acc);

/* The same walk over every `stride`-th group only (a bounded sample of the
 * full walk for CPU timing); acc is written for the sampled groups. */
long long orc_walk_sample(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                          float theta, int groupWidth, int d2Order, int stride, float3* acc);

/* Per-group interaction-list lengths of the same walk (list[g] = accepted
 * nodes of group g). */
/* Group walk (width 32) with bucket leaves of at most leafSize bodies. */
long long orc_walk_buckets(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                           float theta, int leafSize, int width, float3* acc);
/* Group walk (width 32 or 64) with the relative opening criterion. */
long long orc_walk_relative(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                            float theta, float alpha, const float* aMag, const float* groupParam,
                            int d2Order, int width, float3* acc);
/* Every stride-th group of the walk (relative criterion when aMag != NULL):
 * accelerations of those bodies and each sampled group's accepted count. */
long long orc_walk_groups_sample(const float4* pos, int n, const node* nodes, float extX, float eps2, float G,
                                 float theta, float alpha, const float* aMag, const float* groupParam,
                                 int width, int stride, float3* acc, int* listLen);
void orc_walk_list_lengths(const float4* pos, int n, const node* nodes, float extX, float theta,
                           int groupWidth, int d2Order, int* listLen);

/* Symplectic Euler kick-drift (tree.cu:678-703). */
void orc_kick_drift(float4* pos, float3* vel, const float3* acc, int n, float dt);

/* FP64 direct-sum accelerations of the bodies listed in `targets`
 * (ntargets entries; NULL = all n bodies): a_t = sum_j G m_j (x_j - x_t) /
 * (|x_j - x_t|^2 + eps2)^{3/2}.  OpenMP over targets. */
void orc_direct_sum_f64(const float4* pos, int n, const int* targets, int ntargets, double eps2,
                        double G, double* acc);

/* One full reference step on host arrays (bbox, keys, sort, reorder, tree,
 * walk, kick-drift).  pos/vel are replaced by the sorted, updated arrays;
 * perm receives this step's permutation; acc the accelerations (sorted
 * order).  scratch: see orc_step_scratch_bytes().  Returns node count or -1. */
size_t orc_step_scratch_bytes(int n);
int orc_step(float4* pos, float3* vel, int n, int bits, float eps, float G, float theta, float dt,
             int groupWidth, int d2Order, uint32_t* perm, float3* acc, void* scratch,
             long long* interactions);

/* Number of OpenMP threads the oracle will use. */
/* FP64 conserved-quantity sums (see bh_oracle.c). */
void orc_diagnostics_f64(const float4* pos, const float3* vel, int n, double eps2, int withPotential, double* out);
int orc_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif /* BH_ORACLE_H */
