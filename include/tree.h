/*
 * tree.h — bounding box, Morton keys, octree, tree walk and integrator of the
 * B200 Barnes-Hut engine.
 *
 * Drop-in counterpart of the reference's tree.h (tree.h:16-46).  The
 * reference declares CUDA kernels there; a C ABI cannot carry `__global__`
 * functions, so each kernel becomes a launcher with the same name and
 * argument meaning plus a trailing cudaStream_t (0 = legacy default stream):
 *
 *     mortonEncode<<<blocks, 256>>>(pos, keys, idx, n, box);      // reference
 *     mortonEncode(pos, keys, idx, n, box, 0);                    // here
 *
 * Launch geometry is chosen by this library for sm_100a.  The prefix-sum
 * helpers keep their reference signatures.  The reference's exit-on-error
 * behaviour is kept for the functions that had it (sumCreate, prefixSum);
 * launchers report launch errors through bh_last_error() (bh_api.h).
 *
 * The level-at-a-time entry points (identifyNodesAtLevel, createNodes,
 * updateTreeParticles, updateTreeMass) exist for callers that drive the
 * reference's per-level build themselves.  buildTree() (main.h) does not use
 * them: it builds every level in one pass without host round trips.
 */
#ifndef BH_TREE_H
#define BH_TREE_H

#include <stdint.h>
#include <driver_types.h>
#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Reference launch constants (tree.h:16-18). */
#define BOXTHREADS 256
#define BOXBLOCKS 256
#define WARPTHREADS 32

/* tree.h:20 / tree.cu:347-367 — key[i] = interleave of the 21-bit grid
 * coordinates (x<<2 | y<<1 | z per bit), originalIndex[i] = i. */
void mortonEncode(const float4* posMassVals, uint64_t* mortonCodes, uint32_t* originalIndex,
                  int NStars, worldBox rootBox, cudaStream_t stream);

/* tree.h:22 / tree.cu:414-456 — per-block min/max of x,y,z; writes
 * BOXBLOCKS partial corners. */
void localMinMaxFinder(const float4* posMassVals, unsigned int N, float3* minCorner,
                       float3* maxCorner, cudaStream_t stream);

/* tree.h:24 / tree.cu:459-490 — reduces `count` partial corners to one. */
void globalMinMaxReducer(const float3* minCorner, const float3* maxCorner, int count,
                         float3* outMin, float3* outMax, cudaStream_t stream);

/* tree.h:26 / tree.cu:50-78 — flag[i] = 1 when body i starts a level-L node. */
void identifyNodesAtLevel(uint64_t* mortonCodes, int nodeLevel, int starCount,
                          uint32_t* nodeFlags, cudaStream_t stream);

/* tree.h:28 / tree.cu:205-235 — writes the level's node records and links
 * each into its parent's child[] slot. */
void createNodes(const uint64_t* mortonCodes, const uint32_t* flags, const uint32_t* previousFlags,
                 const uint32_t* offsets, const uint32_t* offsetsPrev, node* nodes, int level,
                 int arrayLevelOffset, int prevArrayLevelOffset, int starCount, int maxNodes,
                 cudaStream_t stream);

/* tree.h:30 / tree.cu:181-203 — particleCount from the next sibling or the
 * parent's end. */
void updateTreeParticles(node* nodes, int levelStartIndex, int levelNodeCount, int starCount,
                         cudaStream_t stream);

/* tree.h:32 / tree.cu:89-179 — mass and centre of mass of one level's nodes
 * from their bodies (leaves) or children (internal nodes). */
void updateTreeMass(node* nodes, const float4* positionMassVals, int level, int levelNodes,
                    int levelStartIndex, cudaStream_t stream);

/* tree.h:34 / tree.cu:562-676 — Barnes-Hut acceleration of every body.
 * Groups of 32 Morton-consecutive bodies share one opening decision per node
 * (open if any body of the group fails size^2 < theta^2 d^2); monopole with
 * Plummer softening antiSingularitySquared.  `tree` must come from
 * initialiseTree()/buildTree() of this library. */
void calculateAcceleration(const float4* positionMassArray, treeState tree, float3* accelVals,
                           float antiSingularitySquared, float GVal, float theta, int starCount,
                           cudaStream_t stream);

/* tree.h:36 / tree.cu:678-703 — symplectic Euler: v += a dt; x += v dt. */
void positionUpdater(float4* positionMassArray, float3* velocityVals, float3* accelerationVals,
                     int starCount, float timeStep, cudaStream_t stream);

/* tree.h:42 / tree.cu:241-284 — exclusive-scan object for up to maxCount
 * uint32 flags, plus the build's ping-pong flag/offset arrays. */
treeBuilder* sumCreate(int maxCount);

/* tree.h:38,44 / tree.cu:286-302 — offsets = exclusive prefix sum of flags
 * (maxCount elements) on the legacy default stream. */
void prefixSum(treeBuilder* builder, uint32_t* flags, uint32_t* offsets, int maxCount);

/* tree.cu:304-318 — frees what sumCreate() allocated. */
void sumDestroyer(treeBuilder* sum);

#ifdef __cplusplus
}
#endif

#endif /* BH_TREE_H */
