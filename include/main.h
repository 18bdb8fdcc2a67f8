/*
 * main.h — one-call-per-stage orchestration of a Barnes-Hut step.
 *
 * The reference keeps this orchestration in basicGravity.cu without a header
 * (initialiseTree basicGravity.cu:5-77, createWorldBox :79-113, buildTree
 * :116-325, blockNumCalculator :374-427); its main.h (main.h:4-27) only pulls
 * the other headers together.  This header does both: it includes types.h,
 * tree.h and sorting.h and declares the orchestration functions with the
 * reference's signatures, so the reference's main() loop
 *
 *     initialiseTree(state, N, paddedN, blocks);
 *     for (...) { buildTree(state, &pos, &vel);
 *                 calculateAcceleration(pos, *state, acc, eps*eps, G, theta, N, 0);
 *                 positionUpdater(pos, vel, acc, N, dt, 0); }
 *
 * links against this library unchanged apart from the launch syntax.
 *
 * Contracts kept from the reference:
 *   - buildTree() re-sorts the bodies into Morton order and SWAPS the
 *     caller's pos/vel pointers with the state's second buffers
 *     (basicGravity.cu:217-226): after the call *pos and *vel point at the sorted
 *     arrays and state->indexOut holds the permutation of this step;
 *   - after buildTree() the host fields levelOffsets/levelCount/deepestLevel
 *     are filled and state->nodes holds the tree in the reference layout;
 *   - errors print a message and exit(-1).  The bh_* variants in bh_api.h
 *     return status codes instead.
 * Differences: the whole build runs on the device without per-level host
 * synchronisation (one synchronisation at the end copies the level table);
 * destroyTree() releases what initialiseTree() allocated (the reference has
 * no counterpart).
 */
#ifndef BH_MAIN_H
#define BH_MAIN_H

#include "types.h"
#include "tree.h"
#include "sorting.h"

#ifdef __cplusplus
extern "C" {
#endif

#define THREADCOARSENING 2 /* main.h:25 */
#define THREADPERBLOCK 256 /* main.h:26 */

/* basicGravity.cu:5-77 — allocates the tree for starCount bodies: node array
 * of 8*starCount, keys, indices, bounding-box scratch and the second pos/vel
 * buffers of paddedStarCount entries (zeroed).  integrateBlocks is stored in
 * treeBlocks as in the reference. */
void initialiseTree(treeState* state, int starCount, int paddedStarCount, int integrateBlocks);

/* basicGravity.cu:79-113 — bounding box of the bodies and the Morton grid
 * mapping: extent = max(width, height, depth), scale = (2^21-1)/extent. */
void createWorldBox(const float4* cudaPositionMassVals, const int starCount, float3* cudaMinCorner,
                    float3* cudaMaxCorner, float3* cudaOutputMin, float3* cudaOutputMax,
                    worldBox* outputWorldBox);

/* basicGravity.cu:116-325 — bounding box, keys, sort, reorder (pointer swap),
 * level-wise octree and the upward mass pass. */
void buildTree(treeState* tree, float4** cudaPosMasVals, float3** cudaVelVals);

/* Releases everything initialiseTree() allocated (no reference counterpart). */
void destroyTree(treeState* state);

/* basicGravity.cu:374-427 — the reference's launch-geometry helper: walk
 * blocks of 32 threads, integrate/build blocks of 256, N padded to 32. */
void blockNumCalculator(int* accelerationBlocks, int* treeBuilderBlocks, int* integrateBlocks,
                        int* paddedStarCount, int* integrationThreadsPerBlock,
                        int* treeBuilderThreadsPerBlock, int starCount);

/* basicGravity.cu:351-366. */
int roundNumberToMultiple(int number, int multiple);

#ifdef __cplusplus
}
#endif

#endif /* BH_MAIN_H */
