/*
 * types.h — data structures shared by the host code and the B200 Barnes-Hut
 * engine.
 *
 * Drop-in counterpart of the reference's types.h (types.h:1-107). The
 * structures that cross the C ABI (`node`, `worldBox`, `treeState`,
 * `radixSorter`, `treeBuilder`) keep the reference's member order, types and
 * therefore its byte layout, so a caller written against the reference can
 * pass them to this library unchanged:
 *   node        80 B  (path@0 parent@8 first@12 count@16 child[8]@20 level@52
 *                      massData@64)                       types.h:52-62
 *   treeState  304 B                                       types.h:75-90
 *   worldBox    20 B                                       types.h:25-34
 *   radixSorter / treeBuilder                              types.h:19-23, 64-73
 * The layout is checked at compile time below (C11 / C++11 static asserts).
 *
 * What differs is ownership of the opaque members: in this library
 * `radixSorter.tempStorage` and `treeBuilder.tempStorage` point at this
 * library's own scratch, and a `treeBuilder` returned by initialiseTree() is
 * the first member of a larger private context.  Callers only ever hold the
 * pointers, exactly as with the reference.
 */
#ifndef BH_TYPES_H
#define BH_TYPES_H

#include <stddef.h>
#include <stdint.h>
#include <vector_types.h> /* float3, float4 (CUDA's plain-C vector structs) */

#ifdef __cplusplus
extern "C" {
#endif

/* Host-side 4- and 3-vectors used by the initial-condition and output code
 * (types.h:7-13). */
typedef struct __attribute__((aligned(16))) {
    float x, y, z, m;
} sVec4;

typedef struct {
    float x, y, z;
} sVec3;

typedef struct {
    uint8_t R, G, B;
} RGB;

/* Scratch owned by a sorter created with sorterCreate() (types.h:19-23). */
typedef struct {
    void* tempStorage;
    size_t tempStorageBytes;
    int capacity;
} radixSorter;

/* Cube enclosing all bodies and the float -> integer-grid factor
 * scale = (2^bits - 1) / extent (types.h:25-34). */
typedef struct {
    float minX, minY, minZ;
    float extent;
    float scale;
} worldBox;

/* One octree node in the reference's array-of-structs layout (types.h:52-62).
 * Nodes are stored level by level; within a level in Morton order. child[s]
 * is the index of the child in octant s, or -1. massData = (COM xyz, mass). */
typedef struct {
    uint64_t nodePathFromRoot;
    int parentIndex;
    int firstParticleIndex;
    int particleCount;
    int child[8];
    int treeLevel;
    float4 massData;
} node;

/* Prefix-sum object of the level-wise build (types.h:64-73). */
typedef struct {
    void* tempStorage;
    size_t tempStorageBytes;
    int capacity;
    uint32_t* flagsPing;
    uint32_t* flagsPong;
    uint32_t* offsetsPing;
    uint32_t* offsetsPong;
} treeBuilder;

/* Everything one simulation's tree needs on the device (types.h:75-90).
 * levelOffsets/levelCount/deepestLevel are host copies filled by buildTree(). */
typedef struct {
    node* nodes;
    int maxNodes;
    uint64_t* mortonIn;
    uint64_t* mortonOut;
    uint32_t* indexIn;
    uint32_t* indexOut;
    float3* boundingData[4]; /* block minima, block maxima, global min, global max */
    radixSorter* sorter;
    treeBuilder* builder;
    int levelOffsets[22];
    int levelCount[22];
    int deepestLevel;
    int treeBlocks;
    int starCount;
    float4* sortedPosMassVals;
    float3* sortedVelVals;
} treeState;

/* Disk parameters of the reference's initial conditions (types.h:92-100). */
typedef struct {
    float scaleLength;
    float scaleThickness;
    float totalDiskMass;
    sVec3 rotationAngles; /* yaw, pitch, roll */
    sVec3 galacticCentreLocation;
    sVec3 galacticNetVelocity;
} galaxyDiskParameters;

/* Pair used by the reference's ordered frame writer (types.h:102-105). */
typedef struct {
    float4* positionVal;
    uint32_t* originalIndex;
} sorterPair;

#ifdef __cplusplus
} /* extern "C" */
#define BH_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define BH_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

BH_STATIC_ASSERT(sizeof(node) == 80, "node must be 80 bytes");
BH_STATIC_ASSERT(offsetof(node, parentIndex) == 8, "node.parentIndex @8");
BH_STATIC_ASSERT(offsetof(node, child) == 20, "node.child @20");
BH_STATIC_ASSERT(offsetof(node, treeLevel) == 52, "node.treeLevel @52");
BH_STATIC_ASSERT(offsetof(node, massData) == 64, "node.massData @64");
BH_STATIC_ASSERT(sizeof(treeState) == 304, "treeState must be 304 bytes");
BH_STATIC_ASSERT(sizeof(worldBox) == 20, "worldBox must be 20 bytes");

#endif /* BH_TYPES_H */
