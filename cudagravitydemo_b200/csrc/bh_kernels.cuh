// bh_kernels.cuh — host-side launchers of the sm_100a kernels.  Each kernel
// file defines its kernels and the launchers declared here; capi.cu strings
// them into the reference's stages.
#pragma once

#include "bh_internal.cuh"

// ---- bbox_morton.cu --------------------------------------------------------
constexpr int kBboxMaxGrid = 1024;  // partial-result slots of the box reduction
// partials64 (4 * kBboxMaxGrid doubles) and root (both optional, together):
// the FP64 mass, centre of mass and box of all bodies.
cudaError_t bh_launch_bbox(const float4* pos, int n, float* partials, unsigned* ticket, DevBox* box,
                           float3* outMin, float3* outMax, int bits, int* err, uint32_t* zeroBuf,
                           int zeroWords, cudaStream_t s, double* partials64 = nullptr, DevRoot* root = nullptr);
// keys from a device box (boxPtr) or, when boxPtr is NULL, from boxVal.
// idx and hist may be NULL.
cudaError_t bh_launch_morton(const float4* pos, int n, const DevBox* boxPtr, worldBox boxVal, int bits,
                             uint64_t* keys, uint32_t* idx, uint32_t* hist, int npass, cudaStream_t s,
                             const uint16_t* sysOf = nullptr);
// Batch: per-system world boxes (systems blocks at most) and zeroed histograms.
cudaError_t bh_launch_bbox_segments(const float4* pos, const int* segOff, int systems, DevBox* boxes, int bits,
                                    int* err, uint32_t* zeroBuf, int zeroWords, cudaStream_t s);
cudaError_t bh_launch_local_minmax(const float4* pos, unsigned n, float3* minCorner, float3* maxCorner,
                                   int blocks, cudaStream_t s);
cudaError_t bh_launch_global_minmax(const float3* minCorner, const float3* maxCorner, int count,
                                    float3* outMin, float3* outMax, cudaStream_t s);

// ---- radix_sort.cu ----------------------------------------------------------
int bh_sort_tile();
cudaError_t bh_sort_init();  // raises the dynamic shared-memory limit once
// Look-back of tile 1 against status words whose tile 0 never publishes
// (status[0..511] must be zero): gives up after BH_SPIN_LIMIT round trips and
// sets BH_ERR_TIMEOUT in *err.  Exercises the bounded wait without a fault.
cudaError_t bh_launch_lookback_selftest(const uint32_t* status, int* err, cudaStream_t s);
cudaError_t bh_launch_sort_histogram(const uint64_t* keys, int n, uint32_t* hist, int npass, cudaStream_t s);
cudaError_t bh_launch_sort_pass(const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut,
                                uint32_t* valsOut, int n, int shift, const uint32_t* hist,
                                uint32_t* status, int* tileCounter, int* err, int identityVals,
                                cudaStream_t s);

// ---- octree.cu ----------------------------------------------------------------
int bh_tree_threads();
cudaError_t bh_launch_tree_count(const uint64_t* keys, int n, int bits, uint8_t* delta, int* blockLevel,
                                 cudaStream_t s);
// nCB: per node (child range start, size^2 bits), plus the sentinel at nodeCount;
// nCom: per node centre of mass and mass (compact copy for the upward pass)
// levelTotal: BH_LEVEL_SLOTS ints of scratch; ticket: one device word, zero
// between builds (the kernel re-arms it)
cudaError_t bh_launch_tree_scan(int* blockLevel, int nblocks, int n, int bits, int maxNodes,
                                const DevBox* box, DevTreeInfo* info, int2* nCB, int* levelTotal, unsigned* ticket,
                                int* err, cudaStream_t s);
cudaError_t bh_launch_tree_nodes(const uint64_t* keys, const uint8_t* delta, int n, int bits,
                                 const int* blockLevel, const DevTreeInfo* info, int maxNodes, const DevBox* boxes,
                                 int2* nCB, int* nParent, int* nFirst, int* nMeta, cudaStream_t s);
// cooperative launch; bar: one device word for the grid barrier
cudaError_t bh_launch_tree_mass(const float4* pos, const uint8_t* delta, int n, int bits, const DevTreeInfo* info,
                                const int2* nCB, float4* nCom, WalkNode* wn, const int* nFirst, int* nCount,
                                unsigned* bar, int* err, cudaStream_t s);
cudaError_t bh_launch_tree_export(const uint64_t* keys, int bits, const DevTreeInfo* info,
                                  const WalkNode* wn, const int* nParent, const int* nFirst,
                                  const int* nCount, const int* nMeta, node* out, int n, int maxNodes,
                                  cudaStream_t s);
// auxIn/auxOut: an optional per-body float carried along (NULL: none)
cudaError_t bh_launch_reorder(const float4* posIn, const float3* velIn, const uint32_t* idIn,
                              const uint32_t* perm, float4* posOut, float3* velOut, uint32_t* idOut,
                              int n, cudaStream_t s, const float* auxIn = nullptr, float* auxOut = nullptr);
cudaError_t bh_launch_scatter_by_id(const float4* pos, const float3* vel, const float3* acc,
                                    const uint32_t* ids, float4* posOut, float3* velOut,
                                    float3* accOut, int n, cudaStream_t s, const float* aux = nullptr,
                                    float* auxOut = nullptr);
cudaError_t bh_launch_iota(uint32_t* ids, int n, cudaStream_t s);
// one block that waits about ns nanoseconds on the device (bounded)
cudaError_t bh_launch_hold(unsigned long long ns, cudaStream_t s);
// out[i] = in[ids[i]] for ids in [0, n); an id outside reads nothing, gives
// +inf and sets BH_ERR_INVALID in *err (in/out NULL: the ids are only checked)
cudaError_t bh_launch_gather_by_id(const float* in, const uint32_t* ids, float* out, int n, int* err,
                                   cudaStream_t s);

// ---- walk.cu -------------------------------------------------------------------
struct WalkArgs {
    const float4* pos;
    int n;
    const WalkNode* wn;
    float theta, eps2, G;
    float3* accOut;        // may be NULL
    const float3* velIn;   // fused kick-drift: inputs ...
    float4* posOut;        // ... and outputs (may alias nothing of the inputs)
    float3* velOut;
    const uint32_t* idIn;  // optional body ids carried along
    uint32_t* idOut;
    // fused kick-drift, optional second copies of posOut, velOut and idOut
    // (all three or none; device pointers of mapped page-locked host memory:
    // the result crosses PCIe while the walk runs)
    float4* posHost;
    float3* velHost;
    uint32_t* idHost;
    float dt;
    DevCounters* ctr;
    int* err;
    int* spill;            // bh_walk_spill_ints() ints
    // opening criterion beyond the reference's fixed theta (all optional):
    const float2* groupParam;  // per 32-body group: (theta_g, alpha_g); NULL = theta for all
    bool relative;             // also open when G M s^2 > alpha_g |a_b| d^4 (needs aMagIn)
    float alpha;               // alpha for every group when groupParam is NULL
    const float* aMagIn;       // |a| of each body from the previous step (walk order)
    float* aMagOut;            // |a| of each body from this walk (may be NULL)
    // batch: group g = bodies [x, x + y) walking the tree rooted at node z
    // (groups entries; NULL = groups of 32 consecutive bodies, root node 0)
    const int4* groupTable;
    int groups;
    // bucket leaves: an opened node with at most leafSize bodies (> 1)
    // contributes its bodies (from nFirst[node]) instead of its children
    int leafSize;
    const int* nFirst;
    // bodies per group: 32 (the reference) or 64 (two per lane); groupParam
    // stays per 32-body group (groupParamCount entries)
    int groupWidth;
    int groupParamCount;
    // interaction-list length (accepted nodes) of each group (optional)
    int* groupLen;
    // traversal-stack entries per warp kept in shared memory (0: the
    // default); a multiple of 32 in [BH_WALK_STACK_MIN, BH_WALK_STACK_MAX]
    int stackSmem;
    // optional: the walk takes groups in this order (a permutation of the
    // groups, from bh_launch_group_order); NULL = in index order
    const int* groupOrder;
};
#define BH_WALK_STACK_MIN 128
#define BH_WALK_STACK_MAX 2048
int bh_walk_stack_default();
// order[0..groups) = the groups by decreasing len[] (the last walk's list
// lengths); blockHist: bh_group_order_hist_ints(groups) ints of scratch
int bh_group_order_hist_ints(int groups);
cudaError_t bh_launch_group_order(const int* len, int groups, int* order, int* blockHist, cudaStream_t s);
int bh_walk_grid();          // persistent grid size on the current device
size_t bh_walk_spill_ints(); // ints of stack spill space the walk needs
cudaError_t bh_launch_walk(const WalkArgs& a, bool fused, bool compensated, cudaStream_t s);
cudaError_t bh_launch_kick_drift(float4* pos, float3* vel, const float3* acc, int n, float dt,
                                 cudaStream_t s);

// Learned opening criterion (mlp.cu).  feat: groups x BH_GROUP_FEATURES;
// groupParam: (theta, alpha) per group.
cudaError_t bh_launch_group_features(const float4* pos, const float* aMag, const uint64_t* keys, int n, int bits,
                                     const DevBox* box, const DevRoot* root, float G, float* feat, cudaStream_t s);
cudaError_t bh_launch_mac_select(const float* params, const float* feat, int groups, float logTarget, float thetaCap,
                                 float2* groupParam, cudaStream_t s);
