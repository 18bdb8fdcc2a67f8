// capi.cu — the C ABI of the B200 Barnes-Hut engine: the reference-named
// entry points of tree.h / sorting.h / main.h, their status-returning bh_*
// variants, and the device-resident bh_sim.
//
// A step is the reference's buildTree + calculateAcceleration +
// positionUpdater (basicGravity.cu:116-325, 767-783), issued as stream-ordered
// kernels with no host synchronisation inside:
//   k_bbox (world box on the device, histograms zeroed)
//   k_morton (keys + radix digit histograms)
//   k_sort_pass x ceil(3*bits/8)
//   k_reorder (pos, vel, body ids)
//   k_tree_count, k_tree_scan, k_tree_nodes, k_tree_mass [, k_tree_export]
//   k_walk (+ fused kick-drift)
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "bh_api.h"
#include "bh_internal.cuh"
#include "bh_kernels.cuh"
#include "main.h"

size_t bh_scan_temp_bytes(int maxCount);  // compat.cu

// ------------------------------------------------------------------ status
static thread_local int g_last_status = BH_OK;
static thread_local char g_cuda_err[256] = "";

int bh_note_cuda_error(cudaError_t e) {
    snprintf(g_cuda_err, sizeof g_cuda_err, "%s (%s)", cudaGetErrorString(e), cudaGetErrorName(e));
    return BH_ERR_CUDA;
}

int bh_sm_count() {
    static int count = 0;
    if (count == 0) {
        int dev = 0, c = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && c > 0)
            count = c;
        else
            return 148;
    }
    return count;
}

extern "C" const char* bh_status_string(int s) {
    switch (s) {
    case BH_OK: return "ok";
    case BH_ERR_INVALID: return "invalid argument";
    case BH_ERR_ALLOC: return "allocation failed";
    case BH_ERR_CUDA: return "CUDA error";
    case BH_ERR_DEGENERATE_BOX: return "degenerate bounding box";
    case BH_ERR_NONFINITE: return "non-finite body position";
    case BH_ERR_TREE_OVERFLOW: return "tree node capacity exceeded";
    case BH_ERR_STACK_OVERFLOW: return "walk stack overflow";
    case BH_ERR_TIMEOUT: return "device wait timed out";
    case BH_ERR_INTERNAL: return "internal consistency check failed";
    default: return "unknown status";
    }
}

extern "C" int bh_last_error(void) { return g_last_status; }
extern "C" const char* bh_cuda_error_string(void) { return g_cuda_err; }

static int set_status(int s) {
    g_last_status = s;
    return s;
}
int bh_record_status(int s) { return set_status(s); }

// lowest error bit of a device error word -> status
static int status_from_bits(int bits) {
    for (int s = 1; s <= BH_ERR_INTERNAL; s++)
        if (bits & (int)BH_ERRBIT(s)) return s;
    return BH_OK;
}
int bh_status_from_bits(int bits) { return status_from_bits(bits); }

extern "C" void bh_params_default(bh_params* p) {
    if (!p) return;
    p->bitsPerAxis = 21;
    p->leafSize = 1;
    p->groupWidth = 32;
    p->theta = 0.7f;   // units.c:4
    p->eps = 0.02f;    // basicGravity.cu:466
    p->G = 1.0f;       // units.c:3
    p->dt = 0.08f;     // basicGravity.cu:465
    p->compensated = 1;
    p->exportNodes = 0;
    p->macMode = 0;
    p->alpha = 1e-3f;
    p->errTarget = 5e-3f;
}

static int check_params(const bh_params* p) {
    if (!p) return BH_ERR_INVALID;
    if (p->bitsPerAxis < 1 || p->bitsPerAxis > BH_MAX_BITS) return BH_ERR_INVALID;
    if (p->leafSize < 1 || p->leafSize > BH_MAX_LEAF_SIZE) return BH_ERR_INVALID;
    if (p->groupWidth != 32 && p->groupWidth != 64) return BH_ERR_INVALID;
    if (!(p->theta >= 0.0f) || !(p->eps >= 0.0f)) return BH_ERR_INVALID;
    if (p->macMode < 0 || p->macMode > 2) return BH_ERR_INVALID;
    if (p->macMode == 1 && !(p->alpha > 0.0f)) return BH_ERR_INVALID;
    if (p->macMode == 2 && !(p->errTarget > 0.0f)) return BH_ERR_INVALID;
    return BH_OK;
}

// ------------------------------------------------------------ device context
// Device scratch of one tree of up to `capacity` bodies.  treeState.builder
// points at `tb`, the first member.
struct bh_ctx {
    treeBuilder tb;
    uint32_t magic;
    int capacity;
    int maxNodes;
    int treeBlocks;  // blocks of the tree kernels at capacity
    int sortTiles;   // sort tiles at capacity
    // sort
    uint64_t* keysTmp;
    uint32_t* valsTmp;
    uint32_t* sortHist;    // [8][256]
    uint32_t* sortStatus;  // [8 tile counters padded to 256] + [8][sortTiles][256]
    size_t sortStatusWords;
    // box
    float* bboxPartials;
    unsigned* bboxTicket;
    DevBox* box;
    double* bboxPartials64;  // FP64 root reduction: block partials ...
    DevRoot* root64;         // ... and the root's FP64 mass, centre of mass, box
    // tree
    uint8_t* delta;
    int* blockLevel;
    DevTreeInfo* info;
    WalkNode* wn;
    int2* nCB;     // per node: child range start, size^2 (+ the sentinel)
    int* levelTotal;      // per level node counts (scan scratch)
    unsigned* scanTicket; // last-block ticket of the level scan (zero between builds)
    float4* nCom;  // per node: centre of mass and mass (compact copy)
    int* nParent;
    int* nFirst;
    int* nCount;
    int* nMeta;
    unsigned* gridBar;  // grid barrier word of the upward pass
    // walk
    DevCounters* ctr;
    int* err;
    int* spill;
    bool initialised;
    // second pos/vel buffers allocated by initialiseTree(); buildTree() swaps
    // them with the caller's, so destroyTree() frees these, not the fields
    void* ownedPos;
    void* ownedVel;
};

static const uint32_t kCtxMagic = 0xB4200B42u;

template <typename T>
static int dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
    if (e != cudaSuccess) {
        bh_note_cuda_error(e);
        *p = nullptr;
        return BH_ERR_ALLOC;
    }
    return BH_OK;
}

static void ctx_free(bh_ctx* c) {
    if (!c) return;
    void* ptrs[] = {c->keysTmp, c->valsTmp, c->sortHist, c->sortStatus, c->bboxPartials, c->bboxTicket,
                    c->bboxPartials64, c->root64, c->box, c->delta, c->blockLevel, c->info, c->wn, c->nCB, c->nCom, c->levelTotal, c->scanTicket, c->nParent, c->nFirst,
                    c->nCount, c->nMeta, c->gridBar, c->ctr, c->err, c->spill,
                    c->tb.flagsPing, c->tb.flagsPong, c->tb.offsetsPing, c->tb.offsetsPong,
                    c->tb.tempStorage};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    c->magic = 0;
    delete c;
}

static int sort_init_once() {
    static bool done = false;
    if (!done) {
        BH_CUDA_TRY(bh_sort_init());
        done = true;
    }
    return BH_OK;
}

static int ctx_create(bh_ctx** out, int capacity, int maxNodes) {
    *out = nullptr;
    if (capacity <= 0 || maxNodes <= 0) return BH_ERR_INVALID;
    int st = sort_init_once();
    if (st) return st;
    bh_ctx* c = new (std::nothrow) bh_ctx();
    if (!c) return BH_ERR_ALLOC;
    memset(c, 0, sizeof *c);
    c->magic = kCtxMagic;
    c->capacity = capacity;
    c->maxNodes = maxNodes;
    c->treeBlocks = (capacity + bh_tree_threads() - 1) / bh_tree_threads();
    c->sortTiles = (capacity + bh_sort_tile() - 1) / bh_sort_tile();
    c->sortStatusWords = 256 + (size_t)8 * c->sortTiles * 256;
    const size_t n = (size_t)capacity;
    const size_t m = (size_t)maxNodes;
    if ((st = dalloc(&c->keysTmp, n)) || (st = dalloc(&c->valsTmp, n)) ||
        (st = dalloc(&c->sortHist, 8 * 256)) || (st = dalloc(&c->sortStatus, c->sortStatusWords)) ||
        (st = dalloc(&c->bboxPartials, 6 * kBboxMaxGrid)) || (st = dalloc(&c->bboxTicket, 1)) ||
        (st = dalloc(&c->bboxPartials64, 4 * kBboxMaxGrid)) || (st = dalloc(&c->root64, 1)) ||
        (st = dalloc(&c->box, 1)) || (st = dalloc(&c->delta, n)) ||
        (st = dalloc(&c->blockLevel, (size_t)c->treeBlocks * BH_LEVEL_SLOTS)) ||
        (st = dalloc(&c->info, 1)) || (st = dalloc(&c->wn, m + 1)) || (st = dalloc(&c->nCB, m + 1)) ||
        (st = dalloc(&c->levelTotal, BH_LEVEL_SLOTS)) || (st = dalloc(&c->scanTicket, 1)) ||
        (st = dalloc(&c->nCom, m)) || (st = dalloc(&c->nParent, m)) ||
        (st = dalloc(&c->nFirst, m)) || (st = dalloc(&c->nCount, m)) || (st = dalloc(&c->nMeta, m)) ||
        (st = dalloc(&c->gridBar, 1)) || (st = dalloc(&c->ctr, 1)) ||
        (st = dalloc(&c->err, 1)) || (st = dalloc(&c->spill, bh_walk_spill_ints()))) {
        ctx_free(c);
        return st;
    }
    cudaError_t e;
    if ((e = cudaMemset(c->bboxTicket, 0, sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMemset(c->scanTicket, 0, sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMemset(c->err, 0, sizeof(int))) != cudaSuccess ||
        (e = cudaMemset(c->ctr, 0, sizeof(DevCounters))) != cudaSuccess ||
        (e = cudaMemset(c->info, 0, sizeof(DevTreeInfo))) != cudaSuccess ||
        (e = cudaMemset(c->root64, 0, sizeof(DevRoot))) != cudaSuccess) {
        ctx_free(c);
        return bh_note_cuda_error(e);
    }
    c->tb.capacity = capacity;
    c->initialised = true;
    *out = c;
    return BH_OK;
}

static bh_ctx* ctx_of(const treeState* st) {
    if (!st || !st->builder) return nullptr;
    bh_ctx* c = reinterpret_cast<bh_ctx*>(st->builder);
    return c->magic == kCtxMagic ? c : nullptr;
}

// Stable sort of n pairs by the low keyBits bits.  valsIn == NULL: values are
// the input positions.  histReady: sortHist already holds this input's digit
// counts (the keys kernel produced them).
static int ctx_sort(bh_ctx* c, const uint64_t* keysIn, const uint32_t* valsIn, uint64_t* keysOut,
                    uint32_t* valsOut, int n, int keyBits, bool histReady, cudaStream_t s) {
    const int npass = (keyBits + 7) / 8;
    const int tiles = (n + bh_sort_tile() - 1) / bh_sort_tile();
    BH_CUDA_TRY(cudaMemsetAsync(c->sortStatus, 0, sizeof(uint32_t) * (256 + (size_t)npass * tiles * 256), s));
    if (!histReady) {
        BH_CUDA_TRY(cudaMemsetAsync(c->sortHist, 0, sizeof(uint32_t) * npass * 256, s));
        BH_CUDA_TRY(bh_launch_sort_histogram(keysIn, n, c->sortHist, npass, s));
    }
    const uint64_t* ksrc = keysIn;
    const uint32_t* vsrc = valsIn;
    for (int p = 0; p < npass; p++) {
        const bool toOut = ((npass - 1 - p) % 2) == 0;
        uint64_t* kdst = toOut ? keysOut : c->keysTmp;
        uint32_t* vdst = toOut ? valsOut : c->valsTmp;
        uint32_t* status = c->sortStatus + 256 + (size_t)p * tiles * 256;
        int* counter = reinterpret_cast<int*>(c->sortStatus) + p;
        BH_CUDA_TRY(bh_launch_sort_pass(ksrc, vsrc, kdst, vdst, n, 8 * p, c->sortHist + 256 * p, status,
                                        counter, c->err, (p == 0 && vsrc == nullptr) ? 1 : 0, s));
        ksrc = kdst;
        vsrc = vdst;
    }
    return BH_OK;
}

// Octree of n sorted keys over sorted positions; optional reference export.
// ev (optional, 4 events) is recorded after the count, scan, nodes and mass
// kernels.
// boxes: one world box per system of a batch (nullptr: the context's box)
// beforeMass (optional): an event the upward pass waits for (the bodies'
// reorder, when it runs on another stream; the count, scan and node passes
// read only the sorted keys)
static int ctx_build(bh_ctx* c, const uint64_t* sortedKeys, const float4* sortedPos, int n, int bits,
                     node* exportTo, cudaStream_t s, cudaEvent_t* ev = nullptr, const DevBox* boxes = nullptr,
                     cudaEvent_t beforeMass = nullptr) {
    const int blocks = (n + bh_tree_threads() - 1) / bh_tree_threads();
    BH_CUDA_TRY(bh_launch_tree_count(sortedKeys, n, bits, c->delta, c->blockLevel, s));
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[0], s));
    BH_CUDA_TRY(bh_launch_tree_scan(c->blockLevel, blocks, n, bits, c->maxNodes, c->box, c->info, c->nCB,
                                    c->levelTotal, c->scanTicket, c->err, s));
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[1], s));
    BH_CUDA_TRY(bh_launch_tree_nodes(sortedKeys, c->delta, n, bits, c->blockLevel, c->info, c->maxNodes,
                                     boxes ? boxes : c->box, c->nCB, c->nParent, c->nFirst, c->nMeta, s));
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[2], s));
    if (beforeMass) BH_CUDA_TRY(cudaStreamWaitEvent(s, beforeMass, 0));
    BH_CUDA_TRY(bh_launch_tree_mass(sortedPos, c->delta, n, bits, c->info, c->nCB, c->nCom, c->wn, c->nFirst,
                                    c->nCount, c->gridBar, c->err, s));
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[3], s));
    if (exportTo)
        BH_CUDA_TRY(bh_launch_tree_export(sortedKeys, bits, c->info, c->wn, c->nParent, c->nFirst, c->nCount,
                                          c->nMeta, exportTo, n, c->maxNodes, s));
    return BH_OK;
}

static int ctx_walk(bh_ctx* c, const WalkArgs& a, bool fused, bool compensated, cudaStream_t s) {
    BH_CUDA_TRY(cudaMemsetAsync(c->ctr, 0, sizeof(DevCounters), s));
    BH_CUDA_TRY(bh_launch_walk(a, fused, compensated, s));
    return BH_OK;
}

static int ctx_read_errors(bh_ctx* c, cudaStream_t s, int* bits) {
    BH_CUDA_TRY(cudaMemcpyAsync(bits, c->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    BH_CUDA_TRY(cudaStreamSynchronize(s));
    return BH_OK;
}

// ======================================================== main.h (status)
extern "C" int bh_initialise_tree(treeState* st, int starCount, int paddedStarCount, int integrateBlocks) {
    if (!st || starCount <= 0 || paddedStarCount < starCount) return set_status(BH_ERR_INVALID);
    if ((long long)starCount * 8 > 0x7fffffffLL) return set_status(BH_ERR_INVALID);
    memset(st, 0, sizeof *st);
    const int maxNodes = 8 * starCount;  // basicGravity.cu:11
    bh_ctx* c = nullptr;
    int s = ctx_create(&c, starCount, maxNodes);
    if (s) return set_status(s);
    radixSorter* sorter = nullptr;
    s = bh_sorter_create(&sorter, starCount);
    if (s) {
        ctx_free(c);
        return set_status(s);
    }
    // the reference's builder carries a scan scratch and ping-pong flag and
    // offset arrays (tree.cu:241-284); keep them for per-level callers
    const size_t nb = (size_t)starCount;
    c->tb.tempStorageBytes = bh_scan_temp_bytes(starCount);
    if (cudaMalloc(&c->tb.tempStorage, c->tb.tempStorageBytes) != cudaSuccess || dalloc(&c->tb.flagsPing, nb) ||
        dalloc(&c->tb.flagsPong, nb) || dalloc(&c->tb.offsetsPing, nb) || dalloc(&c->tb.offsetsPong, nb)) {
        bh_sorter_destroy(sorter);
        ctx_free(c);
        return set_status(BH_ERR_ALLOC);
    }
    st->sorter = sorter;
    st->builder = &c->tb;
    st->starCount = starCount;
    st->maxNodes = maxNodes;
    st->treeBlocks = integrateBlocks;
    st->deepestLevel = 0;
    if ((s = dalloc(&st->nodes, (size_t)maxNodes)) || (s = dalloc(&st->mortonIn, (size_t)starCount)) ||
        (s = dalloc(&st->mortonOut, (size_t)starCount)) || (s = dalloc(&st->indexIn, (size_t)starCount)) ||
        (s = dalloc(&st->indexOut, (size_t)starCount)) || (s = dalloc(&st->boundingData[0], BOXBLOCKS)) ||
        (s = dalloc(&st->boundingData[1], BOXBLOCKS)) || (s = dalloc(&st->boundingData[2], 1)) ||
        (s = dalloc(&st->boundingData[3], 1)) || (s = dalloc(&st->sortedPosMassVals, (size_t)paddedStarCount)) ||
        (s = dalloc(&st->sortedVelVals, (size_t)paddedStarCount))) {
        c->ownedPos = st->sortedPosMassVals;
        c->ownedVel = st->sortedVelVals;
        bh_destroy_tree(st);
        return set_status(s);
    }
    c->ownedPos = st->sortedPosMassVals;
    c->ownedVel = st->sortedVelVals;
    cudaError_t e;
    if ((e = cudaMemset(st->sortedPosMassVals, 0, sizeof(float4) * paddedStarCount)) != cudaSuccess ||
        (e = cudaMemset(st->sortedVelVals, 0, sizeof(float3) * paddedStarCount)) != cudaSuccess ||
        (e = bh_launch_iota(st->indexIn, starCount, 0)) != cudaSuccess ||
        (e = cudaDeviceSynchronize()) != cudaSuccess) {
        bh_note_cuda_error(e);
        bh_destroy_tree(st);
        return set_status(BH_ERR_CUDA);
    }
    return set_status(BH_OK);
}

extern "C" int bh_destroy_tree(treeState* st) {
    if (!st) return set_status(BH_ERR_INVALID);
    bh_ctx* c = ctx_of(st);
    void* ptrs[] = {st->nodes, st->mortonIn, st->mortonOut, st->indexIn, st->indexOut,
                    st->boundingData[0], st->boundingData[1], st->boundingData[2], st->boundingData[3],
                    c ? c->ownedPos : nullptr, c ? c->ownedVel : nullptr};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (st->sorter) bh_sorter_destroy(st->sorter);
    if (c) ctx_free(c);
    memset(st, 0, sizeof *st);
    return set_status(BH_OK);
}

extern "C" int bh_build_tree(treeState* st, float4** pos, float3** vel, cudaStream_t s) {
    bh_ctx* c = ctx_of(st);
    if (!c || !pos || !vel || !*pos || !*vel) return set_status(BH_ERR_INVALID);
    const int n = st->starCount, bits = BH_MAX_BITS;
    int rc;
#define TRY(x)                       \
    do {                             \
        if ((rc = (x)) != BH_OK) return set_status(rc); \
    } while (0)
#define TRYC(x) TRY(((x) == cudaSuccess) ? BH_OK : bh_note_cuda_error(cudaGetLastError()))
    TRY(cudaMemsetAsync(c->err, 0, sizeof(int), s) == cudaSuccess ? BH_OK : BH_ERR_CUDA);
    // stage 1: world box (basicGravity.cu:143-155)
    TRYC(bh_launch_bbox(*pos, n, c->bboxPartials, c->bboxTicket, c->box, st->boundingData[2], st->boundingData[3],
                        bits, c->err, c->sortHist, 8 * 256, s, c->bboxPartials64, c->root64));
    // stage 2: keys (basicGravity.cu:176-183)
    worldBox none = {0, 0, 0, 0, 0};
    TRYC(bh_launch_morton(*pos, n, c->box, none, bits, st->mortonIn, st->indexIn, c->sortHist, 8, s));
    // stage 3: sort + reorder + pointer swap (basicGravity.cu:190-226)
    TRY(ctx_sort(c, st->mortonIn, st->indexIn, st->mortonOut, st->indexOut, n, 64, true, s));
    TRYC(bh_launch_reorder(*pos, *vel, nullptr, st->indexOut, st->sortedPosMassVals, st->sortedVelVals, nullptr,
                           n, s));
    float4* tp = *pos;
    *pos = st->sortedPosMassVals;
    st->sortedPosMassVals = tp;
    float3* tv = *vel;
    *vel = st->sortedVelVals;
    st->sortedVelVals = tv;
    // stages 4-5: octree + mass (basicGravity.cu:232-319)
    TRY(ctx_build(c, st->mortonOut, *pos, n, bits, st->nodes, s));
    // level table to the host (the reference keeps it in treeState)
    DevTreeInfo info;
    int errBits = 0;
    TRY(cudaMemcpyAsync(&info, c->info, sizeof info, cudaMemcpyDeviceToHost, s) == cudaSuccess ? BH_OK
                                                                                          : bh_note_cuda_error(cudaGetLastError()));
    TRY(ctx_read_errors(c, s, &errBits));
    for (int L = 0; L < 22; L++) {
        st->levelOffsets[L] = info.levelOffset[L];
        st->levelCount[L] = info.levelCount[L];
    }
    st->deepestLevel = info.deepest;
#undef TRY
#undef TRYC
    return set_status(status_from_bits(errBits));
}

extern "C" int bh_calculate_acceleration(const float4* pos, const treeState* st, float3* acc, float eps2, float G,
                                         float theta, int starCount, cudaStream_t s) {
    bh_ctx* c = ctx_of(st);
    if (!c || !pos || !acc || starCount != st->starCount) return set_status(BH_ERR_INVALID);
    WalkArgs a;
    memset(&a, 0, sizeof a);
    a.pos = pos;
    a.n = starCount;
    a.wn = c->wn;
    a.theta = theta;
    a.eps2 = eps2;
    a.G = G;
    a.accOut = acc;
    a.ctr = c->ctr;
    a.err = c->err;
    a.spill = c->spill;
    return set_status(ctx_walk(c, a, false, true, s));
}

extern "C" int bh_position_updater(float4* pos, float3* vel, const float3* acc, int n, float dt, cudaStream_t s) {
    if (!pos || !vel || !acc || n <= 0) return set_status(BH_ERR_INVALID);
    cudaError_t e = bh_launch_kick_drift(pos, vel, acc, n, dt, s);
    return set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

extern "C" int bh_morton_encode(const float4* pos, uint64_t* keys, uint32_t* idx, int n, worldBox box, int bits,
                                cudaStream_t s) {
    if (!pos || !keys || n <= 0 || bits < 1 || bits > BH_MAX_BITS) return set_status(BH_ERR_INVALID);
    cudaError_t e = bh_launch_morton(pos, n, nullptr, box, bits, keys, idx, nullptr, 0, s);
    return set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

extern "C" int bh_world_box(const float4* pos, int n, int bits, worldBox* boxOut, float3* minOut, float3* maxOut,
                            cudaStream_t s) {
    if (!pos || n <= 0 || !boxOut || bits < 1 || bits > BH_MAX_BITS) return set_status(BH_ERR_INVALID);
    float3* scratch = nullptr;
    int rc = dalloc(&scratch, 2 * BOXBLOCKS + 2);
    if (rc) return set_status(rc);
    cudaError_t e;
    float3 mn, mx;
    if ((e = bh_launch_local_minmax(pos, (unsigned)n, scratch, scratch + BOXBLOCKS, BOXBLOCKS, s)) != cudaSuccess ||
        (e = bh_launch_global_minmax(scratch, scratch + BOXBLOCKS, BOXBLOCKS, scratch + 2 * BOXBLOCKS,
                                     scratch + 2 * BOXBLOCKS + 1, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&mn, scratch + 2 * BOXBLOCKS, sizeof mn, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&mx, scratch + 2 * BOXBLOCKS + 1, sizeof mx, cudaMemcpyDeviceToHost, s)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess) {
        cudaFree(scratch);
        return set_status(bh_note_cuda_error(e));
    }
    cudaFree(scratch);
    // basicGravity.cu:90-112
    const float w = mx.x - mn.x, h = mx.y - mn.y, d = mx.z - mn.z;
    const float extent = fmaxf(w, fmaxf(h, d));
    boxOut->minX = mn.x;
    boxOut->minY = mn.y;
    boxOut->minZ = mn.z;
    boxOut->extent = extent;
    boxOut->scale = (float)((1u << bits) - 1u) / extent;
    if (minOut) *minOut = mn;
    if (maxOut) *maxOut = mx;
    if (!(extent > 0.0f) || !isfinite(extent)) return set_status(BH_ERR_DEGENERATE_BOX);
    return set_status(BH_OK);
}

// ===================================================== main.h (reference)
static void die(const char* msg) {
    printf("%s", msg);
    fflush(stdout);
    exit(-1);
}

extern "C" void initialiseTree(treeState* state, int starCount, int paddedStarCount, int integrateBlocks) {
    int s = bh_initialise_tree(state, starCount, paddedStarCount, integrateBlocks);
    if (s) {
        char msg[256];
        snprintf(msg, sizeof msg, "ERROR: initialiseTree failed: %s %s\n", bh_status_string(s), g_cuda_err);
        die(msg);
    }
}

extern "C" void destroyTree(treeState* state) { bh_destroy_tree(state); }

extern "C" void createWorldBox(const float4* cudaPositionMassVals, const int starCount, float3* cudaMinCorner,
                               float3* cudaMaxCorner, float3* cudaOutputMin, float3* cudaOutputMax,
                               worldBox* outputWorldBox) {
    cudaError_t e;
    float3 mn, mx;
    if ((e = bh_launch_local_minmax(cudaPositionMassVals, (unsigned)starCount, cudaMinCorner, cudaMaxCorner,
                                    BOXBLOCKS, 0)) != cudaSuccess ||
        (e = bh_launch_global_minmax(cudaMinCorner, cudaMaxCorner, BOXBLOCKS, cudaOutputMin, cudaOutputMax, 0)) !=
            cudaSuccess ||
        (e = cudaMemcpy(&mn, cudaOutputMin, sizeof mn, cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (e = cudaMemcpy(&mx, cudaOutputMax, sizeof mx, cudaMemcpyDeviceToHost)) != cudaSuccess) {
        printf("\nCUDA ERROR at: %s:%d\n%s\n", __FILE__, __LINE__, cudaGetErrorString(e));
        fflush(stdout);
        exit(-1);
    }
    const float width = mx.x - mn.x, height = mx.y - mn.y, depth = mx.z - mn.z;
    const float extent = fmaxf(width, fmaxf(height, depth));
    outputWorldBox->extent = extent;
    outputWorldBox->minX = mn.x;
    outputWorldBox->minY = mn.y;
    outputWorldBox->minZ = mn.z;
    outputWorldBox->scale = (float)((1u << 21) - 1u) / extent;
}

extern "C" void buildTree(treeState* tree, float4** cudaPosMasVals, float3** cudaVelVals) {
    int s = bh_build_tree(tree, cudaPosMasVals, cudaVelVals, 0);
    if (s == BH_ERR_DEGENERATE_BOX || s == BH_ERR_NONFINITE) die("\nERROR: rootBox failed to initialise.\n");
    if (s == BH_ERR_TREE_OVERFLOW) {
        DevTreeInfo info;
        bh_ctx* c = ctx_of(tree);
        int level = 0;
        if (c && cudaMemcpy(&info, c->info, sizeof info, cudaMemcpyDeviceToHost) == cudaSuccess)
            level = info.overflowLevel;
        char msg[128];
        snprintf(msg, sizeof msg, "ERROR: Node array overflow at level: %d", level);
        die(msg);
    }
    if (s) {
        char msg[256];
        snprintf(msg, sizeof msg, "ERROR: buildTree failed: %s %s\n", bh_status_string(s), g_cuda_err);
        die(msg);
    }
}

extern "C" int roundNumberToMultiple(int number, int multiple) {
    if (multiple == 0) return number;
    if (multiple < 0) die("Rounding up to a negative number is undefined\n");
    const int r = number % multiple;
    return r == 0 ? number : number + multiple - r;
}

extern "C" void blockNumCalculator(int* accelerationBlocks, int* treeBuilderBlocks, int* integrateBlocks,
                                   int* paddedStarCount, int* integrationThreadsPerBlock,
                                   int* treeBuilderThreadsPerBlock, int starCount) {
    // basicGravity.cu:374-427 (without the CPU-core printout)
    *integrationThreadsPerBlock = 256;
    *treeBuilderThreadsPerBlock = 256;
    *paddedStarCount = roundNumberToMultiple(starCount, WARPTHREADS);
    *accelerationBlocks = *paddedStarCount / WARPTHREADS + (starCount % WARPTHREADS ? 1 : 0);
    *integrateBlocks = *paddedStarCount / 256 + (starCount % 256 ? 1 : 0);
    *treeBuilderBlocks = *paddedStarCount / 256 + (starCount % 256 ? 1 : 0);
}

// ===================================================== tree.h launchers
extern "C" void mortonEncode(const float4* posMassVals, uint64_t* mortonCodes, uint32_t* originalIndex, int NStars,
                             worldBox rootBox, cudaStream_t stream) {
    bh_morton_encode(posMassVals, mortonCodes, originalIndex, NStars, rootBox, BH_MAX_BITS, stream);
}

extern "C" void localMinMaxFinder(const float4* posMassVals, unsigned int N, float3* minCorner, float3* maxCorner,
                                  cudaStream_t stream) {
    cudaError_t e = bh_launch_local_minmax(posMassVals, N, minCorner, maxCorner, BOXBLOCKS, stream);
    set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

extern "C" void globalMinMaxReducer(const float3* minCorner, const float3* maxCorner, int count, float3* outMin,
                                    float3* outMax, cudaStream_t stream) {
    cudaError_t e = bh_launch_global_minmax(minCorner, maxCorner, count, outMin, outMax, stream);
    set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

extern "C" void calculateAcceleration(const float4* positionMassArray, treeState tree, float3* accelVals,
                                      float antiSingularitySquared, float GVal, float theta, int starCount,
                                      cudaStream_t stream) {
    bh_calculate_acceleration(positionMassArray, &tree, accelVals, antiSingularitySquared, GVal, theta, starCount,
                              stream);
}

extern "C" void positionUpdater(float4* positionMassArray, float3* velocityVals, float3* accelerationVals,
                                int starCount, float timeStep, cudaStream_t stream) {
    bh_position_updater(positionMassArray, velocityVals, accelerationVals, starCount, timeStep, stream);
}

// ================================================= sorting.h
// A sorter owns the three-buffer scratch of the onesweep sort.
struct bh_sorter {
    radixSorter pub;  // first member: the pointer callers hold
    uint32_t magic;
    bh_ctx* ctx;      // sort scratch lives in a tree-less context
};
static const uint32_t kSorterMagic = 0x5047A11Du;

static bh_ctx* sort_ctx_create(int capacity) {
    int st = sort_init_once();
    if (st) return nullptr;
    bh_ctx* c = new (std::nothrow) bh_ctx();
    if (!c) return nullptr;
    memset(c, 0, sizeof *c);
    c->magic = kCtxMagic;
    c->capacity = capacity;
    c->sortTiles = (capacity + bh_sort_tile() - 1) / bh_sort_tile();
    c->sortStatusWords = 256 + (size_t)8 * c->sortTiles * 256;
    if (dalloc(&c->keysTmp, (size_t)capacity) || dalloc(&c->valsTmp, (size_t)capacity) ||
        dalloc(&c->sortHist, 8 * 256) || dalloc(&c->sortStatus, c->sortStatusWords) || dalloc(&c->err, 1)) {
        ctx_free(c);
        return nullptr;
    }
    cudaMemset(c->err, 0, sizeof(int));
    return c;
}

extern "C" int bh_sorter_create(radixSorter** out, int maxCount) {
    if (!out) return set_status(BH_ERR_INVALID);
    *out = nullptr;
    if (maxCount <= 0) return set_status(BH_ERR_INVALID);
    bh_sorter* s = new (std::nothrow) bh_sorter();
    if (!s) return set_status(BH_ERR_ALLOC);
    s->ctx = sort_ctx_create(maxCount);
    if (!s->ctx) {
        delete s;
        return set_status(BH_ERR_ALLOC);
    }
    s->magic = kSorterMagic;
    s->pub.tempStorage = s->ctx->keysTmp;
    s->pub.tempStorageBytes = (size_t)maxCount * 12 + s->ctx->sortStatusWords * 4 + 8 * 256 * 4;
    s->pub.capacity = maxCount;
    *out = &s->pub;
    return set_status(BH_OK);
}

static bh_sorter* sorter_of(radixSorter* r) {
    if (!r) return nullptr;
    bh_sorter* s = reinterpret_cast<bh_sorter*>(r);
    return s->magic == kSorterMagic ? s : nullptr;
}

extern "C" int bh_radix_sort_pairs(radixSorter* sorter, const uint64_t* keysIn, uint64_t* keysOut,
                                   const uint32_t* valsIn, uint32_t* valsOut, int n, int keyBits, cudaStream_t s) {
    bh_sorter* so = sorter_of(sorter);
    if (!so || !keysIn || !keysOut || !valsIn || !valsOut) return set_status(BH_ERR_INVALID);
    if (n <= 0 || n > sorter->capacity || keyBits < 1 || keyBits > 64) return set_status(BH_ERR_INVALID);
    return set_status(ctx_sort(so->ctx, keysIn, valsIn, keysOut, valsOut, n, keyBits, false, s));
}

// The device error word of a sorter's passes (a look-back wait that gave up
// sets BH_ERR_TIMEOUT there): read after the work queued on `s`, then cleared.
extern "C" int bh_sorter_errors(radixSorter* sorter, int* errorBits, cudaStream_t s) {
    bh_sorter* so = sorter_of(sorter);
    if (!so) return set_status(BH_ERR_INVALID);
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, so->ctx->err, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaMemsetAsync(so->ctx->err, 0, sizeof(int), s);
    if (e != cudaSuccess) return set_status(bh_note_cuda_error(e));
    if (errorBits) *errorBits = h;
    return set_status(status_from_bits(h));
}

// Failure detection without a fault: the look-back wait run against this
// sorter's own status words, with a predecessor tile that never publishes.
// It gives up and leaves BH_ERR_TIMEOUT in the sorter's error word, where
// bh_sorter_errors() must find it.
extern "C" int bh_selftest_sorter_timeout(radixSorter* sorter, cudaStream_t s) {
    bh_sorter* so = sorter_of(sorter);
    if (!so) return set_status(BH_ERR_INVALID);
    cudaError_t e = cudaMemsetAsync(so->ctx->sortStatus, 0, sizeof(uint32_t) * 2 * 256, s);
    if (e == cudaSuccess) e = bh_launch_lookback_selftest(so->ctx->sortStatus, so->ctx->err, s);
    return set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

extern "C" int bh_sorter_destroy(radixSorter* sorter) {
    bh_sorter* s = sorter_of(sorter);
    if (!s) return set_status(BH_ERR_INVALID);
    ctx_free(s->ctx);
    s->magic = 0;
    delete s;
    return set_status(BH_OK);
}

extern "C" radixSorter* sorterCreate(int maxCount) {
    if (maxCount <= 0) die("ERROR: Attempted to create a radix sort over an array of <= 0 elements.\n");
    radixSorter* r = nullptr;
    if (bh_sorter_create(&r, maxCount)) die("ERROR: Radix sorter creation failed.\n");
    return r;
}

extern "C" void radixSortPairs(radixSorter* sorter, const uint64_t* keysIn, uint64_t* keysOut,
                               const uint32_t* valsIn, uint32_t* valsOut, int numCount) {
    if (!sorter) die("ERROR: Sorter struct passed to radix sort was uninitialised");
    if (numCount <= 0 || numCount > sorter->capacity)
        die("ERROR: Length of array to sort conflicts with capacity of radix sorter.\n");
    int s = bh_radix_sort_pairs(sorter, keysIn, keysOut, valsIn, valsOut, numCount, 64, 0);
    // the reference's form stops on every error: the passes' device error
    // word is read back at once (this waits for the sort)
    if (s == BH_OK) s = bh_sorter_errors(sorter, nullptr, 0);
    if (s) {
        char msg[256];
        snprintf(msg, sizeof msg, "\nCUDA ERROR: %s %s\n", bh_status_string(s), s == BH_ERR_CUDA ? g_cuda_err : "");
        die(msg);
    }
}

extern "C" void sorterDestroyer(radixSorter* sorter) {
    if (!sorter) die("ERROR: Attempted to delete non-existant sorter.\n");
    bh_sorter_destroy(sorter);
}

extern "C" void reorderParticles(const float4* posIn, const float3* velIn, float4* posOut, float3* velOut,
                                 uint32_t* originalIndex, int starCount, cudaStream_t stream) {
    cudaError_t e = bh_launch_reorder(posIn, velIn, nullptr, originalIndex, posOut, velOut, nullptr, starCount, stream);
    set_status(e == cudaSuccess ? BH_OK : bh_note_cuda_error(e));
}

// ================================================================ bh_sim
struct bh_sim {
    bh_ctx* ctx;
    bh_params prm;
    cudaStream_t stream;
    bool ownStream;
    int capacity;
    int n;
    float4 *posA, *posB;
    float3 *velA, *velB;
    uint32_t *idA, *idB;
    uint64_t *keysA, *keysB;
    uint32_t* perm;
    float3* acc;
    node* aos;
    float3* corner;  // global min, max
    float *aMagA, *aMagB;  // |a| per body from the last walk (A: current order, B: sorted)
    float2* groupParam;    // per-group (theta, alpha) of the learned criterion
    int* groupLen;         // interaction-list length of each walk group (last walk)
    int* groupOrder;       // the next walk's group order (longest first)
    int* orderHist;        // its per-block bin counts (scratch)
    bool lengthsValid;     // groupLen holds the last walk's lengths of the current grouping
    int walkStack;         // walk stack entries per warp in shared memory (0: default)
    float* feat;           // per-group features of the learned criterion
    float* mlp;            // its MLP (BH_MLP_PARAMS floats)
    bool mlpLoaded;
    bool aMagValid;        // aMagA holds the last step's |a| for the current bodies
    bool aMagIdOrder;      // ... in body-id order (left by bh_sim_step_host)
    // batch of independent systems (systems == 0: one system)
    int systems;
    int sysBits;           // bits of the system index above the Morton bits
    int* segOffHost;       // systems + 1 body offsets (host)
    int* segOff;           // the same on the device
    uint16_t* sysOf;       // system of every body slot (device)
    DevBox* boxes;         // world box per system (device)
    int4* groupTable[2];   // walk groups of 32 / 64 bodies: first body, count, root node (device)
    // bh_sim_step_host: velocities upload on a second stream while the keys
    // and the sort run; the reorder waits for them
    cudaStream_t copyStream;
    cudaEvent_t velReady, mainReady;
    // bh_sim_step_host_sorted: the ids go up on the copy stream too (the
    // reorder waits for them), the velocities after them, gathered into
    // sorted order there once the sort is done (the walk waits for that);
    // |a| is kept by body id between calls (aMagById), and the last step's
    // walk may write the result into the caller's mapped host arrays
    cudaEvent_t idsReady;
    bool velSeparate;
    float* aMagById;
    int* errHost;  // page-locked copy of the device error word
    float4* hostPos;
    float3* hostVel;
    uint32_t* hostId;
    // a step's side branch runs beside the tree build: the group order (fork
    // at the step's start), the reorder (after the sort) and the learned
    // criterion; the upward pass waits for the reorder, the walk joins all
    cudaStream_t side;
    cudaEvent_t evFork, evSorted, evReordered, evJoin;
    cudaEvent_t waitBeforeReorder;  // set only for that one eagerly enqueued step
    int groups[2];
    treeState ts;
    cudaGraphExec_t graph;
    bool graphReady;
};

static void sim_drop_graph(bh_sim* s) {
    if (s->graphReady) cudaGraphExecDestroy(s->graph);
    s->graphReady = false;
}

extern "C" int bh_sim_create(bh_sim** out, int capacity, const bh_params* prm, cudaStream_t stream) {
    if (!out) return set_status(BH_ERR_INVALID);
    *out = nullptr;
    if (capacity <= 0 || (long long)capacity * 8 > 0x7fffffffLL) return set_status(BH_ERR_INVALID);
    bh_params p;
    if (prm) p = *prm;
    else bh_params_default(&p);
    int rc = check_params(&p);
    if (rc) return set_status(rc);
    bh_sim* s = new (std::nothrow) bh_sim();
    if (!s) return set_status(BH_ERR_ALLOC);
    memset(s, 0, sizeof *s);
    s->prm = p;
    s->capacity = capacity;
    if ((rc = ctx_create(&s->ctx, capacity, 8 * capacity))) {
        delete s;
        return set_status(rc);
    }
    const size_t n = (size_t)capacity;
    if ((rc = dalloc(&s->posA, n)) || (rc = dalloc(&s->posB, n)) || (rc = dalloc(&s->velA, n)) ||
        (rc = dalloc(&s->velB, n)) || (rc = dalloc(&s->idA, n)) || (rc = dalloc(&s->idB, n)) ||
        (rc = dalloc(&s->keysA, n)) || (rc = dalloc(&s->keysB, n)) || (rc = dalloc(&s->perm, n)) ||
        (rc = dalloc(&s->acc, n)) || (rc = dalloc(&s->corner, 2)) || (rc = dalloc(&s->aMagA, n)) ||
        (rc = dalloc(&s->aMagB, n)) || (rc = dalloc(&s->groupParam, (n + 31) / 32)) ||
        (rc = dalloc(&s->groupLen, (n + 31) / 32)) || (rc = dalloc(&s->groupOrder, (n + 31) / 32)) ||
        (rc = dalloc(&s->orderHist, bh_group_order_hist_ints((n + 31) / 32))) ||
        (rc = dalloc(&s->feat, (n + 31) / 32 * BH_GROUP_FEATURES)) || (rc = dalloc(&s->mlp, BH_MLP_PARAMS)) ||
        (p.exportNodes && (rc = dalloc(&s->aos, (size_t)s->ctx->maxNodes)))) {
        bh_sim_destroy(s);
        return set_status(rc);
    }
    if (cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->evFork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->evReordered, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->evSorted, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->evJoin, cudaEventDisableTiming) != cudaSuccess) {
        bh_note_cuda_error(cudaGetLastError());
        bh_sim_destroy(s);
        return set_status(BH_ERR_CUDA);
    }
    if (cudaMemset(s->groupLen, 0, sizeof(int) * ((n + 31) / 32)) != cudaSuccess) {
        bh_note_cuda_error(cudaGetLastError());
        bh_sim_destroy(s);
        return set_status(BH_ERR_CUDA);
    }
    if (stream) {
        s->stream = stream;
    } else {
        cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            bh_note_cuda_error(e);
            bh_sim_destroy(s);
            return set_status(BH_ERR_CUDA);
        }
        s->ownStream = true;
    }
    *out = s;
    return set_status(BH_OK);
}

extern "C" int bh_sim_create_batch(bh_sim** out, int systems, const int* counts, const bh_params* prm,
                                   cudaStream_t stream) {
    if (!out) return set_status(BH_ERR_INVALID);
    *out = nullptr;
    if (systems < 1 || systems > 65535 || !counts) return set_status(BH_ERR_INVALID);
    long long total = 0;
    for (int k = 0; k < systems; k++) {
        if (counts[k] <= 0) return set_status(BH_ERR_INVALID);
        total += counts[k];
    }
    if (total * 8 > 0x7fffffffLL) return set_status(BH_ERR_INVALID);
    bh_params p;
    if (prm) p = *prm;
    else bh_params_default(&p);
    if (p.macMode != 0 || p.exportNodes) return set_status(BH_ERR_INVALID);
    bh_sim* s = nullptr;
    int rc = bh_sim_create(&s, (int)total, &p, stream);
    if (rc) return rc;
    int sysBits = 0;
    while ((1 << sysBits) < systems) sysBits++;
    s->systems = systems;
    s->sysBits = sysBits;
    s->n = 0;
    // groups of 32 (and of 64) bodies that never straddle two systems;
    // system k's tree is rooted at node k (roots are level 0, in system order)
    s->segOffHost = (int*)malloc(sizeof(int) * (systems + 1));
    uint16_t* so = (uint16_t*)malloc(sizeof(uint16_t) * total);
    if (!s->segOffHost || !so) rc = BH_ERR_ALLOC;
    if (!rc) {
        int off = 0;
        for (int k = 0; k < systems; k++) {
            s->segOffHost[k] = off;
            for (int b = 0; b < counts[k]; b++) so[off + b] = (uint16_t)k;
            off += counts[k];
        }
        s->segOffHost[systems] = off;
    }
    if (!rc && ((rc = dalloc(&s->segOff, systems + 1)) || (rc = dalloc(&s->sysOf, (size_t)total)) ||
                (rc = dalloc(&s->boxes, systems))))
        ;
    if (!rc) {
        cudaError_t e = cudaMemcpy(s->segOff, s->segOffHost, sizeof(int) * (systems + 1), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->sysOf, so, sizeof(uint16_t) * total, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) rc = bh_note_cuda_error(e);
    }
    for (int t = 0; t < 2 && !rc; t++) {
        const int width = t ? 64 : 32;
        int groups = 0;
        for (int k = 0; k < systems; k++) groups += (counts[k] + width - 1) / width;
        int4* gt = (int4*)malloc(sizeof(int4) * groups);
        if (!gt) {
            rc = BH_ERR_ALLOC;
            break;
        }
        int g = 0;
        for (int k = 0; k < systems; k++)
            for (int b = 0; b < counts[k]; b += width)
                gt[g++] = make_int4(s->segOffHost[k] + b, counts[k] - b < width ? counts[k] - b : width, k, 0);
        s->groups[t] = groups;
        // per-group lengths and order: a batch can have more groups than
        // bodies / 32 (every system ends in a partial group)
        if (t == 0 && groups > (s->capacity + 31) / 32) {
            cudaFree(s->groupLen);
            cudaFree(s->groupOrder);
            cudaFree(s->orderHist);
            s->groupLen = nullptr;
            s->groupOrder = nullptr;
            s->orderHist = nullptr;
            rc = dalloc(&s->groupLen, groups);
            if (!rc) rc = dalloc(&s->groupOrder, groups);
            if (!rc) rc = dalloc(&s->orderHist, bh_group_order_hist_ints(groups));
            if (!rc && cudaMemset(s->groupLen, 0, sizeof(int) * groups) != cudaSuccess)
                rc = bh_note_cuda_error(cudaGetLastError());
            if (rc) {
                free(gt);
                break;
            }
        }
        rc = dalloc(&s->groupTable[t], groups);
        if (!rc && cudaMemcpy(s->groupTable[t], gt, sizeof(int4) * groups, cudaMemcpyHostToDevice) != cudaSuccess)
            rc = bh_note_cuda_error(cudaGetLastError());
        free(gt);
    }
    free(so);
    if (rc) {
        bh_sim_destroy(s);
        return set_status(rc);
    }
    *out = s;
    return set_status(BH_OK);
}

extern "C" int bh_sim_systems(const bh_sim* s, int* systems, int* offsets) {
    if (!s || !systems) return set_status(BH_ERR_INVALID);
    *systems = s->systems;
    if (offsets && s->systems)
        for (int k = 0; k <= s->systems; k++) offsets[k] = s->segOffHost[k];
    return set_status(BH_OK);
}

extern "C" int bh_sim_destroy(bh_sim* s) {
    if (!s) return set_status(BH_ERR_INVALID);
    if (s->stream) cudaStreamSynchronize(s->stream);
    sim_drop_graph(s);
    void* ptrs[] = {s->posA, s->posB, s->velA, s->velB, s->idA, s->idB, s->keysA, s->keysB, s->perm, s->acc, s->aos,
                    s->corner, s->aMagA, s->aMagB, s->aMagById, s->groupParam, s->groupLen, s->groupOrder, s->orderHist, s->feat, s->mlp,
                    s->segOff, s->sysOf,
                    s->boxes, s->groupTable[0], s->groupTable[1]};
    free(s->segOffHost);
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s->ctx) ctx_free(s->ctx);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->evFork) cudaEventDestroy(s->evFork);
    if (s->evReordered) cudaEventDestroy(s->evReordered);
    if (s->evSorted) cudaEventDestroy(s->evSorted);
    if (s->evJoin) cudaEventDestroy(s->evJoin);
    if (s->copyStream) cudaStreamDestroy(s->copyStream);
    if (s->velReady) cudaEventDestroy(s->velReady);
    if (s->mainReady) cudaEventDestroy(s->mainReady);
    if (s->idsReady) cudaEventDestroy(s->idsReady);
    if (s->errHost) cudaFreeHost(s->errHost);
    if (s->ownStream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return set_status(BH_OK);
}

extern "C" int bh_sim_set_params(bh_sim* s, const bh_params* p) {
    if (!s) return set_status(BH_ERR_INVALID);
    int rc = check_params(p);
    if (rc) return set_status(rc);
    if (s->systems && (p->macMode != 0 || p->exportNodes)) return set_status(BH_ERR_INVALID);
    if (p->exportNodes && !s->aos) {
        rc = dalloc(&s->aos, (size_t)s->ctx->maxNodes);
        if (rc) return set_status(rc);
    }
    s->prm = *p;
    sim_drop_graph(s);
    return set_status(BH_OK);
}

extern "C" int bh_sim_get_params(const bh_sim* s, bh_params* p) {
    if (!s || !p) return set_status(BH_ERR_INVALID);
    *p = s->prm;
    return set_status(BH_OK);
}

extern "C" cudaStream_t bh_sim_stream(const bh_sim* s) { return s ? s->stream : nullptr; }

extern "C" int bh_sim_load(bh_sim* s, const float4* pos, const float3* vel, int n, int fromHost) {
    if (!s || !pos || !vel || n <= 0 || n > s->capacity) return set_status(BH_ERR_INVALID);
    if (s->systems && n != s->capacity) return set_status(BH_ERR_INVALID);  // a batch loads all its bodies
    const cudaMemcpyKind k = fromHost ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    BH_CUDA_TRY(cudaMemcpyAsync(s->posA, pos, sizeof(float4) * n, k, s->stream));
    BH_CUDA_TRY(cudaMemcpyAsync(s->velA, vel, sizeof(float3) * n, k, s->stream));
    BH_CUDA_TRY(bh_launch_iota(s->idA, n, s->stream));
    BH_CUDA_TRY(cudaMemsetAsync(s->ctx->err, 0, sizeof(int), s->stream));
    if (n != s->n || s->aMagValid) sim_drop_graph(s);
    s->n = n;
    s->aMagValid = false;
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_store(bh_sim* s, float4* pos, float3* vel, int toHost) {
    if (!s || s->n <= 0) return set_status(BH_ERR_INVALID);
    const int n = s->n;
    BH_CUDA_TRY(bh_launch_scatter_by_id(s->posA, s->velA, nullptr, s->idA, s->posB, s->velB, nullptr, n, s->stream));
    const cudaMemcpyKind k = toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    if (pos) BH_CUDA_TRY(cudaMemcpyAsync(pos, s->posB, sizeof(float4) * n, k, s->stream));
    if (vel) BH_CUDA_TRY(cudaMemcpyAsync(vel, s->velB, sizeof(float3) * n, k, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_device_state(bh_sim* s, float4** pos, float3** vel, uint32_t** ids, int* n) {
    if (!s) return set_status(BH_ERR_INVALID);
    if (pos) *pos = s->posA;
    if (vel) *vel = s->velA;
    if (ids) *ids = s->idA;
    if (n) *n = s->n;
    return set_status(BH_OK);
}

// the relative / learned criterion needs |a| of the last step
static bool sim_relative(const bh_sim* s) { return s->prm.macMode != 0 && s->aMagValid; }

// Morton bits per axis: a batch keeps its system index above them, so
// 3 * bits + sysBits must fit the 64-bit key.
static int sim_bits(const bh_sim* s) {
    const int b = s->prm.bitsPerAxis;
    if (!s->systems) return b;
    const int room = (64 - s->sysBits) / 3;
    return b < room ? b : room;
}

// build stages shared by a step and an acceleration query: A -> sorted B.
// ev (optional, kProfileStages + 1 events) marks the stage boundaries:
// keys | sort | reorder | tree count | tree scan | tree nodes | tree mass |
// (learned criterion, walk: recorded by sim_enqueue_step).
static const int kProfileStages = 9;
// side (optional, with afterReorder): the stream the reorder runs on, beside
// the tree's count, scan and node passes; afterReorder is recorded on it after
// the reorder and the upward pass waits for it.  afterSort is recorded on the
// main stream once the keys are sorted (needed with side).
static int sim_enqueue_build(bh_sim* s, cudaEvent_t* ev, cudaEvent_t afterReorder = nullptr,
                             cudaStream_t side = nullptr, cudaEvent_t afterSort = nullptr) {
    bh_ctx* c = s->ctx;
    const int n = s->n, bits = sim_bits(s);
    const int keyBits = 3 * bits + (s->systems ? s->sysBits : 0);
    const int npass = (keyBits + 7) / 8;
    cudaStream_t st = s->stream;
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[0], st));
    worldBox none = {0, 0, 0, 0, 0};
    if (s->systems) {
        BH_CUDA_TRY(bh_launch_bbox_segments(s->posA, s->segOff, s->systems, s->boxes, bits, c->err, c->sortHist,
                                            npass * 256, st));
        BH_CUDA_TRY(bh_launch_morton(s->posA, n, s->boxes, none, bits, s->keysA, nullptr, c->sortHist, npass, st,
                                     s->sysOf));
    } else {
        BH_CUDA_TRY(bh_launch_bbox(s->posA, n, c->bboxPartials, c->bboxTicket, c->box, s->corner, s->corner + 1,
                                   bits, c->err, c->sortHist, npass * 256, st, c->bboxPartials64, c->root64));
        BH_CUDA_TRY(bh_launch_morton(s->posA, n, c->box, none, bits, s->keysA, nullptr, c->sortHist, npass, st));
    }
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[1], st));
    int rc = ctx_sort(c, s->keysA, nullptr, s->keysB, s->perm, n, keyBits, true, st);
    if (rc) return rc;
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[2], st));
    cudaStream_t rs = st;  // the reorder's stream
    if (side) {
        BH_CUDA_TRY(cudaEventRecord(afterSort, st));
        BH_CUDA_TRY(cudaStreamWaitEvent(side, afterSort, 0));
        rs = side;
    }
    if (s->waitBeforeReorder) BH_CUDA_TRY(cudaStreamWaitEvent(rs, s->waitBeforeReorder, 0));
    // (velocities gathered separately, on the copy stream, when velSeparate)
    float3* const velIn = s->velSeparate ? nullptr : s->velA;
    float3* const velOut = s->velSeparate ? nullptr : s->velB;
    BH_CUDA_TRY(bh_launch_reorder(s->posA, velIn, s->idA, s->perm, s->posB, velOut, s->idB, n, rs,
                                  sim_relative(s) ? s->aMagA : nullptr, sim_relative(s) ? s->aMagB : nullptr));
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[3], st));
    if (afterReorder) BH_CUDA_TRY(cudaEventRecord(afterReorder, rs));
    return ctx_build(c, s->keysB, s->posB, n, bits, s->prm.exportNodes ? s->aos : nullptr, st, ev ? ev + 4 : nullptr,
                     s->systems ? s->boxes : nullptr, side ? afterReorder : nullptr);
}

// learned criterion: group features and the per-group choice of (theta,
// alpha), after the build and before the walk
// (the features need the reordered bodies, |a|, keys, box and FP64 root, not
// the tree, so a step runs them beside the tree build)
static bool sim_learned_active(const bh_sim* s) { return sim_relative(s) && s->prm.macMode == 2; }

static int sim_enqueue_learned(bh_sim* s, cudaStream_t st) {
    if (!sim_learned_active(s)) return BH_OK;
    if (!s->mlpLoaded) return BH_ERR_INVALID;
    bh_ctx* c = s->ctx;
    const int groups = (s->n + 31) / 32;
    BH_CUDA_TRY(bh_launch_group_features(s->posB, s->aMagB, s->keysB, s->n, s->prm.bitsPerAxis, c->box, c->root64,
                                         s->prm.G, s->feat, st));
    BH_CUDA_TRY(bh_launch_mac_select(s->mlp, s->feat, groups, log10f(s->prm.errTarget), s->prm.theta, s->groupParam,
                                     st));
    return BH_OK;
}

// groups of the walk as it runs now: 32 or 64 bodies, batches by table
static int sim_walk_groups(const bh_sim* s) {
    const int t = s->prm.groupWidth == 64 ? 1 : 0;
    if (s->systems) return s->groups[t];
    return t ? (s->n + 63) / 64 : (s->n + 31) / 32;
}

// opening criterion of the walk over the sorted bodies
static void sim_set_criterion(bh_sim* s, WalkArgs& a) {
    a.leafSize = s->prm.leafSize;
    a.nFirst = s->ctx->nFirst;
    a.groupWidth = s->prm.groupWidth;
    a.groupParamCount = (s->n + 31) / 32;
    a.groupLen = s->groupLen;
    a.stackSmem = s->walkStack;
    if (s->systems) {
        const int t = s->prm.groupWidth == 64 ? 1 : 0;
        a.groupTable = s->groupTable[t];
        a.groups = s->groups[t];
    }
    if (!sim_relative(s)) return;
    a.relative = true;
    a.alpha = s->prm.alpha;
    a.aMagIn = s->aMagB;
    if (s->prm.macMode == 2) a.groupParam = s->groupParam;
}

// ev (optional, kProfileStages + 1 events): the build events, then after the
// walk; with events the stages run one after the other on the simulation's
// stream, without them the group order, the reorder and the learned
// criterion run on the side stream beside the tree build.
static int sim_enqueue_step(bh_sim* s, cudaEvent_t* ev) {
    const bool fork = ev == nullptr;
    int rc = BH_OK;
    if (fork) {
        // side branch: group order from the last walk's lengths right away,
        // the learned criterion once the bodies are reordered
        BH_CUDA_TRY(cudaEventRecord(s->evFork, s->stream));
        BH_CUDA_TRY(cudaStreamWaitEvent(s->side, s->evFork, 0));
        BH_CUDA_TRY(bh_launch_group_order(s->groupLen, sim_walk_groups(s), s->groupOrder, s->orderHist, s->side));
        // the reorder on the side stream too, beside the tree's count, scan
        // and node passes; the upward pass waits for it
        if ((rc = sim_enqueue_build(s, nullptr, s->evReordered, s->side, s->evSorted))) return rc;
        if ((rc = sim_enqueue_learned(s, s->side))) return rc;
        BH_CUDA_TRY(cudaEventRecord(s->evJoin, s->side));
        BH_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->evJoin, 0));
    } else {
        if ((rc = sim_enqueue_build(s, ev))) return rc;
        if ((rc = sim_enqueue_learned(s, s->stream))) return rc;
    }
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[kProfileStages - 1], s->stream));
    if (s->velSeparate) {
        // the velocities, uploaded on the copy stream, into sorted order
        // there once the sort is done; the walk (the first reader) waits
        if (!fork) return BH_ERR_INTERNAL;
        BH_CUDA_TRY(cudaStreamWaitEvent(s->copyStream, s->evSorted, 0));
        BH_CUDA_TRY(bh_launch_reorder(nullptr, s->velA, nullptr, s->perm, nullptr, s->velB, nullptr, s->n,
                                      s->copyStream));
        BH_CUDA_TRY(cudaEventRecord(s->velReady, s->copyStream));
        BH_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->velReady, 0));
    }
    bh_ctx* c = s->ctx;
    WalkArgs a;
    memset(&a, 0, sizeof a);
    a.pos = s->posB;
    a.n = s->n;
    a.wn = c->wn;
    a.theta = s->prm.theta;
    a.eps2 = s->prm.eps * s->prm.eps;
    a.G = s->prm.G;
    a.accOut = nullptr;
    a.velIn = s->velB;
    a.posOut = s->posA;
    a.velOut = s->velA;
    a.idIn = s->idB;
    a.idOut = s->idA;
    a.posHost = s->hostPos;  // NULL except in the last step of bh_sim_step_host_sorted
    a.velHost = s->hostVel;
    a.idHost = s->hostId;
    a.dt = s->prm.dt;
    a.ctr = c->ctr;
    a.err = c->err;
    a.spill = c->spill;
    sim_set_criterion(s, a);
    a.aMagOut = s->aMagA;  // this step's |a|, in the order the next step starts from
    // longest groups first, judged by the last walk's list lengths (stale
    // lengths, e.g. after a load, only make the order less useful)
    if (!fork)
        BH_CUDA_TRY(bh_launch_group_order(s->groupLen, sim_walk_groups(s), s->groupOrder, s->orderHist, s->stream));
    a.groupOrder = s->groupOrder;
    rc = ctx_walk(c, a, true, s->prm.compensated != 0, s->stream);
    if (rc) return rc;
    if (ev) BH_CUDA_TRY(cudaEventRecord(ev[kProfileStages], s->stream));
    return BH_OK;
}

// Kernel launches of one step (the count the benchmark reports).
extern "C" int bh_sim_kernels_per_step(const bh_sim* s) {
    if (!s) return 0;
    const int npass = (3 * sim_bits(s) + (s->systems ? s->sysBits : 0) + 7) / 8;
    return 2 /* box, keys */ + npass + 1 /* reorder */ + 4 /* tree */ + (s->prm.exportNodes ? 1 : 0) +
           (s->prm.macMode == 2 ? 2 : 0) /* features, selection */ + 2 /* group order */ + 1 /* walk */;
}

// nsteps real steps issued stage by stage (no graph, each queued behind a
// short device-side hold) with events between the stages; msOut[9] = mean ms of keys (box + Morton), sort, reorder, tree
// count, tree scan, tree nodes, tree mass (+ export), learned criterion
// (group features + budget selection; 0 in the other modes), walk +
// kick-drift.
extern "C" int bh_sim_profile(bh_sim* s, int nsteps, float* msOut) {
    if (!s || s->n <= 0 || nsteps <= 0 || !msOut) return set_status(BH_ERR_INVALID);
    cudaEvent_t ev[kProfileStages + 1];
    for (int k = 0; k <= kProfileStages; k++) BH_CUDA_TRY(cudaEventCreate(&ev[k]));
    double acc[kProfileStages] = {0};
    int rc = BH_OK;
    for (int it = 0; it < nsteps && rc == BH_OK; it++) {
        // the step's launches queue up behind a 0.5 ms hold, so the stages
        // run back to back as in a graph replay instead of at the host's
        // launch rate
        BH_CUDA_TRY(bh_launch_hold(500000ull, s->stream));
        rc = sim_enqueue_step(s, ev);
        if (rc) break;
        if (cudaEventSynchronize(ev[kProfileStages]) != cudaSuccess) {
            rc = bh_note_cuda_error(cudaGetLastError());
            break;
        }
        for (int k = 0; k < kProfileStages; k++) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            acc[k] += ms;
        }
    }
    for (int k = 0; k <= kProfileStages; k++) cudaEventDestroy(ev[k]);
    for (int k = 0; k < kProfileStages; k++) msOut[k] = (float)(acc[k] / nsteps);
    return set_status(rc);
}

static int sim_capture(bh_sim* s) {
    cudaGraph_t g;
    BH_CUDA_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int rc = sim_enqueue_step(s, nullptr);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (rc) {
        if (e == cudaSuccess) cudaGraphDestroy(g);
        return rc;
    }
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    e = cudaGraphInstantiate(&s->graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return bh_note_cuda_error(e);
    s->graphReady = true;
    return BH_OK;
}

extern "C" int bh_sim_step(bh_sim* s, int nsteps) {
    if (!s || s->n <= 0 || nsteps < 0) return set_status(BH_ERR_INVALID);
    if (s->prm.macMode == 2 && !s->mlpLoaded) return set_status(BH_ERR_INVALID);
    if (nsteps > 0 && s->prm.macMode != 0 && !s->aMagValid) {
        // no accelerations yet: one step with the fixed-theta walk provides them
        int rc = sim_enqueue_step(s, nullptr);
        if (rc) return set_status(rc);
        s->aMagValid = true;
        sim_drop_graph(s);
        nsteps--;
    }
    if (nsteps > 0 && !s->graphReady) {
        int rc = sim_capture(s);
        if (rc) return set_status(rc);
    }
    for (int k = 0; k < nsteps; k++) BH_CUDA_TRY(cudaGraphLaunch(s->graph, s->stream));
    if (nsteps > 0) s->aMagIdOrder = false;
    return set_status(BH_OK);
}

extern "C" int bh_sim_step_host(bh_sim* s, float4* pos, float3* vel, int n, int nsteps) {
    if (!s || !pos || !vel || n <= 0 || n > s->capacity || nsteps < 0) return set_status(BH_ERR_INVALID);
    if (s->systems && n != s->capacity) return set_status(BH_ERR_INVALID);
    if (n != s->n) {
        sim_drop_graph(s);
        s->n = n;
        s->aMagValid = false;
    }
    // |a| is only reusable if the last call left it in body-id order (the
    // order of the bodies this call uploads)
    if (s->aMagValid && !s->aMagIdOrder) {
        s->aMagValid = false;
        sim_drop_graph(s);
    }
    if (nsteps > 0 && s->prm.macMode == 2 && !s->mlpLoaded) return set_status(BH_ERR_INVALID);
    if (!s->copyStream) {
        BH_CUDA_TRY(cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking));
        BH_CUDA_TRY(cudaEventCreateWithFlags(&s->velReady, cudaEventDisableTiming));
        BH_CUDA_TRY(cudaEventCreateWithFlags(&s->mainReady, cudaEventDisableTiming));
    }
    BH_CUDA_TRY(cudaMemcpyAsync(s->posA, pos, sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA_TRY(bh_launch_iota(s->idA, n, s->stream));
    int rc = BH_OK;
    if (nsteps > 0) {
        // the velocities are first read by the reorder: upload them on the
        // copy stream while the box, keys and sort of the first step run
        BH_CUDA_TRY(cudaEventRecord(s->mainReady, s->stream));
        BH_CUDA_TRY(cudaStreamWaitEvent(s->copyStream, s->mainReady, 0));
        BH_CUDA_TRY(cudaMemcpyAsync(s->velA, vel, sizeof(float3) * n, cudaMemcpyHostToDevice, s->copyStream));
        BH_CUDA_TRY(cudaEventRecord(s->velReady, s->copyStream));
        const bool bootstrap = s->prm.macMode != 0 && !s->aMagValid;
        s->waitBeforeReorder = s->velReady;
        rc = sim_enqueue_step(s, nullptr);  // the first step, stage by stage
        s->waitBeforeReorder = nullptr;
        if (rc) return set_status(rc);
        if (bootstrap) {  // its |a| feeds the relative criterion from now on
            s->aMagValid = true;
            sim_drop_graph(s);
        }
        if (nsteps > 1 && (rc = bh_sim_step(s, nsteps - 1))) return rc;
    } else {
        BH_CUDA_TRY(cudaMemcpyAsync(s->velA, vel, sizeof(float3) * n, cudaMemcpyHostToDevice, s->stream));
    }
    // back to body-id order; |a| too, so that the next call, which uploads the
    // bodies in that order, still has the last step's accelerations
    const bool carry = s->aMagValid;
    BH_CUDA_TRY(bh_launch_scatter_by_id(s->posA, s->velA, nullptr, s->idA, s->posB, s->velB, nullptr, n, s->stream,
                                        carry ? s->aMagA : nullptr, carry ? s->aMagB : nullptr));
    BH_CUDA_TRY(cudaMemcpyAsync(pos, s->posB, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA_TRY(cudaMemcpyAsync(vel, s->velB, sizeof(float3) * n, cudaMemcpyDeviceToHost, s->stream));
    if (carry) BH_CUDA_TRY(cudaMemcpyAsync(s->aMagA, s->aMagB, sizeof(float) * n, cudaMemcpyDeviceToDevice, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->aMagIdOrder = carry;
    return set_status(BH_OK);
}

// Device pointer of page-locked, mapped host memory (NULL for pageable memory).
static void* mapped_device_pointer(const void* host) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, host) != cudaSuccess) {
        cudaGetLastError();  // pageable memory on older runtimes: not an error
        return nullptr;
    }
    return at.type == cudaMemoryTypeHost ? at.devicePointer : nullptr;
}

extern "C" int bh_sim_step_host_sorted(bh_sim* s, float4* pos, float3* vel, uint32_t* ids, int n, int nsteps) {
    if (!s || !pos || !vel || !ids || n <= 0 || n > s->capacity || nsteps < 0) return set_status(BH_ERR_INVALID);
    if (s->systems && n != s->capacity) return set_status(BH_ERR_INVALID);
    if (nsteps > 0 && s->prm.macMode == 2 && !s->mlpLoaded) return set_status(BH_ERR_INVALID);
    if (!s->copyStream) {
        BH_CUDA_TRY(cudaStreamCreateWithFlags(&s->copyStream, cudaStreamNonBlocking));
        BH_CUDA_TRY(cudaEventCreateWithFlags(&s->velReady, cudaEventDisableTiming));
        BH_CUDA_TRY(cudaEventCreateWithFlags(&s->mainReady, cudaEventDisableTiming));
    }
    if (!s->idsReady) BH_CUDA_TRY(cudaEventCreateWithFlags(&s->idsReady, cudaEventDisableTiming));
    if (!s->errHost) BH_CUDA_TRY(cudaHostAlloc((void**)&s->errHost, sizeof(int), cudaHostAllocDefault));
    const bool relativeMode = s->prm.macMode != 0;
    if (relativeMode && !s->aMagById) {
        int rc = dalloc(&s->aMagById, (size_t)s->capacity);
        if (rc) return set_status(rc);
    }
    // |a| of the last step (the relative criterion's input) by body id, taken
    // from the device state before this call's bodies replace it
    bool carry = relativeMode && s->aMagValid && s->n == n;
    if (carry) {
        if (s->aMagIdOrder)
            BH_CUDA_TRY(cudaMemcpyAsync(s->aMagById, s->aMagA, sizeof(float) * n, cudaMemcpyDeviceToDevice,
                                        s->stream));
        else
            BH_CUDA_TRY(bh_launch_scatter_by_id(nullptr, nullptr, nullptr, s->idA, nullptr, nullptr, nullptr, n,
                                                s->stream, s->aMagA, s->aMagById));
    }
    if (n != s->n || s->aMagValid != carry) sim_drop_graph(s);
    s->n = n;
    s->aMagValid = carry;
    s->aMagIdOrder = false;
    // the call's own status: the error word starts clear
    BH_CUDA_TRY(cudaMemsetAsync(s->ctx->err, 0, sizeof(int), s->stream));
    // positions on the simulation's stream (the box needs them first); ids,
    // then velocities on the copy stream behind them
    BH_CUDA_TRY(cudaMemcpyAsync(s->posA, pos, sizeof(float4) * n, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA_TRY(cudaEventRecord(s->mainReady, s->stream));
    BH_CUDA_TRY(cudaStreamWaitEvent(s->copyStream, s->mainReady, 0));
    BH_CUDA_TRY(cudaMemcpyAsync(s->idA, ids, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s->copyStream));
    // the ids checked (and |a| brought into their order)
    BH_CUDA_TRY(bh_launch_gather_by_id(carry ? s->aMagById : nullptr, s->idA, carry ? s->aMagA : nullptr, n,
                                       s->ctx->err, s->copyStream));
    BH_CUDA_TRY(cudaEventRecord(s->idsReady, s->copyStream));
    BH_CUDA_TRY(cudaMemcpyAsync(s->velA, vel, sizeof(float3) * n, cudaMemcpyHostToDevice, s->copyStream));
    if (nsteps == 0) {
        BH_CUDA_TRY(cudaEventRecord(s->velReady, s->copyStream));
        BH_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->velReady, 0));
        BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
        return set_status(BH_OK);
    }
    // the last step's walk writes the caller's arrays directly when all three
    // are mapped page-locked memory; otherwise they are copied after it
    float4* const hp = static_cast<float4*>(mapped_device_pointer(pos));
    float3* const hv = static_cast<float3*>(mapped_device_pointer(vel));
    uint32_t* const hi = static_cast<uint32_t*>(mapped_device_pointer(ids));
    const bool direct = hp && hv && hi;
    int rc = BH_OK;
    for (int step = 0; step < nsteps && rc == BH_OK; step++) {
        const bool first = step == 0, last = step == nsteps - 1;
        if (!first && !last) {  // the steps in between: the captured graph
            rc = bh_sim_step(s, nsteps - 2);
            step = nsteps - 2;
            continue;
        }
        const bool bootstrap = relativeMode && !s->aMagValid;
        if (first) {
            s->waitBeforeReorder = s->idsReady;
            s->velSeparate = true;
        }
        if (last && direct) {
            s->hostPos = hp;
            s->hostVel = hv;
            s->hostId = hi;
        }
        rc = sim_enqueue_step(s, nullptr);
        s->waitBeforeReorder = nullptr;
        s->velSeparate = false;
        s->hostPos = nullptr;
        s->hostVel = nullptr;
        s->hostId = nullptr;
        if (rc == BH_OK && bootstrap) {  // its |a| feeds the relative criterion from now on
            s->aMagValid = true;
            sim_drop_graph(s);
        }
    }
    if (rc) {
        cudaStreamSynchronize(s->copyStream);
        cudaStreamSynchronize(s->stream);
        return set_status(rc);
    }
    if (!direct) {
        BH_CUDA_TRY(cudaMemcpyAsync(pos, s->posA, sizeof(float4) * n, cudaMemcpyDeviceToHost, s->stream));
        BH_CUDA_TRY(cudaMemcpyAsync(vel, s->velA, sizeof(float3) * n, cudaMemcpyDeviceToHost, s->stream));
        BH_CUDA_TRY(cudaMemcpyAsync(ids, s->idA, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s->stream));
    }
    BH_CUDA_TRY(cudaMemcpyAsync(s->errHost, s->ctx->err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(status_from_bits(*s->errHost));
}

extern "C" int bh_sim_accelerations(bh_sim* s, float3* acc, int toHost) {
    if (!s || !acc || s->n <= 0) return set_status(BH_ERR_INVALID);
    int rc = sim_enqueue_build(s, nullptr);
    if (rc) return set_status(rc);
    if ((rc = sim_enqueue_learned(s, s->stream))) return set_status(rc);
    bh_ctx* c = s->ctx;
    WalkArgs a;
    memset(&a, 0, sizeof a);
    a.pos = s->posB;
    a.n = s->n;
    a.wn = c->wn;
    a.theta = s->prm.theta;
    a.eps2 = s->prm.eps * s->prm.eps;
    a.G = s->prm.G;
    a.accOut = s->acc;
    a.ctr = c->ctr;
    a.err = c->err;
    a.spill = c->spill;
    sim_set_criterion(s, a);
    rc = ctx_walk(c, a, false, s->prm.compensated != 0, s->stream);
    if (rc) return set_status(rc);
    // sorted order -> body-id order
    float3* dst = acc;
    float3* staging = nullptr;
    if (toHost) {
        staging = reinterpret_cast<float3*>(s->velB);  // scratch between steps
        dst = staging;
    }
    BH_CUDA_TRY(bh_launch_scatter_by_id(nullptr, nullptr, s->acc, s->idB, nullptr, nullptr, dst, s->n, s->stream));
    if (toHost) BH_CUDA_TRY(cudaMemcpyAsync(acc, staging, sizeof(float3) * s->n, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_accel_magnitudes(bh_sim* s, float* aMag, int toHost) {
    if (!s || !aMag || s->n <= 0 || !s->aMagValid) return set_status(BH_ERR_INVALID);
    BH_CUDA_TRY(cudaMemcpyAsync(aMag, s->aMagA, sizeof(float) * s->n,
                                toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_synchronize(bh_sim* s) {
    if (!s) return set_status(BH_ERR_INVALID);
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_diagnostics(bh_sim* s, int withPotential, bh_diagnostics* out) {
    if (!s || !out || s->n <= 0) return set_status(BH_ERR_INVALID);
    return set_status(bh_diagnostics_f64(s->posA, s->velA, s->n, s->prm.eps, s->prm.G, withPotential, out, s->stream));
}

extern "C" int bh_sim_system_diagnostics(bh_sim* s, int withPotential, bh_diagnostics* out) {
    if (!s || !out || s->n <= 0) return set_status(BH_ERR_INVALID);
    if (!s->systems) return bh_sim_diagnostics(s, withPotential, out);
    // bodies never leave their system's segment, so each system is a slice
    for (int k = 0; k < s->systems; k++) {
        const int off = s->segOffHost[k], cnt = s->segOffHost[k + 1] - off;
        int rc = bh_diagnostics_f64(s->posA + off, s->velA + off, cnt, s->prm.eps, s->prm.G, withPotential, &out[k],
                                    s->stream);
        if (rc) return set_status(rc);
    }
    return set_status(BH_OK);
}

// Autotuner: time `trialSteps` graph-replayed steps from the current state
// for every candidate (bucket size, group width), keep the fastest, and put
// the state back.  Then, at that bucket size and width, the walk's
// shared-memory stack depth: a deeper stack spills less to global memory but
// may leave room for fewer resident blocks.
static const int kTuneLeafSizes[] = {1, 2, 4, 8, 16};
static const int kTuneWidths[] = {32, 64};
static const int kTuneStacks[] = {384, 1536};  // besides the default (768)

extern "C" int bh_sim_set_walk_stack(bh_sim* s, int entries) {
    if (!s) return set_status(BH_ERR_INVALID);
    if (entries != 0 && (entries < BH_WALK_STACK_MIN || entries > BH_WALK_STACK_MAX || entries % 32))
        return set_status(BH_ERR_INVALID);
    s->walkStack = entries;
    sim_drop_graph(s);
    return set_status(BH_OK);
}

extern "C" int bh_sim_walk_stack(const bh_sim* s) {
    if (!s) return 0;
    return s->walkStack ? s->walkStack : bh_walk_stack_default();
}

extern "C" int bh_sim_tune(bh_sim* s, int trialSteps, bh_tune_result* out) {
    if (!s || !out || s->n <= 0 || trialSteps <= 0) return set_status(BH_ERR_INVALID);
    const int n = s->n;
    const int nLeaf = (int)(sizeof kTuneLeafSizes / sizeof kTuneLeafSizes[0]);
    const int nShape = nLeaf * (int)(sizeof kTuneWidths / sizeof kTuneWidths[0]);
    const int nStack = (int)(sizeof kTuneStacks / sizeof kTuneStacks[0]);
    const int cands = nShape + nStack;
    static_assert(sizeof kTuneLeafSizes / sizeof kTuneLeafSizes[0] * (sizeof kTuneWidths / sizeof kTuneWidths[0]) +
                          sizeof kTuneStacks / sizeof kTuneStacks[0] <=
                      BH_TUNE_MAX,
                  "tuning table");
    const int keepStack = s->walkStack;
    float4* p0 = nullptr;
    float3* v0 = nullptr;
    uint32_t* i0 = nullptr;
    float* a0 = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = BH_OK;
    if ((rc = dalloc(&p0, n)) || (rc = dalloc(&v0, n)) || (rc = dalloc(&i0, n)) || (rc = dalloc(&a0, n))) {
        cudaFree(p0); cudaFree(v0); cudaFree(i0); cudaFree(a0);
        return set_status(rc);
    }
    const bool aValid = s->aMagValid, aIdOrder = s->aMagIdOrder;
    const bh_params keep = s->prm;
    cudaStream_t st = s->stream;
    auto copy = [&](void* d, const void* src, size_t bytes) {
        return cudaMemcpyAsync(d, src, bytes, cudaMemcpyDeviceToDevice, st) == cudaSuccess ? BH_OK
                                                                                         : bh_note_cuda_error(cudaGetLastError());
    };
    auto save = [&]() {
        int r = copy(p0, s->posA, sizeof(float4) * n);
        if (!r) r = copy(v0, s->velA, sizeof(float3) * n);
        if (!r) r = copy(i0, s->idA, sizeof(uint32_t) * n);
        if (!r) r = copy(a0, s->aMagA, sizeof(float) * n);
        return r;
    };
    auto restore = [&]() {
        int r = copy(s->posA, p0, sizeof(float4) * n);
        if (!r) r = copy(s->velA, v0, sizeof(float3) * n);
        if (!r) r = copy(s->idA, i0, sizeof(uint32_t) * n);
        if (!r) r = copy(s->aMagA, a0, sizeof(float) * n);
        s->aMagValid = aValid;
        s->aMagIdOrder = aIdOrder;
        return r;
    };
    memset(out, 0, sizeof *out);
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) rc = BH_ERR_CUDA;
    if (!rc) rc = save();
    int best = -1, bestShape = -1;
    for (int k = 0; k < cands && !rc; k++) {
        bh_params p = keep;
        int stack = 0;  // the default depth while the shapes are timed
        if (k < nShape) {
            p.leafSize = kTuneLeafSizes[k % nLeaf];
            p.groupWidth = kTuneWidths[k / nLeaf];
        } else {
            if (k == nShape) bestShape = best;  // the shapes are done: tune the stack at the best one
            p.leafSize = kTuneLeafSizes[bestShape % nLeaf];
            p.groupWidth = kTuneWidths[bestShape / nLeaf];
            stack = kTuneStacks[k - nShape];
        }
        s->prm = p;
        s->walkStack = stack;
        sim_drop_graph(s);
        if ((rc = restore())) break;
        if ((rc = bh_sim_step(s, 1))) break;  // bootstrap / graph capture, untimed
        if (cudaEventRecord(e0, st) != cudaSuccess) { rc = BH_ERR_CUDA; break; }
        if ((rc = bh_sim_step(s, trialSteps))) break;
        float ms = 0.f;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            rc = bh_note_cuda_error(cudaGetLastError());
            break;
        }
        out->leafSizes[k] = p.leafSize;
        out->groupWidths[k] = p.groupWidth;
        out->stackEntriesTried[k] = stack ? stack : bh_walk_stack_default();
        out->msPerStep[k] = ms / trialSteps;
        out->candidates = k + 1;
        if (best < 0 || out->msPerStep[k] < out->msPerStep[best]) best = k;
    }
    s->prm = keep;
    s->walkStack = keepStack;
    sim_drop_graph(s);
    if (!rc) rc = restore();
    if (!rc && best >= 0) {
        s->prm.leafSize = out->leafSizes[best];
        s->prm.groupWidth = out->groupWidths[best];
        s->walkStack = best < nShape ? 0 : kTuneStacks[best - nShape];
        out->leafSize = s->prm.leafSize;
        out->groupWidth = s->prm.groupWidth;
        out->stackEntries = out->stackEntriesTried[best];
    }
    if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = bh_note_cuda_error(cudaGetLastError());
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(p0); cudaFree(v0); cudaFree(i0); cudaFree(a0);
    return set_status(rc);
}

extern "C" int bh_sim_set_mac_mlp(bh_sim* s, const float* params) {
    if (!s || !params) return set_status(BH_ERR_INVALID);
    for (int i = 0; i < BH_MLP_PARAMS; i++)
        if (!isfinite(params[i])) return set_status(BH_ERR_INVALID);
    BH_CUDA_TRY(cudaMemcpyAsync(s->mlp, params, sizeof(float) * BH_MLP_PARAMS, cudaMemcpyHostToDevice, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->mlpLoaded = true;
    return set_status(BH_OK);
}

extern "C" int bh_sim_group_features(bh_sim* s, float* feat, uint32_t* ids, int toHost) {
    if (!s || !feat || s->n <= 0 || !s->aMagValid) return set_status(BH_ERR_INVALID);
    int rc = sim_enqueue_build(s, nullptr);
    if (rc) return set_status(rc);
    const int groups = (s->n + 31) / 32;
    BH_CUDA_TRY(bh_launch_group_features(s->posB, s->aMagB, s->keysB, s->n, s->prm.bitsPerAxis, s->ctx->box,
                                         s->ctx->root64, s->prm.G, s->feat, s->stream));
    const cudaMemcpyKind k = toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    BH_CUDA_TRY(cudaMemcpyAsync(feat, s->feat, sizeof(float) * groups * BH_GROUP_FEATURES, k, s->stream));
    if (ids) BH_CUDA_TRY(cudaMemcpyAsync(ids, s->idB, sizeof(uint32_t) * s->n, k, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_group_params(bh_sim* s, float* gp, int toHost) {
    if (!s || !gp || s->n <= 0) return set_status(BH_ERR_INVALID);
    const int groups = (s->n + 31) / 32;
    BH_CUDA_TRY(cudaMemcpyAsync(gp, s->groupParam, sizeof(float2) * groups,
                                toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_group_lengths(bh_sim* s, int* lens, int maxGroups, int* groups, int toHost) {
    if (!s || !lens || !groups || s->n <= 0) return set_status(BH_ERR_INVALID);
    *groups = sim_walk_groups(s);
    if (maxGroups < *groups) return set_status(BH_ERR_INVALID);
    BH_CUDA_TRY(cudaMemcpyAsync(lens, s->groupLen, sizeof(int) * *groups,
                                toHost ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    return set_status(BH_OK);
}

extern "C" int bh_sim_root_f64(bh_sim* s, double out[10]) {
    if (!s || !out || s->n <= 0 || s->systems) return set_status(BH_ERR_INVALID);
    DevRoot r;
    BH_CUDA_TRY(cudaMemcpyAsync(&r, s->ctx->root64, sizeof r, cudaMemcpyDeviceToHost, s->stream));
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    out[0] = r.mass;
    for (int k = 0; k < 3; k++) {
        out[1 + k] = r.com[k];
        out[4 + k] = r.mn[k];
        out[7 + k] = r.mx[k];
    }
    return set_status(BH_OK);
}

extern "C" int bh_sim_stats(bh_sim* s, bh_stats* out) {
    if (!s || !out) return set_status(BH_ERR_INVALID);
    DevTreeInfo info;
    DevCounters ctr;
    int err = 0;
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    BH_CUDA_TRY(cudaMemcpy(&info, s->ctx->info, sizeof info, cudaMemcpyDeviceToHost));
    BH_CUDA_TRY(cudaMemcpy(&ctr, s->ctx->ctr, sizeof ctr, cudaMemcpyDeviceToHost));
    BH_CUDA_TRY(cudaMemcpy(&err, s->ctx->err, sizeof err, cudaMemcpyDeviceToHost));
    memset(out, 0, sizeof *out);
    out->interactions = (long long)ctr.interactions;
    out->nodesTested = (long long)ctr.nodesTested;
    out->nodeCount = info.nodeCount;
    out->deepestLevel = info.deepest;
    for (int L = 0; L < 23; L++) {
        out->levelOffsets[L] = info.levelOffset[L];
        out->levelCount[L] = info.levelCount[L];
    }
    out->errorBits = err;
    out->maxStack = ctr.maxStack;
    out->groupVotes = (long long)ctr.undecided;
    return set_status(status_from_bits(err));
}

extern "C" int bh_sim_tree(bh_sim* s, treeState** state) {
    if (!s || !state) return set_status(BH_ERR_INVALID);
    DevTreeInfo info;
    BH_CUDA_TRY(cudaStreamSynchronize(s->stream));
    BH_CUDA_TRY(cudaMemcpy(&info, s->ctx->info, sizeof info, cudaMemcpyDeviceToHost));
    treeState* t = &s->ts;
    memset(t, 0, sizeof *t);
    t->nodes = s->aos;
    t->maxNodes = s->ctx->maxNodes;
    t->mortonIn = s->keysA;
    t->mortonOut = s->keysB;
    t->indexIn = nullptr;
    t->indexOut = s->perm;
    t->boundingData[2] = s->corner;
    t->boundingData[3] = s->corner + 1;
    t->builder = &s->ctx->tb;
    for (int L = 0; L < 22; L++) {
        t->levelOffsets[L] = info.levelOffset[L];
        t->levelCount[L] = info.levelCount[L];
    }
    t->deepestLevel = info.deepest;
    t->starCount = s->n;
    t->sortedPosMassVals = s->posB;
    t->sortedVelVals = s->velB;
    *state = t;
    return set_status(BH_OK);
}
