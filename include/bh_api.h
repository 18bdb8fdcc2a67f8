/*
 * bh_api.h — status-returning and device-resident API of the B200 Barnes-Hut
 * engine (libbh_b200.so).
 *
 * Everything here sits beside the reference-named entry points of types.h,
 * tree.h, sorting.h and main.h:
 *   - bh_* variants of the reference entry points that return a bh_status
 *     instead of calling exit(-1);
 *   - bh_sim: a device-resident simulation that runs whole steps
 *     (bounding box -> keys -> sort -> reorder -> octree -> walk + kick-drift)
 *     as one CUDA graph per step, with no host synchronisation inside a step;
 *   - seeded initial conditions (Plummer sphere, exponential disk + Hernquist
 *     bulge, two-galaxy merger).
 * All functions are plain C with pointers and sizes.
 */
#ifndef BH_API_H
#define BH_API_H

#include <stdint.h>
#include <driver_types.h>
#include "types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
typedef enum {
    BH_OK = 0,
    BH_ERR_INVALID = 1,         /* bad argument: n <= 0, n > capacity, null pointer, bad params */
    BH_ERR_ALLOC = 2,           /* a device or host allocation failed */
    BH_ERR_CUDA = 3,            /* a CUDA runtime call failed (bh_cuda_error_string) */
    BH_ERR_DEGENERATE_BOX = 4,  /* bounding-box extent is zero or not finite */
    BH_ERR_NONFINITE = 5,       /* a body position is NaN or infinite */
    BH_ERR_TREE_OVERFLOW = 6,   /* the octree needs more nodes than maxNodes */
    BH_ERR_STACK_OVERFLOW = 7,  /* a walk traversal stack exceeded its bound */
    BH_ERR_TIMEOUT = 8,         /* a bounded device-side wait gave up */
    BH_ERR_INTERNAL = 9         /* a device-side consistency check failed (tree links) */
} bh_status;

/* Human-readable name of a status code. */
const char* bh_status_string(int status);
/* Status of the most recent launcher call on this host thread (the launchers
 * of tree.h and sorting.h return void, like the reference's kernels). */
int bh_last_error(void);
/* Text of the last CUDA runtime error seen on this host thread. */
const char* bh_cuda_error_string(void);

/* ------------------------------------------------------------ parameters */
#define BH_MAX_LEAF_SIZE 16

typedef struct {
    int bitsPerAxis;   /* Morton bits per axis, 1..21; 21 reproduces the reference */
    int leafSize;      /* bucket size, 1..BH_MAX_LEAF_SIZE: an opened node with at most this many
                        * bodies contributes its bodies directly; 1 reproduces the reference */
    int groupWidth;    /* bodies sharing one opening decision: 32 (the reference) or 64 (two per lane) */
    float theta;       /* opening angle: a node is accepted when size^2 < theta^2 d^2 */
    float eps;         /* Plummer softening length (eps^2 is added to r^2) */
    float G;           /* gravitational constant */
    float dt;          /* time step of the kick-drift integrator */
    int compensated;   /* 1: Kahan-compensated force sums (blocked), 0: plain FP32 sums */
    int exportNodes;   /* 1: also write the tree in the reference's 80-byte node layout */
    /* Opening criterion.  0: the reference's fixed theta.  1: relative
     * criterion: a node is also opened when G M s^2 > alpha |a_b| d^4 for a
     * body b of the group (|a_b| from the previous step), theta acting as the
     * geometric cap.  2: learned: per group, the MLP of bh_sim_set_mac_mlp()
     * predicts the group's RMS relative force error at each budget of
     * bh_mac_ladder() and the group walks with the largest budget whose
     * prediction meets errTarget (theta stays the cap; a group with a
     * non-finite prediction falls back to the fixed theta 0.5).  Modes 1 and 2
     * need the last step's accelerations: the first step after a load uses
     * mode 0. */
    int macMode;
    float alpha;       /* mode 1: relative-criterion budget */
    float errTarget;   /* mode 2: predicted RMS relative force error each group must meet */
} bh_params;

/* Reference values: 21 bits, leaf 1, group 32, theta 0.7, eps 0.02, G 1,
 * dt 0.08 (units.c:3-4, basicGravity.cu:462-466), compensated sums on,
 * fixed-theta opening (macMode 0). */
void bh_params_default(bh_params* p);

/* ------------------------------------- status variants of main.h / tree.h */
int bh_initialise_tree(treeState* state, int starCount, int paddedStarCount, int integrateBlocks);
int bh_build_tree(treeState* state, float4** pos, float3** vel, cudaStream_t stream);
int bh_destroy_tree(treeState* state);
int bh_calculate_acceleration(const float4* pos, const treeState* state, float3* acc,
                              float antiSingularitySquared, float G, float theta, int starCount,
                              cudaStream_t stream);
int bh_position_updater(float4* pos, float3* vel, const float3* acc, int starCount, float dt,
                        cudaStream_t stream);
/* Device bounding box + world box (basicGravity.cu:79-113) for `bits` bits per
 * axis; writes the world box and the global corners to device memory. */
int bh_world_box(const float4* pos, int n, int bits, worldBox* boxOut /* host */,
                 float3* minOut /* host, may be NULL */, float3* maxOut /* host, may be NULL */,
                 cudaStream_t stream);
/* Morton keys for `bits` bits per axis (bits = 21: the reference's keys). */
int bh_morton_encode(const float4* pos, uint64_t* keys, uint32_t* idx, int n, worldBox box,
                     int bits, cudaStream_t stream);

/* ------------------------------------------------------ device simulation */
typedef struct bh_sim bh_sim;

typedef struct {
    long long interactions;   /* body-node interactions of the last walk */
    long long nodesTested;    /* opening tests of the last walk (per group, not per body) */
    int nodeCount;            /* nodes in the last tree */
    int deepestLevel;         /* deepest level of the last tree */
    int levelOffsets[23];     /* first node of each level (entry deepest+1 = nodeCount) */
    int levelCount[23];
    int errorBits;            /* device error word: 1 << (bh_status - 1) per error seen */
    int maxStack;             /* deepest traversal stack of the last walk (entries, one warp) */
    long long groupVotes;     /* nodes of the last walk that needed the exact per-body group vote */
} bh_stats;

/* Creates a simulation for up to `capacity` bodies on the current device.
 * stream 0 makes the simulation create its own non-blocking stream. */
int bh_sim_create(bh_sim** out, int capacity, const bh_params* params, cudaStream_t stream);
int bh_sim_destroy(bh_sim* sim);
int bh_sim_set_params(bh_sim* sim, const bh_params* params);
int bh_sim_get_params(const bh_sim* sim, bh_params* params);
cudaStream_t bh_sim_stream(const bh_sim* sim);

/* Loads n bodies (pos.w = mass).  fromHost != 0: host arrays (pinned or
 * pageable), else device arrays.  Body ids become 0..n-1. */
int bh_sim_load(bh_sim* sim, const float4* pos, const float3* vel, int n, int fromHost);
/* Copies the current state out in body-id order (the order of the last load).
 * Any of pos/vel may be NULL. */
int bh_sim_store(bh_sim* sim, float4* pos, float3* vel, int toHost);
/* Raw device views of the current state in the simulation's (Morton) order. */
int bh_sim_device_state(bh_sim* sim, float4** pos, float3** vel, uint32_t** ids, int* n);

/* nsteps full steps on the device, asynchronous on the simulation's stream
 * (each step replays one captured CUDA graph). */
int bh_sim_step(bh_sim* sim, int nsteps);
/* End to end: copies pos/vel (host, n bodies) in, runs nsteps steps, copies
 * the result back into the same host arrays in their original order, and
 * synchronises. */
int bh_sim_step_host(bh_sim* sim, float4* pos, float3* vel, int n, int nsteps);
/* End to end in the reference's frame order: pos/vel/ids (host, n bodies in
 * any order, ids[k] = the body id of entry k, each in [0, n)) go in, nsteps
 * steps run, and the arrays come back holding the state after the last step
 * in that step's Morton order with each entry's body id — the order the
 * reference leaves its device arrays in after buildTree + positionUpdater,
 * whose frames it copies out with indexOut (basicGravity.cu:796-800).
 * Feeding the returned arrays back in continues the same simulation
 * bit for bit as bh_sim_step does on the device.  When all three arrays are
 * page-locked and mapped (cudaHostAlloc, cudaMallocHost, or cudaHostRegister
 * with cudaHostRegisterMapped), the last step's walk writes them directly as
 * its groups finish, so the device-to-host transfer overlaps the walk;
 * otherwise they are copied after it.  The relative criteria reuse the last
 * step's |a| by body id.  In a batch each system's bodies must stay within
 * that system's slots (the returned order keeps them there).  Synchronises;
 * returns the status of the device
 * error word, which the call clears first (an id outside [0, n) gives
 * BH_ERR_INVALID).  nsteps = 0 only uploads the bodies. */
int bh_sim_step_host_sorted(bh_sim* sim, float4* pos, float3* vel, uint32_t* ids, int n, int nsteps);
/* Build + walk only: accelerations of the current state, in body-id order
 * (toHost != 0: host array, else device array). */
int bh_sim_accelerations(bh_sim* sim, float3* acc, int toHost);
/* |a| of every body from the last step, in the order of bh_sim_device_state
 * (the input of the relative criterion); BH_ERR_INVALID before any step. */
int bh_sim_accel_magnitudes(bh_sim* sim, float* aMag, int toHost);
/* nsteps real steps issued stage by stage with CUDA events between stages
 * (synchronous; each step's launches queue behind a 0.5 ms device-side hold,
 * so the stages run back to back as in a graph replay); msOut[9] = mean milliseconds of: keys (box + Morton), sort,
 * reorder, tree count, tree scan, tree nodes, tree mass (+ reference-layout
 * export when enabled), learned criterion (group features + budget selection;
 * about 0 in the other modes), walk + kick-drift. */
int bh_sim_profile(bh_sim* sim, int nsteps, float* msOut);
/* Kernel launches one step issues. */
int bh_sim_kernels_per_step(const bh_sim* sim);
/* FP32 FMA throughput of the current device in TFLOP/s (best of `reps`
 * timed runs of a dependent-FMA probe), the walk's roofline denominator. */
int bh_fma_peak_tflops(int reps, float* tflops, cudaStream_t stream);
/* FP64 direct-sum accelerations (device arrays): acc[3*t..3*t+2] for body
 * targets[t] (targets NULL: bodies 0..ntargets-1) against all n bodies. */
int bh_direct_sum_f64(const float4* pos, int n, const int* targets, int ntargets, double eps, double G,
                      double* acc, cudaStream_t stream);
/* Waits for everything enqueued on the simulation's stream. */
int bh_sim_synchronize(bh_sim* sim);

/* ----------------------------------------------- outputDump.bin writer */
/* The reference's dump file (basicGravity.cu:614-635, inputOutput.c:41-58):
 * int32 n, int32 frames, RGB[n] (NULL colours: the reference's 100,100,100),
 * then `frames` frames of float32 x, y, z per body, in body-id order.  Frames
 * are gathered on the device and written while the device keeps stepping;
 * close fails if fewer or more frames than announced were given. */
typedef struct bh_dump bh_dump;
int bh_dump_open(bh_dump** out, const char* path, int n, int frames, const RGB* colours);
/* One frame of device bodies: pos[i] is body ids[i] (ids NULL: body i). */
int bh_dump_frame(bh_dump* dump, const float4* pos, const uint32_t* ids, int n, cudaStream_t stream);
/* One frame of the simulation's current state, on its stream. */
int bh_sim_dump_frame(bh_dump* dump, bh_sim* sim);
int bh_dump_close(bh_dump* dump);

/* ------------------------------------------ batch of independent systems */
/* A simulation of `systems` independent systems (counts[k] bodies each, laid
 * out system after system in every load and store).  Each system gets its
 * own world box and tree; one launch per stage serves all of them (the keys
 * carry the system index above the Morton bits, so one sort orders bodies by
 * system, one build makes a forest with one root per system, one persistent
 * walk serves groups that never straddle two systems), and a step is one
 * CUDA graph.  Fixed-theta opening only (macMode 0), no reference-layout
 * export; Morton bits per axis are capped so that 3 * bits + the system
 * index bits fit 64 (18 for 256 systems).  The simulation is used through
 * every bh_sim_* call; loads must give all bodies. */
int bh_sim_create_batch(bh_sim** out, int systems, const int* counts, const bh_params* params,
                        cudaStream_t stream);
/* Number of systems (0 for a single-system simulation) and, when offsets is
 * not NULL, the systems + 1 body offsets. */
int bh_sim_systems(const bh_sim* sim, int* systems, int* offsets);

/* ----------------------------------------------------------- autotuner */
#define BH_TUNE_MAX 16
typedef struct {
    int leafSize;              /* chosen bucket size ... */
    int groupWidth;            /* ... and walk group width (now set in the simulation's parameters) */
    int candidates;            /* entries filled below */
    int leafSizes[BH_TUNE_MAX];
    int groupWidths[BH_TUNE_MAX];
    float msPerStep[BH_TUNE_MAX];
    int stackEntries;          /* chosen walk stack depth (now set in the simulation) */
    int stackEntriesTried[BH_TUNE_MAX];
} bh_tune_result;
/* Times trialSteps steps (graph replays, events on the simulation's stream)
 * from the current state for every bucket size 1, 2, 4, 8, 16 and group
 * width 32, 64 (walk stack at its default depth), then for the walk stack
 * depths 384 and 1536 at the fastest of those; keeps the fastest candidate in
 * the simulation (parameters and walk stack depth) and restores the state
 * (positions, velocities, ids, last |a|) as it was.  Synchronous. */
int bh_sim_tune(bh_sim* sim, int trialSteps, bh_tune_result* out);

/* Walk traversal-stack entries per warp kept in shared memory (the rest of a
 * deep traversal spills to a per-warp global area): 0 = the default (768), or
 * a multiple of 32 in 128..2048.  More entries spill less; fewer leave room
 * for more resident blocks.  The reference's stack is a fixed int[168] per
 * 32-thread block (tree.cu:586-588). */
int bh_sim_set_walk_stack(bh_sim* sim, int entries);
/* The depth in use (entries per warp). */
int bh_sim_walk_stack(const bh_sim* sim);

/* ------------------------------------------------ FP64 diagnostics */
typedef struct {
    double mass;
    double com[3];              /* centre of mass */
    double comVel[3];           /* its velocity */
    double momentum[3];         /* sum m v */
    double angularMomentum[3];  /* sum m (x cross v), about the origin */
    double kinetic;             /* sum m v^2 / 2 */
    double potential;           /* -(G/2) sum_{i != j} m_i m_j / sqrt(r_ij^2 + eps^2); 0 unless asked */
    double total;               /* kinetic + potential */
} bh_diagnostics;
/* Conserved quantities of n bodies (device arrays), every sum in FP64; the
 * potential is the exact pair sum (O(n^2)), computed when withPotential != 0.
 * Synchronises the stream. */
int bh_diagnostics_f64(const float4* pos, const float3* vel, int n, double eps, double G, int withPotential,
                       bh_diagnostics* out, cudaStream_t stream);
/* The same for the simulation's current state (its eps and G). */
int bh_sim_diagnostics(bh_sim* sim, int withPotential, bh_diagnostics* out);
/* FP64 diagnostics of every system of a batch: out[systems] (one entry when
 * the simulation is not a batch). */
int bh_sim_system_diagnostics(bh_sim* sim, int withPotential, bh_diagnostics* out);

/* ---------------------------- the reference program's demo galaxy, seeded */
typedef struct {
    float totalMass;       /* all bodies, equal masses (5: basicGravity.cu:500) */
    float scaleLength;     /* disk scale length R_d (4: basicGravity.cu:541) */
    float scaleThickness;  /* Laplace scale height (0.3: basicGravity.cu:542) */
    float haloFraction;    /* share of bodies in the uniform-radius halo (0.2: basicGravity.cu:694) */
    float G;               /* for the circular speeds (1: units.c:3) */
    float rotation[3];     /* yaw, pitch, roll in radians (0) */
    float centre[3];       /* position offset (0) */
    float velocity[3];     /* velocity offset (0) */
} bh_demo_params;
void bh_demo_params_default(bh_demo_params* p);
/* The reference's own initial conditions (initialConditions.c:246-382,
 * basicGravity.cu:694-697) on the device: exponential disk by rejection
 * sampling below 5 R_d, Laplace heights, circular speeds of the enclosed disk
 * mass, then a halo with radii uniform in [0, 5 R_d).  Counter-based draws
 * keyed by (seed, body), so the result depends only on the seed (the
 * reference seeds rand() with the clock).  Device arrays; synchronous. */
int bh_ic_demo(float4* pos, float3* vel, int n, const bh_demo_params* params, uint64_t seed, cudaStream_t stream);

/* ------------------------------------------- learned opening criterion */
/* The MLP 8 -> 32 -> 32 -> 1 (ReLU; BF16 tensor-core products, FP32
 * accumulation) as one FP32 block of BH_MLP_PARAMS floats, row-major W[in][out]:
 * W1[8][32] b1[32] W2[32][32] b2[32] W3[32] b3, then the input normalisation
 * mean[8] and 1/std[8] (x_norm = (x - mean) * inv_std).  The first
 * BH_MLP_TRAINED floats are the trained parameters.  Input 0 is log10 alpha,
 * inputs 1..7 the group features of bh_sim_group_features(); the output is
 * the predicted log10 RMS relative force error of the group. */
#define BH_MLP_PARAMS 1393
#define BH_MLP_TRAINED 1377
#define BH_MAC_CANDIDATES 8
#define BH_GROUP_FEATURES 7
/* The budgets (alpha) a learned walk chooses from, increasing. */
int bh_mac_ladder(float alphas[BH_MAC_CANDIDATES]);
/* Loads the MLP (host array of BH_MLP_PARAMS floats) used by macMode 2. */
int bh_sim_set_mac_mlp(bh_sim* sim, const float* params);
/* Builds the tree of the current state as a walk would, then writes the
 * features of every 32-body group (groups x BH_GROUP_FEATURES floats; group
 * g = bodies 32g..32g+31 of the walk order) and the body ids in walk order
 * (n, may be NULL).  Needs the last step's accelerations. */
int bh_sim_group_features(bh_sim* sim, float* feat, uint32_t* ids, int toHost);
/* (theta, alpha) per group chosen by the last learned walk (groups x 2). */
int bh_sim_group_params(bh_sim* sim, float* gp, int toHost);
/* No counterpart in the reference.  Interaction-list length (nodes, or bucket
 * bodies, accepted) of every walk group of the last walk, in walk order: the
 * 32- or 64-body groups of the sorted bodies, or a batch's group table.
 * *groups = the number of groups; lens must hold maxGroups >= *groups ints
 * (BH_ERR_INVALID otherwise, with *groups still set). */
int bh_sim_group_lengths(bh_sim* sim, int* lens, int maxGroups, int* groups, int toHost);

/* No counterpart in the reference (its root reduction is FP32, tree.cu:89-179
 * and :414-490).  The FP64 reduction over all bodies made by the last build's
 * bounding-box pass: out[0] = total mass, out[1..3] = centre of mass,
 * out[4..6] = box minimum, out[7..9] = box maximum (host array).  The FP32
 * tree keeps the reference's rounding; this is what system-level quantities
 * (the learned criterion's distance from the centre of mass) read.  One
 * system only (BH_ERR_INVALID for a batch). */
int bh_sim_root_f64(bh_sim* sim, double out[10]);
/* Device arrays.  Y[r] = MLP(X[r, 0..7]) for `rows` rows. */
int bh_mlp_forward(const float* params, const float* X, int rows, float* Y, cudaStream_t stream);
/* grad[0..BH_MLP_TRAINED) = d/dparams of sum_r (MLP(X[r]) - Y[r])^2 / rows and
 * *loss = sum_r (MLP(X[r]) - Y[r])^2 (both overwritten). */
int bh_mlp_loss_grad(const float* params, const float* X, const float* Y, int rows, float* grad, float* loss,
                     cudaStream_t stream);
/* One pass of Adam (beta 0.9 / 0.999, eps 1e-8) over `rows` rows in batches
 * of `batch`, updating params in place; adamM / adamV (BH_MLP_TRAINED floats
 * each, zero at the start of training) and *step carry the optimiser state;
 * *loss accumulates the squared errors seen (device float). */
int bh_mlp_train_epoch(float* params, const float* X, const float* Y, int rows, float* grad, float* adamM,
                       float* adamV, int batch, int* step, float lr, float* loss, cudaStream_t stream);
/* Self-test of failure detection without a GPU fault: runs the radix sort's
 * decoupled look-back for a tile whose predecessor never publishes its
 * counts; the wait is bounded like every device-side wait in this library,
 * so the kernel records a timeout and returns.  Returns BH_ERR_TIMEOUT when
 * that works (the context stays usable), anything else when it does not.
 * Takes a second or so. */
int bh_selftest_bounded_wait(cudaStream_t stream);
/* Waits for the stream, then reads statistics and the device error word. */
int bh_sim_stats(bh_sim* sim, bh_stats* out);
/* Device pointers into the last tree (reference layout requires exportNodes). */
int bh_sim_tree(bh_sim* sim, treeState** state);

/* ------------------------------------------------- seeded initial conditions */
/* Plummer sphere: total mass M, scale radius a, isotropic velocities drawn
 * from the distribution function, centre of mass and bulk velocity removed. */
int bh_ic_plummer(float4* pos, float3* vel, int n, float M, float a, float G, uint64_t seed);

typedef struct {
    float diskMass;        /* exponential disk mass */
    float diskScale;       /* radial scale length R_d */
    float diskHeight;      /* sech^2 vertical scale height z0 */
    float diskTrunc;       /* disk truncation radius (in R_d) */
    float bulgeMass;       /* Hernquist bulge mass */
    float bulgeScale;      /* Hernquist scale radius */
    float bulgeTrunc;      /* bulge truncation radius (in bulge scale radii) */
    float dispersion;      /* Gaussian velocity dispersion as a fraction of v_c */
    float G;
} bh_galaxy_params;

/* Configuration of the N=1M disk: disk 0.8 (R_d 1, z0 0.1), bulge 0.2 (a 0.2),
 * 10% dispersion, G 1. */
void bh_galaxy_params_default(bh_galaxy_params* g);

/* Exponential disk + Hernquist bulge; circular velocities from the enclosed
 * mass plus Gaussian dispersion.  Bodies are split between disk and bulge in
 * proportion to mass (equal body masses). */
int bh_ic_disk_galaxy(float4* pos, float3* vel, int n, const bh_galaxy_params* g, uint64_t seed);

/* Two disk galaxies of n/2 bodies each on a parabolic orbit: initial
 * separation `separation`, pericentre `pericentre`, the second disk
 * inclined by `inclinationDeg` degrees about the x axis. */
int bh_ic_merger(float4* pos, float3* vel, int n, const bh_galaxy_params* g, float separation,
                 float pericentre, float inclinationDeg, uint64_t seed);

#ifdef __cplusplus
}
#endif

#endif /* BH_API_H */
