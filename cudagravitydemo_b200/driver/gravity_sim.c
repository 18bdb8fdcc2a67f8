/* gravity_sim.c — the simulation program in C over the engine's C ABI.
 *
 * The reference's main() (basicGravity.cu:437-810) builds initial conditions,
 * uploads them, then per step builds the tree, walks it, integrates, and every
 * framesPerWrite = 5 steps writes a frame of outputDump.bin; it prints a
 * progress bar and the time per step.  This program does the same through
 * libbh_b200.so: seeded initial conditions (bh_ic_*; "demo" is the
 * reference's own galaxy, built on the device by bh_ic_demo), a device-resident
 * simulation whose step is one CUDA graph, frames gathered in body-id order
 * on the device (bh_sim_dump_frame), and FP64 energy / momentum at the start
 * and the end.
 *
 *   gravity_sim [-n N] [-steps S] [-ic plummer|disk|merger|demo] [-seed K]
 *               [-theta T] [-eps E] [-dt DT] [-G G] [-bits B]
 *               [-mac 0|1|2] [-alpha A] [-target X] [-mlp weights.f32]
 *               [-every F] [-o outputDump.bin | -o none] [-quiet]
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "bh_api.h"

static double now_s(void) {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static int fail(const char* what, int rc) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, bh_status_string(rc), bh_cuda_error_string());
    return 1;
}

/* inputOutput.c:60-76: percentage, bar, step and time per step on one line */
static void progress(int steps, int step, double msPerStep) {
    const int width = 40;
    double pct = 100.0 * step / (steps > 0 ? steps : 1);
    int filled = (int)(pct / 100.0 * width);
    char bar[41];
    for (int i = 0; i < width; i++) bar[i] = i < filled ? '|' : '-';
    bar[width] = 0;
    fprintf(stdout, "\r %6.2f%% [%s] step: %6d / %d, time (ms): %7.3f", pct, bar, step, steps, msPerStep);
    fflush(stdout);
}

int main(int argc, char** argv) {
    int n = 16384, steps = 100, every = 5, quiet = 0;
    unsigned long long seed = 0;
    const char* ic = "plummer";
    const char* out = "outputDump.bin";
    const char* mlp = NULL;
    bh_params p;
    bh_params_default(&p);
    p.theta = 0.5f;
    p.eps = 0.01f;
    p.dt = 1e-3f;
    for (int i = 1; i < argc; i++) {
        const char* a = argv[i];
        const char* v = i + 1 < argc ? argv[i + 1] : NULL;
        if (!strcmp(a, "-quiet")) { quiet = 1; continue; }
        if (!v) { fprintf(stderr, "missing value for %s\n", a); return 2; }
        i++;
        if (!strcmp(a, "-n")) n = atoi(v);
        else if (!strcmp(a, "-steps")) steps = atoi(v);
        else if (!strcmp(a, "-ic")) ic = v;
        else if (!strcmp(a, "-seed")) seed = strtoull(v, NULL, 10);
        else if (!strcmp(a, "-theta")) p.theta = (float)atof(v);
        else if (!strcmp(a, "-eps")) p.eps = (float)atof(v);
        else if (!strcmp(a, "-dt")) p.dt = (float)atof(v);
        else if (!strcmp(a, "-G")) p.G = (float)atof(v);
        else if (!strcmp(a, "-bits")) p.bitsPerAxis = atoi(v);
        else if (!strcmp(a, "-mac")) p.macMode = atoi(v);
        else if (!strcmp(a, "-alpha")) p.alpha = (float)atof(v);
        else if (!strcmp(a, "-target")) p.errTarget = (float)atof(v);
        else if (!strcmp(a, "-mlp")) mlp = v;
        else if (!strcmp(a, "-every")) every = atoi(v);
        else if (!strcmp(a, "-o")) out = v;
        else { fprintf(stderr, "unknown option %s\n", a); return 2; }
    }
    if (n <= 0 || steps < 0 || every <= 0) { fprintf(stderr, "bad sizes\n"); return 2; }

    float4* pos = (float4*)calloc((size_t)n, sizeof(float4));
    float3* vel = (float3*)calloc((size_t)n, sizeof(float3));
    if (!pos || !vel) { fprintf(stderr, "out of host memory\n"); return 1; }
    int rc;
    bh_galaxy_params g;
    bh_galaxy_params_default(&g);
    if (!strcmp(ic, "plummer")) rc = bh_ic_plummer(pos, vel, n, 1.0f, 1.0f, p.G, seed);
    else if (!strcmp(ic, "disk")) rc = bh_ic_disk_galaxy(pos, vel, n, &g, seed);
    else if (!strcmp(ic, "merger")) rc = bh_ic_merger(pos, vel, n, &g, 20.0f, 2.0f, 30.0f, seed);
    else if (!strcmp(ic, "demo")) rc = 0; /* built on the device below */
    else { fprintf(stderr, "unknown initial conditions %s\n", ic); return 2; }
    if (rc) return fail("initial conditions", rc);

    bh_sim* sim = NULL;
    if ((rc = bh_sim_create(&sim, n, &p, 0))) return fail("bh_sim_create", rc);
    if (p.macMode == 2) {
        if (!mlp) { fprintf(stderr, "-mac 2 needs -mlp weights.f32\n"); return 2; }
        float w[BH_MLP_PARAMS];
        FILE* f = fopen(mlp, "rb");
        if (!f || fread(w, sizeof(float), BH_MLP_PARAMS, f) != BH_MLP_PARAMS) {
            fprintf(stderr, "cannot read %d floats from %s\n", BH_MLP_PARAMS, mlp);
            return 1;
        }
        fclose(f);
        if ((rc = bh_sim_set_mac_mlp(sim, w))) return fail("bh_sim_set_mac_mlp", rc);
    }
    if ((rc = bh_sim_load(sim, pos, vel, n, 1))) return fail("bh_sim_load", rc);
    if (!strcmp(ic, "demo")) { /* the reference's galaxy, written straight into the simulation's state */
        float4* dpos = NULL;
        float3* dvel = NULL;
        bh_demo_params dp;
        bh_demo_params_default(&dp);
        dp.G = p.G;
        if ((rc = bh_sim_device_state(sim, &dpos, &dvel, NULL, NULL))) return fail("bh_sim_device_state", rc);
        if ((rc = bh_ic_demo(dpos, dvel, n, &dp, seed, bh_sim_stream(sim)))) return fail("bh_ic_demo", rc);
    }

    bh_diagnostics d0, d1;
    if ((rc = bh_sim_diagnostics(sim, 1, &d0))) return fail("bh_sim_diagnostics", rc);
    printf("bodies %d, steps %d, initial conditions %s (seed %llu), theta %g, eps %g, dt %g, mode %d\n", n, steps,
           ic, seed, p.theta, p.eps, p.dt, p.macMode);
    printf("E0 = %.12e (T %.6e, W %.6e)\n", d0.total, d0.kinetic, d0.potential);

    bh_dump* dump = NULL;
    const int frames = steps / every; /* basicGravity.cu:625 */
    if (strcmp(out, "none") && (rc = bh_dump_open(&dump, out, n, frames, NULL))) return fail("bh_dump_open", rc);

    const double t0 = now_s();
    double tLast = t0;
    int written = 0;
    for (int i = 0; i < steps; i++) {
        if ((rc = bh_sim_step(sim, 1))) return fail("bh_sim_step", rc);
        if (i % every == 0) { /* basicGravity.cu:793 */
            if (dump && written < frames) {
                if ((rc = bh_sim_dump_frame(dump, sim))) return fail("bh_sim_dump_frame", rc);
                written++;
            }
            if (!quiet) {
                if ((rc = bh_sim_synchronize(sim))) return fail("bh_sim_synchronize", rc);
                const double t = now_s();
                progress(steps, i + 1, 1e3 * (t - tLast) / (i == 0 ? 1 : every));
                tLast = t;
            }
        }
    }
    if ((rc = bh_sim_synchronize(sim))) return fail("bh_sim_synchronize", rc);
    const double elapsed = now_s() - t0;
    if (dump && (rc = bh_dump_close(dump))) return fail("bh_dump_close", rc);
    bh_stats st;
    if ((rc = bh_sim_stats(sim, &st))) return fail("bh_sim_stats", rc);
    if ((rc = bh_sim_diagnostics(sim, 1, &d1))) return fail("bh_sim_diagnostics", rc);
    if (!quiet) printf("\n");
    printf("time %.3f s, %.3f ms/step, %.1f steps/s, last walk %lld interactions, %d nodes\n", elapsed,
           steps ? 1e3 * elapsed / steps : 0.0, steps ? steps / elapsed : 0.0, st.interactions, st.nodeCount);
    double dp = 0.0;
    for (int k = 0; k < 3; k++) dp += (d1.momentum[k] - d0.momentum[k]) * (d1.momentum[k] - d0.momentum[k]);
    printf("E1 = %.12e, relative energy drift %.3e, |dP| %.3e\n", d1.total, (d1.total - d0.total) / fabs(d0.total),
           sqrt(dp));
    if (dump) printf("wrote %d frames to %s\n", written, out);
    bh_sim_destroy(sim);
    free(pos);
    free(vel);
    return 0;
}
