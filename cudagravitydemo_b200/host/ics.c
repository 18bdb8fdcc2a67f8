/*
 * ics.c — seeded initial conditions for the B200 Barnes-Hut engine.
 *
 * The reference seeds its initial conditions from time(0) (basicGravity.cu:460)
 * and samples an exponential disk plus a uniform "halo" sphere
 * (initialConditions.c:246-382).  This file provides reproducible, seeded
 * generators for the workloads the engine is measured on:
 *   - Plummer sphere (radius from the inverse mass CDF, velocities by
 *     rejection sampling of the distribution function q^2 (1-q^2)^{7/2},
 *     after Aarseth, Henon & Wielen 1974);
 *   - exponential disk with a sech^2 vertical profile plus a Hernquist bulge,
 *     circular velocities from the enclosed mass plus Gaussian dispersion;
 *   - two such galaxies on a parabolic orbit.
 * The random numbers come from xoshiro256** (Blackman & Vigna) seeded through
 * splitmix64, so a seed gives the same bodies on every machine.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#include "bh_api.h"

/* ------------------------------------------------------------------ RNG */
typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void rng_seed(rng_t* r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static uint64_t rng_next(rng_t* r) {
    uint64_t* s = r->s;
    uint64_t result = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return result;
}

/* uniform in (0, 1): 53 random bits, never exactly 0 or 1 */
static double rng_uniform(rng_t* r) {
    return ((double)(rng_next(r) >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

static double rng_normal(rng_t* r) { /* Box-Muller */
    double u1 = rng_uniform(r), u2 = rng_uniform(r);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * M_PI * u2);
}

static void rng_direction(rng_t* r, double d[3]) {
    double cz = 2.0 * rng_uniform(r) - 1.0;
    double phi = 2.0 * M_PI * rng_uniform(r);
    double sz = sqrt(1.0 - cz * cz);
    d[0] = sz * cos(phi); d[1] = sz * sin(phi); d[2] = cz;
}

/* ------------------------------------------------------------- Plummer */
static void remove_bulk(float4* pos, float3* vel, int n) {
    double m = 0, cx = 0, cy = 0, cz = 0, vx = 0, vy = 0, vz = 0;
    for (int i = 0; i < n; i++) {
        double w = pos[i].w;
        m += w;
        cx += w * pos[i].x; cy += w * pos[i].y; cz += w * pos[i].z;
        vx += w * vel[i].x; vy += w * vel[i].y; vz += w * vel[i].z;
    }
    if (m <= 0) return;
    cx /= m; cy /= m; cz /= m; vx /= m; vy /= m; vz /= m;
    for (int i = 0; i < n; i++) {
        pos[i].x = (float)(pos[i].x - cx); pos[i].y = (float)(pos[i].y - cy); pos[i].z = (float)(pos[i].z - cz);
        vel[i].x = (float)(vel[i].x - vx); vel[i].y = (float)(vel[i].y - vy); vel[i].z = (float)(vel[i].z - vz);
    }
}

int bh_ic_plummer(float4* pos, float3* vel, int n, float M, float a, float G, uint64_t seed) {
    if (!pos || !vel || n <= 0 || !(M > 0) || !(a > 0)) return BH_ERR_INVALID;
    rng_t r;
    rng_seed(&r, seed);
    const double m = (double)M / n;
    for (int i = 0; i < n; i++) {
        /* enclosed-mass fraction u in (0, 0.999): cuts the 0.1% outermost
         * mass so a few far bodies do not stretch the bounding box */
        double u = 0.999 * rng_uniform(&r);
        double rad = a / sqrt(pow(u, -2.0 / 3.0) - 1.0);
        double d[3];
        rng_direction(&r, d);
        /* speed q * v_esc with q drawn from g(q) = q^2 (1 - q^2)^{7/2} */
        double q, y;
        do {
            q = rng_uniform(&r);
            y = 0.1 * rng_uniform(&r);
        } while (y > q * q * pow(1.0 - q * q, 3.5));
        double vesc = sqrt(2.0 * G * M / sqrt(rad * rad + (double)a * a));
        double v = q * vesc, e[3];
        rng_direction(&r, e);
        pos[i].x = (float)(rad * d[0]); pos[i].y = (float)(rad * d[1]); pos[i].z = (float)(rad * d[2]);
        pos[i].w = (float)m;
        vel[i].x = (float)(v * e[0]); vel[i].y = (float)(v * e[1]); vel[i].z = (float)(v * e[2]);
    }
    remove_bulk(pos, vel, n);
    return BH_OK;
}

/* ------------------------------------------------------- disk + bulge */
void bh_galaxy_params_default(bh_galaxy_params* g) {
    g->diskMass = 0.8f;
    g->diskScale = 1.0f;
    g->diskHeight = 0.1f;
    g->diskTrunc = 5.0f;   /* disk truncated at 5 R_d, as the reference's disk */
    g->bulgeMass = 0.2f;
    g->bulgeScale = 0.2f;
    g->bulgeTrunc = 20.0f; /* Hernquist bulge truncated at 20 scale radii */
    g->dispersion = 0.1f;
    g->G = 1.0f;
}

/* enclosed mass of an exponential disk within cylindrical radius R */
static double disk_enclosed(double Md, double Rd, double R) {
    double x = R / Rd;
    return Md * (1.0 - (1.0 + x) * exp(-x));
}

static double hernquist_enclosed(double Mb, double ab, double r) {
    double q = r / (r + ab);
    return Mb * q * q;
}

/* radius of an exponential disk with enclosed-mass fraction f (Newton on
 * 1 - (1 + x) e^-x = f) */
static double disk_radius(double f, double Rd) {
    double x = 1.0;
    for (int it = 0; it < 60; it++) {
        double e = exp(-x);
        double g = 1.0 - (1.0 + x) * e - f;
        double dg = x * e;
        double step = g / (dg > 1e-300 ? dg : 1e-300);
        x -= step;
        if (x < 1e-12) x = 1e-12;
        if (fabs(step) < 1e-14 * (1.0 + x)) break;
    }
    return x * Rd;
}

/* one galaxy of n bodies at the origin, disk in the x-y plane */
static void galaxy(float4* pos, float3* vel, int n, const bh_galaxy_params* g, rng_t* r) {
    const double Md = g->diskMass, Mb = g->bulgeMass, Mt = Md + Mb;
    const double m = Mt / n;
    int nb = (int)llround((double)n * Mb / Mt);
    int nd = n - nb;
    const double fdMax = 1.0 - (1.0 + g->diskTrunc) * exp(-(double)g->diskTrunc);
    const double rbMax = (double)g->bulgeTrunc * g->bulgeScale;
    const double qb = rbMax / (rbMax + g->bulgeScale);
    const double fbMax = qb * qb;
    for (int i = 0; i < n; i++) {
        double x, y, z, vx, vy, vz;
        if (i < nd) {
            double R = disk_radius(fdMax * rng_uniform(r), g->diskScale);
            double phi = 2.0 * M_PI * rng_uniform(r);
            z = g->diskHeight * atanh(2.0 * rng_uniform(r) - 1.0); /* sech^2 profile */
            x = R * cos(phi);
            y = R * sin(phi);
            double Menc = disk_enclosed(Md, g->diskScale, R) + hernquist_enclosed(Mb, g->bulgeScale, R);
            double vc = sqrt(g->G * Menc / (R > 1e-6 ? R : 1e-6));
            vx = -vc * sin(phi);
            vy = vc * cos(phi);
            vz = 0.0;
            double s = g->dispersion * vc;
            vx += s * rng_normal(r); vy += s * rng_normal(r); vz += s * rng_normal(r);
        } else {
            double sq = sqrt(fbMax * rng_uniform(r));
            double rad = g->bulgeScale * sq / (1.0 - sq);
            double d[3], e[3];
            rng_direction(r, d);
            x = rad * d[0]; y = rad * d[1]; z = rad * d[2];
            double Menc = hernquist_enclosed(Mb, g->bulgeScale, rad) +
                          disk_enclosed(Md, g->diskScale, rad);
            double vc = sqrt(g->G * Menc / (rad > 1e-6 ? rad : 1e-6));
            /* circular speed along a random direction perpendicular to the
             * radius vector (random orbital planes), plus dispersion */
            rng_direction(r, e);
            double dot = e[0] * d[0] + e[1] * d[1] + e[2] * d[2];
            double t[3] = {e[0] - dot * d[0], e[1] - dot * d[1], e[2] - dot * d[2]};
            double tn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
            if (tn < 1e-12) { t[0] = 1; t[1] = t[2] = 0; tn = 1; }
            double s = g->dispersion * vc;
            vx = vc * t[0] / tn + s * rng_normal(r);
            vy = vc * t[1] / tn + s * rng_normal(r);
            vz = vc * t[2] / tn + s * rng_normal(r);
        }
        pos[i].x = (float)x; pos[i].y = (float)y; pos[i].z = (float)z; pos[i].w = (float)m;
        vel[i].x = (float)vx; vel[i].y = (float)vy; vel[i].z = (float)vz;
    }
}

int bh_ic_disk_galaxy(float4* pos, float3* vel, int n, const bh_galaxy_params* g, uint64_t seed) {
    if (!pos || !vel || n <= 0 || !g) return BH_ERR_INVALID;
    if (!(g->diskMass >= 0) || !(g->bulgeMass >= 0) || !(g->diskMass + g->bulgeMass > 0) ||
        !(g->diskScale > 0) || !(g->diskHeight > 0) || !(g->bulgeScale > 0) || !(g->diskTrunc > 0) ||
        !(g->bulgeTrunc > 0))
        return BH_ERR_INVALID;
    rng_t r;
    rng_seed(&r, seed);
    galaxy(pos, vel, n, g, &r);
    remove_bulk(pos, vel, n);
    return BH_OK;
}

int bh_ic_merger(float4* pos, float3* vel, int n, const bh_galaxy_params* g, float separation,
                 float pericentre, float inclinationDeg, uint64_t seed) {
    if (!pos || !vel || n < 2 || !g || !(separation > pericentre) || !(pericentre > 0))
        return BH_ERR_INVALID;
    rng_t r;
    rng_seed(&r, seed);
    int n1 = n / 2, n2 = n - n1;
    galaxy(pos, vel, n1, g, &r);
    galaxy(pos + n1, vel + n1, n2, g, &r);
    /* incline the second disk about the x axis */
    double inc = inclinationDeg * M_PI / 180.0, ci = cos(inc), si = sin(inc);
    for (int i = n1; i < n; i++) {
        double y = pos[i].y, z = pos[i].z;
        pos[i].y = (float)(ci * y - si * z); pos[i].z = (float)(si * y + ci * z);
        double vy = vel[i].y, vz = vel[i].z;
        vel[i].y = (float)(ci * vy - si * vz); vel[i].z = (float)(si * vy + ci * vz);
    }
    /* parabolic relative orbit of two equal masses: speed sqrt(2 G Mt / d),
     * angular momentum sqrt(2 G Mt r_p) */
    double Mg = (double)g->diskMass + g->bulgeMass, Mt = 2.0 * Mg;
    double d = separation;
    double v = sqrt(2.0 * g->G * Mt / d);
    double h = sqrt(2.0 * g->G * Mt * pericentre);
    double vt = h / d;
    double vr = -sqrt(fmax(v * v - vt * vt, 0.0));
    /* relative position along +x, relative velocity (vr, vt, 0) */
    double rel[3] = {d, 0.0, 0.0}, vrel[3] = {vr, vt, 0.0};
    for (int i = 0; i < n; i++) {
        double s = (i < n1) ? -0.5 : 0.5;
        pos[i].x = (float)(pos[i].x + s * rel[0]);
        pos[i].y = (float)(pos[i].y + s * rel[1]);
        pos[i].z = (float)(pos[i].z + s * rel[2]);
        vel[i].x = (float)(vel[i].x + s * vrel[0]);
        vel[i].y = (float)(vel[i].y + s * vrel[1]);
        vel[i].z = (float)(vel[i].z + s * vrel[2]);
    }
    remove_bulk(pos, vel, n);
    return BH_OK;
}
