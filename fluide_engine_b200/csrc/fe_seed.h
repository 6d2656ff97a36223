/*
 * fe_seed.h -- deterministic particle seeding shared by the library and the CPU oracle.
 *
 * Seeding rule (subcell-centre rule): every subcell of edge h/2 whose centre lies inside a
 * region receives one particle at subcell_origin + U[0,1)^3 * h/2.  Subcells are visited with x
 * outermost, then y, then z innermost, and the three uniforms of a particle are drawn x, y, z in
 * that order from a splitmix64 stream started at `seed`.  Positions are produced in FP64 and the
 * caller rounds them to FP32; the oracle receives the same FP32 values widened back to FP64, so
 * both sides start bit-identical.
 *
 * The reference seeds with the unseeded global std::rand() (pic_simulator.cpp:521-548), which is
 * not reproducible; this rule replaces it for the analytic box / sphere scenes.
 */
#ifndef FE_SEED_H
#define FE_SEED_H

#include <stdint.h>
#include <stddef.h>
#include <math.h>

typedef struct {
    uint64_t state;
} fe_rng;

static inline uint64_t fe_rng_next(fe_rng* r)
{
    uint64_t z = (r->state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* Uniform double in [0, 1) with 53 random bits. */
static inline double fe_rng_uniform(fe_rng* r) { return (double)(fe_rng_next(r) >> 11) * (1.0 / 9007199254740992.0); }

/* Region kinds. */
enum { FE_REGION_BOX = 0, FE_REGION_SPHERE = 1 };

typedef struct {
    int kind;          /* FE_REGION_BOX or FE_REGION_SPHERE */
    double lo[3];      /* box: lower corner; sphere: centre */
    double hi[3];      /* box: upper corner; sphere: hi[0] = radius */
    double vel[3];     /* initial velocity of the particles seeded in this region */
} fe_region;

static inline int fe_region_contains(const fe_region* g, double x, double y, double z)
{
    if (g->kind == FE_REGION_BOX)
        return x >= g->lo[0] && x <= g->hi[0] && y >= g->lo[1] && y <= g->hi[1] && z >= g->lo[2] && z <= g->hi[2];
    double dx = x - g->lo[0], dy = y - g->lo[1], dz = z - g->lo[2];
    return dx * dx + dy * dy + dz * dz <= g->hi[0] * g->hi[0];
}

/*
 * Seeds the union of `nreg` regions (a subcell inside several regions is seeded once, with the
 * velocity of the first region that holds it) in a domain of n[3] cells of edge h[3] starting at
 * origin[3].  Writes at most `cap` particles (xyz interleaved) when pos != NULL and returns the
 * number of particles the rule produces, so a first call with pos == NULL sizes the buffers.
 */
static inline size_t fe_seed_regions_host(const fe_region* reg, int nreg, const int n[3], const double origin[3],
                                     const double h[3], uint64_t seed, float* pos, float* vel, size_t cap)
{
    fe_rng rng;
    rng.state = seed;
    size_t count = 0;
    const int m[3] = {2 * n[0], 2 * n[1], 2 * n[2]};
    const double hs[3] = {0.5 * h[0], 0.5 * h[1], 0.5 * h[2]};
    for (int i = 0; i < m[0]; ++i) {
        double cx = origin[0] + (i + 0.5) * hs[0];
        for (int j = 0; j < m[1]; ++j) {
            double cy = origin[1] + (j + 0.5) * hs[1];
            for (int k = 0; k < m[2]; ++k) {
                double cz = origin[2] + (k + 0.5) * hs[2];
                int which = -1;
                for (int g = 0; g < nreg; ++g)
                    if (fe_region_contains(&reg[g], cx, cy, cz)) { which = g; break; }
                if (which < 0) continue;
                double ux = fe_rng_uniform(&rng), uy = fe_rng_uniform(&rng), uz = fe_rng_uniform(&rng);
                if (pos && count < cap) {
                    pos[3 * count + 0] = (float)(origin[0] + i * hs[0] + ux * hs[0]);
                    pos[3 * count + 1] = (float)(origin[1] + j * hs[1] + uy * hs[1]);
                    pos[3 * count + 2] = (float)(origin[2] + k * hs[2] + uz * hs[2]);
                    if (vel) {
                        vel[3 * count + 0] = (float)reg[which].vel[0];
                        vel[3 * count + 1] = (float)reg[which].vel[1];
                        vel[3 * count + 2] = (float)reg[which].vel[2];
                    }
                }
                ++count;
            }
        }
    }
    return count;
}

#endif /* FE_SEED_H */
