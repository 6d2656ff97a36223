/*
 * fe_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU FP64 restatement of the reference substep.
 *
 * Loaded by the tests, the smoke check and the CPU-baseline leg of bench.py as the checker of the
 * CUDA path; never part of the product.  Compiled with -ffp-contract=off so that every multiply and
 * add rounds separately, exactly as the reference's x86-64 build does.
 *
 * Reference file:line citations are relative to the reference project's src/ directory.
 */
#include "fe_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../fluide_engine_b200/csrc/fe_keys.h"
#include "../fluide_engine_b200/csrc/fe_seed.h"

/* Collider SDF value with no colliders (3d/collider_collection.cpp:3,38). */
#define OR_MAX_DISTANCE 1.7976931348623157E+30

typedef struct {
    int x, y, z;
} dim3i;

static inline size_t ix3(dim3i d, int i, int j, int k) { return (size_t)i + (size_t)d.x * ((size_t)j + (size_t)d.y * (size_t)k); }
static inline size_t cnt3(dim3i d) { return (size_t)d.x * (size_t)d.y * (size_t)d.z; }

/* A position-dependent external force (PointField, SwirlField, VolumeField), after the DirectionalField of
 * or_desc::gravity in PICSimulator::_externalForces. */
typedef struct {
    int kind;                    /* OR_FORCE_POINT / SWIRL / VOLUME */
    double origin[3], axis[3];   /* point / swirl origin; swirl axis (normalised, as the SwirlField constructor) */
    double strength;
    double cos_a, sin_a;         /* RotatePointAroundAxis's cos / sin of its 0.0001-degree angle */
    int n[3];                    /* volume field: node grid and its closest-point vectors (3 per node) */
    double o[3], h[3];
    double* field;
} or_force;
#define OR_MAX_FORCES 8

/* A TriangleMeshCollider (3d/triangle_mesh_collider.cpp:4-8): the mesh and its Mesh2SDF on the collider's own node
 * grid. */
typedef struct {
    int n[3];
    double o[3], h[3];
    double* sdf;
    double* V;
    int64_t* T;
    double* N;     /* mesh normals; triangle t's normal is N[T[4t + 3]] */
    size_t nv, nt, nn;
} or_collider;
#define OR_MAX_COLLIDERS 8

struct or_sim {
    or_desc d;
    dim3i n;                 /* cells */
    dim3i du, dv, dw;        /* face array sizes */
    double h[3];             /* gridSpacing = domainSize / gridSize (hybrid_simulator.cpp:8) */
    double xo[3], yo[3], zo[3];       /* velocity-grid data origins */
    double rxo[3], ryo[3], rzo[3];    /* FLIP residual-grid data origins */
    double sdf_origin[3];    /* domain origin + h/2 (hybrid_simulator.cpp:15) */
    size_t np;
    double *pos, *vel, *C;   /* AoS: 3, 3, 9 doubles per particle; C rows cX, cY, cZ */
    double *u, *v, *w;
    double *su, *sv, *sw;    /* FLIPSimulator::_velocityResiduals */
    uint8_t *mu, *mv, *mw;   /* Fluid3::xMarkers/yMarkers/zMarkers */
    double* sdf;             /* Fluid3::sdf */
    uint8_t* marks;          /* SinglePhasePressureSolver::_fluidMarkers */
    double* p;               /* LinearSystem::x, kept between substeps (linear_system.cpp:13-18) */
    double* b;               /* LinearSystem::b */
    int cg_it;
    double cg_res;
    uint8_t *dmu, *dmv, *dmw; /* diffusion face markers (BackwardEulerDiffusionSolver::_fluidMarkers) */
    int diff_it[3];           /* Jacobi iterations of the last diffusion solve, per component */
    or_force forces[OR_MAX_FORCES];
    int nforces;
    or_collider colliders[OR_MAX_COLLIDERS];
    int ncolliders;
    double* csdf;             /* ColliderCollection::_sdf on the n nodes at the domain origin; initially 0 */
    int enclosed_projection;  /* restate the GPU's treatment of enclosed FLUID components (off: the reference) */
};

/* ---------------------------------------------------------------- math_utils.hpp restatements */

/* Clamp(val, maxVal, minVal) (common/math_utils.hpp:13-28). */
static inline double clampd(double val, double maxv, double minv)
{
    if (val < minv) return minv;
    if (val > maxv) return maxv;
    return val;
}

/* Lerp (common/math_utils.hpp:30-34). */
double or_lerp(double a, double b, double f) { return (1 - f) * a + f * b; }

/* Trilerp via Bilerp (common/math_utils.hpp:36-46). c = x000,x100,x010,x110,x001,x101,x011,x111. */
double or_trilerp(const double c[8], double fx, double fy, double fz)
{
    double b0 = or_lerp(or_lerp(c[0], c[1], fx), or_lerp(c[2], c[3], fx), fy);
    double b1 = or_lerp(or_lerp(c[4], c[5], fx), or_lerp(c[6], c[7], fx), fy);
    return or_lerp(b0, b1, fz);
}

/* GetBarycentric with iLow = 0 (common/math_utils.hpp:48-73). */
static inline void barycentric(double x, int iHigh, int* i, double* f)
{
    double s = floor(x);
    int ii = (int)s;
    if (0 == iHigh) {
        ii = 0;
        *f = 0;
    } else if (ii < 0) {
        ii = 0;
        *f = 0;
    } else if (ii > iHigh - 1) {
        ii = iHigh - 1;
        *f = 1;
    } else {
        *f = x - s;
    }
    *i = ii;
}

typedef struct {
    int i[8], j[8], k[8];
} idx8;

/* GetCooridnatesAndWeights (common/math_utils.hpp:75-112). */
static void coords_weights(dim3i size, const double origin[3], const double h[3], const double x[3], idx8* id,
                           double w[8])
{
    int i, j, k;
    double fx, fy, fz;
    double nx = (x[0] - origin[0]) / h[0], ny = (x[1] - origin[1]) / h[1], nz = (x[2] - origin[2]) / h[2];
    barycentric(nx, size.x - 1, &i, &fx);
    barycentric(ny, size.y - 1, &j, &fy);
    barycentric(nz, size.z - 1, &k, &fz);
    int ip1 = i + 1 < size.x - 1 ? i + 1 : size.x - 1;
    int jp1 = j + 1 < size.y - 1 ? j + 1 : size.y - 1;
    int kp1 = k + 1 < size.z - 1 ? k + 1 : size.z - 1;
    const int ii[8] = {i, ip1, i, ip1, i, ip1, i, ip1};
    const int jj[8] = {j, j, jp1, jp1, j, j, jp1, jp1};
    const int kk[8] = {k, k, k, k, kp1, kp1, kp1, kp1};
    for (int t = 0; t < 8; ++t) {
        id->i[t] = ii[t];
        id->j[t] = jj[t];
        id->k[t] = kk[t];
    }
    w[0] = (1.00 - fx) * (1.00 - fy) * (1.00 - fz);
    w[1] = fx * (1.00 - fy) * (1.00 - fz);
    w[2] = (1.00 - fx) * fy * (1.00 - fz);
    w[3] = fx * fy * (1.00 - fz);
    w[4] = (1.00 - fx) * (1.00 - fy) * fz;
    w[5] = fx * (1.00 - fy) * fz;
    w[6] = (1.00 - fx) * fy * fz;
    w[7] = fx * fy * fz;
}

/* GetCooridnatesAndGradientWeights (common/math_utils.hpp:114-176); g[t][0..2] per corner. */
static void coords_grad_weights(dim3i size, const double origin[3], const double h[3], const double x[3], idx8* id,
                                double g[8][3])
{
    int i, j, k;
    double fx, fy, fz;
    double nx = (x[0] - origin[0]) / h[0], ny = (x[1] - origin[1]) / h[1], nz = (x[2] - origin[2]) / h[2];
    double ihx = 1 / h[0], ihy = 1 / h[1], ihz = 1 / h[2];
    barycentric(nx, size.x - 1, &i, &fx);
    barycentric(ny, size.y - 1, &j, &fy);
    barycentric(nz, size.z - 1, &k, &fz);
    int ip1 = i + 1 < size.x - 1 ? i + 1 : size.x - 1;
    int jp1 = j + 1 < size.y - 1 ? j + 1 : size.y - 1;
    int kp1 = k + 1 < size.z - 1 ? k + 1 : size.z - 1;
    const int ii[8] = {i, ip1, i, ip1, i, ip1, i, ip1};
    const int jj[8] = {j, j, jp1, jp1, j, j, jp1, jp1};
    const int kk[8] = {k, k, k, k, kp1, kp1, kp1, kp1};
    for (int t = 0; t < 8; ++t) {
        id->i[t] = ii[t];
        id->j[t] = jj[t];
        id->k[t] = kk[t];
    }
    g[0][0] = -ihx * (1 - fy) * (1 - fz);
    g[0][1] = -ihy * (1 - fx) * (1 - fz);
    g[0][2] = -ihz * (1 - fx) * (1 - fy);
    g[1][0] = ihx * (1 - fy) * (1 - fz);
    g[1][1] = fx * (-ihy) * (1 - fz);
    g[1][2] = fx * (1 - fy) * (-ihz);
    g[2][0] = (-ihx) * fy * (1 - fz);
    g[2][1] = (1 - fx) * ihy * (1 - fz);
    g[2][2] = (1 - fx) * fy * (-ihz);
    g[3][0] = ihx * fy * (1 - fz);
    g[3][1] = fx * ihy * (1 - fz);
    g[3][2] = fx * fy * (-ihz);
    g[4][0] = (-ihx) * (1 - fy) * fz;
    g[4][1] = (1 - fx) * (-ihy) * fz;
    g[4][2] = (1 - fx) * (1 - fy) * ihz;
    g[5][0] = ihx * (1 - fy) * fz;
    g[5][1] = fx * (-ihy) * fz;
    g[5][2] = fx * (1 - fy) * ihz;
    g[6][0] = (-ihx) * fy * fz;
    g[6][1] = (1 - fx) * ihy * fz;
    g[6][2] = (1 - fx) * fy * ihz;
    g[7][0] = ihx * fy * fz;
    g[7][1] = fx * ihy * fz;
    g[7][2] = fx * fy * ihz;
}

/* Clamped trilinear sample shared by FaceCenteredGrid3D::SampleArray
 * (grid_systems/face_centered_grid3d.cpp:339-371) and ScalarGrid3D::Sample (3d/scalar_grid3d.cpp:33-65). */
static double sample3(const double* arr, dim3i size, const double origin[3], const double h[3], const double pos[3])
{
    int i, j, k;
    double fx, fy, fz;
    double nx = (pos[0] - origin[0]) / h[0], ny = (pos[1] - origin[1]) / h[1], nz = (pos[2] - origin[2]) / h[2];
    barycentric(nx, size.x - 1, &i, &fx);
    barycentric(ny, size.y - 1, &j, &fy);
    barycentric(nz, size.z - 1, &k, &fz);
    int ip1 = i + 1 < size.x - 1 ? i + 1 : size.x - 1;
    int jp1 = j + 1 < size.y - 1 ? j + 1 : size.y - 1;
    int kp1 = k + 1 < size.z - 1 ? k + 1 : size.z - 1;
    double c[8] = {arr[ix3(size, i, j, k)],   arr[ix3(size, ip1, j, k)],   arr[ix3(size, i, jp1, k)],
                   arr[ix3(size, ip1, jp1, k)], arr[ix3(size, i, j, kp1)],   arr[ix3(size, ip1, j, kp1)],
                   arr[ix3(size, i, jp1, kp1)], arr[ix3(size, ip1, jp1, kp1)]};
    return or_trilerp(c, fx, fy, fz);
}

double or_sample_face_array(const double* arr, const int size[3], const double origin[3], const double h[3],
                            const double pos[3])
{
    dim3i d = {size[0], size[1], size[2]};
    return sample3(arr, d, origin, h, pos);
}

double or_scalar_sample(const double* arr, const int size[3], const double origin[3], const double h[3],
                        const double pos[3])
{
    dim3i d = {size[0], size[1], size[2]};
    return sample3(arr, d, origin, h, pos);
}

/* ExtrapolateToRegion (common/math_utils.hpp:186-253). */
static void extrapolate_to_region(const double* input, const uint8_t* valid, dim3i size, size_t iters, double* output)
{
    size_t n = cnt3(size);
    uint8_t* valid0 = (uint8_t*)malloc(n);
    uint8_t* valid1 = (uint8_t*)malloc(n);
    memcpy(valid0, valid, n);
    memcpy(valid1, valid, n);
    if (output != input) memcpy(output, input, n * sizeof(double));
    for (size_t it = 0; it < iters; ++it) {
        for (int i = 0; i < size.x; ++i)
            for (int j = 0; j < size.y; ++j)
                for (int k = 0; k < size.z; ++k) {
                    size_t c = ix3(size, i, j, k);
                    if (!valid0[c]) {
                        double sum = 0;
                        unsigned count = 0;
                        if (i + 1 < size.x && valid0[ix3(size, i + 1, j, k)]) { sum += output[ix3(size, i + 1, j, k)]; ++count; }
                        if (i > 0 && valid0[ix3(size, i - 1, j, k)]) { sum += output[ix3(size, i - 1, j, k)]; ++count; }
                        if (j + 1 < size.y && valid0[ix3(size, i, j + 1, k)]) { sum += output[ix3(size, i, j + 1, k)]; ++count; }
                        if (j > 0 && valid0[ix3(size, i, j - 1, k)]) { sum += output[ix3(size, i, j - 1, k)]; ++count; }
                        if (k + 1 < size.z && valid0[ix3(size, i, j, k + 1)]) { sum += output[ix3(size, i, j, k + 1)]; ++count; }
                        if (k > 0 && valid0[ix3(size, i, j, k - 1)]) { sum += output[ix3(size, i, j, k - 1)]; ++count; }
                        if (count > 0) {
                            output[c] = sum / count;
                            valid1[c] = 1;
                        }
                    } else {
                        valid1[c] = 1;
                    }
                }
        /* valid0.Swap(valid1): valid0 takes the grown mask, valid1 the previous one. */
        uint8_t* t = valid0;
        valid0 = valid1;
        valid1 = t;
    }
    free(valid0);
    free(valid1);
}

/* ---------------------------------------------------------------- construction */

static void* xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s); }

or_sim* or_create(const or_desc* d)
{
    if (!d || d->n[0] < 2 || d->n[1] < 2 || d->n[2] < 2) return NULL;
    or_sim* s = (or_sim*)calloc(1, sizeof(or_sim));
    s->d = *d;
    s->n = (dim3i){d->n[0], d->n[1], d->n[2]};
    s->du = (dim3i){d->n[0] + 1, d->n[1], d->n[2]};
    s->dv = (dim3i){d->n[0], d->n[1] + 1, d->n[2]};
    s->dw = (dim3i){d->n[0], d->n[1], d->n[2] + 1};
    for (int a = 0; a < 3; ++a) s->h[a] = d->size[a] / (double)d->n[a]; /* hybrid_simulator.cpp:8 */
    /* FaceCenteredGrid3D::CalculateDataOrigins (grid_systems/face_centered_grid3d.cpp:324-332) runs inside
     * SetGridSpacing before SetOrigin (hybrid_simulator.cpp:11-12), and Grid3D::SetOrigin does not recompute
     * them, so the velocity grid's data origins are taken from origin (0,0,0).  The FLIP residual grid is
     * constructed with the domain origin (flip_simulator.cpp:5). */
    const double zero[3] = {0, 0, 0};
    const double* o = zero;
    s->xo[0] = o[0] + s->h[0] * 0;
    s->xo[1] = o[1] + s->h[1] * 0.5;
    s->xo[2] = o[2] + s->h[2] * 0.5;
    s->yo[0] = o[0] + s->h[0] * 0.5;
    s->yo[1] = o[1] + s->h[1] * 0;
    s->yo[2] = o[2] + s->h[2] * 0.5;
    s->zo[0] = o[0] + s->h[0] * 0.5;
    s->zo[1] = o[1] + s->h[1] * 0.5;
    s->zo[2] = o[2] + s->h[2] * 0;
    o = d->origin;
    s->rxo[0] = o[0] + s->h[0] * 0;
    s->rxo[1] = o[1] + s->h[1] * 0.5;
    s->rxo[2] = o[2] + s->h[2] * 0.5;
    s->ryo[0] = o[0] + s->h[0] * 0.5;
    s->ryo[1] = o[1] + s->h[1] * 0;
    s->ryo[2] = o[2] + s->h[2] * 0.5;
    s->rzo[0] = o[0] + s->h[0] * 0.5;
    s->rzo[1] = o[1] + s->h[1] * 0.5;
    s->rzo[2] = o[2] + s->h[2] * 0;
    for (int a = 0; a < 3; ++a) s->sdf_origin[a] = d->origin[a] + s->h[a] / 2.0;
    size_t nc = cnt3(s->n);
    s->u = (double*)xcalloc(cnt3(s->du), sizeof(double));
    s->v = (double*)xcalloc(cnt3(s->dv), sizeof(double));
    s->w = (double*)xcalloc(cnt3(s->dw), sizeof(double));
    s->su = (double*)xcalloc(cnt3(s->du), sizeof(double));
    s->sv = (double*)xcalloc(cnt3(s->dv), sizeof(double));
    s->sw = (double*)xcalloc(cnt3(s->dw), sizeof(double));
    s->mu = (uint8_t*)xcalloc(cnt3(s->du), 1);
    s->mv = (uint8_t*)xcalloc(cnt3(s->dv), 1);
    s->mw = (uint8_t*)xcalloc(cnt3(s->dw), 1);
    s->sdf = (double*)xcalloc(nc, sizeof(double));
    s->marks = (uint8_t*)xcalloc(nc, 1);
    s->p = (double*)xcalloc(nc, sizeof(double));
    s->b = (double*)xcalloc(nc, sizeof(double));
    s->dmu = (uint8_t*)xcalloc(cnt3(s->du), 1);
    s->dmv = (uint8_t*)xcalloc(cnt3(s->dv), 1);
    s->dmw = (uint8_t*)xcalloc(cnt3(s->dw), 1);
    s->csdf = (double*)xcalloc(cnt3(s->n), sizeof(double));
    return s;
}

void or_destroy(or_sim* s)
{
    if (!s) return;
    free(s->pos); free(s->vel); free(s->C);
    free(s->u); free(s->v); free(s->w);
    free(s->su); free(s->sv); free(s->sw);
    free(s->mu); free(s->mv); free(s->mw);
    free(s->sdf); free(s->marks); free(s->p); free(s->b);
    free(s->dmu); free(s->dmv); free(s->dmw);
    for (int f = 0; f < s->nforces; ++f) free(s->forces[f].field);
    for (int c = 0; c < s->ncolliders; ++c) {
        free(s->colliders[c].sdf); free(s->colliders[c].V); free(s->colliders[c].T); free(s->colliders[c].N);
    }
    free(s->csdf);
    free(s);
}

int or_set_particles(or_sim* s, size_t n, const double* pos, const double* vel, const double* C)
{
    free(s->pos); free(s->vel); free(s->C);
    s->np = n;
    s->pos = (double*)xcalloc(3 * n, sizeof(double));
    s->vel = (double*)xcalloc(3 * n, sizeof(double));
    s->C = (double*)xcalloc(9 * n, sizeof(double));
    if (pos) memcpy(s->pos, pos, 3 * n * sizeof(double));
    if (vel) memcpy(s->vel, vel, 3 * n * sizeof(double));
    if (C) memcpy(s->C, C, 9 * n * sizeof(double));
    return 0;
}

size_t or_num_particles(const or_sim* s) { return s->np; }

void or_get_particles(const or_sim* s, double* pos, double* vel, double* C)
{
    if (pos) memcpy(pos, s->pos, 3 * s->np * sizeof(double));
    if (vel) memcpy(vel, s->vel, 3 * s->np * sizeof(double));
    if (C) memcpy(C, s->C, 9 * s->np * sizeof(double));
}

void or_get_grid(const or_sim* s, double* u, double* v, double* w)
{
    if (u) memcpy(u, s->u, cnt3(s->du) * sizeof(double));
    if (v) memcpy(v, s->v, cnt3(s->dv) * sizeof(double));
    if (w) memcpy(w, s->w, cnt3(s->dw) * sizeof(double));
}

void or_set_grid(or_sim* s, const double* u, const double* v, const double* w)
{
    if (u) memcpy(s->u, u, cnt3(s->du) * sizeof(double));
    if (v) memcpy(s->v, v, cnt3(s->dv) * sizeof(double));
    if (w) memcpy(s->w, w, cnt3(s->dw) * sizeof(double));
}

void or_get_pressure(const or_sim* s, double* p) { memcpy(p, s->p, cnt3(s->n) * sizeof(double)); }
void or_set_pressure(or_sim* s, const double* p) { memcpy(s->p, p, cnt3(s->n) * sizeof(double)); }
void or_get_marks(const or_sim* s, uint8_t* m) { memcpy(m, s->marks, cnt3(s->n)); }
void or_get_sdf(const or_sim* s, double* sdf) { memcpy(sdf, s->sdf, cnt3(s->n) * sizeof(double)); }
void or_get_rhs(const or_sim* s, double* b) { memcpy(b, s->b, cnt3(s->n) * sizeof(double)); }

void or_get_face_markers(const or_sim* s, uint8_t* mu, uint8_t* mv, uint8_t* mw)
{
    if (mu) memcpy(mu, s->mu, cnt3(s->du));
    if (mv) memcpy(mv, s->mv, cnt3(s->dv));
    if (mw) memcpy(mw, s->mw, cnt3(s->dw));
}

void or_get_snapshot(const or_sim* s, double* u, double* v, double* w)
{
    if (u) memcpy(u, s->su, cnt3(s->du) * sizeof(double));
    if (v) memcpy(v, s->sv, cnt3(s->dv) * sizeof(double));
    if (w) memcpy(w, s->sw, cnt3(s->dw) * sizeof(double));
}

/* ---------------------------------------------------------------- P2G */

/* PICSimulator::TransferParticles2Grid (pic_simulator.cpp:356-437), FLIPSimulator (flip_simulator.cpp:25-119)
 * and APICSimulator (apic_simulator.cpp:15-118).  PIC and APIC pass the CELL count as the clamp size
 * (pic_simulator.cpp:389,397,405; apic_simulator.cpp:58,71,84), FLIP the face-array size (flip_simulator.cpp:58). */
void or_stage_p2g(or_sim* s)
{
    size_t nu = cnt3(s->du), nv = cnt3(s->dv), nw = cnt3(s->dw);
    double* uw = (double*)xcalloc(nu, sizeof(double));
    double* vw = (double*)xcalloc(nv, sizeof(double));
    double* ww = (double*)xcalloc(nw, sizeof(double));
    memset(s->u, 0, nu * sizeof(double));
    memset(s->v, 0, nv * sizeof(double));
    memset(s->w, 0, nw * sizeof(double));
    memset(s->mu, 0, nu);
    memset(s->mv, 0, nv);
    memset(s->mw, 0, nw);
    const int flip = s->d.solver == OR_FLIP, apic = s->d.solver == OR_APIC;
    dim3i szu = flip ? s->du : s->n, szv = flip ? s->dv : s->n, szw = flip ? s->dw : s->n;
    const double* O = s->d.origin;
    const double* S = s->d.size;
    double hh[3] = {s->h[0] / 2.0, s->h[1] / 2.0, s->h[2] / 2.0}; /* apic_simulator.cpp:52 */
    for (size_t pi = 0; pi < s->np; ++pi) {
        const double* x = s->pos + 3 * pi;
        const double* vel = s->vel + 3 * pi;
        const double* cx = s->C + 9 * pi;
        idx8 id;
        double wt[8];
        /* u */
        double pc[3] = {x[0], x[1], x[2]};
        if (apic) {
            pc[1] = clampd(pc[1], O[1] + S[1] - hh[1], O[1] + hh[1]);
            pc[2] = clampd(pc[2], O[2] + S[2] - hh[2], O[2] + hh[2]);
        }
        coords_weights(szu, s->xo, s->h, x, &id, wt);
        for (int t = 0; t < 8; ++t) {
            size_t f = ix3(s->du, id.i[t], id.j[t], id.k[t]);
            double val = vel[0];
            if (apic) {
                double g0 = s->xo[0] + s->h[0] * (double)id.i[t];
                double g1 = s->xo[1] + s->h[1] * (double)id.j[t];
                double g2 = s->xo[2] + s->h[2] * (double)id.k[t];
                double term = cx[0] * (g0 - pc[0]) + cx[1] * (g1 - pc[1]) + cx[2] * (g2 - pc[2]);
                val = vel[0] + term;
            }
            s->u[f] += val * wt[t];
            uw[f] += wt[t];
            s->mu[f] = 1;
        }
        /* v */
        pc[0] = x[0]; pc[1] = x[1]; pc[2] = x[2];
        if (apic) {
            pc[0] = clampd(pc[0], O[0] + S[0] - hh[0], O[0] + hh[0]);
            pc[2] = clampd(pc[2], O[2] + S[2] - hh[2], O[2] + hh[2]);
        }
        coords_weights(szv, s->yo, s->h, x, &id, wt);
        for (int t = 0; t < 8; ++t) {
            size_t f = ix3(s->dv, id.i[t], id.j[t], id.k[t]);
            double val = vel[1];
            if (apic) {
                const double* cy = cx + 3;
                double g0 = s->yo[0] + s->h[0] * (double)id.i[t];
                double g1 = s->yo[1] + s->h[1] * (double)id.j[t];
                double g2 = s->yo[2] + s->h[2] * (double)id.k[t];
                double term = cy[0] * (g0 - pc[0]) + cy[1] * (g1 - pc[1]) + cy[2] * (g2 - pc[2]);
                val = vel[1] + term;
            }
            s->v[f] += val * wt[t];
            vw[f] += wt[t];
            s->mv[f] = 1;
        }
        /* w */
        pc[0] = x[0]; pc[1] = x[1]; pc[2] = x[2];
        if (apic) {
            pc[0] = clampd(pc[0], O[0] + S[0] - hh[0], O[0] + hh[0]);
            pc[1] = clampd(pc[1], O[1] + S[1] - hh[1], O[1] + hh[1]);
        }
        coords_weights(szw, s->zo, s->h, x, &id, wt);
        for (int t = 0; t < 8; ++t) {
            size_t f = ix3(s->dw, id.i[t], id.j[t], id.k[t]);
            double val = vel[2];
            if (apic) {
                const double* cz = cx + 6;
                double g0 = s->zo[0] + s->h[0] * (double)id.i[t];
                double g1 = s->zo[1] + s->h[1] * (double)id.j[t];
                double g2 = s->zo[2] + s->h[2] * (double)id.k[t];
                double term = cz[0] * (g0 - pc[0]) + cz[1] * (g1 - pc[1]) + cz[2] * (g2 - pc[2]);
                val = vel[2] + term;
            }
            s->w[f] += val * wt[t];
            ww[f] += wt[t];
            s->mw[f] = 1;
        }
    }
    for (size_t f = 0; f < nu; ++f) if (uw[f] > 0.0) s->u[f] /= uw[f];
    for (size_t f = 0; f < nv; ++f) if (vw[f] > 0.0) s->v[f] /= vw[f];
    for (size_t f = 0; f < nw; ++f) if (ww[f] > 0.0) s->w[f] /= ww[f];
    if (flip) { /* flip_simulator.cpp:107-118 */
        memcpy(s->su, s->u, nu * sizeof(double));
        memcpy(s->sv, s->v, nv * sizeof(double));
        memcpy(s->sw, s->w, nw * sizeof(double));
    }
    free(uw); free(vw); free(ww);
}

/* ---------------------------------------------------------------- particle SDF */

/* HashGridParticleSearcher::GetBucketIndex / GetHashKeyFromBucketIndex with a 64^3 table
 * (particle_systems/hash_grid_particle_searcher.cpp:133-152, particle_system.cpp:30-34). */
static inline int bucket_of(double x, double spacing) { return (int)floor(x / spacing); }
static inline int wrap64(int b)
{
    /* int % size_t converts b to size_t first; for 64 this equals the non-negative modulo. */
    return (int)((size_t)(long long)b % (size_t)64);
}
static inline size_t hash_key(int bx, int by, int bz)
{
    return (size_t)((wrap64(bz) * 64 + wrap64(by)) * 64 + wrap64(bx));
}

/* PICSimulator::BuildSignedDistanceField (pic_simulator.cpp:452-475) with HashGridParticleSearcher::Build and
 * ForEachNearbyPoint (hash_grid_particle_searcher.cpp:14-32, 97-126, 154-204).  ExtrapolateIntoCollider
 * (pic_simulator.cpp:497-519) is the identity with no colliders: every node is valid. */
static void extrapolate_into_collider(or_sim* s);
static double collider_sample(const or_sim* s, const double pos[3]);

void or_stage_sdf(or_sim* s)
{
    double maxH = s->h[0] > (s->h[1] > s->h[2] ? s->h[1] : s->h[2]) ? s->h[0] : (s->h[1] > s->h[2] ? s->h[1] : s->h[2]);
    double radious = 1.2 * maxH / sqrt(2.0);
    double band = 2.0 * radious;
    double spacing = 2 * radious;
    size_t nb = (size_t)64 * 64 * 64;
    size_t* start = (size_t*)xcalloc(nb + 1, sizeof(size_t));
    size_t* list = (size_t*)xcalloc(s->np, sizeof(size_t));
    size_t* key = (size_t*)xcalloc(s->np, sizeof(size_t));
    for (size_t pi = 0; pi < s->np; ++pi) {
        const double* x = s->pos + 3 * pi;
        key[pi] = hash_key(bucket_of(x[0], spacing), bucket_of(x[1], spacing), bucket_of(x[2], spacing));
        start[key[pi] + 1]++;
    }
    for (size_t b = 0; b < nb; ++b) start[b + 1] += start[b];
    size_t* fill = (size_t*)xcalloc(nb, sizeof(size_t));
    for (size_t pi = 0; pi < s->np; ++pi) list[start[key[pi]] + fill[key[pi]]++] = pi; /* push_back order */
    const double R2 = band * band;
    for (int i = 0; i < s->n.x; ++i)
        for (int j = 0; j < s->n.y; ++j)
            for (int k = 0; k < s->n.z; ++k) {
                double q[3] = {s->sdf_origin[0] + i * s->h[0], s->sdf_origin[1] + j * s->h[1],
                               s->sdf_origin[2] + k * s->h[2]}; /* Grid3D::GridIndexToPosition */
                double minDistance = band;
                if (s->np > 0) {
                    int ob[3] = {bucket_of(q[0], spacing), bucket_of(q[1], spacing), bucket_of(q[2], spacing)};
                    int nbk[8][3];
                    for (int t = 0; t < 8; ++t) { nbk[t][0] = ob[0]; nbk[t][1] = ob[1]; nbk[t][2] = ob[2]; }
                    int dx = ((ob[0] + 0.5f) * spacing <= q[0]) ? 1 : -1;
                    int dy = ((ob[1] + 0.5f) * spacing <= q[1]) ? 1 : -1;
                    int dz = ((ob[2] + 0.5f) * spacing <= q[2]) ? 1 : -1;
                    nbk[4][0] += dx; nbk[5][0] += dx; nbk[6][0] += dx; nbk[7][0] += dx;
                    nbk[2][1] += dy; nbk[3][1] += dy; nbk[6][1] += dy; nbk[7][1] += dy;
                    nbk[1][2] += dz; nbk[3][2] += dz; nbk[5][2] += dz; nbk[7][2] += dz;
                    for (int t = 0; t < 8; ++t) {
                        size_t kk = hash_key(nbk[t][0], nbk[t][1], nbk[t][2]);
                        for (size_t e = start[kk]; e < start[kk + 1]; ++e) {
                            const double* x = s->pos + 3 * list[e];
                            double ddx = x[0] - q[0], ddy = x[1] - q[1], ddz = x[2] - q[2];
                            double d2 = ddx * ddx + ddy * ddy + ddz * ddz;
                            if (d2 <= R2) {
                                double dist = sqrt(ddx * ddx + ddy * ddy + ddz * ddz);
                                if (dist < minDistance) minDistance = dist; /* std::min keeps the first on ties */
                            }
                        }
                    }
                }
                s->sdf[ix3(s->n, i, j, k)] = minDistance - radious;
            }
    free(start); free(list); free(key); free(fill);
    if (s->ncolliders > 0) extrapolate_into_collider(s);
}

/* SinglePhasePressureSolver::BuildMarkers (fluid_solvers/single_phase_pressure_solver.cpp:30-48).  Without
 * colliders the collider SDF is positive everywhere, so the BOUNDRY branch is never taken. */
void or_build_markers(or_sim* s)
{
    for (int i = 0; i < s->n.x; ++i)
        for (int j = 0; j < s->n.y; ++j)
            for (int k = 0; k < s->n.z; ++k) {
                /* FaceCenteredGrid3D::GetCellCenterPos (face_centered_grid3d.cpp:318-321) */
                double c[3] = {(s->d.origin[0] + 0.5 * s->h[0]) + s->h[0] * i,
                               (s->d.origin[1] + 0.5 * s->h[1]) + s->h[1] * j,
                               (s->d.origin[2] + 0.5 * s->h[2]) + s->h[2] * k};
                double v = sample3(s->sdf, s->n, s->sdf_origin, s->h, c);
                s->marks[ix3(s->n, i, j, k)] =
                    v < 0 ? OR_FLUID : ((s->ncolliders > 0 && collider_sample(s, c) < 0) ? OR_BOUNDRY : OR_AIR);
            }
}

/* ---------------------------------------------------------------- grid passes */

/* PICSimulator::ExtrapolateVelocityToAir (pic_simulator.cpp:477-495). */
void or_stage_extrapolate(or_sim* s)
{
    size_t iters = (size_t)ceil(s->d.max_cfl);
    size_t nu = cnt3(s->du), nv = cnt3(s->dv), nw = cnt3(s->dw);
    double* prev = (double*)malloc((nu > nv ? (nu > nw ? nu : nw) : (nv > nw ? nv : nw)) * sizeof(double));
    memcpy(prev, s->u, nu * sizeof(double));
    extrapolate_to_region(prev, s->mu, s->du, iters, s->u);
    memcpy(prev, s->v, nv * sizeof(double));
    extrapolate_to_region(prev, s->mv, s->dv, iters, s->v);
    memcpy(prev, s->w, nw * sizeof(double));
    extrapolate_to_region(prev, s->mw, s->dw, iters, s->w);
    free(prev);
}

static void constrain_with_colliders(or_sim* s);

/* BlockedBoundryConditionSolver::ConstrainVelocity (fluid_solvers/blocked_boundry_condition_solver.cpp:18-291).
 * Without colliders only the wall-layer zeroing (:198-244) changes the grid. */
void or_stage_bc(or_sim* s)
{
    if (s->ncolliders > 0) {
        constrain_with_colliders(s);
        return;
    }
    for (int k = 0; k < s->du.z; ++k)
        for (int j = 0; j < s->du.y; ++j) {
            s->u[ix3(s->du, 0, j, k)] = 0;
            s->u[ix3(s->du, s->du.x - 1, j, k)] = 0;
        }
    for (int k = 0; k < s->dv.z; ++k)
        for (int i = 0; i < s->dv.x; ++i) {
            s->v[ix3(s->dv, i, 0, k)] = 0;
            s->v[ix3(s->dv, i, s->dv.y - 1, k)] = 0;
        }
    for (int j = 0; j < s->dw.y; ++j)
        for (int i = 0; i < s->dw.x; ++i) {
            s->w[ix3(s->dw, i, j, 0)] = 0;
            s->w[ix3(s->dw, i, j, s->dw.z - 1)] = 0;
        }
}

/* PICSimulator::ComputeExternalForces (pic_simulator.cpp:203-212) with one DirectionalField
 * (forces/external_force.cpp:4-29, forces/directional_field.cpp:13-16). */
static void apply_position_forces(or_sim* s, double dt);

void or_stage_forces(or_sim* s, double dt)
{
    size_t nu = cnt3(s->du), nv = cnt3(s->dv), nw = cnt3(s->dw);
    for (size_t f = 0; f < nu; ++f) s->u[f] += dt * s->d.gravity[0];
    for (size_t f = 0; f < nv; ++f) s->v[f] += dt * s->d.gravity[1];
    for (size_t f = 0; f < nw; ++f) s->w[f] += dt * s->d.gravity[2];
    apply_position_forces(s, dt);
    or_stage_bc(s);
}

/* ---------------------------------------------------------------- pressure */

typedef struct {
    double c, r, u, f; /* LinearSystemMatrixRow center, right, up, front (linear_system/linear_system.hpp:9-15) */
} row4;

/* BLAS::Dot (linear_system/blas.cpp:4-19): i outer, k inner. */
static double blas_dot(const double* a, const double* b, dim3i n)
{
    double r = 0;
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) r += a[ix3(n, i, j, k)] * b[ix3(n, i, j, k)];
    return r;
}

/* BLAS::Residual (linear_system/blas.cpp:21-36). */
static void blas_residual(const row4* A, const double* x, const double* b, double* out, dim3i n)
{
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                size_t c = ix3(n, i, j, k);
                out[c] = b[c] - A[c].c * x[c] - ((i > 0) ? A[ix3(n, i - 1, j, k)].r * x[ix3(n, i - 1, j, k)] : 0.0) -
                         ((i + 1 < n.x) ? A[c].r * x[ix3(n, i + 1, j, k)] : 0.0) -
                         ((j > 0) ? A[ix3(n, i, j - 1, k)].u * x[ix3(n, i, j - 1, k)] : 0.0) -
                         ((j + 1 < n.y) ? A[c].u * x[ix3(n, i, j + 1, k)] : 0.0) -
                         ((k > 0) ? A[ix3(n, i, j, k - 1)].f * x[ix3(n, i, j, k - 1)] : 0.0) -
                         ((k + 1 < n.z) ? A[c].f * x[ix3(n, i, j, k + 1)] : 0.0);
            }
}

/* BLAS::MatrixVectorMultiplication (linear_system/blas.cpp:68-83). */
static void blas_spmv(const row4* A, const double* v, double* out, dim3i n)
{
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                size_t c = ix3(n, i, j, k);
                out[c] = A[c].c * v[c] + ((i > 0) ? A[ix3(n, i - 1, j, k)].r * v[ix3(n, i - 1, j, k)] : 0.0) +
                         ((i + 1 < n.x) ? A[c].r * v[ix3(n, i + 1, j, k)] : 0.0) +
                         ((j > 0) ? A[ix3(n, i, j - 1, k)].u * v[ix3(n, i, j - 1, k)] : 0.0) +
                         ((j + 1 < n.y) ? A[c].u * v[ix3(n, i, j + 1, k)] : 0.0) +
                         ((k > 0) ? A[ix3(n, i, j, k - 1)].f * v[ix3(n, i, j, k - 1)] : 0.0) +
                         ((k + 1 < n.z) ? A[c].f * v[ix3(n, i, j, k + 1)] : 0.0);
            }
}

/* BLAS::AXpY (linear_system/blas.cpp:38-44): out = a*x + y. */
static void blas_axpy(double a, const double* x, const double* y, double* out, size_t n)
{
    for (size_t c = 0; c < n; ++c) out[c] = a * x[c] + y[c];
}

/* SinglePhasePressureSolver::BuildSystem (fluid_solvers/single_phase_pressure_solver.cpp:99-164);
 * b uses FaceCenteredGrid3D::DivergenceAtCallCenter (grid_systems/face_centered_grid3d.cpp:157-166). */
static void build_system(dim3i n, const double h[3], const uint8_t* m, const double* u, const double* v,
                         const double* w, row4* A, double* b)
{
    dim3i du = {n.x + 1, n.y, n.z}, dv = {n.x, n.y + 1, n.z}, dw = {n.x, n.y, n.z + 1};
    double ih[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]};
    double ih2[3] = {ih[0] * ih[0], ih[1] * ih[1], ih[2] * ih[2]};
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                size_t c = ix3(n, i, j, k);
                row4* row = &A[c];
                row->c = row->r = row->u = row->f = 0.0;
                b[c] = 0.0;
                if (m[c] == OR_FLUID) {
                    double left = u[ix3(du, i, j, k)], right = u[ix3(du, i + 1, j, k)];
                    double down = v[ix3(dv, i, j, k)], up = v[ix3(dv, i, j + 1, k)];
                    double back = w[ix3(dw, i, j, k)], front = w[ix3(dw, i, j, k + 1)];
                    b[c] = (right - left) / h[0] + (up - down) / h[1] + (front - back) / h[2];
                    if (i + 1 < n.x && m[ix3(n, i + 1, j, k)] != OR_BOUNDRY) {
                        row->c += ih2[0];
                        if (m[ix3(n, i + 1, j, k)] == OR_FLUID) row->r -= ih2[0];
                    }
                    if (i > 0 && m[ix3(n, i - 1, j, k)] != OR_BOUNDRY) row->c += ih2[0];
                    if (j + 1 < n.y && m[ix3(n, i, j + 1, k)] != OR_BOUNDRY) {
                        row->c += ih2[1];
                        if (m[ix3(n, i, j + 1, k)] == OR_FLUID) row->u -= ih2[1];
                    }
                    if (j > 0 && m[ix3(n, i, j - 1, k)] != OR_BOUNDRY) row->c += ih2[1];
                    if (k + 1 < n.z && m[ix3(n, i, j, k + 1)] != OR_BOUNDRY) {
                        row->c += ih2[2];
                        if (m[ix3(n, i, j, k + 1)] == OR_FLUID) row->f -= ih2[2];
                    }
                    if (k > 0 && m[ix3(n, i, j, k - 1)] != OR_BOUNDRY) row->c += ih2[2];
                } else {
                    row->c = 1.0;
                }
            }
}

/* ConjugateGradientSolver::Solve (linear_system/conjugate_gradient_solver.cpp:14-55) with tolerance
 * rel * BLAS::L2Norm(b); x is the warm start and is updated in place.  Returns the iteration count. */
static int cg_solve(const row4* A, const double* b, double* x, dim3i n, double rel, int maxIt)
{
    size_t N = cnt3(n);
    double* r = (double*)malloc(N * sizeof(double));
    double* d = (double*)malloc(N * sizeof(double));
    double* q = (double*)malloc(N * sizeof(double));
    double* s = (double*)malloc(N * sizeof(double));
    double tol = rel * sqrt(blas_dot(b, b, n));
    blas_residual(A, x, b, r, n);
    memcpy(d, r, N * sizeof(double));
    double sigmaNew = blas_dot(r, d, n);
    int it = 0, trigger = 0;
    while (sigmaNew > tol * tol && it < maxIt) {
        blas_spmv(A, d, q, n);
        double alpha = sigmaNew / blas_dot(d, q, n);
        blas_axpy(alpha, d, x, x, N);
        if (trigger || (it % 50 == 0 && it > 0)) {
            blas_residual(A, x, b, r, n);
            trigger = 0;
        } else {
            blas_axpy(-alpha, q, r, r, N);
        }
        memcpy(s, r, N * sizeof(double));
        double sigmaOld = sigmaNew;
        sigmaNew = blas_dot(r, s, n);
        if (sigmaNew > sigmaOld) trigger = 1;
        double beta = sigmaNew / sigmaOld;
        blas_axpy(beta, d, s, d, N);
        it++;
    }
    free(r); free(d); free(q); free(s);
    return it;
}

static double true_rel_residual(const row4* A, const double* b, const double* x, dim3i n)
{
    size_t N = cnt3(n);
    double* r = (double*)malloc(N * sizeof(double));
    blas_residual(A, x, b, r, n);
    double rn = sqrt(blas_dot(r, r, n)), bn = sqrt(blas_dot(b, b, n));
    free(r);
    return bn > 0 ? rn / bn : rn;
}

/* SinglePhasePressureSolver::ApplyPressure (fluid_solvers/single_phase_pressure_solver.cpp:56-92): output
 * equals the input except the +x/+y/+z faces of FLUID cells whose neighbour is not BOUNDRY. */
static void apply_pressure(dim3i n, const double h[3], const uint8_t* m, const double* p, double* u, double* v,
                           double* w)
{
    dim3i du = {n.x + 1, n.y, n.z}, dv = {n.x, n.y + 1, n.z}, dw = {n.x, n.y, n.z + 1};
    double sc[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]};
    /* Reads of in(...) are of faces no other cell writes, so updating in place equals out = in + ... */
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                if (m[ix3(n, i, j, k)] != OR_FLUID) continue;
                double pc = p[ix3(n, i, j, k)];
                if (i + 1 < n.x && m[ix3(n, i + 1, j, k)] != OR_BOUNDRY)
                    u[ix3(du, i + 1, j, k)] = u[ix3(du, i + 1, j, k)] + sc[0] * (p[ix3(n, i + 1, j, k)] - pc);
                if (j + 1 < n.y && m[ix3(n, i, j + 1, k)] != OR_BOUNDRY)
                    v[ix3(dv, i, j + 1, k)] = v[ix3(dv, i, j + 1, k)] + sc[1] * (p[ix3(n, i, j + 1, k)] - pc);
                if (k + 1 < n.z && m[ix3(n, i, j, k + 1)] != OR_BOUNDRY)
                    w[ix3(dw, i, j, k + 1)] = w[ix3(dw, i, j, k + 1)] + sc[2] * (p[ix3(n, i, j, k + 1)] - pc);
            }
}

int or_project(const int nn[3], const double h[3], const uint8_t* marks, double* u, double* v, double* w, double* p,
               double rel_tol, int max_it, double* rel_residual)
{
    dim3i n = {nn[0], nn[1], nn[2]};
    size_t N = cnt3(n);
    row4* A = (row4*)malloc(N * sizeof(row4));
    double* b = (double*)malloc(N * sizeof(double));
    build_system(n, h, marks, u, v, w, A, b);
    int it = cg_solve(A, b, p, n, rel_tol, max_it);
    if (rel_residual) *rel_residual = true_rel_residual(A, b, p, n);
    apply_pressure(n, h, marks, p, u, v, w);
    free(A);
    free(b);
    return it;
}

/* PICSimulator::ComputePressure (pic_simulator.cpp:224-229) -> SinglePhasePressureSolver::Solve
 * (fluid_solvers/single_phase_pressure_solver.cpp:21-28), then ApplyBoundryCondition. */
/* Not the reference: the GPU's solvable form of a collider scene's system (enabled by
 * or_set_enclosed_projection; the default follows the reference).  With colliders, FLUID cells can form
 * components that touch no AIR cell (pure-Neumann blocks walled in by BOUNDRY cells and domain walls),
 * whose rows the reference leaves singular and, in general, inconsistent, so its CG cannot converge there.
 * (1) A FLUID cell with no in-domain non-BOUNDRY neighbour has an all-zero row: it becomes an identity row
 * with b = 0 (pressure 0; ApplyPressure never reads it toward a BOUNDRY or out-of-domain face).
 * (2) FLUID cells are grouped into 6-connected components; a component without an AIR neighbour loses the
 * mean of its right-hand side, which leaves a consistent block unchanged and makes an inconsistent one
 * solvable.  Components are found by a union-find over the FLUID cells in cell order. */
static size_t uf_find(size_t* parent, size_t x)
{
    while (parent[x] != x) {
        parent[x] = parent[parent[x]];
        x = parent[x];
    }
    return x;
}

static void project_enclosed(dim3i n, const uint8_t* m, row4* A, double* b, double* p)
{
    size_t N = cnt3(n);
    size_t* parent = (size_t*)malloc(N * sizeof(size_t));
    uint8_t* open = (uint8_t*)calloc(N, 1);
    double* sum = (double*)calloc(N, sizeof(double));
    size_t* cnt = (size_t*)calloc(N, sizeof(size_t));
    for (size_t c = 0; c < N; ++c) parent[c] = c;
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                size_t c = ix3(n, i, j, k);
                if (m[c] != OR_FLUID) continue;
                if (A[c].c == 0.0) { /* (1) all-zero row */
                    A[c].c = 1.0;
                    A[c].r = A[c].u = A[c].f = 0.0;
                    b[c] = 0.0;
                    p[c] = 0.0;
                }
                size_t nb[3] = {i + 1 < n.x ? ix3(n, i + 1, j, k) : c, j + 1 < n.y ? ix3(n, i, j + 1, k) : c,
                                k + 1 < n.z ? ix3(n, i, j, k + 1) : c};
                for (int q = 0; q < 3; ++q) {
                    if (nb[q] == c || m[nb[q]] != OR_FLUID) continue;
                    size_t ra = uf_find(parent, c), rb = uf_find(parent, nb[q]);
                    if (ra != rb) parent[ra > rb ? ra : rb] = ra < rb ? ra : rb;
                }
            }
    for (int i = 0; i < n.x; ++i)
        for (int j = 0; j < n.y; ++j)
            for (int k = 0; k < n.z; ++k) {
                size_t c = ix3(n, i, j, k);
                if (m[c] != OR_FLUID) continue;
                size_t r = uf_find(parent, c);
                if ((i > 0 && m[ix3(n, i - 1, j, k)] == OR_AIR) || (i + 1 < n.x && m[ix3(n, i + 1, j, k)] == OR_AIR) ||
                    (j > 0 && m[ix3(n, i, j - 1, k)] == OR_AIR) || (j + 1 < n.y && m[ix3(n, i, j + 1, k)] == OR_AIR) ||
                    (k > 0 && m[ix3(n, i, j, k - 1)] == OR_AIR) || (k + 1 < n.z && m[ix3(n, i, j, k + 1)] == OR_AIR))
                    open[r] = 1;
                sum[r] += b[c];
                cnt[r] += 1;
            }
    for (size_t c = 0; c < N; ++c) {
        if (m[c] != OR_FLUID) continue;
        size_t r = uf_find(parent, c);
        if (!open[r]) b[c] -= sum[r] / (double)cnt[r];
    }
    free(parent); free(open); free(sum); free(cnt);
}

void or_set_enclosed_projection(or_sim* s, int on) { s->enclosed_projection = on ? 1 : 0; }

void or_stage_pressure(or_sim* s, double dt)
{
    (void)dt; /* neither dt nor density enters the solve (single_phase_pressure_solver.cpp:59-60) */
    or_build_markers(s);
    size_t N = cnt3(s->n);
    row4* A = (row4*)malloc(N * sizeof(row4));
    build_system(s->n, s->h, s->marks, s->u, s->v, s->w, A, s->b);
    if (s->enclosed_projection && s->ncolliders > 0) project_enclosed(s->n, s->marks, A, s->b, s->p);
    s->cg_it = cg_solve(A, s->b, s->p, s->n, s->d.cg_rel_tol, s->d.cg_max_it);
    s->cg_res = true_rel_residual(A, s->b, s->p, s->n);
    apply_pressure(s->n, s->h, s->marks, s->p, s->u, s->v, s->w);
    free(A);
    or_stage_bc(s);
}

/* ---------------------------------------------------------------- diffusion (viscosity) */

/* JacobiIterationSolver::Solve (linear_system/jacobi_iteration_solver.cpp:14-37) with its Relax (:39-76) and
 * CalculateTolerance (:79-83 = sqrt(BLAS::Dot(r, r)) of BLAS::Residual).  The reference's default diffusion
 * solver, CudaJacobiIterationSolver(1000, 5, 1e-14) (fluid_solvers/backward_euler_diffusion_solver.cpp:10),
 * relaxes with the same expression (linear_system/cuda_jacobi_iteration_solver.cu:5-24) on the same check
 * schedule (:49-61); only its residual norm sums in another order.  Returns the iterations run; the result is
 * left in x. */
static int jacobi_solve(const row4* A, const double* b, double* x, dim3i n, int max_it, int check, double tol)
{
    size_t N = cnt3(n);
    double* xt = (double*)xcalloc(N, sizeof(double));
    double* res = (double*)xcalloc(N, sizeof(double));
    double* cur = x; /* system->x */
    double* nxt = xt; /* _xTemp */
    int done = max_it;
    for (int it = 0; it < max_it; ++it) {
        for (int i = 0; i < n.x; ++i)
            for (int j = 0; j < n.y; ++j)
                for (int k = 0; k < n.z; ++k) {
                    size_t c = ix3(n, i, j, k);
                    double r = ((i > 0) ? A[ix3(n, i - 1, j, k)].r * cur[ix3(n, i - 1, j, k)] : 0.0) +
                               ((i + 1 < n.x) ? A[c].r * cur[ix3(n, i + 1, j, k)] : 0.0) +
                               ((j > 0) ? A[ix3(n, i, j - 1, k)].u * cur[ix3(n, i, j - 1, k)] : 0.0) +
                               ((j + 1 < n.y) ? A[c].u * cur[ix3(n, i, j + 1, k)] : 0.0) +
                               ((k > 0) ? A[ix3(n, i, j, k - 1)].f * cur[ix3(n, i, j, k - 1)] : 0.0) +
                               ((k + 1 < n.z) ? A[c].f * cur[ix3(n, i, j, k + 1)] : 0.0);
                    nxt[c] = (b[c] - r) / A[c].c;
                }
        double* t = cur; /* system->x.Swap(_xTemp) */
        cur = nxt;
        nxt = t;
        if (it != 0 && it % check == 0) {
            blas_residual(A, cur, b, res, n);
            if (sqrt(blas_dot(res, res, n)) < tol) {
                done = it + 1;
                break;
            }
        }
    }
    if (cur != x) memcpy(x, cur, N * sizeof(double));
    free(xt);
    free(res);
    return done;
}

/* One component of BackwardEulerDiffusionSolver::Solve (fluid_solvers/backward_euler_diffusion_solver.cpp:
 * 20-49): markers from the fluid SDF sampled at the face positions of the copy-constructed velocity grid,
 * whose data origins include the domain origin (face_centered_grid3d.cpp:11-17,303-316; the collider SDF is
 * positive, so BOUNDRY never occurs), BuildMatrix (:136-198), BuildVectors (:200-242), then the Jacobi solve. */
static int diffuse_component(or_sim* s, double* arr, dim3i sz, const double org[3], const double c[3],
                             uint8_t* mk)
{
    size_t N = cnt3(sz);
    for (int i = 0; i < sz.x; ++i)
        for (int j = 0; j < sz.y; ++j)
            for (int k = 0; k < sz.z; ++k) {
                double pos[3] = {org[0] + s->h[0] * (double)i, org[1] + s->h[1] * (double)j,
                                 org[2] + s->h[2] * (double)k};
                mk[ix3(sz, i, j, k)] = sample3(s->sdf, s->n, s->sdf_origin, s->h, pos) < 0 ? OR_FLUID : OR_AIR;
            }
    row4* A = (row4*)malloc((N ? N : 1) * sizeof(row4));
    double* b = (double*)xcalloc(N, sizeof(double));
    for (int i = 0; i < sz.x; ++i)
        for (int j = 0; j < sz.y; ++j)
            for (int k = 0; k < sz.z; ++k) {
                size_t f = ix3(sz, i, j, k);
                row4* row = &A[f];
                row->c = 1.0;
                row->u = row->f = row->r = 0.0;
                b[f] = arr[f]; /* b = x = arr; BOUNDRY neighbours would add c * arr */
                if (mk[f] != OR_FLUID) continue;
                if (i + 1 < sz.x) {
                    if (mk[ix3(sz, i + 1, j, k)] != OR_AIR) row->c += c[0];
                    if (mk[ix3(sz, i + 1, j, k)] == OR_FLUID) row->r -= c[0];
                }
                if (i > 0 && mk[ix3(sz, i - 1, j, k)] != OR_AIR) row->c += c[0];
                if (j + 1 < sz.y) {
                    if (mk[ix3(sz, i, j + 1, k)] != OR_AIR) row->c += c[1];
                    if (mk[ix3(sz, i, j + 1, k)] == OR_FLUID) row->u -= c[1];
                }
                if (j > 0 && mk[ix3(sz, i, j - 1, k)] != OR_AIR) row->c += c[1];
                if (k + 1 < sz.z) {
                    if (mk[ix3(sz, i, j, k + 1)] != OR_AIR) row->c += c[2];
                    if (mk[ix3(sz, i, j, k + 1)] == OR_FLUID) row->f -= c[2];
                }
                if (k > 0 && mk[ix3(sz, i, j, k - 1)] != OR_AIR) row->c += c[2];
            }
    int its = jacobi_solve(A, b, arr, sz, 1000, 5, 0.00000000000001);
    free(A);
    free(b);
    return its;
}

/* PICSimulator::ComputeDiffusion (pic_simulator.cpp:214-222).  The call passes dt and viscosity swapped
 * into DiffusionSolver::Solve; c = (timeInterval * viscosity) / (h * h) is the same product either way. */
void or_stage_diffusion(or_sim* s, double dt)
{
    if (!(s->d.viscosity > 0.0)) return;
    double c[3];
    for (int a = 0; a < 3; ++a) c[a] = (s->d.viscosity * dt) / (s->h[a] * s->h[a]);
    s->diff_it[0] = diffuse_component(s, s->u, s->du, s->rxo, c, s->dmu);
    s->diff_it[1] = diffuse_component(s, s->v, s->dv, s->ryo, c, s->dmv);
    s->diff_it[2] = diffuse_component(s, s->w, s->dw, s->rzo, c, s->dmw);
    or_stage_bc(s);
}

int or_diffusion_iterations(const or_sim* s, int component)
{
    return (component >= 0 && component < 3) ? s->diff_it[component] : -1;
}

void or_get_diffusion_markers(const or_sim* s, uint8_t* mu, uint8_t* mv, uint8_t* mw)
{
    if (mu) memcpy(mu, s->dmu, cnt3(s->du));
    if (mv) memcpy(mv, s->dmv, cnt3(s->dv));
    if (mw) memcpy(mw, s->dmw, cnt3(s->dw));
}

double or_divergence_l2(const or_sim* s)
{
    double acc = 0;
    for (int k = 0; k < s->n.z; ++k)
        for (int j = 0; j < s->n.y; ++j)
            for (int i = 0; i < s->n.x; ++i) {
                if (s->marks[ix3(s->n, i, j, k)] != OR_FLUID) continue;
                double dv = (s->u[ix3(s->du, i + 1, j, k)] - s->u[ix3(s->du, i, j, k)]) / s->h[0] +
                            (s->v[ix3(s->dv, i, j + 1, k)] - s->v[ix3(s->dv, i, j, k)]) / s->h[1] +
                            (s->w[ix3(s->dw, i, j, k + 1)] - s->w[ix3(s->dw, i, j, k)]) / s->h[2];
                acc += dv * dv;
            }
    return sqrt(acc);
}

/* ---------------------------------------------------------------- G2P and advection */

/* FaceCenteredGrid3D::Sample (grid_systems/face_centered_grid3d.cpp:138-144) on the velocity grid. */
static void sample_velocity(const or_sim* s, const double* u, const double* v, const double* w, const double* xo,
                            const double* yo, const double* zo, const double pos[3], double out[3])
{
    out[0] = sample3(u, s->du, xo, s->h, pos);
    out[1] = sample3(v, s->dv, yo, s->h, pos);
    out[2] = sample3(w, s->dw, zo, s->h, pos);
}

/* TransferGrid2Particles: PIC (pic_simulator.cpp:439-450), FLIP (flip_simulator.cpp:121-161),
 * APIC (apic_simulator.cpp:120-176). */
void or_stage_g2p(or_sim* s)
{
    if (s->d.solver == OR_FLIP) {
        size_t nu = cnt3(s->du), nv = cnt3(s->dv), nw = cnt3(s->dw);
        for (size_t f = 0; f < nu; ++f) s->su[f] = s->u[f] - s->su[f];
        for (size_t f = 0; f < nv; ++f) s->sv[f] = s->v[f] - s->sv[f];
        for (size_t f = 0; f < nw; ++f) s->sw[f] = s->w[f] - s->sw[f];
        double fb = s->d.blend;
        for (size_t pi = 0; pi < s->np; ++pi) {
            double* vel = s->vel + 3 * pi;
            const double* x = s->pos + 3 * pi;
            double dv[3], pic[3];
            sample_velocity(s, s->su, s->sv, s->sw, s->rxo, s->ryo, s->rzo, x, dv);
            double flip[3] = {vel[0] + dv[0], vel[1] + dv[1], vel[2] + dv[2]};
            if (fb > 0.0) {
                sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, x, pic);
                for (int a = 0; a < 3; ++a) flip[a] = (1 - fb) * flip[a] + fb * pic[a];
            }
            vel[0] = flip[0]; vel[1] = flip[1]; vel[2] = flip[2];
        }
        return;
    }
    if (s->d.solver == OR_PIC) {
        for (size_t pi = 0; pi < s->np; ++pi)
            sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, s->pos + 3 * pi, s->vel + 3 * pi);
        return;
    }
    /* APIC */
    const double* O = s->d.origin;
    const double* S = s->d.size;
    double hh[3] = {s->h[0] / 2.0, s->h[1] / 2.0, s->h[2] / 2.0};
    for (size_t pi = 0; pi < s->np; ++pi) {
        const double* x = s->pos + 3 * pi;
        double* c = s->C + 9 * pi;
        sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, x, s->vel + 3 * pi);
        for (int a = 0; a < 9; ++a) c[a] = 0;
        idx8 id;
        double g[8][3];
        double pc[3] = {x[0], clampd(x[1], O[1] + S[1] - hh[1], O[1] + hh[1]), clampd(x[2], O[2] + S[2] - hh[2], O[2] + hh[2])};
        coords_grad_weights(s->n, s->xo, s->h, pc, &id, g);
        for (int t = 0; t < 8; ++t) {
            double val = s->u[ix3(s->du, id.i[t], id.j[t], id.k[t])];
            c[0] += g[t][0] * val; c[1] += g[t][1] * val; c[2] += g[t][2] * val;
        }
        pc[0] = clampd(x[0], O[0] + S[0] - hh[0], O[0] + hh[0]); pc[1] = x[1];
        pc[2] = clampd(x[2], O[2] + S[2] - hh[2], O[2] + hh[2]);
        coords_grad_weights(s->n, s->yo, s->h, pc, &id, g);
        for (int t = 0; t < 8; ++t) {
            double val = s->v[ix3(s->dv, id.i[t], id.j[t], id.k[t])];
            c[3] += g[t][0] * val; c[4] += g[t][1] * val; c[5] += g[t][2] * val;
        }
        pc[0] = clampd(x[0], O[0] + S[0] - hh[0], O[0] + hh[0]);
        pc[1] = clampd(x[1], O[1] + S[1] - hh[1], O[1] + hh[1]); pc[2] = x[2];
        coords_grad_weights(s->n, s->zo, s->h, pc, &id, g);
        for (int t = 0; t < 8; ++t) {
            double val = s->w[ix3(s->dw, id.i[t], id.j[t], id.k[t])];
            c[6] += g[t][0] * val; c[7] += g[t][1] * val; c[8] += g[t][2] * val;
        }
    }
}

static void resolve_collision(const or_collider* c, const double prev[3], double* pos, double* vel);

/* PICSimulator::MoveParticles (pic_simulator.cpp:239-312).  Without colliders the collider response never fires
 * (the collider SDF is positive everywhere).  With colliders, a particle that ends inside the collider SDF makes
 * every collider c resolve particle number c (the loop variable of :300-302 shadows the particle index), from this
 * particle's start position. */
void or_stage_move(or_sim* s, double dt)
{
    unsigned nsub = (unsigned)(s->d.max_cfl > 1.0 ? s->d.max_cfl : 1.0);
    double sdt = dt / nsub;
    const double* O = s->d.origin;
    const double* S = s->d.size;
    for (size_t pi = 0; pi < s->np; ++pi) {
        double* x = s->pos + 3 * pi;
        double* vel = s->vel + 3 * pi;
        double pt0[3] = {x[0], x[1], x[2]}, pt1[3] = {x[0], x[1], x[2]};
        const double pt0s[3] = {x[0], x[1], x[2]}; /* startParticlePosition */
        for (unsigned t = 0; t < nsub; ++t) {
            double v0[3], mid[3], mv[3];
            sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, pt0, v0);
            for (int a = 0; a < 3; ++a) mid[a] = pt0[a] + 0.5 * sdt * v0[a];
            sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, mid, mv);
            for (int a = 0; a < 3; ++a) pt1[a] = pt0[a] + sdt * mv[a];
            for (int a = 0; a < 3; ++a) pt0[a] = pt1[a];
        }
        for (int a = 0; a < 3; ++a) {
            if (pt1[a] <= O[a]) { pt1[a] = O[a]; vel[a] = 0.0; }
            if (pt1[a] >= O[a] + S[a]) { pt1[a] = O[a] + S[a]; vel[a] = 0.0; }
        }
        x[0] = pt1[0]; x[1] = pt1[1]; x[2] = pt1[2];
        if (s->ncolliders > 0 && collider_sample(s, x) < 0) {
            const double start[3] = {pt0s[0], pt0s[1], pt0s[2]};
            for (int c = 0; c < s->ncolliders; ++c)
                if ((size_t)c < s->np) resolve_collision(&s->colliders[c], start, s->pos + 3 * c, s->vel + 3 * c);
        }
    }
}

/* PICSimulator::ComputeAdvection (pic_simulator.cpp:231-237). */
void or_stage_advection(or_sim* s, double dt)
{
    or_stage_extrapolate(s);
    or_stage_bc(s);
    or_stage_g2p(s);
    or_stage_move(s, dt);
}

/* PICSimulator::OnAdvanceTimeStep (pic_simulator.cpp:111-154) with OnBeginAdvanceTimeStep (:156-196).
 * No emitters; BuildCollider leaves the collider SDF at its constant; viscosity 0 skips diffusion. */
void or_substep(or_sim* s, double dt)
{
    or_build_collider(s);
    or_stage_p2g(s);
    or_stage_sdf(s);
    or_stage_extrapolate(s);
    or_stage_bc(s);
    or_stage_forces(s, dt);
    or_stage_diffusion(s, dt);
    or_stage_pressure(s, dt);
    or_stage_advection(s, dt);
}

/* PICSimulator::Cfl (pic_simulator.cpp:80-97). */
double or_cfl(const or_sim* s, double dt)
{
    double maxV = 0.0;
    for (int i = 0; i < s->n.x; ++i)
        for (int j = 0; j < s->n.y; ++j)
            for (int k = 0; k < s->n.z; ++k) {
                double cx = 0.5 * (s->u[ix3(s->du, i, j, k)] + s->u[ix3(s->du, i + 1, j, k)]);
                double cy = 0.5 * (s->v[ix3(s->dv, i, j, k)] + s->v[ix3(s->dv, i, j + 1, k)]);
                double cz = 0.5 * (s->w[ix3(s->dw, i, j, k)] + s->w[ix3(s->dw, i, j, k + 1)]);
                double vx = fabs(cx) + dt * 0.0, vy = fabs(cy) + dt * -9.8, vz = fabs(cz) + dt * 0.0;
                maxV = maxV > vx ? maxV : vx;
                maxV = maxV > vy ? maxV : vy;
                maxV = maxV > vz ? maxV : vz;
            }
    double minH = s->h[0] < (s->h[1] < s->h[2] ? s->h[1] : s->h[2]) ? s->h[0] : (s->h[1] < s->h[2] ? s->h[1] : s->h[2]);
    return maxV * dt / minH;
}

/* PICSimulator::NumberOfSubTimeSteps (pic_simulator.cpp:349-354). */
unsigned or_number_of_substeps(const or_sim* s, double dt)
{
    double c = ceil(or_cfl(s, dt) / s->d.max_cfl);
    return (unsigned)(c > 1.0 ? c : 1.0);
}

/* PhysicsAnimation::AdvanceTimeStep (physics_animation.cpp:64-92). */
int or_advance_time(or_sim* s, double frame_dt)
{
    double remaining = frame_dt;
    int count = 0;
    while (remaining > 0.0000000001) {
        unsigned n = or_number_of_substeps(s, remaining);
        double sub = remaining / (double)n;
        or_substep(s, sub);
        remaining -= sub;
        ++count;
    }
    return count;
}

int or_cg_iterations(const or_sim* s) { return s->cg_it; }
double or_cg_rel_residual(const or_sim* s) { return s->cg_res; }

/* ---------------------------------------------------------------- keys and seeding */

void or_sort_keys(const float* pos, size_t n, const int dims[3], const float origin[3], const float inv_h[3],
                  uint32_t* keys_sorted, uint32_t* perm)
{
    uint32_t space = fe_key_space(dims[0], dims[1], dims[2]);
    uint32_t* key = (uint32_t*)malloc((n ? n : 1) * sizeof(uint32_t));
    size_t* start = (size_t*)calloc((size_t)space + 1, sizeof(size_t));
    for (size_t i = 0; i < n; ++i) {
        key[i] = fe_particle_key(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], origin, inv_h, dims[0], dims[1], dims[2]);
        start[key[i] + 1]++;
    }
    for (uint32_t k = 0; k < space; ++k) start[k + 1] += start[k];
    for (size_t i = 0; i < n; ++i) {
        size_t slot = start[key[i]]++;
        perm[slot] = (uint32_t)i;
        keys_sorted[slot] = key[i];
    }
    free(key);
    free(start);
}

size_t or_seed_regions(const void* regions, int nreg, const int n[3], const double origin[3], const double h[3],
                       uint64_t seed, float* pos, float* vel, size_t cap)
{
    return fe_seed_regions_host((const fe_region*)regions, nreg, n, origin, h, seed, pos, vel, cap);
}

/* ---------------------------------------------------------------- surface (marching cubes + OBJ) */

#include "../fluide_engine_b200/csrc/fe_mc_tables.h"

static const unsigned long long or_mc3d[256] = FE_MC_CASES_3D;
static const unsigned long long or_mc2d[16] = FE_MC_CASES_2D;
static const int or_mc_edge[12][2] = FE_MC_EDGE_CORNERS;

typedef struct {
    double *v, *n;    /* 3 per vertex */
    int64_t* t;       /* 4 per triangle: vertices, normal index */
    size_t nv, nt, cap_v, cap_t;
    int64_t* map;     /* vertex map (MarchingCubeVertexMap): key -> vertex id, -1 = absent */
    size_t map_size;
} or_mesh;

static void mesh_add_vertex(or_mesh* m, const double p[3], const double nrm[3])
{
    if (m->nv < m->cap_v) {
        memcpy(m->v + 3 * m->nv, p, 3 * sizeof(double));
        memcpy(m->n + 3 * m->nv, nrm, 3 * sizeof(double));
    }
    ++m->nv;
}

static void mesh_add_triangle(or_mesh* m, const int64_t f[3])
{
    if (m->nt < m->cap_t) {
        int64_t* t = m->t + 4 * m->nt;
        t[0] = f[0]; t[1] = f[1]; t[2] = f[2];
        t[3] = (int64_t)m->nv - 1; /* mesh->GetNormals().size() - 1 */
    }
    ++m->nt;
}

/* MarchingCubesSolver::GlobalVertexId / GlobalEdgeId (marching_cubes_solver.cpp:157-181): keys on the doubled grid. */
static size_t mc_key(int i, int j, int k, const int n[3], int ox, int oy, int oz)
{
    return ((size_t)(2 * k + oz) * 2 * (size_t)n[1] + (size_t)(2 * j + oy)) * 2 * (size_t)n[0] + (size_t)(2 * i + ox);
}
static const int mc_vertex_off[8][3] = {{0, 0, 0}, {2, 0, 0}, {2, 0, 2}, {0, 0, 2}, {0, 2, 0}, {2, 2, 0}, {2, 2, 2}, {0, 2, 2}};
static const int mc_edge_off[12][3] = {{1, 0, 0}, {2, 0, 1}, {1, 0, 2}, {0, 0, 1}, {1, 2, 0}, {2, 2, 1},
                                       {1, 2, 2}, {0, 2, 1}, {0, 1, 0}, {2, 1, 0}, {2, 1, 2}, {0, 1, 2}};

static double sdfv(const double* s, const int n[3], int i, int j, int k) { return s[(size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k)]; }

/* MarchingCubesSolver::Gradient (marching_cubes_solver.cpp:116-155). */
static void mc_gradient(const double* s, const int n[3], const double h[3], int i, int j, int k, double g[3])
{
    int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
    if (i > n[0] - 2) ip = i; else if (i == 0) im = 0;
    if (j > n[1] - 2) jp = j; else if (j == 0) jm = 0;
    if (k > n[2] - 2) kp = k; else if (k == 0) km = 0;
    const double ih[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]};
    g[0] = 0.5 * ih[0] * (sdfv(s, n, ip, j, k) - sdfv(s, n, im, j, k));
    g[1] = 0.5 * ih[1] * (sdfv(s, n, i, jp, k) - sdfv(s, n, i, jm, k));
    g[2] = 0.5 * ih[2] * (sdfv(s, n, i, j, kp) - sdfv(s, n, i, j, km));
}

/* Grid3D::GridIndexToPosition (common/grid3d.hpp:20-23). */
static void grid_pos(const double o[3], const double h[3], int i, int j, int k, double p[3])
{
    p[0] = o[0] + i * h[0];
    p[1] = o[1] + j * h[1];
    p[2] = o[2] + k * h[2];
}

static int64_t map_get(or_mesh* m, size_t key) { return key < m->map_size ? m->map[key] : -1; }
static void map_put(or_mesh* m, size_t key, int64_t id) { if (key < m->map_size) m->map[key] = id; }

/* SolveSingleCube (marching_cubes_solver.cpp:183-316), iso value 0. */
static void mc_cube(const double* s, const int n[3], const double o[3], const double h[3], int i, int j, int k, or_mesh* m)
{
    static const int cof[8][3] = FE_MC_CORNER_OFFSETS;
    double data[8], nrm[8][3];
    for (int c = 0; c < 8; ++c) {
        data[c] = sdfv(s, n, i + cof[c][0], j + cof[c][1], k + cof[c][2]);
        mc_gradient(s, n, h, i + cof[c][0], j + cof[c][1], k + cof[c][2], nrm[c]);
    }
    int cfg = 0;
    for (int c = 0; c < 8; ++c)
        if (data[c] <= 0.0) cfg |= 1 << c;
    if (cfg == 0 || cfg == 255) return;
    /* BoundingBox3D with origin GridIndexToPosition(i, j, k) and size h; Corner (3d/bounding_box_3d.cpp:23-31) */
    double bo[3];
    grid_pos(o, h, i, j, k, bo);
    static const int index_map[8] = {0, 1, 5, 4, 2, 3, 7, 6};
    double e[12][3], en[12][3];
    for (int ed = 0; ed < 12; ++ed) {
        const int a = or_mc_edge[ed][0], b = or_mc_edge[ed][1];
        if (((cfg >> a) & 1) == ((cfg >> b) & 1)) continue;
        double p0[3], p1[3];
        for (int d = 0; d < 3; ++d) {
            const int ca = index_map[a], cb = index_map[b];
            const double offa = ((ca >> d) & 1) ? 0.5 : -0.5, offb = ((cb >> d) & 1) ? 0.5 : -0.5;
            p0[d] = (h[d] * offa + bo[d]) + 0.5 * h[d];
            p1[d] = (h[d] * offb + bo[d]) + 0.5 * h[d];
        }
        const double phi0 = data[a] - 0.0, phi1 = data[b] - 0.0;
        double alpha = (fabs(phi0) + fabs(phi1) > 0.000000001) ? fabs(phi0) / (fabs(phi0) + fabs(phi1)) : 0.5;
        if (alpha < 0.000001) alpha = 0.000001;
        if (alpha > 0.999999) alpha = 0.999999;
        for (int d = 0; d < 3; ++d) {
            e[ed][d] = (1.0 - alpha) * p0[d] + alpha * p1[d];
            en[ed][d] = (1.0 - alpha) * nrm[a][d] + alpha * nrm[b][d];
        }
    }
    const unsigned long long cs = or_mc3d[cfg];
    const int ntri = (int)(cs >> 60);
    for (int t = 0; t < ntri; ++t) {
        int64_t f[3];
        for (int q = 0; q < 3; ++q) {
            const int ed = (int)((cs >> (4 * (3 * t + q))) & 15);
            const size_t key = mc_key(i, j, k, n, mc_edge_off[ed][0], mc_edge_off[ed][1], mc_edge_off[ed][2]);
            int64_t id = map_get(m, key);
            if (id < 0) {
                /* SafeNormalize: n / |n| when |n|^2 > 0 (Vector3::Normalize, common/vector3.hpp:149-152) */
                double nn[3] = {en[ed][0], en[ed][1], en[ed][2]};
                const double len = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
                if (len * len > 0.0) {
                    const double l2 = sqrt(nn[0] * nn[0] + nn[1] * nn[1] + nn[2] * nn[2]);
                    nn[0] /= l2; nn[1] /= l2; nn[2] /= l2;
                }
                id = (int64_t)m->nv;
                mesh_add_vertex(m, e[ed], nn);
                map_put(m, key, id);
            }
            f[q] = id;
        }
        mesh_add_triangle(m, f);
    }
}

/* SolveSingleSquare (marching_cubes_solver.cpp:497-583): data, keys (4 corners then 4 edges), corners, normal. */
static void mc_square(const double data[4], const size_t keys[8], const double nrm[3], const double corners[4][3], or_mesh* m)
{
    int cfg = 0;
    for (int c = 0; c < 4; ++c)
        if (data[c] <= 0.0) cfg |= 1 << c;
    if (cfg == 0) return;
    double e[4][3];
    for (int ed = 0; ed < 4; ++ed) {
        const int a = ed, b = (ed + 1) & 3;
        if (((cfg >> a) & 1) == ((cfg >> b) & 1)) continue;
        const double phi0 = data[a] - 0.0, phi1 = data[b] - 0.0;
        double alpha = (fabs(phi0) + fabs(phi1) > 1e-12) ? fabs(phi0) / (fabs(phi0) + fabs(phi1)) : (double)0.5f;
        if (alpha < (double)0.000001f) alpha = (double)0.000001f;
        if (alpha > (double)0.999999f) alpha = (double)0.999999f;
        for (int d = 0; d < 3; ++d) e[ed][d] = (1.0 - alpha) * corners[a][d] + alpha * corners[b][d];
    }
    const unsigned long long cs = or_mc2d[cfg];
    const int ntri = (int)(cs >> 60);
    for (int t = 0; t < ntri; ++t) {
        int64_t f[3];
        for (int q = 0; q < 3; ++q) {
            const int iv = (int)((cs >> (4 * (3 * t + q))) & 15);
            const size_t key = keys[iv];
            int64_t id = map_get(m, key);
            if (id < 0) {
                id = (int64_t)m->nv;
                mesh_add_vertex(m, iv < 4 ? corners[iv] : e[iv - 4], nrm);
                map_put(m, key, id);
            }
            f[q] = id;
        }
        mesh_add_triangle(m, f);
    }
}

/* One cap square of the domain face `side` (0 back z-, 1 front z+, 2 left x-, 3 right x+, 4 down y-, 5 up y+) at
 * cube (i, j, k): SolveXY / SolveYZ / SolveXZ (marching_cubes_solver.cpp:318-495) list its corners and keys. */
static void mc_cap(const double* s, const int n[3], const double o[3], const double h[3], int side, int i, int j, int k,
                   or_mesh* m)
{
    /* corner node offsets per side, in the square's corner order; vertex ids (mc_vertex_off) and edge ids */
    static const int corner_off[6][4][3] = {
        {{1, 0, 0}, {0, 0, 0}, {0, 1, 0}, {1, 1, 0}}, {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}},
        {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}}, {{1, 0, 1}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}},
        {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}}, {{1, 1, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}}};
    static const int vid[6][4] = {{1, 0, 4, 5}, {3, 2, 6, 7}, {0, 3, 7, 4}, {2, 1, 5, 6}, {0, 1, 2, 3}, {5, 4, 7, 6}};
    static const int eid[6][4] = {{0, 8, 4, 9}, {2, 10, 6, 11}, {3, 11, 7, 8}, {1, 9, 5, 10}, {0, 1, 2, 3}, {4, 7, 6, 5}};
    static const double normal[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}};
    double data[4], corners[4][3];
    size_t keys[8];
    for (int c = 0; c < 4; ++c) {
        const int a = i + corner_off[side][c][0], b = j + corner_off[side][c][1], d = k + corner_off[side][c][2];
        data[c] = sdfv(s, n, a, b, d);
        grid_pos(o, h, a, b, d, corners[c]);
        keys[c] = mc_key(i, j, k, n, mc_vertex_off[vid[side][c]][0], mc_vertex_off[vid[side][c]][1], mc_vertex_off[vid[side][c]][2]);
        keys[4 + c] = mc_key(i, j, k, n, mc_edge_off[eid[side][c]][0], mc_edge_off[eid[side][c]][1], mc_edge_off[eid[side][c]][2]);
    }
    mc_square(data, keys, normal[side], corners, m);
}

int or_build_surface(const double* sdf, const int n[3], const double origin[3], const double h[3], double* vertices,
                     double* normals, int64_t* tris, size_t cap_v, size_t cap_t, size_t* nv, size_t* nt)
{
    if (n[0] < 2 || n[1] < 2 || n[2] < 2) return -1;
    or_mesh m = {vertices, normals, tris, 0, 0, vertices ? cap_v : 0, tris ? cap_t : 0, NULL, 0};
    m.map_size = 8 * (size_t)n[0] * (size_t)n[1] * (size_t)n[2];
    m.map = (int64_t*)malloc(m.map_size * sizeof(int64_t));
    int64_t* map2 = (int64_t*)malloc(m.map_size * sizeof(int64_t));
    if (!m.map || !map2) { free(m.map); free(map2); return -1; }
#define OR_MAP_RESET(p) for (size_t q_ = 0; q_ < m.map_size; ++q_) (p)[q_] = -1
    /* CalculateXYZMeshPart: i, j, k nested, one vertex map */
    OR_MAP_RESET(m.map);
    for (int i = 0; i < n[0] - 1; ++i)
        for (int j = 0; j < n[1] - 1; ++j)
            for (int k = 0; k < n[2] - 1; ++k) mc_cube(sdf, n, origin, h, i, j, k, &m);
    /* the three cap parts, each with one vertex map per side; a part's two sides alternate per square */
    int64_t* maps[2] = {m.map, map2};
    for (int part = 0; part < 3; ++part) {
        OR_MAP_RESET(maps[0]);
        OR_MAP_RESET(maps[1]);
        const int outer = part == 0 ? n[1] - 1 : n[2] - 1;          /* XY: j, YZ: k, XZ: k */
        const int inner = part == 1 ? n[1] - 1 : n[0] - 1;          /* XY: i, YZ: j, XZ: i */
        for (int a = 0; a < outer; ++a)
            for (int b = 0; b < inner; ++b)
                for (int sd = 0; sd < 2; ++sd) {
                    int i, j, k;
                    if (part == 0) { i = b; j = a; k = sd ? n[2] - 2 : 0; }
                    else if (part == 1) { i = sd ? n[0] - 2 : 0; j = b; k = a; }
                    else { i = b; j = sd ? n[1] - 2 : 0; k = a; }
                    m.map = maps[sd];
                    mc_cap(sdf, n, origin, h, 2 * part + sd, i, j, k, &m);
                }
    }
#undef OR_MAP_RESET
    free(maps[0]);
    free(maps[1]);
    *nv = m.nv;
    *nt = m.nt;
    return 0;
}

/* OBJManager::OnSave (3d/obj_manager.cpp:14-90): std::to_string is printf "%f"; indices are 1-based, the
 * normal index of a triangle is written as size_t (so -1 prints as 0). */
int or_write_obj(const char* path, const char* name, const double* v, const double* vn, size_t nv, const int64_t* t,
                 size_t nt)
{
    FILE* f = fopen(path, "wb");
    if (!f) return -1;
    fprintf(f, "mtllib test.mtl\n");
    fprintf(f, "o %s\n\n", name ? name : "");
    for (size_t i = 0; i < nv; ++i) fprintf(f, "v %f %f %f\n", v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    fprintf(f, "\n");
    for (size_t i = 0; i < nv; ++i) fprintf(f, "vn %f %f %f\n", vn[3 * i], vn[3 * i + 1], vn[3 * i + 2]);
    fprintf(f, "\n");
    fprintf(f, "s off\n\n");
    for (size_t i = 0; i < nt; ++i) {
        const uint64_t nidx = (uint64_t)t[4 * i + 3] + 1u;
        fprintf(f, "f %llu//%llu %llu//%llu %llu//%llu\n", (unsigned long long)t[4 * i] + 1, (unsigned long long)nidx,
                (unsigned long long)t[4 * i + 1] + 1, (unsigned long long)nidx, (unsigned long long)t[4 * i + 2] + 1,
                (unsigned long long)nidx);
    }
    fprintf(f, "\n");
    return fclose(f) == 0 ? 0 : -1;
}

/* ---------------------------------------------------------------- mesh -> SDF, mesh seeding */

static double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static double len3(const double a[3]) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

/* Collisions::ClossestPointOnTriangle (3d/collisions.cpp:21-212): the region-based closest point of a triangle
 * (Eberly, "Distance Between Point and Triangle in 3D"), in the reference's operation order. */
static void closest_on_triangle(const double pt[3], const double p0[3], const double p1[3], const double p2[3], double out[3])
{
    double diff[3], e0[3], e1[3];
    for (int d = 0; d < 3; ++d) { diff[d] = p0[d] - pt[d]; e0[d] = p1[d] - p0[d]; e1[d] = p2[d] - p0[d]; }
    const double a00 = dot3(e0, e0), a01 = dot3(e0, e1), a11 = dot3(e1, e1);
    const double b0 = dot3(diff, e0), b1 = dot3(diff, e1);
    const double dd = a00 * a11 - a01 * a01;
    const double det = (dd < 0.0) ? 0.0 : dd; /* std::max(x, 0.0) = (x < 0.0) ? 0.0 : x (keeps -0.0 and NaN) */
    double s = a01 * b1 - a11 * b0;
    double t = a01 * b0 - a00 * b1;
    if (s + t <= det) {
        if (s < 0) {
            if (t < 0) { /* region 4 */
                if (b0 < 0) {
                    t = 0;
                    if (-b0 >= a00) s = 1; else s = -b0 / a00;
                } else {
                    s = 0;
                    if (b1 >= 0) t = 0; else if (-b1 >= a11) t = 1; else t = -b1 / a11;
                }
            } else { /* region 3 */
                s = 0;
                if (b1 >= 0) t = 0; else if (-b1 >= a11) t = 1; else t = -b1 / a11;
            }
        } else if (t < 0) { /* region 5 */
            t = 0;
            if (b0 >= 0) s = 0; else if (-b0 >= a00) s = 1; else s = -b0 / a00;
        } else { /* region 0 */
            s /= det;
            t /= det;
        }
    } else {
        double tmp0, tmp1, numer, denom;
        if (s < 0) { /* region 2 */
            tmp0 = a01 + b0;
            tmp1 = a11 + b1;
            if (tmp1 > tmp0) {
                numer = tmp1 - tmp0;
                denom = a00 - 2 * a01 + a11;
                if (numer >= denom) { s = 1; t = 0; } else { s = numer / denom; t = 1 - s; }
            } else {
                s = 0;
                if (tmp1 <= 0) t = 1; else if (b1 >= 0) t = 0; else t = -b1 / a11;
            }
        } else if (t < 0) { /* region 6 */
            tmp0 = a01 + b1;
            tmp1 = a00 + b0;
            if (tmp1 > tmp0) {
                numer = tmp1 - tmp0;
                denom = a00 - 2 * a01 + a11;
                if (numer >= denom) { t = 1; s = 0; } else { t = numer / denom; s = 1 - t; }
            } else {
                t = 0;
                if (tmp1 <= 0) s = 1; else if (b0 >= 0) s = 0; else s = -b0 / a00;
            }
        } else { /* region 1 */
            numer = a11 + b1 - a01 - b0;
            if (numer <= 0) { s = 0; t = 1; }
            else {
                denom = a00 - 2 * a01 + a11;
                if (numer >= denom) { s = 1; t = 0; } else { s = numer / denom; t = 1 - s; }
            }
        }
    }
    for (int d = 0; d < 3; ++d) out[d] = (p0[d] + s * e0[d]) + t * e1[d];
}

/* Collisions::DistanceToTriangle (3d/collisions.cpp:214-217). */
double or_distance_to_triangle(const double pt[3], const double p0[3], const double p1[3], const double p2[3])
{
    double c[3], d[3];
    closest_on_triangle(pt, p0, p1, p2, c);
    for (int a = 0; a < 3; ++a) d[a] = c[a] - pt[a];
    return len3(d);
}

/* TriangleMesh::IsInside (3d/triangle_mesh.cpp:120-163): the winding sum of atan2(det, k) over the triangles
 * (half solid angles), inside when |sum| >= 2 pi - 0.001, with abs on the double (its meaning on MSVC, the
 * reference's platform). */
int or_mesh_is_inside(const double* V, const int64_t* T, size_t nt, const double pt[3])
{
    const double PI_ = 3.14159265358979323846;
    double ret = 0;
    for (size_t i = 0; i < nt; ++i) {
        double A[3], B[3], C[3];
        for (int d = 0; d < 3; ++d) {
            A[d] = V[3 * T[4 * i] + d] - pt[d];
            B[d] = V[3 * T[4 * i + 1] + d] - pt[d];
            C[d] = V[3 * T[4 * i + 2] + d] - pt[d];
        }
        double omega = A[0] * B[1] * C[2];
        omega += B[0] * C[1] * A[2];
        omega += C[0] * A[1] * B[2];
        omega -= C[0] * B[1] * A[2];
        omega -= B[0] * A[1] * C[2];
        omega -= A[0] * C[1] * B[2];
        const double na = len3(A), nb = len3(B), nc = len3(C);
        double k = na * nb * nc;
        k += nc * ((A[0] * B[0] + A[1] * B[1]) + A[2] * B[2]);
        k += na * ((B[0] * C[0] + B[1] * C[1]) + B[2] * C[2]);
        k += nb * ((C[0] * A[0] + C[1] * A[1]) + C[2] * A[2]);
        ret += atan2(omega, k);
    }
    return fabs(ret) >= 2.0 * PI_ - 0.001;
}

static int clampi(int v, int maxv, int minv) { return v < minv ? minv : (v > maxv ? maxv : v); }

/* Mesh2SDF::Build (3d/mesh_2_sdf.cpp:14-82): ComputeExactBandDistanceField with bandwidth 1 (the fill value
 * max(h) * (nx + ny + nz); per triangle, the nodes of its index box -- vertex coordinates times 1 / h_x on every
 * axis, truncated, widened by the band and clamped -- take min(distance to the triangle)), then ComputeSigns. */
void or_mesh_to_sdf(const double* V, size_t nv, const int64_t* T, size_t nt, const int n[3], const double origin[3],
                    const double h[3], double* sdf)
{
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    double hmax = h[2];
    if (h[0] >= h[1] && h[0] >= h[2]) hmax = h[0]; else if (h[1] >= h[0] && h[1] >= h[2]) hmax = h[1];
    const double fill = hmax * (double)((size_t)n[0] + (size_t)n[1] + (size_t)n[2]);
    for (size_t c = 0; c < nc; ++c) sdf[c] = fill;
    if (nv == 0) return;
    const int band = 1;
    const double inv = 1.0 / h[0];
    for (size_t t = 0; t < nt; ++t) {
        const double* p = V + 3 * T[4 * t];
        const double* q = V + 3 * T[4 * t + 1];
        const double* r = V + 3 * T[4 * t + 2];
        double f[3][3];
        for (int d = 0; d < 3; ++d) { f[0][d] = p[d] * inv; f[1][d] = q[d] * inv; f[2][d] = r[d] * inv; }
        int lo[3], hi[3];
        for (int d = 0; d < 3; ++d) {
            lo[d] = clampi((int)fmin(f[0][d], fmin(f[1][d], f[2][d])) - band, n[d] - 1, 0);
            hi[d] = clampi((int)fmax(f[0][d], fmax(f[1][d], f[2][d])) + band + 1, n[d] - 1, 0);
        }
        for (int k = lo[2]; k <= hi[2]; ++k)
            for (int j = lo[1]; j <= hi[1]; ++j)
                for (int i = lo[0]; i <= hi[0]; ++i) {
                    double pt[3];
                    grid_pos(origin, h, i, j, k, pt);
                    const double dist = or_distance_to_triangle(pt, p, q, r);
                    size_t c = (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k);
                    if (dist < sdf[c]) sdf[c] = dist;
                }
    }
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                double pt[3];
                grid_pos(origin, h, i, j, k, pt);
                if (or_mesh_is_inside(V, T, nt, pt)) {
                    size_t c = (size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k);
                    sdf[c] = sdf[c] * -1.0;
                }
            }
}

/* PICSimulator::InitializeParticles (pic_simulator.cpp:521-548): the cells (i, j, k) of the velocity grid whose
 * GridIndexToPosition (its origin, the domain origin, + h * index) has a fluid-SDF sample < 0 receive
 * particlesPerBlock particles in [position, position + h).  Writes 1 / 0 per cell. */
void or_seed_cells(const or_sim* s, uint8_t* mask)
{
    for (int k = 0; k < s->n.z; ++k)
        for (int j = 0; j < s->n.y; ++j)
            for (int i = 0; i < s->n.x; ++i) {
                double pt[3];
                grid_pos(s->d.origin, s->h, i, j, k, pt);
                mask[ix3(s->n, i, j, k)] = sample3(s->sdf, s->n, s->sdf_origin, s->h, pt) < 0 ? 1 : 0;
            }
}

void or_set_sdf(or_sim* s, const double* sdf) { memcpy(s->sdf, sdf, cnt3(s->n) * sizeof(double)); }

/* ---------------------------------------------------------------- position-dependent external forces */

static double vlen(double x, double y, double z) { return sqrt(x * x + y * y + z * z); } /* Vector3::GetLength */

/* PointField::Sample (forces/point_field.cpp:16-19, GetDistance :46-49, GetDirection :51-56). */
static void point_sample(const or_force* f, const double p[3], double out[3])
{
    const double len = vlen(p[0] - f->origin[0], p[1] - f->origin[1], p[2] - f->origin[2]);
    const double dist = len >= 1.0 ? len : 1.0;
    double e[3] = {f->origin[0] - p[0], f->origin[1] - p[1], f->origin[2] - p[2]};
    const double el = vlen(e[0], e[1], e[2]); /* Normalize = Divide(length) */
    for (int a = 0; a < 3; ++a) e[a] /= el;
    const double sc = f->strength * (1.0 / dist);
    for (int a = 0; a < 3; ++a) out[a] = sc * e[a];
}

/* Collisions::RotatePointAroundAxis (3d/collisions.cpp:219-237): rotation of p about the line through
 * (a, b, c) with direction (u, v, w), the closed form of the rotation matrix about an arbitrary axis. */
static void rotate_about_axis(const double o[3], const double axis[3], const double p[3], double cA, double sA,
                              double out[3])
{
    const double al = vlen(axis[0], axis[1], axis[2]); /* GetNormalized */
    const double u = axis[0] / al, v = axis[1] / al, w = axis[2] / al;
    const double x = p[0], y = p[1], z = p[2];
    const double a = o[0], b = o[1], c = o[2];
    out[0] = (a * (v * v + w * w) - u * (b * v + c * w - u * x - v * y - w * z)) * (1 - cA) + x * cA +
             ((-1.0 * c) * v + b * w - w * y + v * z) * sA;
    out[1] = (b * (u * u + w * w) - v * (a * u + c * w - u * x - v * y - w * z)) * (1 - cA) + y * cA +
             (c * u - a * w + w * x - u * z) * sA;
    out[2] = (c * (u * u + v * v) - w * (a * u + b * v - u * x - v * y - w * z)) * (1 - cA) + z * cA +
             ((-1.0 * b) * u + a * v - v * x + u * y) * sA;
}

/* SwirlField::Sample (forces/swirlf_field.cpp:16-23) with Collisions::DistanceToAxis (3d/collisions.cpp:239-246),
 * which takes the axis direction as a second point on the axis. */
static void swirl_sample(const or_force* f, const double p[3], double out[3])
{
    const double* o = f->origin;
    const double* ax = f->axis;
    const double d0 = vlen(o[0] - ax[0], o[1] - ax[1], o[2] - ax[2]); /* DistanceToPoint(axisDirection, axisOrigin) */
    double dir[3], vv[3], cl[3];
    for (int a = 0; a < 3; ++a) dir[a] = (ax[a] - o[a]) / d0;
    for (int a = 0; a < 3; ++a) vv[a] = p[a] - o[a];
    const double t = vv[0] * dir[0] + vv[1] * dir[1] + vv[2] * dir[2];
    for (int a = 0; a < 3; ++a) cl[a] = o[a] + t * dir[a];
    double dist = vlen(p[0] - cl[0], p[1] - cl[1], p[2] - cl[2]);
    dist = dist >= 1.0 ? dist : 1.0;
    double r[3], fd[3];
    rotate_about_axis(o, ax, p, f->cos_a, f->sin_a, r);
    for (int a = 0; a < 3; ++a) fd[a] = p[a] - r[a];
    const double fl = vlen(fd[0], fd[1], fd[2]);
    for (int a = 0; a < 3; ++a) fd[a] = fd[a] / fl;
    const double sc = f->strength * (1 / (dist * dist));
    for (int a = 0; a < 3; ++a) out[a] = sc * fd[a];
}

/* VolumeField::Sample (forces/volume_field.cpp:20-58): trilinear closest-point vector, force along its negation
 * with strength / max(|vector|, 1)^2. */
static void volume_sample(const or_force* f, const double p[3], double out[3])
{
    int id[3], ip[3];
    double fr[3];
    for (int a = 0; a < 3; ++a) {
        barycentric((p[a] - f->o[a]) / f->h[a], f->n[a] - 1, &id[a], &fr[a]);
        ip[a] = id[a] + 1 < f->n[a] - 1 ? id[a] + 1 : f->n[a] - 1;
    }
    double sv[3];
    for (int c = 0; c < 3; ++c) {
#define FV(i, j, k) f->field[3 * ((size_t)(i) + (size_t)f->n[0] * ((size_t)(j) + (size_t)f->n[1] * (size_t)(k))) + c]
        const double q[8] = {FV(id[0], id[1], id[2]), FV(ip[0], id[1], id[2]), FV(id[0], ip[1], id[2]),
                             FV(ip[0], ip[1], id[2]), FV(id[0], id[1], ip[2]), FV(ip[0], id[1], ip[2]),
                             FV(id[0], ip[1], ip[2]), FV(ip[0], ip[1], ip[2])};
#undef FV
        sv[c] = or_trilerp(q, fr[0], fr[1], fr[2]);
    }
    const double len = vlen(sv[0], sv[1], sv[2]);
    double fd[3];
    for (int a = 0; a < 3; ++a) fd[a] = (sv[a] / len) * (-1.0);
    const double dist = len >= 1.0 ? len : 1.0;
    const double sc = f->strength * (1 / (dist * dist));
    for (int a = 0; a < 3; ++a) out[a] = sc * fd[a];
}

static void force_sample(const or_force* f, const double p[3], double out[3])
{
    if (f->kind == OR_FORCE_POINT) point_sample(f, p, out);
    else if (f->kind == OR_FORCE_SWIRL) swirl_sample(f, p, out);
    else volume_sample(f, p, out);
}

/* ExternalForce::ApplyExternalForce (forces/external_force.cpp:3-29) of every position-dependent force, in the
 * order added: each face += dt * the force's component at the face position (FaceCenteredGrid3D::GetXPos, ...). */
static void apply_position_forces(or_sim* s, double dt)
{
    const double* org[3] = {s->xo, s->yo, s->zo};
    double* arr[3] = {s->u, s->v, s->w};
    const dim3i dims[3] = {s->du, s->dv, s->dw};
    for (int f = 0; f < s->nforces; ++f)
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < dims[c].z; ++k)
                for (int j = 0; j < dims[c].y; ++j)
                    for (int i = 0; i < dims[c].x; ++i) {
                        const double p[3] = {org[c][0] + s->h[0] * (double)i, org[c][1] + s->h[1] * (double)j,
                                             org[c][2] + s->h[2] * (double)k};
                        double fv[3];
                        force_sample(&s->forces[f], p, fv);
                        arr[c][ix3(dims[c], i, j, k)] += dt * fv[c];
                    }
}

static or_force* new_force(or_sim* s, int kind, double strength)
{
    if (s->nforces >= OR_MAX_FORCES) return NULL;
    or_force* f = &s->forces[s->nforces++];
    memset(f, 0, sizeof(*f));
    f->kind = kind;
    f->strength = strength;
    return f;
}

/* PointField(origin, strength, strengthFallOff) (forces/point_field.cpp:3-5); the fall-off is unused by Sample. */
int or_add_point_field(or_sim* s, const double origin[3], double strength)
{
    or_force* f = new_force(s, OR_FORCE_POINT, strength);
    if (!f) return -1;
    for (int a = 0; a < 3; ++a) f->origin[a] = origin[a];
    return 0;
}

/* SwirlField(origin, axisDirection, strength, strengthFallOff) (forces/swirlf_field.cpp:5-8): the axis is stored
 * normalised; the rotation angle of Sample is 0.0001 degrees (PI from common/math_utils.hpp:11). */
int or_add_swirl_field(or_sim* s, const double origin[3], const double axis[3], double strength)
{
    or_force* f = new_force(s, OR_FORCE_SWIRL, strength);
    if (!f) return -1;
    const double al = vlen(axis[0], axis[1], axis[2]);
    for (int a = 0; a < 3; ++a) {
        f->origin[a] = origin[a];
        f->axis[a] = axis[a] / al;
    }
    const double ang = 0.0001 * 3.14159265358979323846 / 180;
    f->cos_a = cos(ang);
    f->sin_a = sin(ang);
    return 0;
}

/* The closest-point vectors of VolumeField::Initialize (forces/volume_field.cpp:72-89): at every node of the
 * field's grid, closest point on the first nearest triangle (Collisions::ClosestTriangleIdx, 3d/collisions.cpp:
 * 249-265, strict < from 1.7976931348623157e30) minus the node position.  (Initialize also builds a Mesh2SDF
 * that Sample never reads.) */
void or_volume_field_vectors(const double* V, const int64_t* T, size_t nt, const int n[3], const double o[3],
                             const double h[3], double* out)
{
    for (int k = 0; k < n[2]; ++k)
        for (int j = 0; j < n[1]; ++j)
            for (int i = 0; i < n[0]; ++i) {
                const double gp[3] = {o[0] + i * h[0], o[1] + j * h[1], o[2] + k * h[2]};
                double best = 1.7976931348623157E+30;
                size_t idx = 0;
                for (size_t t = 0; t < nt; ++t) {
                    const double d = or_distance_to_triangle(gp, V + 3 * T[4 * t], V + 3 * T[4 * t + 1], V + 3 * T[4 * t + 2]);
                    if (d < best) {
                        best = d;
                        idx = t;
                    }
                }
                double cp[3] = {0, 0, 0};
                if (nt) closest_on_triangle(gp, V + 3 * T[4 * idx], V + 3 * T[4 * idx + 1], V + 3 * T[4 * idx + 2], cp);
                double* dst = out + 3 * ((size_t)i + (size_t)n[0] * ((size_t)j + (size_t)n[1] * (size_t)k));
                for (int a = 0; a < 3; ++a) dst[a] = cp[a] - gp[a];
            }
}

/* VolumeField(mesh, resolution, domain, strength) (forces/volume_field.cpp:5-13): spacing = domain size /
 * resolution, origin = domain origin. */
int or_add_volume_field(or_sim* s, const double* V, const int64_t* T, size_t nt, const int n[3],
                        const double domain_origin[3], const double domain_size[3], double strength)
{
    if (n[0] < 1 || n[1] < 1 || n[2] < 1) return -1;
    or_force* f = new_force(s, OR_FORCE_VOLUME, strength);
    if (!f) return -1;
    for (int a = 0; a < 3; ++a) {
        f->n[a] = n[a];
        f->o[a] = domain_origin[a];
        f->h[a] = domain_size[a] / n[a];
    }
    f->field = (double*)xcalloc(3 * (size_t)n[0] * n[1] * n[2], sizeof(double));
    or_volume_field_vectors(V, T, nt, f->n, f->o, f->h, f->field);
    return 0;
}

/* ---------------------------------------------------------------- colliders */

/* ScalarGrid3D::Sample of the collider SDF (ColliderCollection::_sdf: the n nodes at the velocity grid's origin,
 * the domain origin, spacing h; pic_simulator.cpp:24). */
static double collider_sample(const or_sim* s, const double pos[3])
{
    return sample3(s->csdf, s->n, s->d.origin, s->h, pos);
}

/* TriangleMeshCollider(gridSize, gridOrigin, gridSpacing, mesh) (3d/triangle_mesh_collider.cpp:4-8): Mesh2SDF of
 * the mesh on the collider's own node grid.  N holds the mesh normals (3 doubles each), indexed by the triangles'
 * normal ids as ResolveCollision reads them.  Returns 0 on success. */
int or_add_mesh_collider(or_sim* s, const double* V, size_t nv, const int64_t* T, size_t nt, const double* N,
                         size_t nn, const int n[3], const double origin[3], const double h[3])
{
    if (s->ncolliders >= OR_MAX_COLLIDERS || n[0] < 1 || n[1] < 1 || n[2] < 1) return -1;
    for (size_t t = 0; t < nt; ++t)
        if (T[4 * t + 3] < 0 || (size_t)T[4 * t + 3] >= nn) return -1;
    or_collider* c = &s->colliders[s->ncolliders++];
    memset(c, 0, sizeof(*c));
    for (int a = 0; a < 3; ++a) {
        c->n[a] = n[a];
        c->o[a] = origin[a];
        c->h[a] = h[a];
    }
    c->sdf = (double*)xcalloc((size_t)n[0] * n[1] * n[2], sizeof(double));
    or_mesh_to_sdf(V, nv, T, nt, n, origin, h, c->sdf);
    c->V = (double*)xcalloc(3 * nv, sizeof(double));
    c->T = (int64_t*)xcalloc(4 * nt, sizeof(int64_t));
    c->N = (double*)xcalloc(3 * nn, sizeof(double));
    if (nv) memcpy(c->V, V, 3 * nv * sizeof(double));
    if (nt) memcpy(c->T, T, 4 * nt * sizeof(int64_t));
    if (nn) memcpy(c->N, N, 3 * nn * sizeof(double));
    c->nv = nv;
    c->nt = nt;
    c->nn = nn;
    return 0;
}

/* BoundryConditionSolver::BuildCollider -> ColliderCollection::BuildSdf (3d/collider_collection.cpp:33-50): every
 * node takes the smallest GetClosestDistanceAt (TriangleMeshCollider: its SDF sampled at the node) over the
 * colliders, from 1.7976931348623157e30. */
void or_build_collider(or_sim* s)
{
    for (int k = 0; k < s->n.z; ++k)
        for (int j = 0; j < s->n.y; ++j)
            for (int i = 0; i < s->n.x; ++i) {
                const double p[3] = {s->d.origin[0] + i * s->h[0], s->d.origin[1] + j * s->h[1],
                                     s->d.origin[2] + k * s->h[2]};
                double m = OR_MAX_DISTANCE;
                for (int c = 0; c < s->ncolliders; ++c) {
                    const or_collider* cl = &s->colliders[c];
                    const dim3i d = {cl->n[0], cl->n[1], cl->n[2]};
                    const double v = sample3(cl->sdf, d, cl->o, cl->h, p);
                    if (v < m) m = v;
                }
                s->csdf[ix3(s->n, i, j, k)] = m;
            }
}

void or_get_collider_sdf(const or_sim* s, double* out) { memcpy(out, s->csdf, cnt3(s->n) * sizeof(double)); }

/* PICSimulator::ExtrapolateIntoCollider (pic_simulator.cpp:497-519): fluid SDF nodes where the collider SDF
 * (sampled at the node) is < 0 take ceil(maxCfl) rounds of ExtrapolateToRegion. */
static void extrapolate_into_collider(or_sim* s)
{
    const size_t nc = cnt3(s->n);
    uint8_t* valid = (uint8_t*)xcalloc(nc, 1);
    double* prev = (double*)xcalloc(nc, sizeof(double));
    for (int i = 0; i < s->n.x; ++i)
        for (int j = 0; j < s->n.y; ++j)
            for (int k = 0; k < s->n.z; ++k) {
                const double p[3] = {s->sdf_origin[0] + i * s->h[0], s->sdf_origin[1] + j * s->h[1],
                                     s->sdf_origin[2] + k * s->h[2]};
                valid[ix3(s->n, i, j, k)] = collider_sample(s, p) < 0 ? 0 : 1;
            }
    memcpy(prev, s->sdf, nc * sizeof(double));
    extrapolate_to_region(prev, valid, s->n, (size_t)ceil(s->d.max_cfl), s->sdf);
    free(valid);
    free(prev);
}

/* BlockedBoundryConditionSolver::FractionInsideSdf (fluid_solvers/blocked_boundry_condition_solver.cpp:304-322). */
static double fraction_inside(double phi0, double phi1)
{
    if (phi0 < 0.0 && phi1 < 0.0) return 1;
    if (phi0 < 0.0 && !(phi1 < 0.0)) return phi0 / (phi0 - phi1);
    if (!(phi0 < 0.0) && phi1 < 0.0) return phi1 / (phi1 - phi0);
    return 0;
}

/* ScalarGrid3D::Gradient (3d/scalar_grid3d.cpp:67-90) of the collider SDF: the interpolation weights of the eight
 * surrounding nodes times their clamped central differences. */
static void collider_gradient(const or_sim* s, const double pos[3], double g[3])
{
    idx8 id;
    double w[8];
    coords_weights(s->n, s->d.origin, s->h, pos, &id, w);
    g[0] = g[1] = g[2] = 0.0;
    for (int t = 0; t < 8; ++t) {
        const int i = id.i[t], j = id.j[t], k = id.k[t];
        const double left = s->csdf[ix3(s->n, i > 0 ? i - 1 : i, j, k)];
        const double right = s->csdf[ix3(s->n, i + 1 < s->n.x ? i + 1 : i, j, k)];
        const double down = s->csdf[ix3(s->n, i, j > 0 ? j - 1 : j, k)];
        const double up = s->csdf[ix3(s->n, i, j + 1 < s->n.y ? j + 1 : j, k)];
        const double back = s->csdf[ix3(s->n, i, j, k > 0 ? k - 1 : k)];
        const double front = s->csdf[ix3(s->n, i, j, k + 1 < s->n.z ? k + 1 : k)];
        const double wt = w[t] * 0.5;
        g[0] += (wt * (right - left)) / s->h[0];
        g[1] += (wt * (up - down)) / s->h[1];
        g[2] += (wt * (front - back)) / s->h[2];
    }
}

/* ConstrainVelocity with colliders (fluid_solvers/blocked_boundry_condition_solver.cpp:18-291): faces whose
 * half-cell segment lies inside the collider SDF (FractionInsideSdf of the samples h/2 either side, 1 - clamped
 * fraction not > 0) are zeroed and refilled by ceil(maxCfl) rounds of ExtrapolateToRegion; faces inside the
 * collider then take the tangential part of the sampled velocity (ApplyFriction with coefficient 0: v - n (v . n),
 * n the normalised SDF gradient; 0 where the gradient vanishes); the wall layers are zeroed; and faces between a
 * cell whose collider-SDF node is < 0 and one whose node is not are zeroed. */
static void constrain_with_colliders(or_sim* s)
{
    double* arr[3] = {s->u, s->v, s->w};
    const dim3i dims[3] = {s->du, s->dv, s->dw};
    const double* org[3] = {s->xo, s->yo, s->zo};
    const size_t depth = (size_t)ceil(s->d.max_cfl);
    uint8_t* mk[3];
    double* tmp[3];
    for (int c = 0; c < 3; ++c) {
        const size_t nf = cnt3(dims[c]);
        mk[c] = (uint8_t*)xcalloc(nf, 1);
        tmp[c] = (double*)xcalloc(nf, sizeof(double));
        for (int k = 0; k < dims[c].z; ++k)
            for (int j = 0; j < dims[c].y; ++j)
                for (int i = 0; i < dims[c].x; ++i) {
                    const double p[3] = {org[c][0] + s->h[0] * (double)i, org[c][1] + s->h[1] * (double)j,
                                         org[c][2] + s->h[2] * (double)k};
                    double p0[3] = {p[0], p[1], p[2]}, p1[3] = {p[0], p[1], p[2]};
                    const double off[3] = {c == 0 ? 0.5 * s->h[0] : 0.0, c == 1 ? 0.5 * s->h[1] : 0.0,
                                           c == 2 ? 0.5 * s->h[2] : 0.0};
                    for (int a = 0; a < 3; ++a) {
                        p0[a] = p[a] - off[a];
                        p1[a] = p[a] + off[a];
                    }
                    double frac = fraction_inside(collider_sample(s, p0), collider_sample(s, p1));
                    frac = 1 - clampd(frac, 1.0, 0.0);
                    const size_t f = ix3(dims[c], i, j, k);
                    if (frac > 0.0) {
                        mk[c][f] = 1;
                    } else {
                        arr[c][f] = 0.0;
                        mk[c][f] = 0;
                    }
                }
    }
    for (int c = 0; c < 3; ++c) {
        const size_t nf = cnt3(dims[c]);
        double* prev = (double*)xcalloc(nf, sizeof(double));
        memcpy(prev, arr[c], nf * sizeof(double));
        extrapolate_to_region(prev, mk[c], dims[c], depth, arr[c]);
        free(prev);
    }
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < dims[c].z; ++k)
            for (int j = 0; j < dims[c].y; ++j)
                for (int i = 0; i < dims[c].x; ++i) {
                    const double p[3] = {org[c][0] + s->h[0] * (double)i, org[c][1] + s->h[1] * (double)j,
                                         org[c][2] + s->h[2] * (double)k};
                    const size_t f = ix3(dims[c], i, j, k);
                    if (collider_sample(s, p) < 0) {
                        double vel[3], g[3];
                        sample_velocity(s, s->u, s->v, s->w, s->xo, s->yo, s->zo, p, vel);
                        collider_gradient(s, p, g);
                        const double gl = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
                        if (gl * gl > 0.0) {
                            const double gv = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
                            const double nrm[3] = {g[0] / gv, g[1] / gv, g[2] / gv};
                            const double vr[3] = {vel[0] - 0.0, vel[1] - 0.0, vel[2] - 0.0};
                            const double d = vr[0] * nrm[0] + vr[1] * nrm[1] + vr[2] * nrm[2];
                            tmp[c][f] = (vr[c] - nrm[c] * d) + 0.0;
                        } else {
                            tmp[c][f] = 0.0;
                        }
                    } else {
                        tmp[c][f] = arr[c][f];
                    }
                }
    for (int c = 0; c < 3; ++c) {
        memcpy(arr[c], tmp[c], cnt3(dims[c]) * sizeof(double));
        free(tmp[c]);
        free(mk[c]);
    }
    /* the wall layers (:198-244) */
    for (int k = 0; k < s->du.z; ++k)
        for (int j = 0; j < s->du.y; ++j) {
            s->u[ix3(s->du, 0, j, k)] = 0;
            s->u[ix3(s->du, s->du.x - 1, j, k)] = 0;
        }
    for (int k = 0; k < s->dv.z; ++k)
        for (int i = 0; i < s->dv.x; ++i) {
            s->v[ix3(s->dv, i, 0, k)] = 0;
            s->v[ix3(s->dv, i, s->dv.y - 1, k)] = 0;
        }
    for (int j = 0; j < s->dw.y; ++j)
        for (int i = 0; i < s->dw.x; ++i) {
            s->w[ix3(s->dw, i, j, 0)] = 0;
            s->w[ix3(s->dw, i, j, s->dw.z - 1)] = 0;
        }
    /* faces between BOUNDRY and FLUID cells of the node-value markers (:246-290) */
    const dim3i n = s->n;
    for (int k = 0; k < n.z; ++k)
        for (int j = 0; j < n.y; ++j)
            for (int i = 0; i < n.x; ++i) {
#define CB(a, b, c) (s->csdf[ix3(n, (a), (b), (c))] < 0)
                if (!CB(i, j, k)) continue;
                if (i > 0 && !CB(i - 1, j, k)) s->u[ix3(s->du, i, j, k)] = 0;
                if (i < n.x - 1 && !CB(i + 1, j, k)) s->u[ix3(s->du, i + 1, j, k)] = 0;
                if (j > 0 && !CB(i, j - 1, k)) s->v[ix3(s->dv, i, j, k)] = 0;
                if (j < n.y - 1 && !CB(i, j + 1, k)) s->v[ix3(s->dv, i, j + 1, k)] = 0;
                if (k > 0 && !CB(i, j, k - 1)) s->w[ix3(s->dw, i, j, k)] = 0;
                if (k < n.z - 1 && !CB(i, j, k + 1)) s->w[ix3(s->dw, i, j, k + 1)] = 0;
#undef CB
            }
}

/* TriangleMeshCollider::ResolveCollision (3d/triangle_mesh_collider.cpp:65-100) with radius and restitution 0 and
 * friction 0: the closest point on the first nearest triangle to `prev` (Collisions::ClosestTriangleIdx,
 * ClossestPointOnTriangle) becomes the position; when the position was inside the mesh
 * (TriangleMesh::IsInside), the velocity's normal part toward the triangle's normal is scaled by -0. */
static void resolve_collision(const or_collider* c, const double prev[3], double* pos, double* vel)
{
    double best = OR_MAX_DISTANCE;
    size_t idx = 0;
    for (size_t t = 0; t < c->nt; ++t) {
        const double d = or_distance_to_triangle(prev, c->V + 3 * c->T[4 * t], c->V + 3 * c->T[4 * t + 1],
                                                 c->V + 3 * c->T[4 * t + 2]);
        if (d < best) {
            best = d;
            idx = t;
        }
    }
    double cp[3];
    closest_on_triangle(prev, c->V + 3 * c->T[4 * idx], c->V + 3 * c->T[4 * idx + 1], c->V + 3 * c->T[4 * idx + 2], cp);
    const double* nrm = c->N + 3 * c->T[4 * idx + 3];
    if (or_mesh_is_inside(c->V, c->T, c->nt, pos)) {
        const double rv[3] = {vel[0] - 0.0, vel[1] - 0.0, vel[2] - 0.0};
        const double nd = nrm[0] * rv[0] + nrm[1] * rv[1] + nrm[2] * rv[2];
        double rn[3] = {nd * nrm[0], nd * nrm[1], nd * nrm[2]};
        double rt[3] = {rv[0] - rn[0], rv[1] - rn[1], rv[2] - rn[2]};
        if (nd < 0.0) {
            const double drn[3] = {(-0.0 - 1.0) * rn[0], (-0.0 - 1.0) * rn[1], (-0.0 - 1.0) * rn[2]};
            for (int a = 0; a < 3; ++a) rn[a] *= -0.0;
            if (rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] > 0.0) {
                const double lt = sqrt(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2]);
                const double ln = sqrt(drn[0] * drn[0] + drn[1] * drn[1] + drn[2] * drn[2]);
                const double q = 1.0 - 0.0 * ln / lt;
                const double fs = (q < 0.0) ? 0.0 : q; /* std::max(q, 0.0) */
                for (int a = 0; a < 3; ++a) rt[a] *= fs;
            }
        }
        for (int a = 0; a < 3; ++a) vel[a] = (rn[a] + rt[a]) + 0.0;
    }
    for (int a = 0; a < 3; ++a) pos[a] = cp[a];
}
