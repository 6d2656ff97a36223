// fe_internal.cuh -- shared device state and helpers of the B200 substep kernels.
//
// Layout in HBM (one scene):
//   particles  FP32 struct of arrays px,py,pz,vx,vy,vz (+ c0..c8 for APIC), kept sorted by cell key,
//              double-buffered for the sort's gather; pid = original particle index.
//   MAC grid   FP32 u (nx+1)ny nz, v nx(ny+1)nz, w nx ny(nz+1), x-fastest as the reference's Array3;
//              ping-pong copies for extrapolation, FP32 FLIP snapshot, u8 face markers, FP32 P2G
//              accumulators (numerator, weight).
//   cells      u8 marks (AIR 0 / FLUID 1), FP64 pressure (warm start kept between substeps),
//              FP64 right-hand side, FP32 CG vectors (r, w, s twice; p, x) and the compacted FLUID list.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "../../include/fluide_b200.h"
#include "fe_keys.h"

namespace fe {

constexpr int kMaxRefineDefault = 12;

// NVTX range for the lifetime of the object: each public call (a step, a substep and its phases, a batch step,
// the autotuner, checkpoints, particle transfers, surface extraction) shows as a named range in an NVTX-aware
// profiler; without one attached the push and pop do nothing.
struct TraceRange {
    explicit TraceRange(const char* name) { nvtxRangePushA(name); }
    ~TraceRange() { nvtxRangePop(); }
    TraceRange(const TraceRange&) = delete;
    TraceRange& operator=(const TraceRange&) = delete;
};
constexpr int kMaxCgBlocks = 4096;  // solver blocks one scene can be given (sizes its partial-sum buffer)
// Grid-barrier words of one solver: [0] arrivals of the current launch, [2] statistics counter (kept across
// launches), [32] blocks that have left the current launch (its own 128-byte line).
constexpr int kCgBarWords = 64;
// Grid-reduction totals: 3 rotating slots x 4 groups x 4 sums, every total on its own 128-byte line (16 doubles).
constexpr int kCgTotalsGroups = 4;
constexpr int kCgTotalsStride = 16;
constexpr int kCgTotalsDoubles = 3 * kCgTotalsGroups * 4 * kCgTotalsStride;
// Doubles of one solver's partial buffer for up to max_blocks blocks: the reduction totals, then the per-block
// FLUID counts of the solver's setup.
constexpr size_t cg_partial_doubles(size_t max_blocks) { return kCgTotalsDoubles + max_blocks; }
constexpr int kBatchMaxScenes = 64;
// Entries of a scene's device ring of solve statistics (one per pressure solve; solves wrap around it).
constexpr unsigned kStatsRingEntries = 1u << 16;

struct GridDims {
    int nx, ny, nz;
    int tnx, tny, tnz;      // tiles per axis
    uint32_t key_space;     // tiles * 512
};

// Everything a kernel needs, passed by value.
struct SceneView {
    GridDims g;
    int solver;
    uint64_t np;
    // geometry (FP64 master copies; FP32 views for the particle kernels)
    double h[3], inv_h[3], origin[3], size[3];
    float hf[3], inv_hf[3], originf[3], sizef[3];
    float xo[3], yo[3], zo[3];        // velocity-grid data origins (origin-independent, see fe_scene.cu)
    float rxo[3], ryo[3], rzo[3];     // FLIP residual-grid data origins
    float blend;
    double gravity[3];
    double max_cfl;
    int extrap_depth, rk_substeps;
    // particles
    float *px, *py, *pz, *vx, *vy, *vz;
    float* c[9];
    uint32_t* pid;
    // the sort's scratch: key per particle; rank = a particle's atomic slot in its cell, then (after the sort) the
    // sorted order, slot -> particle; perm = the runs in arbitrary order; cell counts and starts per cell key
    uint32_t *key, *rank, *perm, *cell_count, *cell_start;
    // grid
    float *u, *v, *w;
    float *u2, *v2, *w2;
    float *su, *sv, *sw;
    float *nu, *nv, *nw;   // P2G numerators
    float *du, *dv, *dw;   // P2G weights
    uint8_t *mu, *mv, *mw; // P2G face markers
    uint8_t *mu2, *mv2, *mw2; // extrapolation validity ping-pong
    uint8_t* marks;
    double *p, *b;
    double* pprev;         // the pressure of the substep before the last (time-extrapolated warm start), or null
    // marking tables (per axis, FP64)
    double* q_pos[3];      // sdf node coordinate of each index
    int* q_b0[3];          // hash bucket of the node
    int* q_b1[3];          // the second bucket chosen by the half test
    uint8_t* q_exact[3];   // 1 if the cell-centre sample hits the node exactly
    int* q_i0[3];          // GetBarycentric index of the cell-centre sample
    double* q_f[3];        // GetBarycentric fraction of the cell-centre sample
    double sdf_origin[3];
    double radius, band, bucket;   // r = 1.2 max(h)/sqrt(2), 2r, hash spacing 2r
    uint32_t* crit_list;   // cells whose mark needs the full trilinear sample
    uint32_t* crit_count;
    uint8_t* crit_flag;
    int any_inexact;
};

// Error bookkeeping (fe_scene.cu).
fe_status set_error(fe_status st, const char* fmt, ...);
fe_status cuda_check(cudaError_t e, const char* what);
void count_launch(uint64_t n = 1);

#define FE_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return ::fe::cuda_check(e_, #call);        \
    } while (0)

__host__ __device__ __forceinline__ size_t idx3(int i, int j, int k, int sx, int sy)
{
    return (size_t)i + (size_t)sx * ((size_t)j + (size_t)sy * (size_t)k);
}

// GetBarycentric with iLow = 0 (common/math_utils.hpp:48-73), FP32.
__device__ __forceinline__ void bary(float x, int iHigh, int& i, float& f)
{
    float s = floorf(x);
    int ii = (int)s;  // cvt.rzi saturates, so huge or NaN inputs stay finite
    if (iHigh == 0 || ii < 0 || !(x == x)) {
        ii = 0;
        f = 0.f;
    } else if (ii > iHigh - 1) {
        ii = iHigh - 1;
        f = 1.f;
    } else {
        f = x - s;
    }
    i = ii;
}

// Clamped trilinear sample of a face array (FaceCenteredGrid3D::SampleArray,
// grid_systems/face_centered_grid3d.cpp:339-371), FP32, Lerp order of common/math_utils.hpp:30-46.
__device__ __forceinline__ float lerpf_ref(float a, float b, float f) { return (1.f - f) * a + f * b; }

struct Stencil {
    int i, j, k, ip, jp, kp;
    float fx, fy, fz;
};

__device__ __forceinline__ Stencil stencil(float x, float y, float z, const float o[3], const float ih[3], int sx,
                                           int sy, int sz)
{
    Stencil s;
    bary((x - o[0]) * ih[0], sx - 1, s.i, s.fx);
    bary((y - o[1]) * ih[1], sy - 1, s.j, s.fy);
    bary((z - o[2]) * ih[2], sz - 1, s.k, s.fz);
    s.ip = min(s.i + 1, sx - 1);
    s.jp = min(s.j + 1, sy - 1);
    s.kp = min(s.k + 1, sz - 1);
    return s;
}

__device__ __forceinline__ float sample_st(const float* __restrict__ a, const Stencil& s, int sx, int sy)
{
    float c000 = __ldg(a + idx3(s.i, s.j, s.k, sx, sy)), c100 = __ldg(a + idx3(s.ip, s.j, s.k, sx, sy));
    float c010 = __ldg(a + idx3(s.i, s.jp, s.k, sx, sy)), c110 = __ldg(a + idx3(s.ip, s.jp, s.k, sx, sy));
    float c001 = __ldg(a + idx3(s.i, s.j, s.kp, sx, sy)), c101 = __ldg(a + idx3(s.ip, s.j, s.kp, sx, sy));
    float c011 = __ldg(a + idx3(s.i, s.jp, s.kp, sx, sy)), c111 = __ldg(a + idx3(s.ip, s.jp, s.kp, sx, sy));
    float b0 = lerpf_ref(lerpf_ref(c000, c100, s.fx), lerpf_ref(c010, c110, s.fx), s.fy);
    float b1 = lerpf_ref(lerpf_ref(c001, c101, s.fx), lerpf_ref(c011, c111, s.fx), s.fy);
    return lerpf_ref(b0, b1, s.fz);
}

__device__ __forceinline__ float sample_face(const float* __restrict__ a, float x, float y, float z, const float o[3],
                                             const float ih[3], int sx, int sy, int sz)
{
    Stencil s = stencil(x, y, z, o, ih, sx, sy, sz);
    return sample_st(a, s, sx, sy);
}

// 3D launch over the three face arrays: blocks of 32 x 8 threads tile (i, j); blockIdx.z runs over the z
// layers of u (nz), then v (nz), then w (nz + 1), so every thread gets its face coordinates without integer
// division and a warp's 32 threads read consecutive faces.
constexpr int kTileX = 32, kTileY = 8;
struct FaceCoord {
    int c, i, j, k, sx, sy, sz;
    size_t f;
};
__host__ __device__ inline dim3 face_grid(int nx, int ny, int nz)
{
    return dim3((unsigned)((nx + 1 + kTileX - 1) / kTileX), (unsigned)((ny + 1 + kTileY - 1) / kTileY),
                (unsigned)(3 * nz + 1));
}
__host__ __device__ inline dim3 cell_grid(int nx, int ny, int nz)
{
    return dim3((unsigned)((nx + kTileX - 1) / kTileX), (unsigned)((ny + kTileY - 1) / kTileY), (unsigned)nz);
}
// Block coordinates of a 3D launch: the hardware's, or those of a block of a flat multi-scene launch (block
// `local` of its scene's share, x fastest over the scene's own grid of gx x gy blocks).
struct Blk3 {
    unsigned x, y, z;
};
__device__ __forceinline__ Blk3 hw_blk3() { return {blockIdx.x, blockIdx.y, blockIdx.z}; }
__device__ __forceinline__ Blk3 flat_blk3(uint32_t local, dim3 grid)
{
    return {local % grid.x, (local / grid.x) % grid.y, local / (grid.x * grid.y)};
}
__device__ __forceinline__ bool face_coord(int nx, int ny, int nz, Blk3 b, FaceCoord& fc)
{
    const int z = (int)b.z;
    if (z < nz) { fc.c = 0; fc.k = z; fc.sx = nx + 1; fc.sy = ny; fc.sz = nz; }
    else if (z < 2 * nz) { fc.c = 1; fc.k = z - nz; fc.sx = nx; fc.sy = ny + 1; fc.sz = nz; }
    else { fc.c = 2; fc.k = z - 2 * nz; fc.sx = nx; fc.sy = ny; fc.sz = nz + 1; }
    fc.i = (int)(b.x * kTileX + threadIdx.x);
    fc.j = (int)(b.y * kTileY + threadIdx.y);
    if (fc.i >= fc.sx || fc.j >= fc.sy) return false;
    fc.f = (size_t)fc.i + (size_t)fc.sx * ((size_t)fc.j + (size_t)fc.sy * (size_t)fc.k);
    return true;
}
__device__ __forceinline__ bool face_coord(int nx, int ny, int nz, FaceCoord& fc)
{
    return face_coord(nx, ny, nz, hw_blk3(), fc);
}

// Column launch over the three face arrays: blocks of 32 x 8 threads tile (i, j) as above, and each thread marches
// kColumn consecutive faces along z, so values along z are carried from one face to the next and the index advances
// by one plane per step; grid.z runs over the z chunks of u (nz faces), then v (nz), then w (nz + 1).
constexpr int kColumn = 8;
__host__ __device__ inline dim3 column_grid(int nx, int ny, int nz)
{
    return dim3((unsigned)((nx + 1 + kTileX - 1) / kTileX), (unsigned)((ny + 1 + kTileY - 1) / kTileY),
                (unsigned)(2 * ((nz + kColumn - 1) / kColumn) + (nz + 1 + kColumn - 1) / kColumn));
}
struct FaceColumn {
    int c, i, j, k0, k1, sx, sy, sz;
};
__device__ __forceinline__ bool column_coord(int nx, int ny, int nz, Blk3 b, FaceColumn& fc)
{
    const int cz = (nz + kColumn - 1) / kColumn;
    int z = (int)b.z;
    if (z < cz) { fc.c = 0; fc.sx = nx + 1; fc.sy = ny; fc.sz = nz; }
    else if (z < 2 * cz) { fc.c = 1; z -= cz; fc.sx = nx; fc.sy = ny + 1; fc.sz = nz; }
    else { fc.c = 2; z -= 2 * cz; fc.sx = nx; fc.sy = ny; fc.sz = nz + 1; }
    fc.i = (int)(b.x * kTileX + threadIdx.x);
    fc.j = (int)(b.y * kTileY + threadIdx.y);
    fc.k0 = z * kColumn;
    fc.k1 = min(fc.k0 + kColumn, fc.sz);
    return fc.i < fc.sx && fc.j < fc.sy && fc.k0 < fc.sz;
}

// Viscosity (fe_diffuse.cu): buffers of the implicit diffusion solve, allocated when a scene's viscosity is > 0.
// Face arrays are the three components concatenated (u | v | w) like the velocity buffers.
struct DiffWork {
    unsigned long long* node_dist;  // nx*ny*nz: bits of the smallest particle distance per SDF node (all ones: none)
    uint8_t* mark;                  // faces: FE_CELL_FLUID / FE_CELL_AIR (BackwardEulerDiffusionSolver::_fluidMarkers)
    unsigned long long* list;       // FLUID faces: (face << 9) | (wall << 8) | (component << 6) | FLUID-neighbour mask
    double* x[2];                   // faces: Jacobi iterates (only FLUID entries are used)
    double* snap;                   // faces: an earlier iterate, for the exact early exit
    unsigned* count;                // [0]: list length
    int* its;                       // [4]: Jacobi iterations of the last solve per component, relaxation passes run
    int* tab_i0;                    // [component][axis][index]: GetBarycentric index of each face coordinate
    double* tab_f;                  // same layout: GetBarycentric fraction
    int tab_stride;                 // max(nx, ny, nz) + 1 entries per (component, axis)
    int blocks;                     // blocks of the persistent Jacobi kernel (all co-resident)
};

// Kernel launchers (one per .cu file).
cudaError_t launch_sort(const SceneView& v, cudaStream_t st, void* scan_tmp, size_t scan_tmp_bytes);
size_t sort_scan_tmp_bytes(uint32_t n);
// Exclusive prefix sum of n counts into out[0..n] (out[n] = total); tmp holds sort_scan_tmp_bytes(n).
cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t n, uint32_t* out, void* tmp, size_t tmp_bytes,
                                  cudaStream_t st);
cudaError_t launch_gather(const SceneView& v, const SceneView& dst, cudaStream_t st);
cudaError_t launch_p2g(const SceneView& v, cudaStream_t st);
cudaError_t launch_mark(const SceneView& v, cudaStream_t st);
cudaError_t launch_fluid_sdf(const SceneView& v, double* out, cudaStream_t st);
// Distance bits of the band SDF per node by a particle scatter, then the diffusion face markers (fe_mark.cu).
cudaError_t launch_face_fluid_marks(const SceneView& v, const DiffWork& d, cudaStream_t st);
// The band SDF of v's particles at every node (BuildSignedDistanceField's values, FP64) by the same scatter;
// node_scratch holds nx*ny*nz u64 (fe_mark.cu).
cudaError_t launch_node_sdf(const SceneView& v, unsigned long long* node_scratch, double* sdf, cudaStream_t st);
cudaError_t launch_pre(const SceneView& v, double dt, cudaStream_t st);
cudaError_t launch_post(const SceneView& v, cudaStream_t st);
cudaError_t launch_rhs(const SceneView& v, cudaStream_t st);
cudaError_t launch_apply(const SceneView& v, cudaStream_t st);
cudaError_t launch_g2p(const SceneView& v, double dt, bool do_g2p, bool do_move, cudaStream_t st);
cudaError_t launch_cfl(const SceneView& v, double dt, double* out_max, cudaStream_t st);
cudaError_t launch_divergence(const SceneView& v, double* out, cudaStream_t st);
cudaError_t launch_scatter_out(const SceneView& v, float* pos, float* vel, float* C, cudaStream_t st);

// CG solver (fe_cg.cu).
struct CgWork {
    float *r0, *r1, *w0, *w1, *s0, *s1, *pv, *x;  // FP32 vectors of the multigrid solver (8 x cells)
    // the plain CG's view of the same memory: (r, w, s, p) of a cell in one float4, ping-pong, and its correction
    // (a 9th run of cells after the 8 above)
    float4 *rws0, *rws1;
    float* xcg;
    uint32_t* list;         // compacted FLUID cells: (cell << 6) | in-domain neighbour mask
    double* partial;        // [0, kCgTotalsDoubles) reduction totals, then one FLUID count per block
    unsigned* bar;          // kCgBarWords barrier words
    int* err;
    fe_step_stats* stats;   // device ring of solve statistics
    unsigned stats_cap;     // entries of that ring (solves wrap around it)
    int blocks, threads;
    int cluster;            // thread-block cluster size of the persistent solver launch (0 / 1: no clusters)
};
// Persistent-solver launch shape: `threads` per block (256, 512 or 1024), as many blocks per SM as make 1024
// threads, all co-resident.
cudaError_t cg_prepare(CgWork& w, int device, int threads = 1024, int cluster = 1);
// Bounded-wait limits of the pressure solvers' grid barrier on the current device (spin_limit 0: the default;
// extra_arrivals > 0 makes every barrier wait for blocks that do not exist, so each wait runs out).
cudaError_t set_solver_barrier_limits(unsigned long long spin_limit, unsigned extra_arrivals);

// Multigrid hierarchy of the MG-preconditioned solver (fe_mg_body.cuh): level 0 is the scene grid, whose
// vectors are the solver's own (CgWork); level l >= 1 halves every axis of level l-1 (rounding up) until
// the largest axis is <= 8, and that last level is solved by one block.
constexpr int kMaxMgLevels = 12;
// FE_PRESSURE_AUTO picks the multigrid solver from this many grid cells on.  Measured on B200 over whole
// 240-substep dam-break runs (ms per solve, plain / multigrid): 24^3 0.36 / 0.39, 32^3 0.46 / 0.39, 40^3 0.55 /
// 0.52, 48^3 0.64 / 0.63, 64^3 0.85 / 0.67, 96^3 - / 1.27, 128^3 3.24 / 1.91; at 256^3 the multigrid one wins by
// 8x (the plain CG streams its vectors from HBM about 1,000 times per solve).
constexpr size_t kMgAutoCells = (size_t)1 << 15;
struct MgLevel {
    int nx, ny, nz;
    float ih2[3];      // 1 / h_l^2 per axis, h_l = 2^l h
    uint8_t* mask;     // l >= 1: 1 where some child cell holds fluid
    float* r;          // l >= 1: restricted residual
    float* z;          // l >= 1: correction
    float* t;          // l >= 1: scratch: the level's residual going down, its pre-smoothed correction going up
};
struct MgWork {
    int levels;        // levels in use (0 or 1: no hierarchy, the plain CG solves)
    int block_from;    // levels >= block_from (at most 4096 cells each) are processed by one block alone
    MgLevel lv[kMaxMgLevels];
};
// Level dimensions for an nx x ny x nz grid with spacing h (host); returns the number of levels (>= 2), or 1
// when the grid is too small for a hierarchy.
int mg_plan(int nx, int ny, int nz, const double h[3], MgLevel* out);
// First level (>= 1) from which every level has at most block_cells cells and is processed by one block without
// grid barriers.
int mg_block_from(const MgLevel* lv, int levels, int block_cells);

// One scene of a multi-scene pressure solve (fe_cg.cu k_multi_cg): the scene's grid view and solver
// buffers, its solver settings and the block range [block_start, block_start + block_count) that solves it.
struct MultiCgScene {
    SceneView view;
    CgWork work;
    MgWork mg;                     // the scene's multigrid hierarchy (used when use_mg)
    int use_mg;                    // solve this scene with the multigrid-preconditioned body
    double rel_tol, inner_tol;
    int max_it, max_refine;
    int block_start, block_count;  // this scene's block range, re-split before every solve
    int last_its, last_fluid;      // the previous solve's inner iterations and FLUID cells (-1 / 0: none yet)
    double weight0;                // expected solve work before any solve has run
};
cudaError_t multi_cg_capacity(int device, int* max_blocks, int* threads);
// Re-splits total_blocks among the S scenes in proportion to their last solve's work, then solves them.
cudaError_t launch_multi_cg(MultiCgScene* scenes, int S, int total_blocks, cudaStream_t st);
cudaError_t launch_cg(const SceneView& v, const CgWork& w, double rel_tol, double inner_tol, int max_it, int max_refine,
                      cudaStream_t st);
cudaError_t launch_mgcg(const SceneView& v, const CgWork& w, const MgWork& mg, double rel_tol, double inner_tol,
                        int max_it, int max_refine, cudaStream_t st);

// Surface extraction (fe_surface.cu): items = the node grid's cubes, then its XY, YZ and XZ cap squares (two faces
// each); counts per item, then the mesh from the scanned counts.
size_t mc_items(int nx, int ny, int nz);
cudaError_t launch_mc_count(const SceneView& v, const double* sdf, uint8_t* cfg, uint32_t* nvert, uint32_t* ntri,
                            cudaStream_t st);
cudaError_t launch_mc_emit(const SceneView& v, const double* sdf, const uint8_t* cfg, const uint32_t* vbase,
                           const uint32_t* tbase, double* V, double* N, int64_t* T, cudaStream_t st);

// Scene initialisation from meshes (fe_mesh.cu).  Mesh2SDF onto a node grid (scratch: one u64 per node); the
// InitializeParticles and VolumeEmitter counts per node (particles per block where the rule holds); spawning the
// counted particles at node position + h * U[0,1]^3 into v's arrays from index `base` on.
cudaError_t launch_mesh_to_sdf(const double* V, uint64_t nv, const int64_t* T, uint64_t nt, const int n[3],
                               const double o[3], const double h[3], unsigned long long* scratch, double* sdf,
                               cudaStream_t st);
cudaError_t launch_seed_count(const double* fluid_sdf, const int n[3], const double sdf_o[3], const double h[3],
                              const double vel_o[3], uint32_t ppb, uint32_t* count, cudaStream_t st);
cudaError_t launch_emit_count(const double* emitter_sdf, const int en[3], const double* fluid_sdf, int fnx, int fny,
                              uint32_t ppb, uint32_t* count, cudaStream_t st, const double* collider_sdf = nullptr);
cudaError_t launch_spawn(const int n[3], const double o[3], const double h[3], const uint32_t* count,
                         const uint32_t* offset, uint64_t seed, const SceneView& v, uint64_t base, const float vel[3],
                         cudaStream_t st);

// VolumeField's closest-point vectors on a node grid (fe_mesh.cu): 3 doubles per node, x-fastest.
cudaError_t launch_volume_vectors(const double* V, uint64_t nv, const int64_t* T, uint64_t nt, const int n[3],
                                  const double o[3], const double h[3], double* out, cudaStream_t st);

// Solid colliders (fe_collide.cu).  A TriangleMeshCollider: its Mesh2SDF on its own node grid and its mesh.
constexpr int kMaxColliders = 8;
struct ColliderDev {
    int n[3];
    double o[3], h[3];
    const double* sdf;
    const double* V;   // 3 per vertex
    const int64_t* T;  // 4 per triangle: vertex ids, normal id into N
    const double* N;   // 3 per normal
    uint64_t nv, nt;
};
struct CollideSet {
    int count;
    ColliderDev c[kMaxColliders];
};
enum : uint8_t { kFaceInside = 1, kFaceZero = 2 };
// Per-scene collider buffers: the collider SDF and its fixed classification, and per-substep scratch.
struct CollideWork {
    double* csdf;            // n^3 nodes at the domain origin
    uint8_t* node_valid;     // n^3: ExtrapolateIntoCollider's valid nodes
    uint8_t* cell_boundry;   // n^3: BuildMarkers' BOUNDRY cells (when not FLUID)
    uint8_t* face_open;      // faces (u | v | w): not blocked by the collider
    uint8_t* face_cls;       // faces: kFaceInside / kFaceZero
    uint8_t* vscratch;       // 2 x faces: extrapolation validity ping-pong
    uint8_t* node_vscratch;  // 2 x n^3
    float *ftmp0, *ftmp1;    // faces: extrapolation copies
    float* fric;             // faces: projected velocities of the listed faces (one per fin_list entry)
    uint32_t* face_cnt;      // 2: list lengths found on the device
    uint32_t* blk_list;      // the faces that are not open (fixed with the collider set)
    uint32_t* fin_list;      // the faces ConstrainVelocity rewrites, bit 31: projected onto the tangent plane
    double* fin_nrm;         // 3 per fin_list entry: the unit collider normal at a projected face
    uint32_t n_blk, n_fin;
    double *sdf_a, *sdf_b;   // n^3: fluid SDF ping-pong
    uint32_t* label;         // n^3: FLUID component labels (union-find)
    uint8_t* open_comp;      // n^3 (by root): the component has an AIR neighbour
    double* comp_sum;        // n^3 (by root): right-hand-side sum of the component
    uint32_t* comp_cnt;      // n^3 (by root): its cells
    // collision response (sized by the particle capacity)
    float* start;            // 3 per slot: position before the move
    float* startv;           // 3 per slot: velocity before the move (after the grid-to-particle transfer)
    float* spos;             // 3 per original index: start positions of the flagged particles
    uint32_t* flag;          // cap + 1
    uint32_t* offs;          // cap + 1
    uint32_t* list;          // cap
    double *cp, *nrm;        // 3 per (listed particle, collider)
    uint8_t* ins;            // 1 per (listed particle, collider)
    uint32_t* slot_of;       // kMaxColliders
    uint32_t *act, *act_offs, *act_list;  // (listed particle, collider) entries that reflect, compacted in order
    void* act_tmp;
    size_t act_tmp_bytes;
    void* scan_tmp;
    size_t scan_tmp_bytes;
};
// The move parameters of k_g2p (MoveParticles' RK2 sub-steps and domain clamp) and its final velocity buffers.
struct CollideMove {
    float dt_sub;
    int nsub;
    float lo[3], hi[3];
    const float *u, *v, *w;
};
cudaError_t launch_collider_setup(const SceneView& v, const CollideSet& cs, CollideWork& w, cudaStream_t st);
// count_only: the list lengths into face_cnt; otherwise fill lists sized by those counts.
cudaError_t launch_collider_face_lists(const SceneView& v, CollideWork& w, bool count_only, cudaStream_t st);
cudaError_t launch_collider_bc(const SceneView& v, const CollideWork& w, float* const buf[3], cudaStream_t st);
// Enclosed FLUID components (no AIR neighbour: a pure-Neumann block) lose the mean of their right-hand side.
cudaError_t launch_collider_project_rhs(const SceneView& v, const CollideWork& w, int* err, cudaStream_t st);
cudaError_t launch_collider_marks(const SceneView& v, const CollideWork& w, unsigned long long* node_scratch,
                                  double** fluid_sdf, cudaStream_t st);
cudaError_t launch_collider_keep_start(const SceneView& v, const CollideWork& w, cudaStream_t st);
cudaError_t launch_collider_resolve(const SceneView& v, const CollideSet& cs, const CollideWork& w,
                                    const CollideMove& g, cudaStream_t st);
cudaError_t launch_surface_with_colliders(const double* fluid, const double* csdf, size_t n, double* out,
                                          cudaStream_t st);
cudaError_t launch_add_gravity(const SceneView& v, float* const buf[3], double dt, cudaStream_t st);
cudaError_t launch_extrap_faces(const SceneView& v, float* const src[3], float* const dst_final[3],
                                float* const other[3], const uint8_t* const valid0[3], uint8_t* vscratch, int depth,
                                cudaStream_t st);

// Position-dependent external forces (fe_forces.cu), applied after the pre-solve pass (which adds gravity).
constexpr int kMaxForces = 8;
struct ForceDev {
    int kind;                   // FE_FORCE_POINT / SWIRL / VOLUME
    int n[3];                   // volume: node grid
    double origin[3], axis[3];  // point / swirl origin; swirl axis (normalised)
    double strength;
    double cos_a, sin_a;        // swirl: cos / sin of RotatePointAroundAxis's angle, evaluated on the host
    double o[3], h[3];          // volume: grid origin and spacing
    const double* field;        // volume: closest-point vectors, 3 per node
};
struct ForceList {
    int count;
    ForceDev f[kMaxForces];
};
// u, vv, ww: the velocity buffers the pre-solve pass wrote; faces at the velocity grid's data origins.
cudaError_t launch_forces(const SceneView& v, const ForceList& fl, float* u, float* vv, float* ww, double dt,
                          cudaStream_t st, bool zero_walls = true);

// Viscosity (fe_diffuse.cu): ComputeDiffusion on the velocity buffers u, vv, ww (face markers, FLUID-face list,
// persistent Jacobi solve, wall layers zeroed).  Uses the scene's solver barrier and error words (CgWork).
cudaError_t launch_diffuse(const SceneView& v, const DiffWork& d, const CgWork& w, float* u, float* vv, float* ww,
                           double dt, double viscosity, cudaStream_t st);
cudaError_t diffuse_prepare(DiffWork& d, int device);

// ------------------------------------------------------------------ flat multi-scene launches (batches)
//
// A batch substep launches every transfer and grid pass ONCE for all its scenes: the launch's blocks are a flat
// work list of (scene, block) entries, the scenes' blocks back to back in membership order.  Each kind of launch
// (block shape) has its own prefix of per-scene block counts; a block finds its scene from that prefix (one ballot
// over at most 64 scene ends) and runs the same body as the one-scene kernel with its block index inside the
// scene.  Per-scene data (the two particle buffer sets, scratch, dt-dependent constants) lives in a device table
// built on the host when the membership or dt changes.
enum BatchKind {
    kBkClear,      // 256 threads: the substep's accumulator / count / marker clears
    kBkPart,       // 256 threads, one particle each: marking, transfer and move
    kBkGather,     // 256 threads, 4 particles each: the gather, keys, placement and ranks
    kBkScan,       // 1024 threads, 4096 counts each
    kBkScanSums,   // 1024 threads, one block per scene
    kBkBigcell,    // 1024 threads, striding over the scene's long runs
    kBkP2g,        // one 8^3 cell tile each
    kBkNormalize,  // 256 threads, one face each
    kBkFaces,      // 32 x 8 threads, face_grid
    kBkCells,      // 32 x 8 threads, cell_grid
    kBkFixup,      // 128 threads: marks needing the full SDF sample (scenes with inexact cell-centre samples)
    kBkCount
};

// MoveParticles' and the transfer's launch constants (fe_g2p.cu).
struct G2PArgs {
    float dt_sub;
    int nsub;
    int same_origins;        // the FLIP residual grid's data origins equal the velocity grid's (domain origin 0)
    float dom_lo[3], dom_hi[3];
    const float *u, *v, *w;  // final velocity buffers
};
G2PArgs g2p_args(const SceneView& v, double dt);

// The marking pass's launch constants (fe_mark.cu): band^2, the largest squared distance whose square root is below r,
// the window around r in which an inexact cell-centre sample is recomputed, 1 / bucket spacing, and whether every
// axis' node window around a particle holds at most two nodes (r / h + 1e-6 < 1 on every axis).
struct MarkConst {
    double R2, rin2, crit_eps, inv_bucket;
    int two;
};

constexpr int kBatchClearRanges = 8;
struct BatchScene {
    SceneView src;               // particle buffer set the substep starts from (the sort's input)
    SceneView dst;               // the other set: the gather's output, used by every later pass
    uint32_t* scan_sums;         // the sort's scan scratch (block sums, then the long-run counter)
    uint32_t* long_count;
    uint32_t scan_blocks;
    // byte ranges cleared at the start of the substep: cell counts, P2G numerators / weights / face markers, marks
    uint8_t* clr_ptr[kBatchClearRanges];
    uint64_t clr_bytes[kBatchClearRanges];
    uint32_t clr_val[kBatchClearRanges];
    int nclr;
    float gdt[3];                // dt * gravity, FP32
    MarkConst mark;              // marking constants (fe_mark.cu)
    G2PArgs g2p;
};
struct BatchPlan {
    int count;
    uint32_t start[kBkCount][kBatchMaxScenes + 1];  // per kind: first block of each scene, then the total
    BatchScene sc[kBatchMaxScenes];
};
// Host-side totals of a plan (grid sizes of the flat launches).
struct BatchLaunch {
    const BatchPlan* plan;       // device copy
    uint32_t total[kBkCount];
    int max_depth;               // largest extrapolation depth among the scenes
};

// The block's scene and its block index inside that scene's share of a kind's launch.  Every lane of the block's
// first warps must be active (called at kernel entry).
__device__ __forceinline__ int batch_scene_of(const BatchPlan* __restrict__ plan, int kind, uint32_t& local)
{
    const uint32_t b = blockIdx.x;
    const int lane = (int)((threadIdx.x + threadIdx.y * blockDim.x) & 31);
    const int S = plan->count;
    const uint32_t* st = plan->start[kind];
    const uint32_t e0 = lane < S ? st[lane + 1] : 0xffffffffu;
    const uint32_t e1 = lane + 32 < S ? st[lane + 33] : 0xffffffffu;
    const int s = __popc(__ballot_sync(0xffffffffu, b >= e0)) + __popc(__ballot_sync(0xffffffffu, b >= e1));
    local = b - st[s];
    return s;
}

// Copies a scene's view into the block's shared memory (register-heavy kernels read their scene's fields from there
// instead of keeping loaded copies in registers); ends with a block barrier.
__device__ __forceinline__ void stage_view(SceneView& dst, const SceneView& src)
{
    static_assert(sizeof(SceneView) % 8 == 0, "SceneView is copied in 8-byte words");
    const int t = (int)(threadIdx.x + threadIdx.y * blockDim.x), n = (int)(blockDim.x * blockDim.y);
    for (int i = t; i < (int)(sizeof(SceneView) / 8); i += n)
        reinterpret_cast<unsigned long long*>(&dst)[i] = reinterpret_cast<const unsigned long long*>(&src)[i];
    __syncthreads();
}

// Per-kind block count of one scene (host; the same grids the one-scene launchers use); the sort's kinds come from
// fe_sort.cu.
uint32_t batch_blocks(const SceneView& v, int kind);
uint32_t sort_batch_blocks(const SceneView& v, int kind);
// launch_mark's constants (fe_mark.cu).
MarkConst mark_constants(const SceneView& v);
// Flat launches of one batch substep's passes (fe_sort.cu, fe_p2g.cu, fe_mark.cu, fe_grid.cu, fe_g2p.cu).
cudaError_t launch_multi_clear(const BatchLaunch& L, cudaStream_t st);
cudaError_t launch_multi_sort(const BatchLaunch& L, cudaStream_t st);    // keys, scan, placement, ranks, gather
cudaError_t launch_multi_p2g(const BatchLaunch& L, cudaStream_t st);     // splat + normalise
cudaError_t launch_multi_mark(const BatchLaunch& L, cudaStream_t st);
cudaError_t launch_multi_pre(const BatchLaunch& L, cudaStream_t st);     // extrapolation + walls + gravity
cudaError_t launch_multi_rhs(const BatchLaunch& L, cudaStream_t st);
cudaError_t launch_multi_apply(const BatchLaunch& L, cudaStream_t st);
cudaError_t launch_multi_post(const BatchLaunch& L, cudaStream_t st);    // extrapolation + walls
cudaError_t launch_multi_g2p(const BatchLaunch& L, cudaStream_t st);     // transfer + move

}  // namespace fe
