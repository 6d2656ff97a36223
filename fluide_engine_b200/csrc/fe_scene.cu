// fe_scene.cu -- scene lifecycle, substep orchestration (CUDA graphs) and the C ABI of fluide_b200.h.
//
// One substep is the reference's PICSimulator::OnAdvanceTimeStep (pic_simulator.cpp:111-154) with no
// emitters, no colliders and zero viscosity:
//   SORT -> P2G -> MARK -> PRE (extrapolate, BC, gravity, BC) -> PRESSURE (rhs, CG, apply) ->
//   POST (extrapolate, BC) -> G2P + MOVE
// For a fixed dt a substep is captured once as three CUDA graphs (pre-solve, solve, post-solve) per
// particle-buffer parity (the sort gathers into the other buffer set, so substeps alternate between two
// graph sets) and replayed; the phase split lets the profiled entry point time the CG kernel with events.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <tuple>
#include <vector>

#include "fe_internal.cuh"
#include "fe_seed.h"

namespace fe {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};
static thread_local bool g_capturing = false;
static thread_local uint64_t g_capture_launches = 0;

fe_status set_error(fe_status st, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return st;
}

fe_status cuda_check(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return FE_OK;
    if (e == cudaErrorMemoryAllocation) return set_error(FE_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return set_error(FE_ERR_NO_DEVICE, "%s: %s", what, cudaGetErrorString(e));
    return set_error(FE_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void count_launch(uint64_t n)
{
    if (g_capturing) g_capture_launches += n;
    else g_launches += n;
}

namespace {

__global__ void k_set_particles(SceneView v, const float* pos, const float* vel, const float* C, uint64_t n)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    v.px[i] = pos[3 * i];
    v.py[i] = pos[3 * i + 1];
    v.pz[i] = pos[3 * i + 2];
    v.vx[i] = vel ? vel[3 * i] : 0.f;
    v.vy[i] = vel ? vel[3 * i + 1] : 0.f;
    v.vz[i] = vel ? vel[3 * i + 2] : 0.f;
    v.pid[i] = (uint32_t)i;
    if (v.solver == FE_SOLVER_APIC)
        for (int a = 0; a < 9; ++a) v.c[a][i] = C ? C[9 * i + a] : 0.f;
}

__global__ void k_sorted_keys(SceneView v, uint32_t* out)
{
    uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= v.np) return;
    out[s] = v.key[v.rank[s]];
}

__global__ void k_perm_ids(const uint32_t* perm, const uint32_t* pid_old, uint32_t* out, uint64_t n)
{
    uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= n) return;
    out[s] = pid_old[perm[s]];
}

struct ParticleSet {
    float *px, *py, *pz, *vx, *vy, *vz;
    float* c[9];
    uint32_t* pid;
};

}  // namespace
}  // namespace fe

using namespace fe;

struct fe_scene {
    fe_scene_desc desc;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    SceneView base;            // grid + scratch pointers; particle pointers filled per parity
    ParticleSet set[2];
    int parity = 0;            // which particle set holds the particles
    int grid_cur = 0;          // 0: velocity in buffer A (u,v,w), 1: in buffer B (u2,v2,w2)
    uint64_t cap = 0;
    bool have_particles = false;
    std::vector<void*> allocs;         // grid-lifetime allocations
    std::vector<void*> particle_allocs;
    void* scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    CgWork cg{};
    MgWork mg{};                       // multigrid levels (levels >= 2) once the multigrid solver was wanted
    bool use_mg = false;               // solve with the multigrid-preconditioned CG (if the grid has a hierarchy)
    double* pprev_buf = nullptr;       // pressure of the substep before the last (time-extrapolated warm start)
    int mg_block_cells = 2048;         // multigrid levels of at most this many cells run in one block
    DiffWork diff{};                   // viscosity buffers (allocated once the viscosity is > 0)
    bool diff_ready = false;
    // Surface extraction (fe_surface.cu), allocated on first use: node distances and SDF values, per-item case
    // bytes, counts and their scans, scan scratch, and the last mesh (grown on demand).
    struct {
        unsigned long long* node = nullptr;
        double* sdf = nullptr;
        uint8_t* cfg = nullptr;
        uint32_t *nvert = nullptr, *ntri = nullptr, *vbase = nullptr, *tbase = nullptr;
        void* tmp = nullptr;
        size_t tmp_bytes = 0, items = 0;
        double *V = nullptr, *N = nullptr;
        int64_t* T = nullptr;
        uint64_t cap_v = 0, cap_t = 0, nv = 0, nt = 0;
        bool built = false;
        std::vector<void*> mesh_allocs;
    } surf;
    // true once a substep's sort has run since the particles were set: the other particle set then holds the
    // positions at the start of the last substep, from which the reference's Fluid3::sdf was built
    bool prev_valid = false;
    // Fluid3::sdf holds the mesh SDF of fe_scene_init_from_mesh (in surf.sdf) until the next substep
    bool mesh_sdf = false;
    // BuildCollider has run (at the start of some substep): until then the collider SDF is its initial 0
    // (ColliderCollection's ScalarGrid3D, 3d/collider_collection.cpp:5-8), which no emitter node passes (> 0)
    bool collider_built = false;
    // VolumeEmitters (fe_mesh.cu): each emits at the start of every substep
    struct Emitter {
        int n[3];
        double o[3], h[3];
        double* sdf = nullptr;
        uint32_t* count = nullptr;
        uint32_t* offset = nullptr;
        void* tmp = nullptr;
        size_t tmp_bytes = 0;
        uint32_t ppb = 8;
        float vel[3] = {0, 0, 0};
        uint64_t seed = 0, calls = 0;
        std::vector<void*> allocs;
    };
    std::vector<Emitter> emitters;
    // position-dependent external forces (fe_forces.cu), applied after the pre-solve pass
    std::vector<std::vector<void*>> force_allocs;
    ForceList forces{};
    // solid colliders (fe_collide.cu): the meshes and their SDFs, the collider SDF with its classification, scratch
    CollideSet colliders{};
    std::vector<std::vector<void*>> collider_allocs;
    CollideWork cw{};
    std::vector<void*> cw_grid_allocs, cw_particle_allocs, cw_face_allocs;
    uint64_t cw_cap = 0;
    int cw_ncoll = 0;
    double* collider_fluid_sdf = nullptr;  // Fluid3::sdf of the last collider substep (after ExtrapolateIntoCollider)
    uint64_t epoch = 0;                // bumped when the substep's kernel sequence changes (batches re-capture)
    double* d_scalar = nullptr;        // CFL / divergence result
    float* staging = nullptr;          // interleaved particle staging (9 floats per particle)
    uint32_t* staging_u32 = nullptr;
    fe_step_stats* stats_ring = nullptr;
    // graphs per particle parity, valid for graph_dt: the three phases (profiled steps, batches) and the whole
    // substep as one graph (plain steps)
    cudaGraphExec_t graph[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
    uint64_t graph_kernels[2][3] = {{0, 0, 0}, {0, 0, 0}};
    cudaGraphExec_t whole[2] = {nullptr, nullptr};
    uint64_t whole_kernels[2] = {0, 0};
    double graph_dt = -1.0;
    bool graphs_disabled = false;
    bool last_substep_empty = false;  // the last run_substep had no particles (an emitter scene before emission)
    std::mutex mu;
};

namespace {

SceneView view_of(const fe_scene* s, int parity)
{
    SceneView v = s->base;
    const ParticleSet& p = s->set[parity];
    v.px = p.px; v.py = p.py; v.pz = p.pz;
    v.vx = p.vx; v.vy = p.vy; v.vz = p.vz;
    for (int a = 0; a < 9; ++a) v.c[a] = p.c[a];
    v.pid = p.pid;
    return v;
}

// Device memory of scenes and batches comes from one stream-ordered pool per device that keeps freed
// memory cached (release threshold: unlimited): creating and destroying scenes -- what a server does per job --
// then costs no driver allocation and no device-wide synchronisation once the pool has grown to the working
// set, unlike cudaMalloc / cudaFree (cudaFree waits for the whole device).  Allocations and frees are ordered
// on the stream they are issued on.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices] = {};

cudaError_t device_pool(int device, cudaMemPool_t* out)
{
    if (device < 0 || device >= kMaxPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pool[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        cudaError_t e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = ~0ull;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return e;
        }
        g_pool[device] = pool;
    }
    *out = g_pool[device];
    return cudaSuccess;
}

template <class T>
cudaError_t dalloc(std::vector<void*>& list, T** out, size_t count, int device, cudaStream_t st)
{
    cudaMemPool_t pool;
    cudaError_t e = device_pool(device, &pool);
    if (e != cudaSuccess) return e;
    void* p = nullptr;
    e = cudaMallocFromPoolAsync(&p, count * sizeof(T) + 16, pool, st);
    if (e != cudaSuccess) return e;
    list.push_back(p);
    *out = (T*)p;
    return cudaSuccess;
}

// Returns the allocations to the pool in `st`'s order (after the work already issued on it).
void free_list(std::vector<void*>& list, cudaStream_t st)
{
    for (void* p : list) cudaFreeAsync(p, st);
    list.clear();
}

void drop_graphs(fe_scene* s)
{
    for (int i = 0; i < 2; ++i) {
        for (int ph = 0; ph < 3; ++ph)
            if (s->graph[i][ph]) {
                cudaGraphExecDestroy(s->graph[i][ph]);
                s->graph[i][ph] = nullptr;
            }
        if (s->whole[i]) {
            cudaGraphExecDestroy(s->whole[i]);
            s->whole[i] = nullptr;
        }
    }
    s->graph_dt = -1.0;
}

// GetBarycentric (common/math_utils.hpp:48-73) in FP64 on the host.
void bary_host(double x, int iHigh, int* i, double* f)
{
    double sfl = std::floor(x);
    int ii = (int)sfl;
    if (iHigh == 0 || ii < 0) { ii = 0; *f = 0; }
    else if (ii > iHigh - 1) { ii = iHigh - 1; *f = 1; }
    else *f = x - sfl;
    *i = ii;
}

// Buffers of the viscosity solve (fe_diffuse.cu) and the GetBarycentric tables of the face centres of the copied
// velocity grid (data origins with the domain origin, grid_systems/face_centered_grid3d.cpp:11-17,303-316) in the
// fluid SDF grid (ScalarGrid3D::Sample, 3d/scalar_grid3d.cpp:33-65), computed in FP64 as the reference does.
fe_status alloc_diffusion(fe_scene* s)
{
    if (s->diff_ready) return FE_OK;
    const SceneView& v = s->base;
    for (int a = 0; a < 3; ++a)  // k_sdf_scatter keeps the candidate nodes of one axis in a 64-bit mask
        if (2.0 * v.band * v.inv_h[a] + 2.0 > 64.0)
            return set_error(FE_ERR_BAD_ARG, "cells too anisotropic for the viscosity solve (max(h) / h > 18)");
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    const size_t nf = (size_t)(n[0] + 1) * n[1] * n[2] + (size_t)n[0] * (n[1] + 1) * n[2] +
                      (size_t)n[0] * n[1] * (n[2] + 1);
    auto& L = s->allocs;
    const int dev = s->device;
    cudaStream_t st = s->own_stream;
    DiffWork d{};
    FE_CUDA(dalloc(L, &d.node_dist, nc, dev, st));
    FE_CUDA(dalloc(L, &d.mark, nf, dev, st));
    FE_CUDA(cudaMemsetAsync(d.mark, 0, nf, st));
    FE_CUDA(dalloc(L, &d.list, nf, dev, st));
    FE_CUDA(dalloc(L, &d.x[0], nf, dev, st));
    FE_CUDA(dalloc(L, &d.x[1], nf, dev, st));
    FE_CUDA(dalloc(L, &d.snap, nf, dev, st));
    FE_CUDA(dalloc(L, &d.count, 1, dev, st));
    FE_CUDA(cudaMemsetAsync(d.count, 0, sizeof(unsigned), st));
    FE_CUDA(dalloc(L, &d.its, 4, dev, st));
    FE_CUDA(cudaMemsetAsync(d.its, 0, 4 * sizeof(int), st));
    d.tab_stride = std::max(n[0], std::max(n[1], n[2])) + 1;
    std::vector<int> ti0((size_t)9 * d.tab_stride, 0);
    std::vector<double> tf((size_t)9 * d.tab_stride, 0.0);
    for (int c = 0; c < 3; ++c)
        for (int a = 0; a < 3; ++a) {
            const double org = v.origin[a] + v.h[a] * (a == c ? 0.0 : 0.5);  // CalculateDataOrigins
            const size_t base = (size_t)(3 * c + a) * d.tab_stride;
            for (int i = 0; i < n[a] + (a == c ? 1 : 0); ++i) {
                const double pos = org + v.h[a] * (double)i;                   // GetXPos / GetYPos / GetZPos
                bary_host((pos - v.sdf_origin[a]) / v.h[a], n[a] - 1, &ti0[base + i], &tf[base + i]);
            }
        }
    FE_CUDA(dalloc(L, &d.tab_i0, ti0.size(), dev, st));
    FE_CUDA(dalloc(L, &d.tab_f, tf.size(), dev, st));
    FE_CUDA(cudaMemcpyAsync(d.tab_i0, ti0.data(), ti0.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    FE_CUDA(cudaMemcpyAsync(d.tab_f, tf.data(), tf.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    FE_CUDA(diffuse_prepare(d, dev));
    FE_CUDA(cudaStreamSynchronize(st));  // host tables are freed on return; the buffers are ready for any stream
    s->diff = d;
    s->diff_ready = true;
    return FE_OK;
}

// Multigrid hierarchy of the scene's grid (levels 1 .. L-1, dense; level 0 is the grid itself), allocated once;
// grids too small for a hierarchy keep levels = 0 and solve with the plain CG.
fe_status ensure_mg(fe_scene* s)
{
    if (s->mg.levels >= 2) return FE_OK;
    SceneView& v = s->base;
    auto& L = s->allocs;
    const int dev = s->device;
    cudaStream_t st = s->own_stream;
    MgLevel lv[kMaxMgLevels];
    const int levels = mg_plan(v.g.nx, v.g.ny, v.g.nz, v.h, lv);
    if (levels < 2) return FE_OK;
    for (int l = 1; l < levels; ++l) {
        MgLevel& M = lv[l];
        const size_t cells = (size_t)M.nx * M.ny * M.nz;
        FE_CUDA(dalloc(L, &M.mask, cells, dev, st));
        FE_CUDA(dalloc(L, &M.r, cells, dev, st));
        FE_CUDA(dalloc(L, &M.z, cells, dev, st));
        FE_CUDA(dalloc(L, &M.t, cells, dev, st));
        FE_CUDA(cudaMemsetAsync(M.mask, 0, cells, st));
        FE_CUDA(cudaMemsetAsync(M.r, 0, cells * sizeof(float), st));
        FE_CUDA(cudaMemsetAsync(M.z, 0, cells * sizeof(float), st));
        FE_CUDA(cudaMemsetAsync(M.t, 0, cells * sizeof(float), st));
    }
    for (int l = 0; l < levels; ++l) s->mg.lv[l] = lv[l];
    s->mg.levels = levels;
    s->mg.block_from = mg_block_from(s->mg.lv, levels, s->mg_block_cells);
    return FE_OK;
}

fe_status alloc_grid(fe_scene* s)
{
    SceneView& v = s->base;
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nvv = (size_t)nx * (ny + 1) * nz, nww = (size_t)nx * ny * (nz + 1);
    const size_t nf = nu + nvv + nww;
    auto& L = s->allocs;
    const int dev = s->device;
    cudaStream_t st = s->own_stream;
    float *A, *B, *S, *N, *D;
    uint8_t *M, *M2;
    FE_CUDA(dalloc(L, &A, nf, dev, st));
    FE_CUDA(dalloc(L, &B, nf, dev, st));
    FE_CUDA(dalloc(L, &S, nf, dev, st));
    FE_CUDA(dalloc(L, &N, nf, dev, st));
    FE_CUDA(dalloc(L, &D, nf, dev, st));
    FE_CUDA(dalloc(L, &M, nf, dev, st));
    FE_CUDA(dalloc(L, &M2, 2 * nf, dev, st));
    v.u = A; v.v = A + nu; v.w = A + nu + nvv;
    v.u2 = B; v.v2 = B + nu; v.w2 = B + nu + nvv;
    v.su = S; v.sv = S + nu; v.sw = S + nu + nvv;
    v.nu = N; v.nv = N + nu; v.nw = N + nu + nvv;
    v.du = D; v.dv = D + nu; v.dw = D + nu + nvv;
    v.mu = M; v.mv = M + nu; v.mw = M + nu + nvv;
    v.mu2 = M2; v.mv2 = M2 + nu; v.mw2 = M2 + nu + nvv;
    FE_CUDA(cudaMemsetAsync(A, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(B, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(S, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(M, 0, nf, st));
    FE_CUDA(dalloc(L, &v.marks, nc, dev, st));
    FE_CUDA(cudaMemsetAsync(v.marks, 0, nc, st));
    FE_CUDA(dalloc(L, &v.p, nc, dev, st));
    FE_CUDA(cudaMemsetAsync(v.p, 0, nc * sizeof(double), st));
    FE_CUDA(dalloc(L, &v.b, nc, dev, st));
    FE_CUDA(cudaMemsetAsync(v.b, 0, nc * sizeof(double), st));
    // sort scratch over the key space
    FE_CUDA(dalloc(L, &v.cell_count, v.g.key_space, dev, st));
    FE_CUDA(dalloc(L, &v.cell_start, (size_t)v.g.key_space + 1, dev, st));
    FE_CUDA(cudaMemsetAsync(v.cell_start, 0, ((size_t)v.g.key_space + 1) * sizeof(uint32_t), st));
    s->scan_tmp_bytes = sort_scan_tmp_bytes(v.g.key_space);
    uint8_t* tmp;
    FE_CUDA(dalloc(L, &tmp, s->scan_tmp_bytes, dev, st));
    s->scan_tmp = tmp;
    // CG vectors
    CgWork& w = s->cg;
    float* vec;
    FE_CUDA(dalloc(L, &vec, nc * 9, dev, st));
    FE_CUDA(cudaMemsetAsync(vec, 0, nc * 9 * sizeof(float), st));
    w.r0 = vec; w.r1 = vec + nc; w.w0 = vec + 2 * nc; w.w1 = vec + 3 * nc;
    w.s0 = vec + 4 * nc; w.s1 = vec + 5 * nc; w.pv = vec + 6 * nc; w.x = vec + 7 * nc;
    w.rws0 = reinterpret_cast<float4*>(vec);
    w.rws1 = reinterpret_cast<float4*>(vec + 4 * nc);
    w.xcg = vec + 8 * nc;
    FE_CUDA(dalloc(L, &w.list, nc, dev, st));
    // multigrid levels 1 .. L-1 (dense; level 0 is the grid above)
    s->mg.levels = 0;
    s->use_mg = s->desc.pressure_solver == FE_PRESSURE_MGPCG ||
                (s->desc.pressure_solver == FE_PRESSURE_AUTO && nc >= kMgAutoCells);
    if (s->use_mg) {
        fe_status mst = ensure_mg(s);
        if (mst != FE_OK) return mst;
    }
    FE_CUDA(cg_prepare(w, s->device));
    // 3 rotating totals slots (12 doubles) + per-block FLUID counts of up to kMaxCgBlocks solver blocks
    FE_CUDA(dalloc(L, &w.partial, cg_partial_doubles(kMaxCgBlocks), dev, st));
    FE_CUDA(cudaMemsetAsync(w.partial, 0, cg_partial_doubles(kMaxCgBlocks) * sizeof(double), st));
    FE_CUDA(dalloc(L, &w.bar, kCgBarWords, dev, st));
    FE_CUDA(cudaMemsetAsync(w.bar, 0, kCgBarWords * sizeof(unsigned), st));
    FE_CUDA(dalloc(L, &w.err, 1, dev, st));
    FE_CUDA(cudaMemsetAsync(w.err, 0, sizeof(int), st));
    FE_CUDA(dalloc(L, &s->stats_ring, (size_t)kStatsRingEntries, dev, st));
    w.stats = s->stats_ring;
    w.stats_cap = kStatsRingEntries;
    FE_CUDA(dalloc(L, &s->d_scalar, 4, dev, st));
    // marking tables
    const int n[3] = {nx, ny, nz};
    double maxH = std::max(v.h[0], std::max(v.h[1], v.h[2]));
    v.radius = 1.2 * maxH / std::sqrt(2.0);  // pic_simulator.cpp:458-460
    v.band = 2.0 * v.radius;
    v.bucket = 2 * v.radius;                 // BuildSearcher(..., 2 * radious), pic_simulator.cpp:462
    v.any_inexact = 0;
    for (int a = 0; a < 3; ++a) {
        std::vector<double> qpos(n[a]), qf(n[a]);
        std::vector<int> b0(n[a]), b1(n[a]), i0(n[a]);
        std::vector<uint8_t> ex(n[a]);
        for (int i = 0; i < n[a]; ++i) {
            qpos[i] = v.sdf_origin[a] + i * v.h[a];                          // Grid3D::GridIndexToPosition
            b0[i] = (int)std::floor(qpos[i] / v.bucket);                     // GetBucketIndex
            b1[i] = (((float)b0[i] + 0.5f) * v.bucket <= qpos[i]) ? b0[i] + 1 : b0[i] - 1;  // GetNearbyKeys
            double cc = (v.origin[a] + 0.5 * v.h[a]) + v.h[a] * i;          // GetCellCenterPos
            double t = (cc - v.sdf_origin[a]) / v.h[a];                      // ScalarGrid3D::Sample
            bary_host(t, n[a] - 1, &i0[i], &qf[i]);
            ex[i] = ((qf[i] == 0.0 && i0[i] == i) || (qf[i] == 1.0 && i0[i] + 1 == i)) ? 1 : 0;
            if (!ex[i]) v.any_inexact = 1;
        }
        FE_CUDA(dalloc(L, &v.q_pos[a], n[a], dev, st));
        FE_CUDA(dalloc(L, &v.q_f[a], n[a], dev, st));
        FE_CUDA(dalloc(L, &v.q_b0[a], n[a], dev, st));
        FE_CUDA(dalloc(L, &v.q_b1[a], n[a], dev, st));
        FE_CUDA(dalloc(L, &v.q_i0[a], n[a], dev, st));
        FE_CUDA(dalloc(L, &v.q_exact[a], n[a], dev, st));
        FE_CUDA(cudaMemcpyAsync(v.q_pos[a], qpos.data(), n[a] * sizeof(double), cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.q_f[a], qf.data(), n[a] * sizeof(double), cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.q_b0[a], b0.data(), n[a] * sizeof(int), cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.q_b1[a], b1.data(), n[a] * sizeof(int), cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.q_i0[a], i0.data(), n[a] * sizeof(int), cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.q_exact[a], ex.data(), n[a], cudaMemcpyHostToDevice, st));
        FE_CUDA(cudaStreamSynchronize(st));  // the host tables above are freed at the end of this iteration
    }
    if (v.any_inexact) {
        FE_CUDA(dalloc(L, &v.crit_list, nc, dev, st));
        FE_CUDA(dalloc(L, &v.crit_count, 1, dev, st));
        FE_CUDA(dalloc(L, &v.crit_flag, (nc + 3) & ~(size_t)3, dev, st));
    }
    if (s->desc.viscosity > 0.0) {
        fe_status ds = alloc_diffusion(s);
        if (ds != FE_OK) return ds;
    }
    // everything above is complete before any other stream touches the scene
    FE_CUDA(cudaStreamSynchronize(st));
    return FE_OK;
}

// Allocates both particle sets and the per-particle scratch for `cap` particles; the first `keep` particles of
// the current set are copied into set 0 (which becomes current) before the old buffers are released.
// The fixed face lists of the collider classification (blocked faces; faces ConstrainVelocity rewrites, with their
// normals), counted on the device and allocated to size, so the per-substep passes visit only those faces.
fe_status collider_face_lists(fe_scene* s)
{
    auto& w = s->cw;
    cudaStream_t st = s->stream;
    const size_t nf = (size_t)(s->base.g.nx + 1) * s->base.g.ny * s->base.g.nz +
                      (size_t)s->base.g.nx * (s->base.g.ny + 1) * s->base.g.nz +
                      (size_t)s->base.g.nx * s->base.g.ny * (s->base.g.nz + 1);
    if (nf >= 0x80000000ull) return set_error(FE_ERR_BAD_ARG, "collider scenes need fewer than 2^31 faces");
    FE_CUDA(launch_collider_face_lists(s->base, w, true, st));
    uint32_t cnt[2] = {0, 0};
    FE_CUDA(cudaMemcpyAsync(cnt, w.face_cnt, sizeof cnt, cudaMemcpyDeviceToHost, st));
    FE_CUDA(cudaStreamSynchronize(st));
    free_list(s->cw_face_allocs, st);
    auto& L = s->cw_face_allocs;
    FE_CUDA(dalloc(L, &w.blk_list, std::max<size_t>(cnt[0], 1), s->device, st));
    FE_CUDA(dalloc(L, &w.fin_list, std::max<size_t>(cnt[1], 1), s->device, st));
    FE_CUDA(dalloc(L, &w.fin_nrm, 3 * std::max<size_t>(cnt[1], 1), s->device, st));
    w.n_blk = cnt[0];
    w.n_fin = cnt[1];
    FE_CUDA(launch_collider_face_lists(s->base, w, false, st));
    return FE_OK;
}

// The collision response's buffers, sized by the particle capacity and the collider count.
fe_status collide_particle_buffers(fe_scene* s)
{
    const int ncoll = std::max(s->colliders.count, 1);
    if (s->cw_cap == s->cap && s->cw_ncoll == ncoll && s->cw.ins && s->cw.cp) return FE_OK;
    free_list(s->cw_particle_allocs, s->stream);
    auto& L = s->cw_particle_allocs;
    auto& w = s->cw;
    const uint64_t cap = std::max<uint64_t>(s->cap, 1);
    const uint64_t entries = cap * (uint64_t)ncoll;
    FE_CUDA(dalloc(L, &w.start, 3 * cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.startv, 3 * cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.spos, 3 * cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.flag, cap + 1, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.offs, cap + 1, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.list, cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.cp, 3 * entries, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.nrm, 3 * entries, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.ins, entries, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.act, entries + 1, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.act_offs, entries + 1, s->device, s->stream));
    FE_CUDA(dalloc(L, &w.act_list, entries, s->device, s->stream));
    w.act_tmp_bytes = sort_scan_tmp_bytes((uint32_t)(entries + 1));
    uint8_t* atmp = nullptr;
    FE_CUDA(dalloc(L, &atmp, w.act_tmp_bytes, s->device, s->stream));
    w.act_tmp = atmp;
    FE_CUDA(dalloc(L, &w.slot_of, kMaxColliders, s->device, s->stream));
    w.scan_tmp_bytes = sort_scan_tmp_bytes((uint32_t)(cap + 1));
    uint8_t* tmp = nullptr;
    FE_CUDA(dalloc(L, &tmp, w.scan_tmp_bytes, s->device, s->stream));
    w.scan_tmp = tmp;
    s->cw_cap = s->cap;
    s->cw_ncoll = ncoll;
    return FE_OK;
}

fe_status alloc_particles(fe_scene* s, uint64_t cap, uint64_t keep = 0)
{
    drop_graphs(s);
    std::vector<void*> old = std::move(s->particle_allocs);
    s->particle_allocs.clear();
    const ParticleSet src = s->set[s->parity];
    auto& L = s->particle_allocs;
    const bool apic = s->desc.solver == FE_SOLVER_APIC;
    for (int k = 0; k < 2; ++k) {
        ParticleSet& p = s->set[k];
        FE_CUDA(dalloc(L, &p.px, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.py, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.pz, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.vx, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.vy, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.vz, cap, s->device, s->stream));
        FE_CUDA(dalloc(L, &p.pid, cap, s->device, s->stream));
        for (int a = 0; a < 9; ++a) {
            p.c[a] = nullptr;
            if (apic) FE_CUDA(dalloc(L, &p.c[a], cap, s->device, s->stream));
        }
    }
    SceneView& v = s->base;
    FE_CUDA(dalloc(L, &v.key, cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &v.rank, cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &v.perm, cap, s->device, s->stream));
    FE_CUDA(dalloc(L, &s->staging, cap * 9, s->device, s->stream));
    FE_CUDA(dalloc(L, &s->staging_u32, cap, s->device, s->stream));
    if (keep) {
        const ParticleSet& dst = s->set[0];
        auto cp = [&](void* d, const void* sp, size_t bytes) {
            return cudaMemcpyAsync(d, sp, bytes, cudaMemcpyDeviceToDevice, s->stream);
        };
        const size_t fb = keep * sizeof(float);
        FE_CUDA(cp(dst.px, src.px, fb)); FE_CUDA(cp(dst.py, src.py, fb)); FE_CUDA(cp(dst.pz, src.pz, fb));
        FE_CUDA(cp(dst.vx, src.vx, fb)); FE_CUDA(cp(dst.vy, src.vy, fb)); FE_CUDA(cp(dst.vz, src.vz, fb));
        FE_CUDA(cp(dst.pid, src.pid, keep * sizeof(uint32_t)));
        for (int a = 0; a < 9; ++a)
            if (dst.c[a] && src.c[a]) FE_CUDA(cp(dst.c[a], src.c[a], fb));
        s->parity = 0;
        s->prev_valid = false;  // the other set no longer holds the last substep's start
    }
    free_list(old, s->stream);  // stream order: after the copies
    s->cap = cap;
    if (s->colliders.count > 0) return collide_particle_buffers(s);
    return FE_OK;
}

// Makes the velocity live in buffer `want` (0 = A, 1 = B); only stage-by-stage runs ever need the copy.
cudaError_t ensure_grid(fe_scene* s, int want, cudaStream_t st = nullptr)
{
    if (s->grid_cur == want) return cudaSuccess;
    const SceneView& v = s->base;
    const size_t nf = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz + (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz +
                      (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    float* src = s->grid_cur ? v.u2 : v.u;
    float* dst = want ? v.u2 : v.u;
    s->grid_cur = want;
    return cudaMemcpyAsync(dst, src, nf * sizeof(float), cudaMemcpyDeviceToDevice, st ? st : s->stream);
}

int pressure_buffer(const fe_scene* s) { return (s->base.extrap_depth > 0 && (s->base.extrap_depth & 1)) ? 1 : 0; }

// Internal steps of one substep; the public fe_stage ids map onto ranges of them.
enum { kStepSort, kStepP2g, kStepMark, kStepPre, kStepDiffuse, kStepRhs, kStepCg, kStepApply, kStepPost, kStepG2p,
       kStepMove, kStepCount };

int first_step(int stage)
{
    static const int m[FE_STAGE_COUNT] = {kStepSort, kStepP2g, kStepMark, kStepPre, kStepDiffuse, kStepRhs, kStepPost,
                                          kStepG2p, kStepMove};
    return m[stage];
}
int last_step(int stage)
{
    static const int m[FE_STAGE_COUNT] = {kStepSort, kStepP2g, kStepMark, kStepPre, kStepDiffuse, kStepApply, kStepPost,
                                          kStepG2p, kStepMove};
    return m[stage];
}

// MoveParticles' parameters as k_g2p uses them, for the collision response's replayed moves.
CollideMove collide_move(const SceneView& v, double dt)
{
    CollideMove g;
    g.nsub = v.rk_substeps;
    g.dt_sub = (float)(dt / g.nsub);
    for (int a = 0; a < 3; ++a) {
        g.lo[a] = (float)v.origin[a];
        g.hi[a] = (float)(v.origin[a] + v.size[a]);
    }
    g.u = v.u;
    g.v = v.v;
    g.w = v.w;
    return g;
}

// Enqueues internal steps [first, last] of one substep on s->stream.
// `stream` overrides the scene's stream (a batch runs the pre-solve steps of viscous scenes on its own stream).
// Residual reduction asked of each FP32 inner solve: the scene's setting, or (0) the solver's default.  The plain
// CG asks 1e-4 (the FP32 inner solve's useful limit; a sweep of 1e-2 .. 3e-5 at 128^3 put the fewest iterations
// there).  The multigrid-preconditioned CG, whose iterations each reduce the residual several-fold, splits the
// relative tolerance evenly over the fewest refinements that 1e-4 per inner solve allows: rel_tol^(1/k) with
// k = ceil(log rel_tol / log 1e-4), so 1e-3 per solve at 1e-6 (128^3 dam break, whole run: 2.43 against 2.57 ms
// per solve) and 1e-4 at 1e-8 (256^3 pool: 1e-3 would take a third refinement, 11.2 against 10.4 ms).
double inner_tol(const fe_scene_desc& d, bool multigrid)
{
    if (d.cg_inner_tol > 0.0) return d.cg_inner_tol;
    if (!multigrid || !(d.cg_rel_tol > 0.0) || d.cg_rel_tol >= 1.0) return 1e-4;
    const double k = std::max(1.0, std::ceil(std::log(d.cg_rel_tol) / std::log(1e-4) - 1e-9));
    return std::min(1e-2, std::max(1e-4, std::pow(d.cg_rel_tol, 1.0 / k)));
}

fe_status enqueue_steps(fe_scene* s, double dt, int first, int last, cudaStream_t stream = nullptr)
{
    cudaStream_t st = stream ? stream : s->stream;
    for (int step = first; step <= last; ++step) {
        SceneView v = view_of(s, s->parity);
        switch (step) {
        case kStepSort: {
            FE_CUDA(launch_sort(v, st, s->scan_tmp, s->scan_tmp_bytes));
            SceneView dst = view_of(s, s->parity ^ 1);
            FE_CUDA(launch_gather(v, dst, st));
            s->parity ^= 1;
            s->prev_valid = true;
            s->mesh_sdf = false;
            s->collider_built = true;
            break;
        }
        case kStepP2g:
            FE_CUDA(launch_p2g(v, st));
            s->grid_cur = 0;
            break;
        case kStepMark:
            if (s->colliders.count > 0) FE_CUDA(launch_collider_marks(v, s->cw, s->surf.node, &s->collider_fluid_sdf, st));
            else FE_CUDA(launch_mark(v, st));
            break;
        case kStepPre:
            FE_CUDA(ensure_grid(s, 0, st));
            if (s->colliders.count > 0) {
                // ExtrapolateVelocityToAir, ConstrainVelocity, forces, ConstrainVelocity (pic_simulator.cpp:186-211)
                float* A[3] = {v.u, v.v, v.w};
                float* B[3] = {v.u2, v.v2, v.w2};
                float* const* fin = (v.extrap_depth & 1) ? B : A;
                const uint8_t* mk[3] = {v.mu, v.mv, v.mw};
                if (v.extrap_depth > 0) FE_CUDA(launch_extrap_faces(v, A, fin, B, mk, v.mu2, v.extrap_depth, st));
                FE_CUDA(launch_collider_bc(v, s->cw, fin, st));
                FE_CUDA(launch_add_gravity(v, fin, dt, st));
                if (s->forces.count > 0) FE_CUDA(launch_forces(v, s->forces, fin[0], fin[1], fin[2], dt, st, false));
                FE_CUDA(launch_collider_bc(v, s->cw, fin, st));
                s->grid_cur = pressure_buffer(s);
                break;
            }
            FE_CUDA(launch_pre(v, dt, st));
            s->grid_cur = pressure_buffer(s);
            if (s->forces.count > 0) {
                const int pb = pressure_buffer(s);
                FE_CUDA(launch_forces(v, s->forces, pb ? v.u2 : v.u, pb ? v.v2 : v.v, pb ? v.w2 : v.w, dt, st));
            }
            break;
        case kStepDiffuse:
            if (s->desc.viscosity > 0.0) {
                const int pb = pressure_buffer(s);
                FE_CUDA(ensure_grid(s, pb, st));
                FE_CUDA(launch_diffuse(v, s->diff, s->cg, pb ? v.u2 : v.u, pb ? v.v2 : v.v, pb ? v.w2 : v.w, dt,
                                       s->desc.viscosity, st));
            }
            break;
        case kStepRhs:
            FE_CUDA(ensure_grid(s, pressure_buffer(s), st));
            FE_CUDA(launch_rhs(v, st));
            if (s->colliders.count > 0) FE_CUDA(launch_collider_project_rhs(v, s->cw, s->cg.err, st));
            break;
        case kStepCg:
            if (s->use_mg && s->mg.levels >= 2 && s->colliders.count == 0)
                FE_CUDA(launch_mgcg(v, s->cg, s->mg, s->desc.cg_rel_tol, inner_tol(s->desc, true), s->desc.cg_max_it,
                                    s->desc.max_refine, st));
            else
                FE_CUDA(launch_cg(v, s->cg, s->desc.cg_rel_tol, inner_tol(s->desc, false), s->desc.cg_max_it,
                                  s->desc.max_refine, st));
            break;
        case kStepApply:
            FE_CUDA(ensure_grid(s, pressure_buffer(s), st));
            FE_CUDA(launch_apply(v, st));
            if (s->colliders.count > 0) {  // ComputePressure ends with ApplyBoundryCondition (pic_simulator.cpp:228)
                const int pb = pressure_buffer(s);
                float* P[3] = {pb ? v.u2 : v.u, pb ? v.v2 : v.v, pb ? v.w2 : v.w};
                FE_CUDA(launch_collider_bc(v, s->cw, P, st));
            }
            break;
        case kStepPost:
            FE_CUDA(ensure_grid(s, pressure_buffer(s), st));
            if (s->colliders.count > 0) {  // ExtrapolateVelocityToAir, ConstrainVelocity (pic_simulator.cpp:233-234)
                float* A[3] = {v.u, v.v, v.w};
                float* B[3] = {v.u2, v.v2, v.w2};
                const int d = v.extrap_depth;
                const uint8_t* mk[3] = {v.mu, v.mv, v.mw};
                if (d > 0) FE_CUDA(launch_extrap_faces(v, (d & 1) ? B : A, A, (d & 1) ? A : B, mk, v.mu2, d, st));
                FE_CUDA(launch_collider_bc(v, s->cw, A, st));
            } else {
                FE_CUDA(launch_post(v, st));
            }
            s->grid_cur = 0;
            break;
        case kStepG2p:
            FE_CUDA(ensure_grid(s, 0, st));
            if (last >= kStepMove && s->colliders.count > 0) {
                // the collision response needs the state between the transfer and the move: no fusion
                FE_CUDA(launch_g2p(v, dt, true, false, st));
                FE_CUDA(launch_collider_keep_start(v, s->cw, st));
                FE_CUDA(launch_g2p(v, dt, false, true, st));
                FE_CUDA(launch_collider_resolve(v, s->colliders, s->cw, collide_move(v, dt), st));
                step = kStepMove;
            } else if (last >= kStepMove) {
                FE_CUDA(launch_g2p(v, dt, true, true, st));
                step = kStepMove;
            } else {
                FE_CUDA(launch_g2p(v, dt, true, false, st));
            }
            break;
        case kStepMove:
            FE_CUDA(ensure_grid(s, 0, st));
            if (s->colliders.count > 0) FE_CUDA(launch_collider_keep_start(v, s->cw, st));
            FE_CUDA(launch_g2p(v, dt, false, true, st));
            if (s->colliders.count > 0) FE_CUDA(launch_collider_resolve(v, s->colliders, s->cw, collide_move(v, dt), st));
            break;
        default:
            return set_error(FE_ERR_BAD_ARG, "unknown step %d", step);
        }
    }
    return FE_OK;
}

fe_status enqueue_stages(fe_scene* s, double dt, int first_stage, int last_stage)
{
    return enqueue_steps(s, dt, first_step(first_stage), last_step(last_stage));
}

// The three phases a substep graph is split into: everything before the solve, the solve, the rest.
const int kPhaseFirst[3] = {kStepSort, kStepCg, kStepApply};
const int kPhaseLast[3] = {kStepRhs, kStepCg, kStepMove};
const char* const kPhaseName[3] = {"pre-solve", "pressure solve", "post-solve"};

fe_status check_device_error(fe_scene* s)
{
    int err = 0;
    FE_CUDA(cudaMemcpyAsync(&err, s->cg.err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    if (err) {
        cudaMemsetAsync(s->cg.err, 0, sizeof(int), s->stream);
        cudaMemsetAsync(s->cg.bar, 0, kCgBarWords * sizeof(unsigned), s->stream);  // arrival and exit counts
        cudaMemsetAsync(s->cg.partial, 0, kCgTotalsDoubles * sizeof(double), s->stream);  // totals restart at zero
        cudaStreamSynchronize(s->stream);
        return set_error((fe_status)err, "pressure solve: grid barrier wait exceeded its limit");
    }
    return FE_OK;
}

// Captures steps [first, last] of one substep of particle parity `parity` as one graph.
fe_status capture_one(fe_scene* s, int parity, double dt, int first, int last, cudaGraphExec_t* out, uint64_t* kernels)
{
    const int saved_parity = s->parity, saved_grid = s->grid_cur;
    s->parity = parity;
    s->grid_cur = 0;
    cudaGraph_t g = nullptr;
    g_capturing = true;
    g_capture_launches = 0;
    cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
    fe_status st = e == cudaSuccess ? enqueue_steps(s, dt, first, last) : cuda_check(e, "begin capture");
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
    g_capturing = false;
    s->parity = saved_parity;
    s->grid_cur = saved_grid;
    if (st != FE_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e2 != cudaSuccess) return cuda_check(e2, "end capture");
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_check(e, "graph instantiate");
    *out = exec;
    *kernels = g_capture_launches;
    return FE_OK;
}

fe_status capture_graphs(fe_scene* s, int parity, double dt)
{
    const int saved_parity = s->parity, saved_grid = s->grid_cur;
    s->parity = parity;
    s->grid_cur = 0;
    fe_status result = FE_OK;
    for (int ph = 0; ph < 3 && result == FE_OK; ++ph) {
        cudaGraph_t g = nullptr;
        g_capturing = true;
        g_capture_launches = 0;
        cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
        fe_status st = e == cudaSuccess ? enqueue_steps(s, dt, kPhaseFirst[ph], kPhaseLast[ph])
                                        : cuda_check(e, "begin capture");
        cudaError_t e2 = cudaStreamEndCapture(s->stream, &g);
        g_capturing = false;
        if (st != FE_OK) {
            if (g) cudaGraphDestroy(g);
            result = st;
            break;
        }
        if (e2 != cudaSuccess) {
            result = cuda_check(e2, "end capture");
            break;
        }
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) {
            result = cuda_check(e, "graph instantiate");
            break;
        }
        s->graph[parity][ph] = exec;
        s->graph_kernels[parity][ph] = g_capture_launches;
    }
    s->parity = saved_parity;
    s->grid_cur = saved_grid;
    return result;
}

// One substep: the three phase graphs of the current parity (captured on first use for this dt); when
// `ev` is non-null, events ev[0..3] are recorded before, between and after the phases.
fe_status emit_particles(fe_scene* s);

fe_status run_substep(fe_scene* s, double dt, cudaEvent_t* ev)
{
    TraceRange trace("substep");
    s->last_substep_empty = false;
    if (!s->emitters.empty()) {
        // emitters change the particle count every substep: direct launches, no graphs
        fe_status st = emit_particles(s);
        if (st != FE_OK) return st;
        if (!s->have_particles || s->base.np == 0) {
            // Nothing emitted yet: the reference's substep would only build an all-air grid and the all-positive
            // SDF of no particles, which emits like the initial 0 SDF, so skipping it leaves the same state.
            s->last_substep_empty = true;
            s->collider_built = true;
            s->mesh_sdf = false;  // the substep's SDF of no particles is positive everywhere (emits like the initial 0)
            for (int q = 0; q < 4; ++q)
                if (ev) FE_CUDA(cudaEventRecord(ev[q], s->stream));
            return FE_OK;
        }
        s->last_substep_empty = false;
        for (int ph = 0; ph < 3; ++ph) {
            TraceRange phase(kPhaseName[ph]);
            if (ev) FE_CUDA(cudaEventRecord(ev[ph], s->stream));
            st = enqueue_steps(s, dt, kPhaseFirst[ph], kPhaseLast[ph]);
            if (st != FE_OK) return st;
        }
        if (ev) FE_CUDA(cudaEventRecord(ev[3], s->stream));
        return FE_OK;
    }
    if (!s->graphs_disabled) {
        if (s->graph_dt != dt) {
            drop_graphs(s);
            s->graph_dt = dt;
        }
        const int par = s->parity;
        if (!s->graph[par][0]) {
            fe_status st = capture_graphs(s, par, dt);
            if (st != FE_OK) {
                // Capture is an optimisation; fall back to direct launches.
                cudaGetLastError();
                s->graphs_disabled = true;
                drop_graphs(s);
            }
        }
    }
    if (s->graphs_disabled) {
        for (int ph = 0; ph < 3; ++ph) {
            TraceRange phase(kPhaseName[ph]);
            if (ev) FE_CUDA(cudaEventRecord(ev[ph], s->stream));
            fe_status st = enqueue_steps(s, dt, kPhaseFirst[ph], kPhaseLast[ph]);
            if (st != FE_OK) return st;
        }
        if (ev) FE_CUDA(cudaEventRecord(ev[3], s->stream));
        return FE_OK;
    }
    const int par = s->parity;
    if (!ev && !s->whole[par]) {
        // a plain step replays the whole substep as one graph (profiled steps keep the phase graphs, between
        // which they record events)
        fe_status st = capture_one(s, par, dt, kStepSort, kStepMove, &s->whole[par], &s->whole_kernels[par]);
        if (st != FE_OK) {
            cudaGetLastError();
            s->whole[par] = nullptr;
        }
    }
    if (!ev && s->whole[par]) {
        FE_CUDA(cudaGraphLaunch(s->whole[par], s->stream));
        g_launches += s->whole_kernels[par];
    } else {
        for (int ph = 0; ph < 3; ++ph) {
            TraceRange phase(kPhaseName[ph]);
            if (ev) FE_CUDA(cudaEventRecord(ev[ph], s->stream));
            FE_CUDA(cudaGraphLaunch(s->graph[par][ph], s->stream));
            g_launches += s->graph_kernels[par][ph];
        }
        if (ev) FE_CUDA(cudaEventRecord(ev[3], s->stream));
    }
    s->parity ^= 1;  // the sort inside the first graph flipped the buffer sets
    s->prev_valid = true;
    s->mesh_sdf = false;
    s->collider_built = true;
    s->grid_cur = 0;
    return FE_OK;
}

// The band SDF from which the reference's last Fluid3::sdf was built: the positions at the start of the last
// substep (the other particle set, once a substep has run), else the current particles.  Allocates the surface
// buffers on first use.
fe_status surf_alloc(fe_scene* s)
{
    auto& w = s->surf;
    const SceneView& b = s->base;
    const size_t nc = (size_t)b.g.nx * b.g.ny * b.g.nz;
    if (!w.sdf) {
        cudaStream_t st = s->own_stream;
        FE_CUDA(cudaStreamSynchronize(s->stream));
        w.items = mc_items(b.g.nx, b.g.ny, b.g.nz);
        if (w.items + 1 >= (1ull << 32)) return set_error(FE_ERR_BAD_ARG, "grid too large for surface extraction");
        w.tmp_bytes = sort_scan_tmp_bytes((uint32_t)w.items);
        auto& L = s->allocs;
        FE_CUDA(dalloc(L, &w.node, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.sdf, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.cfg, w.items, s->device, st));
        FE_CUDA(dalloc(L, &w.nvert, w.items, s->device, st));
        FE_CUDA(dalloc(L, &w.ntri, w.items, s->device, st));
        FE_CUDA(dalloc(L, &w.vbase, w.items + 1, s->device, st));
        FE_CUDA(dalloc(L, &w.tbase, w.items + 1, s->device, st));
        uint8_t* tmp;
        FE_CUDA(dalloc(L, &tmp, w.tmp_bytes, s->device, st));
        w.tmp = tmp;
        FE_CUDA(cudaStreamSynchronize(st));
    }
    return FE_OK;
}

// Fluid3::sdf as the reference holds it now, into surf.sdf: the mesh SDF of fe_scene_init_from_mesh until the next
// substep; else the band SDF of the particles at the start of the last substep (or of the current particles before
// any substep).
fe_status surface_sdf(fe_scene* s)
{
    fe_status st = surf_alloc(s);
    if (st != FE_OK) return st;
    if (!s->prev_valid && s->mesh_sdf) return FE_OK;
    if (s->prev_valid && s->colliders.count > 0 && s->collider_fluid_sdf) {  // after ExtrapolateIntoCollider
        const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
        FE_CUDA(cudaMemcpyAsync(s->surf.sdf, s->collider_fluid_sdf, nc * sizeof(double), cudaMemcpyDeviceToDevice,
                                s->stream));
        return FE_OK;
    }
    const SceneView v = view_of(s, s->prev_valid ? (s->parity ^ 1) : s->parity);
    FE_CUDA(launch_node_sdf(v, s->surf.node, s->surf.sdf, s->stream));
    return FE_OK;
}

// PICSimulator::OnBeginAdvanceTimeStep's emitter loop (pic_simulator.cpp:160-163): every VolumeEmitter adds its
// particles to the current set before the substep, reading the fluid SDF the previous substep built (zero -- the
// initial value of Fluid3::sdf -- before any substep and without a mesh initialisation).  The emitter also needs
// the collider SDF > 0 at the node, and the collider SDF is built right after the emitters, so in a scene's first
// substep it still holds its initial 0 and nothing is emitted.  The counts are read back
// to size the particle arrays, so a substep with emitters runs without graphs.
fe_status emit_particles(fe_scene* s)
{
    if (s->emitters.empty() || !s->collider_built) return FE_OK;  // colliderSdf(i, j, k) > 0 fails on the initial 0
    cudaStream_t st = s->stream;
    const double* fluid = nullptr;
    if (s->prev_valid || s->mesh_sdf) {
        fe_status e = surface_sdf(s);
        if (e != FE_OK) return e;
        fluid = s->surf.sdf;
    }
    const SceneView& b = s->base;
    for (auto& em : s->emitters) {
        const size_t nc = (size_t)em.n[0] * em.n[1] * em.n[2];
        FE_CUDA(launch_emit_count(em.sdf, em.n, fluid, b.g.nx, b.g.ny, em.ppb, em.count, st,
                                  s->colliders.count > 0 ? s->cw.csdf : nullptr));
        FE_CUDA(launch_exclusive_scan(em.count, (uint32_t)nc, em.offset, em.tmp, em.tmp_bytes, st));
        uint32_t total = 0;
        FE_CUDA(cudaMemcpyAsync(&total, em.offset + nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        FE_CUDA(cudaStreamSynchronize(st));
        const uint64_t np = s->base.np;
        if (!total) continue;
        if (np + total >= (1ull << 32)) return set_error(FE_ERR_BAD_ARG, "too many particles (2^32)");
        if (np + total > s->cap || !s->set[0].px) {
            fe_status e = alloc_particles(s, std::max<uint64_t>((np + total) * 5 / 4, 1024), np);
            if (e != FE_OK) return e;
        }
        FE_CUDA(launch_spawn(em.n, em.o, em.h, em.count, em.offset, em.seed + 0x9E3779B97F4A7C15ull * ++em.calls,
                             view_of(s, s->parity), np, em.vel, st));
        s->base.np = np + total;
        s->have_particles = true;
            drop_graphs(s);  // graphs are sized by the particle count
    }
    return FE_OK;
}

}  // namespace

extern "C" {

fe_status fe_scene_desc_default(fe_scene_desc* d)
{
    if (!d) return set_error(FE_ERR_BAD_ARG, "null descriptor");
    memset(d, 0, sizeof(*d));
    d->n[0] = d->n[1] = d->n[2] = 32;
    d->size[0] = d->size[1] = d->size[2] = 1.0;
    d->solver = FE_SOLVER_FLIP;
    d->flip_blend = 0.05;
    d->gravity[1] = -9.81;
    d->max_cfl = 3.0;
    d->cg_rel_tol = 1e-6;
    d->cg_max_it = 2000;
    d->cg_inner_tol = 0.0;  // the solver's own default
    d->max_refine = kMaxRefineDefault;
    d->device = 0;
    d->pressure_solver = FE_PRESSURE_AUTO;
    return FE_OK;
}

}  // extern "C"

namespace {

// Applies the fields of `t` that ask for a change (caller holds the scene's lock or owns the scene alone).
fe_status apply_tuning(fe_scene* s, const fe_tuning* t)
{
    if (t->cg_block_threads > 0 && t->cg_block_threads != 256 && t->cg_block_threads != 512 &&
        t->cg_block_threads != 1024)
        return set_error(FE_ERR_BAD_ARG, "cg_block_threads must be 256, 512 or 1024");
    if (t->multigrid > 1) return set_error(FE_ERR_BAD_ARG, "multigrid is 0 or 1");
    if (t->cg_cluster > 16 || (t->cg_cluster > 0 && (t->cg_cluster & (t->cg_cluster - 1)) != 0))
        return set_error(FE_ERR_BAD_ARG, "cg_cluster must be 1, 2, 4, 8 or 16");
    FE_CUDA(cudaSetDevice(s->device));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    const int want_threads = t->cg_block_threads > 0 ? t->cg_block_threads : s->cg.threads;
    const int want_cluster = t->cg_cluster > 0 ? t->cg_cluster : std::max(s->cg.cluster, 1);
    if (want_threads != s->cg.threads || want_cluster != std::max(s->cg.cluster, 1)) {
        CgWork w = s->cg;
        FE_CUDA(cg_prepare(w, s->device, want_threads, want_cluster));
        s->cg.blocks = w.blocks;
        s->cg.threads = w.threads;
        s->cg.cluster = w.cluster;
    }
    if (t->mg_block_level_cells > 0) {
        s->mg_block_cells = t->mg_block_level_cells;
        if (s->mg.levels >= 2) s->mg.block_from = mg_block_from(s->mg.lv, s->mg.levels, s->mg_block_cells);
    }
    if (t->pressure_extrapolation > 1) return set_error(FE_ERR_BAD_ARG, "pressure_extrapolation is 0 or 1");
    if (t->pressure_extrapolation == 1 && !s->pprev_buf) {
        const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
        FE_CUDA(dalloc(s->allocs, &s->pprev_buf, nc, s->device, s->own_stream));
        FE_CUDA(cudaMemsetAsync(s->pprev_buf, 0, nc * sizeof(double), s->own_stream));
        FE_CUDA(cudaStreamSynchronize(s->own_stream));
    }
    if (t->pressure_extrapolation >= 0) s->base.pprev = t->pressure_extrapolation == 1 ? s->pprev_buf : nullptr;
    if (t->multigrid >= 0) {
        if (t->multigrid == 1) {
            fe_status st = ensure_mg(s);
            if (st != FE_OK) return st;
            FE_CUDA(cudaStreamSynchronize(s->own_stream));
        }
        s->use_mg = t->multigrid == 1;
    }
    drop_graphs(s);  // the captured substeps hold the old launch shape and solver
    ++s->epoch;
    return FE_OK;
}

// Tuning chosen by fe_scene_autotune (or stored by the caller) per (device, grid, transfer): scenes created with
// FE_PRESSURE_AUTO start from it.
struct TuneKey {
    int device, nx, ny, nz, solver;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(device, nx, ny, nz, solver) < std::tie(o.device, o.nx, o.ny, o.nz, o.solver);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, fe_tuning> g_tune_cache;

bool tuning_lookup(int device, int nx, int ny, int nz, int solver, fe_tuning* out)
{
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(TuneKey{device, nx, ny, nz, solver});
    if (it == g_tune_cache.end()) return false;
    *out = it->second;
    return true;
}

}  // namespace

extern "C" {

fe_status fe_scene_create(const fe_scene_desc* desc, fe_scene** out)
{
    if (!desc || !out) return set_error(FE_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    for (int a = 0; a < 3; ++a) {
        if (desc->n[a] < 2 || desc->n[a] > 4096) return set_error(FE_ERR_BAD_ARG, "grid size must be in [2, 4096]");
        if (!(desc->size[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "domain size must be positive");
    }
    if ((uint64_t)fe_key_space(desc->n[0], desc->n[1], desc->n[2]) >= (1ull << 32) - 2)
        return set_error(FE_ERR_BAD_ARG, "grid too large for 32-bit cell keys");
    if ((uint64_t)desc->n[0] * desc->n[1] * desc->n[2] >= (1ull << 26))
        return set_error(FE_ERR_BAD_ARG, "at most 2^26 cells per scene (the solver packs cell indices in 26 bits)");
    if (desc->solver < FE_SOLVER_PIC || desc->solver > FE_SOLVER_APIC) return set_error(FE_ERR_BAD_ARG, "bad solver");
    if (!(desc->max_cfl > 0.0) || desc->max_cfl > 64.0) return set_error(FE_ERR_BAD_ARG, "max_cfl must be in (0, 64]");
    if (!(desc->cg_rel_tol > 0.0) || desc->cg_max_it < 1) return set_error(FE_ERR_BAD_ARG, "bad CG settings");
    if (desc->pressure_solver != FE_PRESSURE_AUTO && desc->pressure_solver != FE_PRESSURE_MGPCG &&
        desc->pressure_solver != FE_PRESSURE_CG)
        return set_error(FE_ERR_BAD_ARG, "bad pressure solver %d", desc->pressure_solver);
    if (!(desc->viscosity >= 0.0) || !std::isfinite(desc->viscosity))
        return set_error(FE_ERR_BAD_ARG, "viscosity must be finite and >= 0");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return set_error(FE_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    if (desc->device < 0 || desc->device >= ndev) return set_error(FE_ERR_BAD_ARG, "device %d out of range", desc->device);
    FE_CUDA(cudaSetDevice(desc->device));

    fe_scene* s = new (std::nothrow) fe_scene();
    if (!s) return set_error(FE_ERR_OOM, "host allocation failed");
    s->desc = *desc;
    if (s->desc.cg_inner_tol <= 0.0 || s->desc.cg_inner_tol >= 1.0) s->desc.cg_inner_tol = 0.0;  // per solver
    if (s->desc.max_refine <= 0) s->desc.max_refine = kMaxRefineDefault;
    s->device = desc->device;
    SceneView& v = s->base;
    memset(&v, 0, sizeof(v));
    v.g.nx = desc->n[0];
    v.g.ny = desc->n[1];
    v.g.nz = desc->n[2];
    v.g.tnx = fe_tiles(v.g.nx);
    v.g.tny = fe_tiles(v.g.ny);
    v.g.tnz = fe_tiles(v.g.nz);
    v.g.key_space = fe_key_space(v.g.nx, v.g.ny, v.g.nz);
    v.solver = desc->solver;
    for (int a = 0; a < 3; ++a) {
        v.h[a] = desc->size[a] / (double)desc->n[a];  // hybrid_simulator.cpp:8
        v.inv_h[a] = 1.0 / v.h[a];
        v.origin[a] = desc->origin[a];
        v.size[a] = desc->size[a];
        v.hf[a] = (float)v.h[a];
        v.inv_hf[a] = (float)((double)desc->n[a] / desc->size[a]);
        v.originf[a] = (float)desc->origin[a];
        v.sizef[a] = (float)desc->size[a];
        v.gravity[a] = desc->gravity[a];
        v.sdf_origin[a] = desc->origin[a] + v.h[a] / 2.0;  // hybrid_simulator.cpp:15
    }
    // Velocity-grid data origins: CalculateDataOrigins (grid_systems/face_centered_grid3d.cpp:324-332) runs in
    // SetGridSpacing before SetOrigin (hybrid_simulator.cpp:11-12) and is not re-run, so they ignore the domain
    // origin.  The FLIP residual grid is built with the origin (flip_simulator.cpp:5).
    const double half[3][3] = {{0, 0.5, 0.5}, {0.5, 0, 0.5}, {0.5, 0.5, 0}};
    for (int a = 0; a < 3; ++a) {
        v.xo[a] = (float)(0.0 + v.h[a] * half[0][a]);
        v.yo[a] = (float)(0.0 + v.h[a] * half[1][a]);
        v.zo[a] = (float)(0.0 + v.h[a] * half[2][a]);
        v.rxo[a] = (float)(desc->origin[a] + v.h[a] * half[0][a]);
        v.ryo[a] = (float)(desc->origin[a] + v.h[a] * half[1][a]);
        v.rzo[a] = (float)(desc->origin[a] + v.h[a] * half[2][a]);
    }
    v.blend = (float)desc->flip_blend;
    v.max_cfl = desc->max_cfl;
    v.extrap_depth = (int)std::ceil(desc->max_cfl);                         // pic_simulator.cpp:491
    v.rk_substeps = (int)(unsigned)std::max(desc->max_cfl, 1.0);            // pic_simulator.cpp:255
    fe_status st = FE_OK;
    e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) st = cuda_check(e, "stream create");
    s->stream = s->own_stream;
    if (st == FE_OK) st = alloc_grid(s);
    if (st == FE_OK && desc->max_particles > 0) st = alloc_particles(s, desc->max_particles);
    fe_tuning tuned;
    if (st == FE_OK && desc->pressure_solver == FE_PRESSURE_AUTO &&
        tuning_lookup(s->device, desc->n[0], desc->n[1], desc->n[2], desc->solver, &tuned))
        st = apply_tuning(s, &tuned);
    if (st != FE_OK) {
        if (s->own_stream) {
            cudaStreamSynchronize(s->own_stream);
            free_list(s->allocs, s->own_stream);
            free_list(s->particle_allocs, s->own_stream);
            cudaStreamSynchronize(s->own_stream);
            cudaStreamDestroy(s->own_stream);
        }
        delete s;
        return st;
    }
    *out = s;
    return FE_OK;
}

fe_status fe_scene_destroy(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    cudaSetDevice(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graphs(s);
    // back to the pool in the own stream's order (the scene's work on any stream is complete here)
    free_list(s->allocs, s->own_stream);
    free_list(s->particle_allocs, s->own_stream);
    free_list(s->surf.mesh_allocs, s->own_stream);
    for (auto& e : s->emitters) free_list(e.allocs, s->own_stream);
    for (auto& l : s->force_allocs) free_list(l, s->own_stream);
    for (auto& l : s->collider_allocs) free_list(l, s->own_stream);
    free_list(s->cw_grid_allocs, s->own_stream);
    free_list(s->cw_particle_allocs, s->own_stream);
    free_list(s->cw_face_allocs, s->own_stream);
    cudaStreamDestroy(s->own_stream);  // its pending frees still run
    delete s;
    return FE_OK;
}

fe_status fe_scene_set_particles(fe_scene* s, const float* pos, const float* vel, const float* C, uint64_t n)
{
    TraceRange trace("fe_scene_set_particles");
    if (!s || (!pos && n)) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (n >= (1ull << 32) - 1) return set_error(FE_ERR_BAD_ARG, "at most 2^32-2 particles per scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (n > s->cap || !s->set[0].px) {
        FE_CUDA(cudaStreamSynchronize(s->stream));
        fe_status st = alloc_particles(s, std::max<uint64_t>(n, 1));
        if (st != FE_OK) return st;
    }
    if (n != s->base.np) drop_graphs(s);
    s->base.np = n;
    s->parity = 0;
    if (n) {
        // staging holds 9 floats per particle: pos at [0, 3n), vel at [3n, 6n); C reuses it afterwards
        float* stp = s->staging;
        FE_CUDA(cudaMemcpyAsync(stp, pos, n * 3 * sizeof(float), cudaMemcpyDefault, s->stream));
        if (vel) FE_CUDA(cudaMemcpyAsync(stp + 3 * n, vel, n * 3 * sizeof(float), cudaMemcpyDefault, s->stream));
        SceneView v = view_of(s, 0);
        k_set_particles<<<(unsigned)((n + 255) / 256), 256, 0, s->stream>>>(v, stp, vel ? stp + 3 * n : nullptr,
                                                                          nullptr, n);
        count_launch();
        FE_CUDA(cudaGetLastError());
        if (C && s->desc.solver == FE_SOLVER_APIC) {
            // stream order: the copy below starts after k_set_particles consumed the staging buffer
            FE_CUDA(cudaMemcpyAsync(stp, C, n * 9 * sizeof(float), cudaMemcpyDefault, s->stream));
            for (int a = 0; a < 9; ++a)  // deinterleave: c[a][i] = C[9 i + a]
                FE_CUDA(cudaMemcpy2DAsync(v.c[a], sizeof(float), stp + a, 9 * sizeof(float), sizeof(float), n,
                                          cudaMemcpyDeviceToDevice, s->stream));
        }
    }
    FE_CUDA(cudaStreamSynchronize(s->stream));
    s->have_particles = true;
    s->prev_valid = false;
    return FE_OK;
}

fe_status fe_scene_reset(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& v = s->base;
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    const size_t nf = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz + (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz +
                      (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    cudaStream_t st = s->stream;
    // what fe_scene_create zeroes: both velocity buffers, the FLIP snapshot, face markers, cell marks,
    // pressure (the solver's warm start), right-hand side, sort offsets, solver vectors and scratch
    FE_CUDA(cudaMemsetAsync(v.u, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(v.u2, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(v.su, 0, nf * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(v.mu, 0, nf, st));
    FE_CUDA(cudaMemsetAsync(v.marks, 0, nc, st));
    FE_CUDA(cudaMemsetAsync(v.p, 0, nc * sizeof(double), st));
    FE_CUDA(cudaMemsetAsync(v.b, 0, nc * sizeof(double), st));
    if (s->pprev_buf) FE_CUDA(cudaMemsetAsync(s->pprev_buf, 0, nc * sizeof(double), st));
    FE_CUDA(cudaMemsetAsync(v.cell_start, 0, ((size_t)v.g.key_space + 1) * sizeof(uint32_t), st));
    FE_CUDA(cudaMemsetAsync(s->cg.r0, 0, nc * 9 * sizeof(float), st));
    FE_CUDA(cudaMemsetAsync(s->cg.partial, 0, cg_partial_doubles(kMaxCgBlocks) * sizeof(double), st));
    FE_CUDA(cudaMemsetAsync(s->cg.bar, 0, kCgBarWords * sizeof(unsigned), st));
    FE_CUDA(cudaMemsetAsync(s->cg.err, 0, sizeof(int), st));
    FE_CUDA(cudaStreamSynchronize(st));
    s->grid_cur = 0;
    s->prev_valid = false;
    s->mesh_sdf = false;
    s->collider_built = false;
    s->collider_fluid_sdf = nullptr;
    for (auto& e : s->emitters) free_list(e.allocs, s->stream);
    s->emitters.clear();
    return FE_OK;
}

fe_status fe_scene_get_particles(fe_scene* s, float* pos, float* vel, float* C, uint64_t n)
{
    TraceRange trace("fe_scene_get_particles");
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    if (n != s->base.np) return set_error(FE_ERR_BAD_ARG, "particle count mismatch (%llu vs %llu)",
                                          (unsigned long long)n, (unsigned long long)s->base.np);
    if (!n) return FE_OK;
    FE_CUDA(cudaSetDevice(s->device));
    SceneView v = view_of(s, s->parity);
    float* stp = s->staging;
    const bool wantC = C && s->desc.solver == FE_SOLVER_APIC;
    FE_CUDA(launch_scatter_out(v, pos ? stp : nullptr, vel ? stp + 3 * n : nullptr, nullptr, s->stream));
    if (pos) FE_CUDA(cudaMemcpyAsync(pos, stp, n * 3 * sizeof(float), cudaMemcpyDefault, s->stream));
    if (vel) FE_CUDA(cudaMemcpyAsync(vel, stp + 3 * n, n * 3 * sizeof(float), cudaMemcpyDefault, s->stream));
    if (wantC) {
        FE_CUDA(cudaStreamSynchronize(s->stream));
        FE_CUDA(launch_scatter_out(v, nullptr, nullptr, stp, s->stream));
        FE_CUDA(cudaMemcpyAsync(C, stp, n * 9 * sizeof(float), cudaMemcpyDefault, s->stream));
    } else if (C) {
        std::vector<float> z(n * 9, 0.f);
        FE_CUDA(cudaMemcpyAsync(C, z.data(), n * 9 * sizeof(float), cudaMemcpyDefault, s->stream));
        FE_CUDA(cudaStreamSynchronize(s->stream));
    }
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_num_particles(const fe_scene* s, uint64_t* n)
{
    if (!s || !n) return set_error(FE_ERR_BAD_ARG, "null argument");
    *n = s->base.np;
    return FE_OK;
}

fe_status fe_scene_step(fe_scene* s, double dt, int32_t nsub, fe_step_stats* stats)
{
    TraceRange trace("fe_scene_step");
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    if (!(dt > 0.0) || nsub < 0) return set_error(FE_ERR_BAD_ARG, "dt must be > 0 and nsub >= 0");
    if (!s->have_particles && s->emitters.empty()) return set_error(FE_ERR_STATE, "set particles before stepping");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (stats) FE_CUDA(cudaMemsetAsync(s->cg.bar + 2, 0, sizeof(unsigned), s->stream));
    std::vector<uint8_t> skipped;  // substeps an emitter scene ran without particles (no solve, no stats entry)
    for (int i = 0; i < nsub; ++i) {
        fe_status st = run_substep(s, dt, nullptr);
        if (st != FE_OK) return st;
        if (s->last_substep_empty) {
            skipped.resize(nsub, 0);
            skipped[i] = 1;
        }
    }
    if (stats && nsub > 0 && !skipped.empty()) {
        // the ring holds the solved substeps in order; a skipped substep reports a converged empty solve
        int solved = 0;
        for (int i = 0; i < nsub; ++i) solved += !skipped[i];
        std::vector<fe_step_stats> ring((size_t)std::min(solved, (int)kStatsRingEntries));
        if (!ring.empty())
            FE_CUDA(cudaMemcpyAsync(ring.data(), s->stats_ring, ring.size() * sizeof(fe_step_stats), cudaMemcpyDeviceToHost,
                                    s->stream));
        fe_status st = check_device_error(s);
        if (st != FE_OK) return st;
        size_t k = 0;
        for (int i = 0; i < std::min(nsub, (int)kStatsRingEntries); ++i) {
            fe_step_stats e{};
            e.converged = 1;
            stats[i] = skipped[i] ? e : ring[k++ % std::max<size_t>(ring.size(), 1)];
        }
        return FE_OK;
    }
    if (stats && nsub > 0) {
        const int cnt = std::min(nsub, (int)kStatsRingEntries);
        FE_CUDA(cudaMemcpyAsync(stats, s->stats_ring, cnt * sizeof(fe_step_stats), cudaMemcpyDeviceToHost, s->stream));
        fe_status st = check_device_error(s);
        if (st != FE_OK) return st;
    }
    return FE_OK;
}

fe_status fe_scene_step_profiled(fe_scene* s, double dt, int32_t nsub, fe_step_stats* stats, float* phase_ms)
{
    TraceRange trace("fe_scene_step_profiled");
    if (!s || !phase_ms) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (!(dt > 0.0) || nsub < 0) return set_error(FE_ERR_BAD_ARG, "dt must be > 0 and nsub >= 0");
    if (!s->have_particles) return set_error(FE_ERR_STATE, "set particles before stepping");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    std::vector<cudaEvent_t> ev((size_t)nsub * 4);
    for (auto& e : ev) FE_CUDA(cudaEventCreate(&e));
    fe_status st = FE_OK;
    if (stats) FE_CUDA(cudaMemsetAsync(s->cg.bar + 2, 0, sizeof(unsigned), s->stream));
    for (int i = 0; i < nsub && st == FE_OK; ++i) st = run_substep(s, dt, &ev[(size_t)i * 4]);
    if (st == FE_OK) {
        cudaError_t e = cudaStreamSynchronize(s->stream);
        for (int i = 0; i < nsub && e == cudaSuccess; ++i)
            for (int ph = 0; ph < 3 && e == cudaSuccess; ++ph)
                e = cudaEventElapsedTime(&phase_ms[i * 3 + ph], ev[(size_t)i * 4 + ph], ev[(size_t)i * 4 + ph + 1]);
        st = cuda_check(e, "phase timing");
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st != FE_OK) return st;
    if (stats && nsub > 0) {
        const int cnt = std::min(nsub, (int)kStatsRingEntries);
        FE_CUDA(cudaMemcpyAsync(stats, s->stats_ring, cnt * sizeof(fe_step_stats), cudaMemcpyDeviceToHost, s->stream));
    }
    return check_device_error(s);
}

fe_status fe_scene_cfl(fe_scene* s, double dt, double* cfl)
{
    if (!s || !cfl) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (!s->have_particles || s->base.np == 0) {  // no particles (an emitter scene before emission): speed 0
        *cfl = 0.0;
        return FE_OK;
    }
    FE_CUDA(ensure_grid(s, 0));
    FE_CUDA(launch_cfl(s->base, dt, s->d_scalar, s->stream));
    double m = 0;
    FE_CUDA(cudaMemcpyAsync(&m, s->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    const double minH = std::min(s->base.h[0], std::min(s->base.h[1], s->base.h[2]));
    *cfl = m * dt / minH;  // pic_simulator.cpp:94-96
    return FE_OK;
}

fe_status fe_scene_advance_frame(fe_scene* s, double frame_dt, int32_t* substeps)
{
    TraceRange trace("fe_scene_advance_frame");
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    if (!(frame_dt > 0.0)) return set_error(FE_ERR_BAD_ARG, "frame_dt must be > 0");
    if (!s->have_particles && s->emitters.empty()) return set_error(FE_ERR_STATE, "set particles before stepping");
    double remaining = frame_dt;
    int count = 0;
    while (remaining > 0.0000000001) {  // physics_animation.cpp:76
        double cfl = 0;
        fe_status st = fe_scene_cfl(s, remaining, &cfl);
        if (st != FE_OK) return st;
        const double c = std::ceil(cfl / s->desc.max_cfl);
        const unsigned n = (unsigned)std::max(c, 1.0);  // pic_simulator.cpp:353
        const double sub = remaining / (double)n;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            FE_CUDA(cudaSetDevice(s->device));
            // OnBeginAdvanceTimeStep emits after the substep count was taken from the particles before emission
            st = emit_particles(s);
            if (st != FE_OK) return st;
            if (s->have_particles && s->base.np > 0) {
                st = enqueue_stages(s, sub, FE_STAGE_SORT, FE_STAGE_MOVE);
                if (st != FE_OK) return st;
            } else {
                s->mesh_sdf = false;  // as in run_substep's skipped substep
            }
            s->collider_built = true;
        }
        remaining -= sub;
        ++count;
        if (count > 100000) return set_error(FE_ERR_STATE, "substep count exploded (non-finite velocities?)");
    }
    if (substeps) *substeps = count;
    return check_device_error(s);
}

fe_status fe_scene_run_stages(fe_scene* s, double dt, int32_t first, int32_t last)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    if (first < 0 || last >= FE_STAGE_COUNT || first > last) return set_error(FE_ERR_BAD_ARG, "bad stage range");
    if (!s->have_particles) return set_error(FE_ERR_STATE, "set particles before stepping");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    FE_CUDA(cudaMemsetAsync(s->cg.bar + 2, 0, sizeof(unsigned), s->stream));
    fe_status st = enqueue_stages(s, dt, first, last);
    if (st != FE_OK) return st;
    return check_device_error(s);
}

fe_status fe_scene_get_grid(fe_scene* s, float* u, float* v, float* w, double* p, uint8_t* marks)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& b = s->base;
    const size_t nu = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz, nvv = (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz,
                 nww = (size_t)b.g.nx * b.g.ny * (b.g.nz + 1), nc = (size_t)b.g.nx * b.g.ny * b.g.nz;
    const float* src = s->grid_cur ? b.u2 : b.u;
    if (u) FE_CUDA(cudaMemcpyAsync(u, src, nu * 4, cudaMemcpyDefault, s->stream));
    if (v) FE_CUDA(cudaMemcpyAsync(v, src + nu, nvv * 4, cudaMemcpyDefault, s->stream));
    if (w) FE_CUDA(cudaMemcpyAsync(w, src + nu + nvv, nww * 4, cudaMemcpyDefault, s->stream));
    if (p) FE_CUDA(cudaMemcpyAsync(p, b.p, nc * 8, cudaMemcpyDefault, s->stream));
    if (marks) FE_CUDA(cudaMemcpyAsync(marks, b.marks, nc, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_set_grid(fe_scene* s, const float* u, const float* v, const float* w)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& b = s->base;
    const size_t nu = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz, nvv = (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz,
                 nww = (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
    float* dst = s->grid_cur ? b.u2 : b.u;
    if (u) FE_CUDA(cudaMemcpyAsync(dst, u, nu * 4, cudaMemcpyDefault, s->stream));
    if (v) FE_CUDA(cudaMemcpyAsync(dst + nu, v, nvv * 4, cudaMemcpyDefault, s->stream));
    if (w) FE_CUDA(cudaMemcpyAsync(dst + nu + nvv, w, nww * 4, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_set_pressure(fe_scene* s, const double* p)
{
    if (!s || !p) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    FE_CUDA(cudaMemcpyAsync(s->base.p, p, nc * 8, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_get_face_markers(fe_scene* s, uint8_t* mu, uint8_t* mv, uint8_t* mw)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& b = s->base;
    const size_t nu = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz, nvv = (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz,
                 nww = (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
    if (mu) FE_CUDA(cudaMemcpyAsync(mu, b.mu, nu, cudaMemcpyDefault, s->stream));
    if (mv) FE_CUDA(cudaMemcpyAsync(mv, b.mv, nvv, cudaMemcpyDefault, s->stream));
    if (mw) FE_CUDA(cudaMemcpyAsync(mw, b.mw, nww, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_get_snapshot(fe_scene* s, float* u, float* v, float* w)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& b = s->base;
    const size_t nu = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz, nvv = (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz,
                 nww = (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
    if (u) FE_CUDA(cudaMemcpyAsync(u, b.su, nu * 4, cudaMemcpyDefault, s->stream));
    if (v) FE_CUDA(cudaMemcpyAsync(v, b.sv, nvv * 4, cudaMemcpyDefault, s->stream));
    if (w) FE_CUDA(cudaMemcpyAsync(w, b.sw, nww * 4, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_get_rhs(fe_scene* s, double* b)
{
    if (!s || !b) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    FE_CUDA(cudaMemcpyAsync(b, s->base.b, nc * 8, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_get_fluid_sdf(fe_scene* s, double* sdf)
{
    if (!s || !sdf) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (!s->have_particles && !s->mesh_sdf) return set_error(FE_ERR_STATE, "set particles first");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    fe_status st = surface_sdf(s);
    if (st != FE_OK) return st;
    const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    FE_CUDA(cudaMemcpyAsync(sdf, s->surf.sdf, nc * sizeof(double), cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_set_fluid_sdf(fe_scene* s, const double* sdf)
{
    if (!s || !sdf) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    fe_status st = surf_alloc(s);
    if (st != FE_OK) return st;
    const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    FE_CUDA(cudaMemcpyAsync(s->surf.sdf, sdf, nc * sizeof(double), cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    s->mesh_sdf = true;  // held until the next substep builds the particles' SDF
    s->prev_valid = false;
    return FE_OK;
}

}  // extern "C"

namespace fe {
namespace {

// Copies a mesh (host or device pointers) into pool memory on `st`; the caller frees `list` in stream order.
fe_status upload_mesh(const double* V, uint64_t nv, const int64_t* T, uint64_t nt, int device, cudaStream_t st,
                      std::vector<void*>& list, double** dV, int64_t** dT)
{
    if ((nv && !V) || (nt && !T)) return set_error(FE_ERR_BAD_ARG, "null mesh arrays");
    std::vector<int64_t> check;
    FE_CUDA(dalloc(list, dV, std::max<uint64_t>(3 * nv, 1), device, st));
    FE_CUDA(dalloc(list, dT, std::max<uint64_t>(4 * nt, 1), device, st));
    if (nv) FE_CUDA(cudaMemcpyAsync(*dV, V, 3 * nv * sizeof(double), cudaMemcpyDefault, st));
    if (nt) {
        FE_CUDA(cudaMemcpyAsync(*dT, T, 4 * nt * sizeof(int64_t), cudaMemcpyDefault, st));
        // vertex ids are validated on the host (a device kernel must never read outside the vertex array)
        check.resize(4 * nt);
        FE_CUDA(cudaMemcpyAsync(check.data(), *dT, 4 * nt * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
        FE_CUDA(cudaStreamSynchronize(st));
        for (uint64_t t = 0; t < nt; ++t)
            for (int q = 0; q < 3; ++q)
                if (check[4 * t + q] < 0 || (uint64_t)check[4 * t + q] >= nv)
                    return set_error(FE_ERR_BAD_ARG, "triangle %llu references vertex %lld of %llu", (unsigned long long)t,
                                     (long long)check[4 * t + q], (unsigned long long)nv);
    }
    return FE_OK;
}

// Counted particles (count per node, scanned into offset) appended to the scene's current particles.
fe_status append_counted(fe_scene* s, const int n[3], const double o[3], const double h[3], const uint32_t* count,
                         uint32_t* offset, void* tmp, size_t tmp_bytes, uint64_t seed, const float vel[3])
{
    cudaStream_t st = s->stream;
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    FE_CUDA(launch_exclusive_scan(count, (uint32_t)nc, offset, tmp, tmp_bytes, st));
    uint32_t total = 0;
    FE_CUDA(cudaMemcpyAsync(&total, offset + nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    FE_CUDA(cudaStreamSynchronize(st));
    if (!total) return FE_OK;
    const uint64_t np = s->have_particles ? s->base.np : 0;
    if (np + total >= (1ull << 32)) return set_error(FE_ERR_BAD_ARG, "too many particles (2^32)");
    if (np + total > s->cap || !s->set[0].px) {
        fe_status e = alloc_particles(s, std::max<uint64_t>(np + total, 1), np);
        if (e != FE_OK) return e;
    }
    FE_CUDA(launch_spawn(n, o, h, count, offset, seed, view_of(s, s->parity), np, vel, st));
    FE_CUDA(cudaStreamSynchronize(st));
    s->base.np = np + total;
    s->have_particles = true;
    drop_graphs(s);
    return FE_OK;
}

}  // namespace
}  // namespace fe

extern "C" {

fe_status fe_mesh_to_sdf(const double* vertices, uint64_t n_vertices, const int64_t* triangles, uint64_t n_triangles,
                         const int32_t n[3], const double origin[3], const double spacing[3], double* sdf, int32_t device)
{
    if (!n || !origin || !spacing || !sdf) return set_error(FE_ERR_BAD_ARG, "null argument");
    for (int a = 0; a < 3; ++a)
        if (n[a] < 1 || !(spacing[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "bad grid");
    FE_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    FE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<void*> list;
    double* dV = nullptr;
    int64_t* dT = nullptr;
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    unsigned long long* scratch = nullptr;
    double* dsdf = nullptr;
    const int nn[3] = {n[0], n[1], n[2]};
    fe_status r = upload_mesh(vertices, n_vertices, triangles, n_triangles, device, st, list, &dV, &dT);
    cudaError_t e = cudaSuccess;
    if (r == FE_OK) e = dalloc(list, &scratch, nc, device, st);
    if (r == FE_OK && e == cudaSuccess) e = dalloc(list, &dsdf, nc, device, st);
    if (r == FE_OK && e == cudaSuccess) e = launch_mesh_to_sdf(dV, n_vertices, dT, n_triangles, nn, origin, spacing, scratch, dsdf, st);
    if (r == FE_OK && e == cudaSuccess) e = cudaMemcpyAsync(sdf, dsdf, nc * sizeof(double), cudaMemcpyDefault, st);
    if (r == FE_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    free_list(list, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (r != FE_OK) return r;
    return cuda_check(e, "mesh to sdf");
}

fe_status fe_scene_init_from_mesh(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                  uint64_t n_triangles, uint32_t particles_per_cell, uint64_t seed)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    fe_status r = surf_alloc(s);
    if (r != FE_OK) return r;
    const SceneView& b = s->base;
    const int n[3] = {b.g.nx, b.g.ny, b.g.nz};
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    cudaStream_t st = s->stream;
    std::vector<void*> list;
    double* dV = nullptr;
    int64_t* dT = nullptr;
    r = upload_mesh(vertices, n_vertices, triangles, n_triangles, s->device, st, list, &dV, &dT);
    uint32_t *count = nullptr, *offset = nullptr;
    uint8_t* tmp = nullptr;
    const size_t tmp_bytes = sort_scan_tmp_bytes((uint32_t)nc);
    cudaError_t e = cudaSuccess;
    if (r == FE_OK) e = dalloc(list, &count, nc, s->device, st);
    if (r == FE_OK && e == cudaSuccess) e = dalloc(list, &offset, nc + 1, s->device, st);
    if (r == FE_OK && e == cudaSuccess) e = dalloc(list, &tmp, tmp_bytes, s->device, st);
    // Mesh2SDF into Fluid3::sdf, then InitializeParticles on it
    if (r == FE_OK && e == cudaSuccess)
        e = launch_mesh_to_sdf(dV, n_vertices, dT, n_triangles, n, b.sdf_origin, b.h, s->surf.node, s->surf.sdf, st);
    if (r == FE_OK && e == cudaSuccess) {
        s->mesh_sdf = true;
        s->prev_valid = false;
        e = launch_seed_count(s->surf.sdf, n, b.sdf_origin, b.h, b.origin, particles_per_cell ? particles_per_cell : 16u,
                              count, st);
    }
    if (r == FE_OK && e == cudaSuccess) {
        const float zero[3] = {0.f, 0.f, 0.f};
        r = append_counted(s, n, b.origin, b.h, count, offset, tmp, tmp_bytes, seed, zero);
    }
    free_list(list, st);
    cudaStreamSynchronize(st);
    if (r != FE_OK) return r;
    return cuda_check(e, "init from mesh");
}

fe_status fe_scene_add_volume_emitter(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                      uint64_t n_triangles, const int32_t resolution[3], const double domain_origin[3],
                                      const double domain_size[3], uint32_t particles_per_block, const double velocity[3],
                                      uint64_t seed, int32_t* id)
{
    if (!s || !resolution || !domain_origin || !domain_size || !velocity) return set_error(FE_ERR_BAD_ARG, "null argument");
    const SceneView& b = s->base;
    const int gn[3] = {b.g.nx, b.g.ny, b.g.nz};
    for (int a = 0; a < 3; ++a) {
        if (resolution[a] < 1 || resolution[a] > gn[a])
            return set_error(FE_ERR_BAD_ARG, "emitter resolution must be within the scene's grid (it indexes the fluid SDF)");
        if (!(domain_size[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "bad emitter domain");
    }
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    fe_scene::Emitter em;
    for (int a = 0; a < 3; ++a) {
        em.n[a] = resolution[a];
        em.o[a] = domain_origin[a];
        em.h[a] = domain_size[a] / resolution[a];  // volume_emmiter.cpp:12
        em.vel[a] = (float)velocity[a];
    }
    em.ppb = particles_per_block;
    em.seed = seed;
    const size_t nc = (size_t)em.n[0] * em.n[1] * em.n[2];
    em.tmp_bytes = sort_scan_tmp_bytes((uint32_t)nc);
    cudaStream_t st = s->stream;
    uint8_t* tmp = nullptr;
    FE_CUDA(dalloc(em.allocs, &em.sdf, nc, s->device, st));
    FE_CUDA(dalloc(em.allocs, &em.count, nc, s->device, st));
    FE_CUDA(dalloc(em.allocs, &em.offset, nc + 1, s->device, st));
    FE_CUDA(dalloc(em.allocs, &tmp, em.tmp_bytes, s->device, st));
    em.tmp = tmp;
    s->emitters.push_back(std::move(em));
    const int32_t idx = (int32_t)s->emitters.size() - 1;
    if (id) *id = idx;
    // VolumeEmitter::InitializeFromTriangleMesh: Mesh2SDF onto the emitter's grid
    auto& e2 = s->emitters.back();
    std::vector<void*> list;
    double* dV = nullptr;
    int64_t* dT = nullptr;
    fe_status r = upload_mesh(vertices, n_vertices, triangles, n_triangles, s->device, st, list, &dV, &dT);
    unsigned long long* scratch = nullptr;
    cudaError_t e = cudaSuccess;
    if (r == FE_OK) e = dalloc(list, &scratch, nc, s->device, st);
    if (r == FE_OK && e == cudaSuccess) e = launch_mesh_to_sdf(dV, n_vertices, dT, n_triangles, e2.n, e2.o, e2.h, scratch, e2.sdf, st);
    free_list(list, st);
    cudaStreamSynchronize(st);
    if (r == FE_OK && e != cudaSuccess) r = cuda_check(e, "emitter sdf");
    if (r != FE_OK) {
        free_list(s->emitters.back().allocs, st);
        s->emitters.pop_back();
    }
    return r;
}

fe_status fe_scene_add_force(fe_scene* s, const fe_force_desc* f, int32_t* id)
{
    if (!s || !f) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (f->kind != FE_FORCE_POINT && f->kind != FE_FORCE_SWIRL && f->kind != FE_FORCE_VOLUME)
        return set_error(FE_ERR_BAD_ARG, "unknown force kind %d", (int)f->kind);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->forces.count >= kMaxForces) return set_error(FE_ERR_BAD_ARG, "at most %d position-dependent forces", kMaxForces);
    FE_CUDA(cudaSetDevice(s->device));
    ForceDev d{};
    d.kind = f->kind;
    d.strength = f->strength;
    for (int a = 0; a < 3; ++a) d.origin[a] = f->origin[a];
    std::vector<void*> allocs;
    if (f->kind == FE_FORCE_SWIRL) {
        // SwirlField stores GetNormalized() of its axis; Sample rotates by 0.0001 degrees (PI, math_utils.hpp:11)
        const double al = std::sqrt(f->axis[0] * f->axis[0] + f->axis[1] * f->axis[1] + f->axis[2] * f->axis[2]);
        for (int a = 0; a < 3; ++a) d.axis[a] = f->axis[a] / al;
        const double angle = 0.0001 * 3.14159265358979323846 / 180;
        d.cos_a = std::cos(angle);
        d.sin_a = std::sin(angle);
    } else if (f->kind == FE_FORCE_VOLUME) {
        for (int a = 0; a < 3; ++a) {
            if (f->resolution[a] < 1 || !(f->domain_size[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "bad volume field grid");
            d.n[a] = f->resolution[a];
            d.o[a] = f->domain_origin[a];
            d.h[a] = f->domain_size[a] / f->resolution[a];  // volume_field.cpp:8
        }
        const size_t nc = (size_t)d.n[0] * d.n[1] * d.n[2];
        cudaStream_t st = s->stream;
        double* field = nullptr;
        FE_CUDA(dalloc(allocs, &field, 3 * nc, s->device, st));
        fe_status r = FE_OK;
        cudaError_t e = cudaSuccess;
        if (f->field) {
            e = cudaMemcpyAsync(field, f->field, 3 * nc * sizeof(double), cudaMemcpyDefault, st);
        } else {
            std::vector<void*> list;
            double* dV = nullptr;
            int64_t* dT = nullptr;
            r = upload_mesh(f->vertices, f->n_vertices, f->triangles, f->n_triangles, s->device, st, list, &dV, &dT);
            if (r == FE_OK) e = launch_volume_vectors(dV, f->n_vertices, dT, f->n_triangles, d.n, d.o, d.h, field, st);
            free_list(list, st);
        }
        if (r == FE_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (r == FE_OK && e != cudaSuccess) r = cuda_check(e, "volume field");
        if (r != FE_OK) {
            free_list(allocs, st);
            return r;
        }
        d.field = field;
    }
    drop_graphs(s);  // the captured substeps hold the old force list
    ++s->epoch;
    if (id) *id = s->forces.count;
    s->forces.f[s->forces.count++] = d;
    s->force_allocs.push_back(std::move(allocs));
    return FE_OK;
}

fe_status fe_scene_clear_forces(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (s->forces.count) {
        drop_graphs(s);
        ++s->epoch;
    }
    for (auto& l : s->force_allocs) free_list(l, s->stream);
    s->force_allocs.clear();
    s->forces.count = 0;
    return FE_OK;
}

fe_status fe_volume_field_vectors(const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                  uint64_t n_triangles, const int32_t n[3], const double origin[3],
                                  const double spacing[3], double* out, int32_t device)
{
    if (!n || !origin || !spacing || !out) return set_error(FE_ERR_BAD_ARG, "null argument");
    for (int a = 0; a < 3; ++a)
        if (n[a] < 1 || !(spacing[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "bad grid");
    FE_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    FE_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    std::vector<void*> list;
    double* dV = nullptr;
    int64_t* dT = nullptr;
    double* dout = nullptr;
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    const int nn[3] = {n[0], n[1], n[2]};
    fe_status r = upload_mesh(vertices, n_vertices, triangles, n_triangles, device, st, list, &dV, &dT);
    cudaError_t e = cudaSuccess;
    if (r == FE_OK) e = dalloc(list, &dout, 3 * nc, device, st);
    if (r == FE_OK && e == cudaSuccess) e = launch_volume_vectors(dV, n_vertices, dT, n_triangles, nn, origin, spacing, dout, st);
    if (r == FE_OK && e == cudaSuccess) e = cudaMemcpyAsync(out, dout, 3 * nc * sizeof(double), cudaMemcpyDefault, st);
    if (r == FE_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
    free_list(list, st);
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (r != FE_OK) return r;
    return cuda_check(e, "volume field vectors");
}

fe_status fe_scene_add_mesh_collider(fe_scene* s, const double* vertices, uint64_t n_vertices, const int64_t* triangles,
                                     uint64_t n_triangles, const double* normals, uint64_t n_normals,
                                     const int32_t resolution[3], const double grid_origin[3],
                                     const double grid_spacing[3], int32_t* id)
{
    if (!s || !resolution || !grid_origin || !grid_spacing) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (n_triangles == 0 || n_vertices == 0 || !vertices || !triangles || !normals)
        return set_error(FE_ERR_BAD_ARG, "a collider mesh needs vertices, triangles and normals");
    for (int a = 0; a < 3; ++a)
        if (resolution[a] < 1 || !(grid_spacing[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "bad collider grid");
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->colliders.count >= kMaxColliders) return set_error(FE_ERR_BAD_ARG, "at most %d colliders", kMaxColliders);
    if (s->desc.viscosity > 0.0)
        return set_error(FE_ERR_BAD_ARG, "colliders with viscosity are not supported (BackwardEulerDiffusionSolver's "
                                         "BOUNDRY faces); set the viscosity to 0 first");
    FE_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    // normal ids are validated on the host: ResolveCollision reads normals[triangle.normalIdx]
    std::vector<int64_t> tri(4 * n_triangles);
    FE_CUDA(cudaMemcpy(tri.data(), triangles, tri.size() * sizeof(int64_t), cudaMemcpyDefault));
    for (uint64_t t = 0; t < n_triangles; ++t)
        if (tri[4 * t + 3] < 0 || (uint64_t)tri[4 * t + 3] >= n_normals)
            return set_error(FE_ERR_BAD_ARG, "triangle %llu has normal id %lld of %llu", (unsigned long long)t,
                             (long long)tri[4 * t + 3], (unsigned long long)n_normals);
    fe_status r = surf_alloc(s);  // its node scratch serves the band SDF of the collider marks
    if (r != FE_OK) return r;
    std::vector<void*> allocs;
    double* dV = nullptr;
    int64_t* dT = nullptr;
    r = upload_mesh(vertices, n_vertices, triangles, n_triangles, s->device, st, allocs, &dV, &dT);
    if (r != FE_OK) {
        free_list(allocs, st);
        return r;
    }
    ColliderDev c{};
    for (int a = 0; a < 3; ++a) {
        c.n[a] = resolution[a];
        c.o[a] = grid_origin[a];
        c.h[a] = grid_spacing[a];
    }
    const size_t cn = (size_t)c.n[0] * c.n[1] * c.n[2];
    double *dN = nullptr, *dsdf = nullptr;
    unsigned long long* scratch = nullptr;
    cudaError_t e = dalloc(allocs, &dN, 3 * n_normals, s->device, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dN, normals, 3 * n_normals * sizeof(double), cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = dalloc(allocs, &dsdf, cn, s->device, st);
    std::vector<void*> tmp_list;
    if (e == cudaSuccess) e = dalloc(tmp_list, &scratch, cn, s->device, st);
    // TriangleMeshCollider's constructor: Mesh2SDF of the mesh on its own grid
    if (e == cudaSuccess) e = launch_mesh_to_sdf(dV, n_vertices, dT, n_triangles, c.n, c.o, c.h, scratch, dsdf, st);
    free_list(tmp_list, st);
    if (e != cudaSuccess) {
        free_list(allocs, st);
        return cuda_check(e, "collider");
    }
    c.sdf = dsdf;
    c.V = dV;
    c.T = dT;
    c.N = dN;
    c.nv = n_vertices;
    c.nt = n_triangles;
    // grid-sized buffers on the first collider
    auto& w = s->cw;
    const SceneView& b = s->base;
    if (s->colliders.count == 0) {
        const size_t nc = (size_t)b.g.nx * b.g.ny * b.g.nz;
        const size_t nf = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz + (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz +
                          (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
        auto& L = s->cw_grid_allocs;
        FE_CUDA(dalloc(L, &w.csdf, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.node_valid, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.cell_boundry, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.face_open, nf, s->device, st));
        FE_CUDA(dalloc(L, &w.face_cls, nf, s->device, st));
        FE_CUDA(dalloc(L, &w.vscratch, 2 * nf, s->device, st));
        FE_CUDA(dalloc(L, &w.node_vscratch, 2 * nc, s->device, st));
        FE_CUDA(dalloc(L, &w.ftmp0, nf, s->device, st));
        FE_CUDA(dalloc(L, &w.ftmp1, nf, s->device, st));
        FE_CUDA(dalloc(L, &w.fric, nf, s->device, st));
        FE_CUDA(dalloc(L, &w.face_cnt, 2, s->device, st));
        FE_CUDA(dalloc(L, &w.sdf_a, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.sdf_b, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.label, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.open_comp, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.comp_sum, nc, s->device, st));
        FE_CUDA(dalloc(L, &w.comp_cnt, nc, s->device, st));
    }
    s->colliders.c[s->colliders.count] = c;
    if (id) *id = s->colliders.count;
    s->colliders.count += 1;
    s->collider_allocs.push_back(std::move(allocs));
    // ColliderCollection::BuildSdf gives the same SDF every substep (static colliders): build and classify now
    FE_CUDA(launch_collider_setup(b, s->colliders, w, st));
    r = collider_face_lists(s);
    if (r != FE_OK) return r;
    r = collide_particle_buffers(s);
    if (r != FE_OK) return r;
    FE_CUDA(cudaStreamSynchronize(st));
    s->collider_fluid_sdf = nullptr;
    drop_graphs(s);
    ++s->epoch;
    return FE_OK;
}

fe_status fe_scene_clear_colliders(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (s->colliders.count == 0) return FE_OK;
    for (auto& l : s->collider_allocs) free_list(l, s->stream);
    s->collider_allocs.clear();
    free_list(s->cw_grid_allocs, s->stream);
    free_list(s->cw_particle_allocs, s->stream);
    free_list(s->cw_face_allocs, s->stream);
    s->cw = CollideWork{};
    s->cw_cap = 0;
    s->cw_ncoll = 0;
    s->colliders.count = 0;
    s->collider_fluid_sdf = nullptr;
    drop_graphs(s);
    ++s->epoch;
    return FE_OK;
}

fe_status fe_scene_get_collider_sdf(fe_scene* s, double* sdf)
{
    if (!s || !sdf) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const size_t nc = (size_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    if (s->colliders.count == 0 || !s->collider_built) {
        // ColliderCollection's SDF starts at 0 and is 1.7976931348623157e30 everywhere once built without colliders
        const std::vector<double> c(nc, s->collider_built ? 1.7976931348623157e30 : 0.0);
        FE_CUDA(cudaMemcpy(sdf, c.data(), nc * sizeof(double), cudaMemcpyDefault));
        return FE_OK;
    }
    FE_CUDA(cudaMemcpyAsync(sdf, s->cw.csdf, nc * sizeof(double), cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_set_emitter_sdf(fe_scene* s, int32_t id, const double* sdf)
{
    if (!s || !sdf) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    if (id < 0 || (size_t)id >= s->emitters.size()) return set_error(FE_ERR_BAD_ARG, "no emitter %d", id);
    FE_CUDA(cudaSetDevice(s->device));
    const auto& em = s->emitters[(size_t)id];
    const size_t nc = (size_t)em.n[0] * em.n[1] * em.n[2];
    FE_CUDA(cudaMemcpyAsync(em.sdf, sdf, nc * sizeof(double), cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_clear_emitters(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    for (auto& e : s->emitters) free_list(e.allocs, s->stream);
    s->emitters.clear();
    return FE_OK;
}

fe_status fe_scene_build_surface(fe_scene* s, uint64_t* n_vertices, uint64_t* n_triangles)
{
    TraceRange trace("fe_scene_build_surface");
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    if (!s->have_particles) return set_error(FE_ERR_STATE, "set particles first");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    fe_status st = surface_sdf(s);
    if (st != FE_OK) return st;
    auto& w = s->surf;
    const SceneView& v = s->base;
    cudaStream_t stream = s->stream;
    const double* msdf = w.sdf;
    if (s->colliders.count > 0 && s->collider_built) {  // MarchingCubesSolver::BuildSurface's collider step
        double* mod = reinterpret_cast<double*>(w.node);
        FE_CUDA(launch_surface_with_colliders(w.sdf, s->cw.csdf, (size_t)v.g.nx * v.g.ny * v.g.nz, mod, stream));
        msdf = mod;
    }
    FE_CUDA(launch_mc_count(v, msdf, w.cfg, w.nvert, w.ntri, stream));
    FE_CUDA(launch_exclusive_scan(w.nvert, (uint32_t)w.items, w.vbase, w.tmp, w.tmp_bytes, stream));
    FE_CUDA(launch_exclusive_scan(w.ntri, (uint32_t)w.items, w.tbase, w.tmp, w.tmp_bytes, stream));
    uint32_t tot[2] = {0, 0};
    FE_CUDA(cudaMemcpyAsync(&tot[0], w.vbase + w.items, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    FE_CUDA(cudaMemcpyAsync(&tot[1], w.tbase + w.items, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    if (tot[0] > w.cap_v || tot[1] > w.cap_t) {
        free_list(w.mesh_allocs, stream);
        w.cap_v = std::max<uint64_t>(tot[0], 1) * 5 / 4;
        w.cap_t = std::max<uint64_t>(tot[1], 1) * 5 / 4;
        FE_CUDA(dalloc(w.mesh_allocs, &w.V, 3 * w.cap_v, s->device, stream));
        FE_CUDA(dalloc(w.mesh_allocs, &w.N, 3 * w.cap_v, s->device, stream));
        FE_CUDA(dalloc(w.mesh_allocs, &w.T, 4 * w.cap_t, s->device, stream));
    }
    FE_CUDA(launch_mc_emit(v, msdf, w.cfg, w.vbase, w.tbase, w.V, w.N, w.T, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    w.nv = tot[0];
    w.nt = tot[1];
    w.built = true;
    if (n_vertices) *n_vertices = w.nv;
    if (n_triangles) *n_triangles = w.nt;
    return FE_OK;
}

fe_status fe_scene_get_surface(fe_scene* s, double* vertices, double* normals, int64_t* triangles)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->surf.built) return set_error(FE_ERR_STATE, "build the surface first (fe_scene_build_surface)");
    FE_CUDA(cudaSetDevice(s->device));
    auto& w = s->surf;
    if (vertices && w.nv) FE_CUDA(cudaMemcpyAsync(vertices, w.V, 3 * w.nv * sizeof(double), cudaMemcpyDefault, s->stream));
    if (normals && w.nv) FE_CUDA(cudaMemcpyAsync(normals, w.N, 3 * w.nv * sizeof(double), cudaMemcpyDefault, s->stream));
    if (triangles && w.nt) FE_CUDA(cudaMemcpyAsync(triangles, w.T, 4 * w.nt * sizeof(int64_t), cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_write_surface_obj(fe_scene* s, const char* path, const char* object_name)
{
    if (!s || !path) return set_error(FE_ERR_BAD_ARG, "null argument");
    uint64_t nv = 0, nt = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->surf.built) return set_error(FE_ERR_STATE, "build the surface first (fe_scene_build_surface)");
        nv = s->surf.nv;
        nt = s->surf.nt;
    }
    std::vector<double> V(3 * nv), N(3 * nv);
    std::vector<int64_t> T(4 * nt);
    fe_status st = fe_scene_get_surface(s, V.data(), N.data(), T.data());
    if (st != FE_OK) return st;
    return fe_write_obj(path, object_name, V.data(), N.data(), nv, T.data(), nt);
}

fe_status fe_scene_set_viscosity(fe_scene* s, double viscosity)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    if (!(viscosity >= 0.0) || !std::isfinite(viscosity))
        return set_error(FE_ERR_BAD_ARG, "viscosity must be finite and >= 0");
    std::lock_guard<std::mutex> lk(s->mu);
    if (viscosity > 0.0 && s->colliders.count > 0)
        return set_error(FE_ERR_BAD_ARG, "viscosity with colliders is not supported (BackwardEulerDiffusionSolver's "
                                         "BOUNDRY faces); clear the colliders first");
    FE_CUDA(cudaSetDevice(s->device));
    if (viscosity > 0.0 && !s->diff_ready) {
        FE_CUDA(cudaStreamSynchronize(s->stream));
        fe_status st = alloc_diffusion(s);
        if (st != FE_OK) return st;
    }
    if ((viscosity > 0.0) != (s->desc.viscosity > 0.0) || viscosity != s->desc.viscosity) {
        drop_graphs(s);  // the captured substeps hold the old sequence / coefficients
        ++s->epoch;
    }
    s->desc.viscosity = viscosity;
    return FE_OK;
}

fe_status fe_scene_get_diffusion(fe_scene* s, int32_t* iterations, uint8_t* mu, uint8_t* mv, uint8_t* mw)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    if (!s->diff_ready) return set_error(FE_ERR_STATE, "the scene has never had a viscosity > 0");
    const int nx = s->base.g.nx, ny = s->base.g.ny, nz = s->base.g.nz;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nv = (size_t)nx * (ny + 1) * nz, nw = (size_t)nx * ny * (nz + 1);
    if (iterations) FE_CUDA(cudaMemcpyAsync(iterations, s->diff.its, 4 * sizeof(int32_t), cudaMemcpyDefault, s->stream));
    if (mu) FE_CUDA(cudaMemcpyAsync(mu, s->diff.mark, nu, cudaMemcpyDefault, s->stream));
    if (mv) FE_CUDA(cudaMemcpyAsync(mv, s->diff.mark + nu, nv, cudaMemcpyDefault, s->stream));
    if (mw) FE_CUDA(cudaMemcpyAsync(mw, s->diff.mark + nu + nv, nw, cudaMemcpyDefault, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_get_sort(fe_scene* s, uint32_t* keys, uint32_t* perm, uint64_t n)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    if (n != s->base.np) return set_error(FE_ERR_BAD_ARG, "particle count mismatch");
    if (!n) return FE_OK;
    FE_CUDA(cudaSetDevice(s->device));
    SceneView v = view_of(s, s->parity);
    const unsigned nb = (unsigned)((n + 255) / 256);
    if (keys) {
        k_sorted_keys<<<nb, 256, 0, s->stream>>>(v, s->staging_u32);
        count_launch();
        FE_CUDA(cudaMemcpyAsync(keys, s->staging_u32, n * 4, cudaMemcpyDefault, s->stream));
        FE_CUDA(cudaStreamSynchronize(s->stream));
    }
    if (perm) {
        // slot -> particle id (the ids the particles carried before the last sort)
        SceneView prev = view_of(s, s->parity ^ 1);
        k_perm_ids<<<nb, 256, 0, s->stream>>>(v.rank, prev.pid, s->staging_u32, n);
        count_launch();
        FE_CUDA(cudaMemcpyAsync(perm, s->staging_u32, n * 4, cudaMemcpyDefault, s->stream));
    }
    FE_CUDA(cudaStreamSynchronize(s->stream));
    return FE_OK;
}

fe_status fe_scene_divergence(fe_scene* s, double* l2)
{
    if (!s || !l2) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    FE_CUDA(ensure_grid(s, 0));
    FE_CUDA(launch_divergence(s->base, s->d_scalar, s->stream));
    double acc = 0;
    FE_CUDA(cudaMemcpyAsync(&acc, s->d_scalar, sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    FE_CUDA(cudaStreamSynchronize(s->stream));
    *l2 = std::sqrt(acc);
    return FE_OK;
}

}  // extern "C"

// A scene's simulation state at a substep boundary, on the device: the particles in slot order (every channel and
// the identity permutation), the positions at the start of the last substep (the fluid surface's SDF is built
// from them), the pressure warm start, the current velocity grid (the next frame's CFL reads it) and the host-side
// flags and counters that steer the next substeps.
struct fe_snapshot {
    int device = 0;
    int n[3] = {0, 0, 0};
    int solver = 0;
    uint64_t np = 0;
    std::vector<void*> allocs;
    float* part = nullptr;    // channels x np floats (pos 3, vel 3, C 9 for APIC), then pid (np u32)
    float* prev = nullptr;    // 3 x np: positions at the start of the last substep (when prev_valid)
    double* p = nullptr;      // nc
    double* pprev = nullptr;  // nc: the pressure before that (time-extrapolated warm start), when in use
    float* grid = nullptr;    // nf: the current velocity buffer
    int channels = 0;
    bool prev_valid = false, collider_built = false, last_substep_empty = false, have_particles = false;
    std::vector<uint64_t> emitter_calls;
    uint64_t bytes = 0;
};

extern "C" {

fe_status fe_scene_snapshot(fe_scene* s, fe_snapshot** out)
{
    TraceRange trace("fe_scene_snapshot");
    if (!s || !out) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    const SceneView& b = s->base;
    const size_t nc = (size_t)b.g.nx * b.g.ny * b.g.nz;
    const size_t nf = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz + (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz +
                      (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
    std::unique_ptr<fe_snapshot> sn(new fe_snapshot);
    sn->device = s->device;
    sn->n[0] = b.g.nx;
    sn->n[1] = b.g.ny;
    sn->n[2] = b.g.nz;
    sn->solver = s->desc.solver;
    sn->np = b.np;
    sn->channels = 6 + (s->desc.solver == FE_SOLVER_APIC ? 9 : 0);
    sn->prev_valid = s->prev_valid;
    sn->collider_built = s->collider_built;
    sn->last_substep_empty = s->last_substep_empty;
    sn->have_particles = s->have_particles;
    for (const auto& e : s->emitters) sn->emitter_calls.push_back(e.calls);
    cudaStream_t st = s->stream;
    const int dev = s->device;
    const size_t np = b.np;
    FE_CUDA(dalloc(sn->allocs, &sn->p, nc, dev, st));
    FE_CUDA(dalloc(sn->allocs, &sn->grid, nf, dev, st));
    FE_CUDA(cudaMemcpyAsync(sn->p, b.p, nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
    FE_CUDA(cudaMemcpyAsync(sn->grid, s->grid_cur ? b.u2 : b.u, nf * sizeof(float), cudaMemcpyDeviceToDevice, st));
    sn->bytes = nc * sizeof(double) + nf * sizeof(float);
    if (s->pprev_buf) {
        FE_CUDA(dalloc(sn->allocs, &sn->pprev, nc, dev, st));
        FE_CUDA(cudaMemcpyAsync(sn->pprev, s->pprev_buf, nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
        sn->bytes += nc * sizeof(double);
    }
    if (np) {
        const SceneView v = view_of(s, s->parity);
        FE_CUDA(dalloc(sn->allocs, &sn->part, np * (sn->channels + 1), dev, st));
        const float* ch[15] = {v.px, v.py, v.pz, v.vx, v.vy, v.vz};
        for (int a = 0; a < 9; ++a) ch[6 + a] = v.c[a];
        for (int k = 0; k < sn->channels; ++k)
            FE_CUDA(cudaMemcpyAsync(sn->part + k * np, ch[k], np * sizeof(float), cudaMemcpyDeviceToDevice, st));
        FE_CUDA(cudaMemcpyAsync(sn->part + sn->channels * np, v.pid, np * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                st));
        sn->bytes += np * (sn->channels + 1) * sizeof(float);
        if (s->prev_valid) {
            const SceneView o = view_of(s, s->parity ^ 1);
            FE_CUDA(dalloc(sn->allocs, &sn->prev, 3 * np, dev, st));
            const float* pc[3] = {o.px, o.py, o.pz};
            for (int k = 0; k < 3; ++k)
                FE_CUDA(cudaMemcpyAsync(sn->prev + k * np, pc[k], np * sizeof(float), cudaMemcpyDeviceToDevice, st));
            sn->bytes += 3 * np * sizeof(float);
        }
    }
    FE_CUDA(cudaStreamSynchronize(st));
    *out = sn.release();
    return FE_OK;
}

fe_status fe_scene_restore(fe_scene* s, const fe_snapshot* sn)
{
    TraceRange trace("fe_scene_restore");
    if (!s || !sn) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    const SceneView& b0 = s->base;
    if (sn->device != s->device || sn->n[0] != b0.g.nx || sn->n[1] != b0.g.ny || sn->n[2] != b0.g.nz ||
        sn->solver != s->desc.solver)
        return set_error(FE_ERR_BAD_ARG, "snapshot of another grid, solver or device");
    if (sn->emitter_calls.size() != s->emitters.size())
        return set_error(FE_ERR_BAD_ARG, "snapshot taken with %zu emitters, scene has %zu", sn->emitter_calls.size(),
                         s->emitters.size());
    FE_CUDA(cudaSetDevice(s->device));
    const size_t np = sn->np;
    if (np > s->cap || !s->set[0].px) {
        FE_CUDA(cudaStreamSynchronize(s->stream));
        fe_status st = alloc_particles(s, std::max<uint64_t>(np, 1));
        if (st != FE_OK) return st;
    }
    if (np != s->base.np) drop_graphs(s);
    const SceneView& b = s->base;
    const size_t nc = (size_t)b.g.nx * b.g.ny * b.g.nz;
    const size_t nf = (size_t)(b.g.nx + 1) * b.g.ny * b.g.nz + (size_t)b.g.nx * (b.g.ny + 1) * b.g.nz +
                      (size_t)b.g.nx * b.g.ny * (b.g.nz + 1);
    cudaStream_t st = s->stream;
    s->base.np = np;
    s->parity = 0;
    s->grid_cur = 0;
    FE_CUDA(cudaMemcpyAsync(b.p, sn->p, nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
    FE_CUDA(cudaMemcpyAsync(b.u, sn->grid, nf * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (s->pprev_buf) {
        if (sn->pprev)
            FE_CUDA(cudaMemcpyAsync(s->pprev_buf, sn->pprev, nc * sizeof(double), cudaMemcpyDeviceToDevice, st));
        else
            FE_CUDA(cudaMemsetAsync(s->pprev_buf, 0, nc * sizeof(double), st));
    }
    if (np) {
        const SceneView v = view_of(s, 0);
        float* ch[15] = {v.px, v.py, v.pz, v.vx, v.vy, v.vz};
        for (int a = 0; a < 9; ++a) ch[6 + a] = v.c[a];
        for (int k = 0; k < sn->channels; ++k)
            FE_CUDA(cudaMemcpyAsync(ch[k], sn->part + k * np, np * sizeof(float), cudaMemcpyDeviceToDevice, st));
        FE_CUDA(cudaMemcpyAsync(v.pid, sn->part + sn->channels * np, np * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                                st));
        if (sn->prev) {
            const SceneView o = view_of(s, 1);
            float* pc[3] = {o.px, o.py, o.pz};
            for (int k = 0; k < 3; ++k)
                FE_CUDA(cudaMemcpyAsync(pc[k], sn->prev + k * np, np * sizeof(float), cudaMemcpyDeviceToDevice, st));
        }
    }
    FE_CUDA(cudaStreamSynchronize(st));
    s->prev_valid = sn->prev_valid && sn->prev;
    s->collider_built = sn->collider_built;
    s->last_substep_empty = sn->last_substep_empty;
    s->have_particles = sn->have_particles;
    s->mesh_sdf = false;
    for (size_t i = 0; i < s->emitters.size(); ++i) s->emitters[i].calls = sn->emitter_calls[i];
    return FE_OK;
}

fe_status fe_snapshot_info(const fe_snapshot* sn, uint64_t* particles, uint64_t* bytes)
{
    if (!sn) return set_error(FE_ERR_BAD_ARG, "null snapshot");
    if (particles) *particles = sn->np;
    if (bytes) *bytes = sn->bytes;
    return FE_OK;
}

fe_status fe_snapshot_destroy(fe_snapshot* sn)
{
    if (!sn) return FE_OK;
    cudaSetDevice(sn->device);
    for (void* p : sn->allocs) cudaFreeAsync(p, 0);
    cudaStreamSynchronize(0);
    delete sn;
    return FE_OK;
}

fe_status fe_scene_set_tuning(fe_scene* s, const fe_tuning* t)
{
    if (!s || !t) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    return apply_tuning(s, t);
}

fe_status fe_scene_get_tuning(fe_scene* s, fe_tuning* t)
{
    if (!s || !t) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    t->multigrid = s->use_mg && s->mg.levels >= 2 && s->colliders.count == 0 ? 1 : 0;
    t->cg_block_threads = s->cg.threads;
    t->mg_block_level_cells = s->mg_block_cells;
    t->cg_cluster = std::max(s->cg.cluster, 1);
    t->pressure_extrapolation = s->base.pprev ? 1 : 0;
    return FE_OK;
}

fe_status fe_tuning_store(int32_t device, const int32_t n[3], int32_t solver, const fe_tuning* t)
{
    if (!n || !t) return set_error(FE_ERR_BAD_ARG, "null argument");
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[TuneKey{device, n[0], n[1], n[2], solver}] = *t;
    return FE_OK;
}

fe_status fe_tuning_lookup(int32_t device, const int32_t n[3], int32_t solver, fe_tuning* t)
{
    if (!n || !t) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (!tuning_lookup(device, n[0], n[1], n[2], solver, t)) return set_error(FE_ERR_STATE, "no tuning stored");
    return FE_OK;
}

fe_status fe_scene_autotune(fe_scene* s, double dt, int32_t substeps, int32_t scope, fe_tuning* best, float* best_ms)
{
    TraceRange trace("fe_scene_autotune");
    if (!s || !(dt > 0.0) || substeps < 1 || scope < FE_TUNE_ALL || scope > FE_TUNE_SHAPE)
        return set_error(FE_ERR_BAD_ARG, "bad autotune arguments");
    if (!s->have_particles || s->base.np == 0) return set_error(FE_ERR_STATE, "autotune needs particles");
    // candidates: the plain CG at 256 / 512 / 1024 threads per block and, where the grid has a multigrid hierarchy
    // and no colliders, the multigrid-preconditioned CG at 512 / 1024 threads with one-block levels up to 2048 or
    // 4096 cells
    fe_tuning before;
    fe_status st = fe_scene_get_tuning(s, &before);
    if (st != FE_OK) return st;
    std::vector<fe_tuning> cand;
    MgLevel lv[kMaxMgLevels];
    const SceneView& b = s->base;
    const bool mg_ok = mg_plan(b.g.nx, b.g.ny, b.g.nz, b.h, lv) >= 2 && s->colliders.count == 0;
    if (scope == FE_TUNE_ALL || before.multigrid == 0)
        for (int th : {1024, 512, 256})
            for (int cl : {1, 2}) cand.push_back(fe_tuning{0, th, 4096, cl, -1});
    if (mg_ok && (scope == FE_TUNE_ALL || before.multigrid == 1))
        for (int th : {1024, 512})
            for (int cells : {4096, 2048}) cand.push_back(fe_tuning{1, th, cells, 1, -1});
    fe_snapshot* snap = nullptr;
    st = fe_scene_snapshot(s, &snap);
    if (st != FE_OK) return st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaSetDevice(s->device);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<fe_step_stats> stats((size_t)substeps);
    float best_time = -1.f;
    fe_tuning pick = before;
    for (const fe_tuning& c : cand) {
        if ((st = fe_scene_restore(s, snap)) != FE_OK) break;
        // a choice the device cannot launch (e.g. a cluster shape it does not hold co-resident) is skipped
        if (fe_scene_set_tuning(s, &c) != FE_OK || fe_scene_step(s, dt, 1, nullptr) != FE_OK) {
            cudaGetLastError();
            continue;
        }
        cudaEventRecord(e0, s->stream);
        if (fe_scene_step(s, dt, substeps, stats.data()) != FE_OK) {
            cudaGetLastError();
            continue;
        }
        cudaEventRecord(e1, s->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        bool ok = true;
        for (const auto& x : stats) ok = ok && x.converged == 1;
        if (ok && (best_time < 0.f || ms < best_time)) {
            best_time = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    fe_status st2 = fe_scene_restore(s, snap);
    fe_snapshot_destroy(snap);
    if (st == FE_OK) st = st2;
    if (st == FE_OK) st = fe_scene_set_tuning(s, &pick);
    if (st != FE_OK) {
        fe_scene_set_tuning(s, &before);
        return st;
    }
    fe_scene_get_tuning(s, &pick);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[TuneKey{s->device, b.g.nx, b.g.ny, b.g.nz, s->desc.solver}] = pick;
    }
    if (best) *best = pick;
    if (best_ms) *best_ms = best_time / (float)substeps;
    return FE_OK;
}

fe_status fe_scene_set_stream(fe_scene* s, void* stream)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    s->stream = stream ? (cudaStream_t)stream : s->own_stream;
    return FE_OK;
}

fe_status fe_scene_synchronize(fe_scene* s)
{
    if (!s) return set_error(FE_ERR_BAD_ARG, "null scene");
    std::lock_guard<std::mutex> lk(s->mu);
    FE_CUDA(cudaSetDevice(s->device));
    return check_device_error(s);
}

uint64_t fe_kernel_launch_count(void) { return g_launches.load(); }

fe_status fe_debug_set_barrier_limits(uint64_t spin_limit, uint32_t extra_arrivals)
{
    if (extra_arrivals > 1024u) return set_error(FE_ERR_BAD_ARG, "extra_arrivals must be at most 1024");
    FE_CUDA(set_solver_barrier_limits((unsigned long long)spin_limit, (unsigned)extra_arrivals));
    return FE_OK;
}

uint64_t fe_seed_regions(const void* regions, int32_t nregions, const int32_t n[3], const double origin[3],
                         const double size[3], uint64_t seed, float* pos, float* vel, uint64_t cap)
{
    if (!regions || nregions <= 0 || !n || !origin || !size) return 0;
    const int nn[3] = {n[0], n[1], n[2]};
    const double h[3] = {size[0] / n[0], size[1] / n[1], size[2] / n[2]};
    return fe_seed_regions_host((const fe_region*)regions, nregions, nn, origin, h, seed, pos, vel, cap);
}

const char* fe_last_error(void) { return g_err; }

int32_t fe_abi_version(void) { return 10600; }

}  // extern "C"

// ------------------------------------------------------------------------------------------- batches
//
// A batch advances many independent scenes together: per substep, every scene's pre-solve phase runs on
// its own stream, ONE cooperative launch solves all scenes' pressure systems (k_multi_cg: each scene on its
// own block range with its own barrier, so scenes iterate independently and concurrently), and every
// scene's post-solve phase runs on its own stream again.  The whole batch substep is captured as one CUDA
// graph (fork/join across the scenes' streams) per particle-buffer parity and replayed.

// Scenes of at most this many cells join a batch's flat launches (fe_batch_set_flat).  Off by default: on the B200 the
// per-scene form measured as fast or faster -- the scenes' passes on their own streams run concurrently, so one
// scene's latency-bound pass overlaps another's bandwidth-bound one, while a flat launch runs one kind of pass at a
// time for all scenes (48 scenes of 32^3..128^3: 10.45 ms per substep per-scene, 10.57 with scenes up to 48^3
// flat, 12.44 all flat; 64 scenes of 24^3..48^3: 2.94 against 2.98).  autotune.tune_batch picks it per batch.
constexpr int64_t kFlatMaxCellsDefault = 0;

struct fe_batch {
    std::vector<fe_scene*> scenes;
    int device = 0;
    cudaStream_t stream = nullptr;
    MultiCgScene* table = nullptr;     // device copy of the per-scene solver table
    int total_blocks = 0;
    std::vector<void*> allocs;
    std::vector<cudaEvent_t> events;   // 2 per scene + 2
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    uint64_t graph_kernels[2] = {0, 0};
    double graph_dt = -1.0;
    uint64_t graph_epoch = 0;  // sum of the scenes' epochs when the graphs were captured
    int parity = 0;
    int64_t steps_done = 0;   // substeps since creation: a young batch replays per-scene graphs
    // overlap mode: every scene runs its whole substep (pre-solve, its own cooperative solve on `share` blocks,
    // post-solve) on its own stream, so one scene's latency-bound solve overlaps other scenes' transfer kernels;
    // the shares add up to the multi-scene solve's co-resident capacity, so all solves in flight fit at once
    bool overlap = false;
    bool shares_measured = false;      // shares re-split from measured solve work since the membership was set
    std::vector<int> share;
    // flat launches: every transfer and grid pass of a substep launched once for all flat members over a (scene,
    // block) work list (BatchPlan, fe_internal.cuh), one device plan per batch parity, on the batch stream, while the
    // other scenes run their passes on their own streams
    int64_t flat_max_cells = kFlatMaxCellsDefault;  // scenes up to this many cells run in the flat launches
    std::vector<int> flat_members;   // indices (into scenes) of the scenes in the flat launches, in plan order
    BatchPlan* plan_dev[2] = {nullptr, nullptr};
    BatchLaunch launch[2] = {};
    bool plan_valid = false;
    double plan_dt = -1.0;
    uint64_t plan_epoch = 0;
    int plan_bparity = 0;             // the batch parity the scene parities below were recorded at
    std::vector<int> plan_parity;     // each scene's particle parity at that batch parity
};

// A batch replays its scenes' own phase graphs around the multi-scene solve for its first
// kBatchCaptureAfter substeps (creating a batch then costs no capture, which is what a server with
// changing membership needs); after that the whole batch substep is captured as one graph.
constexpr int64_t kBatchCaptureAfter = 8;

namespace {

// A scene can run in the flat launches when its substep is the plain sequence those launches implement.
bool flat_scene_ok(const fe_scene* s)
{
    return s->desc.viscosity <= 0.0 && s->forces.count == 0 && s->colliders.count == 0 && s->emitters.empty();
}

bool flat_member(const fe_batch* b, const fe_scene* s)
{
    const int64_t cells = (int64_t)s->base.g.nx * s->base.g.ny * s->base.g.nz;
    return !b->overlap && flat_scene_ok(s) && (b->flat_max_cells < 0 || cells <= b->flat_max_cells);
}

// Recomputes the flat members (after a membership or mode change).
void batch_set_flat_members(fe_batch* b)
{
    b->flat_members.clear();
    for (int i = 0; i < (int)b->scenes.size(); ++i)
        if (flat_member(b, b->scenes[i])) b->flat_members.push_back(i);
    b->plan_valid = false;
}

bool batch_flat(const fe_batch* b) { return !b->flat_members.empty(); }
bool is_flat(const fe_batch* b, int i)
{
    return std::binary_search(b->flat_members.begin(), b->flat_members.end(), i);
}

uint64_t batch_epoch(const fe_batch* b)
{
    uint64_t epoch = 0;
    for (const fe_scene* s : b->scenes) epoch += s->epoch;
    return epoch;
}

// The flat plans of both batch parities for the current membership, scene parities and dt (copied to the device
// after the batch stream has drained, so no launch of an earlier plan can still read it).  No device allocation.
fe_status batch_build_plans(fe_batch* b, double dt)
{
    const int S = (int)b->scenes.size();
    const int F = (int)b->flat_members.size();
    FE_CUDA(cudaStreamSynchronize(b->stream));
    std::unique_ptr<BatchPlan> hp(new (std::nothrow) BatchPlan());
    if (!hp) return set_error(FE_ERR_OOM, "host allocation failed");
    for (int q = 0; q < 2; ++q) {
        BatchPlan& P = *hp;
        std::memset(&P, 0, sizeof(BatchPlan));
        P.count = F;
        BatchLaunch& L = b->launch[q];
        L = BatchLaunch{};
        for (int i = 0; i < F; ++i) {
            fe_scene* s = b->scenes[b->flat_members[i]];
            const int par = s->parity ^ q ^ b->parity;
            BatchScene& e = P.sc[i];
            e.src = view_of(s, par);
            e.dst = view_of(s, par ^ 1);
            const SceneView& v = e.dst;
            const uint32_t K = v.g.key_space;
            e.scan_blocks = sort_batch_blocks(v, kBkScan);
            if (sort_scan_tmp_bytes(K) > s->scan_tmp_bytes) return set_error(FE_ERR_STATE, "scan scratch too small");
            e.scan_sums = (uint32_t*)s->scan_tmp;
            e.long_count = e.scan_sums + e.scan_blocks + 1;
            const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz,
                         nww = (size_t)v.g.nx * v.g.ny * (v.g.nz + 1), faces = nu + nvv + nww;
            const size_t cells = (size_t)v.g.nx * v.g.ny * v.g.nz;
            int r = 0;
            auto range = [&](void* ptr, uint64_t bytes, uint32_t val) {
                e.clr_ptr[r] = (uint8_t*)ptr;
                e.clr_bytes[r] = bytes;
                e.clr_val[r] = val;
                ++r;
            };
            // launch_sort's count clear, launch_p2g's accumulator clears, launch_mark's mark (and crit) clears: all
            // these buffers are dead between substeps
            range(v.cell_count, (uint64_t)K * sizeof(uint32_t), 0);
            range(v.nu, faces * sizeof(float), 0);
            range(v.du, faces * sizeof(float), 0);
            range(v.mu, faces, 0);
            range(v.marks, cells, FE_CELL_AIR);
            if (v.any_inexact) {
                range(v.crit_flag, (cells + 3) & ~(size_t)3, 0);
                range(v.crit_count, sizeof(uint32_t), 0);
            }
            e.nclr = r;
            uint64_t clear_bytes = 0;
            for (int k = 0; k < r; ++k) clear_bytes += e.clr_bytes[k];
            e.gdt[0] = (float)(dt * v.gravity[0]);
            e.gdt[1] = (float)(dt * v.gravity[1]);
            e.gdt[2] = (float)(dt * v.gravity[2]);
            e.mark = mark_constants(v);
            e.g2p = g2p_args(v, dt);
            for (int k = 0; k < kBkCount; ++k) {
                // a block clears 256 threads x 16 B x 8 per pass of its range loop
                const uint32_t n = k == kBkClear ? (uint32_t)std::max<uint64_t>(1, (clear_bytes + 32767) / 32768)
                                                 : batch_blocks(v, k);
                P.start[k][i + 1] = P.start[k][i] + n;
            }
            L.max_depth = std::max(L.max_depth, v.extrap_depth);
        }
        for (int k = 0; k < kBkCount; ++k) L.total[k] = P.start[k][F];
        L.plan = b->plan_dev[q];
        FE_CUDA(cudaMemcpy(b->plan_dev[q], &P, sizeof(BatchPlan), cudaMemcpyHostToDevice));
    }
    b->plan_parity.resize(S);
    for (int i = 0; i < S; ++i) b->plan_parity[i] = b->scenes[i]->parity;
    b->plan_bparity = b->parity;
    b->plan_dt = dt;
    b->plan_epoch = batch_epoch(b);
    b->plan_valid = true;
    return FE_OK;
}

// True when the plans match the batch's current state (membership, dt, scene epochs and particle parities).
bool batch_plans_current(const fe_batch* b, double dt)
{
    if (!b->plan_valid || b->plan_dt != dt || b->plan_epoch != batch_epoch(b)) return false;
    const int flip = b->parity ^ b->plan_bparity;
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->scenes[i]->parity != (b->plan_parity[i] ^ flip)) return false;
    return true;
}

// The flat members' pre-solve passes on the batch stream: the clears, the sort and gather, P2G, marking, the pre
// group and the right-hand side, each one launch for all of them.
fe_status batch_flat_pre(fe_batch* b)
{
    if (!batch_flat(b)) return FE_OK;
    const BatchLaunch& L = b->launch[b->parity];
    cudaStream_t st = b->stream;
    FE_CUDA(launch_multi_clear(L, st));
    FE_CUDA(launch_multi_sort(L, st));
    FE_CUDA(launch_multi_p2g(L, st));
    FE_CUDA(launch_multi_mark(L, st));
    FE_CUDA(launch_multi_pre(L, st));
    FE_CUDA(launch_multi_rhs(L, st));
    return FE_OK;
}

// The flat members' post-solve passes on the batch stream: the pressure apply, the post group and the transfer +
// move.
fe_status batch_flat_post(fe_batch* b)
{
    if (!batch_flat(b)) return FE_OK;
    const BatchLaunch& L = b->launch[b->parity];
    cudaStream_t st = b->stream;
    FE_CUDA(launch_multi_apply(L, st));
    FE_CUDA(launch_multi_post(L, st));
    FE_CUDA(launch_multi_g2p(L, st));
    return FE_OK;
}

// Host bookkeeping after a batch substep was enqueued: every scene's sort flipped its particle buffer sets.
void batch_after_substep(fe_batch* b)
{
    for (fe_scene* s : b->scenes) {
        s->parity ^= 1;
        s->prev_valid = true;
        s->mesh_sdf = false;
        s->collider_built = true;
        s->grid_cur = 0;
    }
    b->parity ^= 1;
}

void batch_drop_graphs(fe_batch* b)
{
    for (int i = 0; i < 2; ++i)
        if (b->graph[i]) {
            cudaGraphExecDestroy(b->graph[i]);
            b->graph[i] = nullptr;
        }
    b->graph_dt = -1.0;
}

// The pre-solve steps of a scene with viscosity run on the batch's stream, one scene after another, so that no
// two cooperative Jacobi kernels (fe_diffuse.cu) are ever in flight together; the other scenes' pre-solve steps
// run concurrently on their own streams.
cudaStream_t pre_stream(const fe_batch* b, const fe_scene* s) { return s->desc.viscosity > 0.0 ? b->stream : s->stream; }

// One batch substep on b->stream: the scenes outside the flat launches run their pre-solve passes on their own
// streams (forked from the batch stream; viscous scenes one after another on the batch stream), concurrently with the
// flat launches of the flat members on the batch stream; all join before the multi-scene solve; then the same for
// the post-solve passes.  scene_graphs replays the forked scenes' own phase graphs (young batches, profiled steps);
// otherwise their steps are enqueued directly (the batch graph's capture).  The flat plans must be current.  `ev`
// (optional) gets events before, between and after the three phases.
fe_status batch_enqueue_mixed(fe_batch* b, double dt, bool scene_graphs, cudaEvent_t* ev)
{
    const int S = (int)b->scenes.size();
    cudaEvent_t fork0 = b->events[2 * S], fork1 = b->events[2 * S + 1];
    if (ev) FE_CUDA(cudaEventRecord(ev[0], b->stream));
    FE_CUDA(cudaEventRecord(fork0, b->stream));
    auto pre = [&](fe_scene* s, cudaStream_t ps) -> fe_status {
        if (!scene_graphs) return enqueue_steps(s, dt, kStepSort, kStepRhs, ps);
        FE_CUDA(cudaGraphLaunch(s->graph[s->parity][0], ps));
        g_launches += s->graph_kernels[s->parity][0];
        return FE_OK;
    };
    // forked scenes first, then the viscous ones and the flat launches on the batch stream, then the joins (a join
    // enqueued earlier would make the batch stream's work wait for the forked scenes)
    for (int i = 0; i < S; ++i) {
        fe_scene* s = b->scenes[i];
        const cudaStream_t ps = pre_stream(b, s);
        if (is_flat(b, i) || ps == b->stream) continue;
        FE_CUDA(cudaStreamWaitEvent(ps, fork0, 0));
        fe_status st = pre(s, ps);
        if (st != FE_OK) return st;
        FE_CUDA(cudaEventRecord(b->events[2 * i], ps));
    }
    for (int i = 0; i < S; ++i) {
        fe_scene* s = b->scenes[i];
        if (is_flat(b, i) || pre_stream(b, s) != b->stream) continue;
        fe_status st = pre(s, b->stream);
        if (st != FE_OK) return st;
    }
    fe_status st = batch_flat_pre(b);
    if (st != FE_OK) return st;
    for (int i = 0; i < S; ++i)
        if (!is_flat(b, i) && pre_stream(b, b->scenes[i]) != b->stream)
            FE_CUDA(cudaStreamWaitEvent(b->stream, b->events[2 * i], 0));
    if (ev) FE_CUDA(cudaEventRecord(ev[1], b->stream));
    FE_CUDA(launch_multi_cg(b->table, S, b->total_blocks, b->stream));
    if (ev) FE_CUDA(cudaEventRecord(ev[2], b->stream));
    FE_CUDA(cudaEventRecord(fork1, b->stream));
    for (int i = 0; i < S; ++i) {
        if (is_flat(b, i)) continue;
        fe_scene* s = b->scenes[i];
        FE_CUDA(cudaStreamWaitEvent(s->stream, fork1, 0));
        if (scene_graphs) {
            FE_CUDA(cudaGraphLaunch(s->graph[s->parity][2], s->stream));
            g_launches += s->graph_kernels[s->parity][2];
        } else {
            st = enqueue_steps(s, dt, kStepApply, kStepMove);
            if (st != FE_OK) return st;
        }
        FE_CUDA(cudaEventRecord(b->events[2 * i + 1], s->stream));
    }
    st = batch_flat_post(b);
    if (st != FE_OK) return st;
    for (int i = 0; i < S; ++i)
        if (!is_flat(b, i)) FE_CUDA(cudaStreamWaitEvent(b->stream, b->events[2 * i + 1], 0));
    if (ev) FE_CUDA(cudaEventRecord(ev[3], b->stream));
    return FE_OK;
}

// Enqueues one batch substep on b->stream (the batch graph's capture).
fe_status batch_enqueue(fe_batch* b, double dt) { return batch_enqueue_mixed(b, dt, false, nullptr); }

// One batch substep launched directly: the forked scenes' own captured phase graphs (pre-solve and post-solve,
// captured once per scene and dt) and the flat launches around the multi-scene solve.
fe_status batch_step_scene_graphs(fe_batch* b, double dt, cudaEvent_t* ev = nullptr)
{
    const int S = (int)b->scenes.size();
    if (batch_flat(b) && !batch_plans_current(b, dt)) {
        fe_status st = batch_build_plans(b, dt);
        if (st != FE_OK) return st;
    }
    for (int i = 0; i < S; ++i) {
        if (is_flat(b, i)) continue;
        fe_scene* s = b->scenes[i];
        if (s->graph_dt != dt) {
            drop_graphs(s);
            s->graph_dt = dt;
        }
        if (!s->graph[s->parity][0]) {
            fe_status st = capture_graphs(s, s->parity, dt);
            if (st != FE_OK) return st;
        }
    }
    fe_status st = batch_enqueue_mixed(b, dt, true, ev);
    if (st != FE_OK) return st;
    batch_after_substep(b);  // every scene's sort flipped its particle buffer sets
    return FE_OK;
}

fe_status batch_enqueue_overlap(fe_batch* b, double dt, bool scene_graphs);

// Overlap mode's young-batch substep: the scenes' own phase graphs around each scene's own solve.
fe_status batch_step_overlap_scene_graphs(fe_batch* b, double dt)
{
    for (fe_scene* s : b->scenes) {
        if (s->graph_dt != dt) {
            drop_graphs(s);
            s->graph_dt = dt;
        }
        if (!s->graph[s->parity][0]) {
            fe_status st = capture_graphs(s, s->parity, dt);
            if (st != FE_OK) return st;
        }
    }
    fe_status st = batch_enqueue_overlap(b, dt, true);
    if (st != FE_OK) return st;
    for (fe_scene* s : b->scenes) {
        s->parity ^= 1;  // the pre-solve graph's sort flipped the particle buffer sets
        s->prev_valid = true;
        s->mesh_sdf = false;
        s->collider_built = true;
        s->grid_cur = 0;
    }
    b->parity ^= 1;
    return FE_OK;
}

fe_status batch_check_scenes(fe_scene* const* scenes, int32_t count)
{
    if (!scenes || count < 1) return set_error(FE_ERR_BAD_ARG, "need at least one scene");
    if (count > kBatchMaxScenes) return set_error(FE_ERR_BAD_ARG, "at most %d scenes per batch", kBatchMaxScenes);
    for (int i = 0; i < count; ++i) {
        if (!scenes[i]) return set_error(FE_ERR_BAD_ARG, "null scene %d", i);
        if (scenes[i]->device != scenes[0]->device)
            return set_error(FE_ERR_BAD_ARG, "all scenes of a batch must share a device");
        if (!scenes[i]->have_particles) return set_error(FE_ERR_STATE, "scene %d has no particles", i);
        if (!scenes[i]->emitters.empty())
            return set_error(FE_ERR_BAD_ARG, "scene %d has emitters (its particle count changes every substep): step it alone", i);
        if (scenes[i]->colliders.count > 0)
            return set_error(FE_ERR_BAD_ARG, "scene %d has colliders: step it alone", i);
        for (int j = 0; j < i; ++j)
            if (scenes[j] == scenes[i]) return set_error(FE_ERR_BAD_ARG, "scene %d appears twice", i);
    }
    return FE_OK;
}

// Sets the batch's scenes: the solver table (in the table allocated once for kBatchMaxScenes entries) with
// each scene's first block split, join events, and no captured graphs (the next substeps replay the scenes'
// own phase graphs until the batch graph is captured again).  No device allocation.
fe_status batch_set_members(fe_batch* b, fe_scene* const* scenes, int32_t count)
{
    // Solver blocks per scene before its first solve, proportional to its expected solve work (particle
    // count as a proxy for its FLUID cells x grid extent, as CG iterations grow with the extent), at least
    // one block each; before every later solve k_multi_partition re-splits the blocks by the scenes'
    // measured work.  The multi-scene launch fills the device's co-resident capacity.
    int capacity = 0, threads = 0;
    cudaError_t e = multi_cg_capacity(b->device, &capacity, &threads);
    if (e != cudaSuccess) return cuda_check(e, "multi-scene occupancy");
    capacity = std::min(capacity, kMaxCgBlocks);
    if (capacity < count) return set_error(FE_ERR_BAD_ARG, "more scenes than solver blocks (%d)", capacity);
    std::vector<double> work(count);
    double total_work = 0.0;
    for (int i = 0; i < count; ++i) {
        const GridDims& g = scenes[i]->base.g;
        // about np / 8 FLUID cells x about 3 x extent inner iterations, the scale of a measured solve's work
        work[i] = (double)scenes[i]->base.np / 8.0 * 3.0 * (double)std::max(g.nx, std::max(g.ny, g.nz));
        total_work += work[i];
    }
    std::vector<int> nblk(count, 1);
    int used = count;
    for (int i = 0; i < count; ++i) {
        const int extra = (int)std::floor((capacity - count) * work[i] / std::max(total_work, 1.0));
        nblk[i] += extra;
        used += extra;
    }
    for (int k = 0; used < capacity; ++k, ++used) {  // leftovers to the largest scenes
        int best = 0;
        for (int i = 1; i < count; ++i)
            if (work[i] > work[best]) best = i;
        nblk[(best + k) % count] += 1;
    }
    std::vector<MultiCgScene> table(count);
    int start = 0;
    for (int i = 0; i < count; ++i) {
        fe_scene* s = scenes[i];
        MultiCgScene& t = table[i];
        t.view = s->base;
        t.work = s->cg;
        t.work.cluster = 1;  // the multi-scene solve is not a cluster launch
        t.mg = s->mg;
        t.use_mg = s->use_mg && s->mg.levels >= 2 ? 1 : 0;
        t.rel_tol = s->desc.cg_rel_tol;
        t.inner_tol = inner_tol(s->desc, t.use_mg != 0);
        t.max_it = s->desc.cg_max_it;
        t.max_refine = s->desc.max_refine;
        t.block_start = start;
        t.block_count = nblk[i];
        t.last_its = -1;  // no solve yet: k_multi_partition uses weight0
        t.last_fluid = 0;
        t.weight0 = work[i];
        start += nblk[i];
    }
    batch_drop_graphs(b);
    while ((int)b->events.size() < 2 * count + 2) {
        cudaEvent_t ev;
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return cuda_check(e, "event");
        b->events.push_back(ev);
    }
    if ((e = cudaMemcpy(b->table, table.data(), count * sizeof(MultiCgScene), cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_check(e, "batch setup");
    b->scenes.assign(scenes, scenes + count);
    b->total_blocks = start;
    b->steps_done = 0;
    batch_set_flat_members(b);
    b->share = nblk;
    b->shares_measured = false;
    return FE_OK;
}

// Overlap mode: re-splits the solver blocks among the scenes in proportion to their measured solve work (read back
// from the solver table once the batch has run a few substeps), as k_multi_partition does on the device.
fe_status batch_resplit(fe_batch* b)
{
    const int S = (int)b->scenes.size();
    std::vector<MultiCgScene> table(S);
    FE_CUDA(cudaStreamSynchronize(b->stream));
    FE_CUDA(cudaMemcpy(table.data(), b->table, S * sizeof(MultiCgScene), cudaMemcpyDeviceToHost));
    std::vector<double> work(S);
    double total = 0.0;
    for (int i = 0; i < S; ++i) {
        const MultiCgScene& m = table[i];
        const double per_it = m.use_mg ? 12.0 : 1.0;
        work[i] = m.last_its >= 0 ? (double)m.last_fluid * ((double)m.last_its * per_it + 3.0) : m.weight0;
        work[i] = std::max(work[i], 0.0);
        total += work[i];
    }
    std::vector<int> nblk(S, 1);
    int used = S;
    for (int i = 0; i < S; ++i) {
        const int extra = total > 0.0 ? (int)std::floor((b->total_blocks - S) * work[i] / total) : 0;
        nblk[i] += extra;
        used += extra;
    }
    for (; used < b->total_blocks; ++used) {  // leftovers where the work per block is largest
        int best = 0;
        for (int i = 1; i < S; ++i)
            if (work[i] / nblk[i] > work[best] / nblk[best]) best = i;
        nblk[best] += 1;
    }
    b->share = nblk;
    b->shares_measured = true;
    return FE_OK;
}

bool batch_has_viscosity(const fe_batch* b)
{
    return std::any_of(b->scenes.begin(), b->scenes.end(), [](const fe_scene* s) { return s->desc.viscosity > 0.0; });
}

// Overlap mode, one batch substep: each scene's pre-solve steps, its own solve and its post-solve steps on its own
// stream, forked from and joined to the batch stream; scene_graphs replays the scenes' own phase graphs (young
// batches), otherwise the steps are enqueued directly (for the batch graph's capture).
fe_status batch_enqueue_overlap(fe_batch* b, double dt, bool scene_graphs)
{
    const int S = (int)b->scenes.size();
    cudaEvent_t fork0 = b->events[2 * S];
    FE_CUDA(cudaEventRecord(fork0, b->stream));
    for (int i = 0; i < S; ++i) {
        fe_scene* s = b->scenes[i];
        FE_CUDA(cudaStreamWaitEvent(s->stream, fork0, 0));
        if (scene_graphs) {
            FE_CUDA(cudaGraphLaunch(s->graph[s->parity][0], s->stream));
            g_launches += s->graph_kernels[s->parity][0];
        } else {
            fe_status st = enqueue_steps(s, dt, kStepSort, kStepRhs, s->stream);
            if (st != FE_OK) return st;
        }
        FE_CUDA(launch_multi_cg(b->table + i, 1, b->share[i], s->stream));
        if (scene_graphs) {
            FE_CUDA(cudaGraphLaunch(s->graph[s->parity][2], s->stream));
            g_launches += s->graph_kernels[s->parity][2];
        } else {
            fe_status st = enqueue_steps(s, dt, kStepApply, kStepMove);
            if (st != FE_OK) return st;
        }
        FE_CUDA(cudaEventRecord(b->events[2 * i + 1], s->stream));
        FE_CUDA(cudaStreamWaitEvent(b->stream, b->events[2 * i + 1], 0));
    }
    return FE_OK;
}

fe_status batch_capture(fe_batch* b, int parity, double dt)
{
    const int S = (int)b->scenes.size();
    std::vector<int> par(S), grid(S);
    for (int i = 0; i < S; ++i) {
        par[i] = b->scenes[i]->parity;
        grid[i] = b->scenes[i]->grid_cur;
    }
    cudaGraph_t g = nullptr;
    g_capturing = true;
    g_capture_launches = 0;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    const bool overlap = b->overlap && !batch_has_viscosity(b);
    fe_status st = e == cudaSuccess ? (overlap ? batch_enqueue_overlap(b, dt, false) : batch_enqueue(b, dt))
                                    : cuda_check(e, "begin capture");
    cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
    g_capturing = false;
    for (int i = 0; i < S; ++i) {
        b->scenes[i]->parity = par[i];
        b->scenes[i]->grid_cur = grid[i];
    }
    if (st != FE_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e2 != cudaSuccess) return cuda_check(e2, "end capture");
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_check(e, "graph instantiate");
    b->graph[parity] = exec;
    b->graph_kernels[parity] = g_capture_launches;
    return FE_OK;
}

}  // namespace

extern "C" {

fe_status fe_batch_create(fe_scene* const* scenes, int32_t count, fe_batch** out)
{
    if (!out) return set_error(FE_ERR_BAD_ARG, "null argument");
    *out = nullptr;
    fe_status vst = batch_check_scenes(scenes, count);
    if (vst != FE_OK) return vst;
    const int dev = scenes[0]->device;
    FE_CUDA(cudaSetDevice(dev));
    fe_batch* b = new (std::nothrow) fe_batch();
    if (!b) return set_error(FE_ERR_OOM, "host allocation failed");
    b->scenes.assign(scenes, scenes + count);
    b->device = dev;
    auto fail = [&](fe_status st) {
        if (b->stream) free_list(b->allocs, b->stream);
        for (auto e : b->events) cudaEventDestroy(e);
        if (b->stream) cudaStreamDestroy(b->stream);
        delete b;
        return st;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_check(e, "stream create"));
    if ((e = dalloc(b->allocs, &b->table, kBatchMaxScenes, dev, b->stream)) != cudaSuccess ||
        (e = dalloc(b->allocs, &b->plan_dev[0], 1, dev, b->stream)) != cudaSuccess ||
        (e = dalloc(b->allocs, &b->plan_dev[1], 1, dev, b->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
        return fail(cuda_check(e, "batch allocation"));
    fe_status st = batch_set_members(b, scenes, count);
    if (st != FE_OK) return fail(st);
    // no host synchronisation: a scene's earlier work precedes the batch's work in its own stream order
    *out = b;
    return FE_OK;
}

fe_status fe_batch_set_overlap(fe_batch* b, int32_t on)
{
    if (!b) return set_error(FE_ERR_BAD_ARG, "null batch");
    FE_CUDA(cudaSetDevice(b->device));
    FE_CUDA(cudaStreamSynchronize(b->stream));
    if (b->overlap != (on != 0)) {
        b->overlap = on != 0;
        batch_set_flat_members(b);
        batch_drop_graphs(b);
    }
    return FE_OK;
}

fe_status fe_batch_set_flat(fe_batch* b, int64_t max_cells)
{
    if (!b) return set_error(FE_ERR_BAD_ARG, "null batch");
    FE_CUDA(cudaSetDevice(b->device));
    FE_CUDA(cudaStreamSynchronize(b->stream));
    if (b->flat_max_cells != max_cells) {
        b->flat_max_cells = max_cells;
        batch_set_flat_members(b);
        batch_drop_graphs(b);
    }
    return FE_OK;
}

fe_status fe_batch_set_scenes(fe_batch* b, fe_scene* const* scenes, int32_t count)
{
    if (!b) return set_error(FE_ERR_BAD_ARG, "null batch");
    fe_status st = batch_check_scenes(scenes, count);
    if (st != FE_OK) return st;
    if (scenes[0]->device != b->device) return set_error(FE_ERR_BAD_ARG, "all scenes of a batch must share a device");
    FE_CUDA(cudaSetDevice(b->device));
    FE_CUDA(cudaStreamSynchronize(b->stream));  // no solve of the old membership may still read the table
    return batch_set_members(b, scenes, count);
}

fe_status fe_batch_destroy(fe_batch* b)
{
    if (!b) return set_error(FE_ERR_BAD_ARG, "null batch");
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    free_list(b->allocs, b->stream);
    for (auto e : b->events) cudaEventDestroy(e);
    cudaStreamDestroy(b->stream);
    delete b;
    return FE_OK;
}

fe_status fe_batch_step_profiled(fe_batch* b, double dt, int32_t nsub, fe_step_stats* stats, float* phase_ms)
{
    TraceRange trace("fe_batch_step_profiled");
    if (!b || !phase_ms) return set_error(FE_ERR_BAD_ARG, "null argument");
    if (!(dt > 0.0) || nsub < 0) return set_error(FE_ERR_BAD_ARG, "dt must be > 0 and nsub >= 0");
    const int S = (int)b->scenes.size();
    std::vector<std::unique_lock<std::mutex>> locks;
    for (fe_scene* s : b->scenes) locks.emplace_back(s->mu);
    FE_CUDA(cudaSetDevice(b->device));
    if (stats)
        for (fe_scene* s : b->scenes) FE_CUDA(cudaMemsetAsync(s->cg.bar + 2, 0, sizeof(unsigned), b->stream));
    std::vector<cudaEvent_t> ev((size_t)nsub * 4);
    for (auto& e : ev) FE_CUDA(cudaEventCreate(&e));
    fe_status st = FE_OK;
    for (int it = 0; it < nsub && st == FE_OK; ++it) {
        st = batch_step_scene_graphs(b, dt, &ev[(size_t)it * 4]);
        ++b->steps_done;
    }
    if (st == FE_OK) {
        cudaError_t e = cudaStreamSynchronize(b->stream);
        for (int i = 0; i < nsub && e == cudaSuccess; ++i)
            for (int ph = 0; ph < 3 && e == cudaSuccess; ++ph)
                e = cudaEventElapsedTime(&phase_ms[i * 3 + ph], ev[(size_t)i * 4 + ph], ev[(size_t)i * 4 + ph + 1]);
        st = cuda_check(e, "phase timing");
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (st != FE_OK) return st;
    for (fe_scene* s : b->scenes) {
        fe_status cst = check_device_error(s);
        if (cst != FE_OK) return cst;
    }
    if (stats && nsub > 0) {
        const int cnt = std::min(nsub, (int)kStatsRingEntries);
        for (int i = 0; i < S; ++i)
            FE_CUDA(cudaMemcpy(stats + (size_t)i * nsub, b->scenes[i]->stats_ring, cnt * sizeof(fe_step_stats),
                               cudaMemcpyDeviceToHost));
    }
    return FE_OK;
}

fe_status fe_batch_step(fe_batch* b, double dt, int32_t nsub, fe_step_stats* stats)
{
    TraceRange trace("fe_batch_step");
    if (!b) return set_error(FE_ERR_BAD_ARG, "null batch");
    if (!(dt > 0.0) || nsub < 0) return set_error(FE_ERR_BAD_ARG, "dt must be > 0 and nsub >= 0");
    const int S = (int)b->scenes.size();
    std::vector<std::unique_lock<std::mutex>> locks;
    for (fe_scene* s : b->scenes) locks.emplace_back(s->mu);
    FE_CUDA(cudaSetDevice(b->device));
    if (stats)
        for (fe_scene* s : b->scenes) FE_CUDA(cudaMemsetAsync(s->cg.bar + 2, 0, sizeof(unsigned), b->stream));
    const bool overlap = b->overlap && !batch_has_viscosity(b);
    for (int it = 0; it < nsub; ++it) {
        if (b->steps_done < kBatchCaptureAfter || std::any_of(b->scenes.begin(), b->scenes.end(),
                                                                 [](fe_scene* s) { return s->graphs_disabled; })) {
            fe_status st = overlap ? batch_step_overlap_scene_graphs(b, dt) : batch_step_scene_graphs(b, dt);
            if (st != FE_OK) return st;
            ++b->steps_done;
            continue;
        }
        if (overlap && !b->shares_measured) {
            fe_status st = batch_resplit(b);  // the young substeps measured each scene's solve work
            if (st != FE_OK) return st;
            batch_drop_graphs(b);
        }
        const uint64_t epoch = batch_epoch(b);
        if (b->graph_dt != dt || b->graph_epoch != epoch) {
            batch_drop_graphs(b);
            b->graph_dt = dt;
            b->graph_epoch = epoch;
        }
        if (batch_flat(b) && !batch_plans_current(b, dt)) {
            batch_drop_graphs(b);
            b->graph_dt = dt;
            b->graph_epoch = epoch;
            fe_status st = batch_build_plans(b, dt);
            if (st != FE_OK) return st;
        }
        const int par = b->parity;
        if (!b->graph[par]) {
            fe_status st = batch_capture(b, par, dt);
            if (st != FE_OK) return st;
        }
        FE_CUDA(cudaGraphLaunch(b->graph[par], b->stream));
        g_launches += b->graph_kernels[par];
        ++b->steps_done;
        b->parity ^= 1;
        for (fe_scene* s : b->scenes) {
            s->parity ^= 1;
            s->prev_valid = true;
            s->mesh_sdf = false;
            s->collider_built = true;
            s->grid_cur = 0;
        }
    }
    FE_CUDA(cudaStreamSynchronize(b->stream));
    for (fe_scene* s : b->scenes) {
        fe_status st = check_device_error(s);
        if (st != FE_OK) return st;
    }
    if (stats && nsub > 0) {
        const int cnt = std::min(nsub, (int)kStatsRingEntries);
        for (int i = 0; i < S; ++i)
            FE_CUDA(cudaMemcpy(stats + (size_t)i * nsub, b->scenes[i]->stats_ring, cnt * sizeof(fe_step_stats),
                               cudaMemcpyDeviceToHost));
    }
    return FE_OK;
}

}  // extern "C"
