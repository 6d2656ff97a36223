// fe_noalloc.cu -- fe_project_noalloc: the pressure projection without any device allocation.
//
// Who needs this: code that must not call cudaMalloc / cudaFree (or anything that allocates) on the
// path where it projects a velocity field -- for example a host application's per-frame callback or
// a real-time loop where cudaMalloc's implicit device synchronisation would stall the frame, or a caller
// whose device memory is owned by another allocator (a framework's caching allocator or a fixed arena)
// that must not see foreign allocations.  Such callers pass their own device buffers for the inputs and
// outputs; every scratch byte the solver needs lives in one file-scope __device__ array, sized for at
// most kMaxCells cells, which every device that loads the library holds until the process exits.
//
// The array is reached from host code only through cudaGetSymbolAddress: its name in host code is a
// host-side stand-in, not a device address.  The first call on each device (with that device current)
// resolves the address and caches it together with the current context's id; a call that finds a
// different context (after cudaDeviceReset, say) resolves it again.  Make that first call before any
// stream capture begins.  Each call ends by reading the solve's status back and synchronising the
// stream it was given.  All calls on a device share the one array and it keeps the previous call's
// contents: what must start at zero (barrier words, reduction totals, error flag, statistics counter) is
// cleared on the caller's stream at the start of every call, and calls whose work overlaps on the GPU
// (different streams, or host threads issuing concurrently) race on the array -- serialise them on one
// stream.
//
// It runs exactly the kernels of the scene path's pressure stage (K_rhs, the persistent K_cg, K_apply).
#include <cuda.h>

#include <cstring>
#include <mutex>

#include "fe_internal.cuh"

namespace fe {
namespace {

constexpr uint64_t kMaxCells = 1ull << 18;  // e.g. 64^3 cells
constexpr int kMaxBlocks = 1024;            // persistent CG blocks (one per SM)
constexpr int kStatsRing = 4;

// Byte layout of the scratch array (all offsets multiples of 256).
constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffB = 0;                                                        // FP64 rhs
constexpr size_t kOffVec = align256(kOffB + kMaxCells * sizeof(double));          // 9 FP32 CG vectors
constexpr size_t kOffList = align256(kOffVec + 9 * kMaxCells * sizeof(float));     // compacted FLUID list
constexpr size_t kOffPartial = align256(kOffList + kMaxCells * sizeof(uint32_t));  // partials + totals
constexpr size_t kOffBar = align256(kOffPartial + cg_partial_doubles(kMaxBlocks) * sizeof(double));
constexpr size_t kOffErr = align256(kOffBar + kCgBarWords * sizeof(unsigned));
constexpr size_t kOffStats = align256(kOffErr + sizeof(int));
constexpr size_t kScratchBytes = align256(kOffStats + kStatsRing * sizeof(fe_step_stats));

static __device__ __align__(256) unsigned char g_project_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
struct ScratchSlot {
    unsigned long long ctx_id;  // context the address was resolved in (0: not yet)
    unsigned char* base;
    CgWork work;
};
ScratchSlot g_slot[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

// Id of the calling thread's current context (unique for the life of the process), through the driver
// entry points the runtime hands out; 0 when it cannot be told.
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Set-up for `dev` (current): resolves the scratch array's device address and lays the solver's buffers
// out in it; done again when the device's context has changed since.  No allocation.
fe_status scratch_for(int dev, CgWork* out, unsigned char** base_out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    const unsigned long long ctx = current_context_id();
    ScratchSlot& slot = g_slot[dev];
    if (slot.ctx_id == 0 || ctx == 0 || slot.ctx_id != ctx) {
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_project_scratch);
        if (e != cudaSuccess || !ptr) return cuda_check(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress");
        CgWork w{};
        e = cg_prepare(w, dev);
        if (e != cudaSuccess) return cuda_check(e, "cg occupancy");
        if (w.blocks > kMaxBlocks) return set_error(FE_ERR_BAD_ARG, "device has more than %d SMs", kMaxBlocks);
        unsigned char* base = (unsigned char*)ptr;
        float* vec = (float*)(base + kOffVec);
        const size_t n = kMaxCells;
        w.r0 = vec; w.r1 = vec + n; w.w0 = vec + 2 * n; w.w1 = vec + 3 * n;
        w.s0 = vec + 4 * n; w.s1 = vec + 5 * n; w.pv = vec + 6 * n; w.x = vec + 7 * n;
        w.rws0 = reinterpret_cast<float4*>(vec);
        w.rws1 = reinterpret_cast<float4*>(vec + 4 * n);
        w.xcg = vec + 8 * n;
        w.list = (uint32_t*)(base + kOffList);
        w.partial = (double*)(base + kOffPartial);
        w.bar = (unsigned*)(base + kOffBar);
        w.err = (int*)(base + kOffErr);
        w.stats = (fe_step_stats*)(base + kOffStats);
        w.stats_cap = kStatsRing;
        slot.work = w;
        slot.base = base;
        slot.ctx_id = ctx;
    }
    *out = slot.work;
    *base_out = slot.base;
    return FE_OK;
}

}  // namespace
}  // namespace fe

using namespace fe;

extern "C" fe_status fe_project_noalloc(const int32_t n[3], const double h[3], const uint8_t* marks, float* u,
                                        float* v, float* w, double* p, double rel_tol, int32_t max_it,
                                        void* stream, fe_step_stats* stats)
{
    TraceRange trace("fe_project_noalloc");
    if (!n || !h || !marks || !u || !v || !w || !p) return set_error(FE_ERR_BAD_ARG, "null argument");
    for (int a = 0; a < 3; ++a) {
        if (n[a] < 2) return set_error(FE_ERR_BAD_ARG, "grid size must be >= 2 per axis");
        if (!(h[a] > 0.0)) return set_error(FE_ERR_BAD_ARG, "grid spacing must be positive");
    }
    const uint64_t cells = (uint64_t)n[0] * (uint64_t)n[1] * (uint64_t)n[2];
    if (cells > kMaxCells)
        return set_error(FE_ERR_BAD_ARG,
                         "fe_project_noalloc handles at most %llu cells (got %llu); use a scene for larger grids",
                         (unsigned long long)kMaxCells, (unsigned long long)cells);
    if (!(rel_tol > 0.0) || max_it < 1) return set_error(FE_ERR_BAD_ARG, "bad solver settings");
    int dev = 0;
    FE_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(FE_ERR_BAD_ARG, "device ordinal %d unsupported", dev);
    CgWork work;
    unsigned char* base = nullptr;
    fe_status st = scratch_for(dev, &work, &base);
    if (st != FE_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;

    SceneView view;
    memset(&view, 0, sizeof(view));
    view.g.nx = n[0];
    view.g.ny = n[1];
    view.g.nz = n[2];
    for (int a = 0; a < 3; ++a) {
        view.h[a] = h[a];
        view.inv_h[a] = 1.0 / h[a];
    }
    view.extrap_depth = 0;  // the velocity lives in the caller's u, v, w
    view.u = u;
    view.v = v;
    view.w = w;
    view.marks = (uint8_t*)marks;
    view.p = p;
    view.b = (double*)(base + kOffB);

    // barrier words (arrival and exit counts, statistics counter), reduction totals slots and the error
    // flag start at zero on every call
    FE_CUDA(cudaMemsetAsync(work.bar, 0, kCgBarWords * sizeof(unsigned), s));
    FE_CUDA(cudaMemsetAsync(work.partial, 0, kCgTotalsDoubles * sizeof(double), s));
    FE_CUDA(cudaMemsetAsync(work.err, 0, sizeof(int), s));
    FE_CUDA(launch_rhs(view, s));
    FE_CUDA(launch_cg(view, work, rel_tol, 1e-4, max_it, kMaxRefineDefault, s));
    FE_CUDA(launch_apply(view, s));
    int err = 0;
    if (stats) FE_CUDA(cudaMemcpyAsync(stats, work.stats, sizeof(fe_step_stats), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaMemcpyAsync(&err, work.err, sizeof(int), cudaMemcpyDeviceToHost, s));
    FE_CUDA(cudaStreamSynchronize(s));
    if (err) return set_error((fe_status)err, "pressure solve: grid barrier wait exceeded its limit");
    return FE_OK;
}
