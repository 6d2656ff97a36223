// fe_batch_cg.cu -- the pressure solves of many independent scenes in ONE persistent cooperative kernel.
//
// Each scene's system and algorithm are exactly those of the single-scene solver (fe_cg.cu): FP32
// Chronopoulos-Gear CG inside FP64 iterative refinement on the scene's FLUID cells.  What the batch adds
// is a flat work list over all scenes' FLUID cells, one pass per global iteration and ONE grid-wide
// barrier per global iteration carrying every scene's dot products, so S scenes pay the barrier latency
// once instead of S times.  Scenes converge independently: every scene runs its own state machine
//   RESID  r = b - A p (FP64), test ||r|| <= tol ||b||        -> DONE or INIT
//   INIT   w = A r, e = p = s = 0, first dot products         -> ITER
//   ITER   one Chronopoulos-Gear iteration                    -> ITER or UPDATE
//   UPDATE p += e                                             -> RESID
// advancing one phase per global iteration; a DONE scene's entries are skipped, and the kernel returns
// when every scene is DONE (or hit its caps).  All blocks hold identical copies of the per-scene scalars
// because they are computed from the same barrier totals.
#include "fe_internal.cuh"
#include "fe_batch.cuh"

#include <cuda/atomic>

namespace fe {
namespace {

constexpr int kThreads = 1024;
constexpr unsigned long long kSpinLimit = 1ull << 26;

enum : int { kResid = 0, kInit = 1, kIter = 2, kUpdate = 3, kDone = 4 };
enum : uint32_t { kXm = 1, kXp = 2, kYm = 4, kYp = 8, kZm = 16, kZp = 32 };

__device__ __forceinline__ unsigned next_gen(unsigned g) { return g + 1u == 65535u ? 0u : g + 1u; }

struct Shared {
    double part[kBatchMaxScenes][2];   // block partials of this pass
    double tot[kBatchMaxScenes][2];    // grid totals after the barrier
    // per-scene solver scalars (identical in every block)
    double gamma[kBatchMaxScenes], delta[kBatchMaxScenes], gamma_prev[kBatchMaxScenes], alpha_prev[kBatchMaxScenes];
    double alpha[kBatchMaxScenes], beta[kBatchMaxScenes], stop[kBatchMaxScenes], rnorm[kBatchMaxScenes];
    double bnorm[kBatchMaxScenes];
    int phase[kBatchMaxScenes], cur[kBatchMaxScenes], first[kBatchMaxScenes];
    int iters[kBatchMaxScenes], refines[kBatchMaxScenes], converged[kBatchMaxScenes];
    int fluid[kBatchMaxScenes];
    float af[kBatchMaxScenes], bf[kBatchMaxScenes];
    int active;
    unsigned list_count;
};

// Barrier with S*2 sums: block partials (s.part) are added to the slot of this generation, the last arriver
// zeroes the next slot, waiters read the totals into s.tot.
__device__ __forceinline__ bool batch_reduce(Shared& s, const BatchWork& w, int S, unsigned& gen)
{
    __syncthreads();
    double* totals = w.totals;  // [3][kBatchMaxScenes][2]
    const unsigned g = gen;
    double* slot = totals + (size_t)(g % 3u) * kBatchMaxScenes * 2;
    for (int t = threadIdx.x; t < S * 2; t += blockDim.x) {
        const double x = (&s.part[0][0])[t];
        if (x != 0.0) atomicAdd(slot + t, x);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> word(w.bar[0]);
        const unsigned old = word.fetch_add(1u, cuda::memory_order_acq_rel);
        if ((old & 0xffffu) == gridDim.x - 1) {
            double* next = totals + (size_t)(next_gen(g) % 3u) * kBatchMaxScenes * 2;
            for (int t = 0; t < S * 2; ++t) next[t] = 0.0;
            word.store(next_gen(old >> 16) << 16, cuda::memory_order_release);
        } else {
            cuda::atomic_ref<int, cuda::thread_scope_device> e(*w.err);
            unsigned long long spins = 0;
            while ((word.load(cuda::memory_order_acquire) >> 16) == (old >> 16)) {
                if (++spins > kSpinLimit) {
                    e.store(FE_ERR_TIMEOUT, cuda::memory_order_relaxed);
                    break;
                }
                if ((spins & 1023) == 0 && e.load(cuda::memory_order_relaxed) != 0) break;
            }
        }
        gen = next_gen(g);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < S * 2; t += blockDim.x) (&s.tot[0][0])[t] = __ldcg(slot + t);
    __syncthreads();
    return *(volatile int*)w.err == 0;
}

// Flushes a thread's running partial for scene `sc` into the block partials.
__device__ __forceinline__ void flush(Shared& s, int sc, double a0, double a1)
{
    if (sc < 0) return;
    if (a0 != 0.0) atomicAdd(&s.part[sc][0], a0);
    if (a1 != 0.0) atomicAdd(&s.part[sc][1], a1);
}

__global__ void __launch_bounds__(kThreads, 1) k_batch_cg(BatchWork w, int S, double rel_tol, double inner_tol,
                                                          int max_it, int max_refine)
{
    __shared__ Shared s;
    const int T = gridDim.x * blockDim.x;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned gen = 0;
    if (threadIdx.x == 0)
        gen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(w.bar[0]).load(cuda::memory_order_relaxed) >> 16;
    for (int t = threadIdx.x; t < S * 2; t += blockDim.x) (&s.part[0][0])[t] = 0.0;
    __syncthreads();

    // ---- setup over the concatenated cell space: zero non-FLUID entries, ||b||^2, FLUID counts per block
    const long long total_cells = w.cell_offset[S];
    const long long chunk = (total_cells + gridDim.x - 1) / gridDim.x;
    const long long cb = min(total_cells, (long long)blockIdx.x * chunk), ce = min(total_cells, cb + chunk);
    unsigned my_count = 0;
    {
        int sc = 0;
        double a0 = 0.0, a1 = 0.0;
        int cur_sc = -1;
        for (long long g = cb + threadIdx.x; g < ce; g += blockDim.x) {
            while (g >= w.cell_offset[sc + 1]) ++sc;
            const BatchScene& d = w.scenes[sc];
            const int c = (int)(g - w.cell_offset[sc]);
            if (sc != cur_sc) {
                flush(s, cur_sc, a0, a1);
                a0 = a1 = 0.0;
                cur_sc = sc;
            }
            if (d.marks[c] == FE_CELL_FLUID) {
                a0 += d.b[c] * d.b[c];
                a1 += 1.0;
                ++my_count;
            } else {
                d.p[c] = 0.0;
                d.r0[c] = d.r1[c] = d.w0[c] = d.w1[c] = d.s0[c] = d.s1[c] = 0.f;
            }
        }
        flush(s, cur_sc, a0, a1);
    }
    // block FLUID count for the ordered compaction
    {
        __shared__ unsigned s_cnt;
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        atomicAdd(&s_cnt, my_count);
        __syncthreads();
        if (threadIdx.x == 0) w.block_count[blockIdx.x] = s_cnt;
    }
    if (!batch_reduce(s, w, S, gen)) return;
    if (threadIdx.x == 0) {
        s.active = 0;
        for (int sc = 0; sc < S; ++sc) {
            s.bnorm[sc] = sqrt(s.tot[sc][0]);
            s.fluid[sc] = (int)s.tot[sc][1];
            s.phase[sc] = s.bnorm[sc] == 0.0 ? kDone : kResid;
            s.converged[sc] = s.bnorm[sc] == 0.0 ? 1 : 0;
            s.iters[sc] = s.refines[sc] = 0;
            s.cur[sc] = 0;
            s.rnorm[sc] = 0.0;
            s.active += s.phase[sc] != kDone;
        }
        unsigned before = 0, all = 0;
        for (int b = 0; b < (int)gridDim.x; ++b) {
            const unsigned x = __ldcg(w.block_count + b);
            if (b < (int)blockIdx.x) before += x;
            all += x;
        }
        s.list_count = all;
        w.block_count[gridDim.x + blockIdx.x] = before;  // this block's list offset
    }
    __syncthreads();
    // ordered compaction of this block's FLUID cells: entry = (cell << 6) | mask, scene id alongside
    {
        __shared__ unsigned s_warp[32];
        __shared__ unsigned s_base;
        if (threadIdx.x == 0) s_base = w.block_count[gridDim.x + blockIdx.x];
        __syncthreads();
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
        int sc = 0;
        for (long long g0 = cb; g0 < ce; g0 += blockDim.x) {
            const long long g = g0 + threadIdx.x;
            bool fl = false;
            int c = 0;
            if (g < ce) {
                while (g >= w.cell_offset[sc + 1]) ++sc;
                c = (int)(g - w.cell_offset[sc]);
                fl = w.scenes[sc].marks[c] == FE_CELL_FLUID;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, fl);
            if (lane == 0) s_warp[wid] = __popc(bal);
            __syncthreads();
            unsigned off = 0, tot = 0;
            for (int k = 0; k < nw; ++k) {
                off += k < wid ? s_warp[k] : 0u;
                tot += s_warp[k];
            }
            if (fl) {
                const BatchScene& d = w.scenes[sc];
                const int i = c % d.nx, j = (c / d.nx) % d.ny, k = c / (d.nx * d.ny);
                const uint32_t m = (i > 0 ? kXm : 0u) | (i + 1 < d.nx ? kXp : 0u) | (j > 0 ? kYm : 0u) |
                                   (j + 1 < d.ny ? kYp : 0u) | (k > 0 ? kZm : 0u) | (k + 1 < d.nz ? kZp : 0u);
                const uint32_t slot = s_base + off + __popc(bal & ((1u << lane) - 1u));
                w.list[slot] = ((uint32_t)c << 6) | m;
                w.list_scene[slot] = (uint8_t)sc;
            }
            __syncthreads();
            if (threadIdx.x == 0) s_base += tot;
            __syncthreads();
        }
    }
    for (int t = threadIdx.x; t < S * 2; t += blockDim.x) (&s.part[0][0])[t] = 0.0;
    if (!batch_reduce(s, w, S, gen)) return;  // list complete everywhere (no sums needed)
    const unsigned F = s.list_count;

    int global_it = 0;
    while (s.active > 0 && global_it < 4 * max_it + 64 * max_refine) {
        ++global_it;
        // per-scene coefficients of this pass
        if (threadIdx.x < S) {
            const int sc = threadIdx.x;
            if (s.phase[sc] == kIter) {
                double beta = 0.0, alpha;
                if (s.first[sc]) {
                    alpha = s.gamma[sc] / s.delta[sc];
                } else {
                    beta = s.gamma[sc] / s.gamma_prev[sc];
                    alpha = s.gamma[sc] / (s.delta[sc] - beta * s.gamma[sc] / s.alpha_prev[sc]);
                }
                s.alpha[sc] = alpha;
                s.beta[sc] = beta;
                s.af[sc] = (float)alpha;
                s.bf[sc] = (float)beta;
            }
        }
        for (int t = threadIdx.x; t < S * 2; t += blockDim.x) (&s.part[0][0])[t] = 0.0;
        __syncthreads();
        int cur_sc = -1;
        double a0 = 0.0, a1 = 0.0;
        for (unsigned e = tid; e < F; e += T) {
            const int sc = w.list_scene[e];
            if (sc != cur_sc) {
                flush(s, cur_sc, a0, a1);
                a0 = a1 = 0.0;
                cur_sc = sc;
            }
            const int ph = s.phase[sc];
            if (ph == kDone) continue;
            const BatchScene& d = w.scenes[sc];
            const uint32_t ent = w.list[e];
            const int c = (int)(ent >> 6);
            const uint32_t m = ent & 63u;
            const int sx = d.nx, sxy = d.nx * d.ny;
            if (ph == kResid) {
                const double pc = d.p[c];
                double ax = 0.0, ay = 0.0, az = 0.0;
                if (m & kXm) ax += pc - d.p[c - 1];
                if (m & kXp) ax += pc - d.p[c + 1];
                if (m & kYm) ay += pc - d.p[c - sx];
                if (m & kYp) ay += pc - d.p[c + sx];
                if (m & kZm) az += pc - d.p[c - sxy];
                if (m & kZp) az += pc - d.p[c + sxy];
                const double rr = d.b[c] - (d.ih2d[0] * ax + d.ih2d[1] * ay + d.ih2d[2] * az);
                d.r0[c] = (float)rr;
                a0 += rr * rr;
            } else if (ph == kInit) {
                const float* r = d.r0;
                const float rc = r[c];
                float ax = 0.f, ay = 0.f, az = 0.f;
                if (m & kXm) ax += rc - r[c - 1];
                if (m & kXp) ax += rc - r[c + 1];
                if (m & kYm) ay += rc - r[c - sx];
                if (m & kYp) ay += rc - r[c + sx];
                if (m & kZm) az += rc - r[c - sxy];
                if (m & kZp) az += rc - r[c + sxy];
                const float wc = d.ih2[0] * ax + d.ih2[1] * ay + d.ih2[2] * az;
                d.w0[c] = wc;
                d.x[c] = 0.f;
                d.pv[c] = 0.f;
                d.s0[c] = 0.f;
                a0 += (double)rc * rc;
                a1 += (double)wc * rc;
            } else if (ph == kIter) {
                const int cu = s.cur[sc];
                const float* r = cu ? d.r1 : d.r0;
                const float* wv = cu ? d.w1 : d.w0;
                const float* sv = cu ? d.s1 : d.s0;
                float* rn = cu ? d.r0 : d.r1;
                float* wn = cu ? d.w0 : d.w1;
                float* sn = cu ? d.s0 : d.s1;
                const float af = s.af[sc], bf = s.bf[sc];
                auto rnew = [&](int q) { return r[q] - af * (wv[q] + bf * sv[q]); };
                const float snew = wv[c] + bf * sv[c];
                const float pnew = r[c] + bf * d.pv[c];
                const float rc = r[c] - af * snew;
                float ax = 0.f, ay = 0.f, az = 0.f;
                if (m & kXm) ax += rc - rnew(c - 1);
                if (m & kXp) ax += rc - rnew(c + 1);
                if (m & kYm) ay += rc - rnew(c - sx);
                if (m & kYp) ay += rc - rnew(c + sx);
                if (m & kZm) az += rc - rnew(c - sxy);
                if (m & kZp) az += rc - rnew(c + sxy);
                const float wc = d.ih2[0] * ax + d.ih2[1] * ay + d.ih2[2] * az;
                d.pv[c] = pnew;
                d.x[c] += af * pnew;
                sn[c] = snew;
                rn[c] = rc;
                wn[c] = wc;
                a0 += (double)rc * rc;
                a1 += (double)wc * rc;
            } else {  // kUpdate
                d.p[c] += (double)d.x[c];
            }
        }
        flush(s, cur_sc, a0, a1);
        if (!batch_reduce(s, w, S, gen)) return;
        // advance every scene's state machine from the totals (identical in all blocks)
        if (threadIdx.x < S) {
            const int sc = threadIdx.x;
            const double target = rel_tol * s.bnorm[sc];
            switch (s.phase[sc]) {
            case kResid: {
                s.rnorm[sc] = sqrt(s.tot[sc][0]);
                s.cur[sc] = 0;
                if (s.rnorm[sc] <= target) {
                    s.converged[sc] = 1;
                    s.phase[sc] = kDone;
                } else if (s.refines[sc] >= max_refine || s.iters[sc] >= max_it) {
                    s.phase[sc] = kDone;
                } else {
                    ++s.refines[sc];
                    s.phase[sc] = kInit;
                }
                break;
            }
            case kInit: {
                s.gamma[sc] = s.tot[sc][0];
                s.delta[sc] = s.tot[sc][1];
                const double want = fmax(inner_tol, 0.25 * target / s.rnorm[sc]);
                s.stop[sc] = want * want * s.gamma[sc];
                s.first[sc] = 1;
                s.phase[sc] = kIter;
                break;
            }
            case kIter: {
                const double alpha = s.alpha[sc];
                if (!(alpha > 0.0) || !isfinite(alpha)) {  // FP32 breakdown: leave it to the refinement
                    s.phase[sc] = kUpdate;
                    break;
                }
                ++s.iters[sc];
                s.cur[sc] ^= 1;
                s.first[sc] = 0;
                s.gamma_prev[sc] = s.gamma[sc];
                s.alpha_prev[sc] = alpha;
                s.gamma[sc] = s.tot[sc][0];
                s.delta[sc] = s.tot[sc][1];
                if (s.gamma[sc] <= s.stop[sc] || s.iters[sc] >= max_it) s.phase[sc] = kUpdate;
                break;
            }
            case kUpdate:
                s.phase[sc] = kResid;
                break;
            default:
                break;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int a = 0;
            for (int sc = 0; sc < S; ++sc) a += s.phase[sc] != kDone;
            s.active = a;
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x < S) {
        const int sc = threadIdx.x;
        const BatchScene& d = w.scenes[sc];
        if (d.stats_ring) {
            const unsigned slot = atomicAdd(d.stats_counter, 1u) % (1u << 16);
            fe_step_stats st;
            st.cg_iterations = s.iters[sc];
            st.refinements = s.refines[sc];
            st.converged = s.converged[sc];
            st.fluid_cells = s.fluid[sc];
            st.rel_residual = s.bnorm[sc] > 0.0 ? s.rnorm[sc] / s.bnorm[sc] : s.rnorm[sc];
            st.b_norm = s.bnorm[sc];
            d.stats_ring[slot] = st;
        }
    }
}

}  // namespace

cudaError_t batch_cg_blocks(int device, int* blocks)
{
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_cg, kThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    *blocks = sms;
    return cudaSuccess;
}

cudaError_t launch_batch_cg(const BatchWork& w, int S, double rel_tol, double inner_tol, int max_it, int max_refine,
                            cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)w.blocks);
    cfg.blockDim = dim3((unsigned)kThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_batch_cg, w, S, rel_tol, inner_tol, max_it, max_refine);
    count_launch();
    return e;
}

}  // namespace fe
