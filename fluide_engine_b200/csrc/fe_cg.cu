// fe_cg.cu -- pressure solve: FP32 matrix-free conjugate gradient inside FP64 iterative refinement,
// as one persistent cooperative kernel per solve (K_cg).
//
// Reference system (fluid_solvers/single_phase_pressure_solver.cpp:99-164): for a FLUID cell, b = div u,
// diagonal = sum over in-domain non-BOUNDRY neighbours of 1/h_axis^2, off-diagonal -1/h_axis^2 toward
// FLUID neighbours; non-FLUID rows are identity with b = 0, so their solution is 0.  The reference solves
// it with unpreconditioned CG warm-started from the previous pressure (linear_system/
// conjugate_gradient_solver.cpp:14-55, linear_system.cpp:13-18).
//
// Here the FLUID-cell system is solved matrix-free from the cell marks:
//   setup      the FLUID cells are compacted, in cell order, into one list shared evenly by all threads
//              (block counts -> grid barrier -> block offsets -> ordered block compaction), with a 6-bit
//              in-domain-neighbour mask per entry; every non-FLUID entry of p and of the FP32 vectors is
//              0, which makes the stencil branch-free over neighbours
//   outer FP64 r = b - A p, ||r||, test ||r|| <= tol ||b||; after each inner solve p += e
//   inner FP32 Chronopoulos-Gear CG on A e = r (dot products accumulated in FP64): per iteration ONE pass
//              p = r + beta p, s = w + beta s, e += alpha p, r' = r - alpha s, w' = A r' and the two dot
//              products (r', r') and (w', r'), then ONE grid-wide reduction.  w' = A r' needs the
//              neighbours' r', which each thread recomputes as r - alpha (w + beta s) from the previous
//              iteration's neighbour values; r, w and s ping-pong so those stay intact within the pass.
// The grid-wide barrier is a counter + generation word with a bounded spin: if a block waits longer than
// a few seconds it records FE_ERR_TIMEOUT, every block leaves its loops and the kernel returns, so a stuck
// solve surfaces as a status instead of a hung device.  Dot products travel with the barrier: blocks
// add their partials into a rotating totals slot before arriving and read the totals once after it, so
// all blocks take identical branch decisions.
#include "fe_internal.cuh"

#include <cuda/atomic>

namespace fe {
namespace {

constexpr int kCgThreads = 1024;
constexpr int kMultiThreads = 256;
constexpr int kListCache = 8192;  // FLUID-list entries cached in shared memory per block (32 KB)
constexpr unsigned long long kSpinLimit = 1ull << 26;

struct CgParams {
    double rel_tol, inner_tol;
    int max_it, max_refine;
    fe_step_stats* stats_ring;
    unsigned* stats_counter;
    unsigned stats_cap;
};

// Barrier generations count modulo 65535 (a multiple of 3), so the three rotating totals slots keep their
// order across the wrap.
__device__ __forceinline__ unsigned next_gen(unsigned g) { return g + 1u == 65535u ? 0u : g + 1u; }

// Grid-wide barrier on two words in different 128-byte lines: bar[0] counts arrivals (one acq_rel
// fetch_add per block), bar[32] holds the generation.  The last arriver resets the count, zeroes the totals
// slot of the next generation and bumps the generation with a release store; the others poll the
// generation (bounded) with acquire loads, away from the line the arrivals hit.  The release/acquire pair at
// device scope, with the __syncthreads on either side, orders every thread's memory traffic of the block
// across the barrier.  `gen` is the generation this barrier started in (tracked by thread 0).  Returns
// false when the wait gave up.
__device__ __forceinline__ bool bar_arrive_wait(unsigned* bar, int* err, unsigned nblocks, double* totals, unsigned gen)
{
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> count(bar[0]);
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> genw(bar[32]);
    const unsigned old = count.fetch_add(1u, cuda::memory_order_acq_rel);
    if (old == nblocks - 1) {
        double* next = totals + 4 * (next_gen(gen) % 3u);
#pragma unroll
        for (int k = 0; k < 4; ++k) next[k] = 0.0;
        count.store(0u, cuda::memory_order_relaxed);
        genw.store(next_gen(gen), cuda::memory_order_release);
        return true;
    }
    cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
    unsigned long long spins = 0;
    while (genw.load(cuda::memory_order_acquire) == gen) {
        if (++spins > kSpinLimit) {
            e.store(FE_ERR_TIMEOUT, cuda::memory_order_relaxed);
            return false;
        }
        if ((spins & 1023) == 0 && e.load(cuda::memory_order_relaxed) != 0) return false;
    }
    return true;
}

__device__ __forceinline__ bool grid_sync(const CgWork& w, unsigned& gen, int nblk)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        bar_arrive_wait(w.bar, w.err, (unsigned)nblk, w.partial, gen);
        gen = next_gen(gen);
    }
    __syncthreads();
    return *(volatile int*)w.err == 0;
}

// Grid-wide sum of N doubles fused with the barrier.  Each block reduces to warp 0, whose lane 0 adds
// the block partials into the totals slot of this barrier (FP64 red.add, ordered before the arrival by
// its release) and arrives; after the barrier it reads the totals once.  Three total slots rotate: the
// last arriver of barrier k zeroes slot k+1 before releasing it, and slot k is read only until the
// readers arrive at barrier k+1.  All blocks read the same final totals, so their branch decisions
// agree (the summation order, and hence the last bits, can vary from run to run).  (Per-block slots summed
// by the last arriver avoid the floating-point atomics but put one more L2 round trip on the critical
// path, which measured slower.)
template <int N>
__device__ __forceinline__ bool grid_reduce(double (&v)[N], double* sh /* [132] */, const CgWork& w, unsigned& gen,
                                            int nblk)
{
    static_assert(N <= 4, "at most 4 sums per reduction");
    // warp partials use sh[0, 32 N), the totals sh[128, 128 + N): disjoint, so a warp that races ahead into
    // the next reduction cannot overwrite totals another warp has not read yet
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) sh[wid * N + k] = v[k];
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        double part[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double s = lane < nw ? sh[lane * N + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            part[k] = s;
        }
        if (lane == 0) {
            // slot of this barrier: generation modulo 3; thread 0 tracks the generation itself (it takes
            // part in every barrier), which saves a load round trip per barrier
            double* totals = w.partial;  // [3][4]
            double* slot = totals + 4 * (gen % 3u);  // zeroed by the release of this generation
#pragma unroll
            for (int k = 0; k < N; ++k) atomicAdd(slot + k, part[k]);
            const bool ok = bar_arrive_wait(w.bar, w.err, (unsigned)nblk, totals, gen);
            gen = next_gen(gen);
            if (ok)
#pragma unroll
                for (int k = 0; k < N; ++k) sh[128 + k] = __ldcg(slot + k);
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[128 + k];
    return *(volatile int*)w.err == 0;
}

// Block-wide sum of one double, valid in all threads (setup only).
__device__ __forceinline__ double block_sum1(double x, double* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if (lane == 0) sh[wid] = x;
    __syncthreads();
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += sh[k];
    __syncthreads();
    return s;
}

enum : uint32_t { kXm = 1, kXp = 2, kYm = 4, kYp = 8, kZm = 16, kZp = 32 };

struct Stencil7 {
    int sx;
    int sxy;
    float ih2[3];
};

// (A v)_c for the FLUID row c with in-domain mask m, non-FLUID entries of v being 0.
template <class F>
__device__ __forceinline__ float apply_row(const Stencil7& st, int c, uint32_t m, F val)
{
    const float vc = val(c);
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (m & kXm) ax += vc - val(c - 1);
    if (m & kXp) ax += vc - val(c + 1);
    if (m & kYm) ay += vc - val(c - st.sx);
    if (m & kYp) ay += vc - val(c + st.sx);
    if (m & kZm) az += vc - val(c - st.sxy);
    if (m & kZp) az += vc - val(c + st.sxy);
    return st.ih2[0] * ax + st.ih2[1] * ay + st.ih2[2] * az;
}

// The solver body, run by `nblk` blocks of which this is block `blk` (a whole grid for one scene, or a
// block range of a multi-scene launch, see k_multi_cg); every barrier and reduction spans those blocks.
__device__ __forceinline__ void cg_body(const SceneView& v, const CgWork& w, const CgParams& prm, const int blk,
                                        const int nblk, int* out_its = nullptr, int* out_fluid = nullptr)
{
    __shared__ double sh[32 * 4 + 4];
    __shared__ uint32_t s_warp[32];
    // the FLUID list does not change during a solve: each thread keeps its first list entries in shared
    // memory (entry k of thread t at s_list[k * blockDim.x + t]), which takes one dependent L2 round trip
    // out of every pass
    __shared__ uint32_t s_list[kListCache];
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const int sxy = nx * ny;
    const int nc = sxy * nz;
    const int T = nblk * blockDim.x;
    const int tid = blk * blockDim.x + threadIdx.x;
    const uint8_t* __restrict__ marks = v.marks;
    const double ih2d[3] = {v.inv_h[0] * v.inv_h[0], v.inv_h[1] * v.inv_h[1], v.inv_h[2] * v.inv_h[2]};
    Stencil7 st;
    st.sx = nx;
    st.sxy = sxy;
    st.ih2[0] = (float)ih2d[0];
    st.ih2[1] = (float)ih2d[1];
    st.ih2[2] = (float)ih2d[2];
    double* __restrict__ p64 = v.p;
    const double* __restrict__ b = v.b;
    float* __restrict__ R[2] = {w.r0, w.r1};
    float* __restrict__ W[2] = {w.w0, w.w1};
    float* __restrict__ S[2] = {w.s0, w.s1};
    float* __restrict__ P = w.pv;
    float* __restrict__ X = w.x;
    uint32_t* __restrict__ list = w.list;

    // barrier generation as of this launch (thread 0 keeps it from here on)
    unsigned gen = 0;
    if (threadIdx.x == 0) gen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(w.bar[32]).load(cuda::memory_order_relaxed);

    // ---- setup: zero non-FLUID entries, ||b||^2, per-block FLUID counts over the block's cell range
    const int chunk = (nc + nblk - 1) / nblk;
    const int cb = min(nc, blk * chunk), ce = min(nc, cb + chunk);
    double acc[2] = {0.0, 0.0};
    for (int c = cb + threadIdx.x; c < ce; c += blockDim.x) {
        if (marks[c] == FE_CELL_FLUID) {
            acc[0] += b[c] * b[c];
            acc[1] += 1.0;
        } else {
            p64[c] = 0.0;
            R[0][c] = 0.f;
            R[1][c] = 0.f;
            W[0][c] = 0.f;
            W[1][c] = 0.f;
            S[0][c] = 0.f;
            S[1][c] = 0.f;
        }
    }
    // block offset = FLUID count of all earlier blocks (fixed order), total = all blocks
    const double mine = block_sum1(acc[1], sh);
    if (threadIdx.x == 0) w.partial[16 + blk] = mine;
    double tot[2] = {acc[0], acc[1]};
    if (!grid_reduce<2>(tot, sh, w, gen, nblk)) return;
    const double bnorm = sqrt(tot[0]);
    const int F = (int)tot[1];
    double before = 0.0;
    for (int bb = threadIdx.x; bb < blk; bb += blockDim.x) before += __ldcg(w.partial + 16 + bb);
    before = block_sum1(before, sh);
    // ordered compaction of this block's FLUID cells with their in-domain masks
    uint32_t base = (uint32_t)before;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int c0 = cb; c0 < ce; c0 += blockDim.x) {
        const int c = c0 + threadIdx.x;
        const bool fl = c < ce && marks[c] == FE_CELL_FLUID;
        const unsigned bal = __ballot_sync(0xffffffffu, fl);
        if (lane == 0) s_warp[wid] = __popc(bal);
        __syncthreads();
        uint32_t off = 0, total = 0;
        for (int k = 0; k < nwarp; ++k) {
            const uint32_t x = s_warp[k];
            off += k < wid ? x : 0u;
            total += x;
        }
        if (fl) {
            const int i = c % nx, j = (c / nx) % ny, k = c / sxy;
            uint32_t m = (i > 0 ? kXm : 0u) | (i + 1 < nx ? kXp : 0u) | (j > 0 ? kYm : 0u) | (j + 1 < ny ? kYp : 0u) |
                         (k > 0 ? kZm : 0u) | (k + 1 < nz ? kZp : 0u);
            const uint32_t slot = base + off + __popc(bal & ((1u << lane) - 1u));
            list[slot] = ((uint32_t)c << 6) | m;
        }
        base += total;
        __syncthreads();
    }
    if (!grid_sync(w, gen, nblk)) return;
    const int kc = kListCache / (int)blockDim.x;
    {
        int k = 0;
        for (int e = tid; e < F && k < kc; e += T, ++k) s_list[k * blockDim.x + threadIdx.x] = __ldcg(list + e);
    }
    auto entry = [&](int k, int e) -> uint32_t { return k < kc ? s_list[k * blockDim.x + threadIdx.x] : list[e]; };
    const double target = prm.rel_tol * bnorm;
    if (bnorm == 0.0) {
        for (int e = tid; e < F; e += T) p64[list[e] >> 6] = 0.0;
    }

    int total_it = 0, refinements = 0;
    double rnorm = 0.0;
    bool converged = bnorm == 0.0;
    int cur = 0;  // ping-pong index of r, w, s
    while (!converged) {
        // ---- outer residual r = b - A p in FP64, stored in FP32 for the inner solve
        double racc[1] = {0.0};
        for (int e = tid, k = 0; e < F; e += T, ++k) {
            const uint32_t ent = entry(k, e);
            const int c = (int)(ent >> 6);
            const uint32_t m = ent & 63u;
            const double pc = p64[c];
            double ax = 0.0, ay = 0.0, az = 0.0;
            if (m & kXm) ax += pc - p64[c - 1];
            if (m & kXp) ax += pc - p64[c + 1];
            if (m & kYm) ay += pc - p64[c - nx];
            if (m & kYp) ay += pc - p64[c + nx];
            if (m & kZm) az += pc - p64[c - sxy];
            if (m & kZp) az += pc - p64[c + sxy];
            const double rr = b[c] - (ih2d[0] * ax + ih2d[1] * ay + ih2d[2] * az);
            R[0][c] = (float)rr;
            racc[0] += rr * rr;
        }
        cur = 0;
        if (!grid_reduce<1>(racc, sh, w, gen, nblk)) return;
        rnorm = sqrt(racc[0]);
        if (rnorm <= target) {
            converged = true;
            break;
        }
        if (refinements >= prm.max_refine || total_it >= prm.max_it) break;
        ++refinements;

        // ---- inner Chronopoulos-Gear CG on A e = r; w0 = A r0 and the first dot products
        double d0[2] = {0.0, 0.0};
        for (int e = tid, k = 0; e < F; e += T, ++k) {
            const uint32_t ent = entry(k, e);
            const int c = (int)(ent >> 6);
            const float* __restrict__ r0 = R[0];
            const float wc = apply_row(st, c, ent & 63u, [&](int q) { return r0[q]; });
            const float rc = r0[c];
            W[0][c] = wc;
            X[c] = 0.f;
            P[c] = 0.f;
            S[0][c] = 0.f;
            d0[0] += (double)rc * (double)rc;
            d0[1] += (double)wc * (double)rc;
        }
        if (!grid_reduce<2>(d0, sh, w, gen, nblk)) return;
        double gamma = d0[0], delta = d0[1];
        const double gamma0 = gamma;
        const double want = fmax(prm.inner_tol, 0.25 * target / rnorm);
        const double stop = want * want * gamma0;
        double alpha_prev = 1.0, gamma_prev = 1.0;
        bool first = true;
        while (total_it < prm.max_it) {
            double beta = 0.0, alpha;
            if (first) {
                alpha = gamma / delta;
            } else {
                beta = gamma / gamma_prev;
                alpha = gamma / (delta - beta * gamma / alpha_prev);
            }
            if (!(alpha > 0.0) || !isfinite(alpha)) break;  // FP32 breakdown: leave it to the outer loop
            first = false;
            const float af = (float)alpha, bf = (float)beta;
            const float* __restrict__ r = R[cur];
            const float* __restrict__ wv = W[cur];
            const float* __restrict__ s = S[cur];
            float* __restrict__ rn = R[cur ^ 1];
            float* __restrict__ wn = W[cur ^ 1];
            float* __restrict__ sn = S[cur ^ 1];
            double dd[2] = {0.0, 0.0};
            for (int e = tid, k = 0; e < F; e += T, ++k) {
                const uint32_t ent = entry(k, e);
                const int c = (int)(ent >> 6);
                // r'(q) = r(q) - alpha (w(q) + beta s(q)) for this cell and its neighbours
                auto rnew = [&](int q) { return r[q] - af * (wv[q] + bf * s[q]); };
                const float snew = wv[c] + bf * s[c];
                const float pnew = r[c] + bf * P[c];
                const float rc = r[c] - af * snew;
                const float wc = apply_row(st, c, ent & 63u, rnew);
                P[c] = pnew;
                X[c] += af * pnew;
                sn[c] = snew;
                rn[c] = rc;
                wn[c] = wc;
                dd[0] += (double)rc * (double)rc;
                dd[1] += (double)wc * (double)rc;
            }
            if (!grid_reduce<2>(dd, sh, w, gen, nblk)) return;
            ++total_it;
            cur ^= 1;
            gamma_prev = gamma;
            alpha_prev = alpha;
            gamma = dd[0];
            delta = dd[1];
            if (gamma <= stop) break;
        }
        // ---- p += e (FP64); the next residual pass reads neighbours' p, hence the barrier
        for (int e = tid, k = 0; e < F; e += T, ++k) {
            const int c = (int)(entry(k, e) >> 6);
            p64[c] += (double)X[c];
        }
        if (!grid_sync(w, gen, nblk)) return;
    }
    if (blk == 0 && threadIdx.x == 0 && out_its) {
        *out_its = total_it;
        *out_fluid = F;
    }
    if (blk == 0 && threadIdx.x == 0 && prm.stats_ring) {
        const unsigned slot = atomicAdd(prm.stats_counter, 1u) % prm.stats_cap;
        fe_step_stats s;
        s.cg_iterations = total_it;
        s.refinements = refinements;
        s.converged = converged ? 1 : 0;
        s.fluid_cells = F;
        s.rel_residual = bnorm > 0.0 ? rnorm / bnorm : rnorm;
        s.b_norm = bnorm;
        prm.stats_ring[slot] = s;
    }
}

__global__ void __launch_bounds__(kCgThreads, 1) k_cg(SceneView v, CgWork w, CgParams prm)
{
    cg_body(v, w, prm, blockIdx.x, gridDim.x);
}

// Many scenes in one cooperative launch: blocks [start[s], start[s+1]) solve scene s with their own barrier
// and reductions, so scenes iterate independently and concurrently.
__global__ void __launch_bounds__(kMultiThreads) k_multi_cg(MultiCgScene* __restrict__ scenes, int S)
{
    int sc = 0;
    while (sc + 1 < S && (int)blockIdx.x >= scenes[sc + 1].block_start) ++sc;
    MultiCgScene& m = scenes[sc];
    CgParams prm;
    prm.rel_tol = m.rel_tol;
    prm.inner_tol = m.inner_tol;
    prm.max_it = m.max_it;
    prm.max_refine = m.max_refine;
    prm.stats_ring = m.work.stats;
    prm.stats_counter = m.work.bar + 2;
    prm.stats_cap = 1u << 16;
    int its = 0, fluid = 0;
    const int blk = (int)blockIdx.x - m.block_start;
    cg_body(m.view, m.work, prm, blk, m.block_count, &its, &fluid);
    if (blk == 0 && threadIdx.x == 0) {  // read by the next solve's k_multi_partition
        m.last_its = its;
        m.last_fluid = fluid;
    }
}

// One thread splits total_blocks among the scenes before a multi-scene solve: one block each, the rest in
// proportion to the previous solve's work of the scene (FLUID cells x (inner iterations + 3 residual
// passes); weight0 before its first solve), leftovers to the heaviest scenes.  Scenes then take about
// equally long, instead of the scene with the most iterations finishing last on a small share.
__global__ void k_multi_partition(MultiCgScene* __restrict__ scenes, int S, int total_blocks)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double wsum = 0.0;
    for (int i = 0; i < S; ++i) {
        const MultiCgScene& m = scenes[i];
        const double w = m.last_its >= 0 ? (double)m.last_fluid * (double)(m.last_its + 3) : m.weight0;
        wsum += fmax(w, 0.0);
    }
    const int spare = total_blocks - S;
    int start = 0, used = 0;
    for (int i = 0; i < S; ++i) {
        MultiCgScene& m = scenes[i];
        const double w = fmax(m.last_its >= 0 ? (double)m.last_fluid * (double)(m.last_its + 3) : m.weight0, 0.0);
        const int extra = wsum > 0.0 ? (int)floor(spare * (w / wsum)) : spare / S;
        m.block_count = 1 + extra;
        used += 1 + extra;
    }
    // leftovers (fewer than S) one each to the heaviest scenes, heaviest first
    for (int left = total_blocks - used; left > 0; --left) {
        int best = -1;
        double bw = -1.0;
        for (int i = 0; i < S; ++i) {
            const MultiCgScene& m = scenes[i];
            double w = m.last_its >= 0 ? (double)m.last_fluid * (double)(m.last_its + 3) : m.weight0;
            w = w / (double)m.block_count;  // work per block: give the block where it is most needed
            if (w > bw) {
                bw = w;
                best = i;
            }
        }
        scenes[best].block_count += 1;
    }
    for (int i = 0; i < S; ++i) {
        scenes[i].block_start = start;
        start += scenes[i].block_count;
    }
}

}  // namespace

cudaError_t multi_cg_capacity(int device, int* max_blocks, int* threads)
{
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_multi_cg, kMultiThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    *max_blocks = sms * per_sm;
    *threads = kMultiThreads;
    return cudaSuccess;
}

cudaError_t launch_multi_cg(MultiCgScene* scenes, int S, int total_blocks, cudaStream_t st)
{
    k_multi_partition<<<1, 32, 0, st>>>(scenes, S, total_blocks);
    count_launch();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)total_blocks);
    cfg.blockDim = dim3((unsigned)kMultiThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_multi_cg, scenes, S);
    count_launch();
    return e;
}

cudaError_t cg_prepare(CgWork& w, int device)
{
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg, kCgThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    w.blocks = sms;  // one persistent block per SM
    w.threads = kCgThreads;
    return cudaSuccess;
}

cudaError_t launch_cg(const SceneView& v, const CgWork& w, double rel_tol, double inner_tol, int max_it,
                      int max_refine, cudaStream_t st)
{
    CgParams prm;
    prm.rel_tol = rel_tol;
    prm.inner_tol = inner_tol;
    prm.max_it = max_it;
    prm.max_refine = max_refine;
    prm.stats_ring = w.stats;
    prm.stats_counter = (unsigned*)(w.bar + 2);
    prm.stats_cap = 1u << 16;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)w.blocks);
    cfg.blockDim = dim3((unsigned)w.threads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_cg, v, w, prm);
    count_launch();
    return e;
}

}  // namespace fe
