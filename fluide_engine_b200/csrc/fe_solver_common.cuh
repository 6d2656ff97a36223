// fe_solver_common.cuh -- device pieces shared by the persistent pressure solvers (fe_cg.cu, fe_mgcg.cu):
// the bounded grid barrier, grid-wide FP64 sums fused with it, the 7-point FLUID-row stencil and the setup
// that compacts the FLUID cells into the solver's list.  Internal linkage: each solver file gets its own copy.
#pragma once

#include <cuda/atomic>

#include "fe_internal.cuh"

namespace fe {
namespace {

constexpr int kListCache = 8192;  // FLUID-list entries cached in shared memory per block (32 KB)
constexpr unsigned long long kSpinLimit = 1ull << 26;

// Limits of the bounded grid-barrier wait, in constant memory (one copy per translation unit that includes this
// header): the polls a block makes before it gives up with FE_ERR_TIMEOUT, and arrivals the barrier waits for
// beyond the blocks of the launch.  In normal operation they are kSpinLimit and 0; the failure-detection test
// hook (fe_debug_set_barrier_limits) sets a short limit and one extra arrival, so every wait runs out.
__constant__ unsigned long long c_spin_limit = kSpinLimit;
__constant__ unsigned c_extra_arrivals = 0u;

struct CgParams {
    double rel_tol, inner_tol;
    int max_it, max_refine;
    fe_step_stats* stats_ring;
    unsigned* stats_counter;
    unsigned stats_cap;
};

// ---- Grid barrier.  The barrier words and the totals start every launch at zero: the last block to leave a
// solver kernel puts them back (solver_exit), and the host clears them after a solve that failed.  bar[0] counts
// the arrivals of the whole launch: each arriving block (or cluster leader) adds 1 with a release reduction and
// polls the count with acquire loads until it reaches (gen + 1) x arrivals, so nothing on the critical path resets
// a word or bumps a generation: a barrier costs the release (which waits for the block's own totals adds) and
// the poll.  `gen` is the number of barriers this launch has passed, tracked by every thread.
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Polls bar[0] until it reaches `target` (bounded: FE_ERR_TIMEOUT after the limit; gives up early when another
// block has set the error flag).  False when the wait gave up.
__device__ __forceinline__ bool bar_poll(const unsigned* bar, int* err, unsigned target)
{
    cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
    unsigned long long spins = 0;
    const unsigned long long limit = c_spin_limit;
    while ((int)(ld_acquire(bar) - target) < 0) {
        if (++spins > limit) {
            e.store(FE_ERR_TIMEOUT, cuda::memory_order_relaxed);
            return false;
        }
        if ((spins & 1023) == 0 && e.load(cuda::memory_order_relaxed) != 0) return false;
    }
    return true;
}

// Total k of group g in rotating slot `slot` (one 128-byte line each).
__device__ __forceinline__ double* totals_at(double* partial, unsigned slot, int g, int k)
{
    return partial + (size_t)(((int)slot * kCgTotalsGroups + g) * 4 + k) * kCgTotalsStride;
}

// Last act of every block of a solver kernel (thread 0, after its last barrier): the last block to leave puts
// the arrival count and the totals back to zero for the next launch.  The others have finished all their polls
// and totals reads before their exit add (release), which the last one observes (acquire).
__device__ __forceinline__ void solver_exit(const CgWork& w, int nblk)
{
    if (threadIdx.x != 0) return;
    cuda::atomic_ref<unsigned, cuda::thread_scope_device> left(w.bar[32]);
    if (left.fetch_add(1u, cuda::memory_order_acq_rel) != (unsigned)nblk - 1u) return;
    for (int i = 0; i < 3 * kCgTotalsGroups * 4; ++i) w.partial[(size_t)i * kCgTotalsStride] = 0.0;
    w.bar[0] = 0u;
    left.store(0u, cuda::memory_order_relaxed);
}

// ---- Cluster pre-reduction (CgWork::cluster > 1: the solver was launched in thread-block clusters of that size).
// Inside a cluster the blocks hand their partial sums to the cluster's first block (rank 0, the leader) through
// distributed shared memory and a release add on a counter in the leader's shared memory; only the leader adds into
// the global totals slot and arrives at the grid barrier (arrivals: one per cluster), while every block polls the
// barrier's arrival count as before.  The leader's wait for its cluster is a bounded poll of its own shared memory,
// so an error anywhere still ends every block's waits; the kernel's last step is a cluster barrier (all waits before
// it are bounded), so no block exits while another block of its cluster may still write into its shared memory.
// Shared-memory words of the leader: the partials at sh[kClusterSlots + 4 rank + k], the arrival counter and the
// count of cluster gathers so far behind them.
constexpr int kMaxCluster = 16;
constexpr int kClusterSlots = 132;                         // after the block reduction's 132 doubles
constexpr int kShDoubles = kClusterSlots + 4 * kMaxCluster + 3;  // + the barrier outcome word

__device__ __forceinline__ unsigned* cluster_counter(double* sh) { return reinterpret_cast<unsigned*>(sh + kClusterSlots + 4 * kMaxCluster); }
__device__ __forceinline__ unsigned* cluster_rounds(double* sh) { return reinterpret_cast<unsigned*>(sh + kClusterSlots + 4 * kMaxCluster + 1); }

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Generic address of `p` (this block's shared memory) in the shared memory of cluster block `rank`.
template <class T>
__device__ __forceinline__ T* cluster_map(T* p, unsigned rank)
{
    T* out;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(out) : "l"(p), "r"(rank));
    return out;
}

__device__ __forceinline__ void cluster_barrier_all()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Thread 0 of every block: hands this block's N partials to the leader (peers) or waits for the peers' (leader,
// bounded) and returns the cluster's sums in part.  Returns false when the leader's wait gave up.
template <int N>
__device__ __forceinline__ bool cluster_gather(double* part, double* sh, int cs, int* err)
{
    const unsigned rank = cluster_rank();
    if (rank != 0) {
        double* dst = cluster_map(sh + kClusterSlots + 4 * rank, 0u);
#pragma unroll
        for (int k = 0; k < N; ++k) dst[k] = part[k];
        unsigned* cnt = cluster_map(cluster_counter(sh), 0u);
        asm volatile("red.release.cluster.add.u32 [%0], 1;" ::"l"(cnt) : "memory");
        return true;
    }
    unsigned* rounds = cluster_rounds(sh);
    const unsigned want = (*rounds + 1u) * (unsigned)(cs - 1);
    *rounds += 1u;
    unsigned* cnt = cluster_counter(sh);
    unsigned long long spins = 0;
    const unsigned long long limit = c_spin_limit;
    cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
    while (true) {
        unsigned got;
        asm volatile("ld.acquire.cluster.u32 %0, [%1];" : "=r"(got) : "l"(cnt) : "memory");
        if ((int)(got - want) >= 0) break;
        if (++spins > limit) {
            e.store(FE_ERR_TIMEOUT, cuda::memory_order_relaxed);
            return false;
        }
        if ((spins & 1023) == 0 && e.load(cuda::memory_order_relaxed) != 0) return false;
    }
    for (int r = 1; r < cs; ++r)
#pragma unroll
        for (int k = 0; k < N; ++k) part[k] += sh[kClusterSlots + 4 * r + k];
    return true;
}

// Start of a clustered solver kernel: the leader's counters are zeroed before any block of the cluster can add.
__device__ __forceinline__ void cluster_begin(const CgWork& w, double* sh)
{
    if (w.cluster <= 1) return;
    if (threadIdx.x == 0) {
        *cluster_counter(sh) = 0u;
        *cluster_rounds(sh) = 0u;
    }
    cluster_barrier_all();
}

// End of a clustered solver kernel (every block reaches it: all waits before it are bounded).
__device__ __forceinline__ void cluster_end(const CgWork& w)
{
    if (w.cluster > 1) cluster_barrier_all();
}

// Blocks that arrive at each barrier: every block, or one per cluster; plus the test hook's extra arrivals.
__device__ __forceinline__ int barrier_members(const CgWork& w, int nblk) { return w.cluster > 1 ? nblk / w.cluster : nblk; }

// Copies of the totals: several groups of arriving blocks add into their own copy once there are many arrivals.
__device__ __forceinline__ int totals_groups(int members) { return members > 256 ? kCgTotalsGroups : 1; }

// Warp 0 of every block, at grid barrier `gen` with N partial sums in lane 0's `part` (already reduced over the
// block): the arrival (plain, or through its cluster's leader), the bounded poll by lane 0, and the totals read by
// lanes g N + k of every group g in parallel with the error flag (lane 31).  Lanes k < N return total k in `out`,
// summed over the groups in group order, so every block gets the same bits.  All lanes return whether the waits
// ended and no block has reported an error.  Block 0 then zeroes the slot two barriers ahead: its last readers
// arrived at this barrier, and its next adders only start after this block's next arrival (a release).
template <int N>
__device__ __forceinline__ bool warp0_barrier(double* part, double& out, double* sh, const CgWork& w, unsigned gen,
                                              int nblk, int blk)
{
    const int lane = threadIdx.x & 31;
    const unsigned slot = gen % 3u;
    const int members = barrier_members(w, nblk);
    const int G = totals_groups(members);
    bool ok = true;
    if (lane == 0) {
        bool arrive = true;
        int member = blk;
        if (w.cluster > 1) {
            ok = cluster_gather<N>(part, sh, w.cluster, w.err);
            arrive = cluster_rank() == 0;
            member = blk / w.cluster;
        }
        if (ok && arrive) {
#pragma unroll
            for (int k = 0; k < N; ++k) atomicAdd(totals_at(w.partial, slot, member % G, k), part[k]);
            red_release_add(w.bar, 1u);
        }
        if (ok) ok = bar_poll(w.bar, w.err, (gen + 1u) * (unsigned)(members + (int)c_extra_arrivals));
    }
    __syncwarp();
    double t = 0.0;
    int e = 0;
    if (N > 0 && lane < G * N) t = __ldcg(totals_at(w.partial, slot, lane / (N > 0 ? N : 1), lane % (N > 0 ? N : 1)));
    if (N > 0 && lane == 31) e = __ldcg(w.err);
    ok = __all_sync(0xffffffffu, ok && e == 0) != 0;
    double sum = 0.0;
    for (int g = 0; g < G; ++g)
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double x = __shfl_sync(0xffffffffu, t, g * N + k);
            if (lane == k) sum += x;
        }
    if (blk == 0 && lane < 4 * G) *totals_at(w.partial, (slot + 2u) % 3u, lane >> 2, lane & 3) = 0.0;
    out = sum;
    return ok;
}

// Shared-memory word through which warp 0 hands the barrier's outcome to the whole block.
constexpr int kShFlag = kShDoubles - 1;

__device__ __forceinline__ bool grid_sync(const CgWork& w, unsigned& gen, int nblk, double* sh, int blk)
{
    __syncthreads();
    if (threadIdx.x < 32) {
        double none[1] = {0.0};
        double out;
        const bool ok = warp0_barrier<0>(none, out, sh, w, gen, nblk, blk);
        if (threadIdx.x == 0) sh[kShFlag] = ok ? 0.0 : 1.0;
    }
    ++gen;
    __syncthreads();
    return sh[kShFlag] == 0.0;
}

// Grid-wide sum of N doubles fused with the barrier.  Each block reduces to warp 0, whose lane 0 adds the block
// partials into its group's copy of the totals slot of this barrier (FP64 red.add, ordered before the arrival by
// its release) and arrives; after the barrier warp 0 reads the totals once.  All blocks read the same totals and
// sum the groups in the same order, so their branch decisions agree (the order of the atomic adds, and hence the
// last bits, can vary from run to run).  (Measured alternatives: per-block slots summed by the last arriver, an
// arrival tree, an all-gather of per-block slots, and a generation word bumped by the last arriver all put more
// L2 round trips on the critical path.)
template <int N>
__device__ __forceinline__ bool grid_reduce(double (&v)[N], double* sh /* [kShDoubles] */, const CgWork& w, unsigned& gen,
                                            int nblk, int blk)
{
    static_assert(N >= 1 && N <= 4, "1 to 4 sums per reduction");
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
        double out;
        const bool ok = warp0_barrier<N>(part, out, sh, w, gen, nblk, blk);
        if (lane < N) sh[128 + lane] = out;
        if (lane == 0) sh[kShFlag] = ok ? 0.0 : 1.0;
    }
    ++gen;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[128 + k];
    return sh[kShFlag] == 0.0;
}

// Index of this thread among the nblk x blockDim.x threads of a solver for the loops over the FLUID list and the
// multigrid levels (entry e = index + k x all threads): warps are interleaved across the blocks (warp j of block
// blk is warp j nblk + blk), so a partial last round of the list spreads over every block instead of landing on
// the first blocks -- at 128^3, 3.4 rounds per thread gave blocks 0..56 four rounds and the rest three -- while
// each warp still takes 32 consecutive entries.
__device__ __forceinline__ int solver_thread(int blk, int nblk)
{
    return (((int)(threadIdx.x >> 5) * nblk + blk) << 5) + (int)(threadIdx.x & 31);
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

// Shared memory of one solver block, declared once per kernel and handed to whichever solver body runs.
constexpr int kCoarseMaxCells = 512;  // the multigrid solver's coarsest level lives in shared memory
struct SolverSmem {
    double sh[kShDoubles];                 // block reductions, then the cluster pre-reduction's words
    uint32_t s_warp[32];                   // compaction counts
    uint32_t s_list[kListCache];           // cached FLUID-list entries
    float cz[2][kCoarseMaxCells];          // multigrid: coarsest-level correction (ping-pong)
    float cr[kCoarseMaxCells];             // multigrid: coarsest-level right-hand side
    float cw[kCoarseMaxCells];             // multigrid: coarsest-level omega / diagonal (0 outside the mask)
    uint8_t cb[kCoarseMaxCells];           // multigrid: coarsest-level in-domain neighbour bits
};

// Solver setup shared by the persistent solvers, run by `nblk` blocks of which this is block `blk`: zeroes
// the non-FLUID entries of the pressure and of the FP32 solver vectors (so stencils over them need no branch
// on the cell type), sums ||b||^2, compacts the FLUID cells in cell order into w.list with their
// in-domain-neighbour masks (per-block counts -> grid reduction -> block offsets -> ordered compaction), and
// caches each thread's first list entries in s_list.  Returns false when a grid wait gave up.
// Vector layouts whose non-FLUID entries the setup zeroes: the multigrid solver's separate arrays, the plain CG's
// interleaved (r, w, s, p) cells.
enum { kLayoutSeparate = 0, kLayoutInterleaved = 1 };

struct SolverSetup {
    int F;          // FLUID cells
    double bnorm;   // ||b||_2
    int kc;         // list entries cached per thread
};

// The stencil mask of cell c: in-domain neighbours that are not BOUNDRY (single_phase_pressure_solver.cpp:117-150),
// 0 for non-FLUID cells.  A FLUID cell enclosed by BOUNDRY cells and walls has an all-zero row in the reference's
// system: nothing couples to it and its pressure reaches no face (ApplyPressure skips faces toward BOUNDRY), so it
// is left out of the solve with pressure 0 instead of holding the residual at |b| for every iteration.
__device__ __forceinline__ uint32_t solve_mask(const uint8_t* __restrict__ marks, int c, int nx, int ny, int nz)
{
    if (marks[c] != FE_CELL_FLUID) return 0u;
    const int i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
    const size_t sxy1 = (size_t)nx * ny;
    return (i > 0 && marks[c - 1] != FE_CELL_BOUNDRY ? kXm : 0u) |
           (i + 1 < nx && marks[c + 1] != FE_CELL_BOUNDRY ? kXp : 0u) |
           (j > 0 && marks[c - nx] != FE_CELL_BOUNDRY ? kYm : 0u) |
           (j + 1 < ny && marks[c + nx] != FE_CELL_BOUNDRY ? kYp : 0u) |
           (k > 0 && marks[c - sxy1] != FE_CELL_BOUNDRY ? kZm : 0u) |
           (k + 1 < nz && marks[c + sxy1] != FE_CELL_BOUNDRY ? kZp : 0u);
}

__device__ __forceinline__ bool solver_setup(const SceneView& v, const CgWork& w, const int blk, const int nblk,
                                             unsigned& gen, double* sh, uint32_t* s_warp, uint32_t* s_list,
                                             SolverSetup& out, int layout)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const int sxy = nx * ny;
    const int nc = sxy * nz;
    const int T = nblk * blockDim.x;
    const int tid = solver_thread(blk, nblk);
    const uint8_t* __restrict__ marks = v.marks;
    double* __restrict__ p64 = v.p;
    const double* __restrict__ b = v.b;
    float* __restrict__ R[2] = {w.r0, w.r1};
    float* __restrict__ W[2] = {w.w0, w.w1};
    float* __restrict__ S[2] = {w.s0, w.s1};
    uint32_t* __restrict__ list = w.list;
    gen = 0;  // barriers passed in this launch

    // ---- setup: zero non-FLUID entries, ||b||^2, per-block FLUID counts over the block's cell range
    const int chunk = (nc + nblk - 1) / nblk;
    const int cb = min(nc, blk * chunk), ce = min(nc, cb + chunk);
    double acc[2] = {0.0, 0.0};
    for (int c = cb + threadIdx.x; c < ce; c += blockDim.x) {
        if (solve_mask(marks, c, nx, ny, nz) != 0u) {
            acc[0] += b[c] * b[c];
            acc[1] += 1.0;
        } else {
            p64[c] = 0.0;
            if (layout == kLayoutInterleaved) {  // the single-pass CG's (r, w, s, p) cells
                w.rws0[c] = make_float4(0.f, 0.f, 0.f, 0.f);
                w.rws1[c] = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                R[0][c] = 0.f;
                R[1][c] = 0.f;
                W[0][c] = 0.f;
                W[1][c] = 0.f;
                S[0][c] = 0.f;
                S[1][c] = 0.f;
                w.pv[c] = 0.f;
            }
        }
    }
    // block offset = FLUID count of all earlier blocks (fixed order), total = all blocks
    const double mine = block_sum1(acc[1], sh);
    if (threadIdx.x == 0) w.partial[kCgTotalsDoubles + blk] = mine;
    double tot[2] = {acc[0], acc[1]};
    if (!grid_reduce<2>(tot, sh, w, gen, nblk, blk)) return false;
    const double bnorm = sqrt(tot[0]);
    const int F = (int)tot[1];
    double before = 0.0;
    for (int bb = threadIdx.x; bb < blk; bb += blockDim.x) before += __ldcg(w.partial + kCgTotalsDoubles + bb);
    before = block_sum1(before, sh);
    // ordered compaction of this block's FLUID cells with their in-domain masks
    uint32_t base = (uint32_t)before;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int c0 = cb; c0 < ce; c0 += blockDim.x) {
        const int c = c0 + threadIdx.x;
        const uint32_t m = c < ce ? solve_mask(marks, c, nx, ny, nz) : 0u;
        const bool fl = m != 0u;
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
            const uint32_t slot = base + off + __popc(bal & ((1u << lane) - 1u));
            list[slot] = ((uint32_t)c << 6) | m;
        }
        base += total;
        __syncthreads();
    }
    if (!grid_sync(w, gen, nblk, sh, blk)) return false;
    const int kc = kListCache / (int)blockDim.x;
    {
        int k = 0;
        for (int e = tid; e < F && k < kc; e += T, ++k) s_list[k * blockDim.x + threadIdx.x] = __ldcg(list + e);
    }
    out.F = F;
    out.bnorm = bnorm;
    out.kc = kc;
    return true;
}

}  // namespace
}  // namespace fe
