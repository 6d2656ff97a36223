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
//              A cell's (r, w, s, p) sit together in one float4, so a neighbour costs one 16-byte load and
//              the cell's new state one 16-byte store.
// The grid-wide barrier is an arrival count polled with a bounded spin: if a block waits longer than a few
// seconds it records FE_ERR_TIMEOUT, every block leaves its loops and the kernel returns, so a stuck solve
// surfaces as a status instead of a hung device.  Dot products travel with the barrier: blocks add their
// partials into a rotating totals slot before arriving and read the totals once after it, so all blocks take
// identical branch decisions.
#include <algorithm>

#include "fe_solver_common.cuh"
#include "fe_mg_body.cuh"

namespace fe {
namespace {

constexpr int kCgThreads = 1024;
constexpr int kMultiThreads = 256;

// The solver body, run by `nblk` blocks of which this is block `blk` (a whole grid for one scene, or a
// block range of a multi-scene launch, see k_multi_cg); every barrier and reduction spans those blocks.
__device__ __forceinline__ void cg_body(SolverSmem& smem, const SceneView& v, const CgWork& w, const CgParams& prm,
                                        const int blk, const int nblk, int* out_its = nullptr, int* out_fluid = nullptr)
{
    double* sh = smem.sh;
    uint32_t* s_warp = smem.s_warp;
    // the FLUID list does not change during a solve: each thread keeps its first list entries in shared
    // memory (entry k of thread t at s_list[k * blockDim.x + t]), which takes one dependent L2 round trip
    // out of every pass
    uint32_t* s_list = smem.s_list;
    const int nx = v.g.nx, ny = v.g.ny;
    const int sxy = nx * ny;
    const int T = nblk * blockDim.x;
    const int tid = solver_thread(blk, nblk);
    const double ih2d[3] = {v.inv_h[0] * v.inv_h[0], v.inv_h[1] * v.inv_h[1], v.inv_h[2] * v.inv_h[2]};
    Stencil7 st;
    st.sx = nx;
    st.sxy = sxy;
    st.ih2[0] = (float)ih2d[0];
    st.ih2[1] = (float)ih2d[1];
    st.ih2[2] = (float)ih2d[2];
    double* __restrict__ p64 = v.p;
    const double* __restrict__ b = v.b;
    float4* __restrict__ Q[2] = {w.rws0, w.rws1};  // (r, w, s, p) per cell
    float* __restrict__ R0 = reinterpret_cast<float*>(w.rws0);  // r of cell c at R0[4 c]
    float* __restrict__ X = w.xcg;
    uint32_t* __restrict__ list = w.list;

    unsigned gen = 0;
    SolverSetup su;
    if (!solver_setup(v, w, blk, nblk, gen, sh, s_warp, s_list, su, kLayoutInterleaved)) return;
    const int F = su.F, kc = su.kc;
    const double bnorm = su.bnorm;
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
            R0[4 * (size_t)c] = (float)rr;
            racc[0] += rr * rr;
        }
        cur = 0;
        if (!grid_reduce<1>(racc, sh, w, gen, nblk, blk)) return;
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
            const float wc = apply_row(st, c, ent & 63u, [&](int q) { return R0[4 * (size_t)q]; });
            const float rc = R0[4 * (size_t)c];
            Q[0][c] = make_float4(rc, wc, 0.f, 0.f);
            X[c] = 0.f;
            d0[0] += (double)rc * (double)rc;
            d0[1] += (double)wc * (double)rc;
        }
        if (!grid_reduce<2>(d0, sh, w, gen, nblk, blk)) return;
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
            const float4* __restrict__ q0 = Q[cur];
            float4* __restrict__ q1 = Q[cur ^ 1];
            double dd[2] = {0.0, 0.0};
            for (int e = tid, k = 0; e < F; e += T, ++k) {
                const uint32_t ent = entry(k, e);
                const int c = (int)(ent >> 6);
                // r'(q) = r(q) - alpha (w(q) + beta s(q)) for this cell and its neighbours
                auto rnew = [&](int q) {
                    const float4 t = q0[q];
                    return t.x - af * (t.y + bf * t.z);
                };
                const float4 me = q0[c];
                const float snew = me.y + bf * me.z;
                const float pnew = me.x + bf * me.w;
                const float rc = me.x - af * snew;
                const float wc = apply_row(st, c, ent & 63u, rnew);
                X[c] += af * pnew;
                q1[c] = make_float4(rc, wc, snew, pnew);
                dd[0] += (double)rc * (double)rc;
                dd[1] += (double)wc * (double)rc;
            }
            if (!grid_reduce<2>(dd, sh, w, gen, nblk, blk)) return;
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
        if (!grid_sync(w, gen, nblk, sh, blk)) return;
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
    __shared__ SolverSmem smem;
    cluster_begin(w, smem.sh);
    cg_body(smem, v, w, prm, blockIdx.x, gridDim.x);
    solver_exit(w, gridDim.x);
    cluster_end(w);
}

// The same solve with the multigrid-preconditioned inner loop (fe_mg_body.cuh).
__global__ void __launch_bounds__(kCgThreads, 1) k_mgcg(SceneView v, CgWork w, MgWork mg, CgParams prm)
{
    __shared__ SolverSmem smem;
    cluster_begin(w, smem.sh);
    mg_body(smem, v, w, mg, prm, blockIdx.x, gridDim.x);
    solver_exit(w, gridDim.x);
    cluster_end(w);
}

// Many scenes in one cooperative launch: blocks [start[s], start[s+1]) solve scene s with their own barrier
// and reductions, so scenes iterate independently and concurrently.  Each scene runs the solver body it runs
// alone: the plain CG body, or the multigrid-preconditioned body for scenes tuned to it (both fit the kernel's
// register budget of 3 co-resident 256-thread blocks per SM).
__global__ void __launch_bounds__(kMultiThreads, 3) k_multi_cg(MultiCgScene* __restrict__ scenes, int S)
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
    prm.stats_cap = m.work.stats_cap;
    int its = 0, fluid = 0;
    const int blk = (int)blockIdx.x - m.block_start;
    __shared__ SolverSmem smem;
    if (m.use_mg) mg_body(smem, m.view, m.work, m.mg, prm, blk, m.block_count, &its, &fluid);
    else cg_body(smem, m.view, m.work, prm, blk, m.block_count, &its, &fluid);
    solver_exit(m.work, m.block_count);
    if (blk == 0 && threadIdx.x == 0) {  // read by the next solve's k_multi_partition
        m.last_its = its;
        m.last_fluid = fluid;
    }
}

// Relative cost of one inner iteration per FLUID cell: the multigrid body's passes and grid barriers (4 L - 2 per
// iteration) against the plain body's one.
__device__ __forceinline__ double multi_work(const MultiCgScene& m)
{
    if (m.last_its < 0) return m.weight0;
    const double per_it = m.use_mg ? 12.0 : 1.0;
    return (double)m.last_fluid * ((double)m.last_its * per_it + 3.0);
}

// Splits total_blocks among the scenes before a multi-scene solve: one block each, the rest in proportion to the
// previous solve's work of the scene (FLUID cells x (inner iterations + 3 residual passes); weight0 before its
// first solve), the leftovers (fewer than S) one each to the scenes with the most work per block.  Scenes then
// take about equally long, instead of the scene with the most iterations finishing last on a small share.  One
// thread per scene (S <= kBatchMaxScenes): each scene's work is read once into shared memory, and the ranking of the
// leftovers runs in parallel, so the split costs a few microseconds rather than S^2 dependent global reads.
__global__ void __launch_bounds__(kBatchMaxScenes) k_multi_partition(MultiCgScene* __restrict__ scenes, int S,
                                                                       int total_blocks)
{
    __shared__ double w[kBatchMaxScenes];
    __shared__ int cnt[kBatchMaxScenes];
    __shared__ int start[kBatchMaxScenes];
    __shared__ double wsum_s;
    __shared__ int left_s;
    const int t = threadIdx.x;
    w[t] = t < S ? fmax(multi_work(scenes[t]), 0.0) : 0.0;
    __syncthreads();
    if (t == 0) {
        double wsum = 0.0;
        for (int i = 0; i < S; ++i) wsum += w[i];  // in scene order
        wsum_s = wsum;
    }
    __syncthreads();
    const int spare = total_blocks - S;
    const double wsum = wsum_s;
    if (t < S) cnt[t] = 1 + (wsum > 0.0 ? (int)floor(spare * (w[t] / wsum)) : spare / S);
    __syncthreads();
    if (t == 0) {
        int used = 0;
        for (int i = 0; i < S; ++i) used += cnt[i];
        left_s = total_blocks - used;
    }
    __syncthreads();
    // rank by work per block, heaviest first, ties to the lower index
    int rank = S;
    if (t < S) {
        const double key = w[t] / (double)cnt[t];
        rank = 0;
        for (int j = 0; j < S; ++j) {
            const double kj = w[j] / (double)cnt[j];
            rank += (kj > key || (kj == key && j < t)) ? 1 : 0;
        }
    }
    __syncthreads();  // every rank read the counts before any changes
    if (t < S && rank < left_s) cnt[t] += 1;
    __syncthreads();
    if (t == 0) {
        int st = 0;
        for (int i = 0; i < S; ++i) {
            start[i] = st;
            st += cnt[i];
        }
    }
    __syncthreads();
    if (t < S) {
        scenes[t].block_count = cnt[t];
        scenes[t].block_start = start[t];
    }
}

}  // namespace

cudaError_t set_solver_barrier_limits(unsigned long long spin_limit, unsigned extra_arrivals)
{
    const unsigned long long lim = spin_limit ? spin_limit : kSpinLimit;
    cudaError_t e = cudaMemcpyToSymbol(c_spin_limit, &lim, sizeof(lim));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(c_extra_arrivals, &extra_arrivals, sizeof(extra_arrivals));
}

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
    k_multi_partition<<<1, kBatchMaxScenes, 0, st>>>(scenes, S, total_blocks);
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

cudaError_t cg_prepare(CgWork& w, int device, int threads, int cluster)
{
    if (threads != 256 && threads != 512 && threads != 1024) return cudaErrorInvalidValue;
    if (cluster < 1) cluster = 1;
    if (cluster > kMaxCluster || (cluster & (cluster - 1)) != 0) return cudaErrorInvalidValue;
    int sms = 0, per_sm = 0, per_sm_mg = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg, threads, 0);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_mg, k_mgcg, threads, 0);
    if (e != cudaSuccess) return e;
    // persistent blocks: as many per SM as fill 1024 threads, all co-resident (a cooperative launch)
    const int want = kCgThreads / threads;
    const int per = std::min(want, std::min(per_sm, per_sm_mg));
    if (per < 1) return cudaErrorCooperativeLaunchTooLarge;
    int blocks = sms * per;
    if (cluster > 1) {
        // whole clusters only, as many as the device holds at once for both solver kernels
        int clusters = blocks / cluster;
        for (int kind = 0; kind < 2; ++kind) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)(clusters * cluster));
            cfg.blockDim = dim3((unsigned)threads);
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = (unsigned)cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int n = 0;
            e = kind == 0 ? cudaOccupancyMaxActiveClusters(&n, k_cg, &cfg) : cudaOccupancyMaxActiveClusters(&n, k_mgcg, &cfg);
            if (e != cudaSuccess) return e;
            clusters = std::min(clusters, n);
        }
        if (clusters < 1) return cudaErrorCooperativeLaunchTooLarge;
        blocks = clusters * cluster;
    }
    if (blocks > kMaxCgBlocks) return cudaErrorCooperativeLaunchTooLarge;
    w.blocks = blocks;
    w.threads = threads;
    w.cluster = cluster;
    return cudaSuccess;
}

int mg_plan(int nx, int ny, int nz, const double h[3], MgLevel* out)
{
    int n[3] = {nx, ny, nz};
    double hh[3] = {h[0], h[1], h[2]};
    int levels = 0;
    while (true) {
        MgLevel& L = out[levels];
        L = MgLevel{};
        L.nx = n[0];
        L.ny = n[1];
        L.nz = n[2];
        for (int a = 0; a < 3; ++a) L.ih2[a] = (float)(1.0 / (hh[a] * hh[a]));
        ++levels;
        if (std::max(n[0], std::max(n[1], n[2])) <= 8 || levels == kMaxMgLevels) break;
        for (int a = 0; a < 3; ++a) {
            n[a] = (n[a] + 1) / 2;
            hh[a] *= 2.0;
        }
    }
    // the last level is solved in one block's shared memory: it must have at most 512 cells
    if (levels < 2 || out[levels - 1].nx * out[levels - 1].ny * out[levels - 1].nz > kCoarseMaxCells) return 1;
    return levels;
}

int mg_block_from(const MgLevel* lv, int levels, int block_cells)
{
    int b = levels - 1;
    while (b > 1 && (size_t)lv[b - 1].nx * lv[b - 1].ny * lv[b - 1].nz <= (size_t)block_cells) --b;
    return b;
}

cudaError_t launch_mgcg(const SceneView& v, const CgWork& w, const MgWork& mg, double rel_tol, double inner_tol,
                        int max_it, int max_refine, cudaStream_t st)
{
    CgParams prm;
    prm.rel_tol = rel_tol;
    prm.inner_tol = inner_tol;
    prm.max_it = max_it;
    prm.max_refine = max_refine;
    prm.stats_ring = w.stats;
    prm.stats_counter = (unsigned*)(w.bar + 2);
    prm.stats_cap = w.stats_cap;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)w.blocks);
    cfg.blockDim = dim3((unsigned)w.threads);
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = (unsigned)std::max(w.cluster, 1);
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = w.cluster > 1 ? 2 : 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_mgcg, v, w, mg, prm);
    count_launch();
    return e;
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
    prm.stats_cap = w.stats_cap;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)w.blocks);
    cfg.blockDim = dim3((unsigned)w.threads);
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = (unsigned)std::max(w.cluster, 1);
    attr[1].val.clusterDim.y = 1;
    attr[1].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = w.cluster > 1 ? 2 : 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k_cg, v, w, prm);
    count_launch();
    return e;
}

}  // namespace fe
