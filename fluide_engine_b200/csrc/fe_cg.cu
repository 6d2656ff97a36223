// fe_cg.cu -- pressure solve: FP32 matrix-free conjugate gradient inside FP64 iterative refinement,
// as one persistent cooperative kernel per solve (K_cg).
//
// Reference system (fluid_solvers/single_phase_pressure_solver.cpp:99-164): for a FLUID cell, b = div u,
// diagonal = sum over in-domain non-BOUNDRY neighbours of 1/h_axis^2, off-diagonal -1/h_axis^2 toward
// FLUID neighbours; non-FLUID rows are identity with b = 0, so their solution is 0.  The reference solves
// it with unpreconditioned CG warm-started from the previous pressure (linear_system/
// conjugate_gradient_solver.cpp:14-55, linear_system.cpp:13-18).
//
// Here the FLUID-cell system is solved matrix-free from the cell marks (no stored matrix rows):
//   outer (FP64): r = b - A p, ||r||, convergence test ||r|| <= tol ||b||; p += e after each inner solve
//   inner (FP32): CG on A e = r, dot products accumulated in FP64, until the inner residual fell by
//                 cg_inner_tol (or far enough to meet the outer target)
// Each inner iteration is two passes separated by grid-wide reductions:
//   A: d' = r + beta d, q = A d' (neighbour d' recomputed from the neighbour r and d, so no extra pass),
//      partial d'.q
//   B: x += alpha d', r -= alpha q, partial r.r
// The grid-wide barrier is a counter + generation word with a bounded spin: if a block waits longer than
// ~3 s it records FE_ERR_TIMEOUT, every block leaves its loops and the kernel returns, so a stuck solve
// surfaces as a status instead of a hung device.  Partial sums are written per block and summed by every
// block in the same fixed order, so all blocks take identical branch decisions and results are
// deterministic.  Non-FLUID entries of every vector are held at 0, which makes the stencil branch-free.
#include "fe_internal.cuh"

#include <cuda/atomic>

namespace fe {
namespace {

constexpr int kCgThreads = 1024;
constexpr unsigned long long kSpinLimit = 1ull << 25;

struct CgParams {
    double rel_tol, inner_tol;
    int max_it, max_refine;
    fe_step_stats* stats_ring;
    unsigned* stats_counter;
    unsigned stats_cap;
};

__device__ __forceinline__ bool grid_sync(unsigned* bar, int* err, unsigned nblocks)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> count(bar[0]);
        cuda::atomic_ref<unsigned, cuda::thread_scope_device> gen(bar[1]);
        cuda::atomic_ref<int, cuda::thread_scope_device> e(*err);
        const unsigned g = gen.load(cuda::memory_order_acquire);
        __threadfence();
        if (count.fetch_add(1u, cuda::memory_order_acq_rel) == nblocks - 1) {
            count.store(0u, cuda::memory_order_relaxed);
            gen.store(g + 1u, cuda::memory_order_release);
        } else {
            unsigned long long spins = 0;
            while (gen.load(cuda::memory_order_acquire) == g) {
                if (e.load(cuda::memory_order_relaxed) != 0) break;
                if (++spins > kSpinLimit) {
                    e.store(FE_ERR_TIMEOUT, cuda::memory_order_relaxed);
                    break;
                }
                if (spins > 32) __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return *(volatile int*)err == 0;
}

// Block-wide sum of up to 4 doubles; result valid in all threads.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* sh /* [32 * N] */)
{
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
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double s = lane < nw ? sh[lane * N + k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            v[k] = s;
        }
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < N; ++k) sh[32 * N + k] = v[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = sh[32 * N + k];
    __syncthreads();
}

// Publishes this block's N partials, synchronises the grid and returns the grid-wide sums (identical in
// every block).  Returns false when the barrier gave up.
template <int N>
__device__ __forceinline__ bool grid_reduce(double (&v)[N], double* sh, const CgWork& w)
{
    block_sum<N>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < N; ++k) w.partial[blockIdx.x * 4 + k] = v[k];
    if (!grid_sync(w.bar, w.err, gridDim.x)) return false;
    double s[N];
#pragma unroll
    for (int k = 0; k < N; ++k) s[k] = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < N; ++k) s[k] += __ldcg(w.partial + b * 4 + k);
    block_sum<N>(s, sh);
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = s[k];
    return true;
}

__global__ void __launch_bounds__(kCgThreads, 1) k_cg(SceneView v, CgWork w, CgParams prm)
{
    __shared__ double sh[32 * 4 + 4];
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t sxy = (size_t)nx * ny;
    const size_t nc = sxy * nz;
    const size_t T = (size_t)gridDim.x * blockDim.x;
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const uint8_t* __restrict__ marks = v.marks;
    const double ih2d[3] = {v.inv_h[0] * v.inv_h[0], v.inv_h[1] * v.inv_h[1], v.inv_h[2] * v.inv_h[2]};
    const float ih2[3] = {(float)ih2d[0], (float)ih2d[1], (float)ih2d[2]};
    float* __restrict__ r = w.r;
    float* __restrict__ q = w.q;
    float* __restrict__ x = w.x;
    double* __restrict__ p = v.p;
    const double* __restrict__ b = v.b;

    // Pass 0: ||b||^2 and FLUID count; non-FLUID entries of p and of every FP32 vector set to 0.
    double acc[2] = {0.0, 0.0};
    for (size_t c = tid; c < nc; c += T) {
        if (marks[c] == FE_CELL_FLUID) {
            acc[0] += b[c] * b[c];
            acc[1] += 1.0;
        } else {
            p[c] = 0.0;
            r[c] = 0.f;
            w.d0[c] = 0.f;
            w.d1[c] = 0.f;
            q[c] = 0.f;
            x[c] = 0.f;
        }
    }
    if (!grid_reduce<2>(acc, sh, w)) return;
    const double bnorm = sqrt(acc[0]);
    const int fluid = (int)acc[1];
    const double target = prm.rel_tol * bnorm;

    int total_it = 0, refinements = 0;
    double rnorm = 0.0;
    bool converged = false;
    for (;;) {
        // Outer residual r = b - A p in FP64 (stored in FP32 for the inner solve).
        double racc[2] = {0.0, 0.0};
        for (size_t c = tid; c < nc; c += T) {
            if (marks[c] != FE_CELL_FLUID) continue;
            const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / sxy);
            const double pc = p[c];
            double ap = 0.0;
            if (i > 0) ap += ih2d[0] * (pc - p[c - 1]);
            if (i + 1 < nx) ap += ih2d[0] * (pc - p[c + 1]);
            if (j > 0) ap += ih2d[1] * (pc - p[c - nx]);
            if (j + 1 < ny) ap += ih2d[1] * (pc - p[c + nx]);
            if (k > 0) ap += ih2d[2] * (pc - p[c - sxy]);
            if (k + 1 < nz) ap += ih2d[2] * (pc - p[c + sxy]);
            const double rr = b[c] - ap;
            const float rf = (float)rr;
            r[c] = rf;
            x[c] = 0.f;
            w.d0[c] = 0.f;
            racc[0] += rr * rr;
            racc[1] += (double)rf * (double)rf;
        }
        if (!grid_reduce<2>(racc, sh, w)) return;
        rnorm = sqrt(racc[0]);
        if (rnorm <= target || bnorm == 0.0) {
            converged = true;
            break;
        }
        if (refinements >= prm.max_refine || total_it >= prm.max_it) break;
        ++refinements;

        // Inner FP32 CG on A e = r.
        double rho = racc[1];
        const double rho0 = rho;
        double want = fmax(prm.inner_tol, 0.25 * target / rnorm);
        const double stop = want * want * rho0;
        double beta = 0.0;
        int parity = 0;
        while (total_it < prm.max_it) {
            const float bf = (float)beta;
            float* __restrict__ dold = parity ? w.d1 : w.d0;
            float* __restrict__ dnew = parity ? w.d0 : w.d1;
            double a1[1] = {0.0};
            for (size_t c = tid; c < nc; c += T) {
                if (marks[c] != FE_CELL_FLUID) continue;
                const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / sxy);
                const float dn = r[c] + bf * dold[c];
                float ax = 0.f, ay = 0.f, az = 0.f;
                if (i > 0) ax += dn - (r[c - 1] + bf * dold[c - 1]);
                if (i + 1 < nx) ax += dn - (r[c + 1] + bf * dold[c + 1]);
                if (j > 0) ay += dn - (r[c - nx] + bf * dold[c - nx]);
                if (j + 1 < ny) ay += dn - (r[c + nx] + bf * dold[c + nx]);
                if (k > 0) az += dn - (r[c - sxy] + bf * dold[c - sxy]);
                if (k + 1 < nz) az += dn - (r[c + sxy] + bf * dold[c + sxy]);
                const float qq = ih2[0] * ax + ih2[1] * ay + ih2[2] * az;
                dnew[c] = dn;
                q[c] = qq;
                a1[0] += (double)dn * (double)qq;
            }
            if (!grid_reduce<1>(a1, sh, w)) return;
            if (!(a1[0] > 0.0)) break;  // breakdown (A d = 0): nothing left to reduce in FP32
            const double alpha = rho / a1[0];
            const float af = (float)alpha;
            double a2[1] = {0.0};
            for (size_t c = tid; c < nc; c += T) {
                if (marks[c] != FE_CELL_FLUID) continue;
                x[c] += af * dnew[c];
                const float rn = r[c] - af * q[c];
                r[c] = rn;
                a2[0] += (double)rn * (double)rn;
            }
            if (!grid_reduce<1>(a2, sh, w)) return;
            ++total_it;
            beta = a2[0] / rho;
            rho = a2[0];
            parity ^= 1;
            if (rho <= stop) break;
        }
        // p += e (FP64); the next residual pass reads neighbours' p, hence the barrier.
        for (size_t c = tid; c < nc; c += T)
            if (marks[c] == FE_CELL_FLUID) p[c] += (double)x[c];
        if (!grid_sync(w.bar, w.err, gridDim.x)) return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && prm.stats_ring) {
        const unsigned slot = atomicAdd(prm.stats_counter, 1u) % prm.stats_cap;
        fe_step_stats s;
        s.cg_iterations = total_it;
        s.refinements = refinements;
        s.converged = converged ? 1 : 0;
        s.fluid_cells = fluid;
        s.rel_residual = bnorm > 0.0 ? rnorm / bnorm : rnorm;
        s.b_norm = bnorm;
        prm.stats_ring[slot] = s;
    }
}

}  // namespace

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
