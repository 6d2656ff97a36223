// fe_mg_body.cuh -- multigrid-preconditioned conjugate gradient for the pressure system, as the body of a
// persistent cooperative kernel (k_mgcg, and per scene inside k_multi_cg).
//
// Same system, same FP64 outer refinement and same convergence test as the plain solver (fe_cg.cu; the
// reference system of single_phase_pressure_solver.cpp:99-164 with the reference's relative residual
// target); only the inner FP32 solve of A e = r changes: preconditioned CG whose preconditioner is one
// multigrid V-cycle, which needs about 10-20 inner iterations for a 1e-6 reduction at 32^3..256^3 instead
// of the plain CG's 130..1100.  Results agree with the plain solver and with the reference to the solve
// tolerance (both stop on the same FP64 residual test).
//
// Hierarchy: level l >= 1 halves every axis of level l-1 (rounding up) until the largest axis is <= 8;
// a coarse cell holds fluid when most of its children do (more than half of those inside the grid: 5 of 8); the operator of level l is the same 7-point matrix on the
// coarse cells with spacing 2^l h (AIR neighbours Dirichlet 0, walls Neumann).
// V-cycle (symmetric, so the preconditioner is SPD): one damped-Jacobi sweep (omega = kOmega) down, starting
// from zero (z1 = omega r / D, pointwise, never stored: recomputed wherever a pass needs it); residual;
// restriction = kRestrictScale x the transpose of the prolongation; the coarsest level gets kCoarseSweeps
// Jacobi sweeps from zero in one block's shared memory; up: z = z1 + P z_coarse, then one Jacobi sweep.
// P is cell-centred trilinear: per axis a fine cell takes 3/4 of its parent and 1/4 of the parent's
// neighbour on its side (the parent again at a wall).
//
// Passes (grid barriers) per inner iteration, L levels: A: x, r update fused with level 0's pre-smoothing,
// its residual and the residual's restriction to level 1 (scattered into level 1's right-hand side; carries
// ||r||^2); per level 1 .. L-2 its residual, restricted the same way; the coarsest solve; per level L-2 .. 1
// the pre-smoothed correction z1 + P z_coarse, then the post-smoothing sweep; the same two for level 0 (the
// second carries (r, z)); the search direction p = z + beta p, q = A p (carries (p, q)).  3 L - 1 barriers.
// Each pass computes every value once and stores it (a level's scratch array t, and for level 0 the residual
// vector); neighbours' values of vectors that are updated pointwise (r, p) are recomputed from their stable
// previous values, as in the plain solver.  (Recomputing the pre-smoothed correction at the neighbours inside
// the smoothing sweep, which saves a barrier per level going up, measured slower: 124 against 95 us per inner
// iteration at 128^3.)
#pragma once

#include "fe_solver_common.cuh"

namespace fe {
namespace {

// Jacobi damping of the smoother.  The iteration matrix I - omega D^-1 A contracts for omega < 1 on these M-matrices
// (Gershgorin: D^-1 A has its spectrum in [0, 2]), which keeps the V-cycle symmetric positive definite.  Swept over
// the 240-substep 128^3 dam break (inner iterations, ms per solve): 0.6 27.0 / 2.25, 2/3 26.0 / 2.17, 0.75 24.2 /
// 2.03, 0.8 23.7 / 1.99, 0.85 23.0 / 1.93, 0.9 22.6 / 1.91, 0.95 25.2 / 2.11; 0.9 was also the faster of 0.85 / 0.9
// at 48^3, 64^3, 96^3 and on the 256^3 APIC pool to 1e-8.
constexpr float kOmega = 0.9f;
// Scale of the restriction (the transpose of the trilinear prolongation): 0.0875 / 0.1 / 0.125 gave 25.2 / 26.0 /
// 28.5 inner iterations at omega 2/3 and 22.6 / 22.6 / - at 0.9 on the same run.
constexpr float kRestrictScale = 0.1f;
// Jacobi sweeps from zero on the coarsest level.  Measured over the 240-substep 128^3 dam break (inner iterations,
// ms per solve): 4 sweeps 26.8 / 2.20, 8 25.8 / 2.15, 11 25.8 / 2.16, 15 25.6 / 2.17, 20 25.6 / 2.20, 30 26.0 / 2.28,
// 45 26.4 / 2.41 -- solving the coarsest level more exactly does not pay: its fluid-if-any-child operator is only a
// rough model of the fine one near the free surface, and each sweep costs one block barrier on one SM.
constexpr int kCoarseSweeps = 10;

__device__ __forceinline__ float level_diag(int i, int j, int k, int nx, int ny, int nz, const float* ih2)
{
    return ih2[0] * (float)((i > 0) + (i < nx - 1)) + ih2[1] * (float)((j > 0) + (j < ny - 1)) +
           ih2[2] * (float)((k > 0) + (k < nz - 1));
}

// The Jacobi scale omega / D of cell (i, j, k).  Every pass that applies the smoother (or recomputes a
// neighbour's pre-smoothed value) takes it from here, so the V-cycle applies one operator throughout and
// stays symmetric; the fast division is within 2 ulp of omega / D.
__device__ __forceinline__ float wdiag(int i, int j, int k, int nx, int ny, int nz, const float* ih2)
{
    return __fdividef(kOmega, level_diag(i, j, k, nx, ny, nz, ih2));
}

// Per axis: the two coarse indices of a fine index i and their prolongation weights (the parent twice at
// a wall, 0.75 + 0.25).
__device__ __forceinline__ void prolong_axis(int i, int nc, int& c0, int& c1)
{
    c0 = i >> 1;
    c1 = (i & 1) ? c0 + 1 : c0 - 1;
    if (c1 < 0 || c1 >= nc) c1 = c0;
}

// (P zc)(i, j, k) on the fine level of `fine` (unmasked).
__device__ __forceinline__ float prolong_at(const MgLevel& coarse, int i, int j, int k)
{
    int i0, i1, j0, j1, k0, k1;
    prolong_axis(i, coarse.nx, i0, i1);
    prolong_axis(j, coarse.ny, j0, j1);
    prolong_axis(k, coarse.nz, k0, k1);
    // one 64-bit index for the parent, 32-bit steps (-1, 0 or +1 cell per axis) to the other corners
    const int sx = coarse.nx, sxy = coarse.nx * coarse.ny;
    const float* p = coarse.z + ((size_t)i0 + (size_t)sx * (size_t)j0 + (size_t)sxy * (size_t)k0);
    const int dx = i1 - i0, dy = (j1 - j0) * sx, dz = (k1 - k0) * sxy;
    const float y00 = 0.75f * p[0] + 0.25f * p[dx];
    const float y10 = 0.75f * p[dy] + 0.25f * p[dx + dy];
    const float y01 = 0.75f * p[dz] + 0.25f * p[dx + dz];
    const float y11 = 0.75f * p[dy + dz] + 0.25f * p[dx + dy + dz];
    const float x0 = 0.75f * y00 + 0.25f * y10;
    const float x1 = 0.75f * y01 + 0.25f * y11;
    return 0.75f * x0 + 0.25f * x1;
}

// Level-l residual of the pre-smoothed correction, res = r - A (omega r / D), at cell (i, j, k) of a dense
// level (0 outside the mask); r outside the mask (where the restriction scatter may have added) counts as 0.
__device__ __forceinline__ float level_residual(const MgLevel& L, int i, int j, int k)
{
    const size_t sx = (size_t)L.nx, sxy = (size_t)L.nx * L.ny;
    const size_t c = (size_t)i + sx * j + sxy * k;
    if (!L.mask[c]) return 0.f;
    auto z1 = [&](int a, int b, int d) {
        const size_t q = (size_t)a + sx * b + sxy * d;
        return L.mask[q] ? L.r[q] * wdiag(a, b, d, L.nx, L.ny, L.nz, L.ih2) : 0.f;
    };
    const float rc = L.r[c];
    const float zc = rc * wdiag(i, j, k, L.nx, L.ny, L.nz, L.ih2);
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (i > 0) ax += zc - z1(i - 1, j, k);
    if (i + 1 < L.nx) ax += zc - z1(i + 1, j, k);
    if (j > 0) ay += zc - z1(i, j - 1, k);
    if (j + 1 < L.ny) ay += zc - z1(i, j + 1, k);
    if (k > 0) az += zc - z1(i, j, k - 1);
    if (k + 1 < L.nz) az += zc - z1(i, j, k + 1);
    return rc - (L.ih2[0] * ax + L.ih2[1] * ay + L.ih2[2] * az);
}

// One damped-Jacobi sweep z = t + omega (r - A t) / D at (i, j, k) of level L from the stored t (0 outside
// the mask).
__device__ __forceinline__ float level_smooth(const MgLevel& L, int i, int j, int k)
{
    const size_t sx = (size_t)L.nx, sxy = (size_t)L.nx * L.ny;
    const size_t c = (size_t)i + sx * j + sxy * k;
    if (!L.mask[c]) return 0.f;
    const float* t = L.t;
    const float tc = t[c];
    float ax = 0.f, ay = 0.f, az = 0.f;
    if (i > 0) ax += tc - t[c - 1];
    if (i + 1 < L.nx) ax += tc - t[c + 1];
    if (j > 0) ay += tc - t[c - sx];
    if (j + 1 < L.ny) ay += tc - t[c + sx];
    if (k > 0) az += tc - t[c - sxy];
    if (k + 1 < L.nz) az += tc - t[c + sxy];
    const float At = L.ih2[0] * ax + L.ih2[1] * ay + L.ih2[2] * az;
    return tc + (L.r[c] - At) * wdiag(i, j, k, L.nx, L.ny, L.nz, L.ih2);
}

// Restriction = kRestrictScale x the transpose of the prolongation, as a scatter: fine cell (i, j, k) with residual
// `val` adds kRestrictScale x its prolongation weight x val into every coarse cell whose prolongation reaches it
// (up to 2 per axis; the parent twice at a wall, weight 1), with FP32 atomics into C.r, which must start at zero.
// It lets the pass that computes a level's residual restrict it too, without a barrier and a gather pass between
// them (each coarse cell's sum is formed in arrival order).  Coarse cells outside the mask receive terms too (a
// fine cell at the fluid's edge reaches a parent with no fluid child); every reader of C.r ignores it outside the
// mask, so no mask load stands between the residual and its atomics.
__device__ __forceinline__ void restrict_scatter(const MgLevel& C, int i, int j, int k, float val)
{
    if (val == 0.f) return;
    int i0, i1, j0, j1, k0, k1;
    prolong_axis(i, C.nx, i0, i1);
    prolong_axis(j, C.ny, j0, j1);
    prolong_axis(k, C.nz, k0, k1);
    const int ii[2] = {i0, i1}, jj[2] = {j0, j1}, kk[2] = {k0, k1};
    const float wi[2] = {i1 == i0 ? 1.f : 0.75f, i1 == i0 ? 0.f : 0.25f};
    const float wj[2] = {j1 == j0 ? 1.f : 0.75f, j1 == j0 ? 0.f : 0.25f};
    const float wk[2] = {k1 == k0 ? 1.f : 0.75f, k1 == k0 ? 0.f : 0.25f};
    const float sv = kRestrictScale * val;
    const size_t sx = (size_t)C.nx, sxy = (size_t)C.nx * C.ny;
#pragma unroll
    for (int d = 0; d < 8; ++d) {
        const int a = d & 1, b = (d >> 1) & 1, e = d >> 2;
        const float wgt = wi[a] * wj[b] * wk[e];
        if (wgt == 0.f) continue;
        atomicAdd(C.r + (size_t)ii[a] + sx * (size_t)jj[b] + sxy * (size_t)kk[e], wgt * sv);
    }
}

// The solver body, run by `nblk` blocks of which this is block `blk`; every barrier and reduction spans
// those blocks.  Vectors: r (ping-pong r0/r1), z (w0), q = A p (w1), p (ping-pong s0/s1), the level-0
// residual (pv, 0 outside FLUID), x (the inner solve's correction).
__device__ __forceinline__ void mg_body(SolverSmem& smem, const SceneView& v, const CgWork& w, const MgWork& mg,
                                        const CgParams& prm, const int blk, const int nblk, int* out_its = nullptr,
                                        int* out_fluid = nullptr)
{
    double* sh = smem.sh;
    uint32_t* s_warp = smem.s_warp;
    uint32_t* s_list = smem.s_list;
    float (*s_cz)[kCoarseMaxCells] = smem.cz;
    float* s_cr = smem.cr;
    float* s_cw = smem.cw;
    uint8_t* s_cb = smem.cb;
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const int sxy = nx * ny;
    const int T = nblk * blockDim.x;
    const int tid = solver_thread(blk, nblk);
    const uint8_t* __restrict__ marks = v.marks;
    const double ih2d[3] = {v.inv_h[0] * v.inv_h[0], v.inv_h[1] * v.inv_h[1], v.inv_h[2] * v.inv_h[2]};
    const float ih2[3] = {(float)ih2d[0], (float)ih2d[1], (float)ih2d[2]};
    double* __restrict__ p64 = v.p;
    const double* __restrict__ b = v.b;
    float* __restrict__ R[2] = {w.r0, w.r1};
    float* __restrict__ Z = w.w0;
    float* __restrict__ Q = w.w1;
    float* __restrict__ P[2] = {w.s0, w.s1};
    float* __restrict__ RES = w.pv;
    float* __restrict__ X = w.x;
    uint32_t* __restrict__ list = w.list;
    const int L = mg.levels;

    unsigned gen = 0;
    SolverSetup su;
    if (!solver_setup(v, w, blk, nblk, gen, sh, s_warp, s_list, su, kLayoutSeparate)) return;
    const int F = su.F, kc = su.kc;
    const double bnorm = su.bnorm;
    auto entry = [&](int k, int e) -> uint32_t { return k < kc ? s_list[k * blockDim.x + threadIdx.x] : list[e]; };

    // coarse-level masks, finest first (level 1 from the cell marks): a coarse cell is fluid when more than half of
    // its children are.  Marking it fluid when any child is (a free surface moved outward by up to a coarse cell)
    // models the fine operator poorly where the surface is thin and ragged; measured over the 240-substep 128^3 dam
    // break, inner iterations with "at least k of 8 children": any 22.6, 2 21.0, 3 18.8, 4 17.2, 5 14.6, 6 14.9,
    // 8 17.2 (ms per solve 1.91 / 1.78 / 1.61 / 1.48 / 1.28 / 1.30 / 1.47).  Masks, restriction and prolongation
    // stay a transpose pair, so the V-cycle stays symmetric positive definite for any such choice.
    for (int l = 1; l < L; ++l) {
        const MgLevel& C = mg.lv[l];
        const MgLevel& Fl = mg.lv[l - 1];
        const int ncells = C.nx * C.ny * C.nz;
        for (int t = tid; t < ncells; t += T) {
            const int I = t % C.nx, J = (t / C.nx) % C.ny, K = t / (C.nx * C.ny);
            int fluid = 0, children = 0;
            for (int dk = 0; dk < 2; ++dk)
                for (int dj = 0; dj < 2; ++dj)
                    for (int di = 0; di < 2; ++di) {
                        const int i = 2 * I + di, j = 2 * J + dj, k = 2 * K + dk;
                        if (i >= Fl.nx || j >= Fl.ny || k >= Fl.nz) continue;
                        const size_t f = (size_t)i + (size_t)Fl.nx * j + (size_t)Fl.nx * Fl.ny * k;
                        fluid += l == 1 ? (marks[f] == FE_CELL_FLUID ? 1 : 0) : (Fl.mask[f] ? 1 : 0);
                        ++children;
                    }
            C.mask[t] = 2 * fluid > children ? 1 : 0;
        }
        if (!grid_sync(w, gen, nblk, sh, blk)) return;
    }

    // the coarse right-hand sides start every V-cycle at zero, because the restriction scatters into them: cleared
    // in the outer residual pass and in the level-0 correction pass, which no pass reading them shares
    auto zero_coarse = [&]() {
        for (int l = 1; l < L; ++l) {
            const MgLevel& C = mg.lv[l];
            const int ncells = C.nx * C.ny * C.nz;
            for (int t = tid; t < ncells; t += T) C.r[t] = 0.f;
        }
    };
    const double target = prm.rel_tol * bnorm;
    if (bnorm == 0.0) {
        for (int e = tid; e < F; e += T) p64[list[e] >> 6] = 0.0;
    }
    int total_it = 0, refinements = 0;
    double rnorm = 0.0;
    bool converged = bnorm == 0.0;
    while (!converged) {
        // ---- outer residual r = b - A p in FP64, stored in FP32; the inner solve's vectors start at zero
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
            X[c] = 0.f;
            Q[c] = 0.f;
            P[0][c] = 0.f;
            racc[0] += rr * rr;
        }
        zero_coarse();
        if (!grid_reduce<1>(racc, sh, w, gen, nblk, blk)) return;
        rnorm = sqrt(racc[0]);
        if (rnorm <= target) {
            converged = true;
            break;
        }
        if (refinements >= prm.max_refine || total_it >= prm.max_it) break;
        ++refinements;

        // ---- inner MG-preconditioned CG on A e = r
        const double want = fmax(prm.inner_tol, 0.25 * target / rnorm);
        double stop = 0.0, rho_old = 1.0;
        float alpha = 0.f;
        int cur = 0, pc = 0;  // ping-pong indices of r and p
        bool first = true;
        const Stencil7 st0{nx, sxy, {ih2[0], ih2[1], ih2[2]}};
        while (true) {
            // pass A: x += alpha p, r' = r - alpha q; level 0 pre-smoothing z1 = omega r' / D and its residual
            {
                const float* __restrict__ r = R[cur];
                float* __restrict__ rn = R[cur ^ 1];
                const float* __restrict__ p = P[pc];
                double acc[1] = {0.0};
                for (int e = tid, k = 0; e < F; e += T, ++k) {
                    const uint32_t ent = entry(k, e);
                    const int c = (int)(ent >> 6);
                    const int ci = c % nx, cj = (c / nx) % ny, ck = c / sxy;
                    // neighbour q = c + offset along axis a at coordinate x: D(q) from its coordinates
                    auto z1 = [&](int q) {
                        const int qi = ci + (q == c - 1 ? -1 : q == c + 1 ? 1 : 0);
                        const int qj = cj + (q == c - nx ? -1 : q == c + nx ? 1 : 0);
                        const int qk = ck + (q == c - sxy ? -1 : q == c + sxy ? 1 : 0);
                        return (r[q] - alpha * Q[q]) * wdiag(qi, qj, qk, nx, ny, nz, ih2);
                    };
                    const float rc = r[c] - alpha * Q[c];
                    const float Az1 = apply_row(st0, c, ent & 63u, z1);
                    X[c] += alpha * p[c];
                    rn[c] = rc;
                    restrict_scatter(mg.lv[1], ci, cj, ck, rc - Az1);  // level-0 residual, restricted to level 1
                    acc[0] += (double)rc * (double)rc;
                }
                if (!grid_reduce<1>(acc, sh, w, gen, nblk, blk)) return;
                cur ^= 1;
                if (first) stop = want * want * acc[0];
                else ++total_it;
                if (acc[0] <= stop || !(acc[0] == acc[0]) || total_it >= prm.max_it) break;
            }
            // Per level: the residual, scattered into the next level's r by the restriction (going down);
            // pre-smoothed correction t = z1 + P z_next, one Jacobi sweep into z (going up).  `sync` separates the passes:
            // a grid barrier for the large levels, a block barrier (after a fence that publishes the block's
            // writes to its own L2 reads) for the levels [block_from, L) that the first block processes alone.
            auto level_down = [&](int l, int t0, int stride, auto sync) -> bool {
                const MgLevel& Fl = mg.lv[l];
                const MgLevel& C = mg.lv[l + 1];
                const int nf = Fl.nx * Fl.ny * Fl.nz;
                for (int t = t0; t < nf; t += stride) {
                    const int i = t % Fl.nx, j = (t / Fl.nx) % Fl.ny, k = t / (Fl.nx * Fl.ny);
                    restrict_scatter(C, i, j, k, level_residual(Fl, i, j, k));
                }
                return sync();
            };
            auto level_up = [&](int l, int t0, int stride, auto sync) -> bool {
                const MgLevel& Fl = mg.lv[l];
                const MgLevel& C = mg.lv[l + 1];
                const int nf = Fl.nx * Fl.ny * Fl.nz;
                for (int t = t0; t < nf; t += stride) {
                    const int i = t % Fl.nx, j = (t / Fl.nx) % Fl.ny, k = t / (Fl.nx * Fl.ny);
                    float val = 0.f;
                    if (Fl.mask[t])
                        val = Fl.r[t] * wdiag(i, j, k, Fl.nx, Fl.ny, Fl.nz, Fl.ih2) +
                              prolong_at(C, i, j, k);
                    Fl.t[t] = val;
                }
                if (!sync()) return false;
                for (int t = t0; t < nf; t += stride) {
                    const int i = t % Fl.nx, j = (t / Fl.nx) % Fl.ny, k = t / (Fl.nx * Fl.ny);
                    Fl.z[t] = level_smooth(Fl, i, j, k);
                }
                return sync();
            };
            auto gsync = [&]() { return grid_sync(w, gen, nblk, sh, blk); };
            auto bsync = [&]() {
                __threadfence();
                __syncthreads();
                return true;
            };
            const int LB = mg.block_from;
            for (int l = 1; l < LB; ++l)
                if (!level_down(l, tid, T, gsync)) return;
            if (blk == 0) {
                for (int l = LB; l + 1 < L; ++l) level_down(l, threadIdx.x, blockDim.x, bsync);
                // coarsest level: Jacobi sweeps from zero in shared memory
                const MgLevel& C = mg.lv[L - 1];
                const int ncells = C.nx * C.ny * C.nz;
                // right-hand side, omega / diagonal (0 outside the mask) and neighbour bits, once
                for (int t = threadIdx.x; t < ncells; t += blockDim.x) {
                    const int I = t % C.nx, J = (t / C.nx) % C.ny, K = t / (C.nx * C.ny);
                    const bool in = C.mask[t] != 0;
                    s_cr[t] = in ? C.r[t] : 0.f;
                    s_cw[t] = in ? wdiag(I, J, K, C.nx, C.ny, C.nz, C.ih2) : 0.f;
                    s_cb[t] = (I > 0 ? 1u : 0u) | (I + 1 < C.nx ? 2u : 0u) | (J > 0 ? 4u : 0u) | (J + 1 < C.ny ? 8u : 0u) |
                              (K > 0 ? 16u : 0u) | (K + 1 < C.nz ? 32u : 0u);
                    s_cz[0][t] = 0.f;
                }
                __syncthreads();
                const int csx = C.nx, csxy = C.nx * C.ny;
                int src = 0;
                for (int sw = 0; sw < kCoarseSweeps; ++sw) {
                    for (int t = threadIdx.x; t < ncells; t += blockDim.x) {
                        const float* z = s_cz[src];
                        const float zc = z[t];
                        const uint32_t m = s_cb[t];
                        float ax = 0.f, ay = 0.f, az = 0.f;
                        if (m & 1u) ax += zc - z[t - 1];
                        if (m & 2u) ax += zc - z[t + 1];
                        if (m & 4u) ay += zc - z[t - csx];
                        if (m & 8u) ay += zc - z[t + csx];
                        if (m & 16u) az += zc - z[t - csxy];
                        if (m & 32u) az += zc - z[t + csxy];
                        const float Az = C.ih2[0] * ax + C.ih2[1] * ay + C.ih2[2] * az;
                        s_cz[src ^ 1][t] = zc + s_cw[t] * (s_cr[t] - Az);  // 0 outside the mask (s_cw = 0)
                    }
                    __syncthreads();
                    src ^= 1;
                }
                for (int t = threadIdx.x; t < ncells; t += blockDim.x) C.z[t] = s_cz[src][t];
                bsync();
                for (int l = L - 2; l >= LB; --l) level_up(l, threadIdx.x, blockDim.x, bsync);
            }
            if (!grid_sync(w, gen, nblk, sh, blk)) return;
            for (int l = LB - 1; l >= 1; --l)
                if (!level_up(l, tid, T, gsync)) return;
            // level 0: pre-smoothed correction into the residual vector (free again), then one Jacobi sweep
            double rho;
            {
                const float* __restrict__ r = R[cur];
                const MgLevel& C = mg.lv[1];
                for (int e = tid, k = 0; e < F; e += T, ++k) {
                    const int c = (int)(entry(k, e) >> 6);
                    const int i = c % nx, j = (c / nx) % ny, kk = c / sxy;
                    RES[c] = r[c] * wdiag(i, j, kk, nx, ny, nz, ih2) + prolong_at(C, i, j, kk);
                }
                zero_coarse();
                if (!grid_sync(w, gen, nblk, sh, blk)) return;
                double acc[1] = {0.0};
                for (int e = tid, k = 0; e < F; e += T, ++k) {
                    const uint32_t ent = entry(k, e);
                    const int c = (int)(ent >> 6);
                    const int i = c % nx, j = (c / nx) % ny, kk = c / sxy;
                    const float At = apply_row(st0, c, ent & 63u, [&](int q) { return RES[q]; });
                    const float zc = RES[c] + (r[c] - At) * wdiag(i, j, kk, nx, ny, nz, ih2);
                    Z[c] = zc;
                    acc[0] += (double)r[c] * (double)zc;
                }
                if (!grid_reduce<1>(acc, sh, w, gen, nblk, blk)) return;
                rho = acc[0];
            }
            // search direction: p' = z + beta p, q = A p', (p', q)
            const double beta = first ? 0.0 : rho / rho_old;
            rho_old = rho;
            first = false;
            {
                const float bf = (float)beta;
                const float* __restrict__ p = P[pc];
                float* __restrict__ pn = P[pc ^ 1];
                double acc[1] = {0.0};
                auto pnew = [&](int q) { return Z[q] + bf * p[q]; };
                for (int e = tid, k = 0; e < F; e += T, ++k) {
                    const uint32_t ent = entry(k, e);
                    const int c = (int)(ent >> 6);
                    const float pc_ = pnew(c);
                    const float qc = apply_row(st0, c, ent & 63u, pnew);
                    pn[c] = pc_;
                    Q[c] = qc;
                    acc[0] += (double)pc_ * (double)qc;
                }
                if (!grid_reduce<1>(acc, sh, w, gen, nblk, blk)) return;
                pc ^= 1;
                const double a = rho / acc[0];
                if (!(a > 0.0) || !isfinite(a)) break;  // FP32 breakdown: leave it to the outer loop
                alpha = (float)a;
            }
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

}  // namespace
}  // namespace fe
