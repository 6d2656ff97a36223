// fe_grid.cu -- face-grid passes of the substep.
//
//   K_extrap   one pass of ExtrapolateToRegion (common/math_utils.hpp:186-253): an invalid face takes
//              the mean of its valid 6-neighbours (order i+1, i-1, j+1, j-1, k+1, k-1) and becomes
//              valid.  Passes ping-pong between the two velocity buffers, so ceil(maxCfl) passes before
//              the solve and as many after it leave the result in the buffer the substep started with.
//              The last pass of each group is fused with what follows it in the reference:
//   pre        ExtrapolateVelocityToAir, ApplyBoundryCondition, gravity, ApplyBoundryCondition
//              (pic_simulator.cpp:186-211): wall faces end at 0, every other face gains dt*g.
//   post       ExtrapolateVelocityToAir, ApplyBoundryCondition (pic_simulator.cpp:233-234).
//              With no colliders ApplyBoundryCondition reduces to zeroing the six wall face layers
//              (fluid_solvers/blocked_boundry_condition_solver.cpp:198-244).
//   K_rhs      b = div u on FLUID cells (DivergenceAtCallCenter, grid_systems/face_centered_grid3d.cpp:
//              157-166, evaluated in FP64 from the FP32 faces), 0 elsewhere.
//   K_apply    u_{i+1} += (p_{i+1} - p_i) / h for FLUID cells i toward +x/+y/+z only, except toward BOUNDRY
//              cells (fluid_solvers/single_phase_pressure_solver.cpp:56-92); wall faces are never touched.
//   K_cfl      max over cells of |u_cc| + dt*(0,-9.8,0) component-wise (pic_simulator.cpp:80-97).
#include "fe_internal.cuh"

namespace fe {
namespace {

struct FaceArrays {
    const float* in[3];
    float* out[3];
    const uint8_t* vin[3];
    uint8_t* vout[3];
};

enum { kModePlain = 0, kModePre = 1, kModePost = 2 };


// One column of faces (FaceColumn) of an extrapolation pass.  The face's own value and validity and those of its
// k - 1 and k + 1 neighbours slide along the column (one new plane loaded per step); the i and j neighbours are
// loaded per face.  Same arithmetic as extrap_store, neighbours summed in the same order (i+1, i-1, j+1, j-1, k+1,
// k-1).
template <int MODE>
__device__ __forceinline__ void extrap_column(const FaceArrays& fa, int nx, int ny, int nz, bool write_valid,
                                              float gx, float gy, float gz, Blk3 blk)
{
    FaceColumn fc;
    if (!column_coord(nx, ny, nz, blk, fc)) return;
    const int c = fc.c, i = fc.i, j = fc.j, sx = fc.sx, sy = fc.sy, sz = fc.sz;
    const float* __restrict__ in = c == 0 ? fa.in[0] : (c == 1 ? fa.in[1] : fa.in[2]);
    const uint8_t* __restrict__ vin = c == 0 ? fa.vin[0] : (c == 1 ? fa.vin[1] : fa.vin[2]);
    float* __restrict__ out = c == 0 ? fa.out[0] : (c == 1 ? fa.out[1] : fa.out[2]);
    uint8_t* __restrict__ vout = c == 0 ? fa.vout[0] : (c == 1 ? fa.vout[1] : fa.vout[2]);
    const size_t sxy = (size_t)sx * sy;
    size_t f = (size_t)i + (size_t)sx * ((size_t)j + (size_t)sy * (size_t)fc.k0);
    const bool ip = i + 1 < sx, im = i > 0, jp = j + 1 < sy, jm = j > 0;
    const bool wall_ij = (c == 0 && (i == 0 || i == sx - 1)) || (c == 1 && (j == 0 || j == sy - 1));
    const float g = c == 0 ? gx : (c == 1 ? gy : gz);
    float vm = 0.f, vc = in[f];
    uint8_t am = 0, ac = vin[f];
    if (fc.k0 > 0) {
        vm = in[f - sxy];
        am = vin[f - sxy];
    }
    for (int k = fc.k0; k < fc.k1; ++k, f += sxy) {
        const bool kp = k + 1 < sz;
        const float vp = kp ? in[f + sxy] : 0.f;
        const uint8_t ap = kp ? vin[f + sxy] : (uint8_t)0;
        const uint8_t a0 = ip ? vin[f + 1] : (uint8_t)0, a1 = im ? vin[f - 1] : (uint8_t)0;
        const uint8_t a2 = jp ? vin[f + sx] : (uint8_t)0, a3 = jm ? vin[f - sx] : (uint8_t)0;
        const float v0 = ip ? in[f + 1] : 0.f, v1 = im ? in[f - 1] : 0.f;
        const float v2 = jp ? in[f + sx] : 0.f, v3 = jm ? in[f - sx] : 0.f;
        float val = vc;
        uint8_t valid = ac;
        if (!valid) {
            float sum = 0.f;
            unsigned count = 0;
            if (a0) { sum += v0; ++count; }
            if (a1) { sum += v1; ++count; }
            if (a2) { sum += v2; ++count; }
            if (a3) { sum += v3; ++count; }
            if (ap) { sum += vp; ++count; }
            if (am) { sum += vm; ++count; }
            if (count > 0) {
                val = sum / (float)count;
                valid = 1;
            }
        }
        if (write_valid) vout[f] = valid;
        if (MODE != kModePlain) {
            const bool wall = wall_ij || (c == 2 && (k == 0 || k == sz - 1));
            if (wall) val = 0.f;
            else if (MODE == kModePre) val += g;
        }
        out[f] = val;
        vm = vc;
        am = ac;
        vc = vp;
        ac = ap;
    }
}

template <int MODE>
__global__ void __launch_bounds__(kTileX * kTileY) k_extrap(FaceArrays fa, int nx, int ny, int nz, bool write_valid,
                                                            float gx, float gy, float gz)
{
    extrap_column<MODE>(fa, nx, ny, nz, write_valid, gx, gy, gz, hw_blk3());
}

__device__ __forceinline__ void rhs_body(const SceneView& v, const float* __restrict__ u, const float* __restrict__ vv,
                                         const float* __restrict__ w, Blk3 blk)
{
    const int nx = v.g.nx, ny = v.g.ny;
    const int i = (int)(blk.x * kTileX + threadIdx.x), j = (int)(blk.y * kTileY + threadIdx.y);
    const int k = (int)blk.z;
    if (i >= nx || j >= ny) return;
    const size_t c = idx3(i, j, k, nx, ny);
    double b = 0.0;
    const bool fluid = v.marks[c] == FE_CELL_FLUID;
    if (fluid) {
        const double left = u[idx3(i, j, k, nx + 1, ny)], right = u[idx3(i + 1, j, k, nx + 1, ny)];
        const double down = vv[idx3(i, j, k, nx, ny + 1)], up = vv[idx3(i, j + 1, k, nx, ny + 1)];
        const double back = w[idx3(i, j, k, nx, ny)], front = w[idx3(i, j, k + 1, nx, ny)];
        b = (right - left) / v.h[0] + (up - down) / v.h[1] + (front - back) / v.h[2];
    }
    v.b[c] = b;
    if (v.pprev) {
        // warm start extrapolated in time, 2 p(n-1) - p(n-2), where the cell held pressure in both substeps; the
        // solve still runs to the same residual target, so only its iteration count changes
        const double pn1 = v.p[c], pn2 = v.pprev[c];
        if (fluid && pn1 != 0.0 && pn2 != 0.0) v.p[c] = 2.0 * pn1 - pn2;
        v.pprev[c] = pn1;
    }
}

__global__ void k_rhs(SceneView v, const float* __restrict__ u, const float* __restrict__ vv,
                      const float* __restrict__ w)
{
    rhs_body(v, u, vv, w, hw_blk3());
}

// One column of faces (FaceColumn) of the pressure apply: indices advance by one plane per step.
__device__ __forceinline__ void apply_column(const SceneView& v, float* u, float* vv, float* w, Blk3 blk)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    FaceColumn fc;
    if (!column_coord(nx, ny, nz, blk, fc)) return;
    const double* __restrict__ p = v.p;
    const uint8_t* __restrict__ mk = v.marks;
    const int i = fc.i, j = fc.j;
    const size_t nxy = (size_t)nx * ny;
    if (fc.c == 0) {
        if (i < 1 || i > nx - 1) return;
        const double ih = v.inv_h[0];
        const size_t fs = (size_t)(nx + 1) * ny;
        size_t cm = idx3(i - 1, j, fc.k0, nx, ny), f = idx3(i, j, fc.k0, nx + 1, ny);
        for (int k = fc.k0; k < fc.k1; ++k, cm += nxy, f += fs)
            if (mk[cm] == FE_CELL_FLUID && mk[cm + 1] != FE_CELL_BOUNDRY)
                u[f] = (float)((double)u[f] + ih * (p[cm + 1] - p[cm]));
    } else if (fc.c == 1) {
        if (j < 1 || j > ny - 1) return;
        const double ih = v.inv_h[1];
        const size_t fs = (size_t)nx * (ny + 1);
        size_t cm = idx3(i, j - 1, fc.k0, nx, ny), f = idx3(i, j, fc.k0, nx, ny + 1);
        for (int k = fc.k0; k < fc.k1; ++k, cm += nxy, f += fs)
            if (mk[cm] == FE_CELL_FLUID && mk[cm + nx] != FE_CELL_BOUNDRY)
                vv[f] = (float)((double)vv[f] + ih * (p[cm + nx] - p[cm]));
    } else {
        const double ih = v.inv_h[2];
        const int k0 = max(fc.k0, 1), k1 = min(fc.k1, nz);  // faces k = 1 .. nz - 1
        size_t cm = idx3(i, j, k0 - 1, nx, ny), f = idx3(i, j, k0, nx, ny);
        for (int k = k0; k < k1; ++k, cm += nxy, f += nxy)
            if (mk[cm] == FE_CELL_FLUID && mk[cm + nxy] != FE_CELL_BOUNDRY)
                w[f] = (float)((double)w[f] + ih * (p[cm + nxy] - p[cm]));
    }
}

__global__ void __launch_bounds__(kTileX * kTileY) k_apply(SceneView v, float* u, float* vv, float* w)
{
    apply_column(v, u, vv, w, hw_blk3());
}

__global__ void k_cfl(SceneView v, const float* __restrict__ u, const float* __restrict__ vv,
                      const float* __restrict__ w, double dt, unsigned long long* out_bits)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    double m = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const double cx = 0.5 * ((double)u[idx3(i, j, k, nx + 1, ny)] + (double)u[idx3(i + 1, j, k, nx + 1, ny)]);
        const double cy = 0.5 * ((double)vv[idx3(i, j, k, nx, ny + 1)] + (double)vv[idx3(i, j + 1, k, nx, ny + 1)]);
        const double cz = 0.5 * ((double)w[idx3(i, j, k, nx, ny)] + (double)w[idx3(i, j, k + 1, nx, ny)]);
        m = fmax(m, fabs(cx) + dt * 0.0);
        m = fmax(m, fabs(cy) + dt * -9.8);
        m = fmax(m, fabs(cz) + dt * 0.0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, (unsigned long long)__double_as_longlong(m));
}

__global__ void k_divergence(SceneView v, const float* __restrict__ u, const float* __restrict__ vv,
                             const float* __restrict__ w, double* out)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    double acc = 0.0;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (v.marks[c] != FE_CELL_FLUID) continue;
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const double d = ((double)u[idx3(i + 1, j, k, nx + 1, ny)] - u[idx3(i, j, k, nx + 1, ny)]) / v.h[0] +
                         ((double)vv[idx3(i, j + 1, k, nx, ny + 1)] - vv[idx3(i, j, k, nx, ny + 1)]) / v.h[1] +
                         ((double)w[idx3(i, j, k + 1, nx, ny)] - w[idx3(i, j, k, nx, ny)]) / v.h[2];
        acc += d * d;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out, acc);
}

__global__ void k_scatter_out(SceneView v, float* pos, float* vel, float* C)
{
    uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (s >= v.np) return;
    const uint64_t d = v.pid[s];
    if (pos) { pos[3 * d] = v.px[s]; pos[3 * d + 1] = v.py[s]; pos[3 * d + 2] = v.pz[s]; }
    if (vel) { vel[3 * d] = v.vx[s]; vel[3 * d + 1] = v.vy[s]; vel[3 * d + 2] = v.vz[s]; }
    if (C && v.solver == FE_SOLVER_APIC)
        for (int a = 0; a < 9; ++a) C[9 * d + a] = v.c[a][s];
}

size_t faces_total(const SceneView& v)
{
    return (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz + (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz +
           (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
}

// Runs `depth` extrapolation passes starting from buffer A (v.u..) whose last pass applies MODE;
// the face markers v.mu.. are read-only, the validity ping-pong uses v.mu2.. and the crit scratch.
template <int MODE>
cudaError_t run_extrap_group(const SceneView& v, float* const src[3], float* const dst_final[3], float* const other[3],
                             int depth, float gx, float gy, float gz, cudaStream_t st)
{
    const size_t total = faces_total(v);
    const float* in[3] = {src[0], src[1], src[2]};
    const uint8_t* vin[3] = {v.mu, v.mv, v.mw};
    // validity buffers alternate between two scratch sets laid out inside mu2 (size 2 * faces)
    const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz;
    uint8_t* vset[2][3] = {{v.mu2, v.mu2 + nu, v.mu2 + nu + nvv},
                           {v.mu2 + total, v.mu2 + total + nu, v.mu2 + total + nu + nvv}};
    static_assert(MODE != kModePlain, "the last pass carries the pre or post tail");
    for (int pass = 0; pass < depth; ++pass) {
        const bool last = pass == depth - 1;
        FaceArrays fa;
        float* const* out = last ? dst_final : ((pass & 1) ? src : other);
        for (int c = 0; c < 3; ++c) {
            fa.in[c] = in[c];
            fa.out[c] = out[c];
            fa.vin[c] = vin[c];
            fa.vout[c] = vset[pass & 1][c];
        }
        const dim3 grid = column_grid(v.g.nx, v.g.ny, v.g.nz), block(kTileX, kTileY);
        if (last) k_extrap<MODE><<<grid, block, 0, st>>>(fa, v.g.nx, v.g.ny, v.g.nz, false, gx, gy, gz);
        else k_extrap<kModePlain><<<grid, block, 0, st>>>(fa, v.g.nx, v.g.ny, v.g.nz, true, 0.f, 0.f, 0.f);
        count_launch();
        for (int c = 0; c < 3; ++c) {
            in[c] = out[c];
            vin[c] = vset[pass & 1][c];
        }
    }
    return cudaGetLastError();
}

}  // namespace

// `depth` plain passes of ExtrapolateToRegion (no wall tail) from `src` with the read-only validity `valid0`, the
// last pass writing `dst_final` (which must differ from src); intermediate results alternate between `other` and
// src, the validity between the two face-sized halves of `vscratch`.
cudaError_t launch_extrap_faces(const SceneView& v, float* const src[3], float* const dst_final[3],
                                float* const other[3], const uint8_t* const valid0[3], uint8_t* vscratch, int depth,
                                cudaStream_t st)
{
    const size_t total = faces_total(v);
    const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz;
    const float* in[3] = {src[0], src[1], src[2]};
    const uint8_t* vin[3] = {valid0[0], valid0[1], valid0[2]};
    uint8_t* vset[2][3] = {{vscratch, vscratch + nu, vscratch + nu + nvv},
                           {vscratch + total, vscratch + total + nu, vscratch + total + nu + nvv}};
    for (int pass = 0; pass < depth; ++pass) {
        const bool last = pass == depth - 1;
        FaceArrays fa;
        float* const* out = last ? dst_final : ((pass & 1) ? src : other);
        for (int c = 0; c < 3; ++c) {
            fa.in[c] = in[c];
            fa.out[c] = out[c];
            fa.vin[c] = vin[c];
            fa.vout[c] = vset[pass & 1][c];
        }
        k_extrap<kModePlain><<<column_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(
            fa, v.g.nx, v.g.ny, v.g.nz, !last, 0.f, 0.f, 0.f);
        count_launch();
        for (int c = 0; c < 3; ++c) {
            in[c] = out[c];
            vin[c] = vset[pass & 1][c];
        }
    }
    return cudaGetLastError();
}

namespace {

// One column of faces of the wall tail with no extrapolation: wall faces 0, every other face gains dt g (add_g).
__device__ __forceinline__ void wall_tail_column(float* u, float* vv, float* w, int nx, int ny, int nz, bool add_g,
                                                 float gx, float gy, float gz, Blk3 blk)
{
    FaceColumn fc;
    if (!column_coord(nx, ny, nz, blk, fc)) return;
    const int c = fc.c, i = fc.i, j = fc.j, sx = fc.sx, sy = fc.sy, sz = fc.sz;
    float* a = c == 0 ? u : (c == 1 ? vv : w);
    const size_t sxy = (size_t)sx * sy;
    size_t f = idx3(i, j, fc.k0, sx, sy);
    const bool wall_ij = (c == 0 && (i == 0 || i == sx - 1)) || (c == 1 && (j == 0 || j == sy - 1));
    const float g = c == 0 ? gx : (c == 1 ? gy : gz);
    for (int k = fc.k0; k < fc.k1; ++k, f += sxy) {
        if (wall_ij || (c == 2 && (k == 0 || k == sz - 1))) a[f] = 0.f;
        else if (add_g) a[f] += g;
    }
}

__global__ void __launch_bounds__(kTileX * kTileY) k_wall_tail(float* u, float* vv, float* w, int nx, int ny, int nz,
                                                               bool add_g, float gx, float gy, float gz)
{
    wall_tail_column(u, vv, w, nx, ny, nz, add_g, gx, gy, gz, hw_blk3());
}

// ---- flat multi-scene forms (BatchPlan, fe_internal.cuh)

// The substep's clears of every scene (fill bytes over the plan's ranges), 16-byte stores where aligned.
__global__ void __launch_bounds__(256) k_multi_clear(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkClear, b);
    const BatchScene& e = plan->sc[s];
    const uint32_t nblk = plan->start[kBkClear][s + 1] - plan->start[kBkClear][s];
    const uint64_t stride = (uint64_t)nblk * blockDim.x;
    for (int r = 0; r < e.nclr; ++r) {
        uint8_t* p = e.clr_ptr[r];
        const uint64_t n = e.clr_bytes[r];
        const uint8_t val = (uint8_t)e.clr_val[r];
        const uint32_t w = 0x01010101u * val;
        const uint64_t head = min(n, (uint64_t)((16u - ((uintptr_t)p & 15u)) & 15u));
        const uint64_t nq = (n - head) / 16;
        const uint64_t tail = head + nq * 16;
        if (b == 0 && threadIdx.x < head) p[threadIdx.x] = val;
        if (b == 0 && threadIdx.x < n - tail) p[tail + threadIdx.x] = val;
        uint4* q = (uint4*)(p + head);
        for (uint64_t u = (uint64_t)b * blockDim.x + threadIdx.x; u < nq; u += stride) q[u] = make_uint4(w, w, w, w);
    }
}

// Buffers of pass `pass` of a scene's extrapolation group (run_extrap_group's assignment, evaluated per scene):
// A = (u, v, w), B = (u2, v2, w2); the pre group starts from A and ends in A (even depth) or B (odd); the post
// group starts where the pre group ended and ends in A.
__device__ __forceinline__ void group_arrays(const SceneView& v, bool pre, int pass, int d, FaceArrays& fa)
{
    float* A[3] = {v.u, v.v, v.w};
    float* B[3] = {v.u2, v.v2, v.w2};
    float* const* src = pre ? A : ((d & 1) ? B : A);
    float* const* oth = pre ? B : ((d & 1) ? A : B);
    float* const* fin = pre ? ((d & 1) ? B : A) : A;
    const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz;
    const size_t total = nu + nvv + (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    uint8_t* vs0 = v.mu2 + (size_t)(pass & 1) * total;        // this pass's validity output
    uint8_t* vs1 = v.mu2 + (size_t)((pass - 1) & 1) * total;  // the previous pass's
    // pass p reads what pass p - 1 wrote: src at p = 0, then alternately oth (p odd) and src (p even)
    float* const* in = pass == 0 ? src : ((pass & 1) ? oth : src);
    float* const* out = pass == d - 1 ? fin : ((pass & 1) ? src : oth);
    for (int c = 0; c < 3; ++c) {
        fa.in[c] = in[c];
        fa.out[c] = out[c];
    }
    fa.vin[0] = pass == 0 ? v.mu : vs1;
    fa.vin[1] = pass == 0 ? v.mv : vs1 + nu;
    fa.vin[2] = pass == 0 ? v.mw : vs1 + nu + nvv;
    fa.vout[0] = vs0;
    fa.vout[1] = vs0 + nu;
    fa.vout[2] = vs0 + nu + nvv;
}

// Pass `pass` of every scene's pre (PRE) or post extrapolation group; a scene whose group is shorter skips the pass,
// a scene with no extrapolation runs its wall tail at pass 0.
template <bool PRE>
__global__ void __launch_bounds__(kTileX * kTileY) k_multi_extrap(const BatchPlan* __restrict__ plan, int pass)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkFaces, b);
    const BatchScene& e = plan->sc[s];
    const SceneView& v = e.dst;
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const Blk3 blk = flat_blk3(b, column_grid(nx, ny, nz));
    const int d = v.extrap_depth;
    const float gx = PRE ? e.gdt[0] : 0.f, gy = PRE ? e.gdt[1] : 0.f, gz = PRE ? e.gdt[2] : 0.f;
    if (d <= 0) {
        if (pass == 0) wall_tail_column(v.u, v.v, v.w, nx, ny, nz, PRE, gx, gy, gz, blk);
        return;
    }
    if (pass >= d) return;
    FaceArrays fa;
    group_arrays(v, PRE, pass, d, fa);
    if (pass == d - 1) extrap_column<PRE ? kModePre : kModePost>(fa, nx, ny, nz, false, gx, gy, gz, blk);
    else extrap_column<kModePlain>(fa, nx, ny, nz, true, 0.f, 0.f, 0.f, blk);
}

// The velocity buffers the pressure stage reads and writes: B after an odd pre group, else A.
__device__ __forceinline__ void stage_buffers(const SceneView& v, float*& u, float*& vv, float*& w)
{
    const bool odd = v.extrap_depth > 0 && (v.extrap_depth & 1);
    u = odd ? v.u2 : v.u;
    vv = odd ? v.v2 : v.v;
    w = odd ? v.w2 : v.w;
}

__global__ void __launch_bounds__(kTileX * kTileY) k_multi_rhs(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkCells, b);
    const SceneView& v = plan->sc[s].dst;
    float *u, *vv, *w;
    stage_buffers(v, u, vv, w);
    rhs_body(v, u, vv, w, flat_blk3(b, cell_grid(v.g.nx, v.g.ny, v.g.nz)));
}

__global__ void __launch_bounds__(kTileX * kTileY) k_multi_apply(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkFaces, b);
    const SceneView& v = plan->sc[s].dst;
    float *u, *vv, *w;
    stage_buffers(v, u, vv, w);
    apply_column(v, u, vv, w, flat_blk3(b, column_grid(v.g.nx, v.g.ny, v.g.nz)));
}

}  // namespace

// Buffer convention: A = (v.u, v.v, v.w) holds the substep's velocity at its start and end; B =
// (v.u2, v.v2, v.w2).  With depth d, the pre group leaves the velocity in A if d is even, else in B.
cudaError_t launch_pre(const SceneView& v, double dt, cudaStream_t st)
{
    const float gx = (float)(dt * v.gravity[0]), gy = (float)(dt * v.gravity[1]), gz = (float)(dt * v.gravity[2]);
    float* A[3] = {v.u, v.v, v.w};
    float* B[3] = {v.u2, v.v2, v.w2};
    const int d = v.extrap_depth;
    if (d <= 0) {
        k_wall_tail<<<column_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v.u, v.v, v.w, v.g.nx, v.g.ny,
                                                                                      v.g.nz, true, gx, gy, gz);
        count_launch();
        return cudaGetLastError();
    }
    float* const* fin = (d & 1) ? B : A;
    return run_extrap_group<kModePre>(v, A, fin, B, d, gx, gy, gz, st);
}

cudaError_t launch_post(const SceneView& v, cudaStream_t st)
{
    float* A[3] = {v.u, v.v, v.w};
    float* B[3] = {v.u2, v.v2, v.w2};
    const int d = v.extrap_depth;
    if (d <= 0) {
        k_wall_tail<<<column_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v.u, v.v, v.w, v.g.nx, v.g.ny,
                                                                                      v.g.nz, false, 0, 0, 0);
        count_launch();
        return cudaGetLastError();
    }
    float* const* src = (d & 1) ? B : A;
    float* const* oth = (d & 1) ? A : B;
    // d passes starting at src end in A when d is odd (src = B), and in A when d is even (src = A)
    return run_extrap_group<kModePost>(v, src, A, oth, d, 0.f, 0.f, 0.f, st);
}

static inline void pressure_buffers(const SceneView& v, const float*& u, const float*& vv, const float*& w)
{
    const bool b = v.extrap_depth > 0 && (v.extrap_depth & 1);
    u = b ? v.u2 : v.u;
    vv = b ? v.v2 : v.v;
    w = b ? v.w2 : v.w;
}

cudaError_t launch_rhs(const SceneView& v, cudaStream_t st)
{
    const float *u, *vv, *w;
    pressure_buffers(v, u, vv, w);
    k_rhs<<<cell_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v, u, vv, w);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_apply(const SceneView& v, cudaStream_t st)
{
    const float *u, *vv, *w;
    pressure_buffers(v, u, vv, w);
    k_apply<<<column_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v, (float*)u, (float*)vv, (float*)w);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_cfl(const SceneView& v, double dt, double* out_max, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out_max, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    k_cfl<<<148 * 4, 256, 0, st>>>(v, v.u, v.v, v.w, dt, (unsigned long long*)out_max);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_divergence(const SceneView& v, double* out, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double), st);
    if (e != cudaSuccess) return e;
    k_divergence<<<148 * 4, 256, 0, st>>>(v, v.u, v.v, v.w, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_scatter_out(const SceneView& v, float* pos, float* vel, float* C, cudaStream_t st)
{
    if (v.np == 0) return cudaSuccess;
    k_scatter_out<<<(unsigned)((v.np + 255) / 256), 256, 0, st>>>(v, pos, vel, C);
    count_launch();
    return cudaGetLastError();
}

uint32_t batch_blocks(const SceneView& v, int kind)
{
    const size_t faces = faces_total(v);
    switch (kind) {
    case kBkClear: return 0;  // set by the plan builder from its clear ranges
    case kBkPart: return (uint32_t)((v.np + 255) / 256);
    case kBkP2g: return v.np > 0 ? (uint32_t)(v.g.tnx * v.g.tny * v.g.tnz) : 0u;
    case kBkNormalize: return (uint32_t)((faces + 1023) / 1024);  // four faces per thread
    case kBkFaces: {
        const dim3 g = column_grid(v.g.nx, v.g.ny, v.g.nz);
        return g.x * g.y * g.z;
    }
    case kBkCells: {
        const dim3 g = cell_grid(v.g.nx, v.g.ny, v.g.nz);
        return g.x * g.y * g.z;
    }
    case kBkFixup: return v.np > 0 && v.any_inexact ? 148u : 0u;
    default: return sort_batch_blocks(v, kind);
    }
}

cudaError_t launch_multi_clear(const BatchLaunch& L, cudaStream_t st)
{
    k_multi_clear<<<L.total[kBkClear], 256, 0, st>>>(L.plan);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_multi_pre(const BatchLaunch& L, cudaStream_t st)
{
    for (int pass = 0; pass < (L.max_depth > 0 ? L.max_depth : 1); ++pass) {
        k_multi_extrap<true><<<L.total[kBkFaces], dim3(kTileX, kTileY), 0, st>>>(L.plan, pass);
        count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_multi_post(const BatchLaunch& L, cudaStream_t st)
{
    for (int pass = 0; pass < (L.max_depth > 0 ? L.max_depth : 1); ++pass) {
        k_multi_extrap<false><<<L.total[kBkFaces], dim3(kTileX, kTileY), 0, st>>>(L.plan, pass);
        count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_multi_rhs(const BatchLaunch& L, cudaStream_t st)
{
    k_multi_rhs<<<L.total[kBkCells], dim3(kTileX, kTileY), 0, st>>>(L.plan);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_multi_apply(const BatchLaunch& L, cudaStream_t st)
{
    k_multi_apply<<<L.total[kBkFaces], dim3(kTileX, kTileY), 0, st>>>(L.plan);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
