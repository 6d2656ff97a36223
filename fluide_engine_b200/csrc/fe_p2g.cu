// fe_p2g.cu -- particle -> grid transfer (K_p2g).
//
// Reference: PICSimulator::TransferParticles2Grid (pic_simulator.cpp:356-437), FLIPSimulator
// (flip_simulator.cpp:25-119) and APICSimulator (apic_simulator.cpp:15-118): for every particle and
// every velocity component, trilinear weights w on the 8 surrounding faces (GetCooridnatesAndWeights,
// common/math_utils.hpp:75-112), u += w * value, weight += w, marker = 1; then u /= weight where
// weight > 0.  PIC and APIC clamp the face index with the CELL count, FLIP with the face count.  APIC
// adds C_row . (x_face - x_clamped), the particle position clamped by h/2 on the two transverse axes.
//
// B200 design: one CTA per 8x8x8-cell tile.  The tile's particles are one contiguous run of the
// sorted arrays (fe_keys.h), read once with coalesced loads.  Every face they can touch lies in a
// 10x10x10 box around the tile (one cell of halo on each side covers the clamp quirks), so each CTA
// accumulates numerator, weight and touched-marker of all three components in 24 KB of shared memory
// with shared-memory atomics, then flushes the box to global accumulators: box faces touched by the
// tile get one global red.add each, so a face receives at most 8 global adds (one per neighbouring
// tile), never one per particle.  A second pass divides numerator by weight and, for FLIP, writes the
// snapshot (flip_simulator.cpp:107-118).  Particles whose stencil leaves the box (only possible for a
// domain origin away from zero, where the reference's data origins ignore the origin) fall back to
// direct global adds, so the kernel stays correct for every input.
#include "fe_internal.cuh"

namespace fe {
namespace {

constexpr int kBox = 10;
constexpr int kBoxFaces = kBox * kBox * kBox;
constexpr int kP2gThreads = 256;

template <int SOLVER>
__global__ void __launch_bounds__(kP2gThreads) k_p2g(SceneView v)
{
    __shared__ float s_num[3][kBoxFaces];
    __shared__ float s_den[3][kBoxFaces];
    __shared__ uint8_t s_mk[3][kBoxFaces];

    const int tile = blockIdx.x;
    const int tx = tile % v.g.tnx, ty = (tile / v.g.tnx) % v.g.tny, tz = tile / (v.g.tnx * v.g.tny);
    const int bx = tx * FE_TILE - 1, by = ty * FE_TILE - 1, bz = tz * FE_TILE - 1;  // box origin (face index)
    const uint32_t beg = v.cell_start[(uint32_t)tile * FE_TILE_CELLS];
    const uint32_t end = v.cell_start[(uint32_t)(tile + 1) * FE_TILE_CELLS];
    if (beg == end) return;  // nothing to splat; accumulators were cleared by the caller

    for (int t = threadIdx.x; t < 3 * kBoxFaces; t += blockDim.x) {
        (&s_num[0][0])[t] = 0.f;
        (&s_den[0][0])[t] = 0.f;
        (&s_mk[0][0])[t] = 0;
    }
    __syncthreads();

    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    // face-array sizes and the clamp sizes the reference passes to GetCooridnatesAndWeights
    const int fsx[3] = {nx + 1, nx, nx}, fsy[3] = {ny, ny + 1, ny}, fsz[3] = {nz, nz, nz + 1};
    const bool flip = SOLVER == FE_SOLVER_FLIP;
    const int csx[3] = {flip ? nx + 1 : nx, nx, nx}, csy[3] = {ny, flip ? ny + 1 : ny, ny},
              csz[3] = {nz, nz, flip ? nz + 1 : nz};
    const float* org[3] = {v.xo, v.yo, v.zo};
    float* gnum[3] = {v.nu, v.nv, v.nw};
    float* gden[3] = {v.du, v.dv, v.dw};
    uint8_t* gmk[3] = {v.mu, v.mv, v.mw};
    const float lo[3] = {v.originf[0] + 0.5f * v.hf[0], v.originf[1] + 0.5f * v.hf[1], v.originf[2] + 0.5f * v.hf[2]};
    const float hi[3] = {v.originf[0] + v.sizef[0] - 0.5f * v.hf[0], v.originf[1] + v.sizef[1] - 0.5f * v.hf[1],
                         v.originf[2] + v.sizef[2] - 0.5f * v.hf[2]};

    // Thread -> particle map that keeps a warp's lanes on different cells: with about 8 particles per
    // cell, consecutive particles share their 24 face targets, so lane l of warp w takes particle
    // base + 8 l + w of each 256-particle window and shared-memory atomics rarely collide.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (uint32_t base = beg; base < end; base += blockDim.x) {
        const uint32_t p = base + (uint32_t)(lane * nwarps + warp);
        if (p >= end) continue;
        const float x = v.px[p], y = v.py[p], z = v.pz[p];
        const float vel[3] = {v.vx[p], v.vy[p], v.vz[p]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            Stencil s = stencil(x, y, z, org[c], v.inv_hf, csx[c], csy[c], csz[c]);
            float cr[3] = {0.f, 0.f, 0.f}, pc[3] = {x, y, z};
            if (SOLVER == FE_SOLVER_APIC) {
                cr[0] = v.c[3 * c][p];
                cr[1] = v.c[3 * c + 1][p];
                cr[2] = v.c[3 * c + 2][p];
                // Clamp(val, max, min) on the two transverse axes (apic_simulator.cpp:55-57,68-70,81-83)
#pragma unroll
                for (int a = 0; a < 3; ++a)
                    if (a != c) pc[a] = pc[a] < lo[a] ? lo[a] : (pc[a] > hi[a] ? hi[a] : pc[a]);
            }
            const float wx[2] = {1.f - s.fx, s.fx}, wy[2] = {1.f - s.fy, s.fy}, wz[2] = {1.f - s.fz, s.fz};
            const int ii[2] = {s.i, s.ip}, jj[2] = {s.j, s.jp}, kk[2] = {s.k, s.kp};
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int a = t & 1, b = (t >> 1) & 1, d = t >> 2;
                const float wgt = wx[a] * wy[b] * wz[d];
                float val = vel[c];
                if (SOLVER == FE_SOLVER_APIC) {
                    float gx = org[c][0] + v.hf[0] * (float)ii[a];
                    float gy = org[c][1] + v.hf[1] * (float)jj[b];
                    float gz = org[c][2] + v.hf[2] * (float)kk[d];
                    val += cr[0] * (gx - pc[0]) + cr[1] * (gy - pc[1]) + cr[2] * (gz - pc[2]);
                }
                const int li = ii[a] - bx, lj = jj[b] - by, lk = kk[d] - bz;
                if ((unsigned)li < kBox && (unsigned)lj < kBox && (unsigned)lk < kBox) {
                    const int l = li + kBox * (lj + kBox * lk);
                    atomicAdd(&s_num[c][l], val * wgt);
                    atomicAdd(&s_den[c][l], wgt);
                    s_mk[c][l] = 1;
                } else {
                    const size_t f = idx3(ii[a], jj[b], kk[d], fsx[c], fsy[c]);
                    atomicAdd(gnum[c] + f, val * wgt);
                    atomicAdd(gden[c] + f, wgt);
                    gmk[c][f] = 1;
                }
            }
        }
    }
    __syncthreads();

#pragma unroll
    for (int c = 0; c < 3; ++c) {
        for (int l = threadIdx.x; l < kBoxFaces; l += blockDim.x) {
            if (!s_mk[c][l]) continue;
            const int li = l % kBox, lj = (l / kBox) % kBox, lk = l / (kBox * kBox);
            const int gi = bx + li, gj = by + lj, gk = bz + lk;
            if (gi < 0 || gj < 0 || gk < 0 || gi >= fsx[c] || gj >= fsy[c] || gk >= fsz[c]) continue;
            const size_t f = idx3(gi, gj, gk, fsx[c], fsy[c]);
            atomicAdd(gnum[c] + f, s_num[c][l]);
            atomicAdd(gden[c] + f, s_den[c][l]);
            gmk[c][f] = 1;
        }
    }
}

// u = num / weight where weight > 0 (pic_simulator.cpp:414-436); FLIP also snapshots the result.
template <bool FLIP>
__global__ void k_p2g_normalize(SceneView v, size_t nu, size_t nvv, size_t nww)
{
    size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t total = nu + nvv + nww;
    if (t >= total) return;
    const float* num;
    const float* den;
    float* out;
    float* snap;
    size_t f;
    if (t < nu) { f = t; num = v.nu; den = v.du; out = v.u; snap = v.su; }
    else if (t < nu + nvv) { f = t - nu; num = v.nv; den = v.dv; out = v.v; snap = v.sv; }
    else { f = t - nu - nvv; num = v.nw; den = v.dw; out = v.w; snap = v.sw; }
    const float d = den[f];
    const float val = d > 0.f ? num[f] / d : num[f];
    out[f] = val;
    if (FLIP) snap[f] = val;
}

}  // namespace

cudaError_t launch_p2g(const SceneView& v, cudaStream_t st)
{
    const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz,
                 nww = (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    cudaError_t e;
    // accumulators: numerator and weight arrays are laid out back to back, markers too (fe_scene.cu)
    if ((e = cudaMemsetAsync(v.nu, 0, (nu + nvv + nww) * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(v.du, 0, (nu + nvv + nww) * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(v.mu, 0, nu + nvv + nww, st)) != cudaSuccess) return e;
    const unsigned tiles = (unsigned)(v.g.tnx * v.g.tny * v.g.tnz);
    if (v.np > 0) {
        if (v.solver == FE_SOLVER_PIC) k_p2g<FE_SOLVER_PIC><<<tiles, kP2gThreads, 0, st>>>(v);
        else if (v.solver == FE_SOLVER_FLIP) k_p2g<FE_SOLVER_FLIP><<<tiles, kP2gThreads, 0, st>>>(v);
        else k_p2g<FE_SOLVER_APIC><<<tiles, kP2gThreads, 0, st>>>(v);
        count_launch();
    }
    const size_t total = nu + nvv + nww;
    const unsigned nb = (unsigned)((total + 255) / 256);
    if (v.solver == FE_SOLVER_FLIP) k_p2g_normalize<true><<<nb, 256, 0, st>>>(v, nu, nvv, nww);
    else k_p2g_normalize<false><<<nb, 256, 0, st>>>(v, nu, nvv, nww);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
