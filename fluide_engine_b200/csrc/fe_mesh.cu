// fe_mesh.cu -- scene initialisation from triangle meshes: Mesh2SDF, InitializeParticles, VolumeEmitter.
//
// Reference:
//   Mesh2SDF::Build (3d/mesh_2_sdf.cpp:14-82): every node starts at max(h) * (nx + ny + nz); each triangle's index
//     box (vertex coordinates times 1 / h_x on every axis, truncated, widened by one node below and two above,
//     clamped) takes min(distance to the triangle) (Collisions::DistanceToTriangle, 3d/collisions.cpp:21-217);
//     then every node inside the mesh (TriangleMesh::IsInside, 3d/triangle_mesh.cpp:120-163: the sum of
//     atan2(det(A, B, C), k) over triangles, i.e. half the solid angle, is at least 2 pi - 0.001 in magnitude)
//     is negated.
//   PICSimulator::InitializeParticles (pic_simulator.cpp:521-548): every velocity-grid index (i, j, k) whose
//     position (domain origin + h * index) samples the fluid SDF below 0 receives particlesPerBlock particles at
//     position + h * U[0, 1]^3.
//   VolumeEmitter::Emitt (emmiter/volume_emmiter.cpp:58-86), at the start of every substep: every node of the
//     emitter's own SDF grid with sdf <= 0 whose fluid SDF value (same index, the SDF of the previous substep) is
//     >= 0 receives particlesPerBlock particles at position + h * U[0, 1]^3 with the emitter's velocity.
//
// B200 design: the band distances are one CTA per triangle over its index box, min-combined with 64-bit
// atomicMin on the bits of the non-negative distances (the same minimum as the reference's sequential loop); the
// signs are one thread per node summing the winding terms of all triangles.  The distance arithmetic follows the
// reference's expressions in FP64 with round-to-nearest intrinsics, so distances are bit-identical; the sign test
// sums CUDA's atan2, whose last bits can differ from the host library's, which decides nothing unless a node lies
// within ~1e-12 of the 2 pi - 0.001 threshold (points on the surface sum to pi, points inside to 2 pi).  Seeding
// and emission are count -> scan -> write passes; the random numbers are a counter-based splitmix64 of (seed,
// particle index, axis), deterministic where the reference's std::rand() in a parallel loop is not.
#include <cinttypes>
#include <cstring>

#include "fe_geom.cuh"

namespace fe {
namespace {

// One CTA per triangle (grid-stride): the nodes of its index box take the minimum distance.
__global__ void __launch_bounds__(256) k_mesh_band(MeshView m, NodeGrid g, unsigned long long* __restrict__ bits)
{
    const double inv = dd(1.0, g.h[0]);  // the reference scales every axis by 1 / h_x
    for (uint64_t t = blockIdx.x; t < m.nt; t += gridDim.x) {
        double p[3][3];
        load_vertex(m, m.T[4 * t], p[0]);
        load_vertex(m, m.T[4 * t + 1], p[1]);
        load_vertex(m, m.T[4 * t + 2], p[2]);
        int lo[3], hi[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double f0 = dm(p[0][d], inv), f1 = dm(p[1][d], inv), f2 = dm(p[2][d], inv);
            lo[d] = min(max((int)fmin(f0, fmin(f1, f2)) - 1, 0), g.n[d] - 1);
            hi[d] = min(max((int)fmax(f0, fmax(f1, f2)) + 2, 0), g.n[d] - 1);
        }
        const int sx = hi[0] - lo[0] + 1, sy = hi[1] - lo[1] + 1, sz = hi[2] - lo[2] + 1;
        const int64_t cells = (int64_t)sx * sy * sz;
        for (int64_t q = threadIdx.x; q < cells; q += blockDim.x) {
            const int i = lo[0] + (int)(q % sx), j = lo[1] + (int)((q / sx) % sy), k = lo[2] + (int)(q / ((int64_t)sx * sy));
            const double pt[3] = {grid_pos(g, 0, i), grid_pos(g, 1, j), grid_pos(g, 2, k)};
            const double d = distance_to_triangle(pt, p[0], p[1], p[2]);
            const unsigned long long b = (unsigned long long)__double_as_longlong(d);
            unsigned long long* cell = bits + idx3(i, j, k, g.n[0], g.n[1]);
            if (b < __ldcg(cell)) atomicMin(cell, b);
        }
    }
}

// TriangleMesh::IsInside at every node, then the signed value: -d inside, d outside.
__global__ void __launch_bounds__(256) k_mesh_sign(MeshView m, NodeGrid g, const unsigned long long* __restrict__ bits,
                                                   double* __restrict__ sdf)
{
    const double two_pi_tol = ds(dm(2.0, 3.14159265358979323846), 0.001);
    const size_t nc = (size_t)g.n[0] * g.n[1] * g.n[2];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.n[0]), j = (int)((c / g.n[0]) % g.n[1]), k = (int)(c / ((size_t)g.n[0] * g.n[1]));
        const double pt[3] = {grid_pos(g, 0, i), grid_pos(g, 1, j), grid_pos(g, 2, k)};
        const double d = __longlong_as_double((long long)bits[c]);
        sdf[c] = fabs(winding_sum(m, pt)) >= two_pi_tol ? dm(d, -1.0) : d;
    }
}

__global__ void k_fill_bits(unsigned long long* __restrict__ bits, size_t n, unsigned long long v)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) bits[c] = v;
}

__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t counter)
{
    uint64_t z = seed + (counter + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// InitializeParticles' cell test: 1 where the velocity-grid position samples the fluid SDF below 0.
__global__ void k_seed_count(const double* __restrict__ fluid_sdf, NodeGrid sdf_grid, NodeGrid vel_grid, uint32_t ppb,
                             uint32_t* __restrict__ count)
{
    const size_t nc = (size_t)vel_grid.n[0] * vel_grid.n[1] * vel_grid.n[2];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % vel_grid.n[0]), j = (int)((c / vel_grid.n[0]) % vel_grid.n[1]);
        const int k = (int)(c / ((size_t)vel_grid.n[0] * vel_grid.n[1]));
        const double pos[3] = {grid_pos(vel_grid, 0, i), grid_pos(vel_grid, 1, j), grid_pos(vel_grid, 2, k)};
        count[c] = sample_nodes(fluid_sdf, sdf_grid, pos) < 0.0 ? ppb : 0u;
    }
}

// VolumeEmitter::Emitt's node test: emitter SDF <= 0 and the fluid SDF at the same index >= 0.
__global__ void k_emit_count(const double* __restrict__ emitter_sdf, NodeGrid eg, const double* __restrict__ fluid_sdf,
                             int fnx, int fny, uint32_t ppb, uint32_t* __restrict__ count,
                             const double* __restrict__ collider_sdf)
{
    const size_t nc = (size_t)eg.n[0] * eg.n[1] * eg.n[2];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % eg.n[0]), j = (int)((c / eg.n[0]) % eg.n[1]), k = (int)(c / ((size_t)eg.n[0] * eg.n[1]));
        const double fv = fluid_sdf ? fluid_sdf[idx3(i, j, k, fnx, fny)] : 0.0;
        // colliderSdf(i, j, k) > 0: with no collider every node holds 1.7976931348623157e30
        const bool free_node = collider_sdf ? collider_sdf[idx3(i, j, k, fnx, fny)] > 0.0 : true;
        count[c] = (emitter_sdf[c] <= 0.0 && fv >= 0.0 && free_node) ? ppb : 0u;
    }
}

// Writes the particles of every counted node: node position + h * U[0,1]^3 (FP32), the given velocity, C = 0.
__global__ void k_spawn(NodeGrid g, const uint32_t* __restrict__ count, const uint32_t* __restrict__ offset,
                        uint64_t seed, SceneView v, uint64_t base, float vx, float vy, float vz)
{
    const size_t nc = (size_t)g.n[0] * g.n[1] * g.n[2];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const uint32_t cnt = count[c];
        if (!cnt) continue;
        const int i = (int)(c % g.n[0]), j = (int)((c / g.n[0]) % g.n[1]), k = (int)(c / ((size_t)g.n[0] * g.n[1]));
        const double pos[3] = {grid_pos(g, 0, i), grid_pos(g, 1, j), grid_pos(g, 2, k)};
        for (uint32_t q = 0; q < cnt; ++q) {
            const uint64_t p = base + offset[c] + q;
            const uint64_t id = (uint64_t)offset[c] + q;
            const double x = da(dm(g.h[0], uniform01(seed, 3 * id)), pos[0]);
            const double y = da(dm(g.h[1], uniform01(seed, 3 * id + 1)), pos[1]);
            const double z = da(dm(g.h[2], uniform01(seed, 3 * id + 2)), pos[2]);
            v.px[p] = (float)x; v.py[p] = (float)y; v.pz[p] = (float)z;
            v.vx[p] = vx; v.vy[p] = vy; v.vz[p] = vz;
            v.pid[p] = (uint32_t)p;
            if (v.c[0])
#pragma unroll
                for (int a = 0; a < 9; ++a) v.c[a][p] = 0.f;
        }
    }
}

// VolumeField::Initialize (forces/volume_field.cpp:72-89): at every node of the field's grid, the closest point on
// the first nearest triangle (Collisions::ClosestTriangleIdx, 3d/collisions.cpp:249-265: strict < from
// 1.7976931348623157e30) minus the node position, 3 doubles per node.  One thread per node over all triangles.
__global__ void __launch_bounds__(256) k_volume_vectors(MeshView m, NodeGrid g, double* __restrict__ out)
{
    const size_t nc = (size_t)g.n[0] * g.n[1] * g.n[2];
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % g.n[0]), j = (int)((c / g.n[0]) % g.n[1]), k = (int)(c / ((size_t)g.n[0] * g.n[1]));
        const double gp[3] = {grid_pos(g, 0, i), grid_pos(g, 1, j), grid_pos(g, 2, k)};
        double best = 1.7976931348623157e30;
        uint64_t idx = 0;
        double A[3], B[3], C[3];
        for (uint64_t t = 0; t < m.nt; ++t) {
            load_vertex(m, __ldg(m.T + 4 * t), A);
            load_vertex(m, __ldg(m.T + 4 * t + 1), B);
            load_vertex(m, __ldg(m.T + 4 * t + 2), C);
            const double d = distance_to_triangle(gp, A, B, C);
            if (d < best) {
                best = d;
                idx = t;
            }
        }
        double cp[3] = {0.0, 0.0, 0.0};
        if (m.nt) {
            load_vertex(m, m.T[4 * idx], A);
            load_vertex(m, m.T[4 * idx + 1], B);
            load_vertex(m, m.T[4 * idx + 2], C);
            closest_on_triangle(gp, A, B, C, cp);
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) out[3 * c + a] = ds(cp[a], gp[a]);
    }
}

NodeGrid node_grid(const int n[3], const double o[3], const double h[3])
{
    NodeGrid g;
    for (int a = 0; a < 3; ++a) { g.n[a] = n[a]; g.o[a] = o[a]; g.h[a] = h[a]; }
    return g;
}

}  // namespace

cudaError_t launch_mesh_to_sdf(const double* V, uint64_t nv, const int64_t* T, uint64_t nt, const int n[3],
                               const double o[3], const double h[3], unsigned long long* scratch, double* sdf,
                               cudaStream_t st)
{
    const NodeGrid g = node_grid(n, o, h);
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    const double hmax = (h[0] >= h[1] && h[0] >= h[2]) ? h[0] : ((h[1] >= h[0] && h[1] >= h[2]) ? h[1] : h[2]);
    const double fill = hmax * (double)((size_t)n[0] + (size_t)n[1] + (size_t)n[2]);
    unsigned long long fill_bits;
    std::memcpy(&fill_bits, &fill, sizeof(fill_bits));
    k_fill_bits<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(scratch, nc, fill_bits);
    count_launch();
    MeshView m{V, T, nv, nt};
    if (nv > 0 && nt > 0) {
        k_mesh_band<<<(unsigned)std::min<uint64_t>(nt, 148 * 64), 256, 0, st>>>(m, g, scratch);
        count_launch();
    }
    if (nv == 0) m.nt = 0;  // no vertices: no distances and no triangle to wind around (the fill stays positive)
    k_mesh_sign<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(m, g, scratch, sdf);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_volume_vectors(const double* V, uint64_t nv, const int64_t* T, uint64_t nt, const int n[3],
                                  const double o[3], const double h[3], double* out, cudaStream_t st)
{
    MeshView m;
    m.V = V;
    m.T = T;
    m.nv = nv;
    m.nt = nv ? nt : 0;
    const NodeGrid g = node_grid(n, o, h);
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    k_volume_vectors<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(m, g, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_seed_count(const double* fluid_sdf, const int n[3], const double sdf_o[3], const double h[3],
                              const double vel_o[3], uint32_t ppb, uint32_t* count, cudaStream_t st)
{
    const NodeGrid sg = node_grid(n, sdf_o, h), vg = node_grid(n, vel_o, h);
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    k_seed_count<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(fluid_sdf, sg, vg, ppb, count);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_emit_count(const double* emitter_sdf, const int en[3], const double* fluid_sdf, int fnx, int fny,
                              uint32_t ppb, uint32_t* count, cudaStream_t st, const double* collider_sdf)
{
    const double z[3] = {0, 0, 0};
    const NodeGrid eg = node_grid(en, z, z);
    const size_t nc = (size_t)en[0] * en[1] * en[2];
    k_emit_count<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(emitter_sdf, eg, fluid_sdf, fnx,
                                                                                        fny, ppb, count, collider_sdf);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_spawn(const int n[3], const double o[3], const double h[3], const uint32_t* count,
                         const uint32_t* offset, uint64_t seed, const SceneView& v, uint64_t base, const float vel[3],
                         cudaStream_t st)
{
    const NodeGrid g = node_grid(n, o, h);
    const size_t nc = (size_t)n[0] * n[1] * n[2];
    k_spawn<<<(unsigned)std::min<size_t>((nc + 255) / 256, 148 * 32), 256, 0, st>>>(g, count, offset, seed, v, base, vel[0],
                                                                                   vel[1], vel[2]);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
