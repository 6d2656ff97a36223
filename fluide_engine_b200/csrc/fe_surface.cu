// fe_surface.cu -- fluid surface: marching cubes over the particle SDF, the reference's mesh, vertex for vertex.
//
// Reference: PICSimulator::GetSurface (pic_simulator.cpp:71-78) -> MarchingCubesSolver::BuildSurface
// (3d/marching_cubes_solver.cpp:25-50): with iso value 0 and no colliders, one serial sweep over the cubes of the
// node grid (i outer, j, k inner; SolveSingleCube, :183-316) and then three sweeps that cap the six domain faces
// with marching squares (SolveXY / SolveYZ / SolveXZ, :318-495; a part's two opposite faces alternate per
// square).  A vertex is created the first time a triangle uses its key (an edge of the doubled grid, or for caps
// also a corner node) and is looked up in a map afterwards; the cube sweep has one map, every cap face its own.
// A triangle's normal index is the index of the most recently created vertex.
//
// B200 design: every cube and every cap square is an "item" in the reference's sweep order.  The case tables
// use every crossed edge (and every inside corner of a square), so all items around a key create or look it up,
// and the one that creates it is the first of them in sweep order -- a closed-form function of the key (along
// each axis across the key, the item with the smaller index when both exist).  So:
//   k_mc_count  per item: the case byte, its triangles and the keys it creates;
//   two exclusive scans over items give each item its first vertex and first triangle;
//   k_mc_emit   per item with triangles: creates its keys' vertices (position, normal) at base + rank in its
//               own use order, and resolves the other keys to the creating item's base + rank, recomputed from
//               that item's case byte.
// The arithmetic is the reference's, operation by operation in FP64 with explicit round-to-nearest intrinsics (no
// fused multiply-add), so vertices, normals and triangles are identical to the reference's mesh.
#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <string>
#include <thread>
#include <vector>

#include "fe_internal.cuh"
#include "fe_mc_tables.h"

namespace fe {
namespace {

__constant__ unsigned long long c_case3[256] = FE_MC_CASES_3D;
__constant__ unsigned long long c_case2[16] = FE_MC_CASES_2D;
__constant__ int c_edge_corner[12][2] = FE_MC_EDGE_CORNERS;
__constant__ int c_corner_off[8][3] = FE_MC_CORNER_OFFSETS;
// Doubled-grid offsets of the cube's edges and corners (MarchingCubesSolver::GlobalEdgeId / GlobalVertexId keys).
__constant__ int c_edge_off[12][3] = {{1, 0, 0}, {2, 0, 1}, {1, 0, 2}, {0, 0, 1}, {1, 2, 0}, {2, 2, 1},
                                      {1, 2, 2}, {0, 2, 1}, {0, 1, 0}, {2, 1, 0}, {2, 1, 2}, {0, 1, 2}};
__constant__ int c_vert_off[8][3] = {{0, 0, 0}, {2, 0, 0}, {2, 0, 2}, {0, 0, 2}, {0, 2, 0}, {2, 2, 0}, {2, 2, 2}, {0, 2, 2}};
// Cap squares per face (0 back z-, 1 front z+, 2 left x-, 3 right x+, 4 down y-, 5 up y+): corner node offsets in
// the square's corner order, the cube-vertex ids of those corners and the cube-edge ids of its edges 4..7.
__constant__ int c_cap_corner[6][4][3] = {
    {{1, 0, 0}, {0, 0, 0}, {0, 1, 0}, {1, 1, 0}}, {{0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}},
    {{0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}}, {{1, 0, 1}, {1, 0, 0}, {1, 1, 0}, {1, 1, 1}},
    {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}}, {{1, 1, 0}, {0, 1, 0}, {0, 1, 1}, {1, 1, 1}}};
__constant__ int c_cap_vid[6][4] = {{1, 0, 4, 5}, {3, 2, 6, 7}, {0, 3, 7, 4}, {2, 1, 5, 6}, {0, 1, 2, 3}, {5, 4, 7, 6}};
__constant__ int c_cap_eid[6][4] = {{0, 8, 4, 9}, {2, 10, 6, 11}, {3, 11, 7, 8}, {1, 9, 5, 10}, {0, 1, 2, 3}, {4, 7, 6, 5}};
__constant__ double c_cap_normal[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}};

struct McGrid {
    int n[3];           // nodes per axis (the SDF grid)
    double o[3], h[3];  // its origin and spacing
    const double* sdf;  // node values, x-fastest
    // item ranges: cubes [0, cap0), then the XY, YZ and XZ cap parts
    uint64_t cubes, part0[3];
};

__device__ __forceinline__ double sdf_at(const McGrid& g, int i, int j, int k)
{
    return __ldg(g.sdf + idx3(i, j, k, g.n[0], g.n[1]));
}

// Cap part p: fixed axis, (outer, inner) in-plane axes of its sweep.
__device__ __forceinline__ void cap_axes(int p, int& fixed, int& outer, int& inner)
{
    if (p == 0) { fixed = 2; outer = 1; inner = 0; }       // XY: j outer, i inner
    else if (p == 1) { fixed = 0; outer = 2; inner = 1; }  // YZ: k outer, j inner
    else { fixed = 1; outer = 2; inner = 0; }              // XZ: k outer, i inner
}

// Item -> cube (i, j, k) or cap (part, side, cube coordinates of the square).
struct Item {
    int kind;  // 0 cube, 1 cap
    int side;  // cap face 0..5
    int c[3];  // cube coordinates
};

__device__ __forceinline__ Item decode(const McGrid& g, uint64_t t)
{
    Item it;
    const int m[3] = {g.n[0] - 1, g.n[1] - 1, g.n[2] - 1};
    if (t < g.cubes) {
        it.kind = 0;
        it.side = 0;
        it.c[2] = (int)(t % m[2]);
        const uint64_t r = t / m[2];
        it.c[1] = (int)(r % m[1]);
        it.c[0] = (int)(r / m[1]);
        return it;
    }
    int p = t >= g.part0[2] ? 2 : (t >= g.part0[1] ? 1 : 0);
    const uint64_t l = t - g.part0[p];
    int fixed, outer, inner;
    cap_axes(p, fixed, outer, inner);
    const int sd = (int)(l & 1);
    const uint64_t sq = l >> 1;
    it.kind = 1;
    it.side = 2 * p + sd;
    it.c[inner] = (int)(sq % m[inner]);
    it.c[outer] = (int)(sq / m[inner]);
    it.c[fixed] = sd ? m[fixed] - 1 : 0;
    return it;
}

__device__ __forceinline__ uint64_t encode_cube(const McGrid& g, int i, int j, int k)
{
    return ((uint64_t)i * (g.n[1] - 1) + j) * (g.n[2] - 1) + k;
}

__device__ __forceinline__ uint64_t encode_cap(const McGrid& g, int side, const int c[3])
{
    const int p = side >> 1;
    int fixed, outer, inner;
    cap_axes(p, fixed, outer, inner);
    const int m_inner = g.n[inner] - 1;
    return g.part0[p] + 2 * ((uint64_t)c[outer] * m_inner + c[inner]) + (side & 1);
}

// A key (doubled offsets off[] from the item's cube c) is created by this item iff, along every axis across the
// key (even offset) within the item's sweep dimensions, the key is on the item's upper side or the item is first.
__device__ __forceinline__ bool creates(const int off[3], const int c[3], int skip_axis)
{
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (a != skip_axis && off[a] == 0 && c[a] > 0) return false;
    return true;
}

// Case byte and the packed triangle list of an item.
__device__ __forceinline__ int cube_case(const McGrid& g, int i, int j, int k)
{
    int cfg = 0;
#pragma unroll
    for (int v = 0; v < 8; ++v)
        if (sdf_at(g, i + c_corner_off[v][0], j + c_corner_off[v][1], k + c_corner_off[v][2]) <= 0.0) cfg |= 1 << v;
    return cfg;
}

__device__ __forceinline__ int cap_case(const McGrid& g, int side, const int c[3])
{
    int cfg = 0;
#pragma unroll
    for (int v = 0; v < 4; ++v)
        if (sdf_at(g, c[0] + c_cap_corner[side][v][0], c[1] + c_cap_corner[side][v][1], c[2] + c_cap_corner[side][v][2]) <= 0.0)
            cfg |= 1 << v;
    return cfg;
}

// Doubled offsets of key q (0..11 cube edges; for caps 0..3 corners, 4..7 edges).
__device__ __forceinline__ void key_off(int kind, int side, int q, int off[3])
{
    if (kind == 0) {
        off[0] = c_edge_off[q][0]; off[1] = c_edge_off[q][1]; off[2] = c_edge_off[q][2];
    } else if (q < 4) {
        const int v = c_cap_vid[side][q];
        off[0] = c_vert_off[v][0]; off[1] = c_vert_off[v][1]; off[2] = c_vert_off[v][2];
    } else {
        const int e = c_cap_eid[side][q - 4];
        off[0] = c_edge_off[e][0]; off[1] = c_edge_off[e][1]; off[2] = c_edge_off[e][2];
    }
}

__device__ __forceinline__ int skip_axis_of(int kind, int side) { return kind == 0 ? -1 : (side < 2 ? 2 : (side < 4 ? 0 : 1)); }

// Rank of key `target` among the keys item (kind, side, c) with case `cfg` creates, in its use order; -1 if absent.
__device__ int creation_rank(int kind, int side, const int c[3], int cfg, int target)
{
    const unsigned long long cs = kind == 0 ? c_case3[cfg] : c_case2[cfg];
    const int nv = 3 * (int)(cs >> 60);
    const int skip = skip_axis_of(kind, side);
    unsigned seen = 0u;
    int r = 0;
    for (int t = 0; t < nv; ++t) {
        const int q = (int)((cs >> (4 * t)) & 15);
        if ((seen >> q) & 1u) continue;
        seen |= 1u << q;
        int off[3];
        key_off(kind, side, q, off);
        if (!creates(off, c, skip)) continue;
        if (q == target) return r;
        ++r;
    }
    return -1;
}

__global__ void k_mc_count(McGrid g, uint64_t items, uint8_t* __restrict__ cfg_out, uint32_t* __restrict__ nvert,
                           uint32_t* __restrict__ ntri)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < items; t += (uint64_t)gridDim.x * blockDim.x) {
        const Item it = decode(g, t);
        const int cfg = it.kind == 0 ? cube_case(g, it.c[0], it.c[1], it.c[2]) : cap_case(g, it.side, it.c);
        cfg_out[t] = (uint8_t)cfg;
        const unsigned long long cs = it.kind == 0 ? c_case3[cfg] : c_case2[cfg];
        const int nt = (int)(cs >> 60);
        unsigned used = 0u;
        for (int q = 0; q < 3 * nt; ++q) used |= 1u << ((cs >> (4 * q)) & 15);
        const int skip = skip_axis_of(it.kind, it.side);
        int created = 0;
        for (int q = 0; q < 12; ++q) {
            if (!((used >> q) & 1u)) continue;
            int off[3];
            key_off(it.kind, it.side, q, off);
            if (creates(off, it.c, skip)) ++created;
        }
        nvert[t] = (uint32_t)created;
        ntri[t] = (uint32_t)nt;
    }
}

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

// Grid3D::GridIndexToPosition (common/grid3d.hpp:20-23).
__device__ __forceinline__ double grid_pos(const McGrid& g, int a, int idx) { return da(g.o[a], dm((double)idx, g.h[a])); }

// MarchingCubesSolver::Gradient (marching_cubes_solver.cpp:116-155) at node (i, j, k).
__device__ void gradient(const McGrid& g, int i, int j, int k, double out[3])
{
    int ip = i + 1, im = i - 1, jp = j + 1, jm = j - 1, kp = k + 1, km = k - 1;
    if (i > g.n[0] - 2) ip = i; else if (i == 0) im = 0;
    if (j > g.n[1] - 2) jp = j; else if (j == 0) jm = 0;
    if (k > g.n[2] - 2) kp = k; else if (k == 0) km = 0;
    out[0] = dm(dm(0.5, __ddiv_rn(1.0, g.h[0])), ds(sdf_at(g, ip, j, k), sdf_at(g, im, j, k)));
    out[1] = dm(dm(0.5, __ddiv_rn(1.0, g.h[1])), ds(sdf_at(g, i, jp, k), sdf_at(g, i, jm, k)));
    out[2] = dm(dm(0.5, __ddiv_rn(1.0, g.h[2])), ds(sdf_at(g, i, j, kp), sdf_at(g, i, j, km)));
}

// The vertex (position, normal) of a cube's edge q (SolveSingleCube's e[] and n[], SafeNormalize).
__device__ void cube_vertex(const McGrid& g, const int c[3], int q, double p[3], double nrm[3])
{
    const int a = c_edge_corner[q][0], b = c_edge_corner[q][1];
    const double da0 = sdf_at(g, c[0] + c_corner_off[a][0], c[1] + c_corner_off[a][1], c[2] + c_corner_off[a][2]);
    const double db0 = sdf_at(g, c[0] + c_corner_off[b][0], c[1] + c_corner_off[b][1], c[2] + c_corner_off[b][2]);
    const double phi0 = ds(da0, 0.0), phi1 = ds(db0, 0.0);
    const double s = da(fabs(phi0), fabs(phi1));
    double alpha = s > 0.000000001 ? __ddiv_rn(fabs(phi0), s) : 0.5;
    if (alpha < 0.000001) alpha = 0.000001;
    if (alpha > 0.999999) alpha = 0.999999;
    const double w0 = ds(1.0, alpha);
    double ga[3], gb[3];
    gradient(g, c[0] + c_corner_off[a][0], c[1] + c_corner_off[a][1], c[2] + c_corner_off[a][2], ga);
    gradient(g, c[0] + c_corner_off[b][0], c[1] + c_corner_off[b][1], c[2] + c_corner_off[b][2], gb);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        // BoundingBox3D::Corner (3d/bounding_box_3d.cpp:23-31) of the cube's box: h * (+-1/2) + origin + h / 2
        const double bo = grid_pos(g, d, c[d]);
        const double half = dm(0.5, g.h[d]);
        const double p0 = da(da(dm(g.h[d], c_corner_off[a][d] ? 0.5 : -0.5), bo), half);
        const double p1 = da(da(dm(g.h[d], c_corner_off[b][d] ? 0.5 : -0.5), bo), half);
        p[d] = da(dm(w0, p0), dm(alpha, p1));
        nrm[d] = da(dm(w0, ga[d]), dm(alpha, gb[d]));
    }
    const double len = __dsqrt_rn(da(da(dm(nrm[0], nrm[0]), dm(nrm[1], nrm[1])), dm(nrm[2], nrm[2])));
    if (dm(len, len) > 0.0) {
        nrm[0] = __ddiv_rn(nrm[0], len);
        nrm[1] = __ddiv_rn(nrm[1], len);
        nrm[2] = __ddiv_rn(nrm[2], len);
    }
}

// The vertex of a cap square's key q (SolveSingleSquare: a corner, or the crossing on edge q - 4).
__device__ void cap_vertex(const McGrid& g, int side, const int c[3], int q, double p[3])
{
    if (q < 4) {
#pragma unroll
        for (int d = 0; d < 3; ++d) p[d] = grid_pos(g, d, c[d] + c_cap_corner[side][q][d]);
        return;
    }
    const int a = q - 4, b = (q - 3) & 3;
    int na[3], nb[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        na[d] = c[d] + c_cap_corner[side][a][d];
        nb[d] = c[d] + c_cap_corner[side][b][d];
    }
    const double phi0 = ds(sdf_at(g, na[0], na[1], na[2]), 0.0), phi1 = ds(sdf_at(g, nb[0], nb[1], nb[2]), 0.0);
    const double s = da(fabs(phi0), fabs(phi1));
    double alpha = s > 1e-12 ? __ddiv_rn(fabs(phi0), s) : (double)0.5f;
    if (alpha < (double)0.000001f) alpha = (double)0.000001f;
    if (alpha > (double)0.999999f) alpha = (double)0.999999f;
    const double w0 = ds(1.0, alpha);
#pragma unroll
    for (int d = 0; d < 3; ++d) p[d] = da(dm(w0, grid_pos(g, d, na[d])), dm(alpha, grid_pos(g, d, nb[d])));
}

__global__ void k_mc_emit(McGrid g, uint64_t items, const uint8_t* __restrict__ cfgs, const uint32_t* __restrict__ vbase,
                          const uint32_t* __restrict__ tbase, double* __restrict__ V, double* __restrict__ N,
                          int64_t* __restrict__ T)
{
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < items; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t tb = tbase[t];
        if (tbase[t + 1] == tb) continue;
        const Item it = decode(g, t);
        const int cfg = cfgs[t];
        const unsigned long long cs = it.kind == 0 ? c_case3[cfg] : c_case2[cfg];
        const int ntri = (int)(cs >> 60);
        const int skip = skip_axis_of(it.kind, it.side);
        const int64_t vb = vbase[t];
        int64_t vid[12];
        unsigned seen = 0u;
        int created = 0;
        for (int tri = 0; tri < ntri; ++tri) {
            int64_t f[3];
            for (int q3 = 0; q3 < 3; ++q3) {
                const int q = (int)((cs >> (4 * (3 * tri + q3))) & 15);
                if (!((seen >> q) & 1u)) {
                    seen |= 1u << q;
                    int off[3];
                    key_off(it.kind, it.side, q, off);
                    if (creates(off, it.c, skip)) {
                        const int64_t id = vb + created++;
                        double p[3], nrm[3];
                        if (it.kind == 0) {
                            cube_vertex(g, it.c, q, p, nrm);
                        } else {
                            cap_vertex(g, it.side, it.c, q, p);
                            nrm[0] = c_cap_normal[it.side][0];
                            nrm[1] = c_cap_normal[it.side][1];
                            nrm[2] = c_cap_normal[it.side][2];
                        }
                        V[3 * id] = p[0]; V[3 * id + 1] = p[1]; V[3 * id + 2] = p[2];
                        N[3 * id] = nrm[0]; N[3 * id + 1] = nrm[1]; N[3 * id + 2] = nrm[2];
                        vid[q] = id;
                    } else {
                        // the creating item: one step down along every axis where the key lies on this item's
                        // lower side and an item exists below; there the key's offset is 2
                        int oc[3], ooff[3];
#pragma unroll
                        for (int a = 0; a < 3; ++a) {
                            const bool down = a != skip && off[a] == 0 && it.c[a] > 0;
                            oc[a] = it.c[a] - (down ? 1 : 0);
                            ooff[a] = off[a] + (down ? 2 : 0);
                        }
                        int oq = -1;
                        const int nk = it.kind == 0 ? 12 : 8;
                        for (int k = 0; k < nk && oq < 0; ++k) {
                            int ko[3];
                            key_off(it.kind, it.side, k, ko);
                            if (ko[0] == ooff[0] && ko[1] == ooff[1] && ko[2] == ooff[2]) oq = k;
                        }
                        const uint64_t owner = it.kind == 0 ? encode_cube(g, oc[0], oc[1], oc[2]) : encode_cap(g, it.side, oc);
                        const int r = creation_rank(it.kind, it.side, oc, cfgs[owner], oq);
                        vid[q] = (int64_t)vbase[owner] + r;
                    }
                }
                f[q3] = vid[q];
            }
            int64_t* out = T + 4 * ((int64_t)tb + tri);
            out[0] = f[0];
            out[1] = f[1];
            out[2] = f[2];
            out[3] = vb + created - 1;  // mesh->GetNormals().size() - 1
        }
    }
}

}  // namespace

size_t mc_items(int nx, int ny, int nz)
{
    const size_t mx = nx - 1, my = ny - 1, mz = nz - 1;
    return mx * my * mz + 2 * (my * mx + mz * my + mz * mx);
}

cudaError_t launch_mc_count(const SceneView& v, const double* sdf, uint8_t* cfg, uint32_t* nvert, uint32_t* ntri,
                            cudaStream_t st)
{
    McGrid g;
    g.n[0] = v.g.nx; g.n[1] = v.g.ny; g.n[2] = v.g.nz;
    for (int a = 0; a < 3; ++a) { g.o[a] = v.sdf_origin[a]; g.h[a] = v.h[a]; }
    g.sdf = sdf;
    const uint64_t mx = g.n[0] - 1, my = g.n[1] - 1, mz = g.n[2] - 1;
    g.cubes = mx * my * mz;
    g.part0[0] = g.cubes;
    g.part0[1] = g.part0[0] + 2 * my * mx;
    g.part0[2] = g.part0[1] + 2 * mz * my;
    const uint64_t items = g.part0[2] + 2 * mz * mx;
    const unsigned blocks = (unsigned)std::min<uint64_t>((items + 255) / 256, 148 * 16);
    k_mc_count<<<blocks, 256, 0, st>>>(g, items, cfg, nvert, ntri);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_mc_emit(const SceneView& v, const double* sdf, const uint8_t* cfg, const uint32_t* vbase,
                           const uint32_t* tbase, double* V, double* N, int64_t* T, cudaStream_t st)
{
    McGrid g;
    g.n[0] = v.g.nx; g.n[1] = v.g.ny; g.n[2] = v.g.nz;
    for (int a = 0; a < 3; ++a) { g.o[a] = v.sdf_origin[a]; g.h[a] = v.h[a]; }
    g.sdf = sdf;
    const uint64_t mx = g.n[0] - 1, my = g.n[1] - 1, mz = g.n[2] - 1;
    g.cubes = mx * my * mz;
    g.part0[0] = g.cubes;
    g.part0[1] = g.part0[0] + 2 * my * mx;
    g.part0[2] = g.part0[1] + 2 * mz * my;
    const uint64_t items = g.part0[2] + 2 * mz * mx;
    const unsigned blocks = (unsigned)std::min<uint64_t>((items + 255) / 256, 148 * 16);
    k_mc_emit<<<blocks, 256, 0, st>>>(g, items, cfg, vbase, tbase, V, N, T);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe

// OBJManager::OnSave (3d/obj_manager.cpp:14-90): header, object name, "v" lines, "vn" lines, "s off", and "f a//n
// b//n c//n" with 1-based indices; numbers as std::to_string prints them ("%f"); the normal index is written as
// an unsigned value (a -1 prints as 0).  The lines are formatted by several host threads into per-range
// buffers and written in order, so the file is the same bytes as a serial writer's.
namespace {

template <class F>
void format_ranges(uint64_t n, F line, std::vector<std::string>& parts)
{
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = (unsigned)std::min<uint64_t>(std::min(hw, 32u), (n + 16383) / 16384);
    parts.assign(std::max(nt, 1u), std::string());
    auto work = [&](unsigned t) {
        const uint64_t b = n * t / std::max(nt, 1u), e = n * (t + 1) / std::max(nt, 1u);
        std::string& out = parts[t];
        out.reserve((size_t)(e - b) * 40);
        char buf[160];
        for (uint64_t i = b; i < e; ++i) {
            const int len = line(i, buf, sizeof(buf));
            out.append(buf, (size_t)len);
        }
    };
    if (nt <= 1) {
        work(0);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 1; t < nt; ++t) th.emplace_back(work, t);
    work(0);
    for (auto& x : th) x.join();
}

}  // namespace

extern "C" fe_status fe_write_obj(const char* path, const char* object_name, const double* vertices,
                                  const double* normals, uint64_t n_vertices, const int64_t* triangles,
                                  uint64_t n_triangles)
{
    if (!path || (n_vertices && (!vertices || !normals)) || (n_triangles && !triangles))
        return fe::set_error(FE_ERR_BAD_ARG, "null argument");
    FILE* f = std::fopen(path, "wb");
    if (!f) return fe::set_error(FE_ERR_BAD_ARG, "cannot open %s for writing", path);
    std::vector<std::string> parts;
    auto put = [&](const std::string& str) { std::fwrite(str.data(), 1, str.size(), f); };
    std::fprintf(f, "mtllib test.mtl\no %s\n\n", object_name ? object_name : "");
    format_ranges(n_vertices, [&](uint64_t i, char* b, size_t cap) {
        return std::snprintf(b, cap, "v %f %f %f\n", vertices[3 * i], vertices[3 * i + 1], vertices[3 * i + 2]);
    }, parts);
    for (const auto& p : parts) put(p);
    std::fputs("\n", f);
    format_ranges(n_vertices, [&](uint64_t i, char* b, size_t cap) {
        return std::snprintf(b, cap, "vn %f %f %f\n", normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
    }, parts);
    for (const auto& p : parts) put(p);
    std::fputs("\n", f);
    std::fputs("s off\n\n", f);
    format_ranges(n_triangles, [&](uint64_t i, char* b, size_t cap) {
        const int64_t* t = triangles + 4 * i;
        const uint64_t nn = (uint64_t)t[3] + 1u;
        return std::snprintf(b, cap, "f %" PRIu64 "//%" PRIu64 " %" PRIu64 "//%" PRIu64 " %" PRIu64 "//%" PRIu64 "\n",
                             (uint64_t)t[0] + 1u, nn, (uint64_t)t[1] + 1u, nn, (uint64_t)t[2] + 1u, nn);
    }, parts);
    for (const auto& p : parts) put(p);
    std::fputs("\n", f);
    const bool ok = std::ferror(f) == 0;
    if (std::fclose(f) != 0 || !ok) return fe::set_error(FE_ERR_BAD_ARG, "write to %s failed", path);
    return FE_OK;
}
