// fe_geom.cuh -- FP64 geometry shared by the mesh kernels (fe_mesh.cu) and the collider kernels (fe_collide.cu):
// the reference's point-triangle closest point and distance (Collisions, 3d/collisions.cpp:21-217), the winding
// test of TriangleMesh::IsInside and ScalarGrid3D::Sample on node grids, with explicit round-to-nearest
// intrinsics (no fused multiply-add) so results equal the reference's operation order.
#pragma once

#include "fe_internal.cuh"

namespace fe {
namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dot3(const double a[3], const double b[3]) { return da(da(dm(a[0], b[0]), dm(a[1], b[1])), dm(a[2], b[2])); }
__device__ __forceinline__ double len3(const double a[3]) { return __dsqrt_rn(dot3(a, a)); }

// Collisions::ClossestPointOnTriangle (3d/collisions.cpp:21-212), region by region.
__device__ __forceinline__ void closest_on_triangle(const double pt[3], const double p0[3], const double p1[3], const double p2[3],
                                    double out[3])
{
    double diff[3], e0[3], e1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) { diff[d] = ds(p0[d], pt[d]); e0[d] = ds(p1[d], p0[d]); e1[d] = ds(p2[d], p0[d]); }
    const double a00 = dot3(e0, e0), a01 = dot3(e0, e1), a11 = dot3(e1, e1);
    const double b0 = dot3(diff, e0), b1 = dot3(diff, e1);
    const double dt = ds(dm(a00, a11), dm(a01, a01));
    const double det = dt < 0.0 ? 0.0 : dt;  // std::max(x, 0.0)
    double s = ds(dm(a01, b1), dm(a11, b0));
    double t = ds(dm(a01, b0), dm(a00, b1));
    if (da(s, t) <= det) {
        if (s < 0) {
            if (t < 0) {  // region 4
                if (b0 < 0) {
                    t = 0;
                    s = (-b0 >= a00) ? 1.0 : dd(-b0, a00);
                } else {
                    s = 0;
                    t = (b1 >= 0) ? 0.0 : ((-b1 >= a11) ? 1.0 : dd(-b1, a11));
                }
            } else {  // region 3
                s = 0;
                t = (b1 >= 0) ? 0.0 : ((-b1 >= a11) ? 1.0 : dd(-b1, a11));
            }
        } else if (t < 0) {  // region 5
            t = 0;
            s = (b0 >= 0) ? 0.0 : ((-b0 >= a00) ? 1.0 : dd(-b0, a00));
        } else {  // region 0
            s = dd(s, det);
            t = dd(t, det);
        }
    } else {
        const double denom = da(ds(a00, dm(2.0, a01)), a11);
        if (s < 0) {  // region 2
            const double tmp0 = da(a01, b0), tmp1 = da(a11, b1);
            if (tmp1 > tmp0) {
                const double numer = ds(tmp1, tmp0);
                if (numer >= denom) { s = 1; t = 0; }
                else { s = dd(numer, denom); t = ds(1.0, s); }
            } else {
                s = 0;
                t = (tmp1 <= 0) ? 1.0 : ((b1 >= 0) ? 0.0 : dd(-b1, a11));
            }
        } else if (t < 0) {  // region 6
            const double tmp0 = da(a01, b1), tmp1 = da(a00, b0);
            if (tmp1 > tmp0) {
                const double numer = ds(tmp1, tmp0);
                if (numer >= denom) { t = 1; s = 0; }
                else { t = dd(numer, denom); s = ds(1.0, t); }
            } else {
                t = 0;
                s = (tmp1 <= 0) ? 1.0 : ((b0 >= 0) ? 0.0 : dd(-b0, a00));
            }
        } else {  // region 1
            const double numer = ds(ds(da(a11, b1), a01), b0);
            if (numer <= 0) { s = 0; t = 1; }
            else if (numer >= denom) { s = 1; t = 0; }
            else { s = dd(numer, denom); t = ds(1.0, s); }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) out[d] = da(da(p0[d], dm(s, e0[d])), dm(t, e1[d]));
}

// Collisions::DistanceToTriangle (3d/collisions.cpp:214-217): DistanceToPoint(point, closest point).
__device__ __forceinline__ double distance_to_triangle(const double pt[3], const double p0[3], const double p1[3], const double p2[3])
{
    double c[3];
    closest_on_triangle(pt, p0, p1, p2, c);
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = ds(c[d], pt[d]);
    return len3(c);
}

struct MeshView {
    const double* V;   // 3 per vertex
    const int64_t* T;  // 4 per triangle (three vertex ids, unused normal id)
    uint64_t nv, nt;
};

struct NodeGrid {
    int n[3];
    double o[3], h[3];
};

__device__ __forceinline__ double grid_pos(const NodeGrid& g, int a, int idx) { return da(g.o[a], dm((double)idx, g.h[a])); }

__device__ __forceinline__ void load_vertex(const MeshView& m, int64_t id, double out[3])
{
    out[0] = m.V[3 * id]; out[1] = m.V[3 * id + 1]; out[2] = m.V[3 * id + 2];
}

// The winding sum of TriangleMesh::IsInside (3d/triangle_mesh.cpp:120-163): atan2(det(A, B, C), k) over the
// triangles, A, B, C the vertices relative to the point (half the solid angle each).
__device__ __forceinline__ double winding_sum(const MeshView& m, const double pt[3])
{
    double ret = 0.0;
    for (uint64_t t = 0; t < m.nt; ++t) {
        double A[3], B[3], C[3];
        load_vertex(m, __ldg(m.T + 4 * t), A);
        load_vertex(m, __ldg(m.T + 4 * t + 1), B);
        load_vertex(m, __ldg(m.T + 4 * t + 2), C);
#pragma unroll
        for (int d = 0; d < 3; ++d) { A[d] = ds(A[d], pt[d]); B[d] = ds(B[d], pt[d]); C[d] = ds(C[d], pt[d]); }
        double omega = dm(dm(A[0], B[1]), C[2]);
        omega = da(omega, dm(dm(B[0], C[1]), A[2]));
        omega = da(omega, dm(dm(C[0], A[1]), B[2]));
        omega = ds(omega, dm(dm(C[0], B[1]), A[2]));
        omega = ds(omega, dm(dm(B[0], A[1]), C[2]));
        omega = ds(omega, dm(dm(A[0], C[1]), B[2]));
        const double na = len3(A), nb = len3(B), nc3 = len3(C);
        double kk = dm(dm(na, nb), nc3);
        kk = da(kk, dm(nc3, dot3(A, B)));
        kk = da(kk, dm(na, dot3(B, C)));
        kk = da(kk, dm(nb, dot3(C, A)));
        ret = da(ret, atan2(omega, kk));
    }
    return ret;
}

// TriangleMesh::IsInside: |winding sum| >= 2 pi - 0.001 (abs on the double, its meaning on the reference's platform).
__device__ __forceinline__ bool mesh_inside(const MeshView& m, const double pt[3])
{
    return fabs(winding_sum(m, pt)) >= ds(dm(2.0, 3.14159265358979323846), 0.001);
}

// ScalarGrid3D::Sample (3d/scalar_grid3d.cpp:33-65) of a node grid at a position, with GetBarycentric clamping.
__device__ __forceinline__ double sample_nodes(const double* __restrict__ f, const NodeGrid& g, const double pos[3])
{
    int i0[3];
    double fr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double x = dd(ds(pos[a], g.o[a]), g.h[a]);
        const int hiI = g.n[a] - 1;
        const double fl = floor(x);
        int ii = (int)fl;
        double ff;
        if (hiI == 0 || ii < 0) { ii = 0; ff = 0.0; }
        else if (ii > hiI - 1) { ii = hiI - 1; ff = 1.0; }
        else ff = ds(x, fl);
        i0[a] = ii;
        fr[a] = ff;
    }
    const int ip = min(i0[0] + 1, g.n[0] - 1), jp = min(i0[1] + 1, g.n[1] - 1), kp = min(i0[2] + 1, g.n[2] - 1);
    auto at = [&](int i, int j, int k) { return f[idx3(i, j, k, g.n[0], g.n[1])]; };
    auto lerp = [](double a, double b, double t) { return da(dm(ds(1.0, t), a), dm(t, b)); };
    const double b0 = lerp(lerp(at(i0[0], i0[1], i0[2]), at(ip, i0[1], i0[2]), fr[0]),
                           lerp(at(i0[0], jp, i0[2]), at(ip, jp, i0[2]), fr[0]), fr[1]);
    const double b1 = lerp(lerp(at(i0[0], i0[1], kp), at(ip, i0[1], kp), fr[0]),
                           lerp(at(i0[0], jp, kp), at(ip, jp, kp), fr[0]), fr[1]);
    return lerp(b0, b1, fr[2]);
}

}  // namespace
}  // namespace fe
