// fe_forces.cu -- position-dependent external forces: PointField, SwirlField, VolumeField.
//
// Reference: PICSimulator::ComputeExternalForces (pic_simulator.cpp:203-212) runs, for every force in the order
// added, ExternalForce::ApplyExternalForce (forces/external_force.cpp:3-29): each face of u, v and w adds
// dt * the force's component sampled at the face position (FaceCenteredGrid3D::GetXPos / GetYPos / GetZPos, the
// velocity grid's data origins + h * index), then ApplyBoundryCondition.  Samples:
//   PointField::Sample (forces/point_field.cpp:16-19): strength / max(|p - o|, 1) along (o - p) / |o - p|;
//   SwirlField::Sample (forces/swirlf_field.cpp:16-23): strength / max(d, 1)^2 along the normalised displacement of
//     p by a 0.0001-degree rotation about the axis (Collisions::RotatePointAroundAxis, 3d/collisions.cpp:219-237),
//     d = Collisions::DistanceToAxis (:239-246), which takes the (normalised) axis direction as a second point;
//   VolumeField::Sample (forces/volume_field.cpp:20-58): the trilinear closest-point vector q of its node grid,
//     strength / max(|q|, 1)^2 along -q / |q|.
//
// B200 design: the directional fields are gravity, added by the pre-solve extrapolation pass; the other forces run
// as one pass over all faces after it (one thread per face, the force list in kernel parameters), in FP64 with
// round-to-nearest intrinsics in the reference's operation order, and re-zero the wall layers (ApplyBoundryCondition
// without colliders).  The rotation's cos / sin are of a constant angle and are evaluated once on the host.
#include "fe_internal.cuh"

namespace fe {
namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }
// Vector3::GetLength (common/vector3.hpp:89-92)
__device__ __forceinline__ double vlen(double x, double y, double z)
{
    return __dsqrt_rn(da(da(dm(x, x), dm(y, y)), dm(z, z)));
}

__device__ __forceinline__ void point_sample(const ForceDev& f, const double p[3], double out[3])
{
    const double len = vlen(ds(p[0], f.origin[0]), ds(p[1], f.origin[1]), ds(p[2], f.origin[2]));
    const double dist = len >= 1.0 ? len : 1.0;
    double e[3] = {ds(f.origin[0], p[0]), ds(f.origin[1], p[1]), ds(f.origin[2], p[2])};
    const double el = vlen(e[0], e[1], e[2]);
    const double sc = dm(f.strength, dd(1.0, dist));
#pragma unroll
    for (int a = 0; a < 3; ++a) out[a] = dm(sc, dd(e[a], el));
}

__device__ __forceinline__ void swirl_sample(const ForceDev& f, const double p[3], double out[3])
{
    const double* o = f.origin;
    const double* ax = f.axis;
    const double d0 = vlen(ds(o[0], ax[0]), ds(o[1], ax[1]), ds(o[2], ax[2]));
    double dir[3], cl[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) dir[a] = dd(ds(ax[a], o[a]), d0);
    const double t = da(da(dm(ds(p[0], o[0]), dir[0]), dm(ds(p[1], o[1]), dir[1])), dm(ds(p[2], o[2]), dir[2]));
#pragma unroll
    for (int a = 0; a < 3; ++a) cl[a] = da(o[a], dm(t, dir[a]));
    double dist = vlen(ds(p[0], cl[0]), ds(p[1], cl[1]), ds(p[2], cl[2]));
    dist = dist >= 1.0 ? dist : 1.0;
    // RotatePointAroundAxis(o, axis, p, 0.0001): the axis is normalised again
    const double al = vlen(ax[0], ax[1], ax[2]);
    const double u = dd(ax[0], al), v = dd(ax[1], al), w = dd(ax[2], al);
    const double x = p[0], y = p[1], z = p[2];
    const double a = o[0], b = o[1], c = o[2];
    const double cA = f.cos_a, sA = f.sin_a, omc = ds(1.0, cA);
    const double t1 = ds(dm(a, da(dm(v, v), dm(w, w))),
                         dm(u, ds(ds(ds(da(dm(b, v), dm(c, w)), dm(u, x)), dm(v, y)), dm(w, z))));
    const double t2 = ds(dm(b, da(dm(u, u), dm(w, w))),
                         dm(v, ds(ds(ds(da(dm(a, u), dm(c, w)), dm(u, x)), dm(v, y)), dm(w, z))));
    const double t3 = ds(dm(c, da(dm(u, u), dm(v, v))),
                         dm(w, ds(ds(ds(da(dm(a, u), dm(b, v)), dm(u, x)), dm(v, y)), dm(w, z))));
    const double rx = da(da(dm(t1, omc), dm(x, cA)), dm(da(ds(da(dm(-c, v), dm(b, w)), dm(w, y)), dm(v, z)), sA));
    const double ry = da(da(dm(t2, omc), dm(y, cA)), dm(ds(da(ds(dm(c, u), dm(a, w)), dm(w, x)), dm(u, z)), sA));
    const double rz = da(da(dm(t3, omc), dm(z, cA)), dm(da(ds(da(dm(-b, u), dm(a, v)), dm(v, x)), dm(u, y)), sA));
    const double fd[3] = {ds(x, rx), ds(y, ry), ds(z, rz)};
    const double fl = vlen(fd[0], fd[1], fd[2]);
    const double sc = dm(f.strength, dd(1.0, dm(dist, dist)));
#pragma unroll
    for (int q = 0; q < 3; ++q) out[q] = dm(sc, dd(fd[q], fl));
}

// GetBarycentric (common/math_utils.hpp:48-73) with iLow = 0, iHigh = n - 1.
__device__ __forceinline__ void barycentric(double x, int n, int& i, double& f)
{
    const int hi = n - 1;
    const double fl = floor(x);
    int ii = (int)fl;
    if (hi == 0 || ii < 0) { ii = 0; f = 0.0; }
    else if (ii > hi - 1) { ii = hi - 1; f = 1.0; }
    else f = ds(x, fl);
    i = ii;
}

__device__ __forceinline__ double lerp(double a, double b, double t) { return da(dm(ds(1.0, t), a), dm(t, b)); }

__device__ __forceinline__ void volume_sample(const ForceDev& f, const double p[3], double out[3])
{
    int id[3], ip[3];
    double fr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        barycentric(dd(ds(p[a], f.o[a]), f.h[a]), f.n[a], id[a], fr[a]);
        ip[a] = min(id[a] + 1, f.n[a] - 1);
    }
    const size_t sx = (size_t)f.n[0], sxy = (size_t)f.n[0] * f.n[1];
    auto at = [&](int i, int j, int k, int c) { return __ldg(f.field + 3 * (i + sx * j + sxy * k) + c); };
    double sv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double b0 = lerp(lerp(at(id[0], id[1], id[2], c), at(ip[0], id[1], id[2], c), fr[0]),
                               lerp(at(id[0], ip[1], id[2], c), at(ip[0], ip[1], id[2], c), fr[0]), fr[1]);
        const double b1 = lerp(lerp(at(id[0], id[1], ip[2], c), at(ip[0], id[1], ip[2], c), fr[0]),
                               lerp(at(id[0], ip[1], ip[2], c), at(ip[0], ip[1], ip[2], c), fr[0]), fr[1]);
        sv[c] = lerp(b0, b1, fr[2]);
    }
    const double len = vlen(sv[0], sv[1], sv[2]);
    const double dist = len >= 1.0 ? len : 1.0;
    const double sc = dm(f.strength, dd(1.0, dm(dist, dist)));
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = dm(sc, -dd(sv[c], len));
}

__global__ void __launch_bounds__(kTileX * kTileY) k_forces(float* __restrict__ u, float* __restrict__ v,
                                                            float* __restrict__ w, int nx, int ny, int nz,
                                                            const ForceList fl, double hx, double hy, double hz,
                                                            double dt, bool zero_walls)
{
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    const int c = fc.c;
    float* arr = c == 0 ? u : (c == 1 ? v : w);
    const bool wall = (c == 0 && (fc.i == 0 || fc.i == fc.sx - 1)) || (c == 1 && (fc.j == 0 || fc.j == fc.sy - 1)) ||
                      (c == 2 && (fc.k == 0 || fc.k == fc.sz - 1));
    if (wall && zero_walls) {  // ApplyBoundryCondition re-zeroes the normal component on the six wall layers
        arr[fc.f] = 0.f;
        return;
    }
    // data origin of component c's faces: h / 2 on the other two axes, 0 on its own (0 + h * 0.5 with the velocity
    // grid's origin-independent data origins), plus h * index
    const double p[3] = {da(c == 0 ? 0.0 : dm(hx, 0.5), dm(hx, (double)fc.i)),
                         da(c == 1 ? 0.0 : dm(hy, 0.5), dm(hy, (double)fc.j)),
                         da(c == 2 ? 0.0 : dm(hz, 0.5), dm(hz, (double)fc.k))};
    double x = (double)arr[fc.f];
    for (int q = 0; q < fl.count; ++q) {
        const ForceDev& f = fl.f[q];
        double fv[3];
        if (f.kind == FE_FORCE_POINT) point_sample(f, p, fv);
        else if (f.kind == FE_FORCE_SWIRL) swirl_sample(f, p, fv);
        else volume_sample(f, p, fv);
        x = da(x, dm(dt, c == 0 ? fv[0] : (c == 1 ? fv[1] : fv[2])));  // by value: no local-memory array
    }
    arr[fc.f] = (float)x;
}

}  // namespace

cudaError_t launch_forces(const SceneView& v, const ForceList& fl, float* u, float* vv, float* ww, double dt,
                          cudaStream_t st, bool zero_walls)
{
    if (fl.count <= 0) return cudaSuccess;
    k_forces<<<face_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(u, vv, ww, v.g.nx, v.g.ny, v.g.nz, fl,
                                                                               v.h[0], v.h[1], v.h[2], dt, zero_walls);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
