// fe_collide.cu -- solid colliders (TriangleMeshCollider) on the substep path.
//
// Reference (with colliders the branches below replace the provable no-ops of the collider-free path):
//   ColliderCollection::BuildSdf (3d/collider_collection.cpp:33-50): every node of the collider SDF (the velocity
//     grid's n nodes at the domain origin) is the smallest TriangleMeshCollider::GetClosestDistanceAt, i.e. the
//     collider's own Mesh2SDF grid sampled there (3d/triangle_mesh_collider.cpp:4-23).
//   PICSimulator::ExtrapolateIntoCollider (pic_simulator.cpp:497-519): fluid-SDF nodes where the collider SDF is < 0
//     take ceil(maxCfl) rounds of ExtrapolateToRegion.
//   SinglePhasePressureSolver::BuildMarkers (fluid_solvers/single_phase_pressure_solver.cpp:30-48): FLUID if the
//     fluid SDF at the cell centre is < 0, else BOUNDRY if the collider SDF there is < 0, else AIR.
//   BlockedBoundryConditionSolver::ConstrainVelocity (fluid_solvers/blocked_boundry_condition_solver.cpp:18-291):
//     faces whose half-cell segment lies inside the collider are zeroed and refilled by ExtrapolateToRegion; faces
//     inside the collider take the tangential part of the sampled velocity (ApplyFriction with coefficient 0,
//     :324-333: v - n (v . n), n the normalised collider-SDF gradient, 3d/scalar_grid3d.cpp:67-90); the wall layers
//     and the faces between a cell whose collider-SDF node is < 0 and one whose node is not are zeroed.
//   PICSimulator::MoveParticles (pic_simulator.cpp:296-305): a particle that ends inside the collider SDF makes every
//     collider c run ResolveCollision (3d/triangle_mesh_collider.cpp:65-100) on particle number c -- the collider
//     loop's variable shadows the particle index -- from this particle's start position: particle c moves to the
//     closest point on collider c's mesh and, if it was inside that mesh, loses the normal part of its velocity.
//
// B200 design: the colliders are static, so everything that depends only on the collider SDF is classified once
// when a collider is added (node validity for the SDF extrapolation, BOUNDRY cells, per-face open / inside / zero
// bits).  Per substep: marks = band SDF (the surface path's scatter) -> node extrapolation passes -> cell samples;
// each ConstrainVelocity = block -> face extrapolation passes -> projection of the inside faces (into a scratch
// array, since it samples the whole grid) -> write-back with the zero bits.  The collision response keeps the
// reference's serial semantics without a serial pass over the particles: particles flag themselves by original
// index, a scan lists the inside ones in index order, one thread per (listed particle, collider) finds the closest
// triangle and tests its closest point against the mesh, and a single thread then replays the short chain of
// updates to particles 0 .. colliders-1 in the reference's order.  FP64 geometry throughout (fe_geom.cuh).
#include "fe_geom.cuh"

namespace fe {
namespace {

constexpr double kMaxDistance = 1.7976931348623157e30;  // 3d/collider_collection.cpp:3

__device__ __forceinline__ NodeGrid node_grid_of(const int n[3], const double o[3], const double h[3])
{
    NodeGrid g;
#pragma unroll
    for (int a = 0; a < 3; ++a) { g.n[a] = n[a]; g.o[a] = o[a]; g.h[a] = h[a]; }
    return g;
}

__device__ __forceinline__ MeshView mesh_of(const ColliderDev& c)
{
    MeshView m;
    m.V = c.V;
    m.T = c.T;
    m.nv = c.nv;
    m.nt = c.nt;
    return m;
}

// ColliderCollection::BuildSdf
__global__ void k_collider_sdf(CollideSet cs, int nx, int ny, int nz, double ox, double oy, double oz, double hx,
                               double hy, double hz, double* __restrict__ csdf)
{
    const size_t nc = (size_t)nx * ny * nz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const double p[3] = {da(ox, dm((double)i, hx)), da(oy, dm((double)j, hy)), da(oz, dm((double)k, hz))};
        double m = kMaxDistance;
        for (int q = 0; q < cs.count; ++q) {
            const NodeGrid g = node_grid_of(cs.c[q].n, cs.c[q].o, cs.c[q].h);
            const double d = sample_nodes(cs.c[q].sdf, g, p);
            if (d < m) m = d;
        }
        csdf[c] = m;
    }
}

// Node validity of ExtrapolateIntoCollider and BuildMarkers' BOUNDRY cells (both fixed by the collider SDF).
__global__ void k_collider_cells(SceneView v, const double* __restrict__ csdf, uint8_t* __restrict__ node_valid,
                                 uint8_t* __restrict__ cell_boundry)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    const int n[3] = {nx, ny, nz};
    const NodeGrid cg = node_grid_of(n, v.origin, v.h);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((size_t)nx * ny));
        const int id[3] = {i, j, k};
        double q[3], cc[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            q[a] = da(v.sdf_origin[a], dm((double)id[a], v.h[a]));                        // GridIndexToPosition
            cc[a] = da(da(v.origin[a], dm(0.5, v.h[a])), dm(v.h[a], (double)id[a]));       // GetCellCenterPos
        }
        node_valid[c] = sample_nodes(csdf, cg, q) < 0.0 ? 0 : 1;
        cell_boundry[c] = sample_nodes(csdf, cg, cc) < 0.0 ? 1 : 0;
    }
}

// Per face: open (its half-cell segment is not inside the collider), inside (the face position is), zero (a wall
// face of its component, or a face between a cell whose collider-SDF node is < 0 and one whose node is not).
__global__ void k_collider_faces(SceneView v, const double* __restrict__ csdf, uint8_t* __restrict__ open,
                                 uint8_t* __restrict__ cls)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    const int c = fc.c;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nvv = (size_t)nx * (ny + 1) * nz;
    const size_t g = (c == 0 ? 0 : (c == 1 ? nu : nu + nvv)) + fc.f;
    const int n[3] = {nx, ny, nz};
    const NodeGrid cg = node_grid_of(n, v.origin, v.h);
    const int id[3] = {fc.i, fc.j, fc.k};
    double p[3], p0[3], p1[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        p[a] = da(a == c ? 0.0 : dm(v.h[a], 0.5), dm(v.h[a], (double)id[a]));  // origin-independent data origins
        const double off = a == c ? dm(0.5, v.h[a]) : 0.0;
        p0[a] = ds(p[a], off);
        p1[a] = da(p[a], off);
    }
    const double phi0 = sample_nodes(csdf, cg, p0), phi1 = sample_nodes(csdf, cg, p1);
    double frac;  // FractionInsideSdf (blocked_boundry_condition_solver.cpp:304-322)
    if (phi0 < 0.0 && phi1 < 0.0) frac = 1.0;
    else if (phi0 < 0.0 && !(phi1 < 0.0)) frac = dd(phi0, ds(phi0, phi1));
    else if (!(phi0 < 0.0) && phi1 < 0.0) frac = dd(phi1, ds(phi1, phi0));
    else frac = 0.0;
    frac = ds(1.0, frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac));  // 1 - Clamp(frac, 1, 0)
    uint8_t k = 0;
    if (sample_nodes(csdf, cg, p) < 0.0) k |= kFaceInside;
    const int ic = id[c], lim = c == 0 ? fc.sx : (c == 1 ? fc.sy : fc.sz);
    if (ic == 0 || ic == lim - 1) {
        k |= kFaceZero;
    } else {
        const size_t sxy = (size_t)nx * ny;
        const size_t cell = idx3(fc.i, fc.j, fc.k, nx, ny);  // the cell on the + side; the - side is one step back
        const size_t back = c == 0 ? 1 : (c == 1 ? (size_t)nx : sxy);
        if ((csdf[cell] < 0.0) != (csdf[cell - back] < 0.0)) k |= kFaceZero;
    }
    open[g] = frac > 0.0 ? 1 : 0;
    cls[g] = k;
}

// Faces (u | v | w numbering) as a reference into the three velocity buffers, and their coordinates.
__device__ __forceinline__ float& face_at(float* u, float* vv, float* w, size_t nu, size_t nvv, uint32_t g)
{
    return g < nu ? u[g] : (g < nu + nvv ? vv[g - nu] : w[g - nu - nvv]);
}
__device__ __forceinline__ void face_index_coord(uint32_t g, int nx, int ny, size_t nu, size_t nvv, int& c, int id[3])
{
    size_t f = g;
    int sx = nx, sy = ny;
    if (g < nu) { c = 0; sx = nx + 1; }
    else if (g < nu + nvv) { c = 1; f -= nu; sy = ny + 1; }
    else { c = 2; f -= nu + nvv; }
    id[0] = (int)(f % sx);
    id[1] = (int)((f / sx) % sy);
    id[2] = (int)(f / ((size_t)sx * sy));
}

// ConstrainVelocity: blocked faces to 0 before the extrapolation (the fixed list of faces that are not open).
__global__ void k_bc_block(float* u, float* vv, float* w, size_t nu, size_t nvv, const uint32_t* __restrict__ list,
                           uint32_t n)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x)
        face_at(u, vv, w, nu, nvv, list[e]) = 0.f;
}

// ScalarGrid3D::Gradient of the collider SDF at p.
__device__ void collider_gradient(const double* __restrict__ csdf, const NodeGrid& g, const double p[3], double out[3])
{
    int id[3], ip[3];
    double fr[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double x = dd(ds(p[a], g.o[a]), g.h[a]);
        const int hi = g.n[a] - 1;
        const double fl = floor(x);
        int ii = (int)fl;
        double ff;
        if (hi == 0 || ii < 0) { ii = 0; ff = 0.0; }
        else if (ii > hi - 1) { ii = hi - 1; ff = 1.0; }
        else ff = ds(x, fl);
        id[a] = ii;
        fr[a] = ff;
        ip[a] = min(ii + 1, g.n[a] - 1);
    }
    const double fx = fr[0], fy = fr[1], fz = fr[2];
    const double w[8] = {dm(dm(ds(1.0, fx), ds(1.0, fy)), ds(1.0, fz)), dm(dm(fx, ds(1.0, fy)), ds(1.0, fz)),
                         dm(dm(ds(1.0, fx), fy), ds(1.0, fz)),        dm(dm(fx, fy), ds(1.0, fz)),
                         dm(dm(ds(1.0, fx), ds(1.0, fy)), fz),        dm(dm(fx, ds(1.0, fy)), fz),
                         dm(dm(ds(1.0, fx), fy), fz),                 dm(dm(fx, fy), fz)};
    const int sx = g.n[0], sy = g.n[1], sz = g.n[2];
    auto at = [&](int i, int j, int k) { return __ldg(csdf + idx3(i, j, k, sx, sy)); };
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int i = (t & 1) ? ip[0] : id[0], j = (t & 2) ? ip[1] : id[1], k = (t & 4) ? ip[2] : id[2];
        const double left = at(i > 0 ? i - 1 : i, j, k), right = at(i + 1 < sx ? i + 1 : i, j, k);
        const double down = at(i, j > 0 ? j - 1 : j, k), up = at(i, j + 1 < sy ? j + 1 : j, k);
        const double back = at(i, j, k > 0 ? k - 1 : k), front = at(i, j, k + 1 < sz ? k + 1 : k);
        const double wt = dm(w[t], 0.5);
        r0 = da(r0, dd(dm(wt, ds(right, left)), g.h[0]));
        r1 = da(r1, dd(dm(wt, ds(up, down)), g.h[1]));
        r2 = da(r2, dd(dm(wt, ds(front, back)), g.h[2]));
    }
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
}

// A rewritten face's list entry: its face index, with kFinProject set when it is projected onto the collider's
// tangent plane (inside, not zero, and a non-zero SDF gradient); the other entries are set to 0.
constexpr uint32_t kFinProject = 0x80000000u;

// The fixed face lists of a static collider classification: the blocked faces, and the faces ConstrainVelocity
// rewrites with the unit collider normal (FP64) at the projected ones.  With count_only the kernel only counts
// them into cnt[0] and cnt[1]; list order does not matter (every entry is independent).
__global__ void k_collider_face_lists(SceneView v, const double* __restrict__ csdf, const uint8_t* __restrict__ open,
                                      const uint8_t* __restrict__ cls, uint32_t* cnt, uint32_t* __restrict__ blk,
                                      uint32_t* __restrict__ fin, double* __restrict__ fin_nrm, int count_only)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    const int c = fc.c;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nvv = (size_t)nx * (ny + 1) * nz;
    const size_t g = (c == 0 ? 0 : (c == 1 ? nu : nu + nvv)) + fc.f;
    if (!open[g]) {
        const uint32_t e = atomicAdd(cnt, 1u);
        if (!count_only) blk[e] = (uint32_t)g;
    }
    const uint8_t k = cls[g];
    if (!(k & (kFaceInside | kFaceZero))) return;
    const uint32_t e = atomicAdd(cnt + 1, 1u);
    if (count_only) return;
    uint32_t entry = (uint32_t)g;
    double nrm[3] = {0.0, 0.0, 0.0};
    if (!(k & kFaceZero)) {
        const int id[3] = {fc.i, fc.j, fc.k};
        double p[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[a] = da(a == c ? 0.0 : dm(v.h[a], 0.5), dm(v.h[a], (double)id[a]));
        const int n[3] = {nx, ny, nz};
        const NodeGrid cg = node_grid_of(n, v.origin, v.h);
        double gr[3];
        collider_gradient(csdf, cg, p, gr);
        const double gl = len3(gr);
        if (dm(gl, gl) > 0.0) {
            nrm[0] = dd(gr[0], gl);
            nrm[1] = dd(gr[1], gl);
            nrm[2] = dd(gr[2], gl);
            entry |= kFinProject;
        }
    }
    fin[e] = entry;
    fin_nrm[3 * (size_t)e] = nrm[0];
    fin_nrm[3 * (size_t)e + 1] = nrm[1];
    fin_nrm[3 * (size_t)e + 2] = nrm[2];
}

// ConstrainVelocity's projection of the faces inside the collider (it samples the whole grid, so the results go to
// `tmp`, one per list entry, and are written back by k_bc_finish).
__global__ void k_bc_friction(SceneView v, const float* __restrict__ u, const float* __restrict__ vv,
                              const float* __restrict__ w, const uint32_t* __restrict__ fin,
                              const double* __restrict__ fin_nrm, uint32_t n, float* __restrict__ tmp)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nvv = (size_t)nx * (ny + 1) * nz;
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t entry = fin[e];
        if (!(entry & kFinProject)) continue;
        int c, id[3];
        face_index_coord(entry & ~kFinProject, nx, ny, nu, nvv, c, id);
        double p[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) p[a] = da(a == c ? 0.0 : dm(v.h[a], 0.5), dm(v.h[a], (double)id[a]));
        const float pf[3] = {(float)p[0], (float)p[1], (float)p[2]};
        const double vel[3] = {sample_face(u, pf[0], pf[1], pf[2], v.xo, v.inv_hf, nx + 1, ny, nz),
                               sample_face(vv, pf[0], pf[1], pf[2], v.yo, v.inv_hf, nx, ny + 1, nz),
                               sample_face(w, pf[0], pf[1], pf[2], v.zo, v.inv_hf, nx, ny, nz + 1)};
        const double nrm[3] = {fin_nrm[3 * (size_t)e], fin_nrm[3 * (size_t)e + 1], fin_nrm[3 * (size_t)e + 2]};
        const double d = dot3(vel, nrm);
        const double vc = c == 0 ? vel[0] : (c == 1 ? vel[1] : vel[2]);
        const double ncmp = c == 0 ? nrm[0] : (c == 1 ? nrm[1] : nrm[2]);
        tmp[e] = (float)da(ds(vc, dm(ncmp, d)), 0.0);
    }
}

// ConstrainVelocity's write-back: projected inside faces, every other listed face (zero bit, or no normal) to 0.
__global__ void k_bc_finish(float* u, float* vv, float* w, size_t nu, size_t nvv, const uint32_t* __restrict__ fin,
                            uint32_t n, const float* __restrict__ tmp)
{
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
        const uint32_t entry = fin[e];
        face_at(u, vv, w, nu, nvv, entry & ~kFinProject) = (entry & kFinProject) ? tmp[e] : 0.f;
    }
}

// One pass of ExtrapolateToRegion over the fluid-SDF nodes (FP64), neighbour order i+1, i-1, j+1, j-1, k+1, k-1.
__global__ void k_extrap_nodes(const double* __restrict__ in, double* __restrict__ out, const uint8_t* __restrict__ vin,
                               uint8_t* __restrict__ vout, int nx, int ny, int nz)
{
    const size_t nc = (size_t)nx * ny * nz, sxy = (size_t)nx * ny;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        double val = in[c];
        uint8_t valid = vin[c];
        if (!valid) {
            const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / sxy);
            double sum = 0.0;
            unsigned count = 0;
            if (i + 1 < nx && vin[c + 1]) { sum = da(sum, in[c + 1]); ++count; }
            if (i > 0 && vin[c - 1]) { sum = da(sum, in[c - 1]); ++count; }
            if (j + 1 < ny && vin[c + nx]) { sum = da(sum, in[c + nx]); ++count; }
            if (j > 0 && vin[c - nx]) { sum = da(sum, in[c - nx]); ++count; }
            if (k + 1 < nz && vin[c + sxy]) { sum = da(sum, in[c + sxy]); ++count; }
            if (k > 0 && vin[c - sxy]) { sum = da(sum, in[c - sxy]); ++count; }
            if (count > 0) {
                val = dd(sum, (double)count);
                valid = 1;
            }
        }
        out[c] = val;
        vout[c] = valid;
    }
}

// BuildMarkers with colliders.
__global__ void k_mark_collider(SceneView v, const double* __restrict__ sdf, const uint8_t* __restrict__ cell_boundry)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    const int n[3] = {nx, ny, nz};
    const NodeGrid sg = node_grid_of(n, v.sdf_origin, v.h);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int id[3] = {(int)(c % nx), (int)((c / nx) % ny), (int)(c / ((size_t)nx * ny))};
        double cc[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) cc[a] = da(da(v.origin[a], dm(0.5, v.h[a])), dm(v.h[a], (double)id[a]));
        v.marks[c] = sample_nodes(sdf, sg, cc) < 0.0 ? FE_CELL_FLUID
                                                    : (cell_boundry[c] ? FE_CELL_BOUNDRY : FE_CELL_AIR);
    }
}

// Start positions and velocities of the move (by slot, after TransferGrid2Particles), kept before MoveParticles
// overwrites them.
__global__ void k_keep_start(SceneView v, float* __restrict__ start, float* __restrict__ startv)
{
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    start[3 * p] = v.px[p];
    start[3 * p + 1] = v.py[p];
    start[3 * p + 2] = v.pz[p];
    startv[3 * p] = v.vx[p];
    startv[3 * p + 1] = v.vy[p];
    startv[3 * p + 2] = v.vz[p];
}

// After the move: particles whose new position samples the collider SDF below 0 flag their original index
// (indices >= the collider count; the first ones are replayed serially) and store their start position by index.
__global__ void k_collide_flags(SceneView v, const double* __restrict__ csdf, int ncoll, const float* __restrict__ start,
                                uint32_t* __restrict__ flag, float* __restrict__ spos, uint32_t* __restrict__ slot_of)
{
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    const uint32_t pid = v.pid[p];
    if (pid < (uint32_t)ncoll) {
        slot_of[pid] = (uint32_t)p;
        return;
    }
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    const NodeGrid cg = node_grid_of(n, v.origin, v.h);
    const double q[3] = {v.px[p], v.py[p], v.pz[p]};
    if (sample_nodes(csdf, cg, q) < 0.0) {
        flag[pid] = 1u;
        spos[3 * (size_t)pid] = start[3 * p];
        spos[3 * (size_t)pid + 1] = start[3 * p + 1];
        spos[3 * (size_t)pid + 2] = start[3 * p + 2];
    }
}

__global__ void k_collide_compact(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ offs, uint64_t np,
                                  uint32_t* __restrict__ list)
{
    for (uint64_t pid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; pid < np; pid += (uint64_t)gridDim.x * blockDim.x)
        if (flag[pid]) list[offs[pid]] = (uint32_t)pid;
}

// ResolveCollision's geometry for one start position: the first nearest triangle's closest point and normal.
__device__ void closest_feature(const ColliderDev& c, const double s[3], double cp[3], double nrm[3])
{
    const MeshView m = mesh_of(c);
    double best = kMaxDistance;
    uint64_t idx = 0;
    double A[3], B[3], C[3];
    for (uint64_t t = 0; t < m.nt; ++t) {
        load_vertex(m, __ldg(m.T + 4 * t), A);
        load_vertex(m, __ldg(m.T + 4 * t + 1), B);
        load_vertex(m, __ldg(m.T + 4 * t + 2), C);
        const double d = distance_to_triangle(s, A, B, C);
        if (d < best) {
            best = d;
            idx = t;
        }
    }
    load_vertex(m, m.T[4 * idx], A);
    load_vertex(m, m.T[4 * idx + 1], B);
    load_vertex(m, m.T[4 * idx + 2], C);
    closest_on_triangle(s, A, B, C, cp);
    const int64_t ni = m.T[4 * idx + 3];
    nrm[0] = c.N[3 * ni];
    nrm[1] = c.N[3 * ni + 1];
    nrm[2] = c.N[3 * ni + 2];
}

// Per (listed particle, collider): the closest point and normal from the particle's start, and whether that
// closest point is inside the collider's mesh (the test the next listed particle's resolution makes).
__global__ void k_collide_prep(CollideSet cs, const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                               const float* __restrict__ spos, double* __restrict__ cp, double* __restrict__ nrm,
                               uint8_t* __restrict__ ins)
{
    const uint64_t total = (uint64_t)(*count) * cs.count;
    for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < total; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t entry = e / cs.count;
        const int c = (int)(e % cs.count);
        const uint32_t pid = list[entry];
        const double s[3] = {spos[3 * (size_t)pid], spos[3 * (size_t)pid + 1], spos[3 * (size_t)pid + 2]};
        double q[3], nv[3];
        closest_feature(cs.c[c], s, q, nv);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            cp[3 * e + a] = q[a];
            nrm[3 * e + a] = nv[a];
        }
        ins[e] = mesh_inside(mesh_of(cs.c[c]), q) ? 1 : 0;
    }
}

// Entry k = e * colliders + c reflects particle c iff the previous entry's closest point was inside collider c's
// mesh (entries e >= 1; the first entry's test uses the particle's own position and is made serially).
__global__ void k_collide_active(const uint32_t* __restrict__ count, int ncoll, const uint8_t* __restrict__ ins,
                                 uint32_t* __restrict__ act)
{
    const uint64_t total = (uint64_t)(*count) * ncoll;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= total; k += (uint64_t)gridDim.x * blockDim.x)
        act[k] = (k < total && k >= (uint64_t)ncoll && ins[k - ncoll]) ? 1u : 0u;
}

__global__ void k_collide_active_compact(const uint32_t* __restrict__ count, int ncoll, const uint32_t* __restrict__ act,
                                         const uint32_t* __restrict__ offs, uint32_t* __restrict__ list)
{
    const uint64_t total = (uint64_t)(*count) * ncoll;
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < total; k += (uint64_t)gridDim.x * blockDim.x)
        if (act[k]) list[offs[k]] = (uint32_t)k;
}

// The velocity part of ResolveCollision for a particle inside the mesh (restitution 0, friction 0).
__device__ void reflect(double vel[3], const double nrm[3])
{
    const double rv[3] = {ds(vel[0], 0.0), ds(vel[1], 0.0), ds(vel[2], 0.0)};
    const double nd = dot3(nrm, rv);
    double rn[3] = {dm(nd, nrm[0]), dm(nd, nrm[1]), dm(nd, nrm[2])};
    double rt[3] = {ds(rv[0], rn[0]), ds(rv[1], rn[1]), ds(rv[2], rn[2])};
    if (nd < 0.0) {
        const double drn[3] = {dm(-1.0, rn[0]), dm(-1.0, rn[1]), dm(-1.0, rn[2])};
#pragma unroll
        for (int a = 0; a < 3; ++a) rn[a] = dm(rn[a], -0.0);
        if (dot3(rt, rt) > 0.0) {
            const double q = ds(1.0, dd(dm(0.0, len3(drn)), len3(rt)));
            const double fs = q < 0.0 ? 0.0 : q;
#pragma unroll
            for (int a = 0; a < 3; ++a) rt[a] = dm(rt[a], fs);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) vel[a] = da(da(rn[a], rt[a]), 0.0);
}

// One MoveParticles RK2 path and domain clamp (the k_g2p move in FP32) for a particle whose start a resolution
// changed before its own turn.
__device__ void move_one(const SceneView& v, const CollideMove& g, float pt[3], float vel[3])
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    auto sample = [&](const float x[3], float out[3]) {
        out[0] = sample_face(g.u, x[0], x[1], x[2], v.xo, v.inv_hf, nx + 1, ny, nz);
        out[1] = sample_face(g.v, x[0], x[1], x[2], v.yo, v.inv_hf, nx, ny + 1, nz);
        out[2] = sample_face(g.w, x[0], x[1], x[2], v.zo, v.inv_hf, nx, ny, nz + 1);
    };
    float pt0[3] = {pt[0], pt[1], pt[2]}, pt1[3] = {pt[0], pt[1], pt[2]};
    const float half = 0.5f * g.dt_sub;
    for (int t = 0; t < g.nsub; ++t) {
        float v0[3], vm[3];
        sample(pt0, v0);
        const float mid[3] = {pt0[0] + half * v0[0], pt0[1] + half * v0[1], pt0[2] + half * v0[2]};
        sample(mid, vm);
        for (int a = 0; a < 3; ++a) pt1[a] = pt0[a] + g.dt_sub * vm[a];
        for (int a = 0; a < 3; ++a) pt0[a] = pt1[a];
    }
    for (int a = 0; a < 3; ++a) {
        if (pt1[a] <= g.lo[a]) { pt1[a] = g.lo[a]; vel[a] = 0.f; }
        if (pt1[a] >= g.hi[a]) { pt1[a] = g.hi[a]; vel[a] = 0.f; }
        if (!(pt1[a] == pt1[a])) { pt1[a] = g.lo[a]; vel[a] = 0.f; }
        pt[a] = pt1[a];
    }
}

// The reference's serial order for particles 0 .. nc-1, then the listed particles' resolutions in index order.
// Before its own turn a particle holds its start state (position and TransferGrid2Particles velocity); a
// resolution triggered by an earlier particle can change that state, and its move then starts from there.
__global__ void k_collide_serial(CollideSet cs, SceneView v, CollideMove g, const double* __restrict__ csdf,
                                 const float* __restrict__ start, const float* __restrict__ startv,
                                 const uint32_t* __restrict__ slot_of, const uint32_t* __restrict__ count,
                                 const double* __restrict__ cp, const double* __restrict__ nrm,
                                 const uint32_t* __restrict__ act_offs, const uint32_t* __restrict__ act_list)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int nc = (int)min((uint64_t)cs.count, v.np);
    double P[kMaxColliders][3], V[kMaxColliders][3];
    bool touched[kMaxColliders];
    for (int c = 0; c < nc; ++c) {
        const uint32_t s = slot_of[c];
        P[c][0] = start[3 * s]; P[c][1] = start[3 * s + 1]; P[c][2] = start[3 * s + 2];
        V[c][0] = startv[3 * s]; V[c][1] = startv[3 * s + 1]; V[c][2] = startv[3 * s + 2];
        touched[c] = false;
    }
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    const NodeGrid cg = node_grid_of(n, v.origin, v.h);
    for (int i = 0; i < nc; ++i) {
        const double st[3] = {P[i][0], P[i][1], P[i][2]};  // startParticlePosition
        if (touched[i]) {  // its start is where an earlier resolution put it: move from there
            float pt[3] = {(float)P[i][0], (float)P[i][1], (float)P[i][2]};
            float vel[3] = {(float)V[i][0], (float)V[i][1], (float)V[i][2]};
            move_one(v, g, pt, vel);
            for (int a = 0; a < 3; ++a) { P[i][a] = pt[a]; V[i][a] = vel[a]; }
        } else {  // untouched: the parallel move's result
            const uint32_t s = slot_of[i];
            P[i][0] = v.px[s]; P[i][1] = v.py[s]; P[i][2] = v.pz[s];
            V[i][0] = v.vx[s]; V[i][1] = v.vy[s]; V[i][2] = v.vz[s];
        }
        if (sample_nodes(csdf, cg, P[i]) < 0.0) {
            for (int c = 0; c < nc; ++c) {
                double cpt[3], nv[3];
                closest_feature(cs.c[c], st, cpt, nv);
                if (mesh_inside(mesh_of(cs.c[c]), P[c])) reflect(V[c], nv);
                for (int a = 0; a < 3; ++a) P[c][a] = cpt[a];
                if (c > i) touched[c] = true;
            }
        }
    }
    // The listed particles' resolutions: particle c reflects at entry e when it was inside the mesh, i.e. at the
    // first entry by its own position and later by the previous entry's closest point (ins); the entries where
    // that holds were compacted in order (act_list), and its final position is the last entry's closest point.
    const uint32_t cnt = nc > 0 ? *count : 0u;
    if (cnt > 0) {
        for (int c = 0; c < nc; ++c)
            if (mesh_inside(mesh_of(cs.c[c]), P[c])) reflect(V[c], nrm + 3 * (size_t)c);
        const uint32_t nact = act_offs[(size_t)cnt * cs.count];
        for (uint32_t a = 0; a < nact; ++a) {
            const uint32_t k = act_list[a];
            const int c = (int)(k % cs.count);
            if (c < nc) reflect(V[c], nrm + 3 * (size_t)k);
        }
        for (int c = 0; c < nc; ++c)
            for (int a = 0; a < 3; ++a) P[c][a] = cp[3 * ((size_t)(cnt - 1) * cs.count + c) + a];
    }
    for (int c = 0; c < nc; ++c) {
        const uint32_t s = slot_of[c];
        v.px[s] = (float)P[c][0]; v.py[s] = (float)P[c][1]; v.pz[s] = (float)P[c][2];
        v.vx[s] = (float)V[c][0]; v.vy[s] = (float)V[c][1]; v.vz[s] = (float)V[c][2];
    }
}

// MarchingCubesSolver::BuildSurface with colliders (3d/marching_cubes_solver.cpp:31-37): nodes inside both the fluid
// and the collider take minus the collider SDF.
__global__ void k_surface_with_colliders(const double* __restrict__ fluid, const double* __restrict__ csdf, size_t n,
                                         double* __restrict__ out)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        out[c] = (fluid[c] < 0.0 && csdf[c] < 0.0) ? dm(csdf[c], -1.0) : fluid[c];
}

// ExternalForce::ApplyExternalForce of the DirectionalFields (the scene's gravity) on every face, wall faces
// included: with colliders the boundary condition that follows is the full ConstrainVelocity.
__global__ void k_add_gravity(float* u, float* vv, float* w, int nx, int ny, int nz, float gx, float gy, float gz)
{
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    float* a = fc.c == 0 ? u : (fc.c == 1 ? vv : w);
    a[fc.f] += fc.c == 0 ? gx : (fc.c == 1 ? gy : gz);
}

unsigned node_blocks(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

// Connected FLUID components (union-find with atomicMin links; every loop is bounded and reports through err).
constexpr uint32_t kNoLabel = 0xffffffffu;
constexpr int kFindLimit = 1 << 24;

__device__ __forceinline__ uint32_t find_root(const uint32_t* label, uint32_t x, int* err)
{
    for (int it = 0; it < kFindLimit; ++it) {
        const uint32_t p = __ldcg(label + x);
        if (p == x) return x;
        x = p;
    }
    atomicExch(err, FE_ERR_TIMEOUT);
    return x;
}

__global__ void k_ccl_init(const uint8_t* __restrict__ marks, size_t nc, uint32_t* __restrict__ label,
                           uint8_t* __restrict__ open_comp, double* __restrict__ sum, uint32_t* __restrict__ cnt)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        label[c] = marks[c] == FE_CELL_FLUID ? (uint32_t)c : kNoLabel;
        open_comp[c] = 0;
        sum[c] = 0.0;
        cnt[c] = 0u;
    }
}

__global__ void k_ccl_union(const uint8_t* __restrict__ marks, int nx, int ny, int nz, uint32_t* label, int* err)
{
    const size_t nc = (size_t)nx * ny * nz, sxy = (size_t)nx * ny;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (marks[c] != FE_CELL_FLUID) continue;
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / sxy);
        const size_t nb[3] = {i > 0 ? c - 1 : c, j > 0 ? c - nx : c, k > 0 ? c - sxy : c};
        for (int q = 0; q < 3; ++q) {
            if (nb[q] == c || marks[nb[q]] != FE_CELL_FLUID) continue;
            uint32_t a = (uint32_t)c, b = (uint32_t)nb[q];
            for (int it = 0; it < kFindLimit; ++it) {
                a = find_root(label, a, err);
                b = find_root(label, b, err);
                if (a == b) break;
                if (a > b) { const uint32_t t = a; a = b; b = t; }
                const uint32_t old = atomicMin(label + b, a);  // link the larger root under the smaller
                if (old == b) break;
                b = old;
                if (it == kFindLimit - 1) atomicExch(err, FE_ERR_TIMEOUT);
            }
        }
    }
}

// Roots of components with an AIR neighbour (a Dirichlet condition); every FLUID cell's label becomes its root.
__global__ void k_ccl_classify(const uint8_t* __restrict__ marks, int nx, int ny, int nz, uint32_t* label,
                               uint8_t* __restrict__ open_comp, int* err)
{
    const size_t nc = (size_t)nx * ny * nz, sxy = (size_t)nx * ny;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (marks[c] != FE_CELL_FLUID) continue;
        const uint32_t r = find_root(label, (uint32_t)c, err);
        label[c] = r;
        const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / sxy);
        const bool air = (i > 0 && marks[c - 1] == FE_CELL_AIR) || (i + 1 < nx && marks[c + 1] == FE_CELL_AIR) ||
                         (j > 0 && marks[c - nx] == FE_CELL_AIR) || (j + 1 < ny && marks[c + nx] == FE_CELL_AIR) ||
                         (k > 0 && marks[c - sxy] == FE_CELL_AIR) || (k + 1 < nz && marks[c + sxy] == FE_CELL_AIR);
        if (air && !open_comp[r]) open_comp[r] = 1;
    }
}

// Right-hand-side sums of the enclosed components only (the open ones, the bulk of the fluid, need none).
__global__ void k_ccl_sums(const uint8_t* __restrict__ marks, const double* __restrict__ b, size_t nc,
                           const uint32_t* __restrict__ label, const uint8_t* __restrict__ open_comp,
                           double* __restrict__ sum, uint32_t* __restrict__ cnt)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (marks[c] != FE_CELL_FLUID) continue;
        const uint32_t r = label[c];
        if (open_comp[r]) continue;
        atomicAdd(sum + r, b[c]);
        atomicAdd(cnt + r, 1u);
    }
}

// A component without AIR neighbours is a pure-Neumann block: its right-hand side loses its mean, which leaves a
// consistent system unchanged and makes an inconsistent one solvable.
__global__ void k_ccl_project(const uint8_t* __restrict__ marks, size_t nc, const uint32_t* __restrict__ label,
                              const uint8_t* __restrict__ open_comp, const double* __restrict__ sum,
                              const uint32_t* __restrict__ cnt, double* __restrict__ b)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        if (marks[c] != FE_CELL_FLUID) continue;
        const uint32_t r = label[c];
        if (open_comp[r]) continue;
        b[c] -= sum[r] / (double)cnt[r];
    }
}

// Blocks for a grid-stride pass over a list of n entries (256 threads), at most 8 per SM.
unsigned list_blocks(uint32_t n) { return (unsigned)std::max<uint32_t>(1u, std::min<uint32_t>((n + 255u) / 256u, 148u * 8u)); }

}  // namespace

cudaError_t launch_collider_setup(const SceneView& v, const CollideSet& cs, CollideWork& w, cudaStream_t st)
{
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    k_collider_sdf<<<node_blocks(nc), 256, 0, st>>>(cs, v.g.nx, v.g.ny, v.g.nz, v.origin[0], v.origin[1], v.origin[2],
                                                   v.h[0], v.h[1], v.h[2], w.csdf);
    count_launch();
    k_collider_cells<<<node_blocks(nc), 256, 0, st>>>(v, w.csdf, w.node_valid, w.cell_boundry);
    count_launch();
    k_collider_faces<<<face_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v, w.csdf, w.face_open,
                                                                                          w.face_cls);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_collider_face_lists(const SceneView& v, CollideWork& w, bool count_only, cudaStream_t st)
{
    cudaError_t e = cudaMemsetAsync(w.face_cnt, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_collider_face_lists<<<face_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(
        v, w.csdf, w.face_open, w.face_cls, w.face_cnt, w.blk_list, w.fin_list, w.fin_nrm, count_only ? 1 : 0);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_collider_project_rhs(const SceneView& v, const CollideWork& w, int* err, cudaStream_t st)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    k_ccl_init<<<node_blocks(nc), 256, 0, st>>>(v.marks, nc, w.label, w.open_comp, w.comp_sum, w.comp_cnt);
    count_launch();
    k_ccl_union<<<node_blocks(nc), 256, 0, st>>>(v.marks, nx, ny, nz, w.label, err);
    count_launch();
    k_ccl_classify<<<node_blocks(nc), 256, 0, st>>>(v.marks, nx, ny, nz, w.label, w.open_comp, err);
    count_launch();
    k_ccl_sums<<<node_blocks(nc), 256, 0, st>>>(v.marks, v.b, nc, w.label, w.open_comp, w.comp_sum, w.comp_cnt);
    count_launch();
    k_ccl_project<<<node_blocks(nc), 256, 0, st>>>(v.marks, nc, w.label, w.open_comp, w.comp_sum, w.comp_cnt, v.b);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_collider_bc(const SceneView& v, const CollideWork& w, float* const buf[3], cudaStream_t st)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nu = (size_t)(nx + 1) * ny * nz, nvv = (size_t)nx * (ny + 1) * nz;
    const size_t total = nu + nvv + (size_t)nx * ny * (nz + 1);
    if (w.n_blk > 0) {
        k_bc_block<<<list_blocks(w.n_blk), 256, 0, st>>>(buf[0], buf[1], buf[2], nu, nvv, w.blk_list, w.n_blk);
        count_launch();
    }
    if (v.extrap_depth > 0) {
        // copy into scratch 0, extrapolate from there back into buf (scratch 1 is the ping-pong partner)
        float* s0[3] = {w.ftmp0, w.ftmp0 + nu, w.ftmp0 + nu + nvv};
        float* s1[3] = {w.ftmp1, w.ftmp1 + nu, w.ftmp1 + nu + nvv};
        for (int c = 0; c < 3; ++c) {
            const size_t cnt = c == 0 ? nu : (c == 1 ? nvv : total - nu - nvv);
            cudaError_t e = cudaMemcpyAsync(s0[c], buf[c], cnt * sizeof(float), cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
        }
        const uint8_t* open[3] = {w.face_open, w.face_open + nu, w.face_open + nu + nvv};
        cudaError_t e = launch_extrap_faces(v, s0, buf, s1, open, w.vscratch, v.extrap_depth, st);
        if (e != cudaSuccess) return e;
    }
    if (w.n_fin > 0) {
        k_bc_friction<<<list_blocks(w.n_fin), 256, 0, st>>>(v, buf[0], buf[1], buf[2], w.fin_list, w.fin_nrm, w.n_fin,
                                                            w.fric);
        count_launch();
        k_bc_finish<<<list_blocks(w.n_fin), 256, 0, st>>>(buf[0], buf[1], buf[2], nu, nvv, w.fin_list, w.n_fin, w.fric);
        count_launch();
    }
    return cudaGetLastError();
}

cudaError_t launch_collider_marks(const SceneView& v, const CollideWork& w, unsigned long long* node_scratch,
                                  double** fluid_sdf, cudaStream_t st)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const size_t nc = (size_t)nx * ny * nz;
    cudaError_t e = launch_node_sdf(v, node_scratch, w.sdf_a, st);  // BuildSignedDistanceField
    if (e != cudaSuccess) return e;
    double* in = w.sdf_a;
    double* out = w.sdf_b;
    const uint8_t* vin = w.node_valid;
    for (int pass = 0; pass < v.extrap_depth; ++pass) {  // ExtrapolateIntoCollider
        uint8_t* vout = w.node_vscratch + (pass & 1) * nc;
        k_extrap_nodes<<<node_blocks(nc), 256, 0, st>>>(in, out, vin, vout, nx, ny, nz);
        count_launch();
        vin = vout;
        double* t = in;
        in = out;
        out = t;
    }
    *fluid_sdf = in;
    k_mark_collider<<<node_blocks(nc), 256, 0, st>>>(v, in, w.cell_boundry);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_collider_keep_start(const SceneView& v, const CollideWork& w, cudaStream_t st)
{
    if (v.np == 0) return cudaSuccess;
    k_keep_start<<<(unsigned)((v.np + 255) / 256), 256, 0, st>>>(v, w.start, w.startv);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_collider_resolve(const SceneView& v, const CollideSet& cs, const CollideWork& w,
                                    const CollideMove& g, cudaStream_t st)
{
    if (v.np == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(w.flag, 0, (v.np + 1) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const unsigned nb = (unsigned)((v.np + 255) / 256);
    k_collide_flags<<<nb, 256, 0, st>>>(v, w.csdf, cs.count, w.start, w.flag, w.spos, w.slot_of);
    count_launch();
    e = launch_exclusive_scan(w.flag, (uint32_t)(v.np + 1), w.offs, w.scan_tmp, w.scan_tmp_bytes, st);
    if (e != cudaSuccess) return e;
    k_collide_compact<<<node_blocks(v.np), 256, 0, st>>>(w.flag, w.offs, v.np, w.list);
    count_launch();
    k_collide_prep<<<148 * 8, 128, 0, st>>>(cs, w.list, w.offs + v.np, w.spos, w.cp, w.nrm, w.ins);
    count_launch();
    // entries that reflect (in order): flags over (count * colliders + 1) entries, scanned, compacted; the scan
    // length is the capacity bound because the count lives on the device
    const uint64_t cap_entries = v.np * (uint64_t)cs.count + 1;
    k_collide_active<<<node_blocks(cap_entries), 256, 0, st>>>(w.offs + v.np, cs.count, w.ins, w.act);
    count_launch();
    e = launch_exclusive_scan(w.act, (uint32_t)cap_entries, w.act_offs, w.act_tmp, w.act_tmp_bytes, st);
    if (e != cudaSuccess) return e;
    k_collide_active_compact<<<node_blocks(cap_entries), 256, 0, st>>>(w.offs + v.np, cs.count, w.act, w.act_offs,
                                                                      w.act_list);
    count_launch();
    k_collide_serial<<<1, 32, 0, st>>>(cs, v, g, w.csdf, w.start, w.startv, w.slot_of, w.offs + v.np, w.cp, w.nrm,
                                       w.act_offs + 0, w.act_list);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_add_gravity(const SceneView& v, float* const buf[3], double dt, cudaStream_t st)
{
    k_add_gravity<<<face_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(
        buf[0], buf[1], buf[2], v.g.nx, v.g.ny, v.g.nz, (float)(dt * v.gravity[0]), (float)(dt * v.gravity[1]),
        (float)(dt * v.gravity[2]));
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_surface_with_colliders(const double* fluid, const double* csdf, size_t n, double* out,
                                          cudaStream_t st)
{
    k_surface_with_colliders<<<node_blocks(n), 256, 0, st>>>(fluid, csdf, n, out);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
