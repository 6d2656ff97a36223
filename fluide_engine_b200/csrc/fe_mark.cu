// fe_mark.cu -- FLUID / AIR cell marking (K_mark), bit-exact with the reference.
//
// Reference: PICSimulator::BuildSignedDistanceField (pic_simulator.cpp:452-475) builds, at every
// cell-centred node c, sdf(c) = min(2r, min |p - c| over the particles its hash searcher visits) - r
// with r = 1.2 max(h) / sqrt(2); HashGridParticleSearcher::ForEachNearbyPoint
// (particle_systems/hash_grid_particle_searcher.cpp:97-126,154-204) visits the particles of 8 buckets of
// edge 2r (the node's bucket and, per axis, the neighbour on the side of the node's half) whose squared
// distance is <= (2r)^2.  SinglePhasePressureSolver::BuildMarkers (fluid_solvers/
// single_phase_pressure_solver.cpp:30-48) then marks a cell FLUID iff the trilinear sample of sdf at
// the cell centre is < 0.
//
// When the cell-centre sample lands exactly on node c (every power-of-two grid on an origin-0 domain,
// checked per axis on the host), the mark is FLUID iff some visited particle has |p - c| < r, because
// a - r < 0 <=> a < r in IEEE arithmetic.  K_mark therefore scatters from particles: each particle tests
// the few nodes within r of it with the reference's exact FP64 expressions (no fused multiply-add,
// correctly rounded sqrt, the same bucket membership) and stores FLUID.  On axes where the sample is off
// the node by a rounding error, the sign of the sample equals the sign of the node value unless the
// node value is within ~1e-15 r of zero; such "critical" cells are listed and re-evaluated with the full
// band SDF and the reference's trilinear sample by k_mark_fixup.  The result is byte-identical to the
// reference in every case.
#include <cmath>

#include "fe_internal.cuh"

namespace fe {
namespace {

__device__ __forceinline__ double dist2_ref(double px, double py, double pz, double cx, double cy, double cz)
{
    // (p - c).GetLengthSquared() = x*x + y*y + z*z, left to right, each operation rounded
    double dx = __dsub_rn(px, cx), dy = __dsub_rn(py, cy), dz = __dsub_rn(pz, cz);
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ int bucket_of(double x, double spacing)
{
    return (int)floor(__ddiv_rn(x, spacing));
}

// floor(x / spacing) exactly as the reference computes it; the multiply by the reciprocal decides it
// unless the quotient is within 1e-9 of an integer, where the correctly rounded division is used.
__device__ __forceinline__ int bucket_fast(double x, double spacing, double inv_spacing)
{
    const double q = x * inv_spacing;
    const double fq = floor(q);
    const double fr = q - fq;
    if (fr > 1e-9 && fr < 1.0 - 1e-9) return (int)fq;
    return bucket_of(x, spacing);
}

__device__ __forceinline__ bool visited(const SceneView& v, int pbx, int pby, int pbz, int i, int j, int k)
{
    return (pbx == v.q_b0[0][i] || pbx == v.q_b1[0][i]) && (pby == v.q_b0[1][j] || pby == v.q_b1[1][j]) &&
           (pbz == v.q_b0[2][k] || pbz == v.q_b1[2][k]);
}

// One thread per particle: the nodes within r of it (2 per axis for cubic cells, where 2r = 1.7 h;
// more along an axis whose spacing is finer than max(h)) get the reference's exact FP64 test.
// A node the particle is within band of: FLUID when within r; on grids with inexact cell-centre samples, a node
// whose distance is within crit_eps of r is listed for the full trilinear sample.
__device__ __forceinline__ void mark_node(const SceneView& v, const MarkConst& mc, double d2, int i, int j, int k)
{
    if (!(d2 <= mc.R2)) return;
    const size_t c = idx3(i, j, k, v.g.nx, v.g.ny);
    // sqrt(d2) < r exactly when d2 <= rin2 (correctly rounded sqrt is monotonic): no square root
    if (d2 <= mc.rin2) v.marks[c] = FE_CELL_FLUID;
    if (v.any_inexact && !(v.q_exact[0][i] && v.q_exact[1][j] && v.q_exact[2][k]) &&
        fabs(__dsqrt_rn(d2) - v.radius) <= mc.crit_eps) {
        unsigned* word = (unsigned*)(v.crit_flag + (c & ~(size_t)3));
        unsigned bit = 1u << (8 * (c & 3));
        if (!(atomicOr(word, bit) & bit)) {
            uint32_t slot = atomicAdd(v.crit_count, 1u);
            v.crit_list[slot] = (uint32_t)c;
        }
    }
}

// The common case, every axis' node window holding at most two nodes (cubic cells: 2r = 1.7 h): the 2 x 2 x 2
// candidates are tested without loops, every table load issued first and each node's test predicated, so the
// lanes of a warp stay converged.  Same nodes, same FP64 expressions and bucket tests as mark_body's loops.
__device__ __forceinline__ void mark_body2(const SceneView& v, const MarkConst& mc, uint32_t blk)
{
    const uint64_t p = blk * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    const double X[3] = {(double)v.px[p], (double)v.py[p], (double)v.pz[p]};
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    int node[3][2];
    bool ok[3][2];
    double q[3][2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double t = (X[a] - v.sdf_origin[a]) * v.inv_h[a];
        const double rr = v.radius * v.inv_h[a] + 1e-6;
        const int lo = max((int)floor(t - rr) + 1, 0);
        const int hi = min((int)floor(t + rr), n[a] - 1);
        const int pb = bucket_fast(X[a], v.bucket, mc.inv_bucket);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int idx = min(lo + s, n[a] - 1);  // clamped for the loads; out-of-window nodes are not ok
            node[a][s] = idx;
            ok[a][s] = lo + s <= hi && (pb == v.q_b0[a][idx] || pb == v.q_b1[a][idx]);
            q[a][s] = v.q_pos[a][idx];
        }
    }
#pragma unroll
    for (int sk = 0; sk < 2; ++sk)
#pragma unroll
        for (int sj = 0; sj < 2; ++sj)
#pragma unroll
            for (int si = 0; si < 2; ++si)
                if (ok[2][sk] && ok[1][sj] && ok[0][si])
                    mark_node(v, mc, dist2_ref(X[0], X[1], X[2], q[0][si], q[1][sj], q[2][sk]), node[0][si],
                              node[1][sj], node[2][sk]);
}

__device__ __forceinline__ void mark_body(const SceneView& v, const MarkConst& mc, uint32_t blk)
{
    uint64_t p = blk * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    const double X[3] = {(double)v.px[p], (double)v.py[p], (double)v.pz[p]};
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    const double inv_bucket = mc.inv_bucket;
    int lo[3], hi[3], pb[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // nodes i with |q_i - x| < r, widened by 1e-6 h (the exact test below decides)
        const double t = (X[a] - v.sdf_origin[a]) * v.inv_h[a];
        const double rr = v.radius * v.inv_h[a] + 1e-6;
        lo[a] = max((int)floor(t - rr) + 1, 0);
        hi[a] = min((int)floor(t + rr), n[a] - 1);
        pb[a] = bucket_fast(X[a], v.bucket, inv_bucket);
    }
    for (int k = lo[2]; k <= hi[2]; ++k) {
        if (pb[2] != v.q_b0[2][k] && pb[2] != v.q_b1[2][k]) continue;
        for (int j = lo[1]; j <= hi[1]; ++j) {
            if (pb[1] != v.q_b0[1][j] && pb[1] != v.q_b1[1][j]) continue;
            for (int i = lo[0]; i <= hi[0]; ++i) {
                if (pb[0] != v.q_b0[0][i] && pb[0] != v.q_b1[0][i]) continue;
                mark_node(v, mc, dist2_ref(X[0], X[1], X[2], v.q_pos[0][i], v.q_pos[1][j], v.q_pos[2][k]), i, j, k);
            }
        }
    }
}

__global__ void __launch_bounds__(256) k_mark(SceneView v, MarkConst mc)
{
    if (mc.two) mark_body2(v, mc, blockIdx.x);
    else mark_body(v, mc, blockIdx.x);
}

// Band-limited SDF value of node (i, j, k) exactly as BuildSignedDistanceField computes it.
__device__ double node_sdf(const SceneView& v, int i, int j, int k, double R2)
{
    const double q[3] = {v.q_pos[0][i], v.q_pos[1][j], v.q_pos[2][k]};
    double minDistance = v.band;
    const int c0[3] = {i, j, k};
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    int lo[3], hi[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // particles within the band 2r of the node lie in cells within ceil(2r/h + 0.5) of it
        const int reach = (int)ceil(v.band * v.inv_h[a] + 0.5) + 1;
        lo[a] = max(c0[a] - reach, 0);
        hi[a] = min(c0[a] + reach, n[a] - 1);
    }
    for (int cz = lo[2]; cz <= hi[2]; ++cz)
        for (int cy = lo[1]; cy <= hi[1]; ++cy)
            for (int cx = lo[0]; cx <= hi[0]; ++cx) {
                const uint32_t key = fe_cell_key(cx, cy, cz, n[0], n[1]);
                for (uint32_t p = v.cell_start[key]; p < v.cell_start[key + 1]; ++p) {
                    const double X = v.px[p], Y = v.py[p], Z = v.pz[p];
                    if (!visited(v, bucket_of(X, v.bucket), bucket_of(Y, v.bucket), bucket_of(Z, v.bucket), i, j, k))
                        continue;
                    const double d2 = dist2_ref(X, Y, Z, q[0], q[1], q[2]);
                    if (!(d2 <= R2)) continue;
                    const double dist = __dsqrt_rn(d2);
                    if (dist < minDistance) minDistance = dist;
                }
            }
    return __dsub_rn(minDistance, v.radius);
}

__device__ __forceinline__ double lerp_ref(double a, double b, double f)
{
    return __dadd_rn(__dmul_rn(__dsub_rn(1.0, f), a), __dmul_rn(f, b));
}

// ScalarGrid3D::Sample at the cell centre (3d/scalar_grid3d.cpp:33-65) with exact band SDF values.
__device__ double sample_cell_sdf(const SceneView& v, int i, int j, int k, double R2)
{
    const int i0 = v.q_i0[0][i], j0 = v.q_i0[1][j], k0 = v.q_i0[2][k];
    const double fx = v.q_f[0][i], fy = v.q_f[1][j], fz = v.q_f[2][k];
    const int ip = min(i0 + 1, v.g.nx - 1), jp = min(j0 + 1, v.g.ny - 1), kp = min(k0 + 1, v.g.nz - 1);
    const double c000 = node_sdf(v, i0, j0, k0, R2), c100 = node_sdf(v, ip, j0, k0, R2);
    const double c010 = node_sdf(v, i0, jp, k0, R2), c110 = node_sdf(v, ip, jp, k0, R2);
    const double c001 = node_sdf(v, i0, j0, kp, R2), c101 = node_sdf(v, ip, j0, kp, R2);
    const double c011 = node_sdf(v, i0, jp, kp, R2), c111 = node_sdf(v, ip, jp, kp, R2);
    const double b0 = lerp_ref(lerp_ref(c000, c100, fx), lerp_ref(c010, c110, fx), fy);
    const double b1 = lerp_ref(lerp_ref(c001, c101, fx), lerp_ref(c011, c111, fx), fy);
    return lerp_ref(b0, b1, fz);
}

__device__ __forceinline__ void mark_fixup_body(const SceneView& v, double R2, uint32_t cap, uint32_t blk, uint32_t nblk)
{
    const uint32_t count = min(*v.crit_count, cap);
    for (uint32_t t = blk * blockDim.x + threadIdx.x; t < count; t += nblk * blockDim.x) {
        const uint32_t c = v.crit_list[t];
        const int i = c % v.g.nx, j = (c / v.g.nx) % v.g.ny, k = c / (v.g.nx * v.g.ny);
        v.marks[c] = sample_cell_sdf(v, i, j, k, R2) < 0.0 ? FE_CELL_FLUID : FE_CELL_AIR;
    }
}

__global__ void k_mark_fixup(SceneView v, double R2, uint32_t cap) { mark_fixup_body(v, R2, cap, blockIdx.x, gridDim.x); }

// ---- flat multi-scene forms (BatchPlan, fe_internal.cuh); marks, crit flags and counts are cleared by
// launch_multi_clear
__global__ void __launch_bounds__(256) k_multi_mark(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkPart, b);
    const BatchScene& e = plan->sc[s];
    if (e.mark.two) mark_body2(e.dst, e.mark, b);
    else mark_body(e.dst, e.mark, b);
}

__global__ void __launch_bounds__(128) k_multi_mark_fixup(const BatchPlan* __restrict__ plan)
{
    __shared__ SceneView v;
    uint32_t b;
    const int s = batch_scene_of(plan, kBkFixup, b);
    const BatchScene& e = plan->sc[s];
    stage_view(v, e.dst);
    mark_fixup_body(v, e.mark.R2, (uint32_t)((size_t)v.g.nx * v.g.ny * v.g.nz), b,
                    plan->start[kBkFixup][s + 1] - plan->start[kBkFixup][s]);
}

__global__ void k_fluid_sdf(SceneView v, double R2, double* out)
{
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
        const int i = c % v.g.nx, j = (c / v.g.nx) % v.g.ny, k = c / ((size_t)v.g.nx * v.g.ny);
        out[c] = v.np ? node_sdf(v, i, j, k, R2) : __dsub_rn(v.band, v.radius);
    }
}


// One thread per particle: every SDF node within the band 2r of the particle that the reference's hash search
// would visit from that node and whose squared distance is <= (2r)^2 takes the minimum of that squared distance.
// The node's reference value is min(2r, min over those particles of |p - c|) - r; correctly rounded sqrt is
// monotonic, so min |p - c| = sqrt(min |p - c|^2) exactly, and the square root is taken once per node when the
// markers are sampled.  Squared distances are non-negative doubles, whose bit patterns order like their values,
// so a 64-bit atomicMin on the bits takes the minimum.  Each squared distance is summed in the reference's order,
// (dx^2 + dy^2) + dz^2; a row whose dy^2 + dz^2 already exceeds (2r)^2 is skipped (rounding is monotonic, so the
// full sum would exceed it too), and the bucket test runs once per axis.  Particles sorted by cell hit the same
// nodes as their neighbours; a plain read of the current minimum first (it only decreases, so a stale value is
// still an upper bound) skips most atomics.
__global__ void __launch_bounds__(256) k_sdf_scatter(SceneView v, unsigned long long* __restrict__ node, double R2)
{
    uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    const double X[3] = {(double)v.px[p], (double)v.py[p], (double)v.pz[p]};
    const int n[3] = {v.g.nx, v.g.ny, v.g.nz};
    const double inv_bucket = 1.0 / v.bucket;
    int lo[3], hi[3];
    unsigned long long pass[3];  // bit u: candidate node lo + u is in a bucket the node's search visits
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        // nodes i with |q_i - x| <= 2r, widened by 1e-6 h (the exact test below decides)
        const double t = (X[a] - v.sdf_origin[a]) * v.inv_h[a];
        const double rr = v.band * v.inv_h[a] + 1e-6;
        lo[a] = max((int)floor(t - rr) + 1, 0);
        hi[a] = min(min((int)floor(t + rr), n[a] - 1), lo[a] + 63);  // 2r spans at most 64 nodes per axis
        const int pb = bucket_fast(X[a], v.bucket, inv_bucket);
        pass[a] = 0ull;
        for (int i = lo[a]; i <= hi[a]; ++i)
            if (pb == v.q_b0[a][i] || pb == v.q_b1[a][i]) pass[a] |= 1ull << (i - lo[a]);
    }
    const double* qx = v.q_pos[0];
    for (int k = lo[2]; k <= hi[2]; ++k) {
        if (!((pass[2] >> (k - lo[2])) & 1ull)) continue;
        const double dz = __dsub_rn(X[2], v.q_pos[2][k]);
        const double dz2 = __dmul_rn(dz, dz);
        if (!(dz2 <= R2)) continue;
        for (int j = lo[1]; j <= hi[1]; ++j) {
            if (!((pass[1] >> (j - lo[1])) & 1ull)) continue;
            const double dy = __dsub_rn(X[1], v.q_pos[1][j]);
            const double dy2 = __dmul_rn(dy, dy);
            if (!(__dadd_rn(dy2, dz2) <= R2)) continue;
            for (int i = lo[0]; i <= hi[0]; ++i) {
                if (!((pass[0] >> (i - lo[0])) & 1ull)) continue;
                const double dx = __dsub_rn(X[0], qx[i]);
                const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), dy2), dz2);  // dist2_ref's order
                if (!(d2 <= R2)) continue;
                const unsigned long long bits = (unsigned long long)__double_as_longlong(d2);
                unsigned long long* cell = node + idx3(i, j, k, n[0], n[1]);
                if (bits < __ldcg(cell)) atomicMin(cell, bits);
            }
        }
    }
}

// Node values of BuildSignedDistanceField (pic_simulator.cpp:452-475): min(2r, sqrt(smallest squared distance)) - r.
__device__ __forceinline__ double node_value(unsigned long long raw, double band, double radius)
{
    double m = band;
    if (raw != ~0ull) {
        const double dm = __dsqrt_rn(__longlong_as_double((long long)raw));
        if (dm < m) m = dm;
    }
    return __dsub_rn(m, radius);
}

__global__ void k_node_values(const unsigned long long* __restrict__ node, size_t nc, double band, double radius,
                              double* __restrict__ sdf)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x)
        sdf[c] = node_value(node[c], band, radius);
}

// BackwardEulerDiffusionSolver::BuildX/Y/ZMarkers (fluid_solvers/backward_euler_diffusion_solver.cpp:71-128):
// a face is FLUID iff ScalarGrid3D::Sample (3d/scalar_grid3d.cpp:33-65) of the fluid SDF at the face centre is
// < 0.  The face centres are those of the copied velocity grid (data origins include the domain origin,
// grid_systems/face_centered_grid3d.cpp:11-17,303-316); their GetBarycentric index and fraction per axis come
// from host tables computed in FP64 with the reference's expressions.
__global__ void k_face_mark(SceneView v, DiffWork d)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    const int base = fc.c * 3 * d.tab_stride;
    const int i0 = d.tab_i0[base + fc.i], j0 = d.tab_i0[base + d.tab_stride + fc.j];
    const int k0 = d.tab_i0[base + 2 * d.tab_stride + fc.k];
    const double fx = d.tab_f[base + fc.i], fy = d.tab_f[base + d.tab_stride + fc.j];
    const double fz = d.tab_f[base + 2 * d.tab_stride + fc.k];
    const int ip = min(i0 + 1, nx - 1), jp = min(j0 + 1, ny - 1), kp = min(k0 + 1, nz - 1);
    const unsigned long long* __restrict__ node = d.node_dist;
    // node value min(2r, sqrt(smallest squared distance)) - r (all ones: no particle within the band)
    auto val = [&](int i, int j, int k) { return node_value(__ldg(node + idx3(i, j, k, nx, ny)), v.band, v.radius); };
    const double c000 = val(i0, j0, k0), c100 = val(ip, j0, k0), c010 = val(i0, jp, k0), c110 = val(ip, jp, k0);
    const double c001 = val(i0, j0, kp), c101 = val(ip, j0, kp), c011 = val(i0, jp, kp), c111 = val(ip, jp, kp);
    const double b0 = lerp_ref(lerp_ref(c000, c100, fx), lerp_ref(c010, c110, fx), fy);
    const double b1 = lerp_ref(lerp_ref(c001, c101, fx), lerp_ref(c011, c111, fx), fy);
    const size_t off = fc.c == 0 ? 0 : (fc.c == 1 ? (size_t)(nx + 1) * ny * nz
                                                   : (size_t)(nx + 1) * ny * nz + (size_t)nx * (ny + 1) * nz);
    d.mark[off + fc.f] = lerp_ref(b0, b1, fz) < 0.0 ? FE_CELL_FLUID : FE_CELL_AIR;
}
}  // namespace

// Largest double d with sqrt(d) < r (sqrt correctly rounded, as IEEE 754 requires of the host's and the device's
// square root): the marking test sqrt(d2) < r becomes d2 <= sqrt_below(r), with the same outcome for every d2.
static double sqrt_below(double r)
{
    double t = r * r;
    while (t > 0.0 && std::sqrt(t) >= r) t = std::nextafter(t, 0.0);
    while (std::sqrt(std::nextafter(t, HUGE_VAL)) < r) t = std::nextafter(t, HUGE_VAL);
    return t;
}

cudaError_t launch_multi_mark(const BatchLaunch& L, cudaStream_t st)
{
    if (L.total[kBkPart]) {
        k_multi_mark<<<L.total[kBkPart], 256, 0, st>>>(L.plan);
        count_launch();
    }
    if (L.total[kBkFixup]) {
        k_multi_mark_fixup<<<L.total[kBkFixup], 128, 0, st>>>(L.plan);
        count_launch();
    }
    return cudaGetLastError();
}

// The marking constants of launch_mark: band^2, the largest squared distance whose square root is below r, and the
// window around r in which an inexact cell-centre sample is recomputed.
MarkConst mark_constants(const SceneView& v)
{
    MarkConst mc;
    mc.R2 = v.band * v.band;
    mc.rin2 = sqrt_below(v.radius);
    mc.crit_eps = 1e-9 * v.radius;
    mc.inv_bucket = 1.0 / v.bucket;
    mc.two = 1;
    for (int a = 0; a < 3; ++a)  // window (t - rr, t + rr] with rr = r / h_a + 1e-6 holds at most ceil(2 rr) nodes
        if (!(v.radius * v.inv_h[a] + 1e-6 < 1.0 - 1e-9)) mc.two = 0;
    return mc;
}

cudaError_t launch_mark(const SceneView& v, cudaStream_t st)
{
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    cudaError_t e = cudaMemsetAsync(v.marks, FE_CELL_AIR, nc, st);
    if (e != cudaSuccess) return e;
    const MarkConst mc = mark_constants(v);
    if (v.any_inexact) {
        if ((e = cudaMemsetAsync(v.crit_flag, 0, (nc + 3) & ~(size_t)3, st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(v.crit_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return e;
    }
    if (v.np > 0) {
        k_mark<<<(unsigned)((v.np + 255) / 256), 256, 0, st>>>(v, mc);
        count_launch();
        if (v.any_inexact) {
            k_mark_fixup<<<148, 128, 0, st>>>(v, mc.R2, (uint32_t)nc);
            count_launch();
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_fluid_sdf(const SceneView& v, double* out, cudaStream_t st)
{
    k_fluid_sdf<<<148 * 8, 128, 0, st>>>(v, v.band * v.band, out);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_node_sdf(const SceneView& v, unsigned long long* node, double* sdf, cudaStream_t st)
{
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    cudaError_t e = cudaMemsetAsync(node, 0xff, nc * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (v.np > 0) {
        k_sdf_scatter<<<(unsigned)((v.np + 255) / 256), 256, 0, st>>>(v, node, v.band * v.band);
        count_launch();
    }
    k_node_values<<<(unsigned)((nc + 255) / 256), 256, 0, st>>>(node, nc, v.band, v.radius, sdf);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_face_fluid_marks(const SceneView& v, const DiffWork& d, cudaStream_t st)
{
    const size_t nc = (size_t)v.g.nx * v.g.ny * v.g.nz;
    cudaError_t e = cudaMemsetAsync(d.node_dist, 0xff, nc * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    if (v.np > 0) {
        k_sdf_scatter<<<(unsigned)((v.np + 255) / 256), 256, 0, st>>>(v, d.node_dist, v.band * v.band);
        count_launch();
    }
    k_face_mark<<<face_grid(v.g.nx, v.g.ny, v.g.nz), dim3(kTileX, kTileY), 0, st>>>(v, d);
    count_launch();
    return cudaGetLastError();
}


}  // namespace fe
