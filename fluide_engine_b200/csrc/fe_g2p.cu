// fe_g2p.cu -- grid -> particle transfer fused with advection (K_g2p_adv).
//
// Reference: TransferGrid2Particles of PICSimulator (pic_simulator.cpp:439-450: v = Sample(grid, x)),
// FLIPSimulator (flip_simulator.cpp:121-161: v = Lerp(v + Sample(grid - snapshot, x), Sample(grid, x),
// blend)) and APICSimulator (apic_simulator.cpp:120-176: v = Sample(grid, x), C rows = sum of gradient
// weights (common/math_utils.hpp:114-176) times face values at the position clamped by h/2 on the
// transverse axes, with the CELL count as clamp size); then PICSimulator::MoveParticles
// (pic_simulator.cpp:239-312): max(maxCfl, 1) RK2 midpoint sub-steps on the GRID velocity, clamp to the
// domain box with the clamped component of the particle velocity set to 0.
//
// One thread per particle over the sorted arrays: the particle state is read once and written once
// (FP32), the grid gathers hit L1/L2 because neighbouring threads hold neighbouring particles.
#include "fe_internal.cuh"

namespace fe {
namespace {

// Face values of the six arrays a transfer reads (u, v, w and the FLIP snapshot su, sv, sw).
struct FaceSource {
    const float* g[6];          // u, v, w, su, sv, sw
    int sx[3], sy[3];           // face-array sizes of the components (x, y)
    // Offset of corner (i, j, k) of component comp's stencil and the steps to its other corners (0 where the stencil
    // is clamped onto one face): one 64-bit index, then 32-bit steps (a step spans at most one plane of faces).
    __device__ __forceinline__ size_t corner_base(int comp, const Stencil& st, int& dx, int& dy, int& dz) const
    {
        dx = st.ip - st.i;
        dy = (st.jp - st.j) * sx[comp];
        dz = (st.kp - st.k) * sx[comp] * sy[comp];
        return idx3(st.i, st.j, st.k, sx[comp], sy[comp]);
    }
    // the 8 corner values of array a from its base, in the reference's corner order (x fastest)
    __device__ __forceinline__ void load8(int a, size_t base, int dx, int dy, int dz, float c[8]) const
    {
        const float* p = g[a] + base;
        c[0] = __ldg(p);
        c[1] = __ldg(p + dx);
        c[2] = __ldg(p + dy);
        c[3] = __ldg(p + dx + dy);
        c[4] = __ldg(p + dz);
        c[5] = __ldg(p + dx + dz);
        c[6] = __ldg(p + dy + dz);
        c[7] = __ldg(p + dx + dy + dz);
    }
    __device__ __forceinline__ void corners(int a, const Stencil& st, float c[8]) const
    {
        int dx, dy, dz;
        const size_t base = corner_base(a % 3, st, dx, dy, dz);
        load8(a, base, dx, dy, dz, c);
    }
};

__device__ __forceinline__ float lerp8(const float c[8], const Stencil& s)
{
    const float b0 = lerpf_ref(lerpf_ref(c[0], c[1], s.fx), lerpf_ref(c[2], c[3], s.fx), s.fy);
    const float b1 = lerpf_ref(lerpf_ref(c[4], c[5], s.fx), lerpf_ref(c[6], c[7], s.fx), s.fy);
    return lerpf_ref(b0, b1, s.fz);
}

// GetBarycentric index pair and fraction of a point along one axis of one staggered grid (stencil() per axis).
struct AxisFrac {
    int i, ip;
    float f;
};
__device__ __forceinline__ AxisFrac axis_frac(float x, float o, float ih, int size)
{
    AxisFrac a;
    bary((x - o) * ih, size - 1, a.i, a.f);
    a.ip = min(a.i + 1, size - 1);
    return a;
}
__device__ __forceinline__ Stencil stencil_of(const AxisFrac& a, const AxisFrac& b, const AxisFrac& c)
{
    Stencil s;
    s.i = a.i; s.ip = a.ip; s.fx = a.f;
    s.j = b.i; s.jp = b.ip; s.fy = b.f;
    s.k = c.i; s.kp = c.ip; s.fz = c.f;
    return s;
}

// The three staggered grids' stencils at one point, as stencil() gives them.  Along each axis the two grids that are
// not staggered along it have the same data origin (both offset by half a cell, set side by side with the scene:
// xo[1] == zo[1], yo[0] == zo[0], xo[2] == yo[2], and likewise for the FLIP residual origins) and the same size, so
// their index and fraction are one computation: 6 per point instead of 9.
__device__ __forceinline__ void stencils3(float x, float y, float z, const float ou[3], const float ov[3],
                                          const float ow[3], const float ih[3], int nx, int ny, int nz, Stencil& su,
                                          Stencil& sv, Stencil& sw)
{
    const AxisFrac xf = axis_frac(x, ou[0], ih[0], nx + 1), xc = axis_frac(x, ov[0], ih[0], nx);
    const AxisFrac yf = axis_frac(y, ov[1], ih[1], ny + 1), yc = axis_frac(y, ou[1], ih[1], ny);
    const AxisFrac zf = axis_frac(z, ow[2], ih[2], nz + 1), zc = axis_frac(z, ou[2], ih[2], nz);
    su = stencil_of(xf, yc, zc);
    sv = stencil_of(xc, yf, zc);
    sw = stencil_of(xc, yc, zf);
}

// The grid velocity at a point: the three components' trilinear samples, each stencil built just before its loads
// (the shared fractions of stencils3 carried from one component to the next).
__device__ __forceinline__ void sample_vel(const SceneView& v, const FaceSource& fs, float x, float y, float z,
                                           float out[3])
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const float* ih = v.inv_hf;
    float c[8];
    const AxisFrac xf = axis_frac(x, v.xo[0], ih[0], nx + 1);
    const AxisFrac yc = axis_frac(y, v.xo[1], ih[1], ny);
    const AxisFrac zc = axis_frac(z, v.xo[2], ih[2], nz);
    const Stencil su = stencil_of(xf, yc, zc);
    fs.corners(0, su, c);
    out[0] = lerp8(c, su);
    const AxisFrac xc = axis_frac(x, v.yo[0], ih[0], nx);
    const AxisFrac yf = axis_frac(y, v.yo[1], ih[1], ny + 1);
    const Stencil sv = stencil_of(xc, yf, zc);
    fs.corners(1, sv, c);
    out[1] = lerp8(c, sv);
    const AxisFrac zf = axis_frac(z, v.zo[2], ih[2], nz + 1);
    const Stencil sw = stencil_of(xc, yc, zf);
    fs.corners(2, sw, c);
    out[2] = lerp8(c, sw);
}

// Trilinear sample of (grid - snapshot) with the reference's Lerp tree (the FLIP residual grid,
// flip_simulator.cpp:138-150), and, when `plain` is non-null, the grid's own sample at the same stencil from the
// same face values.
__device__ __forceinline__ float sample_diff(const FaceSource& fs, int comp, const Stencil& s, float* plain)
{
    float a[8], b[8], d[8];
    int dx, dy, dz;
    const size_t base = fs.corner_base(comp, s, dx, dy, dz);  // the grid and its snapshot share the layout
    fs.load8(comp, base, dx, dy, dz, a);
    fs.load8(comp + 3, base, dx, dy, dz, b);
#pragma unroll
    for (int t = 0; t < 8; ++t) d[t] = a[t] - b[t];
    if (plain) *plain = lerp8(a, s);
    return lerp8(d, s);
}

// sum_t gradweight_t * face_t for one velocity component (apic_simulator.cpp:311-336), from the stencil's 8 corner
// values.
__device__ __forceinline__ void apic_row_vals(const float val[8], const Stencil& s, const float ih[3], float out[3])
{
    const float fx = s.fx, fy = s.fy, fz = s.fz;
    const float gx[8] = {-ih[0] * (1 - fy) * (1 - fz), ih[0] * (1 - fy) * (1 - fz), (-ih[0]) * fy * (1 - fz),
                         ih[0] * fy * (1 - fz),        (-ih[0]) * (1 - fy) * fz,   ih[0] * (1 - fy) * fz,
                         (-ih[0]) * fy * fz,           ih[0] * fy * fz};
    const float gy[8] = {-ih[1] * (1 - fx) * (1 - fz), fx * (-ih[1]) * (1 - fz), (1 - fx) * ih[1] * (1 - fz),
                         fx * ih[1] * (1 - fz),        (1 - fx) * (-ih[1]) * fz, fx * (-ih[1]) * fz,
                         (1 - fx) * ih[1] * fz,        fx * ih[1] * fz};
    const float gz[8] = {-ih[2] * (1 - fx) * (1 - fy), fx * (1 - fy) * (-ih[2]), (1 - fx) * fy * (-ih[2]),
                         fx * fy * (-ih[2]),           (1 - fx) * (1 - fy) * ih[2], fx * (1 - fy) * ih[2],
                         (1 - fx) * fy * ih[2],        fx * fy * ih[2]};
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        r0 += gx[t] * val[t];
        r1 += gy[t] * val[t];
        r2 += gz[t] * val[t];
    }
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
}

__device__ __forceinline__ void apic_row(const FaceSource& fs, int comp, const Stencil& s, const float ih[3],
                                         float out[3])
{
    float val[8];
    fs.corners(comp, s, val);
    apic_row_vals(val, s, ih, out);
}

// APIC: component c's grid sample at the particle (stencil s, the velocity grid's face counts as sizes) and its C row.
// The row's stencil is taken at the particle clamped by h/2 on the two transverse axes with the CELL counts as sizes;
// where no clamp moves the particle and its index along the component's own axis is below n - 1 (the two sizes then
// give the same GetBarycentric result), it is s itself, and the row reuses the sample's 8 corner values.
__device__ __forceinline__ float apic_component(const SceneView& v, const FaceSource& fs, int c, const Stencil& s,
                                                const float P[3], const float lo[3], const float hi[3], uint64_t p)
{
    float c8[8];
    fs.corners(c, s, c8);
    const float pic = lerp8(c8, s);
    float q[3] = {P[0], P[1], P[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a)
        if (a != c) q[a] = q[a] < lo[a] ? lo[a] : (q[a] > hi[a] ? hi[a] : q[a]);
    const int n_c = c == 0 ? v.g.nx : (c == 1 ? v.g.ny : v.g.nz);
    const int i_c = c == 0 ? s.i : (c == 1 ? s.j : s.k);
    float row[3];
    if (q[0] == P[0] && q[1] == P[1] && q[2] == P[2] && i_c <= n_c - 2) {
        apic_row_vals(c8, s, v.inv_hf, row);
    } else {
        const float* org = c == 0 ? v.xo : (c == 1 ? v.yo : v.zo);
        apic_row(fs, c, stencil(q[0], q[1], q[2], org, v.inv_hf, v.g.nx, v.g.ny, v.g.nz), v.inv_hf, row);
    }
    v.c[3 * c][p] = row[0];
    v.c[3 * c + 1][p] = row[1];
    v.c[3 * c + 2][p] = row[2];
    return pic;
}

// APIC's transfer at the particle: the grid velocity (as sample_vel) and the three C rows.
__device__ __forceinline__ void sample_vel_apic(const SceneView& v, const FaceSource& fs, float x, float y, float z,
                                                uint64_t p, float out[3])
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const float* ih = v.inv_hf;
    const float lo[3] = {v.originf[0] + 0.5f * v.hf[0], v.originf[1] + 0.5f * v.hf[1], v.originf[2] + 0.5f * v.hf[2]};
    const float hi[3] = {v.originf[0] + v.sizef[0] - 0.5f * v.hf[0], v.originf[1] + v.sizef[1] - 0.5f * v.hf[1],
                         v.originf[2] + v.sizef[2] - 0.5f * v.hf[2]};
    const float P[3] = {x, y, z};
    const AxisFrac xf = axis_frac(x, v.xo[0], ih[0], nx + 1);
    const AxisFrac yc = axis_frac(y, v.xo[1], ih[1], ny);
    const AxisFrac zc = axis_frac(z, v.xo[2], ih[2], nz);
    out[0] = apic_component(v, fs, 0, stencil_of(xf, yc, zc), P, lo, hi, p);
    const AxisFrac xc = axis_frac(x, v.yo[0], ih[0], nx);
    const AxisFrac yf = axis_frac(y, v.yo[1], ih[1], ny + 1);
    out[1] = apic_component(v, fs, 1, stencil_of(xc, yf, zc), P, lo, hi, p);
    const AxisFrac zf = axis_frac(z, v.zo[2], ih[2], nz + 1);
    out[2] = apic_component(v, fs, 2, stencil_of(xc, yc, zf), P, lo, hi, p);
}

// The transfer and move of particle p (pic_simulator.cpp:239-312, flip_simulator.cpp:121-161,
// apic_simulator.cpp:120-176), reading face values through fs.
template <int SOLVER, bool G2P, bool MOVE>
__device__ __forceinline__ void g2p_particle(const SceneView& v, const G2PArgs& g, const FaceSource& fs, uint64_t p)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const float x = v.px[p], y = v.py[p], z = v.pz[p];
    float vel[3];
    float pic[3];
    bool have_pic = false;
    if (G2P) {
        if (SOLVER == FE_SOLVER_FLIP) {
            Stencil su, sv, sw;
            stencils3(x, y, z, v.rxo, v.ryo, v.rzo, v.inv_hf, nx, ny, nz, su, sv, sw);
            const bool share = g.same_origins && v.blend > 0.f;
            float flip[3] = {v.vx[p] + sample_diff(fs, 0, su, share ? &pic[0] : nullptr),
                             v.vy[p] + sample_diff(fs, 1, sv, share ? &pic[1] : nullptr),
                             v.vz[p] + sample_diff(fs, 2, sw, share ? &pic[2] : nullptr)};
            if (v.blend > 0.f) {
                if (!share) sample_vel(v, fs, x, y, z, pic);
                have_pic = true;
#pragma unroll
                for (int a = 0; a < 3; ++a) flip[a] = (1.f - v.blend) * flip[a] + v.blend * pic[a];
            }
            vel[0] = flip[0];
            vel[1] = flip[1];
            vel[2] = flip[2];
        } else {
            if (SOLVER == FE_SOLVER_APIC) sample_vel_apic(v, fs, x, y, z, p, pic);
            else sample_vel(v, fs, x, y, z, pic);
            have_pic = true;
            vel[0] = pic[0];
            vel[1] = pic[1];
            vel[2] = pic[2];
        }
    } else {
        vel[0] = v.vx[p];
        vel[1] = v.vy[p];
        vel[2] = v.vz[p];
    }
    if (MOVE) {
        float pt0[3] = {x, y, z}, pt1[3] = {x, y, z};
        const float half = 0.5f * g.dt_sub;
        for (int t = 0; t < g.nsub; ++t) {
            float v0[3], vm[3];
            if (t == 0 && have_pic) {
                v0[0] = pic[0]; v0[1] = pic[1]; v0[2] = pic[2];
            } else {
                sample_vel(v, fs, pt0[0], pt0[1], pt0[2], v0);
            }
            const float mid[3] = {pt0[0] + half * v0[0], pt0[1] + half * v0[1], pt0[2] + half * v0[2]};
            sample_vel(v, fs, mid[0], mid[1], mid[2], vm);
#pragma unroll
            for (int a = 0; a < 3; ++a) pt1[a] = pt0[a] + g.dt_sub * vm[a];
#pragma unroll
            for (int a = 0; a < 3; ++a) pt0[a] = pt1[a];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (pt1[a] <= g.dom_lo[a]) { pt1[a] = g.dom_lo[a]; vel[a] = 0.f; }
            if (pt1[a] >= g.dom_hi[a]) { pt1[a] = g.dom_hi[a]; vel[a] = 0.f; }
            // a NaN position (diverged input) is pinned to the lower wall so keys stay in range
            if (!(pt1[a] == pt1[a])) { pt1[a] = g.dom_lo[a]; vel[a] = 0.f; }
        }
        v.px[p] = pt1[0];
        v.py[p] = pt1[1];
        v.pz[p] = pt1[2];
    }
    v.vx[p] = vel[0];
    v.vy[p] = vel[1];
    v.vz[p] = vel[2];
}

__device__ __forceinline__ FaceSource global_source(const SceneView& v, const G2PArgs& g)
{
    FaceSource fs;
    fs.g[0] = g.u; fs.g[1] = g.v; fs.g[2] = g.w;
    fs.g[3] = v.su; fs.g[4] = v.sv; fs.g[5] = v.sw;
    fs.sx[0] = v.g.nx + 1; fs.sx[1] = v.g.nx; fs.sx[2] = v.g.nx;
    fs.sy[0] = v.g.ny; fs.sy[1] = v.g.ny + 1; fs.sy[2] = v.g.ny;
    return fs;
}

// One thread per particle over the sorted arrays: neighbouring threads hold neighbouring particles, so the face
// gathers hit L1/L2.  (A variant staging each tile's faces in shared memory, 13^3 per array, measured slower:
// 260 us against 183 us per launch at 128^3 FLIP.)
template <int SOLVER, bool G2P, bool MOVE>
__global__ void __launch_bounds__(256, 4) k_g2p(SceneView v, G2PArgs g)
{
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    g2p_particle<SOLVER, G2P, MOVE>(v, g, global_source(v, g), p);
}

// Flat multi-scene form (BatchPlan, fe_internal.cuh): every scene's particles in one launch, transfer and move
// fused, each block running its scene's transfer kind.
__global__ void __launch_bounds__(256, 4) k_multi_g2p(const BatchPlan* __restrict__ plan)
{
    __shared__ SceneView v;
    uint32_t b;
    const int s = batch_scene_of(plan, kBkPart, b);
    const BatchScene& e = plan->sc[s];
    stage_view(v, e.dst);
    const uint64_t p = b * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    if (v.solver == FE_SOLVER_PIC) g2p_particle<FE_SOLVER_PIC, true, true>(v, e.g2p, global_source(v, e.g2p), p);
    else if (v.solver == FE_SOLVER_FLIP) g2p_particle<FE_SOLVER_FLIP, true, true>(v, e.g2p, global_source(v, e.g2p), p);
    else g2p_particle<FE_SOLVER_APIC, true, true>(v, e.g2p, global_source(v, e.g2p), p);
}

template <int SOLVER>
void launch_solver(const SceneView& v, const G2PArgs& g, bool do_g2p, bool do_move, cudaStream_t st)
{
    const unsigned nb = (unsigned)((v.np + 255) / 256);
    if (do_g2p && do_move) k_g2p<SOLVER, true, true><<<nb, 256, 0, st>>>(v, g);
    else if (do_g2p) k_g2p<SOLVER, true, false><<<nb, 256, 0, st>>>(v, g);
    else k_g2p<SOLVER, false, true><<<nb, 256, 0, st>>>(v, g);
}

}  // namespace

cudaError_t launch_multi_g2p(const BatchLaunch& L, cudaStream_t st)
{
    if (!L.total[kBkPart]) return cudaSuccess;
    k_multi_g2p<<<L.total[kBkPart], 256, 0, st>>>(L.plan);
    count_launch();
    return cudaGetLastError();
}

G2PArgs g2p_args(const SceneView& v, double dt)
{
    G2PArgs g;
    g.nsub = v.rk_substeps;
    g.dt_sub = (float)(dt / g.nsub);
    g.same_origins = 1;
    for (int a = 0; a < 3; ++a)
        g.same_origins &= (v.rxo[a] == v.xo[a] && v.ryo[a] == v.yo[a] && v.rzo[a] == v.zo[a]) ? 1 : 0;
    for (int a = 0; a < 3; ++a) {
        g.dom_lo[a] = (float)v.origin[a];
        g.dom_hi[a] = (float)(v.origin[a] + v.size[a]);
    }
    g.u = v.u;  // after the post group the velocity is back in buffer A
    g.v = v.v;
    g.w = v.w;
    return g;
}

cudaError_t launch_g2p(const SceneView& v, double dt, bool do_g2p, bool do_move, cudaStream_t st)
{
    if (v.np == 0 || (!do_g2p && !do_move)) return cudaSuccess;
    const G2PArgs g = g2p_args(v, dt);
    if (v.solver == FE_SOLVER_PIC) launch_solver<FE_SOLVER_PIC>(v, g, do_g2p, do_move, st);
    else if (v.solver == FE_SOLVER_FLIP) launch_solver<FE_SOLVER_FLIP>(v, g, do_g2p, do_move, st);
    else launch_solver<FE_SOLVER_APIC>(v, g, do_g2p, do_move, st);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
