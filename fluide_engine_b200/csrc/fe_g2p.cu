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

struct G2PArgs {
    float dt_sub;
    int nsub;
    int same_origins;        // the FLIP residual grid's data origins equal the velocity grid's (domain origin 0)
    float dom_lo[3], dom_hi[3];
    const float *u, *v, *w;  // final velocity buffers
};

__device__ __forceinline__ void sample_vel(const SceneView& v, const G2PArgs& g, float x, float y, float z, float out[3])
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    out[0] = sample_face(g.u, x, y, z, v.xo, v.inv_hf, nx + 1, ny, nz);
    out[1] = sample_face(g.v, x, y, z, v.yo, v.inv_hf, nx, ny + 1, nz);
    out[2] = sample_face(g.w, x, y, z, v.zo, v.inv_hf, nx, ny, nz + 1);
}

// Trilinear sample of (a - b) with the reference's Lerp tree: the FLIP residual grid is the per-face
// difference grid - snapshot (flip_simulator.cpp:138-150) sampled like any face array.
__device__ __forceinline__ float sample_diff(const float* __restrict__ a, const float* __restrict__ b, const Stencil& s,
                                             int sx, int sy)
{
#define FE_D(ii, jj, kk) (__ldg(a + idx3(ii, jj, kk, sx, sy)) - __ldg(b + idx3(ii, jj, kk, sx, sy)))
    float b0 = lerpf_ref(lerpf_ref(FE_D(s.i, s.j, s.k), FE_D(s.ip, s.j, s.k), s.fx),
                         lerpf_ref(FE_D(s.i, s.jp, s.k), FE_D(s.ip, s.jp, s.k), s.fx), s.fy);
    float b1 = lerpf_ref(lerpf_ref(FE_D(s.i, s.j, s.kp), FE_D(s.ip, s.j, s.kp), s.fx),
                         lerpf_ref(FE_D(s.i, s.jp, s.kp), FE_D(s.ip, s.jp, s.kp), s.fx), s.fy);
#undef FE_D
    return lerpf_ref(b0, b1, s.fz);
}

// The FLIP residual sample and the plain sample of the same face array at the same stencil (the residual grid and
// the velocity grid share their data origins when the domain origin is zero): one load of each face value serves
// both Lerp trees.
__device__ __forceinline__ void sample_diff_and_plain(const float* __restrict__ a, const float* __restrict__ b,
                                                      const Stencil& s, int sx, int sy, float& diff, float& plain)
{
    float av[8], dv[8];
    const int ii[2] = {s.i, s.ip}, jj[2] = {s.j, s.jp}, kk[2] = {s.k, s.kp};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const size_t f = idx3(ii[t & 1], jj[(t >> 1) & 1], kk[t >> 2], sx, sy);
        av[t] = __ldg(a + f);
        dv[t] = av[t] - __ldg(b + f);
    }
    float b0 = lerpf_ref(lerpf_ref(dv[0], dv[1], s.fx), lerpf_ref(dv[2], dv[3], s.fx), s.fy);
    float b1 = lerpf_ref(lerpf_ref(dv[4], dv[5], s.fx), lerpf_ref(dv[6], dv[7], s.fx), s.fy);
    diff = lerpf_ref(b0, b1, s.fz);
    b0 = lerpf_ref(lerpf_ref(av[0], av[1], s.fx), lerpf_ref(av[2], av[3], s.fx), s.fy);
    b1 = lerpf_ref(lerpf_ref(av[4], av[5], s.fx), lerpf_ref(av[6], av[7], s.fx), s.fy);
    plain = lerpf_ref(b0, b1, s.fz);
}

// sum_t gradweight_t * face_t for one velocity component (apic_simulator.cpp:311-336).
__device__ __forceinline__ void apic_row(const float* __restrict__ a, const Stencil& s, int sx, int sy, const float ih[3],
                                         float out[3])
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
    const int ii[2] = {s.i, s.ip}, jj[2] = {s.j, s.jp}, kk[2] = {s.k, s.kp};
    float r0 = 0.f, r1 = 0.f, r2 = 0.f;
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const float val = __ldg(a + idx3(ii[t & 1], jj[(t >> 1) & 1], kk[t >> 2], sx, sy));
        r0 += gx[t] * val;
        r1 += gy[t] * val;
        r2 += gz[t] * val;
    }
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
}

template <int SOLVER, bool G2P, bool MOVE>
__global__ void __launch_bounds__(256) k_g2p(SceneView v, G2PArgs g)
{
    const uint64_t p = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (p >= v.np) return;
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const float x = v.px[p], y = v.py[p], z = v.pz[p];
    float vel[3];
    float pic[3];
    bool have_pic = false;
    if (G2P) {
        if (SOLVER == FE_SOLVER_FLIP) {
            const Stencil su = stencil(x, y, z, v.rxo, v.inv_hf, nx + 1, ny, nz);
            const Stencil sv = stencil(x, y, z, v.ryo, v.inv_hf, nx, ny + 1, nz);
            const Stencil sw = stencil(x, y, z, v.rzo, v.inv_hf, nx, ny, nz + 1);
            float flip[3];
            if (g.same_origins && v.blend > 0.f) {
                float d[3];
                sample_diff_and_plain(g.u, v.su, su, nx + 1, ny, d[0], pic[0]);
                sample_diff_and_plain(g.v, v.sv, sv, nx, ny + 1, d[1], pic[1]);
                sample_diff_and_plain(g.w, v.sw, sw, nx, ny, d[2], pic[2]);
                flip[0] = v.vx[p] + d[0];
                flip[1] = v.vy[p] + d[1];
                flip[2] = v.vz[p] + d[2];
                have_pic = true;
            } else {
                flip[0] = v.vx[p] + sample_diff(g.u, v.su, su, nx + 1, ny);
                flip[1] = v.vy[p] + sample_diff(g.v, v.sv, sv, nx, ny + 1);
                flip[2] = v.vz[p] + sample_diff(g.w, v.sw, sw, nx, ny);
                if (v.blend > 0.f) {
                    sample_vel(v, g, x, y, z, pic);
                    have_pic = true;
                }
            }
            if (v.blend > 0.f) {
#pragma unroll
                for (int a = 0; a < 3; ++a) flip[a] = (1.f - v.blend) * flip[a] + v.blend * pic[a];
            }
            vel[0] = flip[0];
            vel[1] = flip[1];
            vel[2] = flip[2];
        } else {
            sample_vel(v, g, x, y, z, pic);
            have_pic = true;
            vel[0] = pic[0];
            vel[1] = pic[1];
            vel[2] = pic[2];
            if (SOLVER == FE_SOLVER_APIC) {
                const float lo[3] = {v.originf[0] + 0.5f * v.hf[0], v.originf[1] + 0.5f * v.hf[1],
                                     v.originf[2] + 0.5f * v.hf[2]};
                const float hi[3] = {v.originf[0] + v.sizef[0] - 0.5f * v.hf[0],
                                     v.originf[1] + v.sizef[1] - 0.5f * v.hf[1],
                                     v.originf[2] + v.sizef[2] - 0.5f * v.hf[2]};
                const float P[3] = {x, y, z};
                const float* arr[3] = {g.u, g.v, g.w};
                const float* org[3] = {v.xo, v.yo, v.zo};
                const int fsx[3] = {nx + 1, nx, nx}, fsy[3] = {ny, ny + 1, ny};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float q[3] = {P[0], P[1], P[2]};
#pragma unroll
                    for (int a = 0; a < 3; ++a)
                        if (a != c) q[a] = q[a] < lo[a] ? lo[a] : (q[a] > hi[a] ? hi[a] : q[a]);
                    const Stencil s = stencil(q[0], q[1], q[2], org[c], v.inv_hf, nx, ny, nz);
                    float row[3];
                    apic_row(arr[c], s, fsx[c], fsy[c], v.inv_hf, row);
                    v.c[3 * c][p] = row[0];
                    v.c[3 * c + 1][p] = row[1];
                    v.c[3 * c + 2][p] = row[2];
                }
            }
        }
    } else {
        vel[0] = v.vx[p];
        vel[1] = v.vy[p];
        vel[2] = v.vz[p];
    }
    float P[3] = {x, y, z};
    if (MOVE) {
        float pt0[3] = {x, y, z}, pt1[3] = {x, y, z};
        const float half = 0.5f * g.dt_sub;
        for (int t = 0; t < g.nsub; ++t) {
            float v0[3], vm[3];
            if (t == 0 && have_pic) {
                v0[0] = pic[0]; v0[1] = pic[1]; v0[2] = pic[2];
            } else {
                sample_vel(v, g, pt0[0], pt0[1], pt0[2], v0);
            }
            const float mid[3] = {pt0[0] + half * v0[0], pt0[1] + half * v0[1], pt0[2] + half * v0[2]};
            sample_vel(v, g, mid[0], mid[1], mid[2], vm);
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
        P[0] = pt1[0]; P[1] = pt1[1]; P[2] = pt1[2];
        v.px[p] = P[0];
        v.py[p] = P[1];
        v.pz[p] = P[2];
    }
    v.vx[p] = vel[0];
    v.vy[p] = vel[1];
    v.vz[p] = vel[2];
}

template <int SOLVER>
void launch_solver(const SceneView& v, const G2PArgs& g, bool do_g2p, bool do_move, unsigned nb, cudaStream_t st)
{
    if (do_g2p && do_move) k_g2p<SOLVER, true, true><<<nb, 256, 0, st>>>(v, g);
    else if (do_g2p) k_g2p<SOLVER, true, false><<<nb, 256, 0, st>>>(v, g);
    else k_g2p<SOLVER, false, true><<<nb, 256, 0, st>>>(v, g);
}

}  // namespace

cudaError_t launch_g2p(const SceneView& v, double dt, bool do_g2p, bool do_move, cudaStream_t st)
{
    if (v.np == 0 || (!do_g2p && !do_move)) return cudaSuccess;
    G2PArgs g;
    g.nsub = v.rk_substeps;
    g.dt_sub = (float)(dt / g.nsub);
    for (int a = 0; a < 3; ++a) {
        g.dom_lo[a] = (float)v.origin[a];
        g.dom_hi[a] = (float)(v.origin[a] + v.size[a]);
    }
    g.same_origins = 1;
    for (int a = 0; a < 3; ++a)
        g.same_origins &= (v.rxo[a] == v.xo[a] && v.ryo[a] == v.yo[a] && v.rzo[a] == v.zo[a]) ? 1 : 0;
    g.u = v.u;  // after the post group the velocity is back in buffer A
    g.v = v.v;
    g.w = v.w;
    const unsigned nb = (unsigned)((v.np + 255) / 256);
    if (v.solver == FE_SOLVER_PIC) launch_solver<FE_SOLVER_PIC>(v, g, do_g2p, do_move, nb, st);
    else if (v.solver == FE_SOLVER_FLIP) launch_solver<FE_SOLVER_FLIP>(v, g, do_g2p, do_move, nb, st);
    else launch_solver<FE_SOLVER_APIC>(v, g, do_g2p, do_move, nb, st);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
