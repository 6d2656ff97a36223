// fe_diffuse.cu -- viscosity: implicit (backward Euler) diffusion of the face velocities.
//
// Reference: PICSimulator::ComputeDiffusion (pic_simulator.cpp:214-222) runs, when the viscosity is > 0,
// BackwardEulerDiffusionSolver::Solve (fluid_solvers/backward_euler_diffusion_solver.cpp:20-49) and then
// ApplyBoundryCondition.  Per velocity component the solver
//   1. marks each face FLUID iff the fluid SDF sampled at the face centre is < 0 (:71-128; without colliders the
//      collider SDF is positive everywhere, so BOUNDRY never occurs and b gets no boundary terms);
//   2. builds the rows (:136-242): for a FLUID face, center = 1 + c_a for every in-range non-AIR neighbour in
//      the order +x, -x, +y, -y, +z, -z and -c_a towards every FLUID neighbour; identity rows elsewhere;
//      b = x = the face velocity; c_a = nu dt / h_a^2;
//   3. solves with CudaJacobiIterationSolver(1000, 5, 1e-14) (:10; linear_system/cuda_jacobi_iteration_solver.cu:
//      5-24,41-63): x' = (b - sum of the off-diagonal terms in the order -x, +x, -y, +y, -z, +z) / center, and
//      after relaxation i (0-based) with i != 0 and i % 5 == 0 it stops if ||b - A x||_2 < 1e-14.
//
// Pipeline: launch_face_fluid_marks (fe_mark.cu) gives the face markers from the same band SDF the reference
// builds; k_face_list compacts the FLUID faces of all three components into one list with their FLUID-neighbour
// masks and seeds x0 = b; k_jacobi is one persistent cooperative kernel over that list with one grid barrier per
// relaxation.  All arithmetic is FP64 with the reference's operation order and no fused multiply-add, so on the
// same FP32 grid the iterates equal the reference's bit for bit.  A residual check of iterate p is computed in
// the pass that relaxes p (both read the same neighbours), so checks cost no extra pass: if the check passes,
// iterate p is the result and the speculative p + 1 is dropped.  Each component stops relaxing at its own
// check, as the reference's three separate solves do.  The last step writes the result rounded to FP32 and
// zeroes the six wall layers (ApplyBoundryCondition without colliders).
#include "fe_solver_common.cuh"

namespace fe {
namespace {

constexpr int kJacobiThreads = 1024;
constexpr int kJacobiMaxIt = 1000;      // CudaJacobiIterationSolver(1000, 5, 1e-14)
constexpr int kJacobiCheck = 5;
constexpr double kJacobiTol = 0.00000000000001;

struct FaceArrays3 {
    float* vel[3];
    size_t off[3];  // offset of each component in the concatenated face arrays
};

// One entry per FLUID face (order of the list is free: a Jacobi relaxation is pointwise).  Wall faces of a
// non-FLUID kind keep their value through the solve, so their zeroing is done here.
__global__ void k_face_list(DiffWork d, FaceArrays3 fa, int nx, int ny, int nz)
{
    FaceCoord fc;
    if (!face_coord(nx, ny, nz, fc)) return;
    const int c = fc.c, i = fc.i, j = fc.j, k = fc.k, sx = fc.sx, sy = fc.sy, sz = fc.sz;
    float* vel = c == 0 ? fa.vel[0] : (c == 1 ? fa.vel[1] : fa.vel[2]);
    const size_t g = (c == 0 ? fa.off[0] : (c == 1 ? fa.off[1] : fa.off[2])) + fc.f;
    const bool wall = (c == 0 && (i == 0 || i == sx - 1)) || (c == 1 && (j == 0 || j == sy - 1)) ||
                      (c == 2 && (k == 0 || k == sz - 1));
    const uint8_t* __restrict__ mk = d.mark;
    if (mk[g] != FE_CELL_FLUID) {
        if (wall) vel[fc.f] = 0.f;
        return;
    }
    const size_t sxy = (size_t)sx * sy;
    const uint32_t m = (i > 0 && mk[g - 1] == FE_CELL_FLUID ? kXm : 0u) |
                       (i + 1 < sx && mk[g + 1] == FE_CELL_FLUID ? kXp : 0u) |
                       (j > 0 && mk[g - sx] == FE_CELL_FLUID ? kYm : 0u) |
                       (j + 1 < sy && mk[g + sx] == FE_CELL_FLUID ? kYp : 0u) |
                       (k > 0 && mk[g - sxy] == FE_CELL_FLUID ? kZm : 0u) |
                       (k + 1 < sz && mk[g + sxy] == FE_CELL_FLUID ? kZp : 0u);
    const unsigned long long entry = ((unsigned long long)g << 9) | ((unsigned long long)wall << 8) |
                                     ((unsigned long long)c << 6) | m;
    // warp-aggregated append
    const unsigned act = __activemask();
    const int lane = threadIdx.x & 31;  // blockDim.x == 32: the lane is threadIdx.x
    const int leader = __ffs(act) - 1;
    unsigned base = 0;
    if (lane == leader) base = atomicAdd(d.count, (unsigned)__popc(act));
    base = __shfl_sync(act, base, leader);
    d.list[base + __popc(act & ((1u << lane) - 1u))] = entry;
    d.x[0][g] = (double)vel[fc.f];
}

struct JacobiParams {
    double c[3];   // nu dt / h_a^2
    int sx[3];     // x extent of each component's face array
    int sxy[3];    // x * y extent
};

__global__ void __launch_bounds__(kJacobiThreads, 1) k_jacobi(DiffWork d, CgWork w, FaceArrays3 fa, JacobiParams prm)
{
    __shared__ double sh[32 * 4 + 4];
    const int nblk = gridDim.x, blk = blockIdx.x;
    const unsigned T = (unsigned)nblk * blockDim.x, tid = (unsigned)blk * blockDim.x + threadIdx.x;
    unsigned gen = 0;
    if (threadIdx.x == 0)
        gen = cuda::atomic_ref<unsigned, cuda::thread_scope_device>(w.bar[32]).load(cuda::memory_order_relaxed);
    const unsigned count = __ldcg(d.count);
    const unsigned long long* __restrict__ list = d.list;
    // buffers selected by value (a runtime index into the parameter array would copy it to local memory)
    double* const x0 = d.x[0];
    double* const x1 = d.x[1];
    const double cx = prm.c[0], cy = prm.c[1], cz = prm.c[2];
    const double ncx = -cx, ncy = -cy, ncz = -cz;  // A(.).right / up / front = 0.0 - c_a
    unsigned done = 0u;    // bit c: component c has its result
    unsigned parity = 0u;  // bit c: buffer holding component c's result
    int its[3] = {kJacobiMaxIt, kJacobiMaxIt, kJacobiMaxIt};

    for (int p = 0; p < kJacobiMaxIt; ++p) {
        // iterate p is checked after relaxation p - 1 when p - 1 != 0 and (p - 1) % 5 == 0
        const bool chk = p > 1 && (p - 1) % kJacobiCheck == 0;
        const double* __restrict__ xr = (p & 1) ? x1 : x0;
        double* __restrict__ xw = (p & 1) ? x0 : x1;
        double acc[3] = {0.0, 0.0, 0.0};
        for (unsigned e = tid; e < count; e += T) {
            const unsigned long long ent = __ldg(list + e);
            const unsigned c = (unsigned)(ent >> 6) & 3u;
            if ((done >> c) & 1u) continue;
            const uint32_t m = (uint32_t)ent & 63u;
            const size_t g = (size_t)(ent >> 9);
            const int sx = c == 0 ? prm.sx[0] : (c == 1 ? prm.sx[1] : prm.sx[2]);
            const int sxy = c == 0 ? prm.sxy[0] : (c == 1 ? prm.sxy[1] : prm.sxy[2]);
            const float* vel = c == 0 ? fa.vel[0] : (c == 1 ? fa.vel[1] : fa.vel[2]);
            const size_t off = c == 0 ? fa.off[0] : (c == 1 ? fa.off[1] : fa.off[2]);
            // every load issued before any use
            const double b = (double)__ldg(vel + (g - off));
            const double xl = (m & kXm) ? __ldcg(xr + g - 1) : 0.0;
            const double xh = (m & kXp) ? __ldcg(xr + g + 1) : 0.0;
            const double yl = (m & kYm) ? __ldcg(xr + g - sx) : 0.0;
            const double yh = (m & kYp) ? __ldcg(xr + g + sx) : 0.0;
            const double zl = (m & kZm) ? __ldcg(xr + g - sxy) : 0.0;
            const double zh = (m & kZp) ? __ldcg(xr + g + sxy) : 0.0;
            const double xc = chk ? __ldcg(xr + g) : 0.0;
            // BuildMatrix center: +x, -x, +y, -y, +z, -z
            double cen = 1.0;
            if (m & kXp) cen = __dadd_rn(cen, cx);
            if (m & kXm) cen = __dadd_rn(cen, cx);
            if (m & kYp) cen = __dadd_rn(cen, cy);
            if (m & kYm) cen = __dadd_rn(cen, cy);
            if (m & kZp) cen = __dadd_rn(cen, cz);
            if (m & kZm) cen = __dadd_rn(cen, cz);
            // off-diagonal terms in Relax order; a term of a non-FLUID neighbour is a signed zero in the
            // reference, which changes no sum
            const double t0 = __dmul_rn(ncx, xl), t1 = __dmul_rn(ncx, xh);
            const double t2 = __dmul_rn(ncy, yl), t3 = __dmul_rn(ncy, yh);
            const double t4 = __dmul_rn(ncz, zl), t5 = __dmul_rn(ncz, zh);
            double r = 0.0;
            if (m & kXm) r = __dadd_rn(r, t0);
            if (m & kXp) r = __dadd_rn(r, t1);
            if (m & kYm) r = __dadd_rn(r, t2);
            if (m & kYp) r = __dadd_rn(r, t3);
            if (m & kZm) r = __dadd_rn(r, t4);
            if (m & kZp) r = __dadd_rn(r, t5);
            xw[g] = __ddiv_rn(__dsub_rn(b, r), cen);
            if (chk) {
                // BLAS::Residual: b - center * x - the same terms, left to right
                double rs = __dsub_rn(b, __dmul_rn(cen, xc));
                if (m & kXm) rs = __dsub_rn(rs, t0);
                if (m & kXp) rs = __dsub_rn(rs, t1);
                if (m & kYm) rs = __dsub_rn(rs, t2);
                if (m & kYp) rs = __dsub_rn(rs, t3);
                if (m & kZm) rs = __dsub_rn(rs, t4);
                if (m & kZp) rs = __dsub_rn(rs, t5);
                const double q = rs * rs;
                acc[0] += c == 0 ? q : 0.0;
                acc[1] += c == 1 ? q : 0.0;
                acc[2] += c == 2 ? q : 0.0;
            }
        }
        if (chk) {
            if (!grid_reduce<3>(acc, sh, w, gen, nblk)) return;
#pragma unroll
            for (int c = 0; c < 3; ++c)
                if (!((done >> c) & 1u) && sqrt(acc[c]) < kJacobiTol) {
                    done |= 1u << c;
                    parity |= (unsigned)(p & 1) << c;
                    its[c] = p;
                }
            if (done == 7u) break;
        } else if (!grid_sync(w, gen, nblk)) {
            return;
        }
    }
    // components that never passed a check end with iterate 1000
#pragma unroll
    for (int c = 0; c < 3; ++c)
        if (!((done >> c) & 1u)) parity |= (unsigned)(kJacobiMaxIt & 1) << c;
    // every entry's result was written by this thread itself (entries are assigned to threads the same way in
    // every pass), so no barrier is needed before the write-back
    for (unsigned e = tid; e < count; e += T) {
        const unsigned long long ent = __ldg(list + e);
        const unsigned c = (unsigned)(ent >> 6) & 3u;
        const size_t g = (size_t)(ent >> 9);
        float* vel = c == 0 ? fa.vel[0] : (c == 1 ? fa.vel[1] : fa.vel[2]);
        const size_t off = c == 0 ? fa.off[0] : (c == 1 ? fa.off[1] : fa.off[2]);
        const double* xf = ((parity >> c) & 1u) ? x1 : x0;
        vel[g - off] = ((ent >> 8) & 1u) ? 0.f : (float)__ldcg(xf + g);
    }
    if (blk == 0 && threadIdx.x == 0) {
        d.its[0] = its[0];
        d.its[1] = its[1];
        d.its[2] = its[2];
    }
}

}  // namespace

cudaError_t diffuse_prepare(DiffWork& d, int device)
{
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi, kJacobiThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    d.blocks = sms;  // one persistent block per SM
    return cudaSuccess;
}

cudaError_t launch_diffuse(const SceneView& v, const DiffWork& d, const CgWork& w, float* u, float* vv, float* ww,
                           double dt, double viscosity, cudaStream_t st)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    if (d.blocks < 1) return cudaErrorInitializationError;
    cudaError_t e;
    if ((e = cudaMemsetAsync(d.count, 0, sizeof(unsigned), st)) != cudaSuccess) return e;
    if ((e = launch_face_fluid_marks(v, d, st)) != cudaSuccess) return e;
    FaceArrays3 fa;
    fa.vel[0] = u;
    fa.vel[1] = vv;
    fa.vel[2] = ww;
    fa.off[0] = 0;
    fa.off[1] = (size_t)(nx + 1) * ny * nz;
    fa.off[2] = fa.off[1] + (size_t)nx * (ny + 1) * nz;
    k_face_list<<<face_grid(nx, ny, nz), dim3(kTileX, kTileY), 0, st>>>(d, fa, nx, ny, nz);
    count_launch();
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    JacobiParams prm;
    // PICSimulator::ComputeDiffusion passes dt and the viscosity swapped into Solve; the product is the same
    for (int a = 0; a < 3; ++a) prm.c[a] = (viscosity * dt) / (v.h[a] * v.h[a]);
    prm.sx[0] = nx + 1;
    prm.sxy[0] = (nx + 1) * ny;
    prm.sx[1] = nx;
    prm.sxy[1] = nx * (ny + 1);
    prm.sx[2] = nx;
    prm.sxy[2] = nx * ny;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)d.blocks);
    cfg.blockDim = dim3((unsigned)kJacobiThreads);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_jacobi, d, w, fa, prm);
    count_launch();
    return e;
}

}  // namespace fe
