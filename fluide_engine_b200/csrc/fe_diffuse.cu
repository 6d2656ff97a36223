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
//
// Early exit without changing the result: the 1e-14 test is absolute, so for most grids it never passes (the
// FP64 rounding floor of ||b - A x|| over ~10^6 faces is above it) and the reference runs all 1000 relaxations.
// The Jacobi map is deterministic, so once a component's iterates repeat bit for bit (they settle at a fixed
// point or a short cycle in the last bits) iterate 1000 is known from the cycle; k_jacobi finds the cycle with
// snapshots compared at check passes and stops the component at the pass that writes an iterate equal to
// iterate 1000 (it reports 1000 iterations, as the reference would).
#include "fe_solver_common.cuh"

namespace fe {
namespace {

constexpr int kJacobiThreads = 1024;
constexpr int kJacobiUnroll = 1;  // list entries in flight per thread (more, at fewer threads, measured slower)
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

// Shared-memory cache of a block's slice of the FLUID-face list: the entries and their right-hand sides (FP32
// velocities, exact in FP64), read once per solve instead of once per relaxation.
constexpr int kJacobiCache = 8192;  // 96 KB: the rest of the 256 KB on-chip memory stays L1 for the neighbour reads
constexpr size_t kJacobiSmem = (size_t)kJacobiCache * (sizeof(unsigned long long) + sizeof(float));

// Per-component state of the exact early exit (identical in every thread: it only changes from grid-reduced
// values).  The iterates of a component are eventually periodic once they stop changing in FP64 (period 1) or
// cycle in their last bits.  A snapshot of the iterate read at a check pass is compared with the iterates read
// at later check passes; without a match after 1, 2, 4, ... checks the snapshot moves (Brent's cycle search),
// so a cycle of any length is found once the snapshot lies in it.  Check passes are 5 apart, so the distance M
// = q - s from snapshot pass s to the matching pass q is a multiple of 5 and of the true period (M is a period
// as well).  From s on, the check iterates fall into M / 5 residue classes modulo M, and the checks at s,
// s + 5, ..., q have already tested one iterate of each: all failed, so no later check can pass, and iterate
// 1000 equals iterate k for the first k > q with (1000 - k) % M == 0.
struct CycleState {
    int snap_pass;   // check pass whose iterate is in the snapshot (-1: none)
    int window;      // checks to wait for a match before re-taking the snapshot
    int waited;      // checks since the snapshot
    int target;      // pass count k after which iterate k = iterate 1000 is in buffer k % 2 (0: none)
};

__global__ void __launch_bounds__(kJacobiThreads, 1)
    k_jacobi(DiffWork d, CgWork w, FaceArrays3 fa, JacobiParams prm)
{
    double* __restrict__ snap = d.snap;
    __shared__ double sh[kShDoubles];
    extern __shared__ unsigned long long s_ent[];  // [kJacobiCache] entries, then [kJacobiCache] floats
    float* s_b = (float*)(s_ent + kJacobiCache);
    const int nblk = gridDim.x, blk = blockIdx.x;
    unsigned gen = 0;  // barriers passed in this launch
    const unsigned count = __ldcg(d.count);
    // The list is in face order, component by component; it is dealt to the blocks in tiles of blockDim.x
    // consecutive entries (tile t to block t % nblk), so every block holds a share of each component and the
    // blocks stay balanced after a component stops.  Thread t of a block takes entry t of each of its tiles;
    // slot k * blockDim.x + t of the block's sequence is entry (blk + k nblk) blockDim.x + t of the list.
    constexpr unsigned B = kJacobiThreads;  // == blockDim.x (a constant: slot / B is a shift)
    const unsigned tiles = (count + B - 1) / B;
    const unsigned my_tiles = tiles > (unsigned)blk ? (tiles - blk + nblk - 1) / nblk : 0u;
    const unsigned mine = my_tiles * B;  // slots, some past the end of the list in the last tile
    const unsigned cached = min(mine, (unsigned)kJacobiCache);
    auto list_index = [&](unsigned slot) -> unsigned { return ((unsigned)blk + (slot / B) * nblk) * B + slot % B; };
    const unsigned long long* __restrict__ list = d.list;
    auto rhs_of = [&](unsigned long long ent) -> float {
        const unsigned c = (unsigned)(ent >> 6) & 3u;
        const float* vel = c == 0 ? fa.vel[0] : (c == 1 ? fa.vel[1] : fa.vel[2]);
        const size_t off = c == 0 ? fa.off[0] : (c == 1 ? fa.off[1] : fa.off[2]);
        return __ldg(vel + ((size_t)(ent >> 9) - off));
    };
    for (unsigned i = threadIdx.x; i < cached; i += B) {
        const unsigned e = list_index(i);
        const unsigned long long ent = e < count ? __ldg(list + e) : ~0ull;  // ~0: past the end
        s_ent[i] = ent;
        s_b[i] = e < count ? rhs_of(ent) : 0.f;
    }
    __syncthreads();
    // buffers selected by value (a runtime index into the parameter array would copy it to local memory)
    double* const x0 = d.x[0];
    double* const x1 = d.x[1];
    const double cx = prm.c[0], cy = prm.c[1], cz = prm.c[2];
    const double ncx = -cx, ncy = -cy, ncz = -cz;  // A(.).right / up / front = 0.0 - c_a
    // control state, kept in shared memory (registers are at their 64-per-thread limit): thread 0 updates it
    // from the grid-reduced values after each barrier, every thread reads it after the next __syncthreads
    __shared__ struct {
        unsigned done;       // bit c: component c has its result
        unsigned parity;     // bit c: buffer holding component c's result
        unsigned take, cmp;  // bit c: at the next check pass, take / compare component c's snapshot
        int its[3];
        int passes;
        int stop;
        CycleState cs[3];
    } ctl;
    if (threadIdx.x == 0) {
        ctl.done = ctl.parity = ctl.cmp = 0u;
        ctl.take = 7u;
        ctl.its[0] = ctl.its[1] = ctl.its[2] = kJacobiMaxIt;
        ctl.passes = kJacobiMaxIt;
        ctl.stop = 0;
        for (int c = 0; c < 3; ++c) ctl.cs[c] = CycleState{-1, 1, 0, 0};
    }
    __syncthreads();

    for (int p = 0; p < kJacobiMaxIt; ++p) {
        // iterate p is checked after relaxation p - 1 when p - 1 != 0 and (p - 1) % 5 == 0
        const bool chk = p > 1 && (p - 1) % kJacobiCheck == 0;
        const unsigned done = ctl.done;
        const unsigned take = chk ? ctl.take & ~done : 0u, cmp = chk ? ctl.cmp & ~done : 0u;
        // Iterate p was written by all blocks during the previous pass.  The grid barrier's device-scope
        // acquire (thread 0) followed by __syncthreads orders it before every read below, so L1-cached loads
        // (ld.global.ca) see it; neighbours shared by the block's threads then come from L1 instead of L2.
        // (Not __restrict__ const: that would allow the non-coherent read-only path.)
        const double* xr = (p & 1) ? x1 : x0;
        double* xw = (p & 1) ? x0 : x1;
        double acc[3] = {0.0, 0.0, 0.0};
        unsigned chg = 0u;  // bit c: some face of component c differs from its snapshot (check passes)
        // kJacobiUnroll entries per thread at a time, all their loads issued before any result is computed
        for (unsigned i0 = threadIdx.x; i0 < mine; i0 += kJacobiUnroll * blockDim.x) {
            unsigned long long ent[kJacobiUnroll];
            double bv[kJacobiUnroll], nb[kJacobiUnroll][6], xc[kJacobiUnroll], sv[kJacobiUnroll];
            bool live[kJacobiUnroll];
#pragma unroll
            for (int u = 0; u < kJacobiUnroll; ++u) {
                const unsigned i = i0 + u * blockDim.x;
                const unsigned e = list_index(i);
                live[u] = i < mine && e < count;
                ent[u] = live[u] ? (i < cached ? s_ent[i] : __ldg(list + e)) : 0ull;
                const unsigned c = (unsigned)(ent[u] >> 6) & 3u;
                live[u] = live[u] && !((done >> c) & 1u);
                bv[u] = 0.0;
                xc[u] = sv[u] = 0.0;
#pragma unroll
                for (int k = 0; k < 6; ++k) nb[u][k] = 0.0;
                if (!live[u]) continue;
                const uint32_t m = (uint32_t)ent[u] & 63u;
                const size_t g = (size_t)(ent[u] >> 9);
                const int sx = c == 0 ? prm.sx[0] : (c == 1 ? prm.sx[1] : prm.sx[2]);
                const int sxy = c == 0 ? prm.sxy[0] : (c == 1 ? prm.sxy[1] : prm.sxy[2]);
                bv[u] = (double)(i < cached ? s_b[i] : rhs_of(ent[u]));
                if (m & kXm) nb[u][0] = __ldca(xr + g - 1);
                if (m & kXp) nb[u][1] = __ldca(xr + g + 1);
                if (m & kYm) nb[u][2] = __ldca(xr + g - sx);
                if (m & kYp) nb[u][3] = __ldca(xr + g + sx);
                if (m & kZm) nb[u][4] = __ldca(xr + g - sxy);
                if (m & kZp) nb[u][5] = __ldca(xr + g + sxy);
                if (chk) xc[u] = __ldca(xr + g);
                if ((cmp >> c) & 1u) sv[u] = __ldcg(snap + g);
            }
#pragma unroll
            for (int u = 0; u < kJacobiUnroll; ++u) {
                if (!live[u]) continue;
                const unsigned c = (unsigned)(ent[u] >> 6) & 3u;
                const uint32_t m = (uint32_t)ent[u] & 63u;
                const size_t g = (size_t)(ent[u] >> 9);
                const double b = bv[u];
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
                const double t0 = __dmul_rn(ncx, nb[u][0]), t1 = __dmul_rn(ncx, nb[u][1]);
                const double t2 = __dmul_rn(ncy, nb[u][2]), t3 = __dmul_rn(ncy, nb[u][3]);
                const double t4 = __dmul_rn(ncz, nb[u][4]), t5 = __dmul_rn(ncz, nb[u][5]);
                double r = 0.0;
                if (m & kXm) r = __dadd_rn(r, t0);
                if (m & kXp) r = __dadd_rn(r, t1);
                if (m & kYm) r = __dadd_rn(r, t2);
                if (m & kYp) r = __dadd_rn(r, t3);
                if (m & kZm) r = __dadd_rn(r, t4);
                if (m & kZp) r = __dadd_rn(r, t5);
                xw[g] = __ddiv_rn(__dsub_rn(b, r), cen);
                if (chk) {
                    if ((take >> c) & 1u) snap[g] = xc[u];
                    if (((cmp >> c) & 1u) && __double_as_longlong(xc[u]) != __double_as_longlong(sv[u]))
                        chg |= 1u << c;
                    // BLAS::Residual: b - center * x - the same terms, left to right
                    double rs = __dsub_rn(b, __dmul_rn(cen, xc[u]));
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
        }
        if (chk) {
            // blocks that saw a snapshot mismatch, per component, packed in one exact double (< 1024 blocks)
            const int a0 = __syncthreads_or((int)(chg & 1u)), a1 = __syncthreads_or((int)(chg & 2u));
            const int a2 = __syncthreads_or((int)(chg & 4u));
            double red[4] = {acc[0], acc[1], acc[2],
                             threadIdx.x == 0 ? (a0 ? 1.0 : 0.0) + (a1 ? 1024.0 : 0.0) + (a2 ? 1048576.0 : 0.0) : 0.0};
            if (!grid_reduce<4>(red, sh, w, gen, nblk, blk)) {
                solver_exit(w, nblk);
                return;
            }
            if (threadIdx.x == 0) {
                const double packed = red[3];
                const double changed[3] = {fmod(packed, 1024.0), fmod(floor(packed / 1024.0), 1024.0),
                                           floor(packed / 1048576.0)};
                unsigned next_take = 0u, next_cmp = 0u;
                for (int c = 0; c < 3; ++c) {
                    if ((ctl.done >> c) & 1u) continue;
                    CycleState& st = ctl.cs[c];
                    if (sqrt(red[c]) < kJacobiTol) {  // the reference's stop
                        ctl.done |= 1u << c;
                        ctl.parity |= (unsigned)(p & 1) << c;
                        ctl.its[c] = p;
                        continue;
                    }
                    if (st.target) continue;
                    bool move = false;
                    if ((take >> c) & 1u) {
                        st.snap_pass = p;
                        st.waited = 0;
                    } else if ((cmp >> c) & 1u) {
                        if (changed[c] == 0.0) {
                            // iterate p = iterate snap_pass on every face: period M = p - snap_pass
                            const int M = p - st.snap_pass;
                            st.target = kJacobiMaxIt - M * ((kJacobiMaxIt - (p + 1)) / M);  // in [p + 1, 1000]
                            continue;
                        }
                        if (++st.waited >= st.window) {  // Brent: move the snapshot, double the window
                            move = true;
                            st.window *= 2;
                        }
                    }
                    if (move) next_take |= 1u << c;
                    else if (st.snap_pass >= 0) next_cmp |= 1u << c;
                }
                ctl.take = next_take;
                ctl.cmp = next_cmp;
            }
        } else if (!grid_sync(w, gen, nblk, sh, blk)) {
            solver_exit(w, nblk);
            return;
        }
        if (threadIdx.x == 0) {
            // components whose iterate 1000 was just written (pass p wrote iterate p + 1)
            for (int c = 0; c < 3; ++c)
                if (!((ctl.done >> c) & 1u) && ctl.cs[c].target == p + 1) {
                    ctl.done |= 1u << c;
                    ctl.parity |= (unsigned)((p + 1) & 1) << c;
                }
            if (ctl.done == 7u) {
                ctl.passes = p + 1;
                ctl.stop = 1;
            }
        }
        __syncthreads();
        if (ctl.stop) break;
    }
    // components that never stopped end with iterate 1000
    if (threadIdx.x == 0)
        for (int c = 0; c < 3; ++c)
            if (!((ctl.done >> c) & 1u)) ctl.parity |= (unsigned)(kJacobiMaxIt & 1) << c;
    __syncthreads();
    const unsigned parity = ctl.parity;
    // every entry's result was written by this thread itself (entries are assigned to threads the same way in
    // every pass), so no barrier is needed before the write-back
    for (unsigned i = threadIdx.x; i < mine; i += blockDim.x) {
        const unsigned e = list_index(i);
        if (e >= count) continue;
        const unsigned long long ent = i < cached ? s_ent[i] : __ldg(list + e);
        const unsigned c = (unsigned)(ent >> 6) & 3u;
        const size_t g = (size_t)(ent >> 9);
        float* vel = c == 0 ? fa.vel[0] : (c == 1 ? fa.vel[1] : fa.vel[2]);
        const size_t off = c == 0 ? fa.off[0] : (c == 1 ? fa.off[1] : fa.off[2]);
        const double* xf = ((parity >> c) & 1u) ? x1 : x0;
        vel[g - off] = ((ent >> 8) & 1u) ? 0.f : (float)__ldcg(xf + g);
    }
    if (blk == 0 && threadIdx.x == 0) {
        d.its[0] = ctl.its[0];
        d.its[1] = ctl.its[1];
        d.its[2] = ctl.its[2];
        d.its[3] = ctl.passes;
    }
    solver_exit(w, nblk);
}

}  // namespace

cudaError_t diffuse_prepare(DiffWork& d, int device)
{
    int sms = 0, per_sm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_jacobi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kJacobiSmem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jacobi, kJacobiThreads, kJacobiSmem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    d.blocks = sms;  // one persistent block per SM
    return cudaSuccess;
}

cudaError_t launch_diffuse(const SceneView& v, const DiffWork& d, const CgWork& w, float* u, float* vv, float* ww,
                           double dt, double viscosity, cudaStream_t st)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    if (d.blocks < 1 || d.blocks > 1023) return cudaErrorInitializationError;  // k_jacobi packs block counts in 10 bits
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
    cfg.dynamicSmemBytes = kJacobiSmem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CgWork jw = w;
    jw.cluster = 1;  // the Jacobi kernel shares the solver's barrier words, never its cluster launch
    e = cudaLaunchKernelEx(&cfg, k_jacobi, d, jw, fa, prm);
    count_launch();
    return e;
}

}  // namespace fe
