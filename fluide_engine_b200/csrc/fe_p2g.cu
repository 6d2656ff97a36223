// fe_p2g.cu -- particle -> grid transfer (K_p2g).
//
// Reference: PICSimulator::TransferParticles2Grid (pic_simulator.cpp:356-437), FLIPSimulator
// (flip_simulator.cpp:25-119) and APICSimulator (apic_simulator.cpp:15-118): for every particle and
// every velocity component, trilinear weights w on the 8 surrounding faces (GetCooridnatesAndWeights,
// common/math_utils.hpp:75-112), u += w * value, weight += w, marker = 1; then u /= weight where
// weight > 0.  PIC and APIC clamp the face index with the CELL count, FLIP with the face count.  APIC
// adds C_row . (x_face - x_clamped), the particle position clamped by h/2 on the two transverse axes.
//
// B200 design: one CTA per 8x8x8-cell tile and one thread per cell of it.  The tile's particles are one
// contiguous run of the sorted arrays (fe_keys.h) and a cell's particles a contiguous piece of that run, so
// each thread walks its own cell's particles and sums their contributions in registers.  With the domain origin
// at zero the faces a particle of cell (cx, cy, cz) touches lie in a window around the cell -- faces c and c + 1
// along the component's own axis, c - 1 .. c + 1 along the two others (the clamps of GetBarycentric at the domain
// walls excepted: those particles take the direct path below) -- so a thread's sums live in 18 slots per
// component, (numerator, weight) per window face, plus a touched mask.  Only then does the
// thread add its touched slots into the tile's 10x10x10 face box in shared memory: one shared atomic per
// (cell, face) pair instead of one per (particle, face) pair, and the 32 lanes of an atomic instruction hit 32
// different faces.  Cells with more than kCellCap particles (particles clamped onto a wall pile up in one
// cell) hand the rest to a warp that spreads them over its lanes and combines the lanes' slots by shuffles.
// The box is then flushed to global accumulators: box faces touched by the tile get one global red.add each,
// so a face receives at most 8 global adds (one per neighbouring tile), never one per particle.  A second pass
// divides numerator by weight and, for FLIP, writes the snapshot (flip_simulator.cpp:107-118).  A particle
// whose stencil leaves its cell's window (only possible for a domain origin away from zero, where the
// reference's data origins ignore the origin) takes the direct path instead: shared atomics into the box per
// face, or global adds for faces outside the box, so the kernel stays correct for every input.
#include "fe_internal.cuh"

namespace fe {
namespace {

constexpr int kBox = 10;
constexpr int kBoxFaces = kBox * kBox * kBox;
constexpr int kP2gThreads = FE_TILE_CELLS;  // one thread per cell of a tile
constexpr int kCellCap = 32;                // particles a thread sums for its own cell; the rest go to a warp

// Per-component constants of the transfer (face-array sizes, the clamp sizes the reference passes to
// GetCooridnatesAndWeights, the data origin, the global accumulators).
struct P2gComp {
    int fsx, fsy, fsz;  // face-array sizes
    int csx, csy, csz;  // clamp sizes: FLIP the face counts, PIC / APIC the cell counts
    float org[3];       // data origin of the component's face grid
    float* gnum;
    float* gden;
    uint8_t* gmk;
};

template <int SOLVER>
__device__ __forceinline__ P2gComp p2g_comp(const SceneView& v, int c)
{
    const int nx = v.g.nx, ny = v.g.ny, nz = v.g.nz;
    const bool flip = SOLVER == FE_SOLVER_FLIP;
    P2gComp k;
    k.fsx = nx + (c == 0);
    k.fsy = ny + (c == 1);
    k.fsz = nz + (c == 2);
    k.csx = flip ? k.fsx : nx;
    k.csy = flip ? k.fsy : ny;
    k.csz = flip ? k.fsz : nz;
#pragma unroll
    for (int a = 0; a < 3; ++a) k.org[a] = c == 0 ? v.xo[a] : (c == 1 ? v.yo[a] : v.zo[a]);
    k.gnum = c == 0 ? v.nu : (c == 1 ? v.nv : v.nw);
    k.gden = c == 0 ? v.du : (c == 1 ? v.dv : v.dw);
    k.gmk = c == 0 ? v.mu : (c == 1 ? v.mv : v.mw);
    return k;
}

// A particle's value for component c and its (APIC) clamped position and C row.
template <int SOLVER>
struct P2gParticle {
    float vc;
    float pc[3];
    float cr[3];
};

template <int SOLVER>
__device__ __forceinline__ P2gParticle<SOLVER> load_particle(const SceneView& v, uint32_t p, int c, float x, float y,
                                                             float z, const float lo[3], const float hi[3])
{
    P2gParticle<SOLVER> q;
    q.vc = __ldg((c == 0 ? v.vx : (c == 1 ? v.vy : v.vz)) + p);
    q.pc[0] = x;
    q.pc[1] = y;
    q.pc[2] = z;
    q.cr[0] = q.cr[1] = q.cr[2] = 0.f;
    if (SOLVER == FE_SOLVER_APIC) {
        q.cr[0] = __ldg(v.c[3 * c] + p);
        q.cr[1] = __ldg(v.c[3 * c + 1] + p);
        q.cr[2] = __ldg(v.c[3 * c + 2] + p);
        // Clamp(val, max, min) on the two transverse axes (apic_simulator.cpp:55-57,68-70,81-83)
#pragma unroll
        for (int a = 0; a < 3; ++a)
            if (a != c) q.pc[a] = q.pc[a] < lo[a] ? lo[a] : (q.pc[a] > hi[a] ? hi[a] : q.pc[a]);
    }
    return q;
}

// The particle's 8 faces added one by one: into the box (shared atomics) or, outside it, into the global
// accumulators.  Used for particles whose stencil leaves their cell's window.
template <int SOLVER>
__device__ void splat_direct(const SceneView& v, const P2gComp& k, const Stencil& s, const P2gParticle<SOLVER>& q,
                             int bx, int by, int bz, float* s_num, float* s_den, uint8_t* s_mk)
{
    const float wx[2] = {1.f - s.fx, s.fx}, wy[2] = {1.f - s.fy, s.fy}, wz[2] = {1.f - s.fz, s.fz};
    const int ii[2] = {s.i, s.ip}, jj[2] = {s.j, s.jp}, kk[2] = {s.k, s.kp};
#pragma unroll
    for (int t = 0; t < 8; ++t) {
        const int a = t & 1, b = (t >> 1) & 1, d = t >> 2;
        const float wgt = wx[a] * wy[b] * wz[d];
        float val = q.vc;
        if (SOLVER == FE_SOLVER_APIC) {
            const float gx = k.org[0] + v.hf[0] * (float)ii[a];
            const float gy = k.org[1] + v.hf[1] * (float)jj[b];
            const float gz = k.org[2] + v.hf[2] * (float)kk[d];
            val += q.cr[0] * (gx - q.pc[0]) + q.cr[1] * (gy - q.pc[1]) + q.cr[2] * (gz - q.pc[2]);
        }
        const int li = ii[a] - bx, lj = jj[b] - by, lk = kk[d] - bz;
        if ((unsigned)li < kBox && (unsigned)lj < kBox && (unsigned)lk < kBox) {
            const int l = li + kBox * (lj + kBox * lk);
            atomicAdd(&s_num[l], val * wgt);
            atomicAdd(&s_den[l], wgt);
            s_mk[l] = 1;
        } else {
            const size_t f = idx3(ii[a], jj[b], kk[d], k.fsx, k.fsy);
            atomicAdd(k.gnum + f, val * wgt);
            atomicAdd(k.gden + f, wgt);
            k.gmk[f] = 1;
        }
    }
}

// Window of component C's faces around a cell: along the component's own (staggered) axis a particle of cell c
// touches faces c and c + 1, along the two other axes c - 1 .. c + 1.  Slot (i, j, k) of the window is face
// (cx + lo<C>(0) + i, cy + lo<C>(1) + j, cz + lo<C>(2) + k), slot index i + W0 (j + W1 k).
template <int C> __host__ __device__ constexpr int win(int axis) { return axis == C ? 2 : 3; }
template <int C> __host__ __device__ constexpr int wlo(int axis) { return axis == C ? 0 : -1; }
template <int C> __host__ __device__ constexpr int nslots() { return win<C>(0) * win<C>(1) * win<C>(2); }  // 18
// `count` ones spaced `width` bits apart (bit 0, width, 2 width, ...).
__host__ __device__ constexpr uint32_t rep_bits(int width, int count)
{
    return count <= 0 ? 0u : (rep_bits(width, count - 1) << width) | 1u;
}

// Touched slots of the window from each axis' touched bits (tx over W0, ty over W1, tz over W2): slot (a, b, c)
// is touched when bit a of tx, b of ty and c of tz are, found by spreading each axis' bits over the slot layout.
template <int C>
__host__ __device__ constexpr uint32_t spread_mask(uint32_t tx, uint32_t ty, uint32_t tz)
{
    constexpr int W0 = win<C>(0), W1 = win<C>(1), W2 = win<C>(2);
    uint32_t sy = 0, ez = 0;
    for (int b3 = 0; b3 < W1; ++b3) sy |= ((ty >> b3) & 1u) * (((1u << W0) - 1u) << (W0 * b3));
    for (int c3 = 0; c3 < W2; ++c3) ez |= ((tz >> c3) & 1u) * (((1u << (W0 * W1)) - 1u) << (W0 * W1 * c3));
    return (tx * rep_bits(W0, W1 * W2)) & (sy * rep_bits(W0 * W1, W2)) & ez;
}
// Touched slots of an unclamped particle in the lower half of the cell on every transverse axis (the first two
// faces of each axis); the upper halves shift it by one face per axis.
template <int C>
__host__ __device__ constexpr uint32_t regular_mask()
{
    return spread_mask<C>(3u, 3u, 3u);
}

// One particle of cell (cx, cy, cz) into the cell's 18 slots of component C; returns false (and adds nothing)
// when its stencil leaves the window, in which case the caller takes the direct path.  The trilinear weight of
// slot (i, j, k) is wx_i wy_j wz_k, so the sums are formed as wx_i (wy_j wz_k v) per (j, k) pair: 2 FMAs per slot
// (APIC: v + C . (x_face - x_p) splits the same way, 3 FMAs per slot).
template <int SOLVER, int C>
__device__ __forceinline__ bool splat_slots(const SceneView& v, const P2gComp& k, const Stencil& s,
                                            const P2gParticle<SOLVER>& q, int cx, int cy, int cz,
                                            float (&num)[nslots<C>()], float (&den)[nslots<C>()], uint32_t& mask)
{
    constexpr int W0 = win<C>(0), W1 = win<C>(1), W2 = win<C>(2);
    constexpr int L0 = wlo<C>(0), L1 = wlo<C>(1), L2 = wlo<C>(2);
    const int oi = s.i - cx, oip = s.ip - cx, oj = s.j - cy, ojp = s.jp - cy, ok = s.k - cz, okp = s.kp - cz;
    if (oi < L0 || oip > L0 + W0 - 1 || oj < L1 || ojp > L1 + W1 - 1 || ok < L2 || okp > L2 + W2 - 1) return false;
    float wx[W0], wy[W1], wz[W2];
    // The usual case: no clamp on any axis, so the stencil is the cell's two own-axis faces and, on each transverse
    // axis, the lower or the upper two of the window's three faces (the half of the cell the particle is in).  The
    // weights are then selects of (1 - f, f), the same values the general sums below give, and the touched slots a
    // fixed pattern shifted by those halves.
    auto axis_regular = [](int o, int op, int W, int lo) { return op == o + 1 && (o == lo || (W == 3 && o == lo + 1)); };
    const bool regular = axis_regular(oi, oip, W0, L0) && axis_regular(oj, ojp, W1, L1) && axis_regular(ok, okp, W2, L2);
    if (regular) {
        const bool hx = W0 == 3 && oi == L0 + 1;
        const bool hy = W1 == 3 && oj == L1 + 1;
        const bool hz = W2 == 3 && ok == L2 + 1;
        const float f[3] = {s.fx, s.fy, s.fz};
        const bool h[3] = {hx, hy, hz};
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int W = a == 0 ? W0 : (a == 1 ? W1 : W2);
            float* w = a == 0 ? wx : (a == 1 ? wy : wz);
            const float lo = 1.f - f[a];
            if (W == 2) {
                w[0] = lo;
                w[1] = f[a];
            } else {
                w[0] = h[a] ? 0.f : lo;
                w[1] = h[a] ? lo : f[a];
                w[2 % W] = h[a] ? f[a] : 0.f;
            }
        }
        mask |= regular_mask<C>() << ((hx ? 1 : 0) + W0 * ((hy ? 1 : 0) + W1 * (hz ? 1 : 0)));
    } else {
        // 1D weights and touched bits on the window (i and ip coincide only on a one-face axis)
        uint32_t tx = 0, ty = 0, tz = 0;
#pragma unroll
        for (int r = 0; r < W0; ++r) {
            wx[r] = (oi == L0 + r ? 1.f - s.fx : 0.f) + (oip == L0 + r ? s.fx : 0.f);
            tx |= (oi == L0 + r || oip == L0 + r) ? 1u << r : 0u;
        }
#pragma unroll
        for (int r = 0; r < W1; ++r) {
            wy[r] = (oj == L1 + r ? 1.f - s.fy : 0.f) + (ojp == L1 + r ? s.fy : 0.f);
            ty |= (oj == L1 + r || ojp == L1 + r) ? 1u << r : 0u;
        }
#pragma unroll
        for (int r = 0; r < W2; ++r) {
            wz[r] = (ok == L2 + r ? 1.f - s.fz : 0.f) + (okp == L2 + r ? s.fz : 0.f);
            tz |= (ok == L2 + r || okp == L2 + r) ? 1u << r : 0u;
        }
        mask |= spread_mask<C>(tx, ty, tz);
    }
    float gx[W0];  // APIC: wx_i C_x (x_face_i - x_p)
    float dy[W1], dz[W2];
    if (SOLVER == FE_SOLVER_APIC) {
#pragma unroll
        for (int r = 0; r < W0; ++r) gx[r] = wx[r] * (q.cr[0] * ((k.org[0] + v.hf[0] * (float)(cx + L0 + r)) - q.pc[0]));
#pragma unroll
        for (int r = 0; r < W1; ++r) dy[r] = (k.org[1] + v.hf[1] * (float)(cy + L1 + r)) - q.pc[1];
#pragma unroll
        for (int r = 0; r < W2; ++r) dz[r] = (k.org[2] + v.hf[2] * (float)(cz + L2 + r)) - q.pc[2];
    }
#pragma unroll
    for (int c3 = 0; c3 < W2; ++c3)
#pragma unroll
        for (int b3 = 0; b3 < W1; ++b3) {
            const float a = wy[b3] * wz[c3];
            float val = q.vc;
            if (SOLVER == FE_SOLVER_APIC) val += q.cr[1] * dy[b3] + q.cr[2] * dz[c3];
            const float t = a * val;
#pragma unroll
            for (int a3 = 0; a3 < W0; ++a3) {
                const int slot = a3 + W0 * (b3 + W1 * c3);
                if (SOLVER == FE_SOLVER_APIC) num[slot] += wx[a3] * t + gx[a3] * a;
                else num[slot] += wx[a3] * t;
                den[slot] += wx[a3] * a;
            }
        }
    return true;
}

// Box index of slot `slot` of component C for the cell at tile-local (lx, ly, lz): the box starts one face before
// the tile.
template <int C>
__device__ __forceinline__ int slot_box(int lx, int ly, int lz, int slot)
{
    constexpr int W0 = win<C>(0), W1 = win<C>(1);
    const int a = slot % W0, b = (slot / W0) % W1, c = slot / (W0 * W1);
    return (lx + 1 + wlo<C>(0) + a) + kBox * ((ly + 1 + wlo<C>(1) + b) + kBox * (lz + 1 + wlo<C>(2) + c));
}

// Component C of the cell's particles [pb, pe) (a thread's own cell, or a warp's share of a crowded cell with
// lane stride 32) into the slots.
template <int SOLVER, int C>
__device__ __forceinline__ void cell_component(const SceneView& v, uint32_t pb, uint32_t pe, uint32_t stride, int cx,
                                               int cy, int cz, int bx, int by, int bz, const float lo[3],
                                               const float hi[3], float (&num)[nslots<C>()],
                                               float (&den)[nslots<C>()], uint32_t& mask, float* s_num, float* s_den,
                                               uint8_t* s_mk)
{
    const P2gComp k = p2g_comp<SOLVER>(v, C);
#pragma unroll
    for (int t = 0; t < nslots<C>(); ++t) num[t] = den[t] = 0.f;
    mask = 0;
    for (uint32_t p = pb; p < pe; p += stride) {
        const float x = __ldg(v.px + p), y = __ldg(v.py + p), z = __ldg(v.pz + p);  // read-only during P2G
        const Stencil s = stencil(x, y, z, k.org, v.inv_hf, k.csx, k.csy, k.csz);
        const P2gParticle<SOLVER> q = load_particle<SOLVER>(v, p, C, x, y, z, lo, hi);
        if (!splat_slots<SOLVER, C>(v, k, s, q, cx, cy, cz, num, den, mask))
            splat_direct<SOLVER>(v, k, s, q, bx, by, bz, s_num, s_den, s_mk);
    }
}

template <int SOLVER, int C>
__device__ __forceinline__ void flush_slots(int lx, int ly, int lz, const float (&num)[nslots<C>()],
                                            const float (&den)[nslots<C>()], uint32_t mask, float* s_num, float* s_den,
                                            uint8_t* s_mk)
{
#pragma unroll
    for (int t = 0; t < nslots<C>(); ++t) {
        if (!((mask >> t) & 1u)) continue;
        const int l = slot_box<C>(lx, ly, lz, t);
        atomicAdd(&s_num[l], num[t]);
        atomicAdd(&s_den[l], den[t]);
        s_mk[l] = 1;
    }
}

// A crowded cell's particles past kCellCap, spread over a warp's lanes; the lanes' slots are summed by shuffles
// and lane 0 adds them into the box.
template <int SOLVER, int C>
__device__ __forceinline__ void crowded_component(const SceneView& v, uint32_t ob, uint32_t oe, int ox, int oy, int oz,
                                                  int cx, int cy, int cz, int bx, int by, int bz, const float lo[3],
                                                  const float hi[3], float* s_num, float* s_den, uint8_t* s_mk)
{
    const int lane = threadIdx.x & 31;
    float num[nslots<C>()], den[nslots<C>()];
    uint32_t mask;
    cell_component<SOLVER, C>(v, ob + lane, oe, 32u, cx, cy, cz, bx, by, bz, lo, hi, num, den, mask, s_num, s_den,
                              s_mk);
    mask = __reduce_or_sync(0xffffffffu, mask);
#pragma unroll
    for (int q = 0; q < nslots<C>(); ++q)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            num[q] += __shfl_xor_sync(0xffffffffu, num[q], off);
            den[q] += __shfl_xor_sync(0xffffffffu, den[q], off);
        }
    if (lane == 0) flush_slots<SOLVER, C>(ox, oy, oz, num, den, mask, s_num, s_den, s_mk);
}

template <int SOLVER, int C>
__device__ __forceinline__ void own_component(const SceneView& v, uint32_t pb, uint32_t pe, int lx, int ly, int lz,
                                              int cx, int cy, int cz, int bx, int by, int bz, const float lo[3],
                                              const float hi[3], float* s_num, float* s_den, uint8_t* s_mk)
{
    float num[nslots<C>()], den[nslots<C>()];
    uint32_t mask;
    cell_component<SOLVER, C>(v, pb, pe, 1u, cx, cy, cz, bx, by, bz, lo, hi, num, den, mask, s_num, s_den, s_mk);
    flush_slots<SOLVER, C>(lx, ly, lz, num, den, mask, s_num, s_den, s_mk);
}

// The tile's face box in shared memory (declared by the kernels, so a kernel that runs several transfer kinds holds
// one box, not one per kind).
struct P2gShared {
    float num[3][kBoxFaces];
    float den[3][kBoxFaces];
    uint8_t mk[3][kBoxFaces];
    uint16_t over[FE_TILE_CELLS];  // cells with more than kCellCap particles (tile-local index)
    int nover;
};

template <int SOLVER>
__device__ __forceinline__ void p2g_body(const SceneView& v, int tile, P2gShared& sh)
{
    float (&s_num)[3][kBoxFaces] = sh.num;
    float (&s_den)[3][kBoxFaces] = sh.den;
    uint8_t (&s_mk)[3][kBoxFaces] = sh.mk;
    uint16_t* s_over = sh.over;
    int& s_nover = sh.nover;

    const int tx = tile % v.g.tnx, ty = (tile / v.g.tnx) % v.g.tny, tz = tile / (v.g.tnx * v.g.tny);
    const int bx = tx * FE_TILE - 1, by = ty * FE_TILE - 1, bz = tz * FE_TILE - 1;  // box origin (face index)
    const uint32_t beg = v.cell_start[(uint32_t)tile * FE_TILE_CELLS];
    const uint32_t end = v.cell_start[(uint32_t)(tile + 1) * FE_TILE_CELLS];
    if (beg == end) return;  // nothing to splat; accumulators were cleared by the caller

    for (int t = threadIdx.x; t < 3 * kBoxFaces; t += blockDim.x) {
        (&s_num[0][0])[t] = 0.f;
        (&s_den[0][0])[t] = 0.f;
        (&s_mk[0][0])[t] = 0;
    }
    if (threadIdx.x == 0) s_nover = 0;
    __syncthreads();

    const float lo[3] = {v.originf[0] + 0.5f * v.hf[0], v.originf[1] + 0.5f * v.hf[1], v.originf[2] + 0.5f * v.hf[2]};
    const float hi[3] = {v.originf[0] + v.sizef[0] - 0.5f * v.hf[0], v.originf[1] + v.sizef[1] - 0.5f * v.hf[1],
                         v.originf[2] + v.sizef[2] - 0.5f * v.hf[2]};

    // this thread's cell (tile-local index = key & 511 = threadIdx.x)
    const int lx = threadIdx.x & 7, ly = (threadIdx.x >> 3) & 7, lz = threadIdx.x >> 6;
    const int cx = tx * FE_TILE + lx, cy = ty * FE_TILE + ly, cz = tz * FE_TILE + lz;
    uint32_t pb = 0, pe = 0;
    if (cx < v.g.nx && cy < v.g.ny && cz < v.g.nz) {
        const uint32_t key = (uint32_t)tile * FE_TILE_CELLS + threadIdx.x;
        pb = v.cell_start[key];
        pe = v.cell_start[key + 1];
    }
    if (pe - pb > (uint32_t)kCellCap) {
        s_over[atomicAdd(&s_nover, 1)] = (uint16_t)threadIdx.x;
        pe = pb + kCellCap;
    }
    own_component<SOLVER, 0>(v, pb, pe, lx, ly, lz, cx, cy, cz, bx, by, bz, lo, hi, s_num[0], s_den[0], s_mk[0]);
    own_component<SOLVER, 1>(v, pb, pe, lx, ly, lz, cx, cy, cz, bx, by, bz, lo, hi, s_num[1], s_den[1], s_mk[1]);
    own_component<SOLVER, 2>(v, pb, pe, lx, ly, lz, cx, cy, cz, bx, by, bz, lo, hi, s_num[2], s_den[2], s_mk[2]);
    __syncthreads();

    // crowded cells: a warp per cell, lanes stride over the particles past kCellCap
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int nover = s_nover;
    for (int o = warp; o < nover; o += nwarps) {
        const int t = s_over[o];
        const int ox = t & 7, oy = (t >> 3) & 7, oz = t >> 6;
        const int ocx = tx * FE_TILE + ox, ocy = ty * FE_TILE + oy, ocz = tz * FE_TILE + oz;
        const uint32_t key = (uint32_t)tile * FE_TILE_CELLS + (uint32_t)t;
        const uint32_t ob = v.cell_start[key] + kCellCap, oe = v.cell_start[key + 1];
        crowded_component<SOLVER, 0>(v, ob, oe, ox, oy, oz, ocx, ocy, ocz, bx, by, bz, lo, hi, s_num[0], s_den[0],
                                     s_mk[0]);
        crowded_component<SOLVER, 1>(v, ob, oe, ox, oy, oz, ocx, ocy, ocz, bx, by, bz, lo, hi, s_num[1], s_den[1],
                                     s_mk[1]);
        crowded_component<SOLVER, 2>(v, ob, oe, ox, oy, oz, ocx, ocy, ocz, bx, by, bz, lo, hi, s_num[2], s_den[2],
                                     s_mk[2]);
    }
    __syncthreads();

#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const P2gComp k = p2g_comp<SOLVER>(v, c);
        for (int l = threadIdx.x; l < kBoxFaces; l += blockDim.x) {
            if (!s_mk[c][l]) continue;
            const int li = l % kBox, lj = (l / kBox) % kBox, lk = l / (kBox * kBox);
            const int gi = bx + li, gj = by + lj, gk = bz + lk;
            if (gi < 0 || gj < 0 || gk < 0 || gi >= k.fsx || gj >= k.fsy || gk >= k.fsz) continue;
            const size_t f = idx3(gi, gj, gk, k.fsx, k.fsy);
            atomicAdd(k.gnum + f, s_num[c][l]);
            atomicAdd(k.gden + f, s_den[c][l]);
            k.gmk[f] = 1;
        }
    }
}

template <int SOLVER>
__global__ void __launch_bounds__(kP2gThreads, 1) k_p2g(SceneView v)
{
    __shared__ P2gShared sh;
    p2g_body<SOLVER>(v, (int)blockIdx.x, sh);
}

// u = num / weight where weight > 0 (pic_simulator.cpp:414-436); FLIP also snapshots the result.
template <bool FLIP>
__device__ __forceinline__ float4 normalize4(float4 n, float4 d)
{
    return make_float4(d.x > 0.f ? n.x / d.x : n.x, d.y > 0.f ? n.y / d.y : n.y, d.z > 0.f ? n.z / d.z : n.z,
                       d.w > 0.f ? n.w / d.w : n.w);
}

// The three components are contiguous in every face buffer (u | v | w), so the pass runs over one flat range of
// `total` faces, four per thread with 16-byte accesses when the buffers are 16-byte aligned (they start on the
// allocator's 256-byte boundaries), else face by face.
template <bool FLIP>
__device__ __forceinline__ void normalize_body(const SceneView& v, size_t total, uint32_t blk)
{
    const size_t q = blk * (size_t)blockDim.x + threadIdx.x;
    const size_t f0 = 4 * q;
    if (f0 >= total) return;
    const bool vec = ((reinterpret_cast<uintptr_t>(v.nu) | reinterpret_cast<uintptr_t>(v.du) |
                       reinterpret_cast<uintptr_t>(v.u) | reinterpret_cast<uintptr_t>(v.su)) & 15u) == 0;
    if (vec && f0 + 4 <= total) {
        const float4 o = normalize4<FLIP>(reinterpret_cast<const float4*>(v.nu)[q],
                                          reinterpret_cast<const float4*>(v.du)[q]);
        reinterpret_cast<float4*>(v.u)[q] = o;
        if (FLIP) reinterpret_cast<float4*>(v.su)[q] = o;
        return;
    }
    for (size_t f = f0; f < f0 + 4 && f < total; ++f) {
        const float d = v.du[f];
        const float val = d > 0.f ? v.nu[f] / d : v.nu[f];
        v.u[f] = val;
        if (FLIP) v.su[f] = val;
    }
}
template <bool FLIP>
__global__ void __launch_bounds__(256) k_p2g_normalize(SceneView v, size_t total)
{
    normalize_body<FLIP>(v, total, blockIdx.x);
}

// ---- flat multi-scene forms (BatchPlan, fe_internal.cuh): every scene's tiles in one launch, each block running
// its scene's transfer kind
__global__ void __launch_bounds__(kP2gThreads, 1) k_multi_p2g(const BatchPlan* __restrict__ plan)
{
    __shared__ P2gShared sh;
    __shared__ SceneView v;
    uint32_t b;
    const int s = batch_scene_of(plan, kBkP2g, b);
    stage_view(v, plan->sc[s].dst);
    if (v.solver == FE_SOLVER_PIC) p2g_body<FE_SOLVER_PIC>(v, (int)b, sh);
    else if (v.solver == FE_SOLVER_FLIP) p2g_body<FE_SOLVER_FLIP>(v, (int)b, sh);
    else p2g_body<FE_SOLVER_APIC>(v, (int)b, sh);
}

__global__ void __launch_bounds__(256) k_multi_p2g_normalize(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkNormalize, b);
    const SceneView& v = plan->sc[s].dst;
    const size_t total = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz + (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz +
                         (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    if (v.solver == FE_SOLVER_FLIP) normalize_body<true>(v, total, b);
    else normalize_body<false>(v, total, b);
}

}  // namespace

// Every scene's splat (accumulators cleared by launch_multi_clear) and normalisation: launch_p2g's passes.
cudaError_t launch_multi_p2g(const BatchLaunch& L, cudaStream_t st)
{
    if (L.total[kBkP2g]) {
        k_multi_p2g<<<L.total[kBkP2g], kP2gThreads, 0, st>>>(L.plan);
        count_launch();
    }
    k_multi_p2g_normalize<<<L.total[kBkNormalize], 256, 0, st>>>(L.plan);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_p2g(const SceneView& v, cudaStream_t st)
{
    const size_t nu = (size_t)(v.g.nx + 1) * v.g.ny * v.g.nz, nvv = (size_t)v.g.nx * (v.g.ny + 1) * v.g.nz,
                 nww = (size_t)v.g.nx * v.g.ny * (v.g.nz + 1);
    cudaError_t e;
    // accumulators: numerator and weight arrays are laid out back to back, markers too (fe_scene.cu)
    if ((e = cudaMemsetAsync(v.nu, 0, (nu + nvv + nww) * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(v.du, 0, (nu + nvv + nww) * sizeof(float), st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(v.mu, 0, nu + nvv + nww, st)) != cudaSuccess) return e;
    const unsigned tiles = (unsigned)(v.g.tnx * v.g.tny * v.g.tnz);
    if (v.np > 0) {
        if (v.solver == FE_SOLVER_PIC) k_p2g<FE_SOLVER_PIC><<<tiles, kP2gThreads, 0, st>>>(v);
        else if (v.solver == FE_SOLVER_FLIP) k_p2g<FE_SOLVER_FLIP><<<tiles, kP2gThreads, 0, st>>>(v);
        else k_p2g<FE_SOLVER_APIC><<<tiles, kP2gThreads, 0, st>>>(v);
        count_launch();
    }
    const size_t total = nu + nvv + nww;
    const unsigned nb = (unsigned)((total + 1023) / 1024);
    if (v.solver == FE_SOLVER_FLIP) k_p2g_normalize<true><<<nb, 256, 0, st>>>(v, total);
    else k_p2g_normalize<false><<<nb, 256, 0, st>>>(v, total);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
