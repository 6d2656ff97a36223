// fe_sort.cu -- cell keys and the stable counting sort of particles by key.
//
// The reference has no sort: its P2G scatters from the unsorted particle array with racy += from
// many threads (pic_simulator.cpp:384-412).  Here particles are kept in cell-key order so that every
// 8x8x8 tile's particles form one contiguous run (fe_keys.h); P2G then splats a tile in shared memory
// and the marking scatter writes within a tile's neighbourhood.
//
// Stable counting sort, O(N + K):
//   k_keys     key of each particle, rank = atomic slot in its cell (order among equal keys arbitrary)
//   scan       exclusive prefix sum of the per-cell counts -> cell_start (K + 1 entries)
//   k_place    perm[cell_start[key] + rank] = particle (a cell's run in arbitrary order)
//   k_cellrank each particle's final slot = run start + the number of particles of its run with a smaller
//              index, so the runs end up ordered by particle index and the result is identical to a stable
//              sort by key (the oracle is a CPU stable counting sort of the same keys); O(run length) per
//              particle, all particles of a run in parallel; the particle is written at its final slot of
//              `rank`, which from then on holds the sorted order (slot -> particle) that the gather reads
//   k_bigcell  runs longer than kBigCell (particles piled into one cell, e.g. clamped into a wall corner)
//              are ordered by one block each with a bitonic network instead, so the cost stays
//              O(n log^2 n) per run rather than O(n^2)
//   k_gather   particle arrays permuted into the second buffer set
#include "fe_internal.cuh"

namespace fe {
namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

// The per-particle passes of the sort (keys, placement, ranks) give each thread kSortBatch particles, a block's
// threads stride over them (coalesced), and issue every particle's loads (and atomics) before the first use, so a
// thread keeps several round trips in flight: the passes are bound by load and atomic latency.
constexpr int kSortBatch = 4;

__device__ __forceinline__ void keys_body(const SceneView& v, uint32_t blk)
{
    const uint64_t base = (blk * (uint64_t)blockDim.x) * kSortBatch + threadIdx.x;
    float x[kSortBatch], y[kSortBatch], z[kSortBatch];
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        if (i < v.np) {
            x[b] = v.px[i];
            y[b] = v.py[i];
            z[b] = v.pz[i];
        }
    }
    uint32_t key[kSortBatch], slot[kSortBatch];
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        if (i < v.np) {
            key[b] = fe_particle_key(x[b], y[b], z[b], v.originf, v.inv_hf, v.g.nx, v.g.ny, v.g.nz);
            slot[b] = atomicAdd(v.cell_count + key[b], 1u);
        }
    }
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        if (i < v.np) {
            v.key[i] = key[b];
            v.rank[i] = slot[b];
        }
    }
}

__global__ void __launch_bounds__(256) k_keys(SceneView v) { keys_body(v, blockIdx.x); }

// Inclusive block scan of one value per thread; returns the block total through *total.
__device__ __forceinline__ uint32_t block_incl_scan(uint32_t x, uint32_t* warp_sums, uint32_t* total)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    uint32_t before = wid > 0 ? warp_sums[wid - 1] : 0u;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return x + before;
}

__device__ __forceinline__ void scan_partials_body(const uint32_t* __restrict__ in, uint32_t n,
                                                   uint32_t* __restrict__ block_sums, uint32_t blk, uint32_t* ws)
{
    uint64_t base = (uint64_t)blk * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t)
        if (base + t < n) s += in[base + t];
    uint32_t total;
    block_incl_scan(s, ws, &total);
    if (threadIdx.x == 0) block_sums[blk] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_partials(const uint32_t* __restrict__ in, uint32_t n,
                                                                  uint32_t* __restrict__ block_sums)
{
    __shared__ uint32_t ws[32];
    scan_partials_body(in, n, block_sums, blockIdx.x, ws);
}

// Exclusive scan of the block sums by a single block, looping over chunks of kScanTile.
__device__ __forceinline__ void scan_block_sums_body(uint32_t* __restrict__ sums, uint32_t nb, uint32_t* ws)
{
    uint32_t carry = 0;
    for (uint32_t chunk = 0; chunk < nb; chunk += kScanTile) {
        uint32_t base = chunk + threadIdx.x * kScanItems;
        uint32_t vals[kScanItems];
        uint32_t s = 0;
#pragma unroll
        for (int t = 0; t < kScanItems; ++t) {
            vals[t] = base + t < nb ? sums[base + t] : 0u;
            s += vals[t];
        }
        uint32_t total;
        uint32_t incl = block_incl_scan(s, ws, &total);
        uint32_t run = carry + incl - s;
#pragma unroll
        for (int t = 0; t < kScanItems; ++t) {
            if (base + t < nb) sums[base + t] = run;
            run += vals[t];
        }
        carry += total;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_block_sums(uint32_t* __restrict__ sums, uint32_t nb)
{
    __shared__ uint32_t ws[32];
    scan_block_sums_body(sums, nb, ws);
}

__device__ __forceinline__ void scan_final_body(const uint32_t* __restrict__ in, uint32_t n,
                                                const uint32_t* __restrict__ block_off, uint32_t* __restrict__ out,
                                                uint32_t blk, uint32_t* ws)
{
    uint64_t base = (uint64_t)blk * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    uint32_t vals[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        vals[t] = base + t < n ? in[base + t] : 0u;
        s += vals[t];
    }
    uint32_t total;
    uint32_t incl = block_incl_scan(s, ws, &total);
    uint32_t run = block_off[blk] + incl - s;
#pragma unroll
    for (int t = 0; t < kScanItems; ++t) {
        if (base + t < n) out[base + t] = run;
        run += vals[t];
    }
    if (base + kScanItems >= n && base < n) out[n] = run;  // the thread holding the last element writes the total
}

__global__ void __launch_bounds__(kScanThreads) k_scan_final(const uint32_t* __restrict__ in, uint32_t n,
                                                               const uint32_t* __restrict__ block_off,
                                                               uint32_t* __restrict__ out)
{
    __shared__ uint32_t ws[32];
    scan_final_body(in, n, block_off, out, blockIdx.x, ws);
}

// After the scan the per-cell counts are dead until the next sort, so cell_count doubles as the list of
// long runs (their keys, at most key_space of them); how many there are is counted in the word after the
// scan's block sums (scan scratch holds nb + 2 words).
constexpr uint32_t kBigCell = 1024;
constexpr int kBigCellBlocks = 32;

__device__ __forceinline__ void place_body(const SceneView& v, uint32_t* __restrict__ long_count, uint32_t blk)
{
    const uint64_t base = (blk * (uint64_t)blockDim.x) * kSortBatch + threadIdx.x;
    if (base == 0) *long_count = 0u;  // the long-run list starts empty
    uint32_t key[kSortBatch], slot[kSortBatch], start[kSortBatch];
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        if (i < v.np) {
            key[b] = v.key[i];
            slot[b] = v.rank[i];
        }
    }
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b)
        if (base + (uint64_t)b * blockDim.x < v.np) start[b] = v.cell_start[key[b]];
#pragma unroll
    for (int b = 0; b < kSortBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        if (i < v.np) v.perm[start[b] + slot[b]] = (uint32_t)i;
    }
}

__global__ void __launch_bounds__(256) k_place(SceneView v, uint32_t* __restrict__ long_count)
{
    place_body(v, long_count, blockIdx.x);
}

// rank[final slot of particle x] = x (rank's atomic slots were consumed by k_place; perm, the runs in arbitrary
// order, key and cell_start are only read here, through the read-only path).
__device__ __forceinline__ void cellrank_body(const SceneView& v, uint32_t* __restrict__ long_count, uint32_t blk)
{
    const uint64_t base = (blk * (uint64_t)blockDim.x) * kSortBatch + threadIdx.x;
    const uint32_t* __restrict__ perm = v.perm;
    uint32_t x[kSortBatch], key[kSortBatch], rb[kSortBatch], re[kSortBatch];
#pragma unroll
    for (int q = 0; q < kSortBatch; ++q)
        if (base + (uint64_t)q * blockDim.x < v.np) x[q] = __ldg(perm + base + (uint64_t)q * blockDim.x);
#pragma unroll
    for (int q = 0; q < kSortBatch; ++q)
        if (base + (uint64_t)q * blockDim.x < v.np) key[q] = __ldg(v.key + x[q]);
#pragma unroll
    for (int q = 0; q < kSortBatch; ++q)
        if (base + (uint64_t)q * blockDim.x < v.np) {
            rb[q] = __ldg(v.cell_start + key[q]);
            re[q] = __ldg(v.cell_start + key[q] + 1);
        }
#pragma unroll
    for (int q = 0; q < kSortBatch; ++q) {
        const uint64_t s = base + (uint64_t)q * blockDim.x;
        if (s >= v.np) continue;
        const uint32_t b = rb[q], e = re[q];
        if (e - b > kBigCell) {
            if (s == b) v.cell_count[atomicAdd(long_count, 1u)] = key[q];
            continue;
        }
        uint32_t r = 0;
        for (uint32_t t = b; t < e; ++t) r += __ldg(perm + t) < x[q] ? 1u : 0u;
        v.rank[b + r] = x[q];
    }
}

__global__ void __launch_bounds__(256) k_cellrank(SceneView v, uint32_t* __restrict__ long_count)
{
    cellrank_body(v, long_count, blockIdx.x);
}

// One block per listed long run.  Ascending-only bitonic network (each merge of size k starts with the
// mirrored comparator i <-> i ^ (k - 1), then half-cleaners of distance k/4 .. 1) over the run padded to
// a power of two; padded positions count as +infinity, so a pair whose upper element is past the run's
// end never swaps and is skipped.  Sorted in place in perm, then copied to the run's slots of rank.
__device__ __forceinline__ void bigcell_body(const SceneView& v, const uint32_t* __restrict__ long_count, uint32_t blk,
                                             uint32_t nblk)
{
    const uint32_t count = *long_count;
    for (uint32_t li = blk; li < count; li += nblk) {
        const uint32_t key = v.cell_count[li];
        const uint32_t b = v.cell_start[key], n = v.cell_start[key + 1] - b;
        uint32_t* a = v.perm + b;
        uint32_t P = 1;
        while (P < n) P <<= 1;
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < (P >> 1); i += blockDim.x) {
                    const uint32_t lo = (i / j) * 2u * j + (i % j);
                    const uint32_t hi = j == (k >> 1) ? lo ^ (k - 1u) : lo + j;  // mirrored first, then half-cleaners
                    if (hi < n) {
                        const uint32_t x = a[lo], y = a[hi];
                        if (x > y) {
                            a[lo] = y;
                            a[hi] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t t = threadIdx.x; t < n; t += blockDim.x) v.rank[b + t] = a[t];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(1024) k_bigcell(SceneView v, const uint32_t* __restrict__ long_count)
{
    bigcell_body(v, long_count, blockIdx.x, gridDim.x);
}

// Each thread moves kGatherBatch particles, all their loads issued before any store, so a thread keeps several
// rows of requests in flight instead of one.  The source set is read-only during the pass (the two particle buffer
// sets never alias), so its loads go through the read-only path and may be scheduled ahead of the stores.
constexpr int kGatherBatch = 4;

template <bool APIC>
__device__ __forceinline__ void gather_body(const SceneView& src, const SceneView& dst, uint32_t blk)
{
    const uint64_t base = (blk * (uint64_t)blockDim.x) * kGatherBatch + threadIdx.x;
    uint32_t j[kGatherBatch];
    bool ok[kGatherBatch];
#pragma unroll
    for (int b = 0; b < kGatherBatch; ++b) {
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        ok[b] = i < src.np;
        j[b] = ok[b] ? __ldg(src.rank + i) : 0u;  // the sorted order (slot -> particle)
    }
    float a[kGatherBatch][6];
    uint32_t id[kGatherBatch];
#pragma unroll
    for (int b = 0; b < kGatherBatch; ++b) {
        if (!ok[b]) continue;
        a[b][0] = __ldg(src.px + j[b]);
        a[b][1] = __ldg(src.py + j[b]);
        a[b][2] = __ldg(src.pz + j[b]);
        a[b][3] = __ldg(src.vx + j[b]);
        a[b][4] = __ldg(src.vy + j[b]);
        a[b][5] = __ldg(src.vz + j[b]);
        id[b] = __ldg(src.pid + j[b]);
    }
#pragma unroll
    for (int b = 0; b < kGatherBatch; ++b) {
        if (!ok[b]) continue;
        const uint64_t i = base + (uint64_t)b * blockDim.x;
        dst.px[i] = a[b][0];
        dst.py[i] = a[b][1];
        dst.pz[i] = a[b][2];
        dst.vx[i] = a[b][3];
        dst.vy[i] = a[b][4];
        dst.vz[i] = a[b][5];
        dst.pid[i] = id[b];
    }
    if (APIC) {
#pragma unroll
        for (int c = 0; c < 9; ++c) {
            float t[kGatherBatch];
#pragma unroll
            for (int b = 0; b < kGatherBatch; ++b) t[b] = ok[b] ? __ldg(src.c[c] + j[b]) : 0.f;
#pragma unroll
            for (int b = 0; b < kGatherBatch; ++b)
                if (ok[b]) dst.c[c][base + (uint64_t)b * blockDim.x] = t[b];
        }
    }
}

template <bool APIC>
__global__ void __launch_bounds__(256) k_gather(SceneView src, SceneView dst)
{
    gather_body<APIC>(src, dst, blockIdx.x);
}

// ---- flat multi-scene forms: one launch per pass for every scene of a batch (BatchPlan, fe_internal.cuh)

__global__ void __launch_bounds__(256) k_multi_keys(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkGather, b);
    keys_body(plan->sc[s].src, b);
}

template <int PASS>  // 0: partial sums, 2: final
__global__ void __launch_bounds__(kScanThreads) k_multi_scan(const BatchPlan* __restrict__ plan)
{
    __shared__ uint32_t ws[32];
    uint32_t b;
    const int s = batch_scene_of(plan, kBkScan, b);
    const BatchScene& e = plan->sc[s];
    if (PASS == 0) scan_partials_body(e.src.cell_count, e.src.g.key_space, e.scan_sums, b, ws);
    else scan_final_body(e.src.cell_count, e.src.g.key_space, e.scan_sums, e.src.cell_start, b, ws);
}

__global__ void __launch_bounds__(kScanThreads) k_multi_scan_sums(const BatchPlan* __restrict__ plan)
{
    __shared__ uint32_t ws[32];
    uint32_t b;
    const int s = batch_scene_of(plan, kBkScanSums, b);
    scan_block_sums_body(plan->sc[s].scan_sums, plan->sc[s].scan_blocks, ws);
}

__global__ void __launch_bounds__(256) k_multi_place(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkGather, b);
    place_body(plan->sc[s].src, plan->sc[s].long_count, b);
}

__global__ void __launch_bounds__(256) k_multi_cellrank(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkGather, b);
    cellrank_body(plan->sc[s].src, plan->sc[s].long_count, b);
}

__global__ void __launch_bounds__(1024) k_multi_bigcell(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkBigcell, b);
    bigcell_body(plan->sc[s].src, plan->sc[s].long_count, b, plan->start[kBkBigcell][s + 1] - plan->start[kBkBigcell][s]);
}

__global__ void __launch_bounds__(256) k_multi_gather(const BatchPlan* __restrict__ plan)
{
    uint32_t b;
    const int s = batch_scene_of(plan, kBkGather, b);
    const BatchScene& e = plan->sc[s];
    if (e.src.solver == FE_SOLVER_APIC) gather_body<true>(e.src, e.dst, b);
    else gather_body<false>(e.src, e.dst, b);
}

}  // namespace

// block sums (nb words), one spare, and the long-run counter
size_t sort_scan_tmp_bytes(uint32_t n) { return ((n + kScanTile - 1) / kScanTile + 2) * sizeof(uint32_t); }

cudaError_t launch_exclusive_scan(const uint32_t* in, uint32_t n, uint32_t* out, void* tmp, size_t tmp_bytes,
                                  cudaStream_t st)
{
    if (n == 0) return cudaMemsetAsync(out, 0, sizeof(uint32_t), st);
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (sort_scan_tmp_bytes(n) > tmp_bytes) return cudaErrorInvalidValue;
    uint32_t* sums = (uint32_t*)tmp;
    k_scan_partials<<<nb, kScanThreads, 0, st>>>(in, n, sums);
    k_scan_block_sums<<<1, kScanThreads, 0, st>>>(sums, nb);
    k_scan_final<<<nb, kScanThreads, 0, st>>>(in, n, sums, out);
    count_launch(3);
    return cudaGetLastError();
}

cudaError_t launch_sort(const SceneView& v, cudaStream_t st, void* scan_tmp, size_t scan_tmp_bytes)
{
    const uint32_t K = v.g.key_space;
    cudaError_t e = cudaMemsetAsync(v.cell_count, 0, (size_t)K * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const int T = 256;
    const unsigned pb = (unsigned)((v.np + (uint64_t)T * kSortBatch - 1) / ((uint64_t)T * kSortBatch));
    if (v.np > 0) {
        k_keys<<<pb, T, 0, st>>>(v);
        count_launch();
    }
    uint32_t nb = (K + kScanTile - 1) / kScanTile;
    if (sort_scan_tmp_bytes(K) > scan_tmp_bytes) return cudaErrorInvalidValue;
    uint32_t* sums = (uint32_t*)scan_tmp;
    k_scan_partials<<<nb, kScanThreads, 0, st>>>(v.cell_count, K, sums);
    k_scan_block_sums<<<1, kScanThreads, 0, st>>>(sums, nb);
    k_scan_final<<<nb, kScanThreads, 0, st>>>(v.cell_count, K, sums, v.cell_start);
    count_launch(3);
    if (v.np > 0) {
        uint32_t* long_count = sums + nb + 1;
        k_place<<<pb, T, 0, st>>>(v, long_count);
        k_cellrank<<<pb, T, 0, st>>>(v, long_count);
        k_bigcell<<<kBigCellBlocks, 1024, 0, st>>>(v, long_count);
        count_launch(3);
    }
    return cudaGetLastError();
}

// Blocks of the sort's passes in a batch: kBkBigcell gets a few blocks per scene (long runs are rare).
constexpr uint32_t kMultiBigCellBlocks = 4;

uint32_t sort_batch_blocks(const SceneView& v, int kind)
{
    switch (kind) {
    case kBkGather: return (uint32_t)((v.np + 256 * kGatherBatch - 1) / (256 * kGatherBatch));
    case kBkScan: return (v.g.key_space + kScanTile - 1) / kScanTile;
    case kBkScanSums: return 1;
    case kBkBigcell: return v.np > 0 ? kMultiBigCellBlocks : 0;
    default: return 0;
    }
}

// The sort of every scene: keys, the scan of the cell counts (cleared by launch_multi_clear), placement, ranks and
// long runs, then the gather into the scenes' other buffer sets -- the passes of launch_sort + launch_gather.
cudaError_t launch_multi_sort(const BatchLaunch& L, cudaStream_t st)
{
    const BatchPlan* p = L.plan;
    if (L.total[kBkPart]) k_multi_keys<<<L.total[kBkGather], 256, 0, st>>>(p);
    k_multi_scan<0><<<L.total[kBkScan], kScanThreads, 0, st>>>(p);
    k_multi_scan_sums<<<L.total[kBkScanSums], kScanThreads, 0, st>>>(p);
    k_multi_scan<2><<<L.total[kBkScan], kScanThreads, 0, st>>>(p);
    count_launch(4);
    if (L.total[kBkPart]) {
        k_multi_place<<<L.total[kBkGather], 256, 0, st>>>(p);
        k_multi_cellrank<<<L.total[kBkGather], 256, 0, st>>>(p);
        k_multi_bigcell<<<L.total[kBkBigcell], 1024, 0, st>>>(p);
        k_multi_gather<<<L.total[kBkGather], 256, 0, st>>>(p);
        count_launch(4);
    }
    return cudaGetLastError();
}

cudaError_t launch_gather(const SceneView& v, const SceneView& dst, cudaStream_t st)
{
    if (v.np == 0) return cudaSuccess;
    const int T = 256;
    const unsigned nb = (unsigned)((v.np + (uint64_t)T * kGatherBatch - 1) / ((uint64_t)T * kGatherBatch));
    if (v.solver == FE_SOLVER_APIC) k_gather<true><<<nb, T, 0, st>>>(v, dst);
    else k_gather<false><<<nb, T, 0, st>>>(v, dst);
    count_launch();
    return cudaGetLastError();
}

}  // namespace fe
