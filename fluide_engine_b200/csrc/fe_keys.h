/*
 * fe_keys.h -- particle cell keys shared bit-for-bit by the CUDA path and the CPU oracle.
 *
 * A particle's key is the index of the grid cell that holds it, in tile-major order:
 * the grid is cut into 8x8x8-cell tiles, tiles are numbered x-fastest, and the 512 cells of
 * a tile are numbered x-fastest inside it.  Sorting particles by key therefore makes every
 * tile's particles one contiguous run, which is what the shared-memory P2G splat and the
 * marking scatter rely on.
 *
 * The reference has no cell keys (its P2G scatters straight from the unsorted particle array,
 * pic_simulator.cpp:384-412); the key and its stable sort are a new design element whose oracle
 * is a stable counting sort over the same function evaluated on the CPU.  The function uses
 * only IEEE single-precision subtract and multiply (no fused multiply-add), so host and device
 * produce identical keys from identical FP32 positions.
 */
#ifndef FE_KEYS_H
#define FE_KEYS_H

#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define FE_HD __host__ __device__ __forceinline__
#else
#define FE_HD static inline
#endif

#define FE_TILE_LOG2 3
#define FE_TILE 8
#define FE_TILE_CELLS 512

/* Cell coordinate along one axis: floor((x - origin) * inv_h) clamped to [0, n-1].
 * NaN maps to 0 so a corrupted particle can never index out of bounds. */
FE_HD int fe_cell_coord(float x, float origin, float inv_h, int n)
{
#if defined(__CUDA_ARCH__)
    float t = __fmul_rn(__fsub_rn(x, origin), inv_h);
#else
    volatile float d = x - origin; /* volatile: forbid contraction / excess precision */
    float t = d * inv_h;
#endif
    if (!(t >= 0.0f)) return 0;
    if (t >= (float)n) return n - 1;
    int c = (int)floorf(t);
    return c > n - 1 ? n - 1 : c;
}

/* Number of tiles along an axis of n cells. */
FE_HD int fe_tiles(int n) { return (n + FE_TILE - 1) >> FE_TILE_LOG2; }

/* Key of cell (cx, cy, cz) for a grid of (nx, ny, nz) cells. */
FE_HD uint32_t fe_cell_key(int cx, int cy, int cz, int nx, int ny)
{
    uint32_t tnx = (uint32_t)fe_tiles(nx), tny = (uint32_t)fe_tiles(ny);
    uint32_t tile = ((uint32_t)(cz >> FE_TILE_LOG2) * tny + (uint32_t)(cy >> FE_TILE_LOG2)) * tnx
                    + (uint32_t)(cx >> FE_TILE_LOG2);
    uint32_t local = (((uint32_t)cz & 7u) << 6) | (((uint32_t)cy & 7u) << 3) | ((uint32_t)cx & 7u);
    return (tile << 9) | local;
}

/* Total key space: tiles x 512 (keys of cells outside a partial edge tile stay unused). */
FE_HD uint32_t fe_key_space(int nx, int ny, int nz)
{
    return (uint32_t)fe_tiles(nx) * (uint32_t)fe_tiles(ny) * (uint32_t)fe_tiles(nz) * FE_TILE_CELLS;
}

/* Inverse of fe_cell_key: recovers (cx, cy, cz). */
FE_HD void fe_key_cell(uint32_t key, int nx, int ny, int* cx, int* cy, int* cz)
{
    uint32_t tnx = (uint32_t)fe_tiles(nx), tny = (uint32_t)fe_tiles(ny);
    uint32_t tile = key >> 9, local = key & 511u;
    uint32_t tx = tile % tnx, ty = (tile / tnx) % tny, tz = tile / (tnx * tny);
    *cx = (int)((tx << 3) | (local & 7u));
    *cy = (int)((ty << 3) | ((local >> 3) & 7u));
    *cz = (int)((tz << 3) | (local >> 6));
}

/* Key of a particle at FP32 position (x, y, z). */
FE_HD uint32_t fe_particle_key(float x, float y, float z, const float origin[3], const float inv_h[3],
                               int nx, int ny, int nz)
{
    int cx = fe_cell_coord(x, origin[0], inv_h[0], nx);
    int cy = fe_cell_coord(y, origin[1], inv_h[1], ny);
    int cz = fe_cell_coord(z, origin[2], inv_h[2], nz);
    return fe_cell_key(cx, cy, cz, nx, ny);
}

#endif /* FE_KEYS_H */
