// fe_batch.cuh -- device-side description of a batch of scenes for the batched pressure solve.
#pragma once

#include "fe_internal.cuh"

namespace fe {

constexpr int kBatchMaxScenes = 64;

// One scene as the batched solver sees it: its grid, cell marks, FP64 pressure / rhs, FP32 CG vectors,
// solver settings and statistics ring (all owned by the scene).
struct BatchScene {
    int nx, ny, nz;
    double ih2d[3];
    float ih2[3];
    const uint8_t* marks;
    double *p, *b;
    float *r0, *r1, *w0, *w1, *s0, *s1, *pv, *x;
    fe_step_stats* stats_ring;
    unsigned* stats_counter;
};

struct BatchWork {
    const BatchScene* scenes;   // [S]
    const long long* cell_offset;  // [S + 1] prefix of the scenes' cell counts
    uint32_t* list;             // compacted FLUID entries (cell << 6 | mask), all scenes
    uint8_t* list_scene;        // scene of each entry
    unsigned* block_count;      // [2 * blocks]
    double* totals;             // [3][kBatchMaxScenes][2] rotating barrier totals
    unsigned* bar;              // packed count / generation
    int* err;
    int blocks;
};

cudaError_t batch_cg_blocks(int device, int* blocks);
cudaError_t launch_batch_cg(const BatchWork& w, int S, double rel_tol, double inner_tol, int max_it, int max_refine,
                            cudaStream_t st);

}  // namespace fe
