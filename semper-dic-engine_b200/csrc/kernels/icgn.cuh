// Launch interface of the batched subset solve (icgn.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "dic_types.h"

namespace dic {

constexpr int kSolveThreads = 128;  // unit of the `blocks` grid-size hint: 4 subsets per unit

struct SolveArgs {
    const float* refI;   // reference intensities (Ghost Wall stamped), W x H
    const float* refGx;  // reference gradients
    const float* refGy;
    const float* defI;   // deformed intensities
    int W, H;
    int pitch;           // row pitch of every plane, elements (a multiple of 4 for TMA)
    const uint8_t* pool_valid;  // Hessian pool, indexed by dic_task.node
    const float2* pool_ms;      // (mean, std)
    const double* pool_Hs;      // whole-subset step matrix, 21 doubles per node (upper triangle)
    int dim;                    // subset size (odd)
    int max_n;                  // shared-memory capacity in pixels per warp (>= dim^2)
    int lm;                     // Levenberg-Marquardt damping of the translation DOFs
    const dic_task* tasks;
    const int* n_tasks_dev;  // task count in device memory, or null to use n_tasks
    int n_tasks;
    dic_result* results;     // one per task
    int* queue;              // 3 work counters (zeroed by launch_solve)
    int* deferred;           // n_tasks slots: tasks the fast pass leaves to the general one
    const int* cancel;       // host-mapped cancel flag polled per task, or null
    int* err;                // set to 1 when a TMA wait ran out (the warp then reads global memory)
    int tma_max_polls;       // polls of a TMA completion wait before it gives up (0: kTmaPolls)
    size_t smem_per_warp;    // set by launch_solve
    int tile_w, tile_h;      // TMA box of the deformed tile, set by launch_solve (0: no tile)
    // set by launch_solve from dim and the shared-memory layout
    int half, n, min_valid;
    int off_tile, off_vals, off_valid, off_refok;
    int general_all;  // set by launch_solve: the general pass takes every task (no fast pass)
    int rescue_all;   // set by launch_solve: the rescue pass takes every task (small launches)
    int ref_no_ghost; // the caller's promise: no reference pixel is below the Ghost Wall threshold
                      // (no mask), so the fast pass skips its per-task scan for them
    int fast_stage;   // the caller's choice: the fast pass stages the reference subset (1) or reads
                      // the planes (0); the same results either way
    // Reference planes other than the deformed image's frame: the subset
    // centred at (cx, cy) is read at (cx + ref_dx, cy + ref_dy) of planes with
    // row pitch ref_pitch (0: the same planes frame, pitch). Staged solver only.
    int ref_pitch, ref_dx, ref_dy;
    // How far the warped subset's bounding box outgrows the subset (its
    // side over the subset's, e.g. |cos| + |sin| of a rotation): above 1 the
    // TMA tiles are sized for it (the fast pass then runs its generic
    // instance); 0 or 1: the tiles of an unrotated subset.
    float tile_spread;
};

struct SmemLayout {
    size_t off_h, off_tile, off_vals, off_valid, off_refok, bytes;
};
__host__ __device__ inline SmemLayout smem_layout(int max_n, int tile_w, int tile_h) {
    SmemLayout L;
    L.off_h = 64;      // barrier (8 B) at 0, tile state at 16
    L.off_tile = 640;  // 64 + 2 * 36 * 8 = 640
    L.off_vals = L.off_tile + (((size_t)tile_w * tile_h * 4 + 127) & ~(size_t)127);
    L.off_valid = L.off_vals + (size_t)max_n * 4;
    L.off_refok = L.off_valid + (size_t)max_n;
    L.bytes = (L.off_refok + (size_t)max_n + 127) & ~(size_t)127;
    return L;
}
void tile_box(int dim, int six, int& tw, int& th, float spread = 0.0f);
// Two launches on `st`: the fast pass over every task, then the general pass
// over the tasks it deferred. Scratch: queue (3 ints) and deferred (n ints).
cudaError_t launch_solve(const SolveArgs& a, int six, int grid_blocks, cudaStream_t st);

}  // namespace dic
