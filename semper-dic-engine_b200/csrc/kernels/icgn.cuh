// Launch interface of the batched subset solve (icgn.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "dic_types.h"

namespace dic {

constexpr int kSolveThreads = 128;  // 4 warps per block, one subset per warp

struct SolveArgs {
    const float* refI;   // reference intensities (Ghost Wall stamped), W x H
    const float* refGx;  // reference gradients
    const float* refGy;
    const float* defI;   // deformed intensities
    int W, H;
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
    int* queue;              // work counter, zero before the launch
    const int* cancel;       // host-mapped cancel flag polled per task, or null
    size_t smem_per_warp;    // set by launch_solve
};

size_t solve_smem_per_warp(int max_n);
cudaError_t launch_solve(const SolveArgs& a, int six, int grid_blocks, cudaStream_t st);

}  // namespace dic
