/*
 * semper_dic_cuda.h — the kernel-level C ABI of libsemper_c.so: one entry per
 * device stage of the full-field solve, on device pointers the caller owns.
 * The engine behind semper_c.h is built from these stages; they are exported
 * so that each stage can be driven and checked on its own (the parity tests
 * do, against the CPU restatement) and embedded in other pipelines.
 *
 * Conventions: every pointer named d_* is device memory; images are
 * row-major, width-fastest; float planes have a row pitch (elements) that is
 * a multiple of 4 (16-byte rows, which the TMA tile loads need), input bytes
 * are tight (pitch = width); `stream` is a cudaStream_t (NULL = default
 * stream). Each call enqueues work and returns 0, or a cudaError_t value if a
 * launch failed. Nothing here allocates or synchronises unless stated.
 */
#ifndef SEMPER_DIC_CUDA_H
#define SEMPER_DIC_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "../semper-dic-engine_b200/csrc/kernels/dic_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Image::Image + prepare_data(false) (src/math/image_processor.cpp:9-24, 54-63)
   and, with d_mask, stamp_ghost_wall (src/pipeline/reference_cache.cpp:18-35):
   u8 -> f32 intensity, 4th-order central-difference gradients, -10 where the
   mask is below 128. */
int dic_cuda_image_prep(const uint8_t* d_px, const uint8_t* d_mask, int width, int height, int pitch,
                        float* d_I, float* d_gx, float* d_gy, void* stream);

/* The grid validity scan of run_full_field_impl
   (src/pipeline/full_field_solver.cpp:266-318): d_skip[node] = 1 within
   subset/2 + 19 px of the border or with a masked subset pixel; *d_n_valid is
   incremented once per kept node (zero it first). */
int dic_cuda_grid_scan(const uint8_t* d_mask, int width, int height, int grid_w, int grid_h, int rect_x,
                       int rect_y, int step, int subset, uint8_t* d_skip, int* d_n_valid, void* stream);

/* The Hessian pre-pass: SubsetPrecomputer::compute_hessian_only
   (src/math/subset_precomputer.cpp:42-149) per grid node, FP64 Hessian, plus
   the whole-subset IC-GN step matrix (optimization_engine.cpp:302-315; LM
   damping of the translation DOFs when lm != 0). Outputs per node: valid
   flag, (mean, std) as two floats, the Hessian and the step matrix as 21
   doubles each (upper triangle, row-major; d_H21 may be NULL). */
int dic_cuda_hessian_pool(const float* d_I, const float* d_gx, const float* d_gy, int width, int height,
                          int pitch, const uint8_t* d_skip, int grid_w, int grid_h, int rect_x, int rect_y, int step,
                          int subset, int lm, uint8_t* d_valid, float* d_mean_std, double* d_H21,
                          double* d_Hs21, void* stream);

/* A batch of subset solves, one per dic_task: solve_node
   (src/pipeline/full_field_solver.cpp:119-139) -> calculate_deformation
   (src/math/optimization_engine.cpp:55-118) with IC-GN (:272-465), the
   Simplex rescue (:531-651) and the coarse search (:120-179) as the task's
   mode asks, then the Ghost Wall rejection. Pool arrays are indexed by
   dic_task.node. Two passes run on the stream: the common case (whole-subset
   iterations, no Simplex) for every task, then every path for the tasks the
   first pass handed on. d_scratch holds their work counters and list
   (dic_cuda_solve_scratch_bytes); its contents need no initialisation.
   `blocks` = persistent grid size (0 = one wave). */
int dic_cuda_solve(const float* d_ref_I, const float* d_ref_gx, const float* d_ref_gy, const float* d_def_I,
                   int width, int height, int pitch, const uint8_t* d_pool_valid, const float* d_pool_mean_std,
                   const double* d_pool_Hs21, int subset, int lm, int six, const dic_task* d_tasks, int n_tasks,
                   dic_result* d_results, void* d_scratch, int blocks, void* stream);

/* Bytes of scratch dic_cuda_solve needs for n_tasks tasks. */
size_t dic_cuda_solve_scratch_bytes(int n_tasks);

/* No counterpart in the reference: an addition of this library for callers
   that cannot allocate device memory (a plugin living in a host
   application's memory pool, a process under a fixed device-memory budget,
   code that must not call cudaMalloc mid-run). Same solve, arguments and
   results as dic_cuda_solve, without d_scratch: the scratch is a fixed array
   in the library's device image, so the call allocates nothing. The array
   takes 4 MiB on a GPU once the library's device code is loaded there (with
   CUDA's default lazy module loading, at the first use on that device) and
   is held until exit.
   - n_tasks above DIC_CUDA_SOLVE_NOALLOC_MAX_TASKS returns
     cudaErrorInvalidValue (1) and launches nothing.
   - The first call on a device looks up the array's device address with that
     device current and keeps it for later calls; make that first call before
     any stream capture. The kept address does not survive a reset of the
     device's primary context (cudaDeviceReset): do not use this entry across
     one.
   - Every call shares the one array (the counters are zeroed on `stream` at
     the start of each call): calls whose work overlaps on the GPU, on
     different streams or from different threads, race and must be
     serialised by the caller. */
#define DIC_CUDA_SOLVE_NOALLOC_MAX_TASKS 1048576
int dic_cuda_solve_noalloc(const float* d_ref_I, const float* d_ref_gx, const float* d_ref_gy, const float* d_def_I,
                           int width, int height, int pitch, const uint8_t* d_pool_valid,
                           const float* d_pool_mean_std, const double* d_pool_Hs21, int subset, int lm, int six,
                           const dic_task* d_tasks, int n_tasks, dic_result* d_results, int blocks, void* stream);

/* One pass of StrainCalculator::reject_displacement_outliers
   (src/strain/strain_calculator.cpp:174-224): d_fail from the flags d_ok of
   finished passes; *d_n_fail += failures (zero it first). */
int dic_cuda_median_pass(int grid_w, int grid_h, const float* d_u, const float* d_v, const uint8_t* d_ok,
                         uint8_t* d_fail, int* d_n_fail, void* stream);

/* d_ok[i] = 0 where d_fail[i] (the end of a median-test pass). */
int dic_cuda_clear_failed(int n, uint8_t* d_ok, const uint8_t* d_fail, void* stream);

/* StrainCalculator::compute_vsg_strain (strain_calculator.cpp:27-158), FP64
   normal equations; -1000 where the fit is refused. */
int dic_cuda_vsg(int grid_w, int grid_h, int step, int window, const float* d_u, const float* d_v,
                 const uint8_t* d_valid, float* d_exx, float* d_eyy, float* d_exy, void* stream);

/* Bytes of scratch dic_cuda_pack needs for a grid of n nodes. */
size_t dic_cuda_pack_scratch_bytes(int n);

/* pack_full_field_output (src/pipeline/full_field_solver_stats.cpp:21-91):
   row-major [x y u v exx eyy exy corr] of the first max_points valid nodes
   whose strain was fitted. d_counts[0] += strain drops before the capacity
   cut; d_counts[1] + d_counts[2] = all nodes that would emit (zero d_counts
   first). */
int dic_cuda_pack(int grid_w, int grid_h, int rect_x, int rect_y, int step, int max_points, const uint8_t* d_valid,
                  const float* d_u, const float* d_v, const float* d_corr, const float* d_exx, const float* d_eyy,
                  const float* d_exy, float* d_out, int* d_counts, void* d_scratch, size_t scratch_bytes,
                  void* stream);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SEMPER_DIC_CUDA_H */
