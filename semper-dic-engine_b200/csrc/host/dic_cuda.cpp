// extern "C" kernel-level entry points (include/semper_dic_cuda.h): thin
// wrappers over the launchers in ../kernels.
#include "../../../include/semper_dic_cuda.h"

#include <cuda_runtime.h>

#include "../kernels/icgn.cuh"
#include "../kernels/prep.cuh"
#include "../kernels/strain.cuh"

#define DIC_API extern "C" __attribute__((visibility("default")))

namespace {
cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }
}

DIC_API int dic_cuda_image_prep(const uint8_t* d_px, const uint8_t* d_mask, int width, int height, int pitch,
                                float* d_I, float* d_gx, float* d_gy, void* stream) {
    return (int)dic::launch_image_prep(d_px, d_mask, width, height, pitch, d_I, d_gx, d_gy, S(stream));
}

DIC_API int dic_cuda_grid_scan(const uint8_t* d_mask, int width, int height, int grid_w, int grid_h, int rect_x,
                               int rect_y, int step, int subset, uint8_t* d_skip, int* d_n_valid, void* stream) {
    return (int)dic::launch_grid_scan(d_mask, width, height, grid_w, grid_h, rect_x, rect_y, step, subset, d_skip,
                                      d_n_valid, S(stream));
}

DIC_API int dic_cuda_hessian_pool(const float* d_I, const float* d_gx, const float* d_gy, int width, int height,
                                  int pitch, const uint8_t* d_skip, int grid_w, int grid_h, int rect_x, int rect_y, int step,
                                  int subset, int lm, uint8_t* d_valid, float* d_mean_std, double* d_H21,
                                  double* d_Hs21, void* stream) {
    return (int)dic::launch_pool(d_I, d_gx, d_gy, width, height, pitch, d_skip, grid_w, grid_h, rect_x, rect_y, step, subset,
                                 lm, d_valid, reinterpret_cast<float2*>(d_mean_std), d_H21, d_Hs21, S(stream));
}

DIC_API int dic_cuda_solve(const float* d_ref_I, const float* d_ref_gx, const float* d_ref_gy, const float* d_def_I,
                           int width, int height, int pitch, const uint8_t* d_pool_valid, const float* d_pool_mean_std,
                           const double* d_pool_Hs21, int subset, int lm, int six, const dic_task* d_tasks,
                           int n_tasks, dic_result* d_results, void* d_scratch, int blocks, void* stream) {
    if (n_tasks <= 0) return 0;
    dic::SolveArgs a{};
    a.refI = d_ref_I;
    a.refGx = d_ref_gx;
    a.refGy = d_ref_gy;
    a.defI = d_def_I;
    a.W = width;
    a.H = height;
    a.pitch = pitch;
    a.err = nullptr;
    a.pool_valid = d_pool_valid;
    a.pool_ms = reinterpret_cast<const float2*>(d_pool_mean_std);
    a.pool_Hs = d_pool_Hs21;
    a.dim = subset;
    a.max_n = subset * subset;
    a.lm = lm;
    a.tasks = d_tasks;
    a.n_tasks = n_tasks;
    a.results = d_results;
    a.queue = reinterpret_cast<int*>(d_scratch);
    a.deferred = reinterpret_cast<int*>(d_scratch) + 4;
    if (blocks <= 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int need = (n_tasks + dic::kSolveThreads / 32 - 1) / (dic::kSolveThreads / 32);
        blocks = need < sms * 4 ? need : sms * 4;
    }
    return (int)dic::launch_solve(a, six, blocks, S(stream));
}

DIC_API size_t dic_cuda_solve_scratch_bytes(int n_tasks) { return (size_t)(4 + (n_tasks > 0 ? n_tasks : 0)) * 4; }

DIC_API int dic_cuda_median_pass(int grid_w, int grid_h, const float* d_u, const float* d_v, const uint8_t* d_ok,
                                 uint8_t* d_fail, int* d_n_fail, void* stream) {
    return (int)dic::launch_median_pass(grid_w, grid_h, d_u, d_v, d_ok, d_fail, d_n_fail, S(stream));
}

DIC_API int dic_cuda_clear_failed(int n, uint8_t* d_ok, const uint8_t* d_fail, void* stream) {
    return (int)dic::launch_clear_failed(n, d_ok, d_fail, S(stream));
}

DIC_API int dic_cuda_vsg(int grid_w, int grid_h, int step, int window, const float* d_u, const float* d_v,
                         const uint8_t* d_valid, float* d_exx, float* d_eyy, float* d_exy, void* stream) {
    return (int)dic::launch_vsg(grid_w, grid_h, step, window, d_u, d_v, d_valid, d_exx, d_eyy, d_exy, S(stream));
}

DIC_API size_t dic_cuda_pack_scratch_bytes(int n) { return dic::pack_scratch_bytes(n); }

DIC_API int dic_cuda_pack(int grid_w, int grid_h, int rect_x, int rect_y, int step, int max_points,
                          const uint8_t* d_valid, const float* d_u, const float* d_v, const float* d_corr,
                          const float* d_exx, const float* d_eyy, const float* d_exy, float* d_out, int* d_counts,
                          void* d_scratch, size_t scratch_bytes, void* stream) {
    return (int)dic::launch_pack(grid_w, grid_h, rect_x, rect_y, step, max_points, d_valid, d_u, d_v, d_corr, d_exx,
                                 d_eyy, d_exy, d_out, d_counts, d_counts + 1, d_scratch, scratch_bytes, S(stream));
}
