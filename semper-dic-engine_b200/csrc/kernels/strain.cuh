// Launch interface of the median test, VSG and packing kernels (strain.cu).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

cudaError_t launch_median_pass(int gw, int gh, const float* u, const float* v, const uint8_t* ok, uint8_t* fail,
                               int* n_fail, cudaStream_t st);
cudaError_t launch_clear_failed(int n, uint8_t* ok, const uint8_t* fail, cudaStream_t st);
cudaError_t launch_vsg(int gw, int gh, int step, int window, const float* u, const float* v, const uint8_t* valid,
                       float* exx, float* eyy, float* exy, cudaStream_t st);
size_t pack_scratch_bytes(int n);
cudaError_t launch_pack(int gw, int gh, int rect_x, int rect_y, int step, int max_pts, const uint8_t* valid,
                        const float* u, const float* v, const float* corr, const float* exx, const float* eyy,
                        const float* exy, float* out, int* n_drop, int* n_emit_total2, void* scratch,
                        size_t scratch_bytes, cudaStream_t st);

}  // namespace dic
