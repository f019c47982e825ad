// Launch interface of the image pass, grid scan and Hessian pool (prep.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

cudaError_t launch_image_prep(const uint8_t* px, const uint8_t* mask, int W, int H, int pitch, float* I, float* gx,
                              float* gy, cudaStream_t st);
cudaError_t launch_grid_scan(const uint8_t* mask, int W, int H, int gridW, int gridH, int rect_x, int rect_y,
                             int step, int dim, uint8_t* skip, int* n_valid, cudaStream_t st);
cudaError_t launch_pool(const float* I, const float* gx, const float* gy, int W, int H, int pitch, const uint8_t* skip,
                        int gridW, int gridH, int rect_x, int rect_y, int step, int dim, int lm, uint8_t* valid,
                        float2* ms, double* H21, double* Hs21, cudaStream_t st);

}  // namespace dic
