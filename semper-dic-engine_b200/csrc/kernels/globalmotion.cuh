// Global motion between a reference and a deformed frame on the device: a
// rotation, an isotropic scale and a translation of the ROI, by phase
// correlation (Fourier-Mellin for the rotation and scale). It stands in for
// the AKAZE + RANSAC global model of the anchor seeding
// (src/pipeline/akaze_features.cpp, full_field_anchors.cpp:301-313).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

struct GlobalSimilarity {
    bool locked = false;     // both correlation peaks passed their gates
    double theta = 0.0;      // rotation, rad (x' = C + s R(theta) (X - C) + T)
    double scale = 1.0;
    double tx = 0.0, ty = 0.0;   // T, px
    double cx = 0.0, cy = 0.0;   // C, px: the ROI centre the rotation is about
    double peak_rotation = 0.0;  // height of the log-polar correlation peak
    double peak_translation = 0.0;
    double H[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // reference -> deformed, row-major
    int kernels = 0;             // kernels the estimate launched
};

class GlobalMotion {
public:
    GlobalMotion();
    ~GlobalMotion();
    GlobalMotion(const GlobalMotion&) = delete;
    GlobalMotion& operator=(const GlobalMotion&) = delete;
    // d_ref, d_def: W x H gray bytes on the device; the ROI rect in pixels.
    cudaError_t estimate(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int rx, int ry, int rw, int rh,
                         cudaStream_t st, GlobalSimilarity& out);
    static constexpr int kN = 512;  // FFT size of the downsampled ROI and of the log-polar map

private:
    cudaError_t estimate_impl(const uint8_t* d_ref, const uint8_t* d_def, int W, int rx, int ry, int rw, int rh,
                              cudaStream_t st, GlobalSimilarity& out);
    struct Impl;
    Impl* impl_ = nullptr;
};

}  // namespace dic
