// Device bookkeeping of incremental DIC (incmask.cu): the forward warp of the
// material mask and the Ghost Wall stamp of an adopted reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

// The filled increment field over a grid (node (i, j) at rect + (i, j) * step).
struct MaskField {
    int gridW, gridH, rect_x, rect_y, step;
    const float* U;
    const float* V;
};

// Every material pixel (mask0 >= 128) of the window [X0, X1] x [Y0, Y1]
// sends per_px x per_px samples X to X + U(X) in `out` (zeroed first).
cudaError_t launch_warp_mask(const uint8_t* mask0, int W, int H, int X0, int X1, int Y0, int Y1, int per_px,
                             MaskField f, uint8_t* out, cudaStream_t st);
// 3x3 morphological close in place (tmp: W x H bytes), the border neutral.
cudaError_t launch_close3x3(uint8_t* m, uint8_t* tmp, int W, int H, cudaStream_t st);
// box = {min x, min y, max x, max y} of the nonzero pixels (set to
// {W, H, -1, -1} first by the call).
cudaError_t launch_mask_bbox(const uint8_t* m, int W, int H, int* box, cudaStream_t st);
// I := -10 where mask < 128 (the Ghost Wall), planes with row pitch `pitch`.
cudaError_t launch_stamp_ghost(float* I, int W, int H, int pitch, const uint8_t* mask, cudaStream_t st);

}  // namespace dic
