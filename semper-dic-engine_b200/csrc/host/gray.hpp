// Raw-image conversions at the boundary, as the reference's decoding does
// them with OpenCV (src/io/image_codec.cpp:141-152, cvtColor RGBA2GRAY;
// src/pipeline/full_field_solver.cpp:191-194, resize INTER_NEAREST).
//
// Both are written from their definitions and were checked against OpenCV's
// outputs (Python cv2 4.13): the gray conversion on all 2^24 RGB triples, the
// resize on 2000 random source and target sizes.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace semper_b200 {

// BT.601 luma of an RGBA pixel in 15-bit fixed point: the weights 0.299,
// 0.587 and 0.114 scaled by 2^15 and rounded (9798, 19235), the blue weight
// taking the remainder so that the three sum to exactly 2^15 (3735); the sum
// rounded to nearest by adding half before the shift. Alpha is ignored.
inline uint8_t rgba_luma(const uint8_t* px) {
    const uint32_t y = 9798u * px[0] + 19235u * px[1] + 3735u * px[2] + (1u << 14);
    return (uint8_t)(y >> 15);
}

inline void rgba_to_gray(const uint8_t* rgba, size_t pixels, uint8_t* gray) {
    for (size_t i = 0; i < pixels; ++i) gray[i] = rgba_luma(rgba + 4 * i);
}

// Nearest-neighbour resize of an 8-bit plane (row stride sstride bytes) to
// dw x dh: target pixel x takes source column floor(x * s) with
// s = 1 / (dw / sw) evaluated in double, clamped to the last column (rows
// likewise).
inline void resize_nearest(const uint8_t* src, int sw, int sh, size_t sstride, int dw, int dh,
                           std::vector<uint8_t>& dst) {
    dst.resize((size_t)dw * dh);
    const double sx = 1.0 / ((double)dw / (double)sw), sy = 1.0 / ((double)dh / (double)sh);
    std::vector<int> cols((size_t)dw);
    for (int x = 0; x < dw; ++x) {
        const int c = (int)std::floor((double)x * sx);
        cols[(size_t)x] = c < sw - 1 ? c : sw - 1;
    }
    for (int y = 0; y < dh; ++y) {
        int r = (int)std::floor((double)y * sy);
        if (r > sh - 1) r = sh - 1;
        const uint8_t* row = src + (size_t)r * sstride;
        uint8_t* out = dst.data() + (size_t)y * dw;
        for (int x = 0; x < dw; ++x) out[x] = row[cols[(size_t)x]];
    }
}

}  // namespace semper_b200
