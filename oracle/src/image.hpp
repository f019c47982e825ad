// ORACLE — test infrastructure only. Never linked into the product library.
//
// Image planes and interpolation, restating src/math/image_processor.cpp.
// T is float (the engine's precision, include/semper/types.hpp:9-10) or double
// (the FP64 accuracy judge: the same math in double).
#pragma once
#include <cstdint>
#include <vector>

#include "arith.hpp"

namespace oracle {

template <class T>
struct Image {
    int width = 0, height = 0;
    std::vector<T> I, gx, gy;

    // Image::Image + prepare_data(false) (image_processor.cpp:9-24, 54-63):
    // u8 -> T, then the 4th-order central difference, zero within 2 px of the
    // border. Integer intensities make the numerator exact, so the quotient is
    // the correctly rounded (-a + 8b - 8c + d) / 12 in any evaluation order.
    void prepare(int w, int h, const uint8_t* px) {
        width = w;
        height = h;
        const size_t n = (size_t)w * h;
        I.resize(n);
        for (size_t i = 0; i < n; ++i) I[i] = (T)px[i];
        gradients();
    }

    // The same from already-float intensities (the reference's own test images
    // are sampled straight into the float plane, tests/framework/synthetic.h:160-186).
    void prepare_float(int w, int h, const float* px) {
        width = w;
        height = h;
        const size_t n = (size_t)w * h;
        I.resize(n);
        for (size_t i = 0; i < n; ++i) I[i] = (T)px[i];
        gradients();
    }

    void gradients() {
        const int w = width, h = height;
        const size_t n = (size_t)w * h;
        gx.assign(n, T(0));
        gy.assign(n, T(0));
        for (int y = 2; y < h - 2; ++y) {
            for (int x = 2; x < w - 2; ++x) {
                const size_t k = (size_t)y * w + x;
                gx[k] = (-I[k + 2] + T(8) * I[k + 1] - T(8) * I[k - 1] + I[k - 2]) / T(12);
                gy[k] = (-I[k + 2 * (size_t)w] + T(8) * I[k + w] - T(8) * I[k - w] +
                         I[k - 2 * (size_t)w]) / T(12);
            }
        }
    }

    // stamp_ghost_wall (src/pipeline/reference_cache.cpp:18-35): masked pixels
    // (mask < 128) carry -10 after the gradients were taken from real values.
    void stamp_ghost_wall(const uint8_t* mask) {
        if (!mask) return;
        const size_t n = (size_t)width * height;
        for (size_t i = 0; i < n; ++i)
            if (mask[i] < 128) I[i] = T(-10);
    }
};

// Catmull-Rom (a = -0.5) weights, get_keys_weights (image_processor.cpp:188-195),
// with the fused products the device uses.
template <class T>
inline void cubic_weights(T s, T w[4]) {
    const T s2 = s * s;
    const T s3 = s2 * s;
    w[0] = fmaT(T(-0.5), s, fmaT(T(-0.5), s3, s2));
    w[1] = fmaT(T(-2.5), s2, fmaT(T(1.5), s3, T(1)));
    w[2] = fmaT(T(0.5), s, fmaT(T(-1.5), s3, T(2) * s2));
    w[3] = fmaT(T(0.5), s3, T(-0.5) * s2);
}

// Keys 4th-order 6x6 zones (image_processor.cpp:70-82).
template <class T>
inline T keys_f0(T s) {
    const T s2 = s * s, s3 = s2 * s;
    return fmaT(T(4.0f / 3.0f), s3, fmaT(T(-7.0f / 3.0f), s2, T(1)));
}
template <class T>
inline T keys_f1(T s) {
    const T s2 = s * s, s3 = s2 * s;
    return fmaT(T(-7.0f / 12.0f), s3, fmaT(T(3), s2, fmaT(T(-59.0f / 12.0f), s, T(2.5))));
}
template <class T>
inline T keys_f2(T s) {
    const T s2 = s * s, s3 = s2 * s;
    return fmaT(T(1.0f / 12.0f), s3, fmaT(T(-2.0f / 3.0f), s2, fmaT(T(7.0f / 4.0f), s, T(-1.5))));
}
template <class T>
inline void keys6_weights(T d, T w[6]) {
    w[0] = keys_f2(d + T(2));
    w[1] = keys_f1(d + T(1));
    w[2] = keys_f0(d);
    w[3] = keys_f0(T(1) - d);
    w[4] = keys_f1(T(2) - d);
    w[5] = keys_f2(T(3) - d);
}

// Value at pixel (xi + dx, yi + dy), 0 <= dx, dy <= 1, from the 4x4
// (interpolate_bicubic, :213-242) or 6x6 (interpolate_keys_fourth, :84-134)
// neighbourhood. Callers guarantee the 4 px guard, inside which neither
// kernel demotes to bilinear.
template <class T>
inline T interp(const Image<T>& im, int xi, int yi, T dx, T dy, bool six) {
    const int w = im.width;
    if (!six) {
        T wx[4], wy[4];
        cubic_weights(dx, wx);
        cubic_weights(dy, wy);
        T val = T(0);
        for (int j = 0; j < 4; ++j) {
            const T* r = &im.I[(size_t)(yi - 1 + j) * w + xi - 1];
            T rv = r[0] * wx[0];
            rv = fmaT(r[1], wx[1], rv);
            rv = fmaT(r[2], wx[2], rv);
            rv = fmaT(r[3], wx[3], rv);
            val = (j == 0) ? rv * wy[0] : fmaT(rv, wy[j], val);
        }
        return val;
    }
    T wx[6], wy[6];
    keys6_weights(dx, wx);
    keys6_weights(dy, wy);
    T val = T(0);
    for (int j = 0; j < 6; ++j) {
        const T* r = &im.I[(size_t)(yi - 2 + j) * w + xi - 2];
        T rv = r[0] * wx[0];
        for (int i = 1; i < 6; ++i) rv = fmaT(r[i], wx[i], rv);
        val = (j == 0) ? rv * wy[0] : fmaT(rv, wy[j], val);
    }
    return val;
}

// A warped sample's position relative to the subset centre (cx, cy), kept as
// integer centre + small offset f instead of the reference's double-summed
// absolute coordinate (src/math/optimization_engine.cpp:19-21): the offset
// carries no rounding at the magnitude of the centre at all.
template <class T>
struct Warp6 {
    T w00, w01, w02, w10, w11, w12;  // the 2x3 top of the 3x3 warp matrix
};

template <class T>
inline void warp_offset(const Warp6<T>& W, T ox, T oy, T& fx, T& fy) {
    fx = fmaT(W.w00, ox, fmaT(W.w01, oy, W.w02));
    fy = fmaT(W.w10, ox, fmaT(W.w11, oy, W.w12));
}

// inside_guard (optimization_engine.cpp:28-32) on the split coordinate: the
// pixel cx + f rounds to must lie at least 4 px inside the image.
template <class T>
inline bool guard_ok(T fx, T fy, int cx, int cy, int width, int height) {
    const T rx = fx + T(0.5), ry = fy + T(0.5);
    return rx >= (T)(4 - cx) && rx < (T)(width - 4 - cx) && ry >= (T)(4 - cy) &&
           ry < (T)(height - 4 - cy);
}

// Sample at cx + fx, cy + fy (guard already passed).
template <class T>
inline T sample_at(const Image<T>& im, int cx, int cy, T fx, T fy, bool six) {
    const T flx = std::floor(fx), fly = std::floor(fy);
    return interp(im, cx + (int)flx, cy + (int)fly, fx - flx, fy - fly, six);
}

}  // namespace oracle
