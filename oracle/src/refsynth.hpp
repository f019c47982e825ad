// ORACLE — test infrastructure only. Never linked into the product library.
//
// The reference test suite's analytic speckle, restated so the inputs behind
// its golden fixtures can be regenerated here:
//   SpeckleField, AffineDeformation   tests/framework/synthetic.h:34-187
//   gray8 (clamp, then v + 0.5f)      tests/framework/synthetic_cv.h:17-36
// std::mt19937 / uniform_real_distribution<float> / std::exp come from the same
// C++ standard library the fixtures were captured with (libstdc++); the sum
// over blobs runs in index order. The reference built its tests with
// -ffast-math, so its own images may differ from these in the last bits; the
// fixture comparisons carry tolerances for exactly that.
#pragma once
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

namespace oracle {

struct RefSpeckle {
    std::vector<float> cx, cy, inv2s2, amp;
    RefSpeckle(unsigned seed, int width, int height, int blobs = 400) {
        std::mt19937 rng(seed);
        std::uniform_real_distribution<float> ux(0.0f, (float)width);
        std::uniform_real_distribution<float> uy(0.0f, (float)height);
        std::uniform_real_distribution<float> us(1.5f, 3.5f);
        std::uniform_real_distribution<float> ua(-90.0f, 90.0f);
        for (int i = 0; i < blobs; ++i) {
            cx.push_back(ux(rng));
            cy.push_back(uy(rng));
            const float s = us(rng);
            inv2s2.push_back(1.0f / (2.0f * s * s));
            amp.push_back(ua(rng));
        }
    }
    float sample(float x, float y) const {
        float v = 128.0f;
        for (size_t i = 0; i < cx.size(); ++i) {
            const float dx = x - cx[i], dy = y - cy[i];
            const float r2 = dx * dx + dy * dy;
            if (r2 < 40.0f) v += amp[i] * std::exp(-r2 * inv2s2[i]);
        }
        if (v < 5.0f) v = 5.0f;
        if (v > 250.0f) v = 250.0f;
        return v;
    }
};

struct RefAffine {
    float u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0, cx = 0, cy = 0;
    void inverse_map(float qx, float qy, float& rx, float& ry) const {
        const float bx = qx - cx - u, by = qy - cy - v;
        const float a11 = 1.0f + ux, a12 = uy, a21 = vx, a22 = 1.0f + vy;
        const float det = a11 * a22 - a12 * a21;
        const float px = (a22 * bx - a12 * by) / det;
        const float py = (-a21 * bx + a11 * by) / det;
        rx = cx + px;
        ry = cy + py;
    }
};

inline std::vector<float> ref_image(const RefSpeckle& f, int w, int h) {
    std::vector<float> out((size_t)w * h);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) out[(size_t)y * w + x] = f.sample((float)x, (float)y);
    return out;
}

inline std::vector<float> def_image(const RefSpeckle& f, int w, int h, const RefAffine& d) {
    std::vector<float> out((size_t)w * h);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            float rx, ry;
            d.inverse_map((float)x, (float)y, rx, ry);
            out[(size_t)y * w + x] = f.sample(rx, ry);
        }
    return out;
}

inline std::vector<uint8_t> gray8(const std::vector<float>& img) {
    std::vector<uint8_t> m(img.size());
    for (size_t i = 0; i < img.size(); ++i) {
        float v = img[i];
        if (v < 0.f) v = 0.f;
        if (v > 255.f) v = 255.f;
        m[i] = (uint8_t)(v + 0.5f);
    }
    return m;
}

}  // namespace oracle
