// ORACLE — test infrastructure only. Never linked into the product library.
//
// Displacement median test and VSG strain, restating
// src/strain/strain_calculator.cpp:12-224 and src/util/median.hpp:21-30.
// VSG normal equations in FP64 as the reference; the 3x3 inverse is the
// cofactor form times 1/det, every product and sum separately rounded.
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

namespace oracle {

constexpr double kVsgRadiusTiny = 1.0e-5;
constexpr int kOutlierRadius = 2;
constexpr float kOutlierEpsPx = 0.1f;
constexpr float kOutlierThreshold = 3.0f;
constexpr int kOutlierMinNeighbours = 3;
constexpr int kOutlierMaxPasses = 5;
constexpr float kStrainUninitSentinel = -1000.0f;
constexpr float kStrainFailSentinel = -999.0f;

// vsg_window_node_count (strain_calculator.cpp:12-25).
inline int vsg_window_node_count(int step, int window) {
    if (step <= 0) return 0;
    const float radius = window / 2.0f;
    const int grid_rad = (int)std::ceil(radius / (float)step);
    const double r2 = (double)(radius * radius) + kVsgRadiusTiny;
    int count = 0;
    for (int dy = -grid_rad; dy <= grid_rad; ++dy)
        for (int dx = -grid_rad; dx <= grid_rad; ++dx) {
            const double px = (double)(dx * step), py = (double)(dy * step);
            if (px * px + py * py <= r2) ++count;
        }
    return count;
}

// Median of the (finite) values; mean of the middle pair for an even count.
inline float median_of(std::vector<float> v) {
    if (v.empty()) return 0.0f;
    std::sort(v.begin(), v.end());
    const size_t n = v.size(), mid = n / 2;
    if (n % 2 == 1) return v[mid];
    return 0.5f * (v[mid - 1] + v[mid]);
}

struct DispField {
    int width = 0, height = 0, step = 0;
    std::vector<float> u, v;
    std::vector<unsigned char> valid;
};

// reject_displacement_outliers (strain_calculator.cpp:174-224).
inline int reject_outliers(DispField& f) {
    const int w = f.width, h = f.height, r = kOutlierRadius;
    std::vector<unsigned char> ok = f.valid;
    std::vector<int> failed;
    int rejected = 0;
    auto nres = [](float c, const std::vector<float>& nb) {
        const float med = median_of(nb);
        std::vector<float> sc(nb.size());
        for (size_t i = 0; i < nb.size(); ++i) sc[i] = std::fabs(nb[i] - med);
        const float spread = median_of(sc);
        return std::fabs(c - med) / (spread + kOutlierEpsPx);
    };
    std::vector<float> nu, nv;
    for (int pass = 0; pass < kOutlierMaxPasses; ++pass) {
        failed.clear();
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const int idx = y * w + x;
                if (!ok[idx]) continue;
                nu.clear();
                nv.clear();
                for (int dy = -r; dy <= r; ++dy) {
                    const int ny = y + dy;
                    if (ny < 0 || ny >= h) continue;
                    for (int dx = -r; dx <= r; ++dx) {
                        const int nx = x + dx;
                        if (nx < 0 || nx >= w || (dx == 0 && dy == 0)) continue;
                        const int ni = ny * w + nx;
                        if (!ok[ni]) continue;
                        nu.push_back(f.u[ni]);
                        nv.push_back(f.v[ni]);
                    }
                }
                if ((int)nu.size() < kOutlierMinNeighbours) continue;
                if (nres(f.u[idx], nu) > kOutlierThreshold || nres(f.v[idx], nv) > kOutlierThreshold)
                    failed.push_back(idx);
            }
        if (failed.empty()) break;
        for (int idx : failed) ok[idx] = 0;
        rejected += (int)failed.size();
    }
    for (size_t i = 0; i < ok.size(); ++i)
        if (!ok[i]) f.valid[i] = 0;
    return rejected;
}

struct StrainOut {
    std::vector<float> exx, eyy, exy;
};

// compute_vsg_strain (strain_calculator.cpp:27-158).
inline StrainOut vsg_strain(const DispField& f, int window) {
    StrainOut s;
    const size_t total = (size_t)f.width * f.height;
    s.exx.assign(total, kStrainUninitSentinel);
    s.eyy.assign(total, kStrainUninitSentinel);
    s.exy.assign(total, kStrainUninitSentinel);
    if (f.step <= 0 || window <= 0) return s;
    const float radius = window / 2.0f;
    const int grid_rad = (int)std::ceil(radius / f.step);
    const int expected = vsg_window_node_count(f.step, window);
    const double r2 = (double)(radius * radius) + kVsgRadiusTiny;
    for (int y = 0; y < f.height; ++y)
        for (int x = 0; x < f.width; ++x) {
            const int idx = y * f.width + x;
            if (!f.valid[idx]) continue;
            double A[3][3] = {}, bu[3] = {}, bv[3] = {};
            int cnt = 0;
            for (int dy = -grid_rad; dy <= grid_rad; ++dy)
                for (int dx = -grid_rad; dx <= grid_rad; ++dx) {
                    const int nx = x + dx, ny = y + dy;
                    if (nx < 0 || nx >= f.width || ny < 0 || ny >= f.height) continue;
                    const int ni = ny * f.width + nx;
                    if (!f.valid[ni]) continue;
                    const double px = (double)(dx * f.step), py = (double)(dy * f.step);
                    if (px * px + py * py <= r2) {
                        const double du = (double)f.u[ni], dv = (double)f.v[ni];
                        const double a[3] = {1.0, px, py};
                        for (int i = 0; i < 3; ++i) {
                            for (int j = 0; j < 3; ++j) A[i][j] = A[i][j] + a[i] * a[j];
                            bu[i] = bu[i] + a[i] * du;
                            bv[i] = bv[i] + a[i] * dv;
                        }
                        ++cnt;
                    }
                }
            const double fill = (double)cnt / (double)expected;
            if (!(fill >= 0.90 && cnt >= 3)) continue;
            double anorm = 0.0;
            for (int c = 0; c < 3; ++c) {
                const double cs = std::fabs(A[0][c]) + std::fabs(A[1][c]) + std::fabs(A[2][c]);
                if (cs > anorm) anorm = cs;
            }
            // Cofactors; det expanded along column 0.
            double C[3][3];
            C[0][0] = A[1][1] * A[2][2] - A[1][2] * A[2][1];
            C[1][0] = A[0][2] * A[2][1] - A[0][1] * A[2][2];
            C[2][0] = A[0][1] * A[1][2] - A[0][2] * A[1][1];
            C[0][1] = A[1][2] * A[2][0] - A[1][0] * A[2][2];
            C[1][1] = A[0][0] * A[2][2] - A[0][2] * A[2][0];
            C[2][1] = A[0][2] * A[1][0] - A[0][0] * A[1][2];
            C[0][2] = A[1][0] * A[2][1] - A[1][1] * A[2][0];
            C[1][2] = A[0][1] * A[2][0] - A[0][0] * A[2][1];
            C[2][2] = A[0][0] * A[1][1] - A[0][1] * A[1][0];
            const double det = A[0][0] * C[0][0] + A[1][0] * C[1][0] + A[2][0] * C[2][0];
            if (!(std::fabs(det) > 1e-12)) continue;
            const double idet = 1.0 / det;
            double Ai[3][3];
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Ai[i][j] = C[i][j] * idet;
            double inorm = 0.0;
            for (int c = 0; c < 3; ++c) {
                const double cs = std::fabs(Ai[0][c]) + std::fabs(Ai[1][c]) + std::fabs(Ai[2][c]);
                if (cs > inorm) inorm = cs;
            }
            const double rcond = (anorm * inorm > 0.0) ? (1.0 / (anorm * inorm)) : 0.0;
            if (rcond < 1e-12) continue;
            double cu[3], cv[3];
            for (int i = 0; i < 3; ++i) {
                cu[i] = (Ai[i][0] * bu[0] + Ai[i][1] * bu[1]) + Ai[i][2] * bu[2];
                cv[i] = (Ai[i][0] * bv[0] + Ai[i][1] * bv[1]) + Ai[i][2] * bv[2];
            }
            const double dudx = cu[1], dudy = cu[2], dvdx = cv[1], dvdy = cv[2];
            s.exx[idx] = (float)(0.5 * ((2.0 * dudx + dudx * dudx) + dvdx * dvdx));
            s.eyy[idx] = (float)(0.5 * ((2.0 * dvdy + dudy * dudy) + dvdy * dvdy));
            s.exy[idx] = (float)(0.5 * (((dudy + dvdx) + dudx * dudy) + dvdx * dvdy));
        }
    return s;
}

}  // namespace oracle
