// ORACLE — test infrastructure only. Never linked into the product library.
//
// Incremental (updated-reference) DIC restated on the CPU: the per-node
// bookkeeping and the session logic of src/pipeline/incremental_math.cpp
// (sampling, coasting fits, anchors, mask warping) and
// src/pipeline/incremental_session.cpp (the session), over the restatement's
// own solves (incremental.hpp). The device session of the product is a
// separate implementation; the tests compare the two bit for bit.
//
// One definition differs from the reference's text: the length of a coasting
// step and of a match's shift is the correctly rounded root of the double sum
// of squares (length2 below), where the reference calls the C library's
// hypot, whose last bit is the library's own; the device session uses the
// same definition.
//
// The OpenCV operations the reference uses here are restated from their
// definitions: the exact Euclidean distance transform (distanceTransform,
// DIST_L2 / DIST_MASK_PRECISE) by the separable lower-envelope method of
// Felzenszwalb and Huttenlocher; a 3x3 morphological close (dilate, then
// erode, the image border neutral to both); the bounding box of the nonzero
// pixels.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <vector>

namespace semper_inc {

// The correctly rounded length of (a, b).
inline float length2(float a, float b) { return (float)std::sqrt((double)a * a + (double)b * b); }

// include/semper/tuning.hpp:193-281 and the gates the session uses.
constexpr float kIncTaylorMaxCells = 1.5f;
constexpr int kIncMaskMaxSamplesPerPx = 8;
constexpr int kIncCoastRadiusCells = 8;
constexpr int kIncCoastMinNodes = 6;
constexpr float kIncCoastMaxTravelSubsets = 2.0f;
constexpr float kIncCoastTrustedTravelSubsets = 0.25f;
constexpr float kIncReanchorMaxShiftFraction = 0.3f;
constexpr float kIncReanchorMinShiftPx = 1.0f;
constexpr int kIncAnchorMarginPx = 10;
constexpr float kIncEarlyUpdateDrop = 0.05f;
constexpr float kIncUpdateMinReported = 0.5f;
constexpr int kIncMaskExtrapCells = 3;
constexpr float kCorrInvalid = -1.0f;
constexpr float kCorrAccept = 0.15f;
constexpr int kOutlierRadius = 2;
constexpr float kOutlierEpsPx = 0.1f;
constexpr float kOutlierThreshold = 3.0f;
constexpr int kOutlierMinNeighbours = 3;
constexpr int kOutlierMaxPasses = 5;

// ------------------------------------------------------------ node fields --

// A solved lattice as sampling wants it (incremental_internal.hpp:17-29).
struct NodeField {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0;
    std::vector<float> u, v, ux, uy, vx, vy, corr;
    std::vector<unsigned char> valid;
    float node_x(int gx) const { return (float)(rect_x + gx * step); }
    float node_y(int gy) const { return (float)(rect_y + gy * step); }
    size_t size() const { return (size_t)gridW * gridH; }
};

// The raw per-node result of one solve (FieldCapture).
struct SolveCapture {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0, attempted = 0;
    std::vector<float> u, v, ux, uy, vx, vy, corr;
    std::vector<unsigned char> solved;
    // optional: the flags of the solve's own displacement median test over
    // the same nodes (the packing ran it already), and its rejection count
    std::vector<unsigned char> median_valid;
    int median_rejected = 0;
};

inline float median_inplace(std::vector<float>& v) {
    if (v.empty()) return 0.0f;
    std::sort(v.begin(), v.end());
    const size_t n = v.size(), mid = n / 2;
    if (n % 2 == 1) return v[mid];
    return 0.5f * (v[mid - 1] + v[mid]);
}

// StrainCalculator::reject_displacement_outliers
// (src/strain/strain_calculator.cpp:174-224): the normalized median test
// over a 5x5 neighbourhood, flags from finished passes only. Returns the
// count rejected.
inline int reject_outliers(int w, int h, const std::vector<float>& u, const std::vector<float>& v,
                           std::vector<unsigned char>& valid) {
    std::vector<unsigned char> ok = valid;
    std::vector<int> failed;
    std::vector<float> nu, nv, sc;
    int rejected = 0;
    auto nres = [&](float c, std::vector<float>& nb) {
        std::vector<float> tmp = nb;
        const float med = median_inplace(tmp);
        sc.resize(nb.size());
        for (size_t i = 0; i < nb.size(); ++i) sc[i] = std::fabs(nb[i] - med);
        const float spread = median_inplace(sc);
        return std::fabs(c - med) / (spread + kOutlierEpsPx);
    };
    for (int pass = 0; pass < kOutlierMaxPasses; ++pass) {
        failed.clear();
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const int idx = y * w + x;
                if (!ok[idx]) continue;
                nu.clear();
                nv.clear();
                for (int dy = -kOutlierRadius; dy <= kOutlierRadius; ++dy) {
                    const int ny = y + dy;
                    if (ny < 0 || ny >= h) continue;
                    for (int dx = -kOutlierRadius; dx <= kOutlierRadius; ++dx) {
                        const int nx = x + dx;
                        if (nx < 0 || nx >= w || (dx == 0 && dy == 0)) continue;
                        const int ni = ny * w + nx;
                        if (!ok[ni]) continue;
                        nu.push_back(u[ni]);
                        nv.push_back(v[ni]);
                    }
                }
                if ((int)nu.size() < kOutlierMinNeighbours) continue;
                if (nres(u[idx], nu) > kOutlierThreshold || nres(v[idx], nv) > kOutlierThreshold)
                    failed.push_back(idx);
            }
        if (failed.empty()) break;
        for (int idx : failed) ok[idx] = 0;
        rejected += (int)failed.size();
    }
    for (size_t i = 0; i < ok.size(); ++i)
        if (!ok[i]) valid[i] = 0;
    return rejected;
}

// node_field_from_capture (incremental_math.cpp:19-57): solved nodes with a
// result, less the ones the displacement median test rejects.
inline NodeField node_field_from_capture(const SolveCapture& cap, int* rejected = nullptr) {
    NodeField f;
    f.gridW = cap.gridW;
    f.gridH = cap.gridH;
    f.rect_x = cap.rect_x;
    f.rect_y = cap.rect_y;
    f.step = cap.step;
    const size_t n = f.size();
    f.u.assign(n, 0.0f);
    f.v.assign(n, 0.0f);
    f.ux.assign(n, 0.0f);
    f.uy.assign(n, 0.0f);
    f.vx.assign(n, 0.0f);
    f.vy.assign(n, 0.0f);
    f.corr.assign(n, kCorrInvalid);
    f.valid.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
        if (!(cap.solved[i] && cap.corr[i] >= 0.0f)) continue;
        f.u[i] = cap.u[i];
        f.v[i] = cap.v[i];
        f.ux[i] = cap.ux[i];
        f.uy[i] = cap.uy[i];
        f.vx[i] = cap.vx[i];
        f.vy[i] = cap.vy[i];
        f.corr[i] = cap.corr[i];
        f.valid[i] = 1;
    }
    if (cap.median_valid.size() == n) {
        // the same test on the same nodes, already run by the solve
        for (size_t i = 0; i < n; ++i) f.valid[i] = f.valid[i] && cap.median_valid[i] ? 1 : 0;
        if (rejected) *rejected = cap.median_rejected;
        return f;
    }
    const int dropped = reject_outliers(f.gridW, f.gridH, f.u, f.v, f.valid);
    if (rejected) *rejected = dropped;
    return f;
}

struct IncrementSample {
    bool ok = false;
    bool taylor = false;
    float u = 0.0f, v = 0.0f;
    float corr = 0.0f;
};

// sample_increment (incremental_math.cpp:59-119): the node's own value on a
// node, bilinear inside a cell with four valid corners, else the first-order
// expansion from the nearest valid node of the 4x4 block within
// kIncTaylorMaxCells cells.
inline IncrementSample sample_increment(const NodeField& f, float x, float y) {
    IncrementSample s;
    if (f.gridW <= 0 || f.gridH <= 0 || f.step <= 0) return s;
    const float gx = (x - (float)f.rect_x) / (float)f.step;
    const float gy = (y - (float)f.rect_y) / (float)f.step;
    const int i0 = (int)std::floor(gx), j0 = (int)std::floor(gy);
    const float fx = gx - (float)i0, fy = gy - (float)j0;
    auto idx = [&](int i, int j) { return (size_t)j * f.gridW + i; };
    auto in = [&](int i, int j) { return i >= 0 && i < f.gridW && j >= 0 && j < f.gridH; };
    if (fx == 0.0f && fy == 0.0f && in(i0, j0) && f.valid[idx(i0, j0)]) {
        const size_t k = idx(i0, j0);
        s.ok = true;
        s.u = f.u[k];
        s.v = f.v[k];
        s.corr = f.corr[k];
        return s;
    }
    if (in(i0, j0) && in(i0 + 1, j0 + 1)) {
        const size_t a = idx(i0, j0), b = idx(i0 + 1, j0), c = idx(i0, j0 + 1), d = idx(i0 + 1, j0 + 1);
        if (f.valid[a] && f.valid[b] && f.valid[c] && f.valid[d]) {
            const float wa = (1 - fx) * (1 - fy), wb = fx * (1 - fy);
            const float wc = (1 - fx) * fy, wd = fx * fy;
            s.ok = true;
            s.u = wa * f.u[a] + wb * f.u[b] + wc * f.u[c] + wd * f.u[d];
            s.v = wa * f.v[a] + wb * f.v[b] + wc * f.v[c] + wd * f.v[d];
            s.corr = std::max(std::max(f.corr[a], f.corr[b]), std::max(f.corr[c], f.corr[d]));
            return s;
        }
    }
    const float max_d = kIncTaylorMaxCells * (float)f.step;
    float best_d2 = std::numeric_limits<float>::infinity();
    int bi = -1, bj = -1;
    for (int j = j0 - 1; j <= j0 + 2; ++j)
        for (int i = i0 - 1; i <= i0 + 2; ++i) {
            if (!in(i, j) || !f.valid[idx(i, j)]) continue;
            const float dx = x - f.node_x(i), dy = y - f.node_y(j);
            const float d2 = dx * dx + dy * dy;
            if (d2 < best_d2) {
                best_d2 = d2;
                bi = i;
                bj = j;
            }
        }
    if (bi < 0 || best_d2 > max_d * max_d) return s;
    const size_t k = idx(bi, bj);
    const float dx = x - f.node_x(bi), dy = y - f.node_y(bj);
    s.ok = true;
    s.taylor = true;
    s.u = f.u[k] + f.ux[k] * dx + f.uy[k] * dy;
    s.v = f.v[k] + f.vx[k] * dx + f.vy[k] * dy;
    s.corr = f.corr[k];
    return s;
}

// fit_increment (incremental_math.cpp:121-186): a weighted least-squares
// plane through the valid nodes within radius_px, weights 1 / (1 + (d/step)^2),
// with at least kIncCoastMinNodes nodes whose weighted spread is at least
// one step in both principal directions; its value at (x, y) by Cramer's rule.
inline IncrementSample fit_increment(const NodeField& f, float x, float y, float radius_px) {
    IncrementSample s;
    if (f.gridW <= 0 || f.gridH <= 0 || f.step <= 0 || radius_px <= 0.0f) return s;
    const double step = f.step;
    const int r = (int)std::ceil(radius_px / step);
    const int ic = (int)std::lround((x - f.rect_x) / step);
    const int jc = (int)std::lround((y - f.rect_y) / step);
    const double r2max = (double)radius_px * radius_px;
    double S[3][3] = {{0}}, bu[3] = {0}, bv[3] = {0};
    int n = 0;
    float worst = 0.0f;
    for (int j = std::max(0, jc - r); j <= std::min(f.gridH - 1, jc + r); ++j)
        for (int i = std::max(0, ic - r); i <= std::min(f.gridW - 1, ic + r); ++i) {
            const size_t k = (size_t)j * f.gridW + i;
            if (!f.valid[k]) continue;
            const double dx = f.node_x(i) - x, dy = f.node_y(j) - y;
            const double d2 = dx * dx + dy * dy;
            if (d2 > r2max) continue;
            const double w = 1.0 / (1.0 + d2 / (step * step));
            const double p[3] = {1.0, dx / step, dy / step};
            for (int a = 0; a < 3; ++a) {
                for (int b = 0; b < 3; ++b) S[a][b] += w * p[a] * p[b];
                bu[a] += w * p[a] * f.u[k];
                bv[a] += w * p[a] * f.v[k];
            }
            worst = std::max(worst, f.corr[k]);
            ++n;
        }
    if (n < kIncCoastMinNodes) return s;
    const double W = S[0][0];
    const double mx = S[0][1] / W, my = S[0][2] / W;
    const double cxx = S[1][1] / W - mx * mx, cyy = S[2][2] / W - my * my, cxy = S[1][2] / W - mx * my;
    const double tr = cxx + cyy, det2 = cxx * cyy - cxy * cxy;
    const double lmin = 0.5 * (tr - std::sqrt(std::max(0.0, tr * tr - 4.0 * det2)));
    if (lmin < 1.0) return s;
    auto det3 = [](const double m[3][3]) {
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    };
    const double D = det3(S);
    if (std::abs(D) < 1e-12) return s;
    auto first = [&](const double b[3]) {
        double M[3][3];
        for (int a = 0; a < 3; ++a) {
            M[a][0] = b[a];
            M[a][1] = S[a][1];
            M[a][2] = S[a][2];
        }
        return det3(M) / D;
    };
    s.ok = true;
    s.u = (float)first(bu);
    s.v = (float)first(bv);
    s.corr = worst;
    return s;
}

// Exact Euclidean distance (in cells) from every cell to the nearest cell
// where `inside` is 0; +inf where there is none. Squared distances are exact
// integers (a row pass, then the lower envelope of parabolas down each
// column), the root taken once.
inline std::vector<float> distance_to_zero(int w, int h, const std::vector<unsigned char>& inside) {
    const double INF = std::numeric_limits<double>::infinity();
    // f: squared distance so far (INF: none); out: the lower envelope of the
    // parabolas (q - p)^2 + f(p) over the finite f(p)
    auto edt1 = [&](const double* f, double* out, int n, std::vector<int>& v, std::vector<double>& z) {
        v.assign((size_t)n, 0);
        z.assign((size_t)n + 1, 0.0);
        int k = -1;
        auto cross = [&](int p, int q) { return ((f[q] + (double)q * q) - (f[p] + (double)p * p)) / (2.0 * (q - p)); };
        for (int q = 0; q < n; ++q) {
            if (!(f[q] < INF)) continue;
            if (k < 0) {
                k = 0;
                v[0] = q;
                z[0] = -INF;
                z[1] = INF;
                continue;
            }
            double sv = cross(v[k], q);
            while (sv <= z[k]) {
                --k;
                sv = cross(v[k], q);
            }
            ++k;
            v[k] = q;
            z[k] = sv;
            z[k + 1] = INF;
        }
        if (k < 0) {
            for (int q = 0; q < n; ++q) out[q] = INF;
            return;
        }
        int j = 0;
        for (int q = 0; q < n; ++q) {
            while (z[j + 1] < q) ++j;
            const int p = v[j];
            out[q] = (double)(q - p) * (q - p) + f[p];
        }
    };
    std::vector<int> v;
    std::vector<double> z, g((size_t)w * h), col((size_t)h), colout((size_t)h), row((size_t)w), rowout((size_t)w);
    for (int y = 0; y < h; ++y) {
        for (int x = 0; x < w; ++x) row[x] = inside[(size_t)y * w + x] ? INF : 0.0;
        edt1(row.data(), rowout.data(), w, v, z);
        for (int x = 0; x < w; ++x) g[(size_t)y * w + x] = rowout[x];
    }
    std::vector<float> out((size_t)w * h);
    for (int x = 0; x < w; ++x) {
        for (int y = 0; y < h; ++y) col[y] = g[(size_t)y * w + x];
        edt1(col.data(), colout.data(), h, v, z);
        for (int y = 0; y < h; ++y)
            out[(size_t)y * w + x] = colout[y] < INF ? (float)std::sqrt(colout[y]) : std::numeric_limits<float>::infinity();
    }
    return out;
}

// gap_distance (incremental_math.cpp:188-209): per node, px to the nearest
// unsolved node (`hole`) and to the nearest unsolved or off-grid position
// (`gap`), with a one-node ring standing for "off the grid".
struct GapDistance {
    int w = 0, h = 0;
    std::vector<float> hole, gap;
};

inline GapDistance gap_distance(const NodeField& f) {
    GapDistance g;
    if (f.gridW <= 0 || f.gridH <= 0 || f.step <= 0) return g;
    const int W = f.gridW + 2, H = f.gridH + 2;
    std::vector<unsigned char> solved((size_t)W * H, 0), hole_in((size_t)W * H, 1);
    for (int j = 0; j < f.gridH; ++j)
        for (int i = 0; i < f.gridW; ++i) {
            const unsigned char v = f.valid[(size_t)j * f.gridW + i] ? 1 : 0;
            solved[(size_t)(j + 1) * W + i + 1] = v;
            hole_in[(size_t)(j + 1) * W + i + 1] = v;
        }
    const std::vector<float> dg = distance_to_zero(W, H, solved), dh = distance_to_zero(W, H, hole_in);
    g.w = f.gridW;
    g.h = f.gridH;
    g.gap.resize(f.size());
    g.hole.resize(f.size());
    for (int j = 0; j < f.gridH; ++j)
        for (int i = 0; i < f.gridW; ++i) {
            g.gap[(size_t)j * f.gridW + i] = (float)(dg[(size_t)(j + 1) * W + i + 1] * (double)f.step);
            g.hole[(size_t)j * f.gridW + i] = (float)(dh[(size_t)(j + 1) * W + i + 1] * (double)f.step);
        }
    return g;
}

enum class AnchorNeed { kDrop, kRefresh, kKeep };

// anchor_need (incremental_math.cpp:211-221).
inline AnchorNeed anchor_need(const NodeField& f, const GapDistance& g, float x, float y, int subset_size) {
    if (g.gap.empty()) return AnchorNeed::kKeep;
    const int i = std::min(f.gridW - 1, std::max(0, (int)std::lround((x - f.rect_x) / f.step)));
    const int j = std::min(f.gridH - 1, std::max(0, (int)std::lround((y - f.rect_y) / f.step)));
    if (g.hole[(size_t)j * f.gridW + i] <= (float)(subset_size / 2 + f.step)) return AnchorNeed::kKeep;
    if (g.gap[(size_t)j * f.gridW + i] <= (float)(2 * subset_size + 2 * f.step)) return AnchorNeed::kRefresh;
    return AnchorNeed::kDrop;
}

// A coasting node's subset on the last reference it was measured on
// (incremental_internal.hpp:71-76): a square gray patch around (ax, ay).
struct CoastAnchor {
    std::vector<uint8_t> patch;
    int size = 0;  // side, 2 * (subset / 2 + kIncAnchorMarginPx) + 1
    int ax = 0, ay = 0;
    float dx = 0, dy = 0;
};

// make_anchor (incremental_math.cpp:223-236).
inline bool make_anchor(const uint8_t* gray, int W, int H, float x, float y, int subset_size, CoastAnchor& out) {
    const int ax = (int)std::lround(x), ay = (int)std::lround(y);
    const int r = subset_size / 2 + kIncAnchorMarginPx;
    if (!gray || ax - r < 0 || ay - r < 0 || ax + r >= W || ay + r >= H) return false;
    out.size = 2 * r + 1;
    out.patch.resize((size_t)out.size * out.size);
    for (int j = 0; j < out.size; ++j)
        std::memcpy(&out.patch[(size_t)j * out.size], gray + (size_t)(ay - r + j) * W + (ax - r), out.size);
    out.ax = ax;
    out.ay = ay;
    out.dx = x - (float)ax;
    out.dy = y - (float)ay;
    return true;
}

// The anchor's node through a matched affine map (match_anchor,
// incremental_math.cpp:238-276, after the solve): the match is accepted only
// when it converged, passed kCorrAccept and stays within max_shift.
inline bool accept_anchor_match(const CoastAnchor& a, int status, float score, float u, float v, float ux, float uy,
                                float vx, float vy, float guess_x, float guess_y, float max_shift, float& x,
                                float& y, float& corr) {
    if (status != 0 || !(score <= kCorrAccept)) return false;
    const float nx = (float)a.ax + u + (1.0f + ux) * a.dx + uy * a.dy;
    const float ny = (float)a.ay + v + vx * a.dx + (1.0f + vy) * a.dy;
    if (!(length2(nx - guess_x, ny - guess_y) <= max_shift)) return false;
    x = nx;
    y = ny;
    corr = score;
    return true;
}

struct GridGeom {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0;
};

// fill_field (incremental_math.cpp:281-322): invalid nodes take the mean of
// their filled 4-neighbours, pass by pass, until nothing changes.
inline bool fill_field(int w, int h, std::vector<float>& U, std::vector<float>& V,
                       const std::vector<unsigned char>& valid) {
    const size_t n = (size_t)w * h;
    std::vector<unsigned char> filled(valid.begin(), valid.end());
    bool any = false;
    for (size_t i = 0; i < n; ++i) {
        if (filled[i])
            any = true;
        else {
            U[i] = 0.0f;
            V[i] = 0.0f;
        }
    }
    if (!any) return false;
    std::vector<unsigned char> next;
    std::vector<float> nu(U), nv(V);
    for (int pass = 0; pass < w + h + 2; ++pass) {
        next = filled;
        bool changed = false;
        for (int y = 0; y < h; ++y)
            for (int x = 0; x < w; ++x) {
                const size_t i = (size_t)y * w + x;
                if (filled[i]) continue;
                float su = 0, sv = 0;
                int cnt = 0;
                const int nx[4] = {x - 1, x + 1, x, x};
                const int ny[4] = {y, y, y - 1, y + 1};
                for (int k = 0; k < 4; ++k) {
                    if (nx[k] < 0 || nx[k] >= w || ny[k] < 0 || ny[k] >= h) continue;
                    const size_t j = (size_t)ny[k] * w + nx[k];
                    if (!filled[j]) continue;
                    su += U[j];
                    sv += V[j];
                    ++cnt;
                }
                if (cnt == 0) continue;
                nu[i] = su / (float)cnt;
                nv[i] = sv / (float)cnt;
                next[i] = 1;
                changed = true;
            }
        U = nu;
        V = nv;
        filled.swap(next);
        if (!changed) break;
    }
    return true;
}

// The continuous field over the filled grid (incremental_math.cpp:324-369):
// bilinear inside, the plane through the nearest grid point with that point's
// gradient outside.
struct ContinuousField {
    const GridGeom& g;
    const std::vector<float>& U;
    const std::vector<float>& V;
    void eval(double x, double y, double& u, double& v) const {
        const double gx_raw = (x - g.rect_x) / g.step, gy_raw = (y - g.rect_y) / g.step;
        const double gx = std::max(0.0, std::min(gx_raw, (double)(g.gridW - 1)));
        const double gy = std::max(0.0, std::min(gy_raw, (double)(g.gridH - 1)));
        const double ox = (gx_raw - gx) * g.step, oy = (gy_raw - gy) * g.step;
        int i0 = (int)std::floor(gx), j0 = (int)std::floor(gy);
        i0 = std::max(0, std::min(i0, std::max(g.gridW - 2, 0)));
        j0 = std::max(0, std::min(j0, std::max(g.gridH - 2, 0)));
        const int i1 = std::min(i0 + 1, g.gridW - 1), j1 = std::min(j0 + 1, g.gridH - 1);
        const double tx = (i1 == i0) ? 0.0 : gx - i0, ty = (j1 == j0) ? 0.0 : gy - j0;
        auto at = [&](const std::vector<float>& F, int i, int j) { return (double)F[(size_t)j * g.gridW + i]; };
        auto bil = [&](const std::vector<float>& F, double& val, double& dx, double& dy) {
            const double a = at(F, i0, j0), b = at(F, i1, j0), c = at(F, i0, j1), d = at(F, i1, j1);
            val = a * (1 - tx) * (1 - ty) + b * tx * (1 - ty) + c * (1 - tx) * ty + d * tx * ty;
            dx = (i1 == i0) ? 0.0 : ((b - a) * (1 - ty) + (d - c) * ty) / g.step;
            dy = (j1 == j0) ? 0.0 : ((c - a) * (1 - tx) + (d - b) * tx) / g.step;
        };
        double ux, uy, vx, vy;
        bil(U, u, ux, uy);
        bil(V, v, vx, vy);
        u += ux * ox + uy * oy;
        v += vx * ox + vy * oy;
    }
};

// 3x3 morphological close of a 0/255 mask, the image border neutral to both
// the dilation and the erosion.
inline void close3x3(std::vector<uint8_t>& m, int W, int H) {
    std::vector<uint8_t> d((size_t)W * H);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            uint8_t v = 0;
            for (int dy = -1; dy <= 1 && !v; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx, yy = y + dy;
                    if (xx < 0 || yy < 0 || xx >= W || yy >= H) continue;
                    if (m[(size_t)yy * W + xx]) {
                        v = 255;
                        break;
                    }
                }
            d[(size_t)y * W + x] = v;
        }
#pragma omp parallel for schedule(static)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            uint8_t v = 255;
            for (int dy = -1; dy <= 1 && v; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int xx = x + dx, yy = y + dy;
                    if (xx < 0 || yy < 0 || xx >= W || yy >= H) continue;
                    if (!d[(size_t)yy * W + xx]) {
                        v = 0;
                        break;
                    }
                }
            m[(size_t)y * W + x] = v;
        }
}

// warp_material_mask (incremental_math.cpp:371-447), in two steps. The plan:
// the filled field, the samples per pixel and the frame-0 window; false when
// no node is valid or the window is empty (the warped mask is then empty).
struct MaskWarpPlan {
    std::vector<float> U, V;  // filled over the grid
    int per_px = 2;
    int X0 = 0, X1 = -1, Y0 = 0, Y1 = -1;
};

inline bool plan_mask_warp(const GridGeom& geom, const std::vector<float>& U_in, const std::vector<float>& V_in,
                           const std::vector<unsigned char>& valid, int W, int H, int margin_px, MaskWarpPlan& p) {
    if (geom.gridW <= 0 || geom.gridH <= 0 || geom.step <= 0) return false;
    p.U = U_in;
    p.V = V_in;
    if (!fill_field(geom.gridW, geom.gridH, p.U, p.V, valid)) return false;
    double stretch = 1.0;
    for (int gy = 0; gy < geom.gridH; ++gy)
        for (int gx = 0; gx < geom.gridW; ++gx) {
            const size_t i = (size_t)gy * geom.gridW + gx;
            const size_t ix = gx + 1 < geom.gridW ? i + 1 : i;
            const size_t iy = gy + 1 < geom.gridH ? i + geom.gridW : i;
            const double ux = (p.U[ix] - p.U[i]) / geom.step, uy = (p.U[iy] - p.U[i]) / geom.step;
            const double vx = (p.V[ix] - p.V[i]) / geom.step, vy = (p.V[iy] - p.V[i]) / geom.step;
            stretch = std::max(stretch, std::max(std::abs(1 + ux) + std::abs(uy), std::abs(vx) + std::abs(1 + vy)));
        }
    p.per_px = std::min(kIncMaskMaxSamplesPerPx, std::max(2, (int)std::ceil(stretch / 0.7)));
    p.X0 = std::max(0, geom.rect_x - margin_px);
    p.X1 = std::min(W - 1, geom.rect_x + (geom.gridW - 1) * geom.step + margin_px);
    p.Y0 = std::max(0, geom.rect_y - margin_px);
    p.Y1 = std::min(H - 1, geom.rect_y + (geom.gridH - 1) * geom.step + margin_px);
    return p.X0 <= p.X1 && p.Y0 <= p.Y1;
}

// The scatter: every frame-0 material sample X (per_px x per_px per pixel of
// the window) lands at X + U(X); then the 3x3 close.
inline void scatter_mask_host(const std::vector<uint8_t>& mask0, int W, int H, const GridGeom& geom,
                              const MaskWarpPlan& p, std::vector<uint8_t>& out) {
    out.assign((size_t)W * H, 0);
    const ContinuousField field{geom, p.U, p.V};
    const double hs = 1.0 / p.per_px;
#pragma omp parallel for schedule(static)
    for (int sy = p.Y0; sy <= p.Y1; ++sy) {
        const uint8_t* mrow = mask0.data() + (size_t)sy * W;
        for (int sx = p.X0; sx <= p.X1; ++sx) {
            if (mrow[sx] < 128) continue;
            for (int b = 0; b < p.per_px; ++b)
                for (int a = 0; a < p.per_px; ++a) {
                    const double X = sx - 0.5 + (a + 0.5) * hs, Y = sy - 0.5 + (b + 0.5) * hs;
                    double u, v;
                    field.eval(X, Y, u, v);
                    const long px = std::lround(X + u), py = std::lround(Y + v);
                    if (px < 0 || px >= W || py < 0 || py >= H) continue;
                    // every writer stores the same value: the result does not depend on order
                    out[(size_t)py * W + px] = 255;
                }
        }
    }
    close3x3(out, W, H);
}

inline std::vector<uint8_t> warp_material_mask(const std::vector<uint8_t>& mask0, int W, int H, const GridGeom& geom,
                                               const std::vector<float>& U_in, const std::vector<float>& V_in,
                                               const std::vector<unsigned char>& valid, int margin_px) {
    std::vector<uint8_t> out;
    MaskWarpPlan p;
    if (!plan_mask_warp(geom, U_in, V_in, valid, W, H, margin_px, p)) return std::vector<uint8_t>((size_t)W * H, 0);
    scatter_mask_host(mask0, W, H, geom, p, out);
    return out;
}

struct Rect {
    int x = 0, y = 0, w = 0, h = 0;
    long long area() const { return (long long)w * h; }
};

inline Rect bounding_rect(const std::vector<uint8_t>& m, int W, int H) {
    int x0 = W, y0 = H, x1 = -1, y1 = -1;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x)
            if (m[(size_t)y * W + x]) {
                x0 = std::min(x0, x);
                x1 = std::max(x1, x);
                y0 = std::min(y0, y);
                y1 = std::max(y1, y);
            }
    if (x1 < 0) return Rect{};
    return Rect{x0, y0, x1 - x0 + 1, y1 - y0 + 1};
}

inline Rect intersect(const Rect& a, const Rect& b) {
    const int x0 = std::max(a.x, b.x), y0 = std::max(a.y, b.y);
    const int x1 = std::min(a.x + a.w, b.x + b.w), y1 = std::min(a.y + a.h, b.y + b.h);
    if (x1 <= x0 || y1 <= y0) return Rect{};
    return Rect{x0, y0, x1 - x0, y1 - y0};
}

}  // namespace semper_inc

namespace semper_inc {

// ---------------------------------------------------------------- session --

struct IncParams {
    int rect_x = 0, rect_y = 0, rect_w = 0, rect_h = 0, step = 0, subset_size = 0, strain_window = 0;
    bool six = false;
};

// IncrementalFrameInfo (include/semper/incremental.hpp:38-46).
struct FrameInfo {
    int reference_frame = 0;
    bool reference_updated = false;
    int tracked_points = 0;
    int frame0_points = 0;
    int taylor_fallbacks = 0;
    int lost_this_frame = 0;
};

inline int64_t max_strain_window(const IncParams& p) {
    if (p.step <= 0) return 0;
    const int64_t gmin = std::min(p.rect_w / p.step, p.rect_h / p.step);
    return 2 * (gmin + 1) * (int64_t)p.step;
}

// IncrementalSession (src/pipeline/incremental_session.cpp) over a solver
// backend B, which provides:
//   int  validate(IncParams&, int W, int H)        validate_params (clips the rect)
//   int  vsg_count(int step, int window)           vsg_window_node_count
//   int  set_reference(gray, W, H, mask)           0 or an error
//   int  run(def, mask, const IncParams&, out, capacity, metrics, metrics_len,
//            progress, SolveCapture*)               run_full_field; keeps the
//                                                   prepared deformed frame
//   int  adopt(const uint8_t* mask)                the kept frame becomes the
//                                                   reference, Ghost Wall from mask
//   int  pack(const GridGeom&, window, u, v, corr, solved, out, capacity)
//                                                   pack_full_field_output
//   bool match_anchor(const CoastAnchor&, subset, six, gx, gy, max_shift, x, y, corr)
//                                                   match_anchor on the kept frame
//   Rect warp_mask(mask0, W, H, const GridGeom&, const MaskWarpPlan&, out)
//                                                   the scatter and close of
//                                                   warp_material_mask; returns
//                                                   the bounding box of `out`
template <class B>
class IncrementalCore {
public:
    using Progress = std::function<void(int)>;
    explicit IncrementalCore(B& backend) : b_(backend) {}

    void clear() {
        initialized_ = false;
        width_ = height_ = 0;
        user_mask0_.clear();
        material_mask0_.clear();
        grid0_ = GridGeom();
        frame0_points_ = -1;
        Ubase_.clear();
        Vbase_.clear();
        alive_.clear();
        coast_travel_.clear();
        anchors_.clear();
        ref_index_ = 0;
        frames_since_update_ = 0;
        ref_reported_ = -1;
        adopted_reported_ = -1;
        frame_count_ = 0;
        params_k_ = IncParams();
        mask_k_.clear();
        scratch_.clear();
    }

    bool initialized() const { return initialized_; }
    int frames_processed() const { return frame_count_; }
    int max_points() const { return grid0_.gridW * grid0_.gridH; }

    // IncrementalSession::init (incremental_session.cpp:219-268).
    int init(const uint8_t* ref, int W, int H, const uint8_t* roi_mask, IncParams p, int update_interval) {
        clear();
        if (!ref || W <= 0 || H <= 0) return -3;
        if (update_interval < 0) return -3;
        params_ = p;
        interval_ = update_interval;
        const int rc = b_.validate(params_, W, H);
        if (rc != 0) return rc;
        const int gridW = params_.rect_w / params_.step, gridH = params_.rect_h / params_.step;
        if (b_.vsg_count(params_.step, params_.strain_window) < 3) return -4;
        width_ = W;
        height_ = H;
        grid0_ = GridGeom{gridW, gridH, params_.rect_x, params_.rect_y, params_.step};
        const size_t npx = (size_t)W * H;
        if (roi_mask) {
            user_mask0_.assign(roi_mask, roi_mask + npx);
            material_mask0_.resize(npx);
            for (size_t i = 0; i < npx; ++i) material_mask0_[i] = roi_mask[i] >= 128 ? 255 : 0;
        } else {
            // the ROI rect plus the reach of its edge nodes' subsets at 45 deg
            const int half = (int)std::ceil(params_.subset_size / 2 * std::sqrt(2.0)) + 1;
            material_mask0_.assign(npx, 0);
            const Rect r = intersect(Rect{params_.rect_x - half, params_.rect_y - half, params_.rect_w + 2 * half,
                                          params_.rect_h + 2 * half},
                                     Rect{0, 0, W, H});
            for (int y = r.y; y < r.y + r.h; ++y)
                std::fill(material_mask0_.begin() + (size_t)y * W + r.x, material_mask0_.begin() + (size_t)y * W + r.x + r.w,
                          (uint8_t)255);
        }
        if (b_.set_reference(ref, W, H, user_mask0_.empty() ? nullptr : user_mask0_.data()) != 0) {
            clear();
            return -3;
        }
        const size_t n = (size_t)gridW * gridH;
        Ubase_.assign(n, 0.0f);
        Vbase_.assign(n, 0.0f);
        alive_.assign(n, 1);
        coast_travel_.assign(n, 0.0f);
        initialized_ = true;
        return 0;
    }

    // IncrementalSession::Impl::process (incremental_session.cpp:289-549).
    int process(const uint8_t* def, float* output, int output_capacity, float* metrics, int metrics_len,
                const Progress& progress, FrameInfo* info) {
        if (!initialized_ || output == nullptr || def == nullptr) return -3;
        FrameInfo fi;
        fi.reference_frame = ref_index_;
        const int N = interval_;
        bool will_update = N > 0 && frames_since_update_ + 1 >= N;
        const GridGeom& g0 = grid0_;
        const size_t n0 = (size_t)g0.gridW * g0.gridH;
        if (ref_index_ > 0 && alive_count() == 0) return nothing_to_follow(fi, metrics, metrics_len, progress, info);

        SolveCapture cap;
        std::vector<float> U(n0, 0.0f), V(n0, 0.0f);
        std::vector<unsigned char> valid(n0, 0), carried(n0, 0);
        std::vector<float> coast_step(n0, 0.0f);
        std::vector<AnchorNeed> need(n0, AnchorNeed::kKeep);
        int written = 0, frame0_points = frame0_points_;
        const int subset_size = params_.subset_size;
        const float max_travel = kIncCoastMaxTravelSubsets * (float)subset_size;
        auto carry = [&](size_t i, float du, float dv) {
            const float travel = length2(du, dv);
            if (coast_travel_[i] + travel > max_travel) return;
            U[i] = Ubase_[i] + du;
            V[i] = Vbase_[i] + dv;
            carried[i] = 1;
            coast_step[i] = travel;
        };
        auto coast = [&](size_t i, const NodeField& inc, float px, float py) {
            if (px < 0.0f || py < 0.0f || px > (float)(width_ - 1) || py > (float)(height_ - 1)) return;
            const float radius = (float)(kIncCoastRadiusCells * inc.step);
            const IncrementSample fit = fit_increment(inc, px, py, radius);
            if (!fit.ok) return;
            carry(i, fit.u, fit.v);
        };
        const float trusted_travel = kIncCoastTrustedTravelSubsets * (float)subset_size;
        int reanchored = 0;

        if (ref_index_ == 0) {
            // the same call as a fixed-reference run, straight into the caller's buffer
            const int rc = b_.run(def, user_mask0_.empty() ? nullptr : user_mask0_.data(), params_, output,
                                  output_capacity, metrics, metrics_len, progress, &cap);
            if (rc < 0) return rc;
            written = rc;
            const NodeField nf = node_field_from_capture(cap);
            U = nf.u;
            V = nf.v;
            valid = nf.valid;
            carried = valid;
            if (frame0_points < 0) frame0_points = cap.attempted;
            const GapDistance gd = gap_distance(nf);
            for (size_t i = 0; i < n0; ++i)
                if (valid[i])
                    need[i] = anchor_need(nf, gd, nf.node_x((int)(i % g0.gridW)), nf.node_y((int)(i / g0.gridW)),
                                          subset_size);
        } else {
            const int gw = params_k_.step > 0 ? params_k_.rect_w / params_k_.step : 0;
            const int gh = params_k_.step > 0 ? params_k_.rect_h / params_k_.step : 0;
            scratch_.resize((size_t)std::max(gw * gh, 1) * 8);
            const int rc = b_.run(def, mask_k_.data(), params_k_, scratch_.data(), (int)scratch_.size(), metrics,
                                  metrics_len, progress, &cap);
            if (rc == -2) {
                // nothing of this reference's grid can be solved: the nodes are dropped
                fi.lost_this_frame = alive_count();
                std::fill(alive_.begin(), alive_.end(), 0);
                for (CoastAnchor& a : anchors_) a.size = 0;
                return nothing_to_follow(fi, metrics, metrics_len, progress, info);
            }
            if (rc < 0) return rc;
            const NodeField inc = node_field_from_capture(cap);
            const GapDistance gd = gap_distance(inc);
            std::vector<float> gu(n0, 0.0f), gv(n0, 0.0f), gcorr(n0, kCorrInvalid);
            std::vector<unsigned char> gsolved(n0, 0);
            // Every node's own step depends on that node alone, so the nodes run
            // in parallel; the anchor matches (device solves) then run one by
            // one in node order.
            enum : unsigned char { kNone, kValid, kMatch };
            std::vector<unsigned char> state(n0, kNone), taylor(n0, 0);
            std::vector<float> ncorr(n0, 0.0f);
#pragma omp parallel for schedule(static)
            for (long li = 0; li < (long)n0; ++li) {
                const size_t i = (size_t)li;
                if (!alive_[i]) continue;
                const int gx = (int)(i % g0.gridW), gy = (int)(i / g0.gridW);
                const float x = (float)(g0.rect_x + gx * g0.step), y = (float)(g0.rect_y + gy * g0.step);
                const float px = x + Ubase_[i], py = y + Vbase_[i];
                const IncrementSample smp = sample_increment(inc, px, py);
                if (!smp.ok) {
                    coast(i, inc, px, py);
                    continue;
                }
                U[i] = Ubase_[i] + smp.u;
                V[i] = Vbase_[i] + smp.v;
                ncorr[i] = smp.corr;
                taylor[i] = smp.taylor ? 1 : 0;
                need[i] = anchor_need(inc, gd, px, py, subset_size);
                if (coast_travel_[i] > trusted_travel) {
                    // confirmed only by a direct match of its subset from where it was last clean
                    if (need[i] == AnchorNeed::kKeep || anchor_of(i) == nullptr) {
                        carried[i] = 1;
                        continue;
                    }
                    state[i] = kMatch;
                    continue;
                }
                state[i] = kValid;
            }
            for (size_t i = 0; i < n0; ++i) {
                if (state[i] == kMatch) {
                    const float x = (float)(g0.rect_x + (int)(i % g0.gridW) * g0.step);
                    const float y = (float)(g0.rect_y + (int)(i / g0.gridW) * g0.step);
                    const float max_shift =
                        std::max(kIncReanchorMinShiftPx, kIncReanchorMaxShiftFraction * coast_travel_[i]);
                    float mx = 0.0f, my = 0.0f;
                    if (!b_.match_anchor(*anchor_of(i), subset_size, params_.six, x + U[i], y + V[i], max_shift, mx,
                                         my, ncorr[i])) {
                        carried[i] = 1;
                        continue;
                    }
                    U[i] = mx - x;
                    V[i] = my - y;
                    reanchored++;
                } else if (state[i] != kValid) {
                    continue;
                }
                valid[i] = 1;
                carried[i] = 1;
                if (taylor[i]) fi.taylor_fallbacks++;
                gu[i] = U[i];
                gv[i] = V[i];
                gcorr[i] = ncorr[i];
                gsolved[i] = 1;
            }
            written = b_.pack(g0, params_.strain_window, gu, gv, gcorr, gsolved, output, output_capacity);
            if (written < 0) return written;
        }

        for (unsigned char c : carried) fi.tracked_points += c ? 1 : 0;
        fi.frame0_points = std::max(frame0_points, 0);

        // the update rules: a failed solve never becomes the reference; an
        // early update when the points reported drop (N > 1)
        int ref_reported = ref_reported_;
        const int base = ref_reported >= 0 ? ref_reported : adopted_reported_ >= 0 ? adopted_reported_ : frame0_points;
        if (base > 0 && (float)written < kIncUpdateMinReported * (float)base) {
            will_update = false;
        } else if (N > 1) {
            if (ref_reported < 0)
                ref_reported = written;
            else if ((float)written < (1.0f - kIncEarlyUpdateDrop) * (float)ref_reported)
                will_update = true;
        }

        if (will_update) {
            const int before = (ref_index_ == 0) ? fi.frame0_points : alive_count();
            std::vector<float> coast_travel = coast_travel_;
            // the anchors this update drops and refreshes, applied in place once
            // the new reference is adopted (a failed adoption leaves them as
            // they were)
            std::vector<size_t> drop, refresh;
            for (size_t i = 0; i < n0; ++i) {
                coast_travel[i] = (carried[i] && !valid[i]) ? coast_travel[i] + coast_step[i] : 0.0f;
                if (!carried[i] || (valid[i] && need[i] == AnchorNeed::kDrop)) {
                    if (anchor_of(i)) drop.push_back(i);
                } else if (valid[i] && need[i] == AnchorNeed::kRefresh) {
                    refresh.push_back(i);
                }
            }
            NextReference next = prepare_reference(U, V, carried);
            if (b_.adopt(next.mask_k.data()) != 0) return -3;
            if (anchors_.size() < n0) anchors_.resize(n0);
            for (const size_t i : drop) anchors_[i].size = 0;
            // each node's anchor is its own slot: the copies run in parallel; a
            // patch that does not fit leaves the slot as it was
#pragma omp parallel for schedule(static)
            for (long k = 0; k < (long)refresh.size(); ++k) {
                const size_t i = refresh[(size_t)k];
                const float ax = (float)(g0.rect_x + (int)(i % g0.gridW) * g0.step) + U[i];
                const float ay = (float)(g0.rect_y + (int)(i / g0.gridW) * g0.step) + V[i];
                make_anchor(def, width_, height_, ax, ay, subset_size, anchors_[i]);
            }
            coast_travel_.swap(coast_travel);
            Ubase_.swap(next.Ubase);
            Vbase_.swap(next.Vbase);
            alive_.swap(next.alive);
            mask_k_ = std::move(next.mask_k);
            params_k_ = next.params_k;
            frame_count_++;
            ref_index_ = frame_count_;
            frames_since_update_ = 0;
            ref_reported_ = -1;
            adopted_reported_ = written;
            frame0_points_ = frame0_points;
            fi.reference_updated = true;
            fi.lost_this_frame = std::max(0, before - alive_count());
        } else {
            frame_count_++;
            frames_since_update_++;
            ref_reported_ = ref_reported;
            frame0_points_ = frame0_points;
        }
        (void)reanchored;
        if (info) *info = fi;
        return written;
    }

private:
    struct NextReference {
        std::vector<float> Ubase, Vbase;
        std::vector<unsigned char> alive;
        std::vector<uint8_t> mask_k;
        IncParams params_k;
    };

    int alive_count() const {
        int n = 0;
        for (unsigned char a : alive_) n += a ? 1 : 0;
        return n;
    }

    // prepare_reference (incremental_session.cpp:118-176).
    NextReference prepare_reference(const std::vector<float>& U, const std::vector<float>& V,
                                    const std::vector<unsigned char>& valid) const {
        NextReference r;
        r.Ubase = U;
        r.Vbase = V;
        r.alive = valid;
        const int half = params_.subset_size / 2;
        const int margin = (kIncMaskExtrapCells + 1) * grid0_.step + half;
        MaskWarpPlan plan;
        Rect bb;
        if (plan_mask_warp(grid0_, r.Ubase, r.Vbase, r.alive, width_, height_, margin, plan)) {
            bb = b_.warp_mask(material_mask0_, width_, height_, grid0_, plan, r.mask_k);
        } else {
            r.mask_k.assign((size_t)width_ * height_, 0);
        }
        r.params_k = params_;
        float min_x = 1e30f, min_y = 1e30f, max_x = -1e30f, max_y = -1e30f;
        for (int j = 0; j < grid0_.gridH; ++j)
            for (int i = 0; i < grid0_.gridW; ++i) {
                const size_t n = (size_t)j * grid0_.gridW + i;
                if (!r.alive[n]) continue;
                const float x = grid0_.rect_x + i * grid0_.step + r.Ubase[n];
                const float y = grid0_.rect_y + j * grid0_.step + r.Vbase[n];
                min_x = std::min(min_x, x);
                max_x = std::max(max_x, x);
                min_y = std::min(min_y, y);
                max_y = std::max(max_y, y);
            }
        Rect grid_rect;
        if (min_x <= max_x) {
            const int x0 = (int)std::floor(min_x), y0 = (int)std::floor(min_y);
            grid_rect = intersect(Rect{x0, y0, (int)std::ceil(max_x) - x0 + grid0_.step,
                                       (int)std::ceil(max_y) - y0 + grid0_.step},
                                  Rect{0, 0, width_, height_});
        }
        r.params_k.rect_x = grid_rect.x;
        r.params_k.rect_y = grid_rect.y;
        r.params_k.rect_w = grid_rect.w;
        r.params_k.rect_h = grid_rect.h;
        r.params_k.strain_window = (int)std::min<int64_t>(r.params_k.strain_window, max_strain_window(r.params_k));
        if (bb.area() == 0) std::fill(r.alive.begin(), r.alive.end(), 0);
        return r;
    }

    // nothing_to_follow (incremental_session.cpp:178-196).
    int nothing_to_follow(FrameInfo fi, float* metrics, int metrics_len, const Progress& progress, FrameInfo* info) {
        frame_count_++;
        fi.frame0_points = std::max(frame0_points_, 0);
        if (info) *info = fi;
        if (metrics != nullptr) {
            const int len = metrics_len < 16 ? 0 : metrics_len >= 24 ? 24 : metrics_len == 18 ? 17 : metrics_len;
            std::fill_n(metrics, len, 0.0f);
        }
        if (progress) progress(100);
        return 0;
    }

    B& b_;
    bool initialized_ = false;
    IncParams params_;
    int interval_ = 0;
    int width_ = 0, height_ = 0;
    std::vector<uint8_t> user_mask0_, material_mask0_;
    GridGeom grid0_;
    int frame0_points_ = -1;
    std::vector<float> Ubase_, Vbase_;
    std::vector<unsigned char> alive_;
    std::vector<float> coast_travel_;
    // the coasting anchor of each frame-0 node (size 0: none)
    std::vector<CoastAnchor> anchors_;

    const CoastAnchor* anchor_of(size_t i) const {
        return i < anchors_.size() && anchors_[i].size > 0 ? &anchors_[i] : nullptr;
    }
    int ref_index_ = 0, frames_since_update_ = 0, ref_reported_ = -1, adopted_reported_ = -1, frame_count_ = 0;
    IncParams params_k_;
    std::vector<uint8_t> mask_k_;
    std::vector<float> scratch_;
};

}  // namespace semper_inc
