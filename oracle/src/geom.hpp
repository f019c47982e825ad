// ORACLE — test infrastructure only. Never linked into the product library.
//
// The seeding mesh's planar geometry, written for the CPU restatement on its
// own (the product's host code has its own copy of these operations; a CPU
// test holds the two to the same answers). The reference calls OpenCV here:
//   Delaunay triangulation   cv::Subdiv2D + getTriangleList   (src/pipeline/full_field_mesh.cpp:66-83)
//   affine map of a triangle cv::getAffineTransform           (full_field_mesh.cpp:101)
//   point in triangle        cv::pointPolygonTest             (full_field_mesh.cpp:180, 203)
//   convex hull + area       cv::convexHull, cv::contourArea  (src/pipeline/full_field_anchors.cpp:493-496)
//   homography refit         cv::findHomography (RANSAC)      (full_field_anchors.cpp:552-561)
//   homography_at            src/pipeline/akaze_features.cpp:184-198
// That arithmetic is third-party, so the build fixes its own rules, and this
// file follows them:
//   * the triangulation is Bowyer-Watson over the points rounded to integers,
//     inserted in input order, inside one super-triangle (centred on the
//     points' coordinate range, 20 x (64 x range + 64) from its centre), with
//     an exact in-circle test (a point exactly on a circumcircle does not
//     break the triangle) and new triangles (cavity edge a -> b, point);
//     triangles are listed by their sorted vertex indices;
//   * every floating-point quantity (affine maps, distances, hull area, the
//     normalised DLT homography through a cyclic Jacobi eigen-solver, its
//     inlier refit) is formed by the operations, in the order, that the
//     product's host code uses, so that the two pipelines see the same bits.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <map>
#include <utility>
#include <vector>

namespace oracle_geom {

struct Pt {
    double x, y;
};

struct Tri {
    int a, b, c;  // counter-clockwise
};

// 2 x the signed area of (a, b, c): > 0 for a left turn.
inline int64_t turn(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t cx, int64_t cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

// Sign of the in-circle determinant of d against the ccw triangle (a, b, c):
// > 0 strictly inside its circumcircle. 128-bit: the lifted terms of
// coordinates up to 2^40 stay exact.
inline int in_circle(const int64_t* X, const int64_t* Y, int a, int b, int c, int d) {
    using w = __int128;
    const w ax = X[a] - X[d], ay = Y[a] - Y[d];
    const w bx = X[b] - X[d], by = Y[b] - Y[d];
    const w cx = X[c] - X[d], cy = Y[c] - Y[d];
    const w det = (ax * ax + ay * ay) * (bx * cy - by * cx) - (bx * bx + by * by) * (ax * cy - ay * cx) +
                  (cx * cx + cy * cy) * (ax * by - ay * bx);
    return det > 0 ? 1 : (det < 0 ? -1 : 0);
}

inline std::vector<Tri> delaunay(const std::vector<Pt>& pts) {
    const int n = (int)pts.size();
    if (n < 3) return {};
    std::vector<int64_t> X(n + 3), Y(n + 3);
    int64_t lo = 0, hi = 0;
    for (int i = 0; i < n; ++i) {
        X[i] = std::llround(pts[i].x);
        Y[i] = std::llround(pts[i].y);
        const int64_t a = std::min(X[i], Y[i]), b = std::max(X[i], Y[i]);
        lo = i == 0 ? a : std::min(lo, a);
        hi = i == 0 ? b : std::max(hi, b);
    }
    const int64_t reach = 20 * (std::max<int64_t>(hi - lo, 1) * 64 + 64), c = (lo + hi) / 2;
    X[n] = c - reach, Y[n] = c - reach;
    X[n + 1] = c + reach, Y[n + 1] = c - reach;
    X[n + 2] = c, Y[n + 2] = c + reach;
    std::vector<Tri> mesh{{n, n + 1, n + 2}};
    for (int p = 0; p < n; ++p) {
        // the cavity: every triangle whose circumcircle holds p strictly
        std::vector<Tri> kept, cavity;
        for (const Tri& t : mesh) (in_circle(X.data(), Y.data(), t.a, t.b, t.c, p) > 0 ? cavity : kept).push_back(t);
        // its boundary: the directed edges whose undirected edge occurs once
        std::map<std::pair<int, int>, int> uses;
        for (const Tri& t : cavity)
            for (const auto& e : {std::make_pair(t.a, t.b), std::make_pair(t.b, t.c), std::make_pair(t.c, t.a)})
                ++uses[{std::min(e.first, e.second), std::max(e.first, e.second)}];
        for (const Tri& t : cavity)
            for (const auto& e : {std::make_pair(t.a, t.b), std::make_pair(t.b, t.c), std::make_pair(t.c, t.a)}) {
                if (uses[{std::min(e.first, e.second), std::max(e.first, e.second)}] != 1) continue;
                // a point on the edge would make a flat triangle
                if (turn(X[e.first], Y[e.first], X[e.second], Y[e.second], X[p], Y[p]) > 0)
                    kept.push_back({e.first, e.second, p});
            }
        mesh.swap(kept);
    }
    std::vector<Tri> out;
    for (const Tri& t : mesh)
        if (t.a < n && t.b < n && t.c < n) out.push_back(t);
    auto sorted = [](const Tri& t) {
        int v[3] = {t.a, t.b, t.c};
        std::sort(v, v + 3);
        return std::vector<int>(v, v + 3);
    };
    std::sort(out.begin(), out.end(), [&](const Tri& u, const Tri& v) { return sorted(u) < sorted(v); });
    return out;
}

// X = M0 x + M1 y + M2, Y = M3 x + M4 y + M5 through three point pairs, by
// Cramer's rule on [x y 1]; false when the sources are collinear.
inline bool affine3(const Pt s[3], const Pt d[3], double M[6]) {
    const double det = s[0].x * (s[1].y - s[2].y) - s[0].y * (s[1].x - s[2].x) + (s[1].x * s[2].y - s[2].x * s[1].y);
    if (!(std::fabs(det) > 0.0)) return false;
    for (int r = 0; r < 2; ++r) {
        const double v0 = r ? d[0].y : d[0].x, v1 = r ? d[1].y : d[1].x, v2 = r ? d[2].y : d[2].x;
        const double ca = v0 * (s[1].y - s[2].y) - s[0].y * (v1 - v2) + (v1 * s[2].y - v2 * s[1].y);
        const double cb = s[0].x * (v1 - v2) - v0 * (s[1].x - s[2].x) + (s[1].x * v2 - s[2].x * v1);
        const double cc = s[0].x * (s[1].y * v2 - s[2].y * v1) - s[0].y * (s[1].x * v2 - s[2].x * v1) +
                          v0 * (s[1].x * s[2].y - s[2].x * s[1].y);
        M[3 * r] = ca / det;
        M[3 * r + 1] = cb / det;
        M[3 * r + 2] = cc / det;
    }
    return true;
}

// Inside or on the edge of the triangle (integer coordinates, exact).
inline bool in_triangle(const int64_t X[3], const int64_t Y[3], int64_t qx, int64_t qy) {
    bool neg = false, pos = false;
    for (int k = 0; k < 3; ++k) {
        const int64_t t = turn(X[k], Y[k], X[(k + 1) % 3], Y[(k + 1) % 3], qx, qy);
        neg = neg || t < 0;
        pos = pos || t > 0;
    }
    return !(neg && pos);
}

// pointPolygonTest's measure: the distance to the nearest edge, positive
// inside or on the boundary, negative outside.
inline double signed_distance(const Pt v[3], Pt p) {
    double d2 = 1e300;
    for (int k = 0; k < 3; ++k) {
        const Pt a = v[k], b = v[(k + 1) % 3];
        const double ex = b.x - a.x, ey = b.y - a.y, px = p.x - a.x, py = p.y - a.y;
        const double len2 = ex * ex + ey * ey;
        const double t = std::clamp(len2 > 0.0 ? (px * ex + py * ey) / len2 : 0.0, 0.0, 1.0);
        const double qx = px - t * ex, qy = py - t * ey;
        d2 = std::min(d2, qx * qx + qy * qy);
    }
    const int64_t X[3] = {std::llround(v[0].x), std::llround(v[1].x), std::llround(v[2].x)};
    const int64_t Y[3] = {std::llround(v[0].y), std::llround(v[1].y), std::llround(v[2].y)};
    const double d = std::sqrt(d2);
    return in_triangle(X, Y, std::llround(p.x), std::llround(p.y)) ? d : -d;
}

// Convex hull area: Andrew's monotone chain from the lowest-x (then lowest-y)
// point, lower chain then upper, collinear points dropped; the shoelace sum
// taken in that vertex order.
inline double hull_area(std::vector<Pt> p) {
    const size_t n = p.size();
    if (n < 3) return 0.0;
    std::sort(p.begin(), p.end(), [](const Pt& a, const Pt& b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
    auto cross = [](const Pt& o, const Pt& a, const Pt& b) { return (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x); };
    std::vector<Pt> h;
    for (size_t i = 0; i < n; ++i) {
        while (h.size() >= 2 && cross(h[h.size() - 2], h.back(), p[i]) <= 0) h.pop_back();
        h.push_back(p[i]);
    }
    const size_t lower = h.size() + 1;
    for (size_t i = n - 1; i > 0; --i) {
        while (h.size() >= lower && cross(h[h.size() - 2], h.back(), p[i - 1]) <= 0) h.pop_back();
        h.push_back(p[i - 1]);
    }
    h.pop_back();
    double s = 0.0;
    for (size_t i = 0; i < h.size(); ++i) {
        const Pt& u = h[i];
        const Pt& v = h[(i + 1) % h.size()];
        s += u.x * v.y - v.x * u.y;
    }
    return std::fabs(s) * 0.5;
}

// Cyclic Jacobi on a symmetric 9 x 9 matrix A (destroyed): eigenvalues into
// e, eigenvectors into the columns of V. Sweeps over (p < q) in row order
// until the off-diagonal square sum drops below 1e-30 (at most 100).
inline void eigen_sym9(double A[81], double e[9], double V[81]) {
    constexpr int n = 9;
    for (int i = 0; i < n * n; ++i) V[i] = (i % (n + 1)) == 0 ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (A[q * n + q] - A[p * n + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                auto rotate = [&](double* M, int stride_k, int stride_pq) {
                    for (int k = 0; k < n; ++k) {
                        double& mp = M[k * stride_k + p * stride_pq];
                        double& mq = M[k * stride_k + q * stride_pq];
                        const double u = mp, v = mq;
                        mp = c * u - s * v;
                        mq = s * u + c * v;
                    }
                };
                rotate(A, n, 1);  // columns p, q
                rotate(A, 1, n);  // rows p, q
                rotate(V, n, 1);
            }
    }
    for (int i = 0; i < n; ++i) e[i] = A[i * n + i];
}

// Normalised DLT over the flagged pairs: both point sets moved to their
// centroid and scaled to mean distance sqrt 2, the 9 x 9 normal matrix's
// eigenvector of least eigenvalue, denormalised, scaled to H[8] = 1.
inline bool dlt(const std::vector<Pt>& src, const std::vector<Pt>& dst, const std::vector<char>& use, double H[9]) {
    int m = 0;
    double sx = 0, sy = 0, dx = 0, dy = 0;
    for (size_t i = 0; i < src.size(); ++i)
        if (use[i]) {
            sx += src[i].x;
            sy += src[i].y;
            dx += dst[i].x;
            dy += dst[i].y;
            ++m;
        }
    if (m < 4) return false;
    sx /= m;
    sy /= m;
    dx /= m;
    dy /= m;
    double rs = 0, rd = 0;
    for (size_t i = 0; i < src.size(); ++i)
        if (use[i]) {
            rs += std::hypot(src[i].x - sx, src[i].y - sy);
            rd += std::hypot(dst[i].x - dx, dst[i].y - dy);
        }
    const double ks = rs > 0 ? std::sqrt(2.0) * m / rs : 1.0, kd = rd > 0 ? std::sqrt(2.0) * m / rd : 1.0;
    double N[81] = {};
    for (size_t i = 0; i < src.size(); ++i) {
        if (!use[i]) continue;
        const double x = (src[i].x - sx) * ks, y = (src[i].y - sy) * ks;
        const double u = (dst[i].x - dx) * kd, v = (dst[i].y - dy) * kd;
        const double ru[9] = {-x, -y, -1, 0, 0, 0, u * x, u * y, u};
        const double rv[9] = {0, 0, 0, -x, -y, -1, v * x, v * y, v};
        for (int a = 0; a < 9; ++a)
            for (int b = 0; b < 9; ++b) N[a * 9 + b] += ru[a] * ru[b] + rv[a] * rv[b];
    }
    double e[9], V[81];
    eigen_sym9(N, e, V);
    int k = 0;
    for (int i = 1; i < 9; ++i)
        if (e[i] < e[k]) k = i;
    const double Ts[9] = {ks, 0, -ks * sx, 0, ks, -ks * sy, 0, 0, 1};
    const double Td[9] = {1 / kd, 0, dx, 0, 1 / kd, dy, 0, 0, 1};
    double A[9] = {}, B[9] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int q = 0; q < 3; ++q) A[r * 3 + c] += V[(r * 3 + q) * 9 + k] * Ts[q * 3 + c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int q = 0; q < 3; ++q) B[r * 3 + c] += Td[r * 3 + q] * A[q * 3 + c];
    if (!(std::fabs(B[8]) > 1e-300)) return false;
    for (int i = 0; i < 9; ++i) {
        H[i] = B[i] / B[8];
        if (!std::isfinite(H[i])) return false;
    }
    return true;
}

// The homography with inlier refits at `tol` px until the inlier set holds
// (at most 8 refits); false when fewer than 4 points stay.
inline bool fit_homography(const std::vector<Pt>& src, const std::vector<Pt>& dst, double tol, double H[9]) {
    std::vector<char> use(src.size(), 1);
    if (!dlt(src, dst, use, H)) return false;
    for (int round = 0; round < 8; ++round) {
        std::vector<char> in(src.size(), 0);
        int m = 0;
        for (size_t i = 0; i < src.size(); ++i) {
            const double w = H[6] * src[i].x + H[7] * src[i].y + H[8];
            if (!(std::fabs(w) > 1e-12)) continue;
            const double X = (H[0] * src[i].x + H[1] * src[i].y + H[2]) / w;
            const double Y = (H[3] * src[i].x + H[4] * src[i].y + H[5]) / w;
            if (std::hypot(X - dst[i].x, Y - dst[i].y) <= tol) {
                in[i] = 1;
                ++m;
            }
        }
        if (m < 4) return false;
        if (in == use) break;
        use.swap(in);
        if (!dlt(src, dst, use, H)) return false;
    }
    return true;
}

// The homography's image of (px, py) and its Jacobian there.
inline bool homography_at(const double h[9], double px, double py, double& X, double& Y, double J[4]) {
    const double w = h[6] * px + h[7] * py + h[8];
    if (!std::isfinite(w) || std::fabs(w) < 1e-12) return false;
    X = (h[0] * px + h[1] * py + h[2]) / w;
    Y = (h[3] * px + h[4] * py + h[5]) / w;
    J[0] = (h[0] - X * h[6]) / w;
    J[1] = (h[1] - X * h[7]) / w;
    J[2] = (h[3] - Y * h[6]) / w;
    J[3] = (h[4] - Y * h[7]) / w;
    bool ok = std::isfinite(X) && std::isfinite(Y);
    for (int k = 0; k < 4; ++k) ok = ok && std::isfinite(J[k]);
    return ok;
}

}  // namespace oracle_geom
