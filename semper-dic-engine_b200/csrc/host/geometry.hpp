// Planar geometry for the seeding mesh: the engine's replacements for the
// OpenCV calls the reference makes there (no OpenCV in this build).
//
//   Delaunay triangulation   cv::Subdiv2D + getTriangleList   (src/pipeline/full_field_mesh.cpp:66-83)
//   affine map of a triangle cv::getAffineTransform           (full_field_mesh.cpp:101)
//   point in triangle        cv::pointPolygonTest             (full_field_mesh.cpp:180, 203)
//   convex hull + area       cv::convexHull, cv::contourArea  (src/pipeline/full_field_anchors.cpp:493-496)
//   homography refit         cv::findHomography (RANSAC 1 px) (full_field_anchors.cpp:552-561)
//
// Seed points are grid nodes, so their coordinates are integers: every
// orientation and in-circle predicate here is evaluated exactly in integer
// arithmetic, which makes the triangulation, and which triangle a grid node
// falls in, a pure function of the point set and its order. Co-circular
// quadruples (every cell of a full lattice) keep the diagonal the incremental
// insertion produced; OpenCV resolves them by its own rule, so the triangle
// diagonals (and the guesses interpolated across them) are not pinned to the
// reference's — only the converged solves are.
//
// Header-only; used by the host pipeline of the library and by the CPU
// restatement used in its tests, so both see the same mesh.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

namespace semper_geom {

struct Pt {
    double x, y;
};

struct Tri {
    int a, b, c;  // indices into the input points, counter-clockwise
};

using i128 = __int128;

inline int64_t orient_i(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t cx, int64_t cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

// > 0 when d lies strictly inside the circumcircle of the ccw triangle abc.
inline i128 incircle_i(int64_t ax, int64_t ay, int64_t bx, int64_t by, int64_t cx, int64_t cy,
                       int64_t dx, int64_t dy) {
    const i128 adx = ax - dx, ady = ay - dy, bdx = bx - dx, bdy = by - dy, cdx = cx - dx,
               cdy = cy - dy;
    const i128 al = adx * adx + ady * ady, bl = bdx * bdx + bdy * bdy, cl = cdx * cdx + cdy * cdy;
    return al * (bdx * cdy - bdy * cdx) - bl * (adx * cdy - ady * cdx) + cl * (adx * bdy - ady * bdx);
}

// Bowyer-Watson over integer points, inserted in input order. Returns the
// triangles with no vertex on the enclosing super-triangle, sorted by their
// (min, mid, max) vertex indices so the order is canonical.
inline std::vector<Tri> delaunay(const std::vector<Pt>& pts) {
    const int n = (int)pts.size();
    std::vector<Tri> out;
    if (n < 3) return out;
    std::vector<int64_t> X(n + 3), Y(n + 3);
    int64_t lo = INT64_MAX, hi = INT64_MIN;
    for (int i = 0; i < n; ++i) {
        X[i] = (int64_t)std::llround(pts[i].x);
        Y[i] = (int64_t)std::llround(pts[i].y);
        lo = std::min(lo, std::min(X[i], Y[i]));
        hi = std::max(hi, std::max(X[i], Y[i]));
    }
    const int64_t span = std::max<int64_t>(hi - lo, 1) * 64 + 64;
    const int64_t mid = (lo + hi) / 2;
    // Super triangle far outside the points (ccw).
    X[n] = mid - 20 * span; Y[n] = mid - 20 * span;
    X[n + 1] = mid + 20 * span; Y[n + 1] = mid - 20 * span;
    X[n + 2] = mid; Y[n + 2] = mid + 20 * span;

    // Each triangle carries its circumcircle in double precision, a filter
    // only: a point farther than the radius (with a wide margin) cannot be
    // inside, and every other candidate gets the exact integer test. The
    // triangles found are those of the exact test alone.
    struct Circ {
        double x, y, r2;  // r2 < 0: degenerate, always tested
    };
    auto circ_of = [&](const Tri& T) {
        const double ax = (double)X[T.a], ay = (double)Y[T.a], bx = (double)X[T.b], by = (double)Y[T.b];
        const double cx = (double)X[T.c], cy = (double)Y[T.c];
        const double d = 2.0 * (ax * (by - cy) + bx * (cy - ay) + cx * (ay - by));
        if (!(std::fabs(d) > 0.0)) return Circ{0.0, 0.0, -1.0};
        const double a2 = ax * ax + ay * ay, b2 = bx * bx + by * by, c2 = cx * cx + cy * cy;
        const double ux = (a2 * (by - cy) + b2 * (cy - ay) + c2 * (ay - by)) / d;
        const double uy = (a2 * (cx - bx) + b2 * (ax - cx) + c2 * (bx - ax)) / d;
        return Circ{ux, uy, (ax - ux) * (ax - ux) + (ay - uy) * (ay - uy)};
    };
    std::vector<Tri> tris;
    std::vector<Circ> circs;
    tris.push_back({n, n + 1, n + 2});
    circs.push_back(circ_of(tris.back()));
    std::vector<char> bad;
    std::vector<int> bads;
    struct Edge { int a, b; };
    std::vector<Edge> poly;
    std::vector<Tri> keep;
    std::vector<Circ> keepc;
    for (int p = 0; p < n; ++p) {
        bad.assign(tris.size(), 0);
        bads.clear();
        const double px = (double)X[p], py = (double)Y[p];
        for (size_t t = 0; t < tris.size(); ++t) {
            const Circ& C = circs[t];
            if (C.r2 >= 0.0) {
                const double dx = px - C.x, dy = py - C.y;
                if (dx * dx + dy * dy > C.r2 * (1.0 + 1e-7) + 1.0) continue;
            }
            const Tri& T = tris[t];
            if (incircle_i(X[T.a], Y[T.a], X[T.b], Y[T.b], X[T.c], Y[T.c], X[p], Y[p]) > 0) {
                bad[t] = 1;
                bads.push_back((int)t);
            }
        }
        // the cavity's boundary: the bad triangles' edges that no other bad
        // triangle shares
        poly.clear();
        for (const int t : bads) {
            const int e[3][2] = {{tris[t].a, tris[t].b}, {tris[t].b, tris[t].c}, {tris[t].c, tris[t].a}};
            for (auto& ed : e) {
                bool shared = false;
                for (size_t k = 0; k < bads.size() && !shared; ++k) {
                    const int u = bads[k];
                    if (u == t) continue;
                    const int f[3][2] = {{tris[u].a, tris[u].b}, {tris[u].b, tris[u].c}, {tris[u].c, tris[u].a}};
                    for (auto& fd : f)
                        if ((fd[0] == ed[1] && fd[1] == ed[0]) || (fd[0] == ed[0] && fd[1] == ed[1])) shared = true;
                }
                if (!shared) poly.push_back({ed[0], ed[1]});
            }
        }
        keep.clear();
        keepc.clear();
        for (size_t t = 0; t < tris.size(); ++t)
            if (!bad[t]) {
                keep.push_back(tris[t]);
                keepc.push_back(circs[t]);
            }
        for (const Edge& e : poly) {
            // A point on an existing edge of a bad triangle forms a flat
            // triangle with it; leave that one out.
            if (orient_i(X[e.a], Y[e.a], X[e.b], Y[e.b], X[p], Y[p]) > 0) {
                keep.push_back({e.a, e.b, p});
                keepc.push_back(circ_of(keep.back()));
            }
        }
        tris.swap(keep);
        circs.swap(keepc);
    }
    for (const Tri& t : tris) {
        if (t.a >= n || t.b >= n || t.c >= n) continue;
        out.push_back(t);
    }
    auto key = [](const Tri& t) {
        int v[3] = {t.a, t.b, t.c};
        std::sort(v, v + 3);
        return std::make_tuple(v[0], v[1], v[2]);
    };
    std::sort(out.begin(), out.end(), [&](const Tri& a, const Tri& b) { return key(a) < key(b); });
    return out;
}

// The affine map taking src[k] to dst[k] (k = 0..2): X = M00 x + M01 y + M02,
// Y = M10 x + M11 y + M12. False for collinear sources.
inline bool affine3(const Pt src[3], const Pt dst[3], double M[6]) {
    const double x0 = src[0].x, y0 = src[0].y, x1 = src[1].x, y1 = src[1].y, x2 = src[2].x,
                 y2 = src[2].y;
    const double det = x0 * (y1 - y2) - y0 * (x1 - x2) + (x1 * y2 - x2 * y1);
    if (!(std::fabs(det) > 0.0)) return false;
    for (int r = 0; r < 2; ++r) {
        const double b0 = r == 0 ? dst[0].x : dst[0].y;
        const double b1 = r == 0 ? dst[1].x : dst[1].y;
        const double b2 = r == 0 ? dst[2].x : dst[2].y;
        // Cramer's rule on [x y 1] m = b.
        const double da = b0 * (y1 - y2) - y0 * (b1 - b2) + (b1 * y2 - b2 * y1);
        const double db = x0 * (b1 - b2) - b0 * (x1 - x2) + (x1 * b2 - x2 * b1);
        const double dc = x0 * (y1 * b2 - y2 * b1) - y0 * (x1 * b2 - x2 * b1) + b0 * (x1 * y2 - x2 * y1);
        M[3 * r + 0] = da / det;
        M[3 * r + 1] = db / det;
        M[3 * r + 2] = dc / det;
    }
    return true;
}

// Signed distance from p to the triangle's boundary: positive inside, zero on
// an edge, negative outside (the pointPolygonTest convention).
inline double tri_signed_distance(const Pt v[3], Pt p) {
    double best = 1e300;
    for (int k = 0; k < 3; ++k) {
        const Pt a = v[k], b = v[(k + 1) % 3];
        const double ex = b.x - a.x, ey = b.y - a.y;
        const double px = p.x - a.x, py = p.y - a.y;
        const double len2 = ex * ex + ey * ey;
        double t = len2 > 0.0 ? (px * ex + py * ey) / len2 : 0.0;
        t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
        const double dx = px - t * ex, dy = py - t * ey;
        best = std::min(best, dx * dx + dy * dy);
    }
    const double d = std::sqrt(best);
    // Inside/on test on exact integers (grid coordinates).
    const int64_t X[3] = {std::llround(v[0].x), std::llround(v[1].x), std::llround(v[2].x)};
    const int64_t Y[3] = {std::llround(v[0].y), std::llround(v[1].y), std::llround(v[2].y)};
    const int64_t qx = std::llround(p.x), qy = std::llround(p.y);
    const int64_t o0 = orient_i(X[0], Y[0], X[1], Y[1], qx, qy);
    const int64_t o1 = orient_i(X[1], Y[1], X[2], Y[2], qx, qy);
    const int64_t o2 = orient_i(X[2], Y[2], X[0], Y[0], qx, qy);
    const bool has_neg = o0 < 0 || o1 < 0 || o2 < 0, has_pos = o0 > 0 || o1 > 0 || o2 > 0;
    if (!(has_neg && has_pos)) return d;  // inside or on the boundary
    return -d;
}

// Inside or on the boundary, exactly (integer coordinates).
inline bool tri_contains(const int64_t X[3], const int64_t Y[3], int64_t qx, int64_t qy) {
    const int64_t o0 = orient_i(X[0], Y[0], X[1], Y[1], qx, qy);
    const int64_t o1 = orient_i(X[1], Y[1], X[2], Y[2], qx, qy);
    const int64_t o2 = orient_i(X[2], Y[2], X[0], Y[0], qx, qy);
    const bool has_neg = o0 < 0 || o1 < 0 || o2 < 0, has_pos = o0 > 0 || o1 > 0 || o2 > 0;
    return !(has_neg && has_pos);
}

// Area of the convex hull (monotone chain), shoelace in double.
inline double hull_area(std::vector<Pt> p) {
    if (p.size() < 3) return 0.0;
    std::sort(p.begin(), p.end(), [](const Pt& a, const Pt& b) { return a.x < b.x || (a.x == b.x && a.y < b.y); });
    std::vector<Pt> h(2 * p.size());
    size_t k = 0;
    auto cross = [](const Pt& o, const Pt& a, const Pt& b) {
        return (a.x - o.x) * (b.y - o.y) - (a.y - o.y) * (b.x - o.x);
    };
    for (size_t i = 0; i < p.size(); ++i) {
        while (k >= 2 && cross(h[k - 2], h[k - 1], p[i]) <= 0) --k;
        h[k++] = p[i];
    }
    for (size_t i = p.size() - 1, t = k + 1; i > 0; --i) {
        while (k >= t && cross(h[k - 2], h[k - 1], p[i - 1]) <= 0) --k;
        h[k++] = p[i - 1];
    }
    h.resize(k - 1);
    double a = 0.0;
    for (size_t i = 0; i < h.size(); ++i) {
        const Pt& u = h[i];
        const Pt& v = h[(i + 1) % h.size()];
        a += u.x * v.y - v.x * u.y;
    }
    return std::fabs(a) * 0.5;
}

// Jacobi eigen-decomposition of a symmetric n x n matrix (n <= 9): on return
// d holds the eigenvalues and V (row-major, column k = eigenvector k).
inline void jacobi_eig(int n, double* A, double* d, double* V) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) V[i * n + j] = i == j ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[i * n + j] * A[i * n + j];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[p * n + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double app = A[p * n + p], aqq = A[q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[k * n + p], akq = A[k * n + q];
                    A[k * n + p] = c * akp - s * akq;
                    A[k * n + q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[p * n + k], aqk = A[q * n + k];
                    A[p * n + k] = c * apk - s * aqk;
                    A[q * n + k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[k * n + p], vkq = V[k * n + q];
                    V[k * n + p] = c * vkp - s * vkq;
                    V[k * n + q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; ++i) d[i] = A[i * n + i];
}

// Normalised DLT homography over the points flagged in `use`.
inline bool dlt_homography(const std::vector<Pt>& src, const std::vector<Pt>& dst,
                           const std::vector<char>& use, double H[9]) {
    int m = 0;
    double sx = 0, sy = 0, dx = 0, dy = 0;
    for (size_t i = 0; i < src.size(); ++i)
        if (use[i]) { sx += src[i].x; sy += src[i].y; dx += dst[i].x; dy += dst[i].y; ++m; }
    if (m < 4) return false;
    sx /= m; sy /= m; dx /= m; dy /= m;
    double ss = 0, ds = 0;
    for (size_t i = 0; i < src.size(); ++i)
        if (use[i]) {
            ss += std::hypot(src[i].x - sx, src[i].y - sy);
            ds += std::hypot(dst[i].x - dx, dst[i].y - dy);
        }
    ss = ss > 0 ? std::sqrt(2.0) * m / ss : 1.0;
    ds = ds > 0 ? std::sqrt(2.0) * m / ds : 1.0;
    double AtA[81] = {};
    for (size_t i = 0; i < src.size(); ++i) {
        if (!use[i]) continue;
        const double x = (src[i].x - sx) * ss, y = (src[i].y - sy) * ss;
        const double X = (dst[i].x - dx) * ds, Y = (dst[i].y - dy) * ds;
        const double r1[9] = {-x, -y, -1, 0, 0, 0, X * x, X * y, X};
        const double r2[9] = {0, 0, 0, -x, -y, -1, Y * x, Y * y, Y};
        for (int a = 0; a < 9; ++a)
            for (int b = 0; b < 9; ++b) AtA[a * 9 + b] += r1[a] * r1[b] + r2[a] * r2[b];
    }
    double d[9], V[81];
    jacobi_eig(9, AtA, d, V);
    int k = 0;
    for (int i = 1; i < 9; ++i)
        if (d[i] < d[k]) k = i;
    double Hn[9];
    for (int i = 0; i < 9; ++i) Hn[i] = V[i * 9 + k];
    // H = Tdst^-1 Hn Tsrc
    const double Ts[9] = {ss, 0, -ss * sx, 0, ss, -ss * sy, 0, 0, 1};
    const double Tdi[9] = {1 / ds, 0, dx, 0, 1 / ds, dy, 0, 0, 1};
    double tmp[9] = {}, out[9] = {};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int q = 0; q < 3; ++q) tmp[r * 3 + c] += Hn[r * 3 + q] * Ts[q * 3 + c];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            for (int q = 0; q < 3; ++q) out[r * 3 + c] += Tdi[r * 3 + q] * tmp[q * 3 + c];
    if (!(std::fabs(out[8]) > 1e-300)) return false;
    for (int i = 0; i < 9; ++i) H[i] = out[i] / out[8];
    for (int i = 0; i < 9; ++i)
        if (!std::isfinite(H[i])) return false;
    return true;
}

// Homography fit with outlier rejection at `tol` px: fit all, drop points off
// by more than tol, refit until the inlier set is stable (at most 8 rounds).
// Deterministic, unlike RANSAC; on clean anchors it keeps every point and
// agrees with a least-squares fit, which is what the RANSAC refit converges to.
inline bool fit_homography(const std::vector<Pt>& src, const std::vector<Pt>& dst, double tol, double H[9]) {
    std::vector<char> use(src.size(), 1);
    if (!dlt_homography(src, dst, use, H)) return false;
    for (int round = 0; round < 8; ++round) {
        std::vector<char> nu(src.size(), 0);
        int m = 0;
        for (size_t i = 0; i < src.size(); ++i) {
            const double w = H[6] * src[i].x + H[7] * src[i].y + H[8];
            if (!(std::fabs(w) > 1e-12)) continue;
            const double X = (H[0] * src[i].x + H[1] * src[i].y + H[2]) / w;
            const double Y = (H[3] * src[i].x + H[4] * src[i].y + H[5]) / w;
            if (std::hypot(X - dst[i].x, Y - dst[i].y) <= tol) { nu[i] = 1; ++m; }
        }
        if (m < 4) return false;
        if (nu == use) break;
        use = nu;
        if (!dlt_homography(src, dst, use, H)) return false;
    }
    return true;
}

// seeding::homography_at (src/pipeline/akaze_features.cpp:184-198).
inline bool homography_at(const double h[9], double px, double py, double& X, double& Y, double J[4]) {
    const double w = h[6] * px + h[7] * py + h[8];
    if (!std::isfinite(w) || std::fabs(w) < 1e-12) return false;
    X = (h[0] * px + h[1] * py + h[2]) / w;
    Y = (h[3] * px + h[4] * py + h[5]) / w;
    J[0] = (h[0] - X * h[6]) / w;
    J[1] = (h[1] - X * h[7]) / w;
    J[2] = (h[3] - Y * h[6]) / w;
    J[3] = (h[4] - Y * h[7]) / w;
    return std::isfinite(X) && std::isfinite(Y) && std::isfinite(J[0]) && std::isfinite(J[1]) &&
           std::isfinite(J[2]) && std::isfinite(J[3]);
}

}  // namespace semper_geom
