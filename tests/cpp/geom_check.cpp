// The product's planar geometry (semper-dic-engine_b200/csrc/host/geometry.hpp)
// against the oracle's own (oracle/src/geom.hpp) on seeded point sets: the
// same triangles with the same vertex order, and the same bits from every
// floating-point helper. Prints one line per case and exits non-zero on the
// first difference.
#include <cstdio>
#include <cstring>
#include <random>

#include "geom.hpp"
#include "geometry.hpp"

namespace P = semper_geom;
namespace O = oracle_geom;

static int fails = 0;
#define REQUIRE(c, ...)                      \
    do {                                     \
        if (!(c)) {                          \
            std::printf("FAIL " __VA_ARGS__); \
            std::printf("\n");               \
            ++fails;                         \
        }                                    \
    } while (0)

static bool same(double a, double b) { return std::memcmp(&a, &b, sizeof a) == 0; }

static void check_set(const char* name, const std::vector<P::Pt>& pp, std::mt19937_64& rng) {
    std::vector<O::Pt> op;
    for (const auto& p : pp) op.push_back({p.x, p.y});
    const auto tp = P::delaunay(pp);
    const auto to = O::delaunay(op);
    REQUIRE(tp.size() == to.size(), "%s: %zu vs %zu triangles", name, tp.size(), to.size());
    for (size_t i = 0; i < tp.size() && i < to.size(); ++i)
        REQUIRE(tp[i].a == to[i].a && tp[i].b == to[i].b && tp[i].c == to[i].c, "%s: triangle %zu", name, i);
    // affine maps of every triangle under a random smooth displacement
    std::uniform_real_distribution<double> U(-3.0, 3.0);
    size_t probes = 0;
    for (size_t i = 0; i < tp.size() && i < to.size(); ++i) {
        const int v[3] = {tp[i].a, tp[i].b, tp[i].c};
        P::Pt ps[3], pd[3];
        O::Pt os[3], od[3];
        for (int k = 0; k < 3; ++k) {
            ps[k] = pp[v[k]];
            const double du = U(rng), dv = U(rng);
            pd[k] = {pp[v[k]].x + du, pp[v[k]].y + dv};
            os[k] = {ps[k].x, ps[k].y};
            od[k] = {pd[k].x, pd[k].y};
        }
        double Mp[6], Mo[6];
        const bool bp = P::affine3(ps, pd, Mp), bo = O::affine3(os, od, Mo);
        REQUIRE(bp == bo, "%s: affine3 %zu", name, i);
        for (int k = 0; bp && bo && k < 6; ++k) REQUIRE(same(Mp[k], Mo[k]), "%s: affine3 %zu bits", name, i);
        // distances and containment for points around the triangle
        for (int q = 0; q < 4; ++q) {
            const double qx = std::round(ps[q % 3].x + U(rng) * 4), qy = std::round(ps[q % 3].y + U(rng) * 4);
            REQUIRE(same(P::tri_signed_distance(ps, {qx, qy}), O::signed_distance(os, {qx, qy})),
                    "%s: distance %zu", name, i);
            int64_t X[3], Y[3];
            for (int k = 0; k < 3; ++k) {
                X[k] = std::llround(ps[k].x);
                Y[k] = std::llround(ps[k].y);
            }
            REQUIRE(P::tri_contains(X, Y, (int64_t)qx, (int64_t)qy) == O::in_triangle(X, Y, (int64_t)qx, (int64_t)qy),
                    "%s: contains %zu", name, i);
            ++probes;
        }
    }
    REQUIRE(same(P::hull_area(pp), O::hull_area(op)), "%s: hull area", name);
    // homography refits: a rotation-scale-translation with a little
    // perspective, noise, and a few outliers
    std::normal_distribution<double> N(0.0, 0.3);
    const double th = U(rng) * 0.4, sc = 1.0 + U(rng) * 0.01, p6 = U(rng) * 1e-6, p7 = U(rng) * 1e-6;
    std::vector<P::Pt> dp;
    std::vector<O::Pt> dq;
    for (size_t i = 0; i < pp.size(); ++i) {
        const double x = pp[i].x, y = pp[i].y, w = 1.0 + p6 * x + p7 * y;
        double X = (sc * (std::cos(th) * x - std::sin(th) * y) + 12.5) / w + N(rng);
        double Y = (sc * (std::sin(th) * x + std::cos(th) * y) - 7.25) / w + N(rng);
        if (i % 17 == 5) X += 40.0;
        dp.push_back({X, Y});
        dq.push_back({X, Y});
    }
    for (const double tol : {1.0, 3.0, 6.0}) {
        double Hp[9], Ho[9];
        const bool bp = P::fit_homography(pp, dp, tol, Hp), bo = O::fit_homography(op, dq, tol, Ho);
        REQUIRE(bp == bo, "%s: homography fit at %g", name, tol);
        for (int k = 0; bp && bo && k < 9; ++k) REQUIRE(same(Hp[k], Ho[k]), "%s: homography bits at %g", name, tol);
        if (bp && bo)
            for (size_t i = 0; i < pp.size(); i += 7) {
                double Xp, Yp, Jp[4], Xo, Yo, Jo[4];
                const bool ap = P::homography_at(Hp, pp[i].x, pp[i].y, Xp, Yp, Jp);
                const bool ao = O::homography_at(Ho, pp[i].x, pp[i].y, Xo, Yo, Jo);
                REQUIRE(ap == ao && same(Xp, Xo) && same(Yp, Yo), "%s: homography_at", name);
                for (int k = 0; ap && ao && k < 4; ++k) REQUIRE(same(Jp[k], Jo[k]), "%s: jacobian", name);
            }
    }
    std::printf("%s: %zu points, %zu triangles, %zu probes\n", name, pp.size(), tp.size(), probes);
}

int main() {
    std::mt19937_64 rng(20260);
    // random integer points
    for (int t = 0; t < 6; ++t) {
        std::uniform_int_distribution<int> C(0, t < 3 ? 400 : 4000);
        std::vector<P::Pt> pts;
        for (int i = 0; i < 40 + 60 * t; ++i) pts.push_back({(double)C(rng), (double)C(rng)});
        char name[32];
        std::snprintf(name, sizeof name, "random %d", t);
        check_set(name, pts, rng);
    }
    // full lattices (every cell co-circular), in row order and shuffled
    for (int t = 0; t < 4; ++t) {
        std::vector<P::Pt> pts;
        const int nx = 6 + 5 * t, ny = 5 + 4 * t, sx = 8 * (t + 1), sy = 12 * (t + 1);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) pts.push_back({(double)(100 + i * sx), (double)(40 + j * sy)});
        if (t % 2) std::shuffle(pts.begin(), pts.end(), rng);
        char name[32];
        std::snprintf(name, sizeof name, "lattice %d", t);
        check_set(name, pts, rng);
    }
    // anchor lattices with holes (anchors that failed)
    for (int t = 0; t < 4; ++t) {
        std::bernoulli_distribution keep(0.8);
        std::vector<P::Pt> pts;
        for (int j = 0; j < 18; ++j)
            for (int i = 0; i < 18; ++i)
                if (keep(rng)) pts.push_back({(double)(676 + i * 161), (double)(676 + j * 161)});
        char name[32];
        std::snprintf(name, sizeof name, "anchors %d", t);
        check_set(name, pts, rng);
    }
    std::printf(fails ? "%d differences\n" : "same\n", fails);
    return fails ? 1 : 0;
}
