// ORACLE — test infrastructure only. Never linked into the product library.
//
// The full-field solve restated from the reference's orchestration:
//   validate_params / clip_axis      src/pipeline/full_field_solver.cpp:77-117
//   run_full_field_impl              src/pipeline/full_field_solver.cpp:141-586
//   plan_anchor_lattice, mark_kept   src/pipeline/full_field_anchors.cpp:64-168
//   solve_anchor_seeds (lattice)     src/pipeline/full_field_anchors.cpp:283-574
//   publish_anchor_results           src/pipeline/full_field_anchors.cpp:576-607
//   build_mesh_guess_field           src/pipeline/full_field_mesh.cpp:32-282
//   run_path_a / _b / _c             src/pipeline/full_field_path_{a,b,c}.cpp
//   pack_full_field_output, metrics  src/pipeline/full_field_solver_stats.cpp:21-91,182-280
//
// The global-motion model (the reference's AKAZE homography, OpenCV) is an
// input here: none, or a 3x3 homography supplied by the caller. The planar
// geometry that the reference takes from OpenCV is the oracle's own (geom.hpp),
// under the rules the build fixed for it.
#pragma once
#include <chrono>
#include <cstdint>
#include <deque>
#include <queue>
#include <vector>

#include "geom.hpp"
#include "solver.hpp"
#include "strain.hpp"

namespace oracle {

constexpr float kCorrInvalid = -1.0f;
constexpr float kAnchorSparseCoverage = 0.05f;
constexpr int kAnchorTarget = 256;
constexpr int kAnchorStrideMin = 1;
constexpr float kAnchorAcceptScore = 0.40f;
constexpr float kAnchorMedianTol = 1.0f;
constexpr float kAnchorFullFraction = 0.60f;
constexpr int kAnchorFullMinVertices = 10;
constexpr float kAnchorFullCoverage = 0.30f;
constexpr double kAnchorRefitRansacPx = 1.0;
constexpr int kAnchorRefitMinPoints = 8;
constexpr float kSimilarityMinCornerPx = 4.0f;
constexpr float kSimilarityKeepFraction = 0.90f;
constexpr int kPathCMaxCandidates = 9;
constexpr int kPathBBatchNodes = 32;
constexpr int kMetricsLen = 24;

enum MeshAssign { kMeshNone = 0, kMeshInTriangle = 1, kMeshExtrapolated = 2, kMeshAnchor = 3, kMeshHomography = 4 };
enum class MeshQuality { NONE, SPARSE, FULL };

struct Params {
    int rect_x = 0, rect_y = 0, rect_w = 0, rect_h = 0, step = 0, subset_size = 0, strain_window = 0;
    bool six = false;
};

struct GridPoint {
    float x = 0, y = 0, u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0, corr = 0;
    bool solved = false;
    int mesh = kMeshNone;
    bool used_simplex = false;
    int icgn_iters = 0;
};

// Per-node result of a solve, for callers that build on the raw field
// (FieldCapture, src/pipeline/full_field_internal.hpp:247-261).
struct Capture {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0, attempted = 0;
    std::vector<GridPoint> grid;
};

inline int metrics_prefix_len(int len) {
    return len < 16 ? 0 : len >= kMetricsLen ? kMetricsLen : len == 18 ? 17 : len;
}

inline bool clip_axis(int& lo, int& len, int step, int extent) {
    int64_t a = lo;
    const int64_t b = std::min<int64_t>((int64_t)lo + (int64_t)len, extent);
    if (a < 0) a += ((-a + step - 1) / step) * (int64_t)step;
    if (b <= a) return false;
    lo = (int)a;
    len = (int)(b - a);
    return true;
}

inline int64_t max_strain_window(const Params& p) {
    if (p.step <= 0) return 0;
    const int64_t gmin = std::min(p.rect_w / p.step, p.rect_h / p.step);
    return 2 * (gmin + 1) * (int64_t)p.step;
}

inline int validate_params(Params& p, int width, int height) {
    if (width <= 0 || height <= 0) return -3;
    if ((int64_t)width * (int64_t)height > (int64_t)INT32_MAX) return -3;
    if (p.step <= 0) return -2;
    if (p.subset_size < 3 || p.subset_size % 2 == 0) return -3;
    if (p.rect_w <= 0 || p.rect_h <= 0) return -2;
    if (!clip_axis(p.rect_x, p.rect_w, p.step, width)) return -2;
    if (!clip_axis(p.rect_y, p.rect_h, p.step, height)) return -2;
    if (p.rect_w / p.step <= 0 || p.rect_h / p.step <= 0) return -2;
    if ((int64_t)p.strain_window > max_strain_window(p)) return -3;
    return 0;
}

inline int lattice_count(int n, int stride) {
    if (n <= 0 || stride <= 0) return 0;
    int c = (n + stride - 1) / stride;
    if ((c - 1) * stride != n - 1) c++;
    return c;
}

struct Lattice {
    int sx = 1, sy = 1, nx = 0, ny = 0;
};

inline Lattice plan_lattice(int gw, int gh) {
    Lattice out;
    if (gw <= 0 || gh <= 0) return out;
    int stride = (int)std::lround(std::sqrt((double)(gw * gh) / (double)kAnchorTarget));
    stride = std::max(kAnchorStrideMin, stride);
    const int budget = lattice_count(gw, stride) * lattice_count(gh, stride);
    int sx = stride, sy = stride;
    while (sx > 1 && lattice_count(gw, sx) < 3) --sx;
    while (sy > 1 && lattice_count(gh, sy) < 3) --sy;
    while (lattice_count(gw, sx) * lattice_count(gh, sy) > budget) {
        const bool gx = lattice_count(gw, sx + 1) >= 3, gy = lattice_count(gh, sy + 1) >= 3;
        if (!gx && !gy) break;
        if (gx && (!gy || lattice_count(gw, sx) >= lattice_count(gh, sy))) ++sx;
        else ++sy;
    }
    out.sx = sx;
    out.sy = sy;
    out.nx = lattice_count(gw, sx);
    out.ny = lattice_count(gh, sy);
    return out;
}

struct Anchor {
    int gx = 0, gy = 0;
    float rx = 0, ry = 0, u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0, corr = 0;
    int iters = 0;
    bool used_simplex = false, vertex = false, output = false, kept = false;
};

// mark_kept_anchors (full_field_anchors.cpp:122-168).
inline void mark_kept(std::vector<Anchor>& a, int LW, int LH, const std::vector<float>& ru,
                      const std::vector<float>& rv) {
    for (int lj = 0; lj < LH; ++lj)
        for (int li = 0; li < LW; ++li) {
            const size_t idx = (size_t)lj * LW + li;
            a[idx].kept = false;
            if (!a[idx].vertex) continue;
            std::vector<float> nu, nv;
            for (int dj = -1; dj <= 1; ++dj)
                for (int di = -1; di <= 1; ++di) {
                    if (di == 0 && dj == 0) continue;
                    const int nj = lj + dj, ni = li + di;
                    if (ni < 0 || ni >= LW || nj < 0 || nj >= LH) continue;
                    const size_t k = (size_t)nj * LW + ni;
                    if (!a[k].vertex) continue;
                    nu.push_back(ru[k]);
                    nv.push_back(rv[k]);
                }
            if (nu.size() < 3) continue;
            const float mu = median_of(nu), mv = median_of(nv);
            if (std::fabs(ru[idx] - mu) > kAnchorMedianTol || std::fabs(rv[idx] - mv) > kAnchorMedianTol) continue;
            a[idx].kept = true;
        }
}

struct Stats {
    int icgn_iters = 0, points = 0, simp_calls = 0, simp_saved = 0, simp_dead = 0;
    double icgn_ms = 0, simp_ms = 0;
};

template <class T>
inline void record_simplex(Stats& s, const Result<T>& r) {
    s.simp_calls++;
    if (r.status == 0 && r.score <= T(kCorrAccept)) s.simp_saved++;
    else s.simp_dead++;
}

template <class T>
struct RefCache {
    bool has = false;
    int width = 0, height = 0;
    Image<T> ref;
    // grid scan + Hessian pool, keyed on the grid and the mask
    bool grid_valid = false;
    Params key;
    std::vector<uint8_t> mask_key;
    int gridW = 0, gridH = 0, total_valid = 0;
    std::vector<unsigned char> skip;
    std::vector<PoolEntry<T>> pool;

    void set(int w, int h, const uint8_t* gray, const uint8_t* mask) {
        has = true;
        width = w;
        height = h;
        ref.prepare(w, h, gray);
        ref.stamp_ghost_wall(mask);
        grid_valid = false;
    }
};

struct SolveInfo {
    MeshQuality quality = MeshQuality::NONE;
    float coverage = 0;
    bool locked = false;
    int accepted = 0, attempted = 0, solved = 0;
};

struct PackOut {
    int valid_count = 0, dropped_outlier = 0, dropped_post = 0;
};

// pack_full_field_output (full_field_solver_stats.cpp:21-91) over a grid:
// the displacement median test, VSG strain, then the row-major packing of
// the first points that fit, strain failures dropped.
inline PackOut pack_field(const std::vector<GridPoint>& grid, int gridW, int gridH, int step, int window, float* out,
                          int capacity) {
    PackOut po;
    const size_t NG = (size_t)gridW * gridH;
    DispField df;
    df.width = gridW; df.height = gridH; df.step = step;
    df.u.assign(NG, 0.f); df.v.assign(NG, 0.f); df.valid.assign(NG, 0);
    for (size_t i = 0; i < NG; ++i)
        if (grid[i].solved && grid[i].corr >= 0.f) {
            df.u[i] = grid[i].u;
            df.v[i] = grid[i].v;
            df.valid[i] = 1;
        }
    po.dropped_outlier = reject_outliers(df);
    const StrainOut so = vsg_strain(df, window);
    bool trunc = false;
    for (int y = 0; y < gridH && !trunc; ++y)
        for (int x = 0; x < gridW; ++x) {
            const size_t idx = (size_t)y * gridW + x;
            if (!df.valid[idx]) continue;
            if ((po.valid_count + 1) * 8 > capacity) { trunc = true; break; }
            if (so.exx[idx] <= kStrainFailSentinel) { po.dropped_post++; continue; }
            float* o = out + (size_t)po.valid_count * 8;
            o[0] = grid[idx].x; o[1] = grid[idx].y; o[2] = df.u[idx]; o[3] = df.v[idx];
            o[4] = so.exx[idx]; o[5] = so.eyy[idx]; o[6] = so.exy[idx]; o[7] = grid[idx].corr;
            po.valid_count++;
        }
    return po;
}

template <class T>
int run_full_field(RefCache<T>& cache, const uint8_t* def_gray, const uint8_t* mask, Params params,
                   float* out, int capacity, float* metrics, int metrics_len, const double* model_H,
                   Capture* capture = nullptr, Image<T>* keep_def = nullptr, const float* anchor_uv = nullptr,
                   int anchor_n = 0) {
    using clk = std::chrono::high_resolution_clock;
    auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
    const auto t_total = clk::now();
    if (out == nullptr || !cache.has || def_gray == nullptr) return -3;
    const int rc = validate_params(params, cache.width, cache.height);
    if (rc != 0) return rc;
    if (capacity < 0) capacity = 0;
    const int W = cache.width, H = cache.height;

    Image<T> def;
    def.prepare(W, H, def_gray);

    const int gridW = params.rect_w / params.step, gridH = params.rect_h / params.step;
    if (vsg_window_node_count(params.step, params.strain_window) < 3) return -4;

    std::vector<GridPoint> grid((size_t)gridW * gridH);
    auto G = [&](int x, int y) -> GridPoint& { return grid[(size_t)y * gridW + x]; };
    const bool cached = cache.grid_valid && cache.key.rect_x == params.rect_x &&
                        cache.key.rect_y == params.rect_y && cache.key.rect_w == params.rect_w &&
                        cache.key.rect_h == params.rect_h && cache.key.step == params.step &&
                        cache.key.subset_size == params.subset_size &&
                        cache.mask_key == (mask ? std::vector<uint8_t>(mask, mask + (size_t)W * H)
                                                : std::vector<uint8_t>()) &&
                        cache.gridW == gridW && cache.gridH == gridH;
    int total_valid = 0;
    const auto t_prepass = clk::now();
    if (cached) {
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                GridPoint& g = G(x, y);
                g.x = (float)(params.rect_x + x * params.step);
                g.y = (float)(params.rect_y + y * params.step);
                g.corr = kCorrInvalid;
                g.solved = cache.skip[(size_t)y * gridW + x] != 0;
            }
        total_valid = cache.total_valid;
    } else {
        cache.grid_valid = false;
        const int hs = params.subset_size / 2, buf = hs + 4 + 15;
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                const int rx = params.rect_x + x * params.step, ry = params.rect_y + y * params.step;
                bool skip = rx - buf < 0 || rx + buf >= W || ry - buf < 0 || ry + buf >= H;
                if (!skip && mask) {
                    for (int dy = -hs; dy <= hs && !skip; ++dy)
                        for (int dx = -hs; dx <= hs; ++dx)
                            if (mask[(size_t)(ry + dy) * W + rx + dx] < 128) { skip = true; break; }
                }
                if (!skip) ++total_valid;
                GridPoint& g = G(x, y);
                g.x = (float)rx;
                g.y = (float)ry;
                g.corr = kCorrInvalid;
                g.solved = skip;
            }
    }
    if (total_valid == 0) return -2;

    if (!cached) {
        cache.pool.assign((size_t)gridW * gridH, PoolEntry<T>());
#pragma omp parallel for schedule(static)
        for (int i = 0; i < gridW * gridH; ++i) {
            const int gx = i % gridW, gy = i / gridW;
            if (grid[i].solved) continue;
            cache.pool[i] = compute_hessian_only(cache.ref, params.rect_x + gx * params.step,
                                                 params.rect_y + gy * params.step, params.subset_size);
        }
        cache.key = params;
        cache.mask_key = mask ? std::vector<uint8_t>(mask, mask + (size_t)W * H) : std::vector<uint8_t>();
        cache.gridW = gridW;
        cache.gridH = gridH;
        cache.skip.assign((size_t)gridW * gridH, 0);
        for (size_t i = 0; i < grid.size(); ++i) cache.skip[i] = grid[i].solved ? 1 : 0;
        cache.total_valid = total_valid;
        cache.grid_valid = true;
    }
    const double ms_prepass = ms_since(t_prepass);
    const std::vector<PoolEntry<T>>& pool = cache.pool;
    const int dim = params.subset_size;

    auto solve_at = [&](Engine<T>& eng, Subset<T>& sub, int gx, int gy, const T g[6], InitMode mode) {
        return solve_node(eng, sub, cache.ref, def, params.rect_x + gx * params.step,
                          params.rect_y + gy * params.step, dim, pool[(size_t)gy * gridW + gx], g, mode);
    };
    auto make_engine = [&]() {
        Engine<T> e;
        e.lm = true;
        e.six = params.six;
        return e;
    };

    // ------------------------------------------------ anchor lattice (L1) --
    const auto t_seed = clk::now();
    Stats st_anchor, st_a, st_b;
    SolveInfo seeds;
    std::vector<Anchor> anchors;
    std::vector<oracle_geom::Pt> ref_pts, def_pts;
    float globalU = 0, globalV = 0;
    bool have_model = model_H != nullptr, model_full = false, model_rejected = false;
    double t_u = 0, t_v = 0;
    const double gcx = params.rect_x + 0.5 * params.rect_w, gcy = params.rect_y + 0.5 * params.rect_h;
    auto model_at = [&](double x, double y, float g6[6]) {
        double X, Y, J[4];
        if (!oracle_geom::homography_at(model_H, x, y, X, Y, J)) return false;
        g6[0] = (float)(X - x); g6[1] = (float)(Y - y);
        g6[2] = (float)(J[0] - 1.0); g6[3] = (float)J[1];
        g6[4] = (float)J[2]; g6[5] = (float)(J[3] - 1.0);
        return true;
    };
    if (have_model) {
        float g6[6];
        if (!model_at(gcx, gcy, g6)) have_model = false;
        else {
            t_u = g6[0];
            t_v = g6[1];
            const double xs[2] = {(double)params.rect_x, (double)(params.rect_x + params.rect_w)};
            const double ys[2] = {(double)params.rect_y, (double)(params.rect_y + params.rect_h)};
            for (double x : xs)
                for (double y : ys)
                    if (!model_at(x, y, g6) || std::hypot(g6[0] - t_u, g6[1] - t_v) > kSimilarityMinCornerPx)
                        model_full = true;
        }
    }
    seeds.locked = have_model;
    std::vector<double> homography;  // empty = none
    if (have_model) homography.assign(model_H, model_H + 9);

    const Lattice lat = plan_lattice(gridW, gridH);
    std::vector<int> lat_x, lat_y;
    for (int gx = 0; gx < gridW; gx += lat.sx) lat_x.push_back(gx);
    if (lat_x.back() != gridW - 1) lat_x.push_back(gridW - 1);
    for (int gy = 0; gy < gridH; gy += lat.sy) lat_y.push_back(gy);
    if (lat_y.back() != gridH - 1) lat_y.push_back(gridH - 1);
    const int LW = (int)lat_x.size(), LH = (int)lat_y.size();

    auto solve_lattice = [&](bool sim) -> float {
        seeds = SolveInfo{};
        seeds.locked = have_model;
        globalU = (float)t_u;
        globalV = (float)t_v;
        ref_pts.clear();
        def_pts.clear();
        anchors.assign((size_t)LW * LH, Anchor{});
        const InitMode mode = have_model ? INIT_NO_SIMPLEX : INIT_AUTO_SEARCH;
        std::vector<NodeSolve<T>> ns(anchors.size());
        std::vector<char> tried(anchors.size(), 0);
        int attempted = 0;
        for (size_t i = 0; i < anchors.size(); ++i) {
            const int gx = lat_x[i % LW], gy = lat_y[i / LW];
            if (!G(gx, gy).solved) { tried[i] = 1; ++attempted; }
        }
#pragma omp parallel for schedule(dynamic, 4)
        for (int i = 0; i < (int)anchors.size(); ++i) {
            if (!tried[i]) continue;
            const int gx = lat_x[i % LW], gy = lat_y[i / LW];
            const int rx = params.rect_x + gx * params.step, ry = params.rect_y + gy * params.step;
            float gs[6] = {globalU, globalV, 0, 0, 0, 0};
            if (sim && !model_at(rx, ry, gs)) { gs[0] = globalU; gs[1] = globalV; gs[2] = gs[3] = gs[4] = gs[5] = 0; }
            // a per-anchor displacement guess under the model (the device's
            // learned seeding hands its network's guesses over here)
            if (sim && anchor_n == LW * LH && std::isfinite(anchor_uv[2 * i]) && std::isfinite(anchor_uv[2 * i + 1])) {
                gs[0] = anchor_uv[2 * i];
                gs[1] = anchor_uv[2 * i + 1];
            }
            T g[6];
            for (int k = 0; k < 6; ++k) g[k] = (T)gs[k];
            Engine<T> eng = make_engine();
            Subset<T> sub;
            ns[i] = solve_at(eng, sub, gx, gy, g, mode);
        }
        for (size_t i = 0; i < anchors.size(); ++i) {
            if (!tried[i] || !ns[i].initialized) continue;
            const Result<T>& r = ns[i].res;
            st_anchor.icgn_iters += r.iters;
            if (ns[i].rescue) record_simplex(st_anchor, r);
            if (r.status != 0) continue;
            Anchor& a = anchors[i];
            a.gx = lat_x[i % LW];
            a.gy = lat_y[i / LW];
            a.rx = (float)(params.rect_x + a.gx * params.step);
            a.ry = (float)(params.rect_y + a.gy * params.step);
            a.u = (float)r.u; a.v = (float)r.v; a.ux = (float)r.ux; a.uy = (float)r.uy;
            a.vx = (float)r.vx; a.vy = (float)r.vy; a.corr = (float)r.score;
            a.iters = r.iters;
            a.used_simplex = ns[i].rescue;
            a.vertex = (float)r.score <= kAnchorAcceptScore;
            a.output = (float)r.score <= kCorrAccept;
        }
        seeds.attempted = attempted;
        std::vector<float> ru(anchors.size(), 0.f), rv(anchors.size(), 0.f);
        for (size_t i = 0; i < anchors.size(); ++i) {
            const Anchor& a = anchors[i];
            if (!a.vertex) continue;
            float g[6] = {0, 0, 0, 0, 0, 0};
            if (sim && !model_at(a.rx, a.ry, g)) { g[0] = globalU; g[1] = globalV; }
            ru[i] = a.u - g[0];
            rv[i] = a.v - g[1];
        }
        mark_kept(anchors, LW, LH, ru, rv);
        std::vector<float> us, vs;
        for (const Anchor& a : anchors) {
            if (!a.kept) continue;
            ref_pts.push_back({(double)a.rx, (double)a.ry});
            def_pts.push_back({(double)(a.rx + a.u), (double)(a.ry + a.v)});
            us.push_back(a.u);
            vs.push_back(a.v);
            if (a.output) seeds.solved++;
        }
        seeds.accepted = (int)ref_pts.size();
        if (seeds.accepted >= 3) {
            globalU = median_of(us);
            globalV = median_of(vs);
            const float roi_area = (float)(params.rect_w * params.rect_h);
            seeds.coverage = roi_area > 0.f ? (float)oracle_geom::hull_area(ref_pts) / roi_area : 0.f;
        }
        const float frac = seeds.attempted > 0 ? (float)seeds.accepted / (float)seeds.attempted : 0.f;
        if (seeds.accepted >= kAnchorFullMinVertices && frac >= kAnchorFullFraction &&
            seeds.coverage >= kAnchorFullCoverage)
            seeds.quality = MeshQuality::FULL;
        else if (seeds.accepted >= 3 && seeds.coverage >= kAnchorSparseCoverage)
            seeds.quality = MeshQuality::SPARSE;
        else
            seeds.quality = MeshQuality::NONE;
        return frac;
    };

    if (LW >= 2 && LH >= 2) {
        if (!model_full) {
            solve_lattice(false);
        } else {
            const float kept = solve_lattice(true);
            if (seeds.quality != MeshQuality::FULL || kept < kSimilarityKeepFraction) {
                solve_lattice(false);
                model_rejected = true;
            }
        }
        bool refitted = false;
        if (seeds.accepted >= kAnchorRefitMinPoints) {
            double Hf[9];
            if (oracle_geom::fit_homography(ref_pts, def_pts, kAnchorRefitRansacPx, Hf)) {
                homography.assign(Hf, Hf + 9);
                refitted = true;
            }
        }
        if (model_rejected && !refitted) homography.clear();
    } else {
        globalU = (float)t_u;
        globalV = (float)t_v;
    }
    const double ms_seed = ms_since(t_seed);

    // publish_anchor_results
    for (const Anchor& a : anchors) {
        if (!a.output || !a.kept) continue;
        GridPoint& g = G(a.gx, a.gy);
        g.x = a.rx; g.y = a.ry; g.u = a.u; g.v = a.v; g.ux = a.ux; g.uy = a.uy; g.vx = a.vx; g.vy = a.vy;
        g.corr = a.corr;
        g.solved = true;
        g.mesh = kMeshAnchor;
        g.used_simplex = a.used_simplex;
        g.icgn_iters = a.iters;
        st_anchor.points++;
    }

    const bool have_seed = seeds.solved > 0 || seeds.accepted >= 3;
    const bool exec_c = seeds.quality == MeshQuality::NONE && !have_seed;

    // ------------------------------------------------------- mesh guesses --
    const auto t_mesh = clk::now();
    const size_t NG = (size_t)gridW * gridH;
    std::vector<float> gu(NG, globalU), gv(NG, globalV), gux(NG, 0.f), guy(NG, 0.f), gvx(NG, 0.f), gvy(NG, 0.f);
    std::vector<unsigned char> in_mesh(NG, 0);
    struct ATri { oracle_geom::Pt p[3]; int64_t X[3], Y[3]; double u, v, ux, uy, vx, vy; float bx, by, bw, bh; };
    std::vector<ATri> tris;
    {
        std::vector<oracle_geom::Pt> ins;
        std::vector<int> ins_of;
        for (size_t i = 0; i < ref_pts.size(); ++i)
            if (ref_pts[i].x > 0 && ref_pts[i].x < W && ref_pts[i].y > 0 && ref_pts[i].y < H) {
                ins.push_back(ref_pts[i]);
                ins_of.push_back((int)i);
            }
        for (const oracle_geom::Tri& t : oracle_geom::delaunay(ins)) {
            ATri at;
            const int vi[3] = {t.a, t.b, t.c};
            oracle_geom::Pt dst[3];
            for (int k = 0; k < 3; ++k) {
                at.p[k] = ins[vi[k]];
                dst[k] = def_pts[ins_of[vi[k]]];
                at.X[k] = std::llround(at.p[k].x);
                at.Y[k] = std::llround(at.p[k].y);
            }
            double M[6];
            if (!oracle_geom::affine3(at.p, dst, M)) continue;
            const double detF = M[0] * M[4] - M[1] * M[3];
            if (!std::isfinite(detF) || std::fabs(detF) <= 1e-3) continue;
            at.ux = M[0] - 1.0; at.uy = M[1]; at.vx = M[3]; at.vy = M[4] - 1.0; at.u = M[2]; at.v = M[5];
            const float mnx = (float)std::min({at.p[0].x, at.p[1].x, at.p[2].x});
            const float mxx = (float)std::max({at.p[0].x, at.p[1].x, at.p[2].x});
            const float mny = (float)std::min({at.p[0].y, at.p[1].y, at.p[2].y});
            const float mxy = (float)std::max({at.p[0].y, at.p[1].y, at.p[2].y});
            at.bx = mnx - 15.0f; at.by = mny - 15.0f; at.bw = (mxx - mnx) + 30.0f; at.bh = (mxy - mny) + 30.0f;
            tris.push_back(at);
        }
    }
    auto assign = [&](size_t idx, const ATri& t, double px, double py, int tag) {
        gu[idx] = (float)(t.ux * px + t.uy * py + t.u);
        gv[idx] = (float)(t.vx * px + t.vy * py + t.v);
        gux[idx] = (float)t.ux; guy[idx] = (float)t.uy; gvx[idx] = (float)t.vx; gvy[idx] = (float)t.vy;
        in_mesh[idx] = 1;
        grid[idx].mesh = tag;
    };
    for (int y = 0; y < gridH; ++y)
        for (int x = 0; x < gridW; ++x) {
            if (G(x, y).solved) continue;
            const float px = (float)(params.rect_x + x * params.step), py = (float)(params.rect_y + y * params.step);
            const size_t idx = (size_t)y * gridW + x;
            for (const ATri& t : tris) {
                if (px < t.bx || px > t.bx + t.bw || py < t.by || py > t.by + t.bh) continue;
                if (oracle_geom::in_triangle(t.X, t.Y, (int64_t)px, (int64_t)py)) {
                    assign(idx, t, px, py, kMeshInTriangle);
                    break;
                }
            }
        }
    if (seeds.quality == MeshQuality::FULL) {
        const float LIM = -3.0f * params.step;
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                const size_t idx = (size_t)y * gridW + x;
                if (in_mesh[idx] || grid[idx].solved) continue;
                const float px = (float)(params.rect_x + x * params.step), py = (float)(params.rect_y + y * params.step);
                float best = LIM - 1.0f;
                int bi = -1;
                for (size_t ti = 0; ti < tris.size(); ++ti) {
                    const ATri& t = tris[ti];
                    if (px < t.bx + LIM || px > t.bx + t.bw - LIM || py < t.by + LIM || py > t.by + t.bh - LIM) continue;
                    const double d = oracle_geom::signed_distance(t.p, {px, py});
                    if (d >= LIM && (float)d > best) { best = (float)d; bi = (int)ti; }
                }
                if (bi >= 0) assign(idx, tris[bi], px, py, kMeshExtrapolated);
            }
    }
    if (homography.size() == 9) {
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                const size_t idx = (size_t)y * gridW + x;
                if (in_mesh[idx] || grid[idx].solved) continue;
                const double px = params.rect_x + (double)x * params.step, py = params.rect_y + (double)y * params.step;
                double X, Y, J[4];
                if (!oracle_geom::homography_at(homography.data(), px, py, X, Y, J)) continue;
                gu[idx] = (float)(X - px); gv[idx] = (float)(Y - py);
                gux[idx] = (float)(J[0] - 1.0); guy[idx] = (float)J[1];
                gvx[idx] = (float)J[2]; gvy[idx] = (float)(J[3] - 1.0);
                in_mesh[idx] = 1;
                grid[idx].mesh = kMeshHomography;
            }
    }
    const float stepf = (float)params.step;
    auto smooth = [&](std::vector<float>& f, const std::vector<float>* ax, const std::vector<float>* ay) {
        const std::vector<float> tmp = f;
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                const size_t idx = (size_t)y * gridW + x;
                if (!in_mesh[idx]) continue;
                float sum = 0.f;
                int cnt = 0, sdx = 0, sdy = 0;
                for (int dy = -2; dy <= 2; ++dy)
                    for (int dx = -2; dx <= 2; ++dx) {
                        const int ny = y + dy, nx = x + dx;
                        if (nx >= 0 && nx < gridW && ny >= 0 && ny < gridH && in_mesh[(size_t)ny * gridW + nx]) {
                            sum += tmp[(size_t)ny * gridW + nx];
                            ++cnt; sdx += dx; sdy += dy;
                        }
                    }
                if (cnt == 0) continue;
                f[idx] = sum / cnt;
                if (ax && (sdx != 0 || sdy != 0))
                    f[idx] -= ((*ax)[idx] * sdx + (*ay)[idx] * sdy) * stepf / cnt;
            }
    };
    smooth(gux, nullptr, nullptr);
    smooth(guy, nullptr, nullptr);
    smooth(gvx, nullptr, nullptr);
    smooth(gvy, nullptr, nullptr);
    smooth(gu, &gux, &guy);
    smooth(gv, &gvx, &gvy);
    const double ms_mesh = ms_since(t_mesh);

    // ------------------------------------------------------------ Path C --
    int pc_x = gridW / 2, pc_y = gridH / 2;
    if (exec_c) {
        std::vector<int> cand;
        if (!ref_pts.empty()) {
            const float gcx2 = params.rect_x + (gridW / 2.f) * params.step, gcy2 = params.rect_y + (gridH / 2.f) * params.step;
            float md = 1e9f;
            int bi = -1;
            for (size_t i = 0; i < ref_pts.size(); ++i) {
                const float dx = (float)ref_pts[i].x - gcx2, dy = (float)ref_pts[i].y - gcy2;
                const float d = dx * dx + dy * dy;
                if (d < md) { md = d; bi = (int)i; }
            }
            if (bi >= 0) {
                const int gx = std::max(0, std::min(gridW - 1, (int)std::round(((float)ref_pts[bi].x - params.rect_x) / params.step)));
                const int gy = std::max(0, std::min(gridH - 1, (int)std::round(((float)ref_pts[bi].y - params.rect_y) / params.step)));
                if (!G(gx, gy).solved) cand.push_back(gy * gridW + gx);
            }
        }
        {
            const float cxg = gridW / 2.0f, cyg = gridH / 2.0f;
            std::vector<std::pair<float, int>> fr;
            for (int y = 0; y < gridH; ++y)
                for (int x = 0; x < gridW; ++x) {
                    if (G(x, y).solved) continue;
                    const float dx = x - cxg, dy = y - cyg;
                    fr.emplace_back(dx * dx + dy * dy, y * gridW + x);
                }
            std::stable_sort(fr.begin(), fr.end(), [](const std::pair<float, int>& a, const std::pair<float, int>& b) { return a.first < b.first; });
            for (const auto& f : fr) {
                if ((int)cand.size() >= kPathCMaxCandidates) break;
                if (!cand.empty() && cand.front() == f.second) continue;
                cand.push_back(f.second);
            }
        }
        bool ok = false;
        if (cand.empty()) {
            if (!seeds.locked) return -2;
        }
        const T g[6] = {(T)globalU, (T)globalV, 0, 0, 0, 0};
        for (int fi : cand) {
            Engine<T> eng = make_engine();
            Subset<T> sub;
            const NodeSolve<T> ns = solve_at(eng, sub, fi % gridW, fi / gridW, g, INIT_AUTO_SEARCH);
            if (!ns.initialized) continue;
            if (ns.res.status == 0 && ns.res.score <= T(kCorrAccept)) {
                pc_x = fi % gridW;
                pc_y = fi / gridW;
                globalU = (float)ns.res.u;
                globalV = (float)ns.res.v;
                ok = true;
                break;
            }
        }
        if (!ok && !cand.empty()) {
            pc_x = cand.front() % gridW;
            pc_y = cand.front() / gridW;
            if (!seeds.locked) return -5;
        }
    }

    // ------------------------------------------------------------ Path A --
    const auto t_a = clk::now();
    {
        std::vector<NodeSolve<T>> ns(NG);
        std::vector<char> run(NG, 0);
        for (size_t i = 0; i < NG; ++i) run[i] = in_mesh[i] && !grid[i].solved;
#pragma omp parallel for schedule(dynamic, 32)
        for (int i = 0; i < (int)NG; ++i) {
            if (!run[i]) continue;
            const T g[6] = {(T)gu[i], (T)gv[i], (T)gux[i], (T)guy[i], (T)gvx[i], (T)gvy[i]};
            const bool outside = grid[i].mesh == kMeshExtrapolated || grid[i].mesh == kMeshHomography;
            Engine<T> eng = make_engine();
            Subset<T> sub;
            ns[i] = solve_at(eng, sub, i % gridW, i / gridW, g, outside ? INIT_NO_SIMPLEX : INIT_NO_SEARCH);
        }
        for (size_t i = 0; i < NG; ++i) {
            if (!run[i] || !ns[i].initialized) continue;
            const Result<T>& r = ns[i].res;
            st_a.icgn_iters += r.iters;
            if (ns[i].rescue) record_simplex(st_a, r);
            GridPoint& g = grid[i];
            if (r.status == 0 && r.score <= T(kCorrAccept)) {
                g.u = (float)r.u; g.v = (float)r.v; g.ux = (float)r.ux; g.uy = (float)r.uy;
                g.vx = (float)r.vx; g.vy = (float)r.vy; g.corr = (float)r.score;
                g.solved = true;
                g.used_simplex = ns[i].rescue;
                g.icgn_iters = r.iters;
                st_a.points++;
            } else {
                g.solved = false;
                g.corr = kCorrInvalid;
                g.used_simplex = ns[i].rescue;
                g.icgn_iters = r.iters;
            }
        }
    }
    const double ms_a = ms_since(t_a);

    // ------------------------------------------------------------ Path B --
    const auto t_b = clk::now();
    {
        struct Seed { int x, y; float u, v, ux, uy, vx, vy, c; };
        struct Order {
            bool operator()(const Seed& a, const Seed& b) const {
                if (a.c != b.c) return a.c > b.c;
                if (a.y != b.y) return a.y > b.y;
                return a.x > b.x;
            }
        };
        std::priority_queue<Seed, std::vector<Seed>, Order> q;
        std::vector<unsigned char> claimed(NG);
        for (size_t i = 0; i < NG; ++i) claimed[i] = grid[i].solved ? 1 : 0;
        const int dx4[] = {1, -1, 0, 0}, dy4[] = {0, 0, 1, -1};
        std::vector<Seed> boundary, gseeds;
        const Seed pcs{pc_x, pc_y, globalU, globalV, 0, 0, 0, 0, 0};
        bool pcs_queued = false;
        for (int y = 0; y < gridH; ++y)
            for (int x = 0; x < gridW; ++x) {
                const GridPoint& g = G(x, y);
                if (!g.solved || g.corr < 0.f) continue;
                bool touch = false;
                for (int k = 0; k < 4; ++k) {
                    const int nx = x + dx4[k], ny = y + dy4[k];
                    if (nx >= 0 && nx < gridW && ny >= 0 && ny < gridH && !G(nx, ny).solved) { touch = true; break; }
                }
                if (touch) boundary.push_back({x, y, g.u, g.v, g.ux, g.uy, g.vx, g.vy, g.corr});
            }
        if (boundary.empty()) {
            struct Cand { int ix, iy; float u, v, dc, mag; };
            std::vector<Cand> cands;
            const float gcx2 = params.rect_x + (gridW / 2.f) * params.step, gcy2 = params.rect_y + (gridH / 2.f) * params.step;
            for (size_t fi = 0; fi < ref_pts.size(); ++fi) {
                const float fx = (float)ref_pts[fi].x, fy = (float)ref_pts[fi].y;
                const int ix = (int)std::round((fx - params.rect_x) / (float)params.step);
                const int iy = (int)std::round((fy - params.rect_y) / (float)params.step);
                if (ix < 0 || ix >= gridW || iy < 0 || iy >= gridH || G(ix, iy).solved) continue;
                const float du = (float)def_pts[fi].x - fx, dv = (float)def_pts[fi].y - fy;
                const float wx = (float)(params.rect_x + ix * params.step), wy = (float)(params.rect_y + iy * params.step);
                const float dc = std::sqrt((wx - gcx2) * (wx - gcx2) + (wy - gcy2) * (wy - gcy2));
                cands.push_back({ix, iy, du, dv, dc, std::sqrt(du * du + dv * dv)});
            }
            if (cands.empty()) {
                gseeds.push_back(pcs);
                pcs_queued = true;
            } else {
                std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) {
                    const float ma = std::floor(a.mag), mb = std::floor(b.mag);
                    if (ma != mb) return ma < mb;
                    if (a.dc != b.dc) return a.dc < b.dc;
                    if (a.iy != b.iy) return a.iy < b.iy;
                    return a.ix < b.ix;
                });
                for (size_t k = 0; k < cands.size() && k < 5; ++k)
                    gseeds.push_back({cands[k].ix, cands[k].iy, cands[k].u, cands[k].v, 0, 0, 0, 0, 0});
            }
        }
        for (const Seed& s : boundary) q.push(s);

        struct Task { int x, y; float g[6]; NodeSolve<T> ns; };
        auto solve_task = [&](Task& t) {
            Engine<T> eng = make_engine();
            Subset<T> sub;
            const T g[6] = {(T)t.g[0], (T)t.g[1], (T)t.g[2], (T)t.g[3], (T)t.g[4], (T)t.g[5]};
            t.ns = solve_at(eng, sub, t.x, t.y, g, INIT_NO_SEARCH);
        };
        auto commit = [&](const Task& t) {
            if (!t.ns.initialized) return;
            const Result<T>& r = t.ns.res;
            st_b.icgn_iters += r.iters;
            if (t.ns.rescue) record_simplex(st_b, r);
            GridPoint& g = G(t.x, t.y);
            if (r.status == 0 && r.score <= T(kCorrAccept)) {
                g.u = (float)r.u; g.v = (float)r.v; g.ux = (float)r.ux; g.uy = (float)r.uy;
                g.vx = (float)r.vx; g.vy = (float)r.vy; g.corr = (float)r.score;
                g.solved = true;
                g.used_simplex = t.ns.rescue;
                g.icgn_iters = r.iters;
                st_b.points++;
                q.push({t.x, t.y, g.u, g.v, g.ux, g.uy, g.vx, g.vy, g.corr});
            } else {
                g.corr = kCorrInvalid;
                g.used_simplex = t.ns.rescue;
                g.icgn_iters = r.iters;
            }
        };
        for (const Seed& s : gseeds) {
            const size_t f = (size_t)s.y * gridW + s.x;
            if (claimed[f]) continue;
            claimed[f] = 1;
            Task t{s.x, s.y, {s.u, s.v, 0, 0, 0, 0}, {}};
            solve_task(t);
            commit(t);
        }
        if (q.empty() && !gseeds.empty() && !pcs_queued) {
            const size_t f = (size_t)pcs.y * gridW + pcs.x;
            if (pcs.x >= 0 && pcs.x < gridW && pcs.y >= 0 && pcs.y < gridH && !claimed[f]) {
                claimed[f] = 1;
                Task t{pcs.x, pcs.y, {pcs.u, pcs.v, 0, 0, 0, 0}, {}};
                solve_task(t);
                commit(t);
            }
        }
        std::deque<std::vector<Task>> rounds;
        auto claim = [&]() -> bool {
            if (q.empty()) return false;
            std::vector<Task> r;
            int popped = 0;
            while (!q.empty() && popped < kPathBBatchNodes) {
                const Seed c = q.top();
                q.pop();
                ++popped;
                for (int k = 0; k < 4; ++k) {
                    const int nx = c.x + dx4[k], ny = c.y + dy4[k];
                    if (nx < 0 || nx >= gridW || ny < 0 || ny >= gridH) continue;
                    const size_t f = (size_t)ny * gridW + nx;
                    if (claimed[f]) continue;
                    claimed[f] = 1;
                    grid[f].solved = true;
                    const float ddx = (float)((nx - c.x) * params.step), ddy = (float)((ny - c.y) * params.step);
                    Task t{nx, ny, {c.u + c.ux * ddx + c.uy * ddy, c.v + c.vx * ddx + c.vy * ddy, c.ux, c.uy, c.vx, c.vy}, {}};
                    r.push_back(t);
                }
            }
            rounds.push_back(std::move(r));
            return true;
        };
        while (rounds.size() < 2 && claim()) {}
        while (!rounds.empty()) {
            std::vector<Task>& r = rounds.front();
#pragma omp parallel for schedule(dynamic, 1)
            for (int k = 0; k < (int)r.size(); ++k) solve_task(r[k]);
            for (const Task& t : r) commit(t);
            rounds.pop_front();
            while (rounds.size() < 2 && claim()) {}
        }
    }
    const double ms_b = ms_since(t_b);

    if (capture) {
        capture->gridW = gridW; capture->gridH = gridH;
        capture->rect_x = params.rect_x; capture->rect_y = params.rect_y;
        capture->step = params.step; capture->attempted = total_valid;
        capture->grid = grid;
    }

    // ---------------------------------------------------- pack + strain --
    const auto t_strain = clk::now();
    const PackOut po = pack_field(grid, gridW, gridH, params.step, params.strain_window, out, capacity);
    const int valid_count = po.valid_count, dropped_outlier = po.dropped_outlier, dropped_post = po.dropped_post;
    const double ms_strain = ms_since(t_strain);
    const double ms_total = ms_since(t_total);

    const int ncopy = metrics_prefix_len(metrics_len);
    if (metrics && ncopy > 0) {
        const int iters = st_a.icgn_iters + st_b.icgn_iters + st_anchor.icgn_iters;
        float m[kMetricsLen];
        m[0] = (float)total_valid;
        m[1] = (float)valid_count;
        m[2] = (float)(total_valid - valid_count);
        m[3] = (float)st_a.points;
        m[4] = (float)st_b.points;
        m[5] = (float)(st_a.simp_calls + st_b.simp_calls + st_anchor.simp_calls);
        m[6] = (float)(st_a.simp_saved + st_b.simp_saved + st_anchor.simp_saved);
        m[7] = (float)(st_a.simp_dead + st_b.simp_dead + st_anchor.simp_dead);
        m[8] = valid_count > 0 ? (float)iters / (float)valid_count : 0.f;
        m[9] = (float)ms_total;
        m[10] = (float)ms_seed;
        m[11] = (float)ms_prepass;
        m[12] = (float)ms_mesh;
        m[13] = (float)ms_strain;
        m[14] = ms_total > 0 ? (float)(valid_count / ms_total) : 0.f;
        m[15] = total_valid > 0 ? ((float)valid_count / total_valid) * 100.0f : 0.f;
        m[16] = seeds.quality == MeshQuality::FULL ? 2.f : seeds.quality == MeshQuality::SPARSE ? 1.f : 0.f;
        m[17] = 0.f;
        m[18] = (float)(ms_a + ms_b);
        m[19] = (float)st_anchor.points;
        m[20] = (float)dropped_post;
        m[21] = seeds.locked ? 1.f : 0.f;
        m[22] = seeds.coverage;
        m[23] = (float)dropped_outlier;
        for (int i = 0; i < ncopy; ++i) metrics[i] = m[i];
    }
    if (keep_def) *keep_def = std::move(def);
    return valid_count;
}

}  // namespace oracle
