// ORACLE — test infrastructure only. Never linked into the product library.
//
// The incremental session over the CPU restatement: the session logic and
// the per-node math of incremental_session.hpp, every solve, adoption and
// packing the restatement's own (pipeline.hpp, solver.hpp).
#pragma once

#include <functional>

#include "incremental_session.hpp"
#include "pipeline.hpp"

namespace oracle {

struct IncBackend {
    RefCache<float> cache;
    Image<float> kept;  // the prepared deformed frame of the last run
    bool has_kept = false;

    static Params to_params(const semper_inc::IncParams& p) {
        Params q;
        q.rect_x = p.rect_x; q.rect_y = p.rect_y; q.rect_w = p.rect_w; q.rect_h = p.rect_h;
        q.step = p.step; q.subset_size = p.subset_size; q.strain_window = p.strain_window; q.six = p.six;
        return q;
    }

    int validate(semper_inc::IncParams& p, int W, int H) {
        Params q = to_params(p);
        const int rc = validate_params(q, W, H);
        p.rect_x = q.rect_x; p.rect_y = q.rect_y; p.rect_w = q.rect_w; p.rect_h = q.rect_h;
        return rc;
    }
    int vsg_count(int step, int window) { return vsg_window_node_count(step, window); }
    int set_reference(const uint8_t* gray, int W, int H, const uint8_t* mask) {
        cache.set(W, H, gray, mask);
        has_kept = false;
        return 0;
    }
    int run(const uint8_t* def, const uint8_t* mask, const semper_inc::IncParams& p, float* out, int capacity,
            float* metrics, int metrics_len, const std::function<void(int)>& progress, semper_inc::SolveCapture* sc) {
        Capture c;
        Image<float> keep;
        const int rc = run_full_field<float>(cache, def, mask, to_params(p), out, capacity, metrics, metrics_len,
                                             nullptr, &c, &keep);
        if (rc < 0) return rc;
        if (progress) progress(100);
        kept = std::move(keep);
        has_kept = true;
        const size_t n = c.grid.size();
        sc->gridW = c.gridW; sc->gridH = c.gridH; sc->rect_x = c.rect_x; sc->rect_y = c.rect_y;
        sc->step = c.step; sc->attempted = c.attempted;
        sc->u.resize(n); sc->v.resize(n); sc->ux.resize(n); sc->uy.resize(n); sc->vx.resize(n); sc->vy.resize(n);
        sc->corr.resize(n); sc->solved.resize(n);
        for (size_t i = 0; i < n; ++i) {
            const GridPoint& g = c.grid[i];
            sc->u[i] = g.u; sc->v[i] = g.v; sc->ux[i] = g.ux; sc->uy[i] = g.uy; sc->vx[i] = g.vx; sc->vy[i] = g.vy;
            sc->corr[i] = g.corr;
            sc->solved[i] = g.solved ? 1 : 0;
        }
        return rc;
    }
    // ReferenceCache::adopt (reference_cache.cpp:82-108): the kept frame with
    // the Ghost Wall of `mask`; the grid scan and pool are rebuilt.
    int adopt(const uint8_t* mask) {
        if (!has_kept) return -3;
        cache.ref = std::move(kept);
        cache.ref.stamp_ghost_wall(mask);
        cache.grid_valid = false;
        cache.has = true;
        has_kept = false;
        return 0;
    }
    int pack(const semper_inc::GridGeom& g, int window, const std::vector<float>& u, const std::vector<float>& v,
             const std::vector<float>& corr, const std::vector<unsigned char>& solved, float* out, int capacity) {
        std::vector<GridPoint> grid((size_t)g.gridW * g.gridH);
        for (int y = 0; y < g.gridH; ++y)
            for (int x = 0; x < g.gridW; ++x) {
                const size_t i = (size_t)y * g.gridW + x;
                GridPoint& gp = grid[i];
                gp.x = (float)(g.rect_x + x * g.step);
                gp.y = (float)(g.rect_y + y * g.step);
                gp.u = u[i];
                gp.v = v[i];
                gp.corr = corr[i];
                gp.solved = solved[i] != 0;
            }
        return pack_field(grid, g.gridW, g.gridH, g.step, window, out, capacity).valid_count;
    }
    semper_inc::Rect warp_mask(const std::vector<uint8_t>& mask0, int W, int H, const semper_inc::GridGeom& g,
                               const semper_inc::MaskWarpPlan& p, std::vector<uint8_t>& out) {
        semper_inc::scatter_mask_host(mask0, W, H, g, p, out);
        return semper_inc::bounding_rect(out, W, H);
    }
    // match_anchor (incremental_math.cpp:238-276) on the kept frame.
    bool match_anchor(const semper_inc::CoastAnchor& a, int subset, bool six, float gx, float gy, float max_shift,
                      float& x, float& y, float& corr) {
        if (!has_kept || a.patch.empty()) return false;
        return match_on(a, kept, subset, six, gx, gy, max_shift, x, y, corr);
    }

    static bool match_on(const semper_inc::CoastAnchor& a, const Image<float>& def, int subset, bool six, float gx,
                         float gy, float max_shift, float& x, float& y, float& corr) {
        Image<float> P;
        P.prepare(a.size, a.size, a.patch.data());
        const int c = a.size / 2;
        const PoolEntry<float> e = compute_hessian_only(P, c, c, subset);
        Subset<float> sub;
        fill_subset(sub, P, c, c, subset, e);
        if (!sub.ok) return false;
        sub.cx = a.ax;
        sub.cy = a.ay;
        Engine<float> eng;
        eng.lm = true;
        eng.six = six;
        const float g[6] = {gx - a.dx - (float)a.ax, gy - a.dy - (float)a.ay, 0.f, 0.f, 0.f, 0.f};
        const Result<float> r = eng.solve(sub, def, g, INIT_NO_SEARCH);
        return semper_inc::accept_anchor_match(a, r.status, r.score, r.u, r.v, r.ux, r.uy, r.vx, r.vy, gx, gy,
                                               max_shift, x, y, corr);
    }
};

struct IncSession {
    IncBackend backend;
    semper_inc::IncrementalCore<IncBackend> core{backend};
};

}  // namespace oracle
