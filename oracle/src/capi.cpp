// ORACLE — test infrastructure only. Never linked into the product library.
//
// extern "C" surface of the CPU restatement, for the parity tests (ctypes)
// and the CPU baseline leg of the benchmark. Every function here is a thin
// call into the templated restatement in pipeline.hpp / solver.hpp / strain.hpp.
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "incremental.hpp"
#include "pipeline.hpp"
#include "refsynth.hpp"

using namespace oracle;

namespace {

struct Handle {
    bool fp64 = false;
    RefCache<float> c32;
    RefCache<double> c64;
};

Params to_params(const int32_t p[8]) {
    Params q;
    q.rect_x = p[0]; q.rect_y = p[1]; q.rect_w = p[2]; q.rect_h = p[3];
    q.step = p[4]; q.subset_size = p[5]; q.strain_window = p[6]; q.six = p[7] != 0;
    return q;
}

template <class T>
void do_solve_nodes(const uint8_t* ref, const uint8_t* def, int w, int h, const uint8_t* mask, int dim,
                    int lm, int six, int n, const int32_t* xy, const float* guess, const int32_t* mode,
                    float* fout, int32_t* iout) {
    Image<T> R, D;
    R.prepare(w, h, ref);
    R.stamp_ghost_wall(mask);
    D.prepare(w, h, def);
#pragma omp parallel for schedule(dynamic, 4)
    for (int k = 0; k < n; ++k) {
        const int x = xy[2 * k], y = xy[2 * k + 1];
        const PoolEntry<T> e = compute_hessian_only(R, x, y, dim);
        Engine<T> eng;
        eng.lm = lm != 0;
        eng.six = six != 0;
        Subset<T> sub;
        T g[6];
        for (int j = 0; j < 6; ++j) g[j] = (T)guess[6 * k + j];
        const NodeSolve<T> ns = solve_node(eng, sub, R, D, x, y, dim, e, g, (InitMode)mode[k]);
        const Result<T>& r = ns.res;
        float* f = fout + 7 * (size_t)k;
        f[0] = (float)r.u; f[1] = (float)r.v; f[2] = (float)r.ux; f[3] = (float)r.uy;
        f[4] = (float)r.vx; f[5] = (float)r.vy; f[6] = (float)r.score;
        int32_t* q = iout + 6 * (size_t)k;
        q[0] = ns.initialized ? 1 : 0;
        q[1] = r.status;
        q[2] = r.iters;
        q[3] = r.invalid_ref;
        q[4] = ns.rescue ? 1 : 0;
        q[5] = r.trigger_iters;
    }
}

}  // namespace

extern "C" {

void* oracle_create(int fp64) {
    Handle* h = new Handle();
    h->fp64 = fp64 != 0;
    return h;
}

void oracle_destroy(void* p) { delete static_cast<Handle*>(p); }

int oracle_set_reference(void* p, const uint8_t* gray, int w, int h, const uint8_t* mask) {
    Handle* H = static_cast<Handle*>(p);
    if (!gray || w <= 0 || h <= 0) return -3;
    if (H->fp64) H->c64.set(w, h, gray, mask);
    else H->c32.set(w, h, gray, mask);
    return 0;
}

int oracle_run(void* p, const uint8_t* def, const uint8_t* mask, const int32_t* params, float* out,
               int cap, float* metrics, int mlen, const double* model_H) {
    Handle* H = static_cast<Handle*>(p);
    const Params q = to_params(params);
    if (H->fp64) return run_full_field<double>(H->c64, def, mask, q, out, cap, metrics, mlen, model_H);
    return run_full_field<float>(H->c32, def, mask, q, out, cap, metrics, mlen, model_H);
}

// oracle_run with per-anchor displacement guesses under the model: anchor_uv
// [anchor_n][2] in the anchor lattice's row-major order (NaN: none), used when
// anchor_n equals the lattice's size.
int oracle_run_guided(void* p, const uint8_t* def, const uint8_t* mask, const int32_t* params, float* out,
                      int cap, float* metrics, int mlen, const double* model_H, const float* anchor_uv,
                      int anchor_n) {
    Handle* H = static_cast<Handle*>(p);
    const Params q = to_params(params);
    if (H->fp64)
        return run_full_field<double>(H->c64, def, mask, q, out, cap, metrics, mlen, model_H, nullptr, nullptr,
                                      anchor_uv, anchor_n);
    return run_full_field<float>(H->c32, def, mask, q, out, cap, metrics, mlen, model_H, nullptr, nullptr,
                                 anchor_uv, anchor_n);
}

// Per-node raw results of the last kind of solve (Capture), for the device
// pipeline's intermediate parity checks: per grid node
// [u v ux uy vx vy corr] + [solved mesh icgn_iters used_simplex].
int oracle_run_capture(void* p, const uint8_t* def, const uint8_t* mask, const int32_t* params,
                       float* out, int cap, float* metrics, int mlen, const double* model_H,
                       float* gf, int32_t* gi, int max_nodes) {
    Handle* H = static_cast<Handle*>(p);
    const Params q = to_params(params);
    Capture c;
    int rc;
    if (H->fp64) rc = run_full_field<double>(H->c64, def, mask, q, out, cap, metrics, mlen, model_H, &c);
    else rc = run_full_field<float>(H->c32, def, mask, q, out, cap, metrics, mlen, model_H, &c);
    if (rc < 0) return rc;
    const int n = (int)c.grid.size();
    for (int i = 0; i < n && i < max_nodes; ++i) {
        const GridPoint& g = c.grid[i];
        float* f = gf + 7 * (size_t)i;
        f[0] = g.u; f[1] = g.v; f[2] = g.ux; f[3] = g.uy; f[4] = g.vx; f[5] = g.vy; f[6] = g.corr;
        int32_t* s = gi + 4 * (size_t)i;
        s[0] = g.solved; s[1] = g.mesh; s[2] = g.icgn_iters; s[3] = g.used_simplex;
    }
    return rc;
}

// Image planes after prepare_data + Ghost Wall (float precision).
void oracle_prepare(const uint8_t* gray, int w, int h, const uint8_t* mask, float* I, float* gx, float* gy) {
    Image<float> im;
    im.prepare(w, h, gray);
    im.stamp_ghost_wall(mask);
    const size_t n = (size_t)w * h;
    std::memcpy(I, im.I.data(), n * 4);
    std::memcpy(gx, im.gx.data(), n * 4);
    std::memcpy(gy, im.gy.data(), n * 4);
}

// Hessian pool entries at the given centres: valid, mean, std, H (21 doubles,
// upper triangle row-major).
void oracle_pool(const uint8_t* gray, int w, int h, const uint8_t* mask, int dim, int n,
                 const int32_t* xy, int32_t* valid, float* mean_std, double* H21) {
    Image<float> im;
    im.prepare(w, h, gray);
    im.stamp_ghost_wall(mask);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
        const PoolEntry<float> e = compute_hessian_only(im, xy[2 * k], xy[2 * k + 1], dim);
        valid[k] = e.valid ? 1 : 0;
        mean_std[2 * k] = e.mean;
        mean_std[2 * k + 1] = e.std_dev;
        int q = 0;
        for (int r = 0; r < 6; ++r)
            for (int c = r; c < 6; ++c) H21[21 * (size_t)k + q++] = e.H[r][c];
    }
}

// solve_node at each (x, y) with its own guess and mode. fout: 7 floats per
// node [u v ux uy vx vy score]; iout: 6 ints [initialized status iters
// invalid_ref rescue trigger_iters].
void oracle_solve_nodes(int fp64, const uint8_t* ref, const uint8_t* def, int w, int h, const uint8_t* mask,
                        int dim, int lm, int six, int n, const int32_t* xy, const float* guess,
                        const int32_t* mode, float* fout, int32_t* iout) {
    if (fp64) do_solve_nodes<double>(ref, def, w, h, mask, dim, lm, six, n, xy, guess, mode, fout, iout);
    else do_solve_nodes<float>(ref, def, w, h, mask, dim, lm, six, n, xy, guess, mode, fout, iout);
}

// Median test then VSG over a displacement grid. valid is updated in place;
// returns the number of rejected points. strain: 3 floats per node.
int oracle_median_vsg(int gw, int gh, int step, int window, const float* u, const float* v,
                      uint8_t* valid, float* strain) {
    DispField f;
    f.width = gw; f.height = gh; f.step = step;
    f.u.assign(u, u + (size_t)gw * gh);
    f.v.assign(v, v + (size_t)gw * gh);
    f.valid.assign(valid, valid + (size_t)gw * gh);
    const int rej = reject_outliers(f);
    const StrainOut s = vsg_strain(f, window);
    for (size_t i = 0; i < f.valid.size(); ++i) {
        valid[i] = f.valid[i];
        strain[3 * i] = s.exx[i];
        strain[3 * i + 1] = s.eyy[i];
        strain[3 * i + 2] = s.exy[i];
    }
    return rej;
}

int oracle_vsg_window_node_count(int step, int window) { return vsg_window_node_count(step, window); }

// The GoldenCorpus run (tests/integration/test_golden_corpus.cpp:54-127):
// 512x512 speckle (seed 42), subset 27, 18x18 grid from 60 step 22, the
// translate and affine scenarios, precompute_subset + INIT_NO_SIMPLEX from a
// zero guess with the default engine (no LM). Returns the record count.
int oracle_corpus(int use6, int fp64, int32_t* ixy, float* vals, int maxn) {
    const int W = 512, H = 512, D = 27;
    const float sc[2][6] = {{3.2f, -1.7f, 0, 0, 0, 0}, {2.1f, 1.4f, 0.015f, -0.008f, 0.006f, 0.012f}};
    int cnt = 0;
    for (int s = 0; s < 2; ++s) {
        RefSpeckle field(42, W, H);
        RefAffine d;
        d.u = sc[s][0]; d.v = sc[s][1]; d.ux = sc[s][2]; d.uy = sc[s][3]; d.vx = sc[s][4]; d.vy = sc[s][5];
        d.cx = W / 2.0f; d.cy = H / 2.0f;
        const std::vector<float> rf = ref_image(field, W, H), df = def_image(field, W, H, d);
        auto run = [&](auto tag) {
            using T = decltype(tag);
            Image<T> R, Dm;
            R.prepare_float(W, H, rf.data());
            Dm.prepare_float(W, H, df.data());
            for (int y = 60; y <= 452; y += 22)
                for (int x = 60; x <= 452; x += 22) {
                    const PoolEntry<T> e = compute_hessian_only(R, x, y, D);
                    Subset<T> sub;
                    fill_subset(sub, R, x, y, D, e);
                    if (!sub.ok) continue;
                    Engine<T> eng;
                    eng.six = use6 != 0;
                    const T g[6] = {0, 0, 0, 0, 0, 0};
                    const Result<T> r = eng.solve(sub, Dm, g, INIT_NO_SIMPLEX);
                    if (cnt < maxn) {
                        ixy[3 * cnt] = x; ixy[3 * cnt + 1] = y; ixy[3 * cnt + 2] = r.status;
                        float* o = vals + 7 * (size_t)cnt;
                        o[0] = (float)r.u; o[1] = (float)r.v; o[2] = (float)r.ux; o[3] = (float)r.uy;
                        o[4] = (float)r.vx; o[5] = (float)r.vy; o[6] = (float)r.score;
                    }
                    ++cnt;
                }
        };
        if (fp64) run(double(0));
        else run(float(0));
    }
    return cnt;
}

// The FullFieldGolden inputs (tests/integration/test_full_field_golden.cpp:60-99):
// 320x320, SpeckleField seed 11 with 600 blobs, gray8; scenario 0 translate
// (3, 2), scenario 1 affine (2, -1.5, 0.012, -0.006, 0.005, 0.010) about the
// centre.
void oracle_ff_inputs(int scenario, uint8_t* ref, uint8_t* def) {
    const int W = 320, H = 320;
    RefSpeckle field(11, W, H, 600);
    const std::vector<uint8_t> r = gray8(ref_image(field, W, H));
    RefAffine d;
    if (scenario == 0) { d.u = 3.0f; d.v = 2.0f; }
    else { d.u = 2.0f; d.v = -1.5f; d.ux = 0.012f; d.uy = -0.006f; d.vx = 0.005f; d.vy = 0.010f; }
    d.cx = W / 2.0f; d.cy = H / 2.0f;
    const std::vector<uint8_t> dd = gray8(def_image(field, W, H, d));
    std::memcpy(ref, r.data(), r.size());
    std::memcpy(def, dd.data(), dd.size());
}

// ---- incremental session and its per-node math (incremental_session.hpp) ----

void* oracle_inc_create() { return new IncSession(); }
void oracle_inc_destroy(void* p) { delete static_cast<IncSession*>(p); }

int oracle_inc_init(void* p, const uint8_t* ref, int w, int h, const uint8_t* mask, const int32_t prm[8],
                    int interval) {
    IncSession* S = static_cast<IncSession*>(p);
    semper_inc::IncParams q;
    q.rect_x = prm[0]; q.rect_y = prm[1]; q.rect_w = prm[2]; q.rect_h = prm[3];
    q.step = prm[4]; q.subset_size = prm[5]; q.strain_window = prm[6]; q.six = prm[7] != 0;
    return S->core.init(ref, w, h, mask, q, interval);
}

// info: reference_frame, reference_updated, tracked_points, frame0_points, taylor_fallbacks, lost_this_frame
int oracle_inc_process(void* p, const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len,
                       int32_t info[6]) {
    IncSession* S = static_cast<IncSession*>(p);
    semper_inc::FrameInfo fi;
    const int rc = S->core.process(def, out, capacity, metrics, metrics_len, nullptr, &fi);
    if (info) {
        info[0] = fi.reference_frame; info[1] = fi.reference_updated ? 1 : 0; info[2] = fi.tracked_points;
        info[3] = fi.frame0_points; info[4] = fi.taylor_fallbacks; info[5] = fi.lost_this_frame;
    }
    return rc;
}

static semper_inc::NodeField make_field(int gw, int gh, int rx, int ry, int step, const float* u, const float* v,
                                        const float* ux, const float* uy, const float* vx, const float* vy,
                                        const float* corr, const uint8_t* valid) {
    semper_inc::NodeField f;
    f.gridW = gw; f.gridH = gh; f.rect_x = rx; f.rect_y = ry; f.step = step;
    const size_t n = (size_t)gw * gh;
    f.u.assign(u, u + n); f.v.assign(v, v + n); f.ux.assign(ux, ux + n); f.uy.assign(uy, uy + n);
    f.vx.assign(vx, vx + n); f.vy.assign(vy, vy + n); f.corr.assign(corr, corr + n); f.valid.assign(valid, valid + n);
    return f;
}

// res: u, v, corr, taylor; returns ok
int oracle_inc_sample(int gw, int gh, int rx, int ry, int step, const float* u, const float* v, const float* ux,
                      const float* uy, const float* vx, const float* vy, const float* corr, const uint8_t* valid,
                      float x, float y, float* res) {
    const semper_inc::IncrementSample s =
        semper_inc::sample_increment(make_field(gw, gh, rx, ry, step, u, v, ux, uy, vx, vy, corr, valid), x, y);
    res[0] = s.u; res[1] = s.v; res[2] = s.corr; res[3] = s.taylor ? 1.f : 0.f;
    return s.ok ? 1 : 0;
}

int oracle_inc_fit(int gw, int gh, int rx, int ry, int step, const float* u, const float* v, const float* ux,
                   const float* uy, const float* vx, const float* vy, const float* corr, const uint8_t* valid,
                   float x, float y, float radius, float* res) {
    const semper_inc::IncrementSample s = semper_inc::fit_increment(
        make_field(gw, gh, rx, ry, step, u, v, ux, uy, vx, vy, corr, valid), x, y, radius);
    res[0] = s.u; res[1] = s.v; res[2] = s.corr;
    return s.ok ? 1 : 0;
}

// 0 drop, 1 refresh, 2 keep
int oracle_inc_anchor_need(int gw, int gh, int rx, int ry, int step, const float* u, const float* v,
                           const float* ux, const float* uy, const float* vx, const float* vy, const float* corr,
                           const uint8_t* valid, float x, float y, int subset) {
    const semper_inc::NodeField f = make_field(gw, gh, rx, ry, step, u, v, ux, uy, vx, vy, corr, valid);
    const semper_inc::AnchorNeed n = semper_inc::anchor_need(f, semper_inc::gap_distance(f), x, y, subset);
    return n == semper_inc::AnchorNeed::kDrop ? 0 : n == semper_inc::AnchorNeed::kRefresh ? 1 : 2;
}

// the node field's valid flags after node_field_from_capture; returns the count rejected
int oracle_inc_node_field(int gw, int gh, const float* u, const float* v, const float* corr, const uint8_t* solved,
                          uint8_t* valid_out) {
    semper_inc::SolveCapture c;
    c.gridW = gw; c.gridH = gh; c.step = 10;
    const size_t n = (size_t)gw * gh;
    c.u.assign(u, u + n); c.v.assign(v, v + n);
    c.ux.assign(n, 0.f); c.uy.assign(n, 0.f); c.vx.assign(n, 0.f); c.vy.assign(n, 0.f);
    c.corr.assign(corr, corr + n); c.solved.assign(solved, solved + n);
    int rejected = 0;
    const semper_inc::NodeField f = semper_inc::node_field_from_capture(c, &rejected);
    std::memcpy(valid_out, f.valid.data(), n);
    return rejected;
}

void oracle_inc_warp_mask(const uint8_t* mask0, int W, int H, int gw, int gh, int rx, int ry, int step,
                          const float* U, const float* V, const uint8_t* valid, int margin, uint8_t* out) {
    const size_t n = (size_t)gw * gh;
    const std::vector<uint8_t> m(mask0, mask0 + (size_t)W * H);
    const std::vector<uint8_t> w = semper_inc::warp_material_mask(
        m, W, H, semper_inc::GridGeom{gw, gh, rx, ry, step}, std::vector<float>(U, U + n),
        std::vector<float>(V, V + n), std::vector<unsigned char>(valid, valid + n), margin);
    std::memcpy(out, w.data(), w.size());
}

// make_anchor on `ref` at (x, y), then match_anchor on `def`; xyc: x, y, corr,
// and the anchor's ax, ay, dx, dy. Returns -1 when no anchor is cut, else 0/1.
int oracle_inc_match(const uint8_t* ref, const uint8_t* def, int W, int H, float x, float y, int subset, float gx,
                     float gy, float max_shift, float* xyc) {
    semper_inc::CoastAnchor a;
    if (!semper_inc::make_anchor(ref, W, H, x, y, subset, a)) return -1;
    Image<float> D;
    D.prepare(W, H, def);
    xyc[3] = (float)a.ax; xyc[4] = (float)a.ay; xyc[5] = a.dx; xyc[6] = a.dy;
    float mx = 0, my = 0, corr = 0;
    const bool ok = IncBackend::match_on(a, D, subset, false, gx, gy, max_shift, mx, my, corr);
    if (ok) { xyc[0] = mx; xyc[1] = my; xyc[2] = corr; }
    return ok ? 1 : 0;
}

}  // extern "C"
