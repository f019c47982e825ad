// IncrementalSession on the device engine (include/semper/incremental.hpp:
// 74-117; behaviour of src/pipeline/incremental_session.cpp:120-549).
//
// The session follows every frame-0 grid node through a chain of references.
// Its per-node state (total displacement at the current reference, whether
// the node is still followed, how far it has coasted) lives in device memory,
// and each frame runs over it as a handful of kernels (incnode.cu): the
// increment solve of the frame against the current reference, the anchor need
// of the increment field, one node step (sample the increment where the node
// now is, or coast on a fitted plane), the packing of the totals on the
// frame-0 grid, and at a reference update the bookkeeping, the fill and
// forward warp of the material mask and the adoption of the solved frame.
// The host keeps what is O(1) per frame (the update schedule, the rect of the
// next reference) and the coasting anchors, whose direct matches are device
// solves run from here for the few nodes the node step lists.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "../kernels/incnode.cuh"
#include "incremental.hpp"

namespace semper_b200 {

namespace {

// include/semper/tuning.hpp:193-281, the session's gates.
constexpr int kCoastRadiusCells = 8;
constexpr float kCoastMaxTravelSubsets = 2.0f;
constexpr float kCoastTrustedTravelSubsets = 0.25f;
constexpr float kReanchorMaxShiftFraction = 0.3f;
constexpr float kReanchorMinShiftPx = 1.0f;
constexpr int kAnchorMarginPx = 10;
constexpr float kEarlyUpdateDrop = 0.05f;
constexpr float kUpdateMinReported = 0.5f;
constexpr int kMaskExtrapCells = 3;
constexpr int kMaskMaxSamplesPerPx = 8;
constexpr float kCorrAccept = 0.15f;

double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

struct Box {
    int x = 0, y = 0, w = 0, h = 0;
    long long area() const { return (long long)w * h; }
};

Box overlap(const Box& a, const Box& b) {
    const int x0 = std::max(a.x, b.x), y0 = std::max(a.y, b.y);
    const int x1 = std::min(a.x + a.w, b.x + b.w), y1 = std::min(a.y + a.h, b.y + b.h);
    if (x1 <= x0 || y1 <= y0) return Box{};
    return Box{x0, y0, x1 - x0, y1 - y0};
}

float key_to_float(int k) {
    const int b = k >= 0 ? k : k ^ 0x7fffffff;
    float f;
    std::memcpy(&f, &b, sizeof f);
    return f;
}

// The correctly rounded length of (a, b) (the node step's coast travel uses
// the same definition).
float length2(float a, float b) { return (float)std::sqrt((double)a * a + (double)b * b); }

// A coasting node's subset on the reference where it was last clean: a square
// patch of gray around the pixel (ax, ay), and the node's offset from it.
struct Anchor {
    std::vector<uint8_t> patch;
    int side = 0;  // 0: none
    int ax = 0, ay = 0;
    float dx = 0.0f, dy = 0.0f;
};

// Cut the anchor of a node at (x, y) from a frame (make_anchor,
// incremental_math.cpp:223-236): false, and the anchor unchanged, when the
// patch would leave the frame.
bool cut_anchor(const uint8_t* gray, int W, int H, float x, float y, int subset, Anchor& a) {
    const int ax = (int)std::lround(x), ay = (int)std::lround(y);
    const int r = subset / 2 + kAnchorMarginPx;
    if (ax - r < 0 || ay - r < 0 || ax + r >= W || ay + r >= H) return false;
    a.side = 2 * r + 1;
    a.patch.resize((size_t)a.side * a.side);
    for (int j = 0; j < a.side; ++j)
        std::memcpy(&a.patch[(size_t)j * a.side], gray + (size_t)(ay - r + j) * W + (ax - r), (size_t)a.side);
    a.ax = ax;
    a.ay = ay;
    a.dx = x - (float)ax;
    a.dy = y - (float)ay;
    return true;
}

int64_t strain_window_cap(const Params& p) {
    if (p.step <= 0) return 0;
    const int64_t gmin = std::min(p.rect_w / p.step, p.rect_h / p.step);
    return 2 * (gmin + 1) * (int64_t)p.step;
}

}  // namespace

struct IncrementalSession::Impl {
    Engine engine;
    FrameProfile prof;

    bool ready = false;
    Params params;  // the frame-0 solve (rect clipped)
    int interval = 0;
    int W = 0, H = 0;
    std::vector<uint8_t> user_mask0, material0;
    bool material0_on_device = false;  // the engine holds material0 since the last mask warp
    std::vector<uint8_t> spare_mask;   // a W x H buffer for the next warped mask
    dic::IncGrid g0{};
    int n0 = 0;
    int frame0_points = -1;

    // per-node state on the device, and one frame's results
    DevBuf<float> ubase, vbase, travel, travel_next, U, V, corr, cstep, gu, gv, gcorr;
    DevBuf<uint8_t> alive, alive_next, anchored, flags, need, gsolved;
    DevBuf<float> fillU[2], fillV[2];
    DevBuf<uint8_t> filled[2];
    DevBuf<int> counters, match_list, refresh_list, drop_list;
    DevBuf<float> match_info, refresh_xy;
    DevBuf<dic::IncMatch> match_rec;
    int alive_nodes = 0;

    std::vector<Anchor> anchors;
    std::vector<uint8_t> anchored_h;

    // the schedule of references
    int ref_index = 0, since_update = 0, ref_reported = -1, adopted_reported = -1, frames = 0;
    Params params_k;
    std::vector<uint8_t> mask_k;
    std::vector<float> scratch;

    cudaStream_t st() const { return engine.stream(); }
    void sync() { check(cudaStreamSynchronize(st()), "sync"); }

    void clear() {
        ready = false;
        W = H = 0;
        user_mask0.clear();
        material0.clear();
        material0_on_device = false;
        g0 = dic::IncGrid{};
        n0 = 0;
        frame0_points = -1;
        alive_nodes = 0;
        anchors.clear();
        anchored_h.clear();
        ref_index = since_update = frames = 0;
        ref_reported = adopted_reported = -1;
        params_k = Params();
        mask_k.clear();
        scratch.clear();
    }

    dic::IncState state() { return dic::IncState{ubase.p, vbase.p, alive.p, travel.p, anchored.p}; }
    dic::IncFrame frame() { return dic::IncFrame{U.p, V.p, corr.p, cstep.p, flags.p}; }

    static dic::IncField field_of(const DeviceField& d) {
        return dic::IncField{d.gridW, d.gridH, d.rect_x, d.rect_y, d.step, d.u, d.v, d.ux, d.uy, d.vx, d.vy,
                             d.corr,  d.solved, d.ok};
    }

    void ensure_nodes(size_t n) {
        for (DevBuf<float>* b : {&ubase, &vbase, &travel, &travel_next, &U, &V, &corr, &cstep, &gu, &gv, &gcorr,
                                 &fillU[0], &fillU[1], &fillV[0], &fillV[1], &match_info, &refresh_xy})
            b->ensure(std::max(b->n, 3 * n));
        for (DevBuf<uint8_t>* b : {&alive, &alive_next, &anchored, &flags, &gsolved, &filled[0], &filled[1]})
            b->ensure(std::max(b->n, n));
        for (DevBuf<int>* b : {&match_list, &refresh_list, &drop_list}) b->ensure(std::max(b->n, n));
        match_rec.ensure(std::max(match_rec.n, n));
        counters.ensure(dic::kIncCounters);
    }

    void zero_counters() { check(cudaMemsetAsync(counters.p, 0, dic::kIncCounters * sizeof(int), st()), "memset"); }

    void counters_to_host(int* h, int first, int count) {
        check(cudaMemcpyAsync(h, counters.p + first, count * sizeof(int), cudaMemcpyDeviceToHost, st()), "D2H");
        sync();
    }

    void upload_anchored() {
        check(cudaMemcpyAsync(anchored.p, anchored_h.data(), (size_t)n0, cudaMemcpyHostToDevice, st()),
              "H2D anchors");
    }

    int init(const uint8_t* ref, int w, int h, const uint8_t* roi_mask, const Params& p_in, int update_interval);
    int process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len, Progress progress,
                FrameInfo* info);
    int nothing_to_follow(FrameInfo fi, float* metrics, int metrics_len, const Progress& progress, FrameInfo* info);
    bool match(int node, float gx, float gy, float travel_k, float& mx, float& my, float& mcorr);
    bool warp_mask(const uint8_t* alive_flags, const float* Ut, const float* Vt, std::vector<uint8_t>& out, Box& bb);
};

// init (incremental_session.cpp:219-268).
int IncrementalSession::Impl::init(const uint8_t* ref, int w, int h, const uint8_t* roi_mask, const Params& p_in,
                                   int update_interval) {
    clear();
    if (!ref || w <= 0 || h <= 0 || update_interval < 0) return -3;
    params = p_in;
    interval = update_interval;
    const int rc = check_params(params, w, h);
    if (rc != 0) return rc;
    if (vsg_window_nodes(params.step, params.strain_window) < 3) return -4;
    W = w;
    H = h;
    g0 = dic::IncGrid{params.rect_w / params.step, params.rect_h / params.step, params.rect_x, params.rect_y,
                      params.step};
    n0 = g0.gw * g0.gh;
    const size_t npx = (size_t)W * H;
    if (roi_mask) {
        user_mask0.assign(roi_mask, roi_mask + npx);
        material0.resize(npx);
        for (size_t i = 0; i < npx; ++i) material0[i] = roi_mask[i] >= 128 ? 255 : 0;
        material0_on_device = false;
    } else {
        // the ROI rect widened by the reach of its edge nodes' subsets at 45 deg
        const int reach = (int)std::ceil(params.subset_size / 2 * std::sqrt(2.0)) + 1;
        material0.assign(npx, 0);
        const Box r = overlap(Box{params.rect_x - reach, params.rect_y - reach, params.rect_w + 2 * reach,
                                  params.rect_h + 2 * reach},
                              Box{0, 0, W, H});
        for (int y = r.y; y < r.y + r.h; ++y) std::memset(material0.data() + (size_t)y * W + r.x, 255, (size_t)r.w);
        material0_on_device = false;
    }
    if (engine.set_reference(ref, W, H, user_mask0.empty() ? nullptr : user_mask0.data()) != 0) {
        clear();
        return -3;
    }
    ensure_nodes((size_t)n0);
    check(cudaMemsetAsync(ubase.p, 0, (size_t)n0 * 4, st()), "memset");
    check(cudaMemsetAsync(vbase.p, 0, (size_t)n0 * 4, st()), "memset");
    check(cudaMemsetAsync(travel.p, 0, (size_t)n0 * 4, st()), "memset");
    check(cudaMemsetAsync(alive.p, 1, (size_t)n0, st()), "memset");
    check(cudaMemsetAsync(anchored.p, 0, (size_t)n0, st()), "memset");
    sync();
    alive_nodes = n0;
    anchors.assign((size_t)n0, Anchor{});
    anchored_h.assign((size_t)n0, 0);
    ready = true;
    return 0;
}

// nothing_to_follow (incremental_session.cpp:178-196): a frame with no node
// left to follow reports nothing and counts as processed.
int IncrementalSession::Impl::nothing_to_follow(FrameInfo fi, float* metrics, int metrics_len,
                                                const Progress& progress, FrameInfo* info) {
    frames++;
    fi.frame0_points = std::max(frame0_points, 0);
    if (info) *info = fi;
    if (metrics != nullptr) {
        const int len = metrics_len < 16 ? 0 : metrics_len >= 24 ? 24 : metrics_len == 18 ? 17 : metrics_len;
        std::fill_n(metrics, len, 0.0f);
    }
    if (progress) progress(100);
    return 0;
}

// match_anchor (incremental_math.cpp:238-276): the node's subset as cut on
// the reference where it was last clean, solved on the frame just run from
// the guess (gx, gy) of where the node is; accepted when it converges within
// kCorrAccept and lands within the allowed shift of the guess.
bool IncrementalSession::Impl::match(int node, float gx, float gy, float travel_k, float& mx, float& my,
                                     float& mcorr) {
    const Anchor& a = anchors[(size_t)node];
    const auto t0 = std::chrono::steady_clock::now();
    prof.matches++;
    const float max_shift = std::max(kReanchorMinShiftPx, kReanchorMaxShiftFraction * travel_k);
    const PatchSolve r = engine.solve_patch(a.patch.data(), a.side, a.ax, a.ay, gx - a.dx - (float)a.ax,
                                            gy - a.dy - (float)a.ay, params.subset_size, params.six);
    prof.match += ms_since(t0);
    if (!r.initialized || r.status != 0 || !(r.score <= kCorrAccept)) return false;
    const float nx = (float)a.ax + r.u + (1.0f + r.ux) * a.dx + r.uy * a.dy;
    const float ny = (float)a.ay + r.v + r.vx * a.dx + (1.0f + r.vy) * a.dy;
    if (!(length2(nx - gx, ny - gy) <= max_shift)) return false;
    mx = nx;
    my = ny;
    mcorr = r.score;
    return true;
}

// The forward warp of the frame-0 material mask onto the next reference
// (warp_material_mask, incremental_math.cpp:371-447): the totals of the
// followed nodes filled over the whole grid (Jacobi passes on the device),
// the samples per pixel from the field's largest local stretch, the window
// of frame 0 the grid covers, then the scatter and close on the device.
// False, with an empty mask, when no node is followed or the window is empty.
bool IncrementalSession::Impl::warp_mask(const uint8_t* alive_flags, const float* Ut, const float* Vt,
                                         std::vector<uint8_t>& out, Box& bb) {
    const auto t0 = std::chrono::steady_clock::now();
    const int half = params.subset_size / 2;
    const int margin = (kMaskExtrapCells + 1) * g0.step + half;
    int any = 0;
    zero_counters();
    check(dic::launch_inc_fill_init(n0, Ut, Vt, alive_flags, fillU[0].p, fillV[0].p, filled[0].p, counters.p, st()),
          "fill init");
    counters_to_host(&any, 13, 1);
    // every byte is written below: zeros on the early returns, the device's
    // mask otherwise (so a recycled buffer is not cleared first)
    if (out.size() != (size_t)W * H) out.assign((size_t)W * H, 0);
    bb = Box{};
    if (!any) {
        std::fill(out.begin(), out.end(), 0);
        prof.warp_mask += ms_since(t0);
        return false;
    }
    // fill passes in groups: a pass after the field is complete changes
    // nothing, so a group may overrun; the flag of each group's last pass
    // says whether to go on
    int cur = 0;
    const int max_passes = g0.gw + g0.gh + 2;
    constexpr int kGroup = 8;
    for (int pass = 0; pass < max_passes;) {
        const int group = std::min(kGroup, max_passes - pass);
        for (int k = 0; k < group; ++k, ++pass) {
            if (k == group - 1) check(cudaMemsetAsync(counters.p + 12, 0, sizeof(int), st()), "memset");
            check(dic::launch_inc_fill_pass(g0.gw, g0.gh, fillU[cur].p, fillV[cur].p, filled[cur].p, fillU[1 - cur].p,
                                            fillV[1 - cur].p, filled[1 - cur].p, counters.p, st()),
                  "fill pass");
            cur = 1 - cur;
        }
        int changed = 0;
        counters_to_host(&changed, 12, 1);
        if (!changed) break;
    }
    const double one = 1.0;
    check(cudaMemcpyAsync(counters.p + 10, &one, sizeof one, cudaMemcpyHostToDevice, st()), "H2D");
    check(dic::launch_inc_stretch(g0.gw, g0.gh, g0.step, fillU[cur].p, fillV[cur].p, counters.p, st()), "stretch");
    double stretch = 1.0;
    check(cudaMemcpyAsync(&stretch, counters.p + 10, sizeof stretch, cudaMemcpyDeviceToHost, st()), "D2H");
    sync();
    const int per_px = std::min(kMaskMaxSamplesPerPx, std::max(2, (int)std::ceil(stretch / 0.7)));
    const int X0 = std::max(0, g0.rect_x - margin), X1 = std::min(W - 1, g0.rect_x + (g0.gw - 1) * g0.step + margin);
    const int Y0 = std::max(0, g0.rect_y - margin), Y1 = std::min(H - 1, g0.rect_y + (g0.gh - 1) * g0.step + margin);
    if (X0 > X1 || Y0 > Y1) {
        std::fill(out.begin(), out.end(), 0);
        prof.warp_mask += ms_since(t0);
        return false;
    }
    int box[4] = {0, 0, 0, 0};
    const bool resident = material0_on_device;
    material0_on_device = true;
    if (engine.warp_mask(material0.data(), W, H, g0.gw, g0.gh, g0.rect_x, g0.rect_y, g0.step, fillU[cur].p,
                         fillV[cur].p, X0, X1, Y0, Y1, per_px, out.data(), box, resident) != 0)
        throw std::runtime_error("mask warp");
    bb = Box{box[0], box[1], box[2], box[3]};
    prof.warp_mask += ms_since(t0);
    return true;
}

// process_frame (incremental_session.cpp:289-549).
int IncrementalSession::Impl::process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len,
                                      Progress progress, FrameInfo* info) {
    if (!ready || out == nullptr || def == nullptr) return -3;
    FrameInfo fi;
    fi.reference_frame = ref_index;
    const int N = interval;
    bool will_update = N > 0 && since_update + 1 >= N;
    if (ref_index > 0 && alive_nodes == 0) return nothing_to_follow(fi, metrics, metrics_len, progress, info);

    int written = 0, frame0 = frame0_points;
    int hc[2] = {0, 0};
    const dic::IncFrame fr = frame();
    if (ref_index == 0) {
        // the same call as a fixed-reference run, straight into the caller's buffer
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = engine.run(def, user_mask0.empty() ? nullptr : user_mask0.data(), params, out, capacity,
                                  metrics, metrics_len, nullptr, progress, nullptr);
        prof.run += ms_since(t0);
        prof.runs++;
        if (rc < 0) return rc;
        written = rc;
        const DeviceField df = engine.last_field();
        if (frame0 < 0) frame0 = df.attempted;
        const dic::IncField f = field_of(df);
        need.ensure(std::max(need.n, (size_t)std::max(n0, 1)));
        zero_counters();
        check(dic::launch_inc_need(f, params.subset_size, need.p, st()), "need");
        check(dic::launch_inc_first(f, need.p, fr, st()), "first frame");
        check(dic::launch_inc_finish(n0, fr, nullptr, nullptr, nullptr, nullptr, counters.p, st()), "finish");
        counters_to_host(hc, 0, 2);
    } else {
        const int gw = params_k.step > 0 ? params_k.rect_w / params_k.step : 0;
        const int gh = params_k.step > 0 ? params_k.rect_h / params_k.step : 0;
        scratch.resize((size_t)std::max(gw * gh, 1) * 8);
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = engine.run(def, mask_k.data(), params_k, scratch.data(), (int)scratch.size(), metrics,
                                  metrics_len, nullptr, progress, nullptr);
        prof.run += ms_since(t0);
        prof.runs++;
        if (rc == -2) {
            // nothing of this reference's grid can be solved: every node is dropped
            fi.lost_this_frame = alive_nodes;
            check(cudaMemsetAsync(alive.p, 0, (size_t)n0, st()), "memset");
            for (Anchor& a : anchors) a.side = 0;
            std::fill(anchored_h.begin(), anchored_h.end(), 0);
            upload_anchored();
            sync();
            alive_nodes = 0;
            return nothing_to_follow(fi, metrics, metrics_len, progress, info);
        }
        if (rc < 0) return rc;
        const dic::IncField f = field_of(engine.last_field());
        need.ensure(std::max(need.n, (size_t)std::max(f.gw * f.gh, 1)));
        zero_counters();
        check(dic::launch_inc_need(f, params.subset_size, need.p, st()), "need");
        const float subset = (float)params.subset_size;
        const dic::IncStepArgs a{W,
                                 H,
                                 params.subset_size,
                                 kCoastMaxTravelSubsets * subset,
                                 kCoastTrustedTravelSubsets * subset,
                                 (float)(kCoastRadiusCells * f.step)};
        check(dic::launch_inc_step(g0, state(), f, need.p, a, fr, counters.p, match_list.p, match_info.p, st()),
              "node step");
        int m = 0;
        counters_to_host(&m, 2, 1);
        if (m > 0) {
            // the listed nodes' anchor matches, device solves run from here
            std::vector<int> nodes((size_t)m);
            std::vector<float> info3((size_t)m * 3);
            check(cudaMemcpyAsync(nodes.data(), match_list.p, (size_t)m * 4, cudaMemcpyDeviceToHost, st()), "D2H");
            check(cudaMemcpyAsync(info3.data(), match_info.p, (size_t)m * 12, cudaMemcpyDeviceToHost, st()), "D2H");
            sync();
            std::vector<int> order((size_t)m);
            for (int t = 0; t < m; ++t) order[(size_t)t] = t;
            std::sort(order.begin(), order.end(), [&](int p, int q) { return nodes[(size_t)p] < nodes[(size_t)q]; });
            std::vector<dic::IncMatch> rec((size_t)m);
            for (int t = 0; t < m; ++t) {
                const int s = order[(size_t)t], k = nodes[(size_t)s];
                const float x = (float)(g0.rect_x + (k % g0.gw) * g0.step);
                const float y = (float)(g0.rect_y + (k / g0.gw) * g0.step);
                const float Uk = info3[(size_t)s * 3], Vk = info3[(size_t)s * 3 + 1], tk = info3[(size_t)s * 3 + 2];
                float mx = 0.0f, my = 0.0f, mc = 0.0f;
                dic::IncMatch r{k, 0, 0.0f, 0.0f, 0.0f};
                if (match(k, x + Uk, y + Vk, tk, mx, my, mc)) {
                    r.ok = 1;
                    r.U = mx - x;
                    r.V = my - y;
                    r.corr = mc;
                }
                rec[(size_t)t] = r;
            }
            check(cudaMemcpyAsync(match_rec.p, rec.data(), rec.size() * sizeof(dic::IncMatch),
                                  cudaMemcpyHostToDevice, st()),
                  "H2D matches");
            check(dic::launch_inc_apply_matches(m, match_rec.p, fr, st()), "apply matches");
        }
        check(dic::launch_inc_finish(n0, fr, gu.p, gv.p, gcorr.p, gsolved.p, counters.p, st()), "finish");
        counters_to_host(hc, 0, 2);
        fi.taylor_fallbacks = hc[1];
        const auto t1 = std::chrono::steady_clock::now();
        written = engine.pack_field(g0.gw, g0.gh, g0.rect_x, g0.rect_y, g0.step, params.strain_window, gu.p, gv.p,
                                    gcorr.p, gsolved.p, out, capacity);
        prof.pack += ms_since(t1);
        if (written < 0) return written;
    }
    fi.tracked_points = hc[0];
    fi.frame0_points = std::max(frame0, 0);

    // the update rules: a failed solve never becomes the reference; an early
    // update when the points reported drop (N > 1)
    int rep = ref_reported;
    const int base = rep >= 0 ? rep : adopted_reported >= 0 ? adopted_reported : frame0;
    if (base > 0 && (float)written < kUpdateMinReported * (float)base) {
        will_update = false;
    } else if (N > 1) {
        if (rep < 0)
            rep = written;
        else if ((float)written < (1.0f - kEarlyUpdateDrop) * (float)rep)
            will_update = true;
    }

    if (!will_update) {
        frames++;
        since_update++;
        ref_reported = rep;
        frame0_points = frame0;
        if (info) *info = fi;
        return written;
    }

    // ------------------------------------------------------------ update
    const int before = ref_index == 0 ? fi.frame0_points : alive_nodes;
    const int init_keys[4] = {INT_MAX, INT_MAX, INT_MIN, INT_MIN};
    zero_counters();
    check(cudaMemcpyAsync(counters.p + 6, init_keys, sizeof init_keys, cudaMemcpyHostToDevice, st()), "H2D");
    check(dic::launch_inc_update(g0, state(), fr, travel_next.p, alive_next.p, counters.p, refresh_list.p,
                                 refresh_xy.p, drop_list.p, st()),
          "update");
    int hu[10] = {0};
    counters_to_host(hu, 0, 10);
    const int n_refresh = hu[3], n_drop = hu[4];
    int alive_new = hu[5];
    std::vector<int> refresh((size_t)n_refresh), drop((size_t)n_drop);
    std::vector<float> rxy((size_t)n_refresh * 2);
    if (n_refresh > 0) {
        check(cudaMemcpyAsync(refresh.data(), refresh_list.p, (size_t)n_refresh * 4, cudaMemcpyDeviceToHost, st()),
              "D2H");
        check(cudaMemcpyAsync(rxy.data(), refresh_xy.p, (size_t)n_refresh * 8, cudaMemcpyDeviceToHost, st()), "D2H");
    }
    if (n_drop > 0)
        check(cudaMemcpyAsync(drop.data(), drop_list.p, (size_t)n_drop * 4, cudaMemcpyDeviceToHost, st()), "D2H");
    sync();

    // the next reference: the warped material mask, and the rect that holds
    // every followed node (widened by a step) inside the frame
    std::vector<uint8_t> next_mask = std::move(spare_mask);  // the buffer of the mask before last
    Box bb;
    const bool warped = warp_mask(alive_next.p, U.p, V.p, next_mask, bb);
    Params next = params;
    Box grid_rect;
    if (alive_new > 0) {
        const float min_x = key_to_float(hu[6]), min_y = key_to_float(hu[7]);
        const float max_x = key_to_float(hu[8]), max_y = key_to_float(hu[9]);
        const int x0 = (int)std::floor(min_x), y0 = (int)std::floor(min_y);
        grid_rect = overlap(Box{x0, y0, (int)std::ceil(max_x) - x0 + g0.step, (int)std::ceil(max_y) - y0 + g0.step},
                            Box{0, 0, W, H});
    }
    next.rect_x = grid_rect.x;
    next.rect_y = grid_rect.y;
    next.rect_w = grid_rect.w;
    next.rect_h = grid_rect.h;
    next.strain_window = (int)std::min<int64_t>(next.strain_window, strain_window_cap(next));
    if (bb.area() == 0) {
        check(cudaMemsetAsync(alive_next.p, 0, (size_t)n0, st()), "memset");
        alive_new = 0;
    }
    const auto t2 = std::chrono::steady_clock::now();
    // the warped mask is still on the device where the warp left it
    if (engine.adopt_last_deformed(next_mask.data(), warped) != 0) return -3;
    prof.adopt += ms_since(t2);

    // anchors: drop, then cut the refreshed ones on the frame just adopted
    for (const int k : drop) {
        anchors[(size_t)k].side = 0;
        anchored_h[(size_t)k] = 0;
    }
#pragma omp parallel for schedule(static)
    for (long t = 0; t < (long)refresh.size(); ++t) {
        const int k = refresh[(size_t)t];
        if (cut_anchor(def, W, H, rxy[2 * (size_t)t], rxy[2 * (size_t)t + 1], params.subset_size,
                       anchors[(size_t)k]))
            anchored_h[(size_t)k] = 1;
    }
    if (n_drop > 0 || n_refresh > 0) upload_anchored();

    std::swap(ubase.p, U.p);
    std::swap(ubase.n, U.n);
    std::swap(vbase.p, V.p);
    std::swap(vbase.n, V.n);
    std::swap(alive.p, alive_next.p);
    std::swap(alive.n, alive_next.n);
    std::swap(travel.p, travel_next.p);
    std::swap(travel.n, travel_next.n);
    alive_nodes = alive_new;
    std::swap(mask_k, next_mask);
    spare_mask = std::move(next_mask);
    params_k = next;
    frames++;
    ref_index = frames;
    since_update = 0;
    ref_reported = -1;
    adopted_reported = written;
    frame0_points = frame0;
    fi.reference_updated = true;
    fi.lost_this_frame = std::max(0, before - alive_nodes);
    sync();
    if (info) *info = fi;
    return written;
}

IncrementalSession::IncrementalSession() : impl_(new Impl()) {
    // The session solves without a global model: a frame moves little against
    // its (updated) reference, and the restatement it is checked against runs
    // the same way.
    impl_->engine.set_global_motion(false);
}
IncrementalSession::~IncrementalSession() = default;

void IncrementalSession::reset() {
    impl_->clear();
    impl_->engine.reset();
}

bool IncrementalSession::initialized() const { return impl_->ready; }
int IncrementalSession::frames_processed() const { return impl_->frames; }
Engine& IncrementalSession::engine() { return impl_->engine; }
const FrameProfile& IncrementalSession::last_profile() const { return impl_->prof; }

int IncrementalSession::init(const uint8_t* ref, int w, int h, const uint8_t* mask, const Params& p,
                             int update_interval) {
    impl_->engine.reset();
    return impl_->init(ref, w, h, mask, p, update_interval);
}

int IncrementalSession::process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len,
                                Progress progress, FrameInfo* info) {
    FrameInfo fi;
    impl_->prof = FrameProfile{};
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    try {
        rc = impl_->process(def, out, capacity, metrics, metrics_len, progress, &fi);
    } catch (...) {
        // a cancel seen by a solve outside the frame's full-field run (an
        // anchor match) ends the frame the same way
        if (!impl_->engine.cancel_requested()) throw;
        rc = -99;
    }
    impl_->prof.total = ms_since(t0);
    if (info) *info = fi;
    return rc;
}

}  // namespace semper_b200
