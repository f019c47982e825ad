// IncrementalSession over the device engine: the session logic of
// incremental_core.hpp, every solve, adoption and packing on the device.
#include "incremental.hpp"

#include <chrono>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "incremental_core.hpp"

namespace semper_b200 {

namespace {

Params to_params(const semper_inc::IncParams& p) {
    Params q;
    q.rect_x = p.rect_x;
    q.rect_y = p.rect_y;
    q.rect_w = p.rect_w;
    q.rect_h = p.rect_h;
    q.step = p.step;
    q.subset_size = p.subset_size;
    q.strain_window = p.strain_window;
    q.six = p.six;
    return q;
}

semper_inc::IncParams from_params(const Params& q) {
    semper_inc::IncParams p;
    p.rect_x = q.rect_x;
    p.rect_y = q.rect_y;
    p.rect_w = q.rect_w;
    p.rect_h = q.rect_h;
    p.step = q.step;
    p.subset_size = q.subset_size;
    p.strain_window = q.strain_window;
    p.six = q.six;
    return p;
}

double ms_since(std::chrono::steady_clock::time_point t) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}

// The solver backend of the session: the device engine.
struct DeviceBackend {
    Engine& e;
    FrameProfile prof;

    int validate(semper_inc::IncParams& p, int W, int H) {
        Params q = to_params(p);
        const int rc = check_params(q, W, H);
        p = from_params(q);
        return rc;
    }
    int vsg_count(int step, int window) { return vsg_window_nodes(step, window); }
    int set_reference(const uint8_t* gray, int W, int H, const uint8_t* mask) {
        return e.set_reference(gray, W, H, mask);
    }
    int run(const uint8_t* def, const uint8_t* mask, const semper_inc::IncParams& p, float* out, int capacity,
            float* metrics, int metrics_len, const std::function<void(int)>& progress,
            semper_inc::SolveCapture* cap) {
        Capture c;
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = e.run(def, mask, to_params(p), out, capacity, metrics, metrics_len, nullptr, progress, &c);
        prof.run += ms_since(t0);
        prof.runs++;
        if (rc < 0) return rc;
        cap->gridW = c.gridW;
        cap->gridH = c.gridH;
        cap->rect_x = c.rect_x;
        cap->rect_y = c.rect_y;
        cap->step = c.step;
        cap->attempted = c.attempted;
        cap->u = std::move(c.u);
        cap->v = std::move(c.v);
        cap->ux = std::move(c.ux);
        cap->uy = std::move(c.uy);
        cap->vx = std::move(c.vx);
        cap->vy = std::move(c.vy);
        cap->corr = std::move(c.corr);
        cap->solved = std::move(c.solved);
        cap->median_valid = std::move(c.median_valid);
        cap->median_rejected = c.median_rejected;
        return rc;
    }
    int adopt(const uint8_t* mask) {
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = e.adopt_last_deformed(mask);
        prof.adopt += ms_since(t0);
        return rc;
    }
    int pack(const semper_inc::GridGeom& g, int window, const std::vector<float>& u, const std::vector<float>& v,
             const std::vector<float>& corr, const std::vector<unsigned char>& solved, float* out, int capacity) {
        const auto t0 = std::chrono::steady_clock::now();
        const int rc = e.pack_field(g.gridW, g.gridH, g.rect_x, g.rect_y, g.step, window, u.data(), v.data(),
                                    corr.data(), solved.data(), out, capacity);
        prof.pack += ms_since(t0);
        return rc;
    }
    semper_inc::Rect warp_mask(const std::vector<uint8_t>& mask0, int W, int H, const semper_inc::GridGeom& g,
                               const semper_inc::MaskWarpPlan& p, std::vector<uint8_t>& out) {
        const auto t0 = std::chrono::steady_clock::now();
        out.resize((size_t)W * H);
        int box[4] = {0, 0, 0, 0};
        if (e.warp_mask(mask0.data(), W, H, g.gridW, g.gridH, g.rect_x, g.rect_y, g.step, p.U.data(), p.V.data(),
                        p.X0, p.X1, p.Y0, p.Y1, p.per_px, out.data(), box) != 0)
            throw std::runtime_error("mask warp");
        prof.warp_mask += ms_since(t0);
        return semper_inc::Rect{box[0], box[1], box[2], box[3]};
    }
    bool match_anchor(const semper_inc::CoastAnchor& a, int subset, bool six, float gx, float gy, float max_shift,
                      float& x, float& y, float& corr) {
        // guess for the centre pixel: the node's guess less its offset from it
        const auto t0 = std::chrono::steady_clock::now();
        prof.matches++;
        struct Add {
            double& m;
            std::chrono::steady_clock::time_point t;
            ~Add() { m += ms_since(t); }
        } add{prof.match, t0};
        const PatchSolve r = e.solve_patch(a.patch.data(), a.size, a.ax, a.ay, gx - a.dx - (float)a.ax,
                                           gy - a.dy - (float)a.ay, subset, six);
        if (!r.initialized) return false;
        return semper_inc::accept_anchor_match(a, r.status, r.score, r.u, r.v, r.ux, r.uy, r.vx, r.vy, gx, gy,
                                               max_shift, x, y, corr);
    }
};

}  // namespace

struct IncrementalSession::Impl {
    Engine engine;
    DeviceBackend backend{engine, FrameProfile{}};
    semper_inc::IncrementalCore<DeviceBackend> core{backend};
};

// The session solves without a global model: the motion between a frame and
// its (updated) reference stays small, and the restatement the session is
// checked against runs the same way.
IncrementalSession::IncrementalSession() : impl_(new Impl()) { impl_->engine.set_global_motion(false); }
IncrementalSession::~IncrementalSession() = default;

void IncrementalSession::reset() {
    impl_->core.clear();
    impl_->engine.reset();
}

bool IncrementalSession::initialized() const { return impl_->core.initialized(); }
int IncrementalSession::frames_processed() const { return impl_->core.frames_processed(); }
Engine& IncrementalSession::engine() { return impl_->engine; }

int IncrementalSession::init(const uint8_t* ref, int w, int h, const uint8_t* mask, const Params& p,
                             int update_interval) {
    impl_->engine.reset();
    return impl_->core.init(ref, w, h, mask, from_params(p), update_interval);
}

const FrameProfile& IncrementalSession::last_profile() const { return impl_->backend.prof; }

int IncrementalSession::process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len,
                                Progress progress, FrameInfo* info) {
    semper_inc::FrameInfo fi;
    impl_->backend.prof = FrameProfile{};
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    try {
        rc = impl_->core.process(def, out, capacity, metrics, metrics_len, progress, &fi);
    } catch (...) {
        // a cancel seen by a solve outside the frame's full-field run (an
        // anchor match) ends the frame the same way
        if (!impl_->engine.cancel_requested()) throw;
        rc = -99;
    }
    impl_->backend.prof.total = ms_since(t0);
    if (info) {
        info->reference_frame = fi.reference_frame;
        info->reference_updated = fi.reference_updated;
        info->tracked_points = fi.tracked_points;
        info->frame0_points = fi.frame0_points;
        info->taylor_fallbacks = fi.taylor_fallbacks;
        info->lost_this_frame = fi.lost_this_frame;
    }
    return rc;
}

}  // namespace semper_b200
