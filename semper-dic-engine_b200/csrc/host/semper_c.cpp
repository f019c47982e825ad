// The C ABI (include/semper_c.h) over the device engine: a thin translation,
// no algorithm. Restates adapters/c/semper_c.cpp:25-238 on this library's
// engine — per-handle busy guard, per-handle cancel token with the reference's
// cancel window (include/semper/cancel.hpp:53-110), and an exception barrier
// at every entry (include/semper/guarded_call.hpp:22-44).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

#include "../../../include/semper_b200_ext.h"
#include "../../../include/semper_c.h"
#include "engine.hpp"
#include "gray.hpp"
#include "incremental.hpp"
#include "proposal.hpp"

using semper_b200::Engine;
using semper_b200::IncrementalSession;
using semper_b200::Params;

namespace {

template <class R, class F>
R guarded(R on_error, F&& body) noexcept {
    try {
        return body();
    } catch (...) {
        return on_error;
    }
}

// CancelToken + CancelScope on the engine's mapped flag.
struct CancelWindow {
    std::atomic<bool> open{false};
};

class HandleCall {
public:
    explicit HandleCall(std::atomic<bool>& b) noexcept : busy_(b), owned_(!b.exchange(true, std::memory_order_acquire)) {}
    ~HandleCall() {
        if (owned_) busy_.store(false, std::memory_order_release);
    }
    bool owned() const { return owned_; }

private:
    std::atomic<bool>& busy_;
    bool owned_;
};

Params to_params(const semper_params* p) {
    Params q;
    q.rect_x = p->rect_x;
    q.rect_y = p->rect_y;
    q.rect_w = p->rect_w;
    q.rect_h = p->rect_h;
    q.step = p->step;
    q.subset_size = p->subset_size;
    q.strain_window = p->strain_window;
    q.six = p->use_6x6_interpolator != 0;
    return q;
}

// io::decode_gray for raw buffers (src/io/image_codec.cpp:126-160): ALPHA_8
// when len == w*h, RGBA when len == 4*w*h (cvtColor RGBA2GRAY's fixed-point
// BT.601 luma, gray.hpp). Encoded images are not decoded by this build: empty
// result (a raw buffer is taken as raw even when its first bytes look like an
// image file's signature).
bool decode_raw(const uint8_t* data, size_t len, int w, int h, std::vector<uint8_t>& out) {
    if (!data || len == 0 || w <= 0 || h <= 0) return false;
    const uint64_t px = (uint64_t)w * (uint64_t)h;
    if (px > (uint64_t)INT32_MAX) return false;
    if ((uint64_t)len == px) {
        out.assign(data, data + px);
        return true;
    }
    if ((uint64_t)len == 4 * px) {
        out.resize(px);
        semper_b200::rgba_to_gray(data, (size_t)px, out.data());
        return true;
    }
    return false;
}

// decode_mask: no bytes is no mask; bytes that do not decode are an error.
bool decode_mask(const uint8_t* m, size_t len, int w, int h, std::vector<uint8_t>& out, bool& has) {
    has = false;
    if (m == nullptr || len == 0) return true;
    if (!decode_raw(m, len, w, h, out)) return false;
    has = true;
    return true;
}

}  // namespace

struct semper_engine {
    Engine engine;
    CancelWindow window;
    std::atomic<bool> busy{false};
    bool has_model = false;
    double model[9] = {};
};

struct semper_incremental {
    std::unique_ptr<IncrementalSession> session;
    CancelWindow window;
    int width = 0, height = 0;
    std::atomic<bool> busy{false};
};

namespace {

// CancelToken::begin / enter / end on an engine's flag.
void window_begin(Engine& e, CancelWindow& w) {
    e.clear_cancel();
    w.open.store(true, std::memory_order_release);
}
void window_enter(Engine& e, CancelWindow& w) {
    if (!w.open.exchange(false, std::memory_order_acq_rel)) e.clear_cancel();
}
struct WindowScope {
    Engine& e;
    CancelWindow& w;
    WindowScope(Engine& e_, CancelWindow& w_) : e(e_), w(w_) { window_begin(e, w); }
    ~WindowScope() { w.open.store(false, std::memory_order_release); }
};

}  // namespace

extern "C" {

SEMPER_C_API semper_engine* semper_create(void) {
    return guarded<semper_engine*>(nullptr, [] { return new semper_engine(); });
}

SEMPER_C_API void semper_destroy(semper_engine* eng) { delete eng; }

SEMPER_C_API int semper_set_reference(semper_engine* eng, const uint8_t* img, size_t img_len, const uint8_t* mask,
                                      size_t mask_len, int expected_w, int expected_h) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    guarded(0, [&] {
        eng->engine.reset();
        return 0;
    });
    if (img == nullptr || img_len == 0) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        std::vector<uint8_t> ref, m;
        if (!decode_raw(img, img_len, expected_w, expected_h, ref)) return SEMPER_ERR_INIT;
        bool has_mask = false;
        if (!decode_mask(mask, mask_len, expected_w, expected_h, m, has_mask)) return SEMPER_ERR_INIT;
        return eng->engine.set_reference(ref.data(), expected_w, expected_h, has_mask ? m.data() : nullptr) == 0
                   ? 0
                   : SEMPER_ERR_INIT;
    });
}

SEMPER_C_API int semper_run(semper_engine* eng, const uint8_t* def, size_t def_len, const uint8_t* mask,
                            size_t mask_len, const semper_params* params, float* out, int out_capacity,
                            float* metrics, int metrics_len, semper_progress_cb cb, void* user) {
    if (eng == nullptr || def == nullptr || def_len == 0 || params == nullptr || out == nullptr || out_capacity < 0)
        return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        WindowScope scope(eng->engine, eng->window);
        if (!eng->engine.has_reference()) return SEMPER_ERR_INIT;
        const int w = eng->engine.width(), h = eng->engine.height();
        std::vector<uint8_t> d, m;
        const uint8_t* frame = def;  // a raw 8-bit frame is used in place
        if ((uint64_t)def_len != (uint64_t)w * (uint64_t)h) {
            if (!decode_raw(def, def_len, w, h, d)) return SEMPER_ERR_INIT;
            frame = d.data();
        }
        bool has_mask = false;
        if (!decode_mask(mask, mask_len, w, h, m, has_mask)) return SEMPER_ERR_INIT;
        semper_b200::Progress progress;
        if (cb) progress = [cb, user](int pct) { cb(pct, user); };
        window_enter(eng->engine, eng->window);
        return eng->engine.run(frame, has_mask ? m.data() : nullptr, to_params(params), out, out_capacity,
                               metrics, metrics_len, eng->has_model ? eng->model : nullptr, progress);
    });
}

SEMPER_C_API void semper_cancel(semper_engine* eng) {
    if (eng != nullptr) eng->engine.request_cancel();
}

SEMPER_C_API const char* semper_version(void) { return "0.6.1"; }

SEMPER_C_API int semper_b200_run_device(semper_engine* eng, const uint8_t* d_def, const semper_params* params,
                                        float* d_out, int out_capacity, float* metrics, int metrics_len) {
    if (eng == nullptr || d_def == nullptr || params == nullptr || d_out == nullptr || out_capacity < 0)
        return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        WindowScope scope(eng->engine, eng->window);
        if (!eng->engine.has_reference()) return SEMPER_ERR_INIT;
        window_enter(eng->engine, eng->window);
        return eng->engine.run_device(d_def, nullptr, to_params(params), d_out, out_capacity, metrics, metrics_len,
                                      eng->has_model ? eng->model : nullptr);
    });
}

SEMPER_C_API void* semper_b200_stream(semper_engine* eng) {
    return eng ? (void*)eng->engine.stream() : nullptr;
}

SEMPER_C_API int semper_b200_last_timings(semper_engine* eng, float times[8], long long counts[5]) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    const semper_b200::PhaseTimes& t = eng->engine.last_times();
    if (times) {
        const float v[8] = {t.prep, t.pool, t.seed, t.mesh, t.path_a, t.path_b, t.strain, t.total};
        for (int i = 0; i < 8; ++i) times[i] = v[i];
    }
    if (counts) {
        counts[0] = t.icgn_iters;
        counts[1] = t.pixel_iters;
        counts[2] = t.path_a_tasks;
        counts[3] = t.path_a_pixel_iters;
        counts[4] = t.launches;
    }
    return 0;
}

SEMPER_C_API int semper_b200_fast_pass_shape(semper_engine* eng, int subset_size, int six) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    return eng->engine.fast_pass_shape(subset_size, six != 0);
}

SEMPER_C_API int semper_b200_incremental_profile(semper_incremental* inc, double out[16]) {
    if (inc == nullptr || out == nullptr) return SEMPER_ERR_INIT;
    const semper_b200::FrameProfile& f = inc->session->last_profile();
    const semper_b200::PhaseTimes& t = inc->session->engine().last_times();
    const double v[16] = {f.total, f.run, f.match, f.warp_mask, f.adopt, f.pack, (double)f.matches, (double)f.runs,
                          t.prep, t.pool, t.seed, t.mesh, t.path_a, t.path_b, t.strain, t.total};
    for (int i = 0; i < 16; ++i) out[i] = v[i];
    return 0;
}

SEMPER_C_API int semper_b200_set_global_model(semper_engine* eng, const double* h9) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    eng->has_model = h9 != nullptr;
    if (h9)
        for (int i = 0; i < 9; ++i) eng->model[i] = h9[i];
    return 0;
}

SEMPER_C_API int semper_b200_set_tma_wait_limit(semper_engine* eng, int polls) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    eng->engine.set_tma_wait_limit(polls);
    return 0;
}

SEMPER_C_API int semper_b200_last_tma_timeout(semper_engine* eng) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    return eng->engine.last_tma_timeout();
}

SEMPER_C_API int semper_b200_set_global_motion(semper_engine* eng, int on) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    eng->engine.set_global_motion(on != 0);
    return 0;
}

SEMPER_C_API int semper_b200_last_global_motion(semper_engine* eng, double out[18]) {
    if (eng == nullptr || out == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    const dic::GlobalSimilarity& g = eng->engine.last_global();
    out[0] = g.locked ? 1.0 : 0.0;
    out[1] = g.theta;
    out[2] = g.scale;
    out[3] = g.tx;
    out[4] = g.ty;
    out[5] = g.cx;
    out[6] = g.cy;
    out[7] = g.peak_rotation;
    out[8] = g.peak_translation;
    for (int i = 0; i < 9; ++i) out[9 + i] = g.H[i];
    return 0;
}

SEMPER_C_API semper_incremental* semper_incremental_create(void) {
    return guarded<semper_incremental*>(nullptr, [] {
        auto* inc = new semper_incremental();
        inc->session.reset(new IncrementalSession());
        return inc;
    });
}

SEMPER_C_API void semper_incremental_destroy(semper_incremental* inc) { delete inc; }

SEMPER_C_API int semper_incremental_init(semper_incremental* inc, const uint8_t* ref, size_t ref_len,
                                         const uint8_t* mask, size_t mask_len, int expected_w, int expected_h,
                                         const semper_params* params, int32_t update_interval) {
    if (inc == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(inc->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    guarded(0, [&] {
        inc->session->reset();
        return 0;
    });
    inc->width = inc->height = 0;
    if (ref == nullptr || ref_len == 0 || params == nullptr) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        std::vector<uint8_t> r, m;
        if (!decode_raw(ref, ref_len, expected_w, expected_h, r)) return SEMPER_ERR_INIT;
        bool has_mask = false;
        if (!decode_mask(mask, mask_len, expected_w, expected_h, m, has_mask)) return SEMPER_ERR_INIT;
        const int rc = inc->session->init(r.data(), expected_w, expected_h, has_mask ? m.data() : nullptr,
                                          to_params(params), update_interval);
        inc->width = rc == 0 ? expected_w : 0;
        inc->height = rc == 0 ? expected_h : 0;
        return rc;
    });
}

SEMPER_C_API int semper_incremental_process(semper_incremental* inc, const uint8_t* def, size_t def_len, float* out,
                                            int out_capacity, float* metrics, int metrics_len,
                                            semper_incremental_info* info, semper_progress_cb cb, void* user) {
    if (inc == nullptr || def == nullptr || def_len == 0 || out == nullptr || out_capacity < 0)
        return SEMPER_ERR_INIT;
    HandleCall call(inc->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    if (!inc->session->initialized()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        Engine& e = inc->session->engine();
        WindowScope scope(e, inc->window);
        std::vector<uint8_t> d;
        if (!decode_raw(def, def_len, inc->width, inc->height, d)) return SEMPER_ERR_INIT;
        semper_b200::Progress progress;
        if (cb) progress = [cb, user](int pct) { cb(pct, user); };
        window_enter(e, inc->window);
        semper_b200::FrameInfo fi;
        const int rc = inc->session->process(d.data(), out, out_capacity, metrics, metrics_len, progress, &fi);
        if (info != nullptr && rc >= 0) {
            info->reference_frame = fi.reference_frame;
            info->reference_updated = fi.reference_updated ? 1 : 0;
            info->tracked_points = fi.tracked_points;
            info->frame0_points = fi.frame0_points;
            info->taylor_fallbacks = fi.taylor_fallbacks;
            info->lost_this_frame = fi.lost_this_frame;
        }
        return rc;
    });
}

SEMPER_C_API void semper_incremental_cancel(semper_incremental* inc) {
    if (inc != nullptr && inc->session) inc->session->engine().request_cancel();
}

}  // extern "C"

struct semper_b200_proposal {
    std::unique_ptr<semper_b200::ProposalNet> net;
};

namespace {

dic::PpSynth synth_cfg(const float cfg[6]) {
    dic::PpSynth c;
    c.max_rot = cfg[0];
    c.max_stretch = cfg[1];
    c.max_shear = cfg[2];
    c.max_shift = cfg[3];
    c.noise = cfg[4];
    c.f = (int)cfg[5];
    return c;
}

// Synthetic pairs must fit the speckle image with their whole warped reach.
bool synth_ok(const uint8_t* speckle, int32_t w, int32_t h, const float* cfg) {
    if (!speckle || !cfg || w < 64 || h < 64) return false;
    const int f = (int)cfg[5];
    if (f < 1 || f > 16 || !(cfg[1] >= 0.0f && cfg[1] < 0.5f) || !(cfg[2] >= 0.0f && cfg[2] < 0.5f) ||
        !(cfg[3] >= 0.0f) || !(cfg[4] >= 0.0f))
        return false;
    const float reach = 32.0f * f * 1.4143f * (1.0f + cfg[1] + cfg[2]) + cfg[3] + 4.0f;
    return 2.0f * reach < (float)std::min(w, h);
}

}  // namespace

extern "C" {

SEMPER_C_API semper_b200_proposal* semper_b200_proposal_create(int32_t max_batch) {
    return guarded<semper_b200_proposal*>(nullptr, [&] {
        auto* p = new semper_b200_proposal();
        p->net.reset(new semper_b200::ProposalNet(max_batch));
        return p;
    });
}

SEMPER_C_API void semper_b200_proposal_destroy(semper_b200_proposal* p) { delete p; }

SEMPER_C_API int64_t semper_b200_proposal_param_count(void) {
    return (int64_t)semper_b200::ProposalNet::param_count();
}

SEMPER_C_API int semper_b200_proposal_set_params(semper_b200_proposal* p, const float* params, int64_t n) {
    if (!p || !params || n != (int64_t)semper_b200::ProposalNet::param_count()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->set_params(params);
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_get_params(semper_b200_proposal* p, float* params, int64_t n) {
    if (!p || !params || n != (int64_t)semper_b200::ProposalNet::param_count()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->get_params(params);
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_forward(semper_b200_proposal* p, const float* x, int32_t batch, float* out) {
    if (!p || !x || !out || batch <= 0 || batch > p->net->max_batch()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->forward_host(x, batch, out);
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_gradients(semper_b200_proposal* p, const float* x, const float* target,
                                                int32_t batch, float* grads, float* loss) {
    if (!p || !x || !target || !grads || batch <= 0 || batch > p->net->max_batch()) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        const float l = p->net->gradients_host(x, target, batch, grads);
        if (loss) *loss = l;
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_synth(semper_b200_proposal* p, const uint8_t* speckle, int32_t w, int32_t h,
                                            const float cfg[6], uint64_t seed, int32_t batch, float* x,
                                            float* target) {
    if (!p || !x || !target || batch <= 0 || batch > p->net->max_batch() || !synth_ok(speckle, w, h, cfg))
        return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->synth_host(speckle, w, h, synth_cfg(cfg), seed, batch, x, target);
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_train(semper_b200_proposal* p, const uint8_t* speckle, int32_t w, int32_t h,
                                            const float cfg[6], int32_t steps, int32_t batch, float lr,
                                            uint64_t seed, float* losses) {
    if (!p || steps < 0 || batch <= 0 || batch > p->net->max_batch() || !synth_ok(speckle, w, h, cfg))
        return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->train(speckle, w, h, synth_cfg(cfg), steps, batch, lr, seed, losses);
        return 0;
    });
}

SEMPER_C_API int semper_b200_proposal_predict_warped(semper_b200_proposal* p, const uint8_t* ref,
                                                     const uint8_t* def, int32_t w, int32_t h, const float* maps,
                                                     int32_t batch, int32_t f, float* out) {
    if (!p || !ref || !def || !maps || !out || w < 2 || h < 2 || f < 1 || f > 16 || batch <= 0 ||
        batch > p->net->max_batch())
        return SEMPER_ERR_INIT;
    for (int32_t k = 0; k < 8 * batch; ++k)
        if (!std::isfinite(maps[k]) || (k % 8 < 2 && std::fabs(maps[k]) > 1e7f)) return SEMPER_ERR_INIT;
    return guarded(SEMPER_ERR_INIT, [&] {
        p->net->predict_warped_host(ref, def, w, h, maps, batch, f, out);
        return 0;
    });
}

SEMPER_C_API int semper_b200_set_proposal(semper_engine* eng, semper_b200_proposal* p, int learned) {
    if (eng == nullptr) return SEMPER_ERR_INIT;
    HandleCall call(eng->busy);
    if (!call.owned()) return SEMPER_ERR_INIT;
    if (learned < 0 || learned > 2) return SEMPER_ERR_INIT;
    eng->engine.set_proposal(p ? p->net.get() : nullptr, learned);
    return 0;
}

SEMPER_C_API int semper_b200_learned_guesses(semper_engine* eng, float* uv, int32_t capacity) {
    if (eng == nullptr || capacity < 0 || (uv == nullptr && capacity > 0)) return SEMPER_ERR_INIT;
    const std::vector<float>& g = eng->engine.last_learned().anchor_uv;
    const int32_t n = (int32_t)(g.size() / 2);
    if (capacity < 2 * n) return n;
    std::copy(g.begin(), g.end(), uv);
    return n;
}

SEMPER_C_API int semper_b200_last_learned(semper_engine* eng, double out[18]) {
    if (eng == nullptr || out == nullptr) return SEMPER_ERR_INIT;
    const semper_b200::LearnedSeed& L = eng->engine.last_learned();
    const double v[9] = {L.ran ? 1.0 : 0.0, L.proposed ? 1.0 : 0.0, L.kept ? 1.0 : 0.0, (double)L.pairs,
                         (double)L.inliers, (double)L.anchors, L.err_mean, L.err_max, L.ms};
    for (int i = 0; i < 9; ++i) out[i] = v[i];
    for (int i = 0; i < 9; ++i) out[9 + i] = L.H[i];
    return 0;
}

}  // extern "C"
