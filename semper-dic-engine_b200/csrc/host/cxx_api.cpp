// The C++ API (include/semper/pipeline.hpp, incremental.hpp, cancel.hpp) over
// the device engine and the device incremental session: argument checks,
// image views made contiguous, ROI masks resized to the reference, and the
// caller's cancel token carried to the engine's flag while a solve runs.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../../../include/semper/incremental.hpp"
#include "../../../include/semper/pipeline.hpp"
#include "engine.hpp"
#include "gray.hpp"
#include "incremental.hpp"

namespace Semper {
namespace pipeline {

namespace {

CancelToken g_token;

// The pixels of a view as one contiguous width x height block: the view's own
// memory when its rows are packed, else a copy in `keep`.
const uint8_t* packed(const GrayView& v, std::vector<uint8_t>& keep) {
    if (v.row_bytes() == (size_t)v.width) return v.data;
    keep.resize((size_t)v.width * v.height);
    for (int y = 0; y < v.height; ++y)
        std::copy(v.data + (size_t)y * v.row_bytes(), v.data + (size_t)y * v.row_bytes() + v.width,
                  keep.data() + (size_t)y * v.width);
    return keep.data();
}

// An ROI mask for a w x h image: none for an empty view, the view itself
// (made contiguous) at the right size, else its nearest-neighbour resize
// (full_field_solver.cpp:191-194). False for a malformed view.
bool mask_for(const GrayView& m, int w, int h, std::vector<uint8_t>& keep, const uint8_t*& out) {
    out = nullptr;
    if (m.data == nullptr && m.width == 0 && m.height == 0) return true;
    if (m.empty()) return m.data == nullptr && m.width >= 0;
    if (m.width == w && m.height == h) {
        out = packed(m, keep);
        return true;
    }
    semper_b200::resize_nearest(m.data, m.width, m.height, m.row_bytes(), w, h, keep);
    out = keep.data();
    return true;
}

semper_b200::Params to_params(const FullFieldParams& p) {
    semper_b200::Params q;
    q.rect_x = p.rect_x;
    q.rect_y = p.rect_y;
    q.rect_w = p.rect_w;
    q.rect_h = p.rect_h;
    q.step = p.step;
    q.subset_size = p.subset_size;
    q.strain_window = p.strain_window;
    q.six = p.use_6x6_interpolator;
    return q;
}

// While a solve runs, a request on the caller's token reaches the engine's
// flag (which the host steps and the device kernels poll) within about a
// millisecond.
class CancelRelay {
public:
    CancelRelay(CancelToken& t, semper_b200::Engine& e) : t_(t), e_(e) {
        t_.enter();
        e_.clear_cancel();
        if (t_.requested()) e_.request_cancel();
        th_ = std::thread([this] {
            while (!done_.load(std::memory_order_acquire)) {
                if (t_.requested()) e_.request_cancel();
                std::this_thread::sleep_for(std::chrono::microseconds(500));
            }
        });
    }
    ~CancelRelay() {
        done_.store(true, std::memory_order_release);
        th_.join();
    }

private:
    CancelToken& t_;
    semper_b200::Engine& e_;
    std::atomic<bool> done_{false};
    std::thread th_;
};

semper_b200::Progress progress_of(const ProgressCallback& cb) {
    if (!cb) return nullptr;
    return [cb](int pct) { cb(pct); };
}

}  // namespace

void request_cancel() { g_token.request(); }
void clear_cancel() { g_token.clear(); }
bool cancel_requested() { return g_token.requested(); }
namespace detail {
CancelToken& global_cancel_token() noexcept { return g_token; }
}  // namespace detail

// ------------------------------------------------------------ ReferenceCache

struct ReferenceCache::Impl {
    semper_b200::Engine engine;
    bool has = false;
};

ReferenceCache::ReferenceCache() : impl(new Impl()) {}
ReferenceCache::~ReferenceCache() = default;

void ReferenceCache::reset() {
    impl->engine.reset();
    impl->has = false;
    width = height = 0;
}

void ReferenceCache::set_from_gray(const GrayView& gray, const GrayView& roi_mask) {
    reset();
    if (gray.empty()) throw std::invalid_argument("set_from_gray: empty image");
    std::vector<uint8_t> gkeep, mkeep;
    const uint8_t* g = packed(gray, gkeep);
    const uint8_t* m = nullptr;
    if (!mask_for(roi_mask, gray.width, gray.height, mkeep, m))
        throw std::invalid_argument("set_from_gray: malformed mask");
    if (impl->engine.set_reference(g, gray.width, gray.height, m) != 0)
        throw std::runtime_error("set_from_gray: the reference could not be prepared");
    impl->has = true;
    width = gray.width;
    height = gray.height;
}

int run_full_field(ReferenceCache& cache, const GrayView& def_gray, const GrayView& roi_mask,
                   const FullFieldParams& params, float* output_ptr, int output_capacity, float* metrics,
                   int metrics_len, CancelToken& cancel, ProgressCallback on_progress) {
    if (!cache.impl || !cache.impl->has || output_ptr == nullptr || output_capacity < 0) return -3;
    if (def_gray.empty() || def_gray.width != cache.width || def_gray.height != cache.height) return -3;
    try {
        std::vector<uint8_t> dkeep, mkeep;
        const uint8_t* d = packed(def_gray, dkeep);
        const uint8_t* m = nullptr;
        if (!mask_for(roi_mask, cache.width, cache.height, mkeep, m)) return -3;
        CancelRelay relay(cancel, cache.impl->engine);
        return cache.impl->engine.run(d, m, to_params(params), output_ptr, output_capacity, metrics, metrics_len,
                                      nullptr, progress_of(on_progress));
    } catch (const std::exception&) {
        return -3;
    }
}

int run_full_field(ReferenceCache& cache, const GrayView& def_gray, const GrayView& roi_mask,
                   const FullFieldParams& params, float* output_ptr, int output_capacity, float* metrics,
                   int metrics_len, ProgressCallback on_progress) {
    return run_full_field(cache, def_gray, roi_mask, params, output_ptr, output_capacity, metrics, metrics_len,
                          g_token, std::move(on_progress));
}

// ------------------------------------------------------ IncrementalSession

struct IncrementalSession::Impl {
    semper_b200::IncrementalSession session;
    int width = 0, height = 0, max_points = 0;
};

IncrementalSession::IncrementalSession() : impl_(new Impl()) {}
IncrementalSession::~IncrementalSession() = default;
IncrementalSession::IncrementalSession(IncrementalSession&&) noexcept = default;
IncrementalSession& IncrementalSession::operator=(IncrementalSession&&) noexcept = default;

int IncrementalSession::init(const GrayView& ref_gray, const GrayView& roi_mask, const IncrementalParams& params) {
    if (!impl_) impl_.reset(new Impl());
    impl_->session.reset();
    impl_->width = impl_->height = impl_->max_points = 0;
    if (ref_gray.empty() || params.update_interval < 0) return -3;
    try {
        std::vector<uint8_t> gkeep, mkeep;
        const uint8_t* g = packed(ref_gray, gkeep);
        const uint8_t* m = nullptr;
        if (!mask_for(roi_mask, ref_gray.width, ref_gray.height, mkeep, m)) return -3;
        const semper_b200::Params p = to_params(params.field);
        const int rc = impl_->session.init(g, ref_gray.width, ref_gray.height, m, p, params.update_interval);
        if (rc != 0) return rc;
        semper_b200::Params clipped = p;
        semper_b200::check_params(clipped, ref_gray.width, ref_gray.height);
        impl_->width = ref_gray.width;
        impl_->height = ref_gray.height;
        impl_->max_points = (clipped.rect_w / clipped.step) * (clipped.rect_h / clipped.step);
        return 0;
    } catch (const std::exception&) {
        impl_->session.reset();
        return -3;
    }
}

int IncrementalSession::process_frame(const GrayView& def_gray, float* output, int output_capacity, float* metrics,
                                      int metrics_len, CancelToken& cancel, ProgressCallback on_progress,
                                      IncrementalFrameInfo* info) {
    if (!impl_ || !impl_->session.initialized() || output == nullptr || output_capacity < 0) return -3;
    if (def_gray.empty() || def_gray.width != impl_->width || def_gray.height != impl_->height) return -3;
    try {
        std::vector<uint8_t> dkeep;
        const uint8_t* d = packed(def_gray, dkeep);
        semper_b200::FrameInfo fi;
        int rc;
        {
            CancelRelay relay(cancel, impl_->session.engine());
            rc = impl_->session.process(d, output, output_capacity, metrics, metrics_len, progress_of(on_progress),
                                        &fi);
        }
        if (info) {
            info->reference_frame = fi.reference_frame;
            info->reference_updated = fi.reference_updated;
            info->tracked_points = fi.tracked_points;
            info->frame0_points = fi.frame0_points;
            info->taylor_fallbacks = fi.taylor_fallbacks;
            info->lost_this_frame = fi.lost_this_frame;
        }
        return rc;
    } catch (const std::exception&) {
        return -3;
    }
}

int IncrementalSession::process_frame(const GrayView& def_gray, float* output, int output_capacity, float* metrics,
                                      int metrics_len, ProgressCallback on_progress, IncrementalFrameInfo* info) {
    return process_frame(def_gray, output, output_capacity, metrics, metrics_len, g_token, std::move(on_progress),
                         info);
}

void IncrementalSession::reset() {
    if (!impl_) return;
    impl_->session.reset();
    impl_->width = impl_->height = impl_->max_points = 0;
}
bool IncrementalSession::initialized() const { return impl_ && impl_->session.initialized(); }
int IncrementalSession::frames_processed() const { return impl_ ? impl_->session.frames_processed() : 0; }
int IncrementalSession::max_points() const { return impl_ ? impl_->max_points : 0; }
void IncrementalSession::set_debug_dir(std::string) {}

}  // namespace pipeline
}  // namespace Semper
