// IncrementalSession over the device engine: see incremental.hpp.
#include "incremental.hpp"

#include <cmath>
#include <cstring>

namespace semper_b200 {

struct IncrementalSession::Impl {
    Engine engine;
    bool init = false;
    Params params;
    int interval = 0;
    int W = 0, H = 0;
    std::vector<uint8_t> mask;
    int frames = 0;
    int frame0_points = 0;
};

IncrementalSession::IncrementalSession() : impl_(new Impl()) {}
IncrementalSession::~IncrementalSession() = default;

void IncrementalSession::reset() {
    impl_->init = false;
    impl_->frames = 0;
    impl_->engine.reset();
}

bool IncrementalSession::initialized() const { return impl_->init; }
int IncrementalSession::frames_processed() const { return impl_->frames; }
Engine& IncrementalSession::engine() { return impl_->engine; }

int IncrementalSession::init(const uint8_t* ref, int w, int h, const uint8_t* mask, const Params& p,
                             int update_interval) {
    reset();
    if (!ref || w <= 0 || h <= 0 || update_interval < 0) return -3;
    Impl& I = *impl_;
    if (I.engine.set_reference(ref, w, h, mask) != 0) return -3;
    I.params = p;
    I.interval = update_interval;
    I.W = w;
    I.H = h;
    I.mask = mask ? std::vector<uint8_t>(mask, mask + (size_t)w * h) : std::vector<uint8_t>();
    if (update_interval != 0) return -3;  // only the fixed-reference mode in this build so far
    I.init = true;
    return 0;
}

int IncrementalSession::process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len,
                                Progress progress, FrameInfo* info) {
    Impl& I = *impl_;
    if (!I.init) return -3;
    const int rc = I.engine.run(def, I.mask.empty() ? nullptr : I.mask.data(), I.params, out, capacity, metrics,
                                metrics_len, nullptr, progress);
    if (rc >= 0) {
        I.frames++;
        if (info) {
            info->reference_frame = 0;
            info->reference_updated = false;
            info->frame0_points = 0;
            info->tracked_points = 0;
        }
    }
    return rc;
}

}  // namespace semper_b200
