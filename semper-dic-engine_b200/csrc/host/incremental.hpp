// IncrementalSession on the device engine (include/semper/incremental.hpp:74-117).
#pragma once
#include <cstdint>
#include <memory>
#include <vector>

#include "engine.hpp"

namespace semper_b200 {

struct FrameInfo {
    int reference_frame = 0;
    bool reference_updated = false;
    int tracked_points = 0;
    int frame0_points = 0;
    int taylor_fallbacks = 0;
    int lost_this_frame = 0;
};

// Host wall time of the last process() call by step, ms, and the number of
// anchor matches it made (measurement only).
struct FrameProfile {
    double total = 0, run = 0, match = 0, warp_mask = 0, adopt = 0, pack = 0;
    int matches = 0, runs = 0;
};

class IncrementalSession {
public:
    IncrementalSession();
    ~IncrementalSession();
    // init (src/pipeline/incremental_session.cpp:120-268): 0, -2, -3, -4.
    int init(const uint8_t* ref, int w, int h, const uint8_t* mask, const Params& p, int update_interval);
    // process_frame (incremental_session.cpp:270-549).
    int process(const uint8_t* def, float* out, int capacity, float* metrics, int metrics_len, Progress progress,
                FrameInfo* info);
    void reset();
    bool initialized() const;
    int frames_processed() const;
    Engine& engine();
    const FrameProfile& last_profile() const;

    struct Impl;

private:
    std::unique_ptr<Impl> impl_;
};

}  // namespace semper_b200
