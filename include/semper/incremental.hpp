/*
 * semper/incremental.hpp — incremental (updated-reference) DIC as a C++ API:
 * a drop-in for the reference's Semper::pipeline::IncrementalSession
 * (include/semper/incremental.hpp:1-122), solved on the GPU by this library.
 * Images are GrayView (semper/pipeline.hpp), with cv::Mat overloads when
 * OpenCV's headers are on the include path. Link against libsemper_b200.so.
 */
#ifndef SEMPER_INCREMENTAL_HPP
#define SEMPER_INCREMENTAL_HPP

#include <memory>
#include <string>

#include <semper/cancel.hpp>
#include <semper/pipeline.hpp>

namespace Semper {
namespace pipeline {

/* The frame-0 grid (`field`, as for run_full_field) and how many solved
   frames pass before the reference moves to the latest one (0: never, 1:
   every frame, N: every N frames or at a 5 % drop of reported points)
   (incremental.hpp:15-37). */
struct IncrementalParams {
    FullFieldParams field;
    int update_interval = 1;
};

/* Per-frame bookkeeping in frame-0 node counts (incremental.hpp:39-47). */
struct IncrementalFrameInfo {
    int reference_frame = 0;
    bool reference_updated = false;
    int tracked_points = 0;
    int frame0_points = 0;
    int taylor_fallbacks = 0;
    int lost_this_frame = 0;
};

/* Total displacement from frame 0 at the frame-0 grid, through a chain of
   references (incremental.hpp:49-118). One session per sequence, one call at
   a time. */
class SEMPER_CXX_API IncrementalSession {
public:
    IncrementalSession();
    ~IncrementalSession();
    IncrementalSession(const IncrementalSession&) = delete;
    IncrementalSession& operator=(const IncrementalSession&) = delete;
    IncrementalSession(IncrementalSession&&) noexcept;
    IncrementalSession& operator=(IncrementalSession&&) noexcept;

    /* Start at frame 0. 0, or -2 (ROI), -3 (empty image, bad interval),
       kBadStrainWindow. `roi_mask` may be empty or of any size. */
    int init(const GrayView& ref_gray, const GrayView& roi_mask, const IncrementalParams& params);

    /* Solve the next frame: the points written (>= 0) or a negative code as
       run_full_field (-3 also when not initialised or for a frame of another
       size). Cancelled by request_cancel(). */
    int process_frame(const GrayView& def_gray, float* output, int output_capacity, float* metrics,
                      int metrics_len, ProgressCallback on_progress = nullptr,
                      IncrementalFrameInfo* info = nullptr);
    /* The same, cancelled by `cancel` only. */
    int process_frame(const GrayView& def_gray, float* output, int output_capacity, float* metrics,
                      int metrics_len, CancelToken& cancel, ProgressCallback on_progress = nullptr,
                      IncrementalFrameInfo* info = nullptr);

#ifdef SEMPER_HAVE_OPENCV
    int init(const cv::Mat& ref_gray, const cv::Mat& roi_mask, const IncrementalParams& params) {
        return init(gray_view(ref_gray), gray_view(roi_mask), params);
    }
    int process_frame(const cv::Mat& def_gray, float* output, int output_capacity, float* metrics,
                      int metrics_len, ProgressCallback on_progress = nullptr,
                      IncrementalFrameInfo* info = nullptr) {
        return process_frame(gray_view(def_gray), output, output_capacity, metrics, metrics_len,
                             std::move(on_progress), info);
    }
    int process_frame(const cv::Mat& def_gray, float* output, int output_capacity, float* metrics,
                      int metrics_len, CancelToken& cancel, ProgressCallback on_progress = nullptr,
                      IncrementalFrameInfo* info = nullptr) {
        return process_frame(gray_view(def_gray), output, output_capacity, metrics, metrics_len, cancel,
                             std::move(on_progress), info);
    }
#endif

    void reset();
    bool initialized() const;
    /* Frames solved so far (frame 0 not counted). */
    int frames_processed() const;
    /* The most points one frame can return (the frame-0 grid's node count). */
    int max_points() const;
    /* Accepted for the reference's interface; this build writes no debug
       output. */
    void set_debug_dir(std::string dir);

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace pipeline
}  // namespace Semper

#endif
