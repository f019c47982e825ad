/*
 * semper/pipeline.hpp — the full-field solve as a C++ API: a drop-in for the
 * reference's Semper::pipeline::ReferenceCache and run_full_field
 * (include/semper/pipeline.hpp:35-115), solved on the GPU by this library.
 *
 * Images are passed as GrayView, a view of 8-bit gray pixels in host memory
 * (rows `stride` bytes apart). When OpenCV's headers are on the include path,
 * the reference's cv::Mat overloads are available too (inline, converting a
 * CV_8UC1 matrix to a view); this library itself does not use OpenCV.
 *
 * Link against libsemper_b200.so.
 */
#ifndef SEMPER_PIPELINE_HPP
#define SEMPER_PIPELINE_HPP

#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>

#include <semper/cancel.hpp>

#if defined(__has_include)
#if __has_include(<opencv2/core.hpp>)
#include <opencv2/core.hpp>
#define SEMPER_HAVE_OPENCV 1
#endif
#endif

namespace Semper {
namespace pipeline {

using ProgressCallback = std::function<void(int percentage)>;

/* 8-bit gray pixels in host memory: `height` rows of `width` bytes, rows
   `stride` bytes apart (0: width). An empty view (null data) stands for no
   image, e.g. no ROI mask. */
struct GrayView {
    const uint8_t* data = nullptr;
    int width = 0;
    int height = 0;
    size_t stride = 0;
    bool empty() const { return data == nullptr || width <= 0 || height <= 0; }
    size_t row_bytes() const { return stride ? stride : (size_t)width; }
};

#ifdef SEMPER_HAVE_OPENCV
/* A CV_8UC1 matrix as a view (an empty view for an empty matrix; a matrix of
   another type gives an empty view with width -1, which the calls reject). */
inline GrayView gray_view(const cv::Mat& m) {
    GrayView v;
    if (m.empty()) return v;
    if (m.type() != CV_8UC1) {
        v.width = -1;
        return v;
    }
    v.data = m.data;
    v.width = m.cols;
    v.height = m.rows;
    v.stride = m.step[0];
    return v;
}
#endif

/* The solve settings (pipeline.hpp:66-72). */
struct FullFieldParams {
    int rect_x = 0, rect_y = 0, rect_w = 0, rect_h = 0;
    int step = 0;
    int subset_size = 0;
    int strain_window = 0;
    bool use_6x6_interpolator = false;
};

/* The reference image and everything derived from it alone, kept between
   solves (pipeline.hpp:35-64): here the prepared planes, the grid scan and
   the Hessian pool live in GPU memory, reused by every solve on the same
   reference, ROI and settings. Non-copyable, non-movable. `mutex` is for the
   caller (the library does not lock it), as in the reference. */
struct SEMPER_CXX_API ReferenceCache {
    int width = 0;
    int height = 0;
    std::mutex mutex;

    ReferenceCache();
    ~ReferenceCache();
    ReferenceCache(const ReferenceCache&) = delete;
    ReferenceCache& operator=(const ReferenceCache&) = delete;
    ReferenceCache(ReferenceCache&&) = delete;
    ReferenceCache& operator=(ReferenceCache&&) = delete;

    /* Drop the reference. */
    void reset();
    /* Take `gray` as the reference; `roi_mask` (empty, or any size: resized
       to the reference by nearest neighbour) marks material >= 128. The old
       reference is dropped first; throws std::invalid_argument for an empty
       or malformed image and std::runtime_error when the GPU fails. */
    void set_from_gray(const GrayView& gray, const GrayView& roi_mask = GrayView());
#ifdef SEMPER_HAVE_OPENCV
    void set_from_gray(const cv::Mat& gray_in, const cv::Mat& roi_mask) {
        set_from_gray(gray_view(gray_in), gray_view(roi_mask));
    }
#endif

    struct Impl;
    std::unique_ptr<Impl> impl;
};

/* Run the full-field solve of `def_gray` against the cached reference
   (pipeline.hpp:74-96). Returns the points written to `output_ptr` (8 floats
   each: x, y, u, v, exx, eyy, exy, corr; never more than output_capacity
   floats), or -2 (ROI), -3 (no reference, an image of another size, a bad
   argument), kBadStrainWindow, kSeedFailed, kCancelled. `metrics` (may be
   null) receives the prefix of the 24 engine metrics that metrics_len allows.
   `roi_mask` may be empty or of any size (resized as for the reference).
   Cancelled by request_cancel() (the process-wide token). */
SEMPER_CXX_API int run_full_field(ReferenceCache& cache, const GrayView& def_gray, const GrayView& roi_mask,
                                  const FullFieldParams& params, float* output_ptr, int output_capacity,
                                  float* metrics, int metrics_len, ProgressCallback on_progress = nullptr);

/* The same, cancelled by the caller's own token only (pipeline.hpp:98-112). */
SEMPER_CXX_API int run_full_field(ReferenceCache& cache, const GrayView& def_gray, const GrayView& roi_mask,
                                  const FullFieldParams& params, float* output_ptr, int output_capacity,
                                  float* metrics, int metrics_len, CancelToken& cancel,
                                  ProgressCallback on_progress = nullptr);

#ifdef SEMPER_HAVE_OPENCV
inline int run_full_field(ReferenceCache& cache, const cv::Mat& def_gray, const cv::Mat& roi_mask,
                          const FullFieldParams& params, float* output_ptr, int output_capacity, float* metrics,
                          int metrics_len, ProgressCallback on_progress = nullptr) {
    return run_full_field(cache, gray_view(def_gray), gray_view(roi_mask), params, output_ptr, output_capacity,
                          metrics, metrics_len, std::move(on_progress));
}
inline int run_full_field(ReferenceCache& cache, const cv::Mat& def_gray, const cv::Mat& roi_mask,
                          const FullFieldParams& params, float* output_ptr, int output_capacity, float* metrics,
                          int metrics_len, CancelToken& cancel, ProgressCallback on_progress = nullptr) {
    return run_full_field(cache, gray_view(def_gray), gray_view(roi_mask), params, output_ptr, output_capacity,
                          metrics, metrics_len, cancel, std::move(on_progress));
}
#endif

}  // namespace pipeline
}  // namespace Semper

#endif
