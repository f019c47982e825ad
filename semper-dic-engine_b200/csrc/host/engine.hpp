// Host side of the B200 full-field solve: the reference cache held on the
// device and run_full_field over it.
//
// Mirrors Semper::pipeline::ReferenceCache (include/semper/pipeline.hpp:35-64)
// and run_full_field / run_full_field_impl (src/pipeline/full_field_solver.cpp:
// 44-59, 141-586) with a raw 8-bit gray view in place of cv::Mat. Every
// data-parallel stage runs as a kernel; the orchestration between them (the
// lattice median test, routing, Delaunay mesh, Path B's deterministic rounds,
// metrics) runs here, on exactly the reference's rules.
#pragma once
#include <atomic>
#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../kernels/dic_types.h"
#include "../kernels/globalmotion.cuh"

namespace semper_b200 {

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

void check(cudaError_t e, const char* what);

// A growable device allocation.
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    // Room for count elements. A buffer that must grow gets half as much again
    // as it had (or count, when more): sizes that creep up frame by frame
    // (an incremental session's grid follows the material) then reallocate a
    // few times, not every frame; cudaFree waits for the whole device.
    void ensure(size_t count) {
        if (count <= n && p) return;
        size_t want = count == 0 ? 1 : count;
        if (p && n + n / 2 > want) want = n + n / 2;
        release();
        check(cudaMalloc(&p, want * sizeof(T)), "cudaMalloc");
        n = want;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

struct Params {
    int rect_x = 0, rect_y = 0, rect_w = 0, rect_h = 0, step = 0, subset_size = 0, strain_window = 0;
    bool six = false;
};

using Progress = std::function<void(int)>;

// The per-node state a caller can take after the solve (FieldCapture,
// src/pipeline/full_field_internal.hpp:247-261).
struct Capture {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0, attempted = 0;
    std::vector<float> u, v, ux, uy, vx, vy, corr;
    std::vector<uint8_t> solved;
    // the nodes holding a result (solved, corr >= 0) that pass the
    // displacement median test of the packing, and how many it rejected
    std::vector<uint8_t> median_valid;
    int median_rejected = 0;
};

// The per-node state of the last solve, left in device memory (the same
// nodes as Capture): valid until the next call on the engine that solves or
// packs. `ok` holds the packing's displacement median flags.
struct DeviceField {
    int gridW = 0, gridH = 0, rect_x = 0, rect_y = 0, step = 0, attempted = 0;
    const float *u = nullptr, *v = nullptr, *ux = nullptr, *uy = nullptr, *vx = nullptr, *vy = nullptr,
                *corr = nullptr;
    const uint8_t* solved = nullptr;
    const uint8_t* ok = nullptr;
};

// Timings of one solve's device phases, measured with CUDA events on the
// engine's stream (ms).
struct PhaseTimes {
    float prep = 0, pool = 0, seed = 0, mesh = 0, path_a = 0, path_b = 0, strain = 0, total = 0;
    long long icgn_iters = 0;   // IC-GN iterations of every subset solve
    long long pixel_iters = 0;  // subset pixels x iterations (the IC-GN work)
    int path_a_tasks = 0;
    long long path_a_pixel_iters = 0;  // the same for the Path A launch alone
    int launches = 0;                  // kernels this library launched during the solve
};

// validate_params (full_field_solver.cpp:97-111): clips the rect; 0 or a
// negative code.
int check_params(Params& p, int width, int height);
// StrainCalculator::vsg_window_node_count (strain_calculator.cpp:12-25).
int vsg_window_nodes(int step, int window);

class ProposalNet;

// What the learned seeding did in the last run: whether it ran, the model it
// proposed (reference -> deformed homography, fitted to the network's patch
// predictions), whether the anchor lattice kept that model (else the
// global-motion estimate took over), and the proposal's error against the
// lattice's own IC-GN solutions (px, over the anchors solved under it).
struct LearnedSeed {
    bool ran = false, proposed = false, kept = false;
    double H[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    int pairs = 0, inliers = 0, anchors = 0;
    float err_mean = 0.0f, err_max = 0.0f;
    float ms = 0.0f;  // device time of the network's stages
    // the network's displacement guess per anchor-lattice node (row-major,
    // 2 floats each, NaN where none) under the proposed model
    std::vector<float> anchor_uv;
};

// The raw result of one patch-subset solve (match_anchor's solve).
struct PatchSolve {
    bool initialized = false;
    int status = 0;
    float score = 0, u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0;
};

class Engine {
public:
    Engine();
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // ReferenceCache::set_from_gray: w x h gray bytes (host), optional mask of
    // the same size (host). The previous reference is dropped first.
    int set_reference(const uint8_t* gray, int w, int h, const uint8_t* mask);
    // The deformed frame of the last solve becomes the reference
    // (ReferenceCache::adopt, src/pipeline/reference_cache.cpp:82-108): its
    // prepared planes are taken over on the device. mask_on_device: the mask
    // is the one the last warp_mask call left on the device (not uploaded
    // again).
    int adopt_last_deformed(const uint8_t* mask, bool mask_on_device = false);
    void reset();
    bool has_reference() const { return has_ref_; }
    int width() const { return W_; }
    int height() const { return H_; }

    // run_full_field over a host deformed image (w x h bytes): host in, host out.
    int run(const uint8_t* def_gray, const uint8_t* mask, Params p, float* out, int capacity, float* metrics,
            int metrics_len, const double* model_H = nullptr, Progress progress = nullptr,
            Capture* capture = nullptr);

    // The same with the deformed image already on the device and the packed
    // output left on the device (d_out, capacity floats).
    int run_device(const uint8_t* d_def, const uint8_t* mask, Params p, float* d_out, int capacity,
                   float* metrics, int metrics_len, const double* model_H = nullptr, Progress progress = nullptr,
                   Capture* capture = nullptr);

    // The field of the last run, in device memory.
    DeviceField last_field() const;

    // pack_full_field_output over a grid (gW x gH nodes at rect + i * step;
    // u, v, corr, solved in host or device memory): the displacement median
    // test, VSG strain and packing on the device, out (host) receiving the
    // points. Returns the points written.
    int pack_field(int gW, int gH, int rect_x, int rect_y, int step, int window, const float* u, const float* v,
                   const float* corr, const uint8_t* solved, float* out, int capacity);

    // match_anchor's solve (incremental_math.cpp:238-276): the subset (side
    // `subset`) at the centre of a size x size gray patch, whose centre pixel
    // sits at (ax, ay), solved in NO_SEARCH mode on the deformed frame of the
    // last run from the guess (gu, gv) of its displacement.
    PatchSolve solve_patch(const uint8_t* patch, int size, int ax, int ay, float gu, float gv, int subset, bool six);

    // warp_material_mask's scatter and close (incremental_math.cpp:371-447)
    // on the device (U, V in host or device memory): every material pixel (mask0 >= 128) of the window
    // [X0, X1] x [Y0, Y1] sends per_px x per_px samples X to X + U(X), U the
    // filled field of the grid; then a 3x3 close. out (host, W x H) receives
    // the mask; box = {x, y, w, h} of its nonzero pixels (all 0 if none).
    // mask0_resident: mask0 is the one the last call uploaded, unchanged.
    int warp_mask(const uint8_t* mask0, int W, int H, int gridW, int gridH, int rect_x, int rect_y, int step,
                  const float* U, const float* V, int X0, int X1, int Y0, int Y1, int per_px, uint8_t* out,
                  int box[4], bool mask0_resident = false);

    void request_cancel() { h_cancel_[0] = 1; }
    void clear_cancel() { h_cancel_[0] = 0; }
    bool cancel_requested() const { return h_cancel_[0] != 0; }

    // Global motion (the stand-in for the AKAZE + RANSAC model,
    // full_field_anchors.cpp:204-279): with no model passed to run, the
    // similarity between the reference and the deformed ROI is estimated on
    // the device and, when both of its correlation peaks pass, seeds the
    // anchor lattice as the reference's global model does. On by default.
    void set_global_motion(bool on) { global_motion_ = on; }
    bool global_motion() const { return global_motion_; }
    // The estimate of the last run (locked false: none, or none used).
    const dic::GlobalSimilarity& last_global() const { return last_global_; }

    // Learned seeding: with a proposal network set (not owned), a run with no
    // model given proposes its global model from the network's predictions on
    // patch pairs of the reference and the deformed frame, and the anchor
    // lattice judges it by the reference's keep rule. `mode` 1: the proposal
    // first, and if the lattice rejects it, the global-motion estimate; mode
    // 2: the global-motion estimate first, and the proposal only when the
    // estimate does not lock or the lattice rejects its model (if the lattice
    // rejects the proposal too, the run seeds as from the estimate alone);
    // 0: off.
    void set_proposal(ProposalNet* net, int mode) {
        proposal_ = net;
        learned_ = mode != 0 && net != nullptr;
        learned_rescue_ = learned_ && mode == 2;
    }
    const LearnedSeed& last_learned() const { return last_learned_; }

    cudaStream_t stream() const { return stream_; }
    const PhaseTimes& last_times() const { return times_; }
    // The fast pass's shape the autotuner kept for (subset size, interpolator):
    // 0 the reference read from the planes, 1 staged in shared memory, -1 not
    // decided yet.
    int fast_pass_shape(int subset_size, bool six) const;
    // Grid blocks of the persistent solve kernel (0: automatic).
    void set_solve_blocks(int b) { solve_blocks_ = b; }
    // Polls of the solve's bounded TMA completion waits (0: the default,
    // about 0.1 s). A wait that runs out makes that warp read global memory,
    // with the same results; a small limit makes that path run.
    void set_tma_wait_limit(int polls) { tma_polls_ = polls > 0 ? polls : 0; }
    // Whether a TMA wait of the last run ran out (1) or not (0).
    int last_tma_timeout() const { return last_tma_timeout_; }

    struct Impl;

private:
    std::unique_ptr<Impl> impl_;
    cudaStream_t stream_ = nullptr;
    volatile int* h_cancel_ = nullptr;  // host-mapped pinned flag
    int* d_cancel_ = nullptr;
    bool has_ref_ = false;
    int W_ = 0, H_ = 0;
    int solve_blocks_ = 0;
    int tma_polls_ = 0;
    int last_tma_timeout_ = 0;
    bool global_motion_ = true;
    dic::GlobalSimilarity last_global_;
    ProposalNet* proposal_ = nullptr;
    bool learned_ = false;
    bool learned_rescue_ = false;  // the proposal only where the global-motion estimate fails
    LearnedSeed last_learned_;
    PhaseTimes times_;
    friend struct Impl;
};

}  // namespace semper_b200
