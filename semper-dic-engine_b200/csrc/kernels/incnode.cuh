// Per-node kernels of the incremental session (IncrementalSession,
// src/pipeline/incremental_session.cpp:289-549, over the per-node math of
// src/pipeline/incremental_math.cpp:19-447). The session's state lives on the
// device, one entry per frame-0 grid node; each frame runs a few launches
// over all nodes and hands the host only counts and short node lists.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

// A solved lattice on the device: the increment field of one solve
// (FieldCapture, src/pipeline/full_field_internal.hpp:247-261). A node holds a
// usable increment when it solved with a result (corr >= 0) and passed the
// packing's displacement median test (`ok`).
struct IncField {
    int gw, gh, rect_x, rect_y, step;
    const float *u, *v, *ux, *uy, *vx, *vy, *corr;
    const uint8_t* solved;
    const uint8_t* ok;
};

// The frame-0 grid the totals live on.
struct IncGrid {
    int gw, gh, rect_x, rect_y, step;
};

// Session state, one entry per frame-0 node.
struct IncState {
    float* ubase;             // total displacement at the current reference
    float* vbase;
    uint8_t* alive;           // the node is still followed
    float* travel;            // distance coasted since its last measurement
    const uint8_t* anchored;  // the node has a coasting anchor (host mirror)
};

// One frame's per-node results.
enum : uint8_t {
    kIncCarried = 1,   // the node has a total this frame
    kIncValid = 2,     // measured this frame (sampled, or matched)
    kIncTaylor = 4,    // its sample was the first-order expansion
    kIncMatch = 8,     // to be confirmed by an anchor match (host)
    kIncNeedShift = 4  // bits 4-5: the anchor need (0 drop, 1 refresh, 2 keep)
};
struct IncFrame {
    float* U;      // the new totals
    float* V;
    float* corr;   // ZNSSD of the measurement
    float* cstep;  // this frame's coasting step
    uint8_t* flags;
};

// Counters written by the launches (ints): [0] carried nodes, [1] valid nodes
// with a Taylor sample, [2] matches listed, [3] refresh listed, [4] drop
// listed, [5] alive after an update, [6..9] grid rect of alive nodes as
// ordered-int floats (min x, min y, max x, max y), [10..11] stretch as the
// bits of a double, [12] fill changed, [13] fill found a valid node.
constexpr int kIncCounters = 16;

// Anchor need of every node of an increment field (the nearest-node lookup of
// anchor_need, incremental_math.cpp:211-221, done by the caller): 0 drop,
// 1 refresh, 2 keep.
cudaError_t launch_inc_need(const IncField& f, int subset, uint8_t* need, cudaStream_t st);

// The first frame on frame 0's own grid: the totals are the solve's field.
cudaError_t launch_inc_first(const IncField& f, const uint8_t* need, const IncFrame& fr, cudaStream_t st);

// A frame against an updated reference: every alive node samples the
// increment at its current position (or coasts on a fitted plane), and is
// listed for an anchor match when it has coasted too far to be trusted (list
// slot t: match_list[t] the node, match_info[3t..3t+2] its sampled total U, V
// and its coast travel; counters[2] the count).
struct IncStepArgs {
    int width, height, subset;
    float max_travel, trusted_travel, coast_radius;
};
cudaError_t launch_inc_step(const IncGrid& g, const IncState& s, const IncField& f, const uint8_t* need,
                            const IncStepArgs& a, const IncFrame& fr, int* counters, int* match_list,
                            float* match_info, cudaStream_t st);

// An anchor match the host ran for a listed node: ok when it confirmed the
// node (then U, V, corr are its measurement).
struct IncMatch {
    int node;
    int ok;
    float U, V, corr;
};
cudaError_t launch_inc_apply_matches(int m, const IncMatch* rec, const IncFrame& fr, cudaStream_t st);

// Frame results into the packing's inputs, and the counts of carried nodes
// and Taylor samples (gu null: counts only).
cudaError_t launch_inc_finish(int n, const IncFrame& fr, float* gu, float* gv, float* gcorr, uint8_t* gsolved,
                              int* counters, cudaStream_t st);

// The update's bookkeeping: the coast travel carried on and the alive flags
// of the next reference (into travel_next, alive_next), anchors to drop and to
// refresh listed (refresh entries with the node's position on the new
// reference), the alive count and the grid rect of the alive nodes
// (counters[6..9] set to INT_MAX, INT_MAX, INT_MIN, INT_MIN first).
cudaError_t launch_inc_update(const IncGrid& g, const IncState& s, const IncFrame& fr, float* travel_next,
                              uint8_t* alive_next, int* counters, int* refresh_list, float* refresh_xy,
                              int* drop_list, cudaStream_t st);

// fill_field (incremental_math.cpp:281-322) as Jacobi passes over the totals:
// init copies U, V with invalid nodes zeroed; each pass fills the invalid
// nodes that have a filled 4-neighbour with their mean (reading the previous
// pass) and sets counters[12] when it filled any.
cudaError_t launch_inc_fill_init(int n, const float* U, const float* V, const uint8_t* valid, float* fu, float* fv,
                                 uint8_t* filled, int* counters, cudaStream_t st);
cudaError_t launch_inc_fill_pass(int gw, int gh, const float* fu, const float* fv, const uint8_t* filled, float* nu,
                                 float* nv, uint8_t* nfilled, int* counters, cudaStream_t st);
// The largest local stretch of the filled field, at least the value whose
// bits counters[10..11] hold as a double (set to 1.0 first).
cudaError_t launch_inc_stretch(int gw, int gh, int step, const float* fu, const float* fv, int* counters,
                               cudaStream_t st);

}  // namespace dic
