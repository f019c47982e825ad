/*
 * semper_b200_ext.h — extensions of this B200 build over the reference C ABI.
 * No counterpart in the reference; they exist for callers that keep frames on
 * the GPU, for measurement, and to feed the solve a global-motion model.
 * They take the same engine handle as semper_c.h and follow its threading
 * rules (one call at a time per handle; -3 when the handle is busy).
 */
#ifndef SEMPER_B200_EXT_H
#define SEMPER_B200_EXT_H

#include <stddef.h>
#include <stdint.h>

#include "semper_c.h"

#ifdef __cplusplus
extern "C" {
#endif

/* semper_run with the deformed frame already in device memory (d_def: w*h
   bytes, the reference's size) and the packed output left in device memory
   (d_out: out_capacity floats). Same return codes, metrics and cancel
   semantics as semper_run; no mask. */
SEMPER_C_API int semper_b200_run_device(semper_engine* eng, const uint8_t* d_def, const semper_params* params,
                                        float* d_out, int out_capacity, float* metrics, int metrics_len);

/* The CUDA stream (cudaStream_t) the engine's work runs on. */
SEMPER_C_API void* semper_b200_stream(semper_engine* eng);

/* Device timings of the last solve, ms, measured with CUDA events on the
   engine stream: [prep, pool, seeding, mesh, path A solve, path B, strain+pack,
   total]; counts: [IC-GN iterations, subset-pixel x iterations of every solve,
   Path A tasks, subset-pixel x iterations of the Path A launch, kernels
   launched]. Returns 0, or -3 for a NULL handle. */
SEMPER_C_API int semper_b200_last_timings(semper_engine* eng, float times[8], long long counts[5]);

/* The shape of the Path A fast pass the engine's autotuner kept for this
   subset size and interpolator (six != 0: 6x6 Keys): 0 reads the reference
   subset from the prepared planes, 1 stages it in shared memory, -1 while
   undecided (the first four large Path A launches alternate between them).
   Both shapes give the same results. Returns -3 for a NULL handle. */
SEMPER_C_API int semper_b200_fast_pass_shape(semper_engine* eng, int subset_size, int six);

/* Where the last semper_incremental_process call spent its time (host wall
   clock, ms): out[0] the whole call, [1] its full-field solves, [2] its
   anchor matches, [3] the material-mask warp, [4] the reference adoption,
   [5] the packing of the carried field; [6] anchor matches made, [7] solves
   run; then the device phases of its last solve as semper_b200_last_timings
   gives them ([8..15]). For measurement. Returns 0, or -3 for a NULL handle. */
SEMPER_C_API int semper_b200_incremental_profile(semper_incremental* inc, double out[16]);

/* The solve's bounded waits for its TMA tile copies: at most `polls` polls
   of the copy's mbarrier (0: the default, about 0.1 s) before a wait gives
   up. A warp whose wait ran out reads the deformed image from global memory
   instead, with identical arithmetic and results, and waits (bounded) for the
   late copy before it exits. A small limit exercises that path. Returns 0, or
   -3 for a NULL or busy handle. */
SEMPER_C_API int semper_b200_set_tma_wait_limit(semper_engine* eng, int polls);

/* 1 when a TMA wait of the last run on this handle ran out, else 0; -3 for a
   NULL handle. */
SEMPER_C_API int semper_b200_last_tma_timeout(semper_engine* eng);

/* A global-motion model for the following runs on this handle: a 3x3
   homography, reference -> deformed, row-major (the role of the reference's
   AKAZE front end, src/pipeline/full_field_anchors.cpp:204-279). NULL clears
   it. Returns 0, or -3 for a NULL handle. */
SEMPER_C_API int semper_b200_set_global_model(semper_engine* eng, const double* h9);

/* Switches the device global-motion estimate on (on != 0, the default) or
   off. With no model set by semper_b200_set_global_model, each run estimates
   a similarity (rotation, isotropic scale, translation) between the reference
   and the deformed ROI by phase correlation and, when both correlation peaks
   pass their gates, seeds the anchor lattice with it as the reference seeds
   from its AKAZE homography (src/pipeline/full_field_anchors.cpp:204-279).
   Returns 0, or -3 for a NULL or busy handle. */
SEMPER_C_API int semper_b200_set_global_motion(semper_engine* eng, int on);

/* The estimate of the last run: out[0] 1 when it was locked and used, else 0;
   out[1] rotation (rad); out[2] scale; out[3..4] translation (px); out[5..6]
   the centre of rotation (px); out[7..8] the rotation and translation
   correlation peaks; out[9..17] the homography, reference -> deformed,
   row-major. All zero but the identity homography when no estimate ran.
   Returns 0, or -3 for a NULL or busy handle. */
SEMPER_C_API int semper_b200_last_global_motion(semper_engine* eng, double out[18]);

/* Batched solves: many independent pairs, each with its own size, mask and
   settings, solved concurrently on the current device (or several GPUs,
   semper_b200_batch_create_on). No counterpart in the
   reference (its callers loop over semper_set_reference + semper_run); each
   job's result, metrics and return code are exactly those of that loop on a
   fresh handle. */
typedef struct semper_b200_job {
    const uint8_t* reference; /* width*height gray bytes */
    const uint8_t* deformed;  /* width*height gray bytes */
    const uint8_t* mask;      /* width*height bytes (>= 128: material), or NULL */
    int32_t width, height;
    semper_params params;
    float* out;               /* out_capacity floats: packed points, as semper_run */
    int32_t out_capacity;
    float* metrics;           /* metrics_len floats, or NULL */
    int32_t metrics_len;
    int32_t result;           /* written: semper_run's return value for this job */
} semper_b200_job;

typedef struct semper_b200_batch semper_b200_batch;

/* A batch runner with `workers` engines (<= 0: 8), each with its own stream
   and host thread, on the current device. NULL on failure. */
SEMPER_C_API semper_b200_batch* semper_b200_batch_create(int32_t workers);
/* The same with the engines spread over `n_devices` GPUs: engine i on
   devices[i % n_devices], so a batch's jobs spread over the GPUs as the
   workers take them (each job solved on one GPU, with the results a lone
   engine gives it). n_devices 0: the current device. NULL on failure. */
SEMPER_C_API semper_b200_batch* semper_b200_batch_create_on(int32_t workers, const int32_t* devices,
                                                             int32_t n_devices);
SEMPER_C_API void semper_b200_batch_destroy(semper_b200_batch* b);
/* Solves every job (largest first, spread over the workers) and returns 0
   when all have run (each job's own code is in its `result`), or -3 for a
   NULL or busy runner. Job buffers must stay valid until it returns. */
SEMPER_C_API int semper_b200_batch_run(semper_b200_batch* b, semper_b200_job* jobs, int32_t n_jobs);
/* The first internal failure (a CUDA error) of the last batch_run, "" when
   none; valid until the next call on the runner. */
SEMPER_C_API const char* semper_b200_batch_last_error(semper_b200_batch* b);

/* Batched incremental sequences (no counterpart in the reference; each
   sequence is solved exactly as its own semper_incremental handle would solve
   it, src/pipeline/incremental_session.cpp:120-549). The runner holds
   `sequences` sessions, each with its own engine and stream. One process
   call advances every listed sequence by one frame, the sequences
   concurrently (a host thread each), so their kernels and copies interleave
   on the device and one sequence's host steps overlap the others' solves. */
typedef struct semper_b200_inc_batch semper_b200_inc_batch;

typedef struct semper_b200_inc_frame {
    int32_t sequence;          /* which session, 0 <= sequence < sequences */
    const uint8_t* frame;      /* width*height bytes, raw 8-bit gray, the sequence's size */
    float* out;                /* out_capacity floats: packed points, as semper_incremental_process */
    int32_t out_capacity;
    float* metrics;            /* metrics_len floats, or NULL */
    int32_t metrics_len;
    semper_incremental_info info; /* written */
    int32_t result;            /* written: semper_incremental_process's return value for this frame */
} semper_b200_inc_frame;

/* NULL on failure or for sequences <= 0. */
SEMPER_C_API semper_b200_inc_batch* semper_b200_inc_batch_create(int32_t sequences);
/* The same with sequence q's session on devices[q % n_devices] (n_devices 0:
   the current device). */
SEMPER_C_API semper_b200_inc_batch* semper_b200_inc_batch_create_on(int32_t sequences, const int32_t* devices,
                                                                     int32_t n_devices);
SEMPER_C_API void semper_b200_inc_batch_destroy(semper_b200_inc_batch* b);
/* semper_incremental_init of one sequence on raw 8-bit frames of width x
   height (mask: the same size, or NULL). Same return codes. */
SEMPER_C_API int semper_b200_inc_batch_init(semper_b200_inc_batch* b, int32_t sequence, const uint8_t* reference,
                                            const uint8_t* mask, int32_t width, int32_t height,
                                            const semper_params* params, int32_t update_interval);
/* One frame for each entry; entries must name distinct sequences. Returns 0
   when every entry has run (each entry's own code is in its `result`), or -3
   for a NULL or busy runner, a sequence out of range or named twice. Frame
   and output buffers must stay valid until it returns. */
SEMPER_C_API int semper_b200_inc_batch_process(semper_b200_inc_batch* b, semper_b200_inc_frame* frames, int32_t n);

/* The learned seed proposal network (no counterpart in the reference): two
   64x64 patches in, the 6-parameter affine map between them out; BF16
   tensor-core kernels with FP32 accumulation for inference and training.
   Parameters are `semper_b200_proposal_param_count()` floats in the layout
   w0 b0 ... w4 b4 (convolutions [co][kh][kw][ci]) w5 b5 w6 b6 (dense
   [out][in]). Patches are [batch][64][64][2] floats (NHWC), outputs
   [batch][6]: A = I + [[o0, o1], [o2, o3]], t = 16 (o4, o5) in patch
   pixels. Every call returns 0, or -3 for a NULL handle or a bad argument. */
typedef struct semper_b200_proposal semper_b200_proposal;
SEMPER_C_API semper_b200_proposal* semper_b200_proposal_create(int32_t max_batch);
SEMPER_C_API void semper_b200_proposal_destroy(semper_b200_proposal* p);
SEMPER_C_API int64_t semper_b200_proposal_param_count(void);
SEMPER_C_API int semper_b200_proposal_set_params(semper_b200_proposal* p, const float* params, int64_t n);
SEMPER_C_API int semper_b200_proposal_get_params(semper_b200_proposal* p, float* params, int64_t n);
/* Forward over a batch of patch pairs (host memory). */
SEMPER_C_API int semper_b200_proposal_forward(semper_b200_proposal* p, const float* x, int32_t batch, float* out);
/* The loss of `target` [batch][6] (the mean squared displacement error of the
   affine map at a 3x3 grid of patch points, patch px^2) and the gradient of
   every parameter. */
SEMPER_C_API int semper_b200_proposal_gradients(semper_b200_proposal* p, const float* x, const float* target,
                                                int32_t batch, float* grads, float* loss);
/* Synthetic pairs from a w x h u8 speckle image: cfg = {max rotation (rad),
   max stretch, max shear, max shift (px), noise (gray levels), box factor}. */
SEMPER_C_API int semper_b200_proposal_synth(semper_b200_proposal* p, const uint8_t* speckle, int32_t w, int32_t h,
                                            const float cfg[6], uint64_t seed, int32_t batch, float* x,
                                            float* target);
/* `steps` Adam steps on batches of synthetic pairs; losses[steps] (may be
   NULL) receives each batch's loss. */
SEMPER_C_API int semper_b200_proposal_train(semper_b200_proposal* p, const uint8_t* speckle, int32_t w, int32_t h,
                                            const float cfg[6], int32_t steps, int32_t batch, float lr,
                                            uint64_t seed, float* losses);

/* Predictions for patch pairs cut from two w x h u8 frames (host memory,
   packed rows) at box factor f: pair k's first patch is the f x f box average
   of `ref` around (maps[8k], maps[8k+1]); its second samples `def`
   bilinearly at x' = A X + b for each sample X of the first, with
   A = [[maps[8k+2], maps[8k+3]], [maps[8k+4], maps[8k+5]]] and
   b = (maps[8k+6], maps[8k+7]); pixels outside the frame read its nearest
   edge. out [batch][6] is the residual map the network sees between them. */
SEMPER_C_API int semper_b200_proposal_predict_warped(semper_b200_proposal* p, const uint8_t* ref,
                                                     const uint8_t* def, int32_t w, int32_t h, const float* maps,
                                                     int32_t batch, int32_t f, float* out);

/* Learned seeding on an engine handle: with a proposal network (NULL: none),
   a run with no model set proposes its global model from the network's
   predictions on patch pairs of the reference and the deformed frame, and
   the anchor lattice keeps or rejects it by the reference's keep rule
   (full_field_anchors.cpp:204-279). learned 1: the proposal first, a rejected
   proposal falling back to the global-motion estimate; learned 2 (rescue):
   the global-motion estimate first, the proposal only when the estimate does
   not lock (and the plain lattice falls short of full quality) or the lattice
   rejects its model, and a rejected proposal leaving the run as the estimate
   seeded it; 0: off. The network must stay alive while the handle may use
   it, and serves one run at a time (handles that share a network must not
   run at once: its buffers are reused by every call). Returns 0, or -3 for
   a NULL or busy handle or another mode. */
SEMPER_C_API int semper_b200_set_proposal(semper_engine* eng, semper_b200_proposal* p, int learned);

/* The last run's learned seeding: out[0] 1 when it ran, [1] a model was
   proposed, [2] the lattice kept it; [3] patch pairs, [4] inlier pairs of the
   fit, [5] anchors that judged it, [6] their mean and [7] largest distance
   from the proposal (px), [8] device time of the network's stages (ms),
   [9..17] the proposed homography (row-major). Returns 0, or -3. */
SEMPER_C_API int semper_b200_last_learned(semper_engine* eng, double out[18]);

/* The last run's per-anchor guesses of the learned seeding: for every node of
   the anchor lattice (row-major), the displacement (u, v) the network put
   forward under the proposed model, NaN where none. Returns the node count n
   (the guesses are copied when capacity >= 2n floats), or -3. */
SEMPER_C_API int semper_b200_learned_guesses(semper_engine* eng, float* uv, int32_t capacity);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SEMPER_B200_EXT_H */
