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

/* A global-motion model for the following runs on this handle: a 3x3
   homography, reference -> deformed, row-major (the role of the reference's
   AKAZE front end, src/pipeline/full_field_anchors.cpp:204-279). NULL clears
   it. Returns 0, or -3 for a NULL handle. */
SEMPER_C_API int semper_b200_set_global_model(semper_engine* eng, const double* h9);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SEMPER_B200_EXT_H */
