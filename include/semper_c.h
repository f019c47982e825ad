/*
 * semper_c.h — the C ABI of the DIC engine, as exported by libsemper_c.so of
 * this build (the B200 implementation). Drop-in for the reference's
 * include/semper/semper_c.h:83-197: the same eleven entry points, argument
 * meanings, struct layouts, return codes and threading rules, so a caller
 * compiled against the reference header links and runs against this library
 * unchanged. The layouts are frozen by the reference's contract
 * (docs/CONTRACT.md A.4, tests/c/contract.c:20-40) and must stay identical.
 *
 * Differences from the reference, all at the input-decoding edge:
 *   - images and masks are raw buffers: ALPHA_8 (w*h bytes) or RGBA
 *     (4*w*h bytes, converted to gray with BT.601 weights); encoded PNG/JPEG/
 *     TIFF bytes are not decoded and return SEMPER_ERR_INIT;
 *   - a mask must have the image's size (no nearest-neighbour resize).
 */
#ifndef SEMPER_C_H
#define SEMPER_C_H

#include <stddef.h>
#include <stdint.h>

#if defined(_WIN32) || defined(__CYGWIN__)
#  if defined(SEMPER_C_BUILD)
#    define SEMPER_C_API __declspec(dllexport)
#  else
#    define SEMPER_C_API __declspec(dllimport)
#  endif
#else
#  define SEMPER_C_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque engine handle (reference semper_c.h:44). Owns a device context, the
   reference cache on the GPU and a cancel flag. */
typedef struct semper_engine semper_engine;

/* Solve parameters, eight int32 at offsets 0..28 (reference semper_c.h:46-52). */
typedef struct semper_params {
    int32_t rect_x, rect_y, rect_w, rect_h; /* region of interest, pixels */
    int32_t step;                           /* grid spacing, pixels */
    int32_t subset_size;                    /* odd subset edge, pixels */
    int32_t strain_window;                  /* VSG window, pixels */
    int32_t use_6x6_interpolator;           /* 0: 4x4 Catmull-Rom, 1: 6x6 Keys */
} semper_params;

/* Return codes (reference semper_c.h:55-65). >= 0 is a point count. */
#define SEMPER_ERR_ROI           (-2)
#define SEMPER_ERR_INIT          (-3)
#define SEMPER_ERR_STRAIN_WINDOW (-4)
#define SEMPER_ERR_SEED          (-5)
#define SEMPER_ERR_CANCELLED     (-99)

typedef void (*semper_progress_cb)(int percentage, void* user);

#define SEMPER_FLOATS_PER_POINT 8  /* [x, y, u, v, exx, eyy, exy, corr] */
#define SEMPER_METRICS_LEN 24

/* reference semper_c.h:95-96 */
SEMPER_C_API semper_engine* semper_create(void);
SEMPER_C_API void           semper_destroy(semper_engine* eng);

/* Cache the reference image on the device (reference semper_c.h:98-113;
   adapters/c/semper_c.cpp:105-124). The previous reference is dropped first. */
SEMPER_C_API int semper_set_reference(semper_engine* eng,
                                      const uint8_t* img, size_t img_len,
                                      const uint8_t* mask, size_t mask_len,
                                      int expected_w, int expected_h);

/* One full-field solve of `def` against the cached reference
   (reference semper_c.h:115-133; adapters/c/semper_c.cpp:126-153). */
SEMPER_C_API int semper_run(semper_engine* eng,
                            const uint8_t* def, size_t def_len,
                            const uint8_t* mask, size_t mask_len,
                            const semper_params* params,
                            float* out, int out_capacity,
                            float* metrics, int metrics_len,
                            semper_progress_cb cb, void* user);

/* Thread-safe cancel of the run in flight (reference semper_c.h:136). */
SEMPER_C_API void semper_cancel(semper_engine* eng);

/* "MAJOR.MINOR.PATCH" of the engine contract implemented (reference semper_c.h:139). */
SEMPER_C_API const char* semper_version(void);

/* Incremental sessions (reference semper_c.h:141-197). */
typedef struct semper_incremental semper_incremental;

/* Six int32, 24 bytes (reference semper_c.h:155-162). */
typedef struct semper_incremental_info {
    int32_t reference_frame;
    int32_t reference_updated;
    int32_t tracked_points;
    int32_t frame0_points;
    int32_t taylor_fallbacks;
    int32_t lost_this_frame;
} semper_incremental_info;

SEMPER_C_API semper_incremental* semper_incremental_create(void);
SEMPER_C_API void                semper_incremental_destroy(semper_incremental* inc);

SEMPER_C_API int semper_incremental_init(semper_incremental* inc,
                                         const uint8_t* ref, size_t ref_len,
                                         const uint8_t* mask, size_t mask_len,
                                         int expected_w, int expected_h,
                                         const semper_params* params,
                                         int32_t update_interval);

SEMPER_C_API int semper_incremental_process(semper_incremental* inc,
                                            const uint8_t* def, size_t def_len,
                                            float* out, int out_capacity,
                                            float* metrics, int metrics_len,
                                            semper_incremental_info* info,
                                            semper_progress_cb cb, void* user);

SEMPER_C_API void semper_incremental_cancel(semper_incremental* inc);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* SEMPER_C_H */
