// Plain-old-data records exchanged between the host pipeline and the DIC
// kernels. C layout, no CUDA or C++ types, so the same header serves the
// host C++ code, the .cu files and the C-ABI declarations.
#ifndef SEMPER_DIC_TYPES_H
#define SEMPER_DIC_TYPES_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Initialization modes, src/math/optimization_engine.cpp:55-118
   (include/semper/types.hpp:14-18). */
enum { DIC_INIT_AUTO_SEARCH = 0, DIC_INIT_NO_SEARCH = 1, DIC_INIT_NO_SIMPLEX = 2 };

/* One subset solve: pool row `node`, centre (cx, cy), 6-DOF guess
   [u v ux uy vx vy], mode. 40 bytes. */
typedef struct dic_task {
    int32_t node;
    int32_t cx, cy;
    int32_t mode;
    float g[6];
} dic_task;

/* The solve's outcome (AnalysisResult, include/semper/types.hpp:23-39) after
   the Ghost Wall rejection of solve_node. flags: bit 0 = the subset was
   initialised (fit the image, valid pool entry), bit 1 = a Simplex ran.
   48 bytes. */
typedef struct dic_result {
    float u, v, ux, uy, vx, vy, score;
    int32_t status, iters, trigger_iters, invalid_ref, flags;
} dic_result;

enum { DIC_RES_INITIALIZED = 1, DIC_RES_RESCUE = 2 };

#ifdef __cplusplus
}
#endif
#endif
