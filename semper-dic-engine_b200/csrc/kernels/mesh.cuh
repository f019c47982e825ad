// Launch interface and records of the mesh-guess and Path A kernels (mesh.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "dic_types.h"

namespace dic {

// One Delaunay triangle of the anchor mesh with its affine map
// (u = ux x + uy y + u, v = vx x + vy y + v, absolute coordinates) and the
// bounding box of the reference (vertex box grown by 15 px on every side).
struct MeshTri {
    double px[3], py[3];
    long long X[3], Y[3];
    double u, v, ux, uy, vx, vy;
    float bx, by, bw, bh;
};

struct Homog {
    double h[9];
};

// Per-node 6-DOF guesses and the in-mesh flag (MeshGuessField).
struct MeshGrid {
    float *gu, *gv, *gux, *guy, *gvx, *gvy;
    uint8_t* in_mesh;
};

// Per-node solve state (GridPoint, without the debug-only fields).
struct FieldGrid {
    float *u, *v, *ux, *uy, *vx, *vy, *corr;
    uint8_t* solved;
    int* iters;
};

struct PathStats {
    unsigned long long icgn_iters;
    int points, simp_calls, simp_saved, simp_dead;
};

struct BoundarySeed {
    int node;
    float v[7];  // u v ux uy vx vy corr
};

struct ScatterRec {
    int node;
    int solved;
    int write_values;
    float v[7];  // u v ux uy vx vy corr
};

cudaError_t launch_boundary(int gw, int gh, FieldGrid f, BoundarySeed* out, int* n_out, cudaStream_t st);
cudaError_t launch_scatter(int n, const ScatterRec* recs, FieldGrid f, cudaStream_t st);
cudaError_t launch_valid(int n, FieldGrid f, uint8_t* valid, cudaStream_t st);
cudaError_t launch_fill(float* p, int n, float v, cudaStream_t st);
cudaError_t launch_init_guess(int n, float gU, float gV, MeshGrid g, cudaStream_t st);
cudaError_t launch_mesh_assign(int gw, int gh, int rect_x, int rect_y, int step, const MeshTri* tris, int ntri,
                               int full, const Homog* h, const uint8_t* solved, uint8_t* tag, MeshGrid g,
                               cudaStream_t st);
cudaError_t launch_smooth(int gw, int gh, int step, MeshGrid g, float* tmp, cudaStream_t st);
cudaError_t launch_path_a_tasks(int gw, int gh, int rect_x, int rect_y, int step, const uint8_t* solved,
                                const uint8_t* tag, MeshGrid g, dic_task* tasks, int* n_tasks, cudaStream_t st);
cudaError_t launch_commit(const dic_task* tasks, const int* n_tasks, int max_tasks, const dic_result* res,
                          FieldGrid f, PathStats* stats, cudaStream_t st);

}  // namespace dic
