// The mesh guess field over the grid and Path A's task list.
//
//   in-triangle guesses, extrapolation, homography guesses, 5x5 smoothing
//       build_mesh_guess_field (src/pipeline/full_field_mesh.cpp:168-280)
//   Path A task list and commit
//       run_path_a (src/pipeline/full_field_path_a.cpp:40-113)
//
// One thread per grid node. Grid coordinates and triangle vertices are
// integers, so the inside/on-edge test is exact (int64 orientation); the
// affine guesses are evaluated in FP64 and rounded to float, as the reference.
#include <cuda_runtime.h>

#include "common.cuh"
#include "mesh.cuh"

namespace dic {

namespace {

__device__ __forceinline__ long long orient(long long ax, long long ay, long long bx, long long by, long long cx,
                                            long long cy) {
    return (bx - ax) * (cy - ay) - (by - ay) * (cx - ax);
}

__device__ __forceinline__ bool contains(const MeshTri& t, long long qx, long long qy) {
    const long long o0 = orient(t.X[0], t.Y[0], t.X[1], t.Y[1], qx, qy);
    const long long o1 = orient(t.X[1], t.Y[1], t.X[2], t.Y[2], qx, qy);
    const long long o2 = orient(t.X[2], t.Y[2], t.X[0], t.Y[0], qx, qy);
    const bool neg = o0 < 0 || o1 < 0 || o2 < 0, pos = o0 > 0 || o1 > 0 || o2 > 0;
    return !(neg && pos);
}

__device__ double signed_distance(const MeshTri& t, double px, double py) {
    double best = 1e300;
    for (int k = 0; k < 3; ++k) {
        const double ax = t.px[k], ay = t.py[k], bx = t.px[(k + 1) % 3], by = t.py[(k + 1) % 3];
        const double ex = bx - ax, ey = by - ay;
        const double qx = px - ax, qy = py - ay;
        const double len2 = ex * ex + ey * ey;
        double s = len2 > 0.0 ? (qx * ex + qy * ey) / len2 : 0.0;
        s = s < 0.0 ? 0.0 : (s > 1.0 ? 1.0 : s);
        const double dx = qx - s * ex, dy = qy - s * ey;
        const double d2 = dx * dx + dy * dy;
        best = best < d2 ? best : d2;
    }
    const double d = sqrt(best);
    return contains(t, llrint(px), llrint(py)) ? d : -d;
}

__device__ __forceinline__ void put_tri(const MeshTri& t, double px, double py, size_t idx, MeshGrid g) {
    g.gu[idx] = (float)(t.ux * px + t.uy * py + t.u);
    g.gv[idx] = (float)(t.vx * px + t.vy * py + t.v);
    g.gux[idx] = (float)t.ux;
    g.guy[idx] = (float)t.uy;
    g.gvx[idx] = (float)t.vx;
    g.gvy[idx] = (float)t.vy;
    g.in_mesh[idx] = 1;
}

__global__ void init_guess_kernel(int n, float gU, float gV, MeshGrid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    g.gu[idx] = gU;
    g.gv[idx] = gV;
    g.gux[idx] = g.guy[idx] = g.gvx[idx] = g.gvy[idx] = 0.0f;
    g.in_mesh[idx] = 0;
}

__global__ void assign_kernel(int gw, int gh, int rect_x, int rect_y, int step, const MeshTri* __restrict__ tris,
                              int ntri, const uint8_t* __restrict__ solved, uint8_t* __restrict__ tag, MeshGrid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || solved[idx]) return;
    const float px = (float)(rect_x + (idx % gw) * step), py = (float)(rect_y + (idx / gw) * step);
    for (int ti = 0; ti < ntri; ++ti) {
        const MeshTri& t = tris[ti];
        if (px < t.bx || px > t.bx + t.bw || py < t.by || py > t.by + t.bh) continue;
        if (contains(t, (long long)px, (long long)py)) {
            put_tri(t, px, py, idx, g);
            tag[idx] = 1;  // kMeshInTriangle
            return;
        }
    }
}

__global__ void extrap_kernel(int gw, int gh, int rect_x, int rect_y, int step, const MeshTri* __restrict__ tris,
                              int ntri, const uint8_t* __restrict__ solved, uint8_t* __restrict__ tag, MeshGrid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || solved[idx] || g.in_mesh[idx]) return;
    const float px = (float)(rect_x + (idx % gw) * step), py = (float)(rect_y + (idx / gw) * step);
    const float LIM = -3.0f * step;
    float best = LIM - 1.0f;
    int bi = -1;
    for (int ti = 0; ti < ntri; ++ti) {
        const MeshTri& t = tris[ti];
        if (px < t.bx + LIM || px > t.bx + t.bw - LIM || py < t.by + LIM || py > t.by + t.bh - LIM) continue;
        const double d = signed_distance(t, px, py);
        if (d >= LIM && (float)d > best) {
            best = (float)d;
            bi = ti;
        }
    }
    if (bi >= 0) {
        put_tri(tris[bi], px, py, idx, g);
        tag[idx] = 2;  // kMeshExtrapolated
    }
}

__global__ void homography_kernel(int gw, int gh, int rect_x, int rect_y, int step, Homog h,
                                  const uint8_t* __restrict__ solved, uint8_t* __restrict__ tag, MeshGrid g) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || solved[idx] || g.in_mesh[idx]) return;
    const double px = rect_x + (double)(idx % gw) * step, py = rect_y + (double)(idx / gw) * step;
    const double w = h.h[6] * px + h.h[7] * py + h.h[8];
    if (!finite_d(w) || fabs(w) < 1e-12) return;
    const double X = (h.h[0] * px + h.h[1] * py + h.h[2]) / w;
    const double Y = (h.h[3] * px + h.h[4] * py + h.h[5]) / w;
    const double J0 = (h.h[0] - X * h.h[6]) / w, J1 = (h.h[1] - X * h.h[7]) / w;
    const double J2 = (h.h[3] - Y * h.h[6]) / w, J3 = (h.h[4] - Y * h.h[7]) / w;
    if (!(finite_d(X) && finite_d(Y) && finite_d(J0) && finite_d(J1) && finite_d(J2) && finite_d(J3))) return;
    g.gu[idx] = (float)(X - px);
    g.gv[idx] = (float)(Y - py);
    g.gux[idx] = (float)(J0 - 1.0);
    g.guy[idx] = (float)J1;
    g.gvx[idx] = (float)J2;
    g.gvy[idx] = (float)(J3 - 1.0);
    g.in_mesh[idx] = 1;
    tag[idx] = 4;  // kMeshHomography
}

// 5x5 box average over in-mesh neighbours; with ax/ay, u/v are carried back
// from the box centroid along the node's smoothed gradient.
__global__ void smooth_kernel(int gw, int gh, float stepf, const float* __restrict__ src, float* __restrict__ dst,
                              const float* __restrict__ ax, const float* __restrict__ ay,
                              const uint8_t* __restrict__ in_mesh) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh) return;
    const float own = src[idx];
    if (!in_mesh[idx]) {
        dst[idx] = own;
        return;
    }
    const int x = idx % gw, y = idx / gw;
    float sum = 0.0f;
    int cnt = 0, sdx = 0, sdy = 0;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            const int ny = y + dy, nx = x + dx;
            if (nx >= 0 && nx < gw && ny >= 0 && ny < gh && in_mesh[ny * gw + nx]) {
                sum += src[ny * gw + nx];
                ++cnt;
                sdx += dx;
                sdy += dy;
            }
        }
    if (cnt == 0) {
        dst[idx] = own;
        return;
    }
    float r = sum / cnt;
    if (ax && (sdx != 0 || sdy != 0)) r -= (ax[idx] * sdx + ay[idx] * sdy) * stepf / cnt;
    dst[idx] = r;
}

// Path A's task list: every in-mesh node not yet solved; NO_SEARCH inside a
// triangle, NO_SIMPLEX for a guess from outside the mesh.
__global__ void path_a_tasks_kernel(int gw, int gh, int rect_x, int rect_y, int step,
                                    const uint8_t* __restrict__ solved, const uint8_t* __restrict__ tag, MeshGrid g,
                                    dic_task* __restrict__ tasks, int* __restrict__ n_tasks) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || !g.in_mesh[idx] || solved[idx]) return;
    const int slot = atomicAdd(n_tasks, 1);
    dic_task t;
    t.node = idx;
    t.cx = rect_x + (idx % gw) * step;
    t.cy = rect_y + (idx / gw) * step;
    t.mode = (tag[idx] == 2 || tag[idx] == 4) ? DIC_INIT_NO_SIMPLEX : DIC_INIT_NO_SEARCH;
    t.g[0] = g.gu[idx];
    t.g[1] = g.gv[idx];
    t.g[2] = g.gux[idx];
    t.g[3] = g.guy[idx];
    t.g[4] = g.gvx[idx];
    t.g[5] = g.gvy[idx];
    tasks[slot] = t;
}

// Writes solved tasks into the grid with the output gate (status 0, ZNSSD <=
// kCorrAccept) and accumulates the Path A telemetry.
__global__ void commit_kernel(const dic_task* __restrict__ tasks, const int* __restrict__ n_tasks,
                              const dic_result* __restrict__ res, FieldGrid f, PathStats* __restrict__ st) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    dic_result r{};
    bool live = t < *n_tasks;
    if (live) r = res[t];
    live = live && (r.flags & DIC_RES_INITIALIZED);
    const bool good = live && r.status == 0 && r.score <= 0.15f;
    const bool rescued = live && (r.flags & DIC_RES_RESCUE);
    if (live) {
        const int node = tasks[t].node;
        f.iters[node] = r.iters;
        if (good) {
            f.u[node] = r.u; f.v[node] = r.v; f.ux[node] = r.ux; f.uy[node] = r.uy;
            f.vx[node] = r.vx; f.vy[node] = r.vy; f.corr[node] = r.score;
            f.solved[node] = 1;
        } else {
            f.solved[node] = 0;
            f.corr[node] = -1.0f;
        }
    }
    // the counts, summed over the warp first: one atomic per counter and warp
    // instead of one per task on the same few addresses (integer sums, so the
    // totals do not depend on the order)
    const unsigned full = 0xffffffffu;
    const unsigned iters = __reduce_add_sync(full, live ? (unsigned)r.iters : 0u);
    const unsigned calls = __reduce_add_sync(full, rescued ? 1u : 0u);
    const unsigned saved = __reduce_add_sync(full, rescued && good ? 1u : 0u);
    const unsigned points = __reduce_add_sync(full, good ? 1u : 0u);
    if ((threadIdx.x & 31) == 0) {
        if (iters) atomicAdd(&st->icgn_iters, (unsigned long long)iters);
        if (calls) {
            atomicAdd(&st->simp_calls, (int)calls);
            if (saved) atomicAdd(&st->simp_saved, (int)saved);
            if (calls - saved) atomicAdd(&st->simp_dead, (int)(calls - saved));
        }
        if (points) atomicAdd(&st->points, (int)points);
    }
}

// Path B's boundary seeds: solved nodes with a valid score and an unsolved
// 4-neighbour (full_field_path_b.cpp:172-184), compacted in any order (the
// reliability queue orders them).
__global__ void boundary_kernel(int gw, int gh, FieldGrid f, BoundarySeed* __restrict__ out, int* __restrict__ n_out) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || !f.solved[idx] || f.corr[idx] < 0.0f) return;
    const int x = idx % gw, y = idx / gw;
    const bool touch = (x + 1 < gw && !f.solved[idx + 1]) || (x > 0 && !f.solved[idx - 1]) ||
                       (y + 1 < gh && !f.solved[idx + gw]) || (y > 0 && !f.solved[idx - gw]);
    if (!touch) return;
    const int slot = atomicAdd(n_out, 1);
    BoundarySeed b;
    b.node = idx;
    b.v[0] = f.u[idx]; b.v[1] = f.v[idx]; b.v[2] = f.ux[idx]; b.v[3] = f.uy[idx];
    b.v[4] = f.vx[idx]; b.v[5] = f.vy[idx]; b.v[6] = f.corr[idx];
    out[slot] = b;
}

// Writes host-side decisions (anchors, Path B commits) into the grid.
__global__ void scatter_kernel(int n, const ScatterRec* __restrict__ recs, FieldGrid f) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const ScatterRec r = recs[k];
    f.solved[r.node] = (uint8_t)r.solved;
    f.corr[r.node] = r.v[6];
    if (r.write_values) {
        f.u[r.node] = r.v[0]; f.v[r.node] = r.v[1]; f.ux[r.node] = r.v[2]; f.uy[r.node] = r.v[3];
        f.vx[r.node] = r.v[4]; f.vy[r.node] = r.v[5];
    }
}

// The packing input: solved nodes with a valid score.
__global__ void valid_kernel(int n, FieldGrid f, uint8_t* __restrict__ valid) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) valid[idx] = (f.solved[idx] && f.corr[idx] >= 0.0f) ? 1 : 0;
}

__global__ void fill_kernel(float* __restrict__ p, int n, float v) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) p[idx] = v;
}

}  // namespace

cudaError_t launch_fill(float* p, int n, float v, cudaStream_t st) {
    fill_kernel<<<(n + 255) / 256, 256, 0, st>>>(p, n, v);
    return cudaGetLastError();
}

cudaError_t launch_init_guess(int n, float gU, float gV, MeshGrid g, cudaStream_t st) {
    init_guess_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, gU, gV, g);
    return cudaGetLastError();
}

cudaError_t launch_mesh_assign(int gw, int gh, int rect_x, int rect_y, int step, const MeshTri* tris, int ntri,
                               int full, const Homog* h, const uint8_t* solved, uint8_t* tag, MeshGrid g,
                               cudaStream_t st) {
    const int n = gw * gh;
    if (ntri > 0) assign_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, rect_x, rect_y, step, tris, ntri, solved, tag, g);
    if (ntri > 0 && full)
        extrap_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, rect_x, rect_y, step, tris, ntri, solved, tag, g);
    if (h) homography_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, rect_x, rect_y, step, *h, solved, tag, g);
    return cudaGetLastError();
}

cudaError_t launch_smooth(int gw, int gh, int step, MeshGrid g, float* tmp, cudaStream_t st) {
    const int n = gw * gh;
    const float stepf = (float)step;
    float* fields[6] = {g.gux, g.guy, g.gvx, g.gvy, g.gu, g.gv};
    for (int k = 0; k < 6; ++k) {
        cudaError_t e = cudaMemcpyAsync(tmp, fields[k], sizeof(float) * n, cudaMemcpyDeviceToDevice, st);
        if (e != cudaSuccess) return e;
        const float* ax = k == 4 ? g.gux : (k == 5 ? g.gvx : nullptr);
        const float* ay = k == 4 ? g.guy : (k == 5 ? g.gvy : nullptr);
        smooth_kernel<<<(n + 255) / 256, 256, 0, st>>>(gw, gh, stepf, tmp, fields[k], ax, ay, g.in_mesh);
    }
    return cudaGetLastError();
}

cudaError_t launch_path_a_tasks(int gw, int gh, int rect_x, int rect_y, int step, const uint8_t* solved,
                                const uint8_t* tag, MeshGrid g, dic_task* tasks, int* n_tasks, cudaStream_t st) {
    const int n = gw * gh;
    path_a_tasks_kernel<<<(n + 255) / 256, 256, 0, st>>>(gw, gh, rect_x, rect_y, step, solved, tag, g, tasks, n_tasks);
    return cudaGetLastError();
}

cudaError_t launch_commit(const dic_task* tasks, const int* n_tasks, int max_tasks, const dic_result* res,
                          FieldGrid f, PathStats* stats, cudaStream_t st) {
    commit_kernel<<<(max_tasks + 255) / 256, 256, 0, st>>>(tasks, n_tasks, res, f, stats);
    return cudaGetLastError();
}

cudaError_t launch_boundary(int gw, int gh, FieldGrid f, BoundarySeed* out, int* n_out, cudaStream_t st) {
    const int n = gw * gh;
    boundary_kernel<<<(n + 255) / 256, 256, 0, st>>>(gw, gh, f, out, n_out);
    return cudaGetLastError();
}

cudaError_t launch_scatter(int n, const ScatterRec* recs, FieldGrid f, cudaStream_t st) {
    if (n > 0) scatter_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, recs, f);
    return cudaGetLastError();
}

cudaError_t launch_valid(int n, FieldGrid f, uint8_t* valid, cudaStream_t st) {
    valid_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, f, valid);
    return cudaGetLastError();
}

}  // namespace dic
