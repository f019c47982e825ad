// Device bookkeeping of incremental DIC: warp_material_mask
// (src/pipeline/incremental_math.cpp:371-447) and stamp_ghost_wall
// (src/pipeline/reference_cache.cpp:18-35). The warp evaluates the same IEEE
// double expressions as the host restatement (no contraction: -fmad=false),
// so both give the same mask.
#include "incmask.cuh"

namespace dic {

namespace {

// The continuous field of the grid at (x, y): bilinear inside, the plane
// through the nearest grid point with that point's gradient outside.
__device__ __forceinline__ void field_eval(const MaskField& g, double x, double y, double& u, double& v) {
    const double gx_raw = (x - g.rect_x) / g.step, gy_raw = (y - g.rect_y) / g.step;
    const double gx = fmax(0.0, fmin(gx_raw, (double)(g.gridW - 1)));
    const double gy = fmax(0.0, fmin(gy_raw, (double)(g.gridH - 1)));
    const double ox = (gx_raw - gx) * g.step, oy = (gy_raw - gy) * g.step;
    int i0 = (int)floor(gx), j0 = (int)floor(gy);
    i0 = max(0, min(i0, max(g.gridW - 2, 0)));
    j0 = max(0, min(j0, max(g.gridH - 2, 0)));
    const int i1 = min(i0 + 1, g.gridW - 1), j1 = min(j0 + 1, g.gridH - 1);
    const double tx = (i1 == i0) ? 0.0 : gx - i0, ty = (j1 == j0) ? 0.0 : gy - j0;
    const size_t k00 = (size_t)j0 * g.gridW + i0, k10 = (size_t)j0 * g.gridW + i1;
    const size_t k01 = (size_t)j1 * g.gridW + i0, k11 = (size_t)j1 * g.gridW + i1;
    {
        const double a = g.U[k00], b = g.U[k10], c = g.U[k01], d = g.U[k11];
        u = a * (1 - tx) * (1 - ty) + b * tx * (1 - ty) + c * (1 - tx) * ty + d * tx * ty;
        const double dx = (i1 == i0) ? 0.0 : ((b - a) * (1 - ty) + (d - c) * ty) / g.step;
        const double dy = (j1 == j0) ? 0.0 : ((c - a) * (1 - tx) + (d - b) * tx) / g.step;
        u += dx * ox + dy * oy;
    }
    {
        const double a = g.V[k00], b = g.V[k10], c = g.V[k01], d = g.V[k11];
        v = a * (1 - tx) * (1 - ty) + b * tx * (1 - ty) + c * (1 - tx) * ty + d * tx * ty;
        const double dx = (i1 == i0) ? 0.0 : ((b - a) * (1 - ty) + (d - c) * ty) / g.step;
        const double dy = (j1 == j0) ? 0.0 : ((c - a) * (1 - tx) + (d - b) * tx) / g.step;
        v += dx * ox + dy * oy;
    }
}

// one thread per window pixel; every writer stores 255, so order does not matter
__global__ void warp_mask_kernel(const uint8_t* __restrict__ mask0, int W, int H, int X0, int X1, int Y0, int Y1,
                                 int per_px, MaskField f, uint8_t* out) {
    const int sx = X0 + blockIdx.x * blockDim.x + threadIdx.x, sy = Y0 + blockIdx.y;
    if (sx > X1 || sy > Y1) return;
    if (mask0[(size_t)sy * W + sx] < 128) return;
    const double hs = 1.0 / per_px;
    for (int b = 0; b < per_px; ++b)
        for (int a = 0; a < per_px; ++a) {
            const double X = sx - 0.5 + (a + 0.5) * hs, Y = sy - 0.5 + (b + 0.5) * hs;
            double u, v;
            field_eval(f, X, Y, u, v);
            const long long px = llround(X + u), py = llround(Y + v);
            if (px < 0 || px >= W || py < 0 || py >= H) continue;
            out[(size_t)py * W + px] = 255;
        }
}

template <bool DILATE>
__global__ void morph3x3_kernel(const uint8_t* __restrict__ in, uint8_t* __restrict__ out, int W, int H) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    uint8_t v = DILATE ? 0 : 255;
    for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
            const int xx = x + dx, yy = y + dy;
            if (xx < 0 || yy < 0 || xx >= W || yy >= H) continue;
            const uint8_t p = in[(size_t)yy * W + xx];
            if (DILATE && p) v = 255;
            if (!DILATE && !p) v = 0;
        }
    out[(size_t)y * W + x] = v;
}

__global__ void bbox_kernel(const uint8_t* __restrict__ m, int W, int H, int* box) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H || !m[(size_t)y * W + x]) return;
    atomicMin(box + 0, x);
    atomicMin(box + 1, y);
    atomicMax(box + 2, x);
    atomicMax(box + 3, y);
}

__global__ void box_init_kernel(int* box, int W, int H) {
    box[0] = W;
    box[1] = H;
    box[2] = -1;
    box[3] = -1;
}

__global__ void stamp_kernel(float* I, int W, int H, int pitch, const uint8_t* __restrict__ mask) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W || y >= H) return;
    if (mask[(size_t)y * W + x] < 128) I[(size_t)y * pitch + x] = -10.0f;
}

}  // namespace

cudaError_t launch_warp_mask(const uint8_t* mask0, int W, int H, int X0, int X1, int Y0, int Y1, int per_px,
                             MaskField f, uint8_t* out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, (size_t)W * H, st);
    if (e != cudaSuccess) return e;
    if (X0 > X1 || Y0 > Y1) return cudaSuccess;
    const int w = X1 - X0 + 1;
    warp_mask_kernel<<<dim3((w + 127) / 128, Y1 - Y0 + 1), 128, 0, st>>>(mask0, W, H, X0, X1, Y0, Y1, per_px, f, out);
    return cudaGetLastError();
}

cudaError_t launch_close3x3(uint8_t* m, uint8_t* tmp, int W, int H, cudaStream_t st) {
    const dim3 grid((W + 255) / 256, H);
    morph3x3_kernel<true><<<grid, 256, 0, st>>>(m, tmp, W, H);
    morph3x3_kernel<false><<<grid, 256, 0, st>>>(tmp, m, W, H);
    return cudaGetLastError();
}

cudaError_t launch_mask_bbox(const uint8_t* m, int W, int H, int* box, cudaStream_t st) {
    box_init_kernel<<<1, 1, 0, st>>>(box, W, H);
    bbox_kernel<<<dim3((W + 255) / 256, H), 256, 0, st>>>(m, W, H, box);
    return cudaGetLastError();
}

cudaError_t launch_stamp_ghost(float* I, int W, int H, int pitch, const uint8_t* mask, cudaStream_t st) {
    stamp_kernel<<<dim3((W + 255) / 256, H), 256, 0, st>>>(I, W, H, pitch, mask);
    return cudaGetLastError();
}

}  // namespace dic
