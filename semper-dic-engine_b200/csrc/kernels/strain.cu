// Displacement median test, VSG strain and output packing over the grid.
//
//   median test   StrainCalculator::reject_displacement_outliers
//                 (src/strain/strain_calculator.cpp:174-224; src/util/median.hpp:21-30)
//   VSG           StrainCalculator::compute_vsg_strain (strain_calculator.cpp:27-158), FP64
//   packing       pack_full_field_output (src/pipeline/full_field_solver_stats.cpp:21-91)
//
// One thread per grid node; the grid arrays are SoA (u, v, flags, strains).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include "common.cuh"
#include "strain.cuh"

namespace dic {

namespace {

// Median of a[0..n) (n <= 24), sorting in place: mean of the middle pair for
// an even count.
__device__ __forceinline__ float median_sort(float* a, int n) {
    for (int i = 1; i < n; ++i) {
        const float v = a[i];
        int j = i - 1;
        while (j >= 0 && a[j] > v) {
            a[j + 1] = a[j];
            --j;
        }
        a[j + 1] = v;
    }
    const int mid = n / 2;
    if (n & 1) return a[mid];
    return 0.5f * (a[mid - 1] + a[mid]);
}

__device__ __forceinline__ float norm_residual(float c, float* nb, int n) {
    float s[24];
    const float med = median_sort(nb, n);
    for (int i = 0; i < n; ++i) s[i] = fabsf(nb[i] - med);
    const float spread = median_sort(s, n);
    return fabsf(c - med) / (spread + 0.1f);
}

// One pass of the normalized median test: reads the flags of finished passes
// (ok), writes this pass's failures.
__global__ void median_kernel(int gw, int gh, const float* __restrict__ u, const float* __restrict__ v,
                              const uint8_t* __restrict__ ok, uint8_t* __restrict__ fail, int* __restrict__ n_fail) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh) return;
    fail[idx] = 0;
    if (!ok[idx]) return;
    const int x = idx % gw, y = idx / gw;
    float nu[24], nv[24];
    int n = 0;
    for (int dy = -2; dy <= 2; ++dy) {
        const int ny = y + dy;
        if (ny < 0 || ny >= gh) continue;
        for (int dx = -2; dx <= 2; ++dx) {
            const int nx = x + dx;
            if (nx < 0 || nx >= gw || (dx == 0 && dy == 0)) continue;
            const int ni = ny * gw + nx;
            if (!ok[ni]) continue;
            nu[n] = u[ni];
            nv[n] = v[ni];
            ++n;
        }
    }
    if (n < 3) return;
    if (norm_residual(u[idx], nu, n) > 3.0f || norm_residual(v[idx], nv, n) > 3.0f) {
        fail[idx] = 1;
        atomicAdd(n_fail, 1);
    }
}

__global__ void clear_failed_kernel(int n, uint8_t* __restrict__ ok, const uint8_t* __restrict__ fail) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n && fail[idx]) ok[idx] = 0;
}

// The VSG plane fit per valid node; FP64 normal equations, every product and
// sum separately rounded (this file is compiled with -fmad=false).
__global__ void vsg_kernel(int gw, int gh, int step, int grid_rad, double r2, int expected,
                           const float* __restrict__ u, const float* __restrict__ v,
                           const uint8_t* __restrict__ valid, float* __restrict__ exx, float* __restrict__ eyy,
                           float* __restrict__ exy) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh) return;
    exx[idx] = eyy[idx] = exy[idx] = -1000.0f;
    if (!valid[idx]) return;
    const int x = idx % gw, y = idx / gw;
    double A00 = 0, A01 = 0, A02 = 0, A10 = 0, A11 = 0, A12 = 0, A20 = 0, A21 = 0, A22 = 0;
    double bu0 = 0, bu1 = 0, bu2 = 0, bv0 = 0, bv1 = 0, bv2 = 0;
    int cnt = 0;
    for (int dy = -grid_rad; dy <= grid_rad; ++dy) {
        for (int dx = -grid_rad; dx <= grid_rad; ++dx) {
            const int nx = x + dx, ny = y + dy;
            if (nx < 0 || nx >= gw || ny < 0 || ny >= gh) continue;
            const int ni = ny * gw + nx;
            if (!valid[ni]) continue;
            const double px = (double)(dx * step), py = (double)(dy * step);
            if (px * px + py * py <= r2) {
                const double du = (double)u[ni], dv = (double)v[ni];
                A00 = A00 + 1.0 * 1.0; A01 = A01 + 1.0 * px; A02 = A02 + 1.0 * py;
                A10 = A10 + px * 1.0;  A11 = A11 + px * px;  A12 = A12 + px * py;
                A20 = A20 + py * 1.0;  A21 = A21 + py * px;  A22 = A22 + py * py;
                bu0 = bu0 + 1.0 * du; bu1 = bu1 + px * du; bu2 = bu2 + py * du;
                bv0 = bv0 + 1.0 * dv; bv1 = bv1 + px * dv; bv2 = bv2 + py * dv;
                ++cnt;
            }
        }
    }
    const double fill = (double)cnt / (double)expected;
    if (!(fill >= 0.90 && cnt >= 3)) return;
    double anorm = 0.0;
    {
        const double c0 = fabs(A00) + fabs(A10) + fabs(A20);
        const double c1 = fabs(A01) + fabs(A11) + fabs(A21);
        const double c2 = fabs(A02) + fabs(A12) + fabs(A22);
        if (c0 > anorm) anorm = c0;
        if (c1 > anorm) anorm = c1;
        if (c2 > anorm) anorm = c2;
    }
    const double C00 = A11 * A22 - A12 * A21;
    const double C10 = A02 * A21 - A01 * A22;
    const double C20 = A01 * A12 - A02 * A11;
    const double C01 = A12 * A20 - A10 * A22;
    const double C11 = A00 * A22 - A02 * A20;
    const double C21 = A02 * A10 - A00 * A12;
    const double C02 = A10 * A21 - A11 * A20;
    const double C12 = A01 * A20 - A00 * A21;
    const double C22 = A00 * A11 - A01 * A10;
    const double det = A00 * C00 + A10 * C10 + A20 * C20;
    if (!(fabs(det) > 1e-12)) return;
    const double id = 1.0 / det;
    const double I00 = C00 * id, I01 = C01 * id, I02 = C02 * id;
    const double I10 = C10 * id, I11 = C11 * id, I12 = C12 * id;
    const double I20 = C20 * id, I21 = C21 * id, I22 = C22 * id;
    double inorm = 0.0;
    {
        const double c0 = fabs(I00) + fabs(I10) + fabs(I20);
        const double c1 = fabs(I01) + fabs(I11) + fabs(I21);
        const double c2 = fabs(I02) + fabs(I12) + fabs(I22);
        if (c0 > inorm) inorm = c0;
        if (c1 > inorm) inorm = c1;
        if (c2 > inorm) inorm = c2;
    }
    const double rcond = (anorm * inorm > 0.0) ? (1.0 / (anorm * inorm)) : 0.0;
    if (rcond < 1e-12) return;
    const double dudx = (I10 * bu0 + I11 * bu1) + I12 * bu2;
    const double dudy = (I20 * bu0 + I21 * bu1) + I22 * bu2;
    const double dvdx = (I10 * bv0 + I11 * bv1) + I12 * bv2;
    const double dvdy = (I20 * bv0 + I21 * bv1) + I22 * bv2;
    exx[idx] = (float)(0.5 * ((2.0 * dudx + dudx * dudx) + dvdx * dvdx));
    eyy[idx] = (float)(0.5 * ((2.0 * dvdy + dudy * dudy) + dvdy * dvdy));
    exy[idx] = (float)(0.5 * (((dudy + dvdx) + dudx * dudy) + dvdx * dvdy));
}

__global__ void emit_kernel(int n, const uint8_t* __restrict__ valid, const float* __restrict__ exx,
                            int* __restrict__ emit) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n) emit[idx] = (valid[idx] && !(exx[idx] <= -999.0f)) ? 1 : 0;
}

// Row-major packing of [x y u v exx eyy exy corr] for the first max_pts
// emitting nodes; counts the strain drops before the capacity cut.
__global__ void pack_kernel(int gw, int gh, int rect_x, int rect_y, int step, int max_pts,
                            const uint8_t* __restrict__ valid, const int* __restrict__ pos,
                            const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ corr,
                            const float* __restrict__ exx, const float* __restrict__ eyy,
                            const float* __restrict__ exy, float* __restrict__ out, int* __restrict__ n_drop) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= gw * gh || !valid[idx]) return;
    const int p = pos[idx];
    if (exx[idx] <= -999.0f) {
        if (p < max_pts) atomicAdd(n_drop, 1);
        return;
    }
    if (p >= max_pts) return;
    float* o = out + (size_t)p * 8;
    o[0] = (float)(rect_x + (idx % gw) * step);
    o[1] = (float)(rect_y + (idx / gw) * step);
    o[2] = u[idx];
    o[3] = v[idx];
    o[4] = exx[idx];
    o[5] = eyy[idx];
    o[6] = exy[idx];
    o[7] = corr[idx];
}

}  // namespace

cudaError_t launch_median_pass(int gw, int gh, const float* u, const float* v, const uint8_t* ok, uint8_t* fail,
                               int* n_fail, cudaStream_t st) {
    const int n = gw * gh;
    median_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, u, v, ok, fail, n_fail);
    return cudaGetLastError();
}

cudaError_t launch_clear_failed(int n, uint8_t* ok, const uint8_t* fail, cudaStream_t st) {
    clear_failed_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, ok, fail);
    return cudaGetLastError();
}

cudaError_t launch_vsg(int gw, int gh, int step, int window, const float* u, const float* v, const uint8_t* valid,
                       float* exx, float* eyy, float* exy, cudaStream_t st) {
    const float radius = window / 2.0f;
    const int grid_rad = (int)ceilf(radius / (float)step);
    const double r2 = (double)(radius * radius) + 1.0e-5;
    int expected = 0;
    for (int dy = -grid_rad; dy <= grid_rad; ++dy)
        for (int dx = -grid_rad; dx <= grid_rad; ++dx) {
            const double px = (double)(dx * step), py = (double)(dy * step);
            if (px * px + py * py <= r2) ++expected;
        }
    const int n = gw * gh;
    vsg_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, step, grid_rad, r2, expected, u, v, valid, exx, eyy, exy);
    return cudaGetLastError();
}

size_t pack_scratch_bytes(int n) {
    size_t tmp = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tmp, (int*)nullptr, (int*)nullptr, n);
    return tmp + 2 * sizeof(int) * (size_t)n + 256;
}

cudaError_t launch_pack(int gw, int gh, int rect_x, int rect_y, int step, int max_pts, const uint8_t* valid,
                        const float* u, const float* v, const float* corr, const float* exx, const float* eyy,
                        const float* exy, float* out, int* n_drop, int* n_emit_total, void* scratch,
                        size_t scratch_bytes, cudaStream_t st) {
    const int n = gw * gh;
    int* emit = reinterpret_cast<int*>(scratch);
    int* pos = emit + n;
    void* tmp = pos + n;
    size_t tmp_bytes = scratch_bytes - 2 * sizeof(int) * (size_t)n;
    emit_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, valid, exx, emit);
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, emit, pos, n, st);
    if (e != cudaSuccess) return e;
    pack_kernel<<<(n + 127) / 128, 128, 0, st>>>(gw, gh, rect_x, rect_y, step, max_pts, valid, pos, u, v, corr, exx,
                                                  eyy, exy, out, n_drop);
    // total emits = pos[n-1] + emit[n-1]: both go to n_emit_total[0..1]
    e = cudaMemcpyAsync(n_emit_total, pos + (n - 1), sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    e = cudaMemcpyAsync(n_emit_total + 1, emit + (n - 1), sizeof(int), cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

}  // namespace dic
