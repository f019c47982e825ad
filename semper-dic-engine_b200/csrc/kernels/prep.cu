// Reference/deformed image preparation, the grid validity scan, and the
// per-node Hessian pool.
//
//   image pass      Image::Image + prepare_data(false) (src/math/image_processor.cpp:9-24,54-63)
//                   + stamp_ghost_wall (src/pipeline/reference_cache.cpp:18-35)
//   grid scan       src/pipeline/full_field_solver.cpp:266-318
//   Hessian pool    SubsetPrecomputer::compute_hessian_only (src/math/subset_precomputer.cpp:42-149)
//                   + hessian::well_conditioned (src/math/hessian.hpp:40-52), FP64
#include <cuda_runtime.h>

#include "common.cuh"
#include "prep.cuh"

namespace dic {

namespace {

// x / 12 correctly rounded for an integer-valued x with |x| <= 2295 (the
// gradient numerators of 8-bit images): the quotient by the rounded
// reciprocal, then one FMA residual correction (Markstein's method for a
// divisor known in advance). For these numerators the result equals the IEEE
// quotient bit for bit; the tests compare the planes with the CPU
// restatement's divisions.
__device__ __forceinline__ float div12(float x) {
    const float inv = 1.0f / 12.0f;  // RN(1/12), folded at compile time
    const float q = x * inv;
    const float r = __fmaf_rn(-q, 12.0f, x);
    return __fmaf_rn(r, inv, q);
}

// One thread per 4 horizontally adjacent pixels: u8 -> f32 intensity and the
// 4th-order central-difference gradients (zero within 2 px of the border),
// then the Ghost Wall where the mask is below 128. Integer numerators make
// the gradient the correctly rounded quotient in any order. Stores are float4
// when the row pitch allows it (W % 4 == 0), scalar otherwise.
__global__ void image_kernel(const uint8_t* __restrict__ px, const uint8_t* __restrict__ mask, int W,
                             int H, int pitch, float* __restrict__ I, float* __restrict__ gx,
                             float* __restrict__ gy) {
    const int x0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int y = blockIdx.y;
    if (x0 >= pitch || y >= H) return;
    const size_t row = (size_t)y * W;
    const size_t orow = (size_t)y * pitch;
    float vi[4], vx[4], vy[4];
    // Interior threads of 4-byte-aligned rows read their bytes as words: three
    // of the row (x0 - 4 .. x0 + 7) and one of each of the four rows above and
    // below; the same integer numerators as the byte path.
    const bool words = ((W & 3) == 0) && ((reinterpret_cast<uintptr_t>(px) & 3) == 0) && x0 >= 4 && x0 + 8 <= W &&
                       y >= 2 && y < H - 2;
    if (words) {
        const uint32_t* r = reinterpret_cast<const uint32_t*>(px + row) + (x0 >> 2);
        const size_t wr = (size_t)W >> 2;
        const uint32_t a = __ldg(r - 1), b = __ldg(r), c = __ldg(r + 1);
        const uint32_t u1 = __ldg(r - wr), u2 = __ldg(r - 2 * wr), d1 = __ldg(r + wr), d2 = __ldg(r + 2 * wr);
        int v[12];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            v[k] = (int)((a >> (8 * k)) & 0xffu);
            v[4 + k] = (int)((b >> (8 * k)) & 0xffu);
            v[8 + k] = (int)((c >> (8 * k)) & 0xffu);
        }
        uint32_t m = 0xffffffffu;
        if (mask) {
            if ((reinterpret_cast<uintptr_t>(mask) & 3) == 0)
                m = __ldg(reinterpret_cast<const uint32_t*>(mask + row) + (x0 >> 2));
            else
                m = (uint32_t)__ldg(mask + row + x0) | ((uint32_t)__ldg(mask + row + x0 + 1) << 8) |
                    ((uint32_t)__ldg(mask + row + x0 + 2) << 16) | ((uint32_t)__ldg(mask + row + x0 + 3) << 24);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int nx = -v[6 + k] + 8 * v[5 + k] - 8 * v[3 + k] + v[2 + k];
            const int ny = -(int)((d2 >> (8 * k)) & 0xffu) + 8 * (int)((d1 >> (8 * k)) & 0xffu) -
                           8 * (int)((u1 >> (8 * k)) & 0xffu) + (int)((u2 >> (8 * k)) & 0xffu);
            vi[k] = (float)v[4 + k];
            vx[k] = div12((float)nx);
            vy[k] = div12((float)ny);
            if (((m >> (8 * k)) & 0xffu) < 128u) vi[k] = -10.0f;
        }
    }
#pragma unroll
    for (int k = 0; k < 4 && !words; ++k) {
        const int x = x0 + k;
        vi[k] = vx[k] = vy[k] = 0.0f;
        if (x >= W) continue;
        const size_t p = row + x;
        vi[k] = (float)__ldg(px + p);
        if (x >= 2 && x < W - 2 && y >= 2 && y < H - 2) {
            const int nx = -(int)__ldg(px + p + 2) + 8 * (int)__ldg(px + p + 1) - 8 * (int)__ldg(px + p - 1) +
                           (int)__ldg(px + p - 2);
            const int ny = -(int)__ldg(px + p + 2 * (size_t)W) + 8 * (int)__ldg(px + p + W) -
                           8 * (int)__ldg(px + p - W) + (int)__ldg(px + p - 2 * (size_t)W);
            vx[k] = div12((float)nx);
            vy[k] = div12((float)ny);
        }
        if (mask && __ldg(mask + p) < 128) vi[k] = -10.0f;
    }
    if ((pitch & 3) == 0) {
        reinterpret_cast<float4*>(I + orow)[x0 >> 2] = make_float4(vi[0], vi[1], vi[2], vi[3]);
        reinterpret_cast<float4*>(gx + orow)[x0 >> 2] = make_float4(vx[0], vx[1], vx[2], vx[3]);
        reinterpret_cast<float4*>(gy + orow)[x0 >> 2] = make_float4(vy[0], vy[1], vy[2], vy[3]);
    } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (x0 + k >= pitch) break;
            I[orow + x0 + k] = vi[k];
            gx[orow + x0 + k] = vx[k];
            gy[orow + x0 + k] = vy[k];
        }
    }
}

// One warp per grid node: skip within half + 19 px of the border, or when any
// subset pixel is masked (< 128).
__global__ void scan_kernel(const uint8_t* __restrict__ mask, int W, int H, int gridW, int gridH, int rect_x,
                            int rect_y, int step, int dim, uint8_t* __restrict__ skip, int* __restrict__ n_valid) {
    const int node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (node >= gridW * gridH) return;
    const int gx = node % gridW, gy = node / gridW;
    const int rx = rect_x + gx * step, ry = rect_y + gy * step;
    const int hs = dim / 2, buf = hs + 4 + 15;
    bool s = rx - buf < 0 || rx + buf >= W || ry - buf < 0 || ry + buf >= H;
    if (!s && mask) {
        int bad = 0;
        for (int i = lane; i < dim * dim; i += 32) {
            const int dy = i / dim - hs, dx = i % dim - hs;
            if (__ldg(mask + (size_t)(ry + dy) * W + rx + dx) < 128) bad = 1;
        }
        s = __any_sync(kFull, bad) != 0;
    }
    if (lane == 0) {
        skip[node] = s ? 1 : 0;
        if (!s) atomicAdd(n_valid, 1);
    }
}

// One warp per node of the pool: mean and std over non-Ghost pixels (FP32,
// lane partial sums + butterfly) and the 21-entry Gauss-Newton Hessian
// (FP64), written to Hs21 for pool_finish_kernel. A node that is skipped,
// off the image or less than half valid is marked invalid here (flag 0) and
// left alone by the finish; the others get flag 2 ("sums ready").
__global__ void pool_sums_kernel(const float* __restrict__ I, const float* __restrict__ Gx,
                                 const float* __restrict__ Gy, int W, int H, int pitch,
                                 const uint8_t* __restrict__ skip, int gridW, int gridH, int rect_x, int rect_y,
                                 int step, int dim, uint8_t* __restrict__ valid, float2* __restrict__ ms,
                                 double* __restrict__ Hs21) {
    const int node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (node >= gridW * gridH) return;
    const int half = dim / 2, n = dim * dim;
    const int cx = rect_x + (node % gridW) * step, cy = rect_y + (node / gridW) * step;
    const bool ok_dim = dim >= 3 && (dim & 1);
    const bool on = cx - half >= 0 && cx + half < W && cy - half >= 0 && cy + half < H;
    auto invalid = [&]() {
        if (lane == 0) {
            valid[node] = 0;
            ms[node] = make_float2(0.0f, 1.0f);
        }
        if (lane < 21) Hs21[(size_t)node * 21 + lane] = 0.0;
    };
    if ((skip && skip[node]) || !ok_dim || !on) {
        invalid();
        return;
    }
    const size_t base = (size_t)(cy - half) * pitch + (cx - half);
    const int q = 32 / dim, r = 32 - q * dim;

    float part = 0.0f;
    int cnt = 0;
    {
        int row = lane / dim, col = lane - row * dim;
        for (int i = lane; i < n; i += 32) {
            const float v = __ldg(I + base + (size_t)row * pitch + col);
            if (!(v < -5.0f)) {
                part = part + v;
                ++cnt;
            }
            col += r; row += q;
            if (col >= dim) { col -= dim; ++row; }
        }
    }
    cnt = wsum(cnt);
    const float sum = wsum(part);
    if ((float)cnt < (float)n * 0.5f) {
        invalid();
        return;
    }
    const float mean = sum / (float)cnt;
    part = 0.0f;
    {
        int row = lane / dim, col = lane - row * dim;
        for (int i = lane; i < n; i += 32) {
            const float v = __ldg(I + base + (size_t)row * pitch + col);
            if (!(v < -5.0f)) {
                const float d = v - mean;
                part = __fmaf_rn(d, d, part);
            }
            col += r; row += q;
            if (col >= dim) { col -= dim; ++row; }
        }
    }
    float sd = sqrtf(wsum(part) / (float)cnt);
    if (sd < 1e-5f) sd = 1.0f;
    const float inv = 1.0f / sd;

    double hp[21];
#pragma unroll
    for (int k = 0; k < 21; ++k) hp[k] = 0.0;
    {
        int row = lane / dim, col = lane - row * dim;
        for (int i = lane; i < n; i += 32) {
            const size_t p = base + (size_t)row * pitch + col;
            if (!(__ldg(I + p) < -5.0f)) {
                const float g0 = __ldg(Gx + p) * inv, g1 = __ldg(Gy + p) * inv;
                const float fx = (float)(col - half), fy = (float)(row - half);
                const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                                     (double)(g1 * fx), (double)(g1 * fy)};
                int k = 0;
#pragma unroll
                for (int a = 0; a < 6; ++a)
#pragma unroll
                    for (int b = a; b < 6; ++b, ++k) hp[k] = __fma_rn(s[a], s[b], hp[k]);
            }
            col += r; row += q;
            if (col >= dim) { col -= dim; ++row; }
        }
    }
#pragma unroll
    for (int k = 0; k < 21; ++k) hp[k] = wsum(hp[k]);
    if (lane < 21) {
        double v = 0.0;
#pragma unroll
        for (int k = 0; k < 21; ++k)
            if (k == lane) v = hp[k];
        Hs21[(size_t)node * 21 + lane] = v;
    }
    if (lane == 0) {
        valid[node] = 2;
        ms[node] = make_float2(mean, sd);
    }
}

// One thread per node whose sums are ready: the 2x2 and scaled-rcond checks
// and the step matrix of a whole-subset iteration (optimization_engine.cpp:
// 302-315): the LM-damped inverse when damping is on and the damped matrix is
// well conditioned, else the plain inverse. Hs21 holds the Hessian on entry
// (copied to H21 when given) and the step matrix on return. The 6x6 FP64 work
// is serial per node, so nodes run one per thread rather than one per warp.
__global__ void pool_finish_kernel(int nodes, int half, int lm, uint8_t* __restrict__ valid,
                                   double* __restrict__ H21, double* __restrict__ Hs21) {
    const int node = blockIdx.x * blockDim.x + threadIdx.x;
    if (node >= nodes || valid[node] != 2) return;
    double* o = Hs21 + (size_t)node * 21;
    double Hm[6][6], Hs[6][6];
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = a; b < 6; ++b) {
            Hm[a][b] = o[tri21(a, b)];
            Hm[b][a] = Hm[a][b];
        }
    if (H21)
#pragma unroll
        for (int k = 0; k < 21; ++k) H21[(size_t)node * 21 + k] = o[k];
    const bool good = cond2x2_ok(Hm) && well_conditioned_r(Hm, half);
    uint8_t v = good ? 1 : 0;
    bool done = false, factored = false;
    if (good && lm) {
        double Hd[6][6];
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = 0; b < 6; ++b) Hd[a][b] = Hm[a][b];
        Hd[0][0] += (double)0.05f;
        Hd[1][1] += (double)0.05f;
        if (well_conditioned_r(Hd, half) && inverse6_r(Hd, Hs, factored)) done = true;
    }
    if (good && !done && !inverse6_r(Hm, Hs, factored)) v = 0;
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
        for (int b = a; b < 6; ++b) o[tri21(a, b)] = good ? Hs[a][b] : 0.0;
    valid[node] = v;
}

}  // namespace

cudaError_t launch_image_prep(const uint8_t* px, const uint8_t* mask, int W, int H, int pitch, float* I, float* gx,
                              float* gy, cudaStream_t st) {
    const int threads = 128;
    const int per_row = (pitch + 3) / 4;
    dim3 grid((per_row + threads - 1) / threads, H);
    image_kernel<<<grid, threads, 0, st>>>(px, mask, W, H, pitch, I, gx, gy);
    return cudaGetLastError();
}

cudaError_t launch_grid_scan(const uint8_t* mask, int W, int H, int gridW, int gridH, int rect_x, int rect_y,
                             int step, int dim, uint8_t* skip, int* n_valid, cudaStream_t st) {
    const int nodes = gridW * gridH;
    const int wpb = 8;
    scan_kernel<<<(nodes + wpb - 1) / wpb, wpb * 32, 0, st>>>(mask, W, H, gridW, gridH, rect_x, rect_y, step, dim,
                                                               skip, n_valid);
    return cudaGetLastError();
}

cudaError_t launch_pool(const float* I, const float* gx, const float* gy, int W, int H, int pitch, const uint8_t* skip,
                        int gridW, int gridH, int rect_x, int rect_y, int step, int dim, int lm, uint8_t* valid,
                        float2* ms, double* H21, double* Hs21, cudaStream_t st) {
    const int nodes = gridW * gridH;
    const int wpb = 4;
    pool_sums_kernel<<<(nodes + wpb - 1) / wpb, wpb * 32, 0, st>>>(I, gx, gy, W, H, pitch, skip, gridW, gridH,
                                                                    rect_x, rect_y, step, dim, valid, ms, Hs21);
    if (H21) {
        const cudaError_t e = cudaMemsetAsync(H21, 0, (size_t)nodes * 21 * sizeof(double), st);
        if (e != cudaSuccess) return e;
    }
    pool_finish_kernel<<<(nodes + 127) / 128, 128, 0, st>>>(nodes, dim / 2, lm, valid, H21, Hs21);
    return cudaGetLastError();
}

}  // namespace dic
