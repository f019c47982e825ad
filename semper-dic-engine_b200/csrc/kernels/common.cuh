// Device building blocks shared by the DIC kernels (sm_100a).
//
// Arithmetic contract. Every kernel file is compiled with -fmad=false, so no
// multiply-add is fused unless written as __fmaf_rn / __fma_rn here. Subset
// reductions put pixel i (row-major in the subset) in lane i % 32, accumulate
// in increasing i, and finish with an xor butterfly; IEEE addition being
// commutative, every lane ends with the same bits. The CPU restatement used by
// the tests follows the same contract, so results agree bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace dic {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float wsum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __dadd_rn(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ int wsum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ bool finite_f(float f) {
    return (__float_as_uint(f) & 0x7f800000u) != 0x7f800000u;
}
__device__ __forceinline__ bool finite_d(double d) {
    return ((unsigned long long)__double_as_longlong(d) & 0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}

// Catmull-Rom weights (src/math/image_processor.cpp:188-195) with the fused
// products of the contract.
__device__ __forceinline__ void cubic_weights(float s, float w[4]) {
    const float s2 = s * s, s3 = s2 * s;
    w[0] = __fmaf_rn(-0.5f, s, __fmaf_rn(-0.5f, s3, s2));
    w[1] = __fmaf_rn(-2.5f, s2, __fmaf_rn(1.5f, s3, 1.0f));
    w[2] = __fmaf_rn(0.5f, s, __fmaf_rn(-1.5f, s3, 2.0f * s2));
    w[3] = __fmaf_rn(0.5f, s3, -0.5f * s2);
}

// Keys 4th-order zones (image_processor.cpp:70-82).
__device__ __forceinline__ float keys_f0(float s) {
    const float s2 = s * s, s3 = s2 * s;
    return __fmaf_rn(4.0f / 3.0f, s3, __fmaf_rn(-7.0f / 3.0f, s2, 1.0f));
}
__device__ __forceinline__ float keys_f1(float s) {
    const float s2 = s * s, s3 = s2 * s;
    return __fmaf_rn(-7.0f / 12.0f, s3, __fmaf_rn(3.0f, s2, __fmaf_rn(-59.0f / 12.0f, s, 2.5f)));
}
__device__ __forceinline__ float keys_f2(float s) {
    const float s2 = s * s, s3 = s2 * s;
    return __fmaf_rn(1.0f / 12.0f, s3, __fmaf_rn(-2.0f / 3.0f, s2, __fmaf_rn(7.0f / 4.0f, s, -1.5f)));
}
__device__ __forceinline__ void keys6_weights(float d, float w[6]) {
    w[0] = keys_f2(d + 2.0f);
    w[1] = keys_f1(d + 1.0f);
    w[2] = keys_f0(d);
    w[3] = keys_f0(1.0f - d);
    w[4] = keys_f1(2.0f - d);
    w[5] = keys_f2(3.0f - d);
}

// Interpolated value at (xi + dx, yi + dy) from a row-major float plane with
// row pitch `pitch` (elements); base points at element (0, 0) of the plane.
__device__ __forceinline__ float interp4(const float* __restrict__ base, int pitch, int xi, int yi,
                                         float dx, float dy) {
    float wx[4], wy[4];
    cubic_weights(dx, wx);
    cubic_weights(dy, wy);
    const float* r = base + (size_t)(yi - 1) * pitch + (xi - 1);
    float val = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float* q = r + (size_t)j * pitch;
        float rv = __ldg(q) * wx[0];
        rv = __fmaf_rn(__ldg(q + 1), wx[1], rv);
        rv = __fmaf_rn(__ldg(q + 2), wx[2], rv);
        rv = __fmaf_rn(__ldg(q + 3), wx[3], rv);
        val = (j == 0) ? rv * wy[0] : __fmaf_rn(rv, wy[j], val);
    }
    return val;
}

__device__ __forceinline__ float interp6(const float* __restrict__ base, int pitch, int xi, int yi,
                                         float dx, float dy) {
    float wx[6], wy[6];
    keys6_weights(dx, wx);
    keys6_weights(dy, wy);
    const float* r = base + (size_t)(yi - 2) * pitch + (xi - 2);
    float val = 0.0f;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const float* q = r + (size_t)j * pitch;
        float rv = __ldg(q) * wx[0];
#pragma unroll
        for (int i = 1; i < 6; ++i) rv = __fmaf_rn(__ldg(q + i), wx[i], rv);
        val = (j == 0) ? rv * wy[0] : __fmaf_rn(rv, wy[j], val);
    }
    return val;
}

// The same from a shared-memory tile (row pitch `pitch`), same arithmetic.
__device__ __forceinline__ float interp4s(const float* base, int pitch, int xi, int yi, float dx, float dy) {
    float wx[4], wy[4];
    cubic_weights(dx, wx);
    cubic_weights(dy, wy);
    const float* r = base + (yi - 1) * pitch + (xi - 1);
    float val = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float* q = r + j * pitch;
        float rv = q[0] * wx[0];
        rv = __fmaf_rn(q[1], wx[1], rv);
        rv = __fmaf_rn(q[2], wx[2], rv);
        rv = __fmaf_rn(q[3], wx[3], rv);
        val = (j == 0) ? rv * wy[0] : __fmaf_rn(rv, wy[j], val);
    }
    return val;
}

__device__ __forceinline__ float interp6s(const float* base, int pitch, int xi, int yi, float dx, float dy) {
    float wx[6], wy[6];
    keys6_weights(dx, wx);
    keys6_weights(dy, wy);
    const float* r = base + (yi - 2) * pitch + (xi - 2);
    float val = 0.0f;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        const float* q = r + j * pitch;
        float rv = q[0] * wx[0];
#pragma unroll
        for (int i = 1; i < 6; ++i) rv = __fmaf_rn(q[i], wx[i], rv);
        val = (j == 0) ? rv * wy[0] : __fmaf_rn(rv, wy[j], val);
    }
    return val;
}

// Two pixels at once on the paired FP32 instructions of sm_100 (each half an
// IEEE single-precision operation rounded to nearest, so every value is the
// one the scalar form gives): the Catmull-Rom weights of two offsets and
// interp4s of two samples from the same tile.
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }

__device__ __forceinline__ void cubic_weights_x2(float2 s, float2 w[4]) {
    const float2 s2 = __fmul2_rn(s, s), s3 = __fmul2_rn(s2, s);
    w[0] = __ffma2_rn(f2(-0.5f), s, __ffma2_rn(f2(-0.5f), s3, s2));
    w[1] = __ffma2_rn(f2(-2.5f), s2, __ffma2_rn(f2(1.5f), s3, f2(1.0f)));
    w[2] = __ffma2_rn(f2(0.5f), s, __ffma2_rn(f2(-1.5f), s3, __fmul2_rn(f2(2.0f), s2)));
    w[3] = __ffma2_rn(f2(0.5f), s3, __fmul2_rn(f2(-0.5f), s2));
}

// Pixel A at (xa + dx.x, ya + dy.x), pixel B at (xb + dx.y, yb + dy.y).
__device__ __forceinline__ float2 interp4s_x2(const float* base, int pitch, int xa, int ya, int xb, int yb, float2 dx,
                                              float2 dy) {
    float2 wx[4], wy[4];
    cubic_weights_x2(dx, wx);
    cubic_weights_x2(dy, wy);
    const float* ra = base + (ya - 1) * pitch + (xa - 1);
    const float* rb = base + (yb - 1) * pitch + (xb - 1);
    float2 val = f2(0.0f);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float* qa = ra + j * pitch;
        const float* qb = rb + j * pitch;
        float2 rv = __fmul2_rn(make_float2(qa[0], qb[0]), wx[0]);
        rv = __ffma2_rn(make_float2(qa[1], qb[1]), wx[1], rv);
        rv = __ffma2_rn(make_float2(qa[2], qb[2]), wx[2], rv);
        rv = __ffma2_rn(make_float2(qa[3], qb[3]), wx[3], rv);
        val = (j == 0) ? __fmul2_rn(rv, wy[0]) : __ffma2_rn(rv, wy[j], val);
    }
    return val;
}

// The 6x6 FP64 helpers of the Hessian: Cholesky, explicit inverse, and the
// scaled 1-norm reciprocal condition (src/math/hessian.hpp:40-52). The `_r`
// forms are fully unrolled, so their matrices live in registers; the
// out-of-line forms copy their arguments in and out around them, for callers
// that are short of registers. Both perform the same operations in the same
// order.
__device__ __forceinline__ bool cholesky6_r(const double (&A)[6][6], double (&L)[6][6]) {
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) L[i][j] = 0.0;
    bool ok = true;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double s = A[j][j];
#pragma unroll
        for (int k = 0; k < j; ++k) s = s - L[j][k] * L[j][k];
        ok = ok && (s > 0.0) && finite_d(s);
        const double d = sqrt(s);
        L[j][j] = d;
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double t = A[i][j];
#pragma unroll
            for (int k = 0; k < j; ++k) t = t - L[i][k] * L[j][k];
            L[i][j] = t / d;
        }
        if (!ok) return false;
    }
    return true;
}

// Ai is written whenever the factorisation succeeds (factored), even when a
// non-finite entry makes the result false.
__device__ __forceinline__ bool inverse6_r(const double (&A)[6][6], double (&Ai)[6][6], bool& factored) {
    double L[6][6];
    factored = cholesky6_r(A, L);
    if (!factored) return false;
    double Li[6][6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
        for (int j = 0; j < 6; ++j) Li[i][j] = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        Li[c][c] = 1.0 / L[c][c];
#pragma unroll
        for (int i = c + 1; i < 6; ++i) {
            double t = 0.0;
#pragma unroll
            for (int k = c; k < i; ++k) t = t + L[i][k] * Li[k][c];
            Li[i][c] = -t / L[i][i];
        }
    }
    bool ok = true;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = r; c < 6; ++c) {
            double t = 0.0;
#pragma unroll
            for (int k = c; k < 6; ++k) t = t + Li[k][r] * Li[k][c];
            Ai[r][c] = t;
            Ai[c][r] = t;
            ok = ok && finite_d(t);
        }
    return ok;
}

__device__ __forceinline__ bool well_conditioned_r(const double (&H)[6][6], int half) {
    const double s = half > 1 ? 1.0 / (double)half : 1.0;
    const double d[6] = {1.0, 1.0, s, s, s, s};
    double Hn[6][6], Hi[6][6];
    bool fin = true;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            Hn[r][c] = (d[r] * H[r][c]) * d[c];
            fin = fin && finite_d(Hn[r][c]);
        }
    if (!fin) return false;
    bool factored;
    if (!inverse6_r(Hn, Hi, factored)) return false;
    double na = 0.0, ni = 0.0;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double a = 0.0, b = 0.0;
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            a = a + fabs(Hn[r][c]);
            b = b + fabs(Hi[r][c]);
        }
        na = fmax(na, a);
        ni = fmax(ni, b);
    }
    return 1.0 / (na * ni) > (double)1e-6f;
}

static __device__ __noinline__ bool inverse6(const double A[6][6], double Ai[6][6]) {
    double a[6][6], ai[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 6; ++c) a[r][c] = A[r][c];
    bool factored;
    const bool ok = inverse6_r(a, ai, factored);
    if (factored) {
#pragma unroll
        for (int r = 0; r < 6; ++r)
#pragma unroll
            for (int c = 0; c < 6; ++c) Ai[r][c] = ai[r][c];
    }
    return ok;
}

static __device__ __noinline__ bool well_conditioned(const double H[6][6], int half) {
    double h[6][6];
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 6; ++c) h[r][c] = H[r][c];
    return well_conditioned_r(h, half);
}

// Warp-collective forms of inverse6_r and well_conditioned_r, for a block
// whose other warps wait on the result: every entry is formed by the same
// operations in the same order as in the one-thread forms, so the results
// agree bit for bit. The chain of one column (square root, divisions) is the
// critical path instead of the whole factorisation. Matrices are 36 doubles,
// row-major, in shared memory; every lane of the warp takes part.
//
// Cholesky with lane i < 6 holding row i of L, the triangular inverse with
// lane c < 6 holding column c of L^-1, and the product L^-T L^-1 with lane
// m < 21 forming upper-triangle entry m. scr: 72 doubles. Ai is written when
// the factorisation succeeds (factored), as by inverse6.
__device__ __forceinline__ bool inverse6_warp(const double* A, double* Ai, double* scr, bool& factored) {
    const int lane = threadIdx.x & 31;
    double* Ls = scr;       // L, row-major
    double* Lis = scr + 36;  // L^-1, row-major
    double Lr[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) Lr[c] = 0.0;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double Lj[6];
#pragma unroll
        for (int k = 0; k < j; ++k) Lj[k] = __shfl_sync(kFull, Lr[k], j);
        int okj = 1;
        if (lane == j) {
            double s = A[j * 6 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) s = s - Lr[k] * Lr[k];
            okj = (s > 0.0) && finite_d(s);
            Lr[j] = sqrt(s);
        }
        const double d = __shfl_sync(kFull, Lr[j], j);
        okj = __shfl_sync(kFull, okj, j);
        if (lane > j && lane < 6) {
            double t = A[lane * 6 + j];
#pragma unroll
            for (int k = 0; k < j; ++k) t = t - Lr[k] * Lj[k];
            Lr[j] = t / d;
        }
        if (!okj) {
            factored = false;
            return false;
        }
    }
    factored = true;
    if (lane < 6) {
#pragma unroll
        for (int c = 0; c < 6; ++c) Ls[lane * 6 + c] = Lr[c];
    }
    __syncwarp();
    if (lane < 6) {
        const int c = lane;
        double Lc[6];
#pragma unroll
        for (int i = 0; i < 6; ++i) {
            Lc[i] = 0.0;
            if (i == c) {
                Lc[i] = 1.0 / Ls[i * 6 + i];
            } else if (i > c) {
                double t = 0.0;
#pragma unroll
                for (int k = 0; k < i; ++k)
                    if (k >= c) t = t + Ls[i * 6 + k] * Lc[k];
                Lc[i] = -t / Ls[i * 6 + i];
            }
        }
#pragma unroll
        for (int i = 0; i < 6; ++i) Lis[i * 6 + c] = Lc[i];
    }
    __syncwarp();
    bool ok = true;
    if (lane < 21) {
        int r = 0, m = lane;
        while (m >= 6 - r) {
            m -= 6 - r;
            ++r;
        }
        const int c = r + m;
        double t = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k)
            if (k >= c) t = t + Lis[k * 6 + r] * Lis[k * 6 + c];
        Ai[r * 6 + c] = t;
        Ai[c * 6 + r] = t;
        ok = finite_d(t);
    }
    ok = __all_sync(kFull, ok);
    __syncwarp();
    return ok;
}

// well_conditioned_r on H (shared memory); scr: 180 doubles.
__device__ __forceinline__ bool well_conditioned_warp(const double* H, int half, double* scr) {
    const int lane = threadIdx.x & 31;
    double* Hn = scr;
    double* Hi = scr + 36;
    double* sub = scr + 72;
    const double s = half > 1 ? 1.0 / (double)half : 1.0;
    bool fin = true;
    for (int e = lane; e < 36; e += 32) {
        const int r = e / 6, c = e - (e / 6) * 6;
        const double dr = r < 2 ? 1.0 : s, dc = c < 2 ? 1.0 : s;
        const double h = (dr * H[e]) * dc;
        Hn[e] = h;
        fin = fin && finite_d(h);
    }
    fin = __all_sync(kFull, fin);
    __syncwarp();
    if (!fin) return false;
    bool factored;
    if (!inverse6_warp(Hn, Hi, sub, factored)) return false;
    double a = 0.0, b = 0.0;
    if (lane < 6) {
#pragma unroll
        for (int r = 0; r < 6; ++r) {
            a = a + fabs(Hn[r * 6 + lane]);
            b = b + fabs(Hi[r * 6 + lane]);
        }
    }
    // the largest column sums; fmax of non-negative, non-NaN values in any order
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) {
        a = fmax(a, __shfl_xor_sync(kFull, a, o));
        b = fmax(b, __shfl_xor_sync(kFull, b, o));
    }
    const double na = __shfl_sync(kFull, a, 0), ni = __shfl_sync(kFull, b, 0);
    __syncwarp();
    return 1.0 / (na * ni) > (double)1e-6f;
}

__device__ __forceinline__ bool cond2x2_ok(const double (&H)[6][6]) {
    const double det = H[0][0] * H[1][1] - H[1][0] * H[0][1];
    const double nrm = H[0][0] * H[0][0] + H[0][1] * H[0][1] + H[1][0] * H[1][0] + H[1][1] * H[1][1];
    const double cond = fabs(det) > 1e-12 ? nrm / fabs(det) : 1.0e13;
    return !(cond > 1.0e12);
}

// Index of (r, c), r <= c, in the 21-entry upper triangle (row-major).
__host__ __device__ constexpr int tri21(int r, int c) { return r * 6 - (r * (r - 1)) / 2 + (c - r); }
// The row and column of upper-triangle entry m (the inverse of tri21).
__host__ __device__ constexpr int tri_row(int m) {
    int r = 0;
    while (m >= 6 - r) {
        m -= 6 - r;
        ++r;
    }
    return r;
}
__host__ __device__ constexpr int tri_col(int m) { return tri_row(m) + (m - tri21(tri_row(m), tri_row(m))); }

}  // namespace dic
