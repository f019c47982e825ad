// The learned seed proposal network (proposal.cuh) on sm_100a.
//
// Every product of the network — the five convolutions and two dense layers,
// forward, and their input and weight gradients backward — is one GEMM on
// the tensor cores: mma.sync m16n8k16 with bfloat16 operands and FP32
// accumulation. Convolutions are implicit GEMMs: the operand loaders gather
// the 3x3, stride-2 windows of the NHWC activations (im2col) as they stage a
// tile in shared memory, so no column matrix is written; a weight gradient
// reduces over the batch with split-K and FP32 atomics. Bias, ReLU, the loss,
// the column-to-image adjoint and Adam are small elementwise kernels. FP32
// values (weights, back-propagated gradients) are rounded to bfloat16 (nearest
// even) as the loaders read them, which is where the CPU restatement rounds
// them too.
#include "proposal.cuh"

#include <cuda_bf16.h>

namespace dic {

PpLayout pp_layout() {
    PpLayout L{};
    size_t o = 0;
    for (int l = 0; l < 5; ++l) {
        L.w[l] = o;
        o += (size_t)kPpChannels[l + 1] * 9 * kPpChannels[l];
        L.b[l] = o;
        o += (size_t)kPpChannels[l + 1];
    }
    L.w[5] = o;
    o += (size_t)kPpFc1 * kPpFc0;
    L.b[5] = o;
    o += kPpFc1;
    L.w[6] = o;
    o += (size_t)kPpOut * kPpFc1;
    L.b[6] = o;
    o += kPpOut;
    L.total = o;
    return L;
}

namespace {

__device__ __forceinline__ uint16_t to_bf16(float x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t*>(&h);
}
__device__ __forceinline__ float from_bf16(uint16_t u) { return __uint_as_float((uint32_t)u << 16); }

// Operand loaders: the bfloat16 bits of element (r, k) of a GEMM operand,
// A(m, k) or B^T(n, k); callers keep (r, k) in range.
struct LdBfRow {  // bf16 matrix, element (r, k) at p[r * ld + k]
    const uint16_t* p;
    int ld;
    __device__ uint16_t operator()(int r, int k) const { return p[(size_t)r * ld + k]; }
};
struct LdBfCol {  // bf16 matrix read transposed: element (r, k) at p[k * ld + r]
    const uint16_t* p;
    int ld;
    __device__ uint16_t operator()(int r, int k) const { return p[(size_t)k * ld + r]; }
};
struct LdF32Row {  // FP32 matrix, rounded: element (r, k) at p[r * ld + k]
    const float* p;
    int ld;
    __device__ uint16_t operator()(int r, int k) const { return to_bf16(p[(size_t)r * ld + k]); }
};
struct LdF32Col {  // FP32 matrix read transposed, rounded: element (r, k) at p[k * ld + r]
    const float* p;
    int ld;
    __device__ uint16_t operator()(int r, int k) const { return to_bf16(p[(size_t)k * ld + r]); }
};
// The 3x3, stride-2, padding-1 windows of an NHWC bf16 tensor [B, H, W, C]
// as a matrix: row m = (b, i, j) of the H/2 x W/2 output, column k = (kh, kw,
// c); zero outside the image. `Transposed` swaps the roles of the indices.
template <bool Transposed>
struct LdIm2Col {
    const uint16_t* x;
    int H, W, C;
    __device__ uint16_t operator()(int r, int c) const {
        const int m = Transposed ? c : r, k = Transposed ? r : c;
        const int Ho = H >> 1, Wo = W >> 1;
        const int b = m / (Ho * Wo), rem = m - b * (Ho * Wo);
        const int i = rem / Wo, j = rem - i * Wo;
        const int kh = k / (3 * C), kr = k - kh * 3 * C;
        const int kw = kr / C, ch = kr - kw * C;
        const int y = 2 * i + kh - 1, xx = 2 * j + kw - 1;
        if (y < 0 || y >= H || xx < 0 || xx >= W) return 0;
        return x[(((size_t)b * H + y) * W + xx) * C + ch];
    }
};

__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// C[M x N] (row stride ldc) = sum over k of A(m, k) B^T(n, k), FP32. A block
// of 4 warps computes a 64 x 64 tile, each warp 32 x 32 (2 x 4 mma tiles);
// K is walked 16 at a time through shared memory (pairs of bf16 packed in a
// word, rows padded to 9 words so the fragment reads meet distinct banks).
// Blocks along z take `kchunk`-long slices of K; with `atomic` they add into
// C (zeroed first), else they store, block z at C + z * slice (slice 0: all
// into C), so that split partials can be summed later in a fixed order.
template <class LA, class LB>
__global__ void __launch_bounds__(128) gemm_kernel(LA A, LB Bt, int M, int N, int K, float* C, int ldc, int kchunk,
                                                   int atomic, size_t slice) {
    __shared__ uint32_t As[64][9];
    __shared__ uint32_t Bs[64][9];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int k_begin = blockIdx.z * kchunk;
    const int k_end = min(K, k_begin + kchunk);
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0f;
    for (int k0 = k_begin; k0 < k_end; k0 += 16) {
        for (int e = tid; e < 64 * 8; e += 128) {
            const int r = e >> 3, kp = e & 7, k = k0 + 2 * kp;
            const int m = m0 + r, n = n0 + r;
            uint32_t va = 0, vb = 0;
            if (m < M) {
                if (k < k_end) va = A(m, k);
                if (k + 1 < k_end) va |= (uint32_t)A(m, k + 1) << 16;
            }
            if (n < N) {
                if (k < k_end) vb = Bt(n, k);
                if (k + 1 < k_end) vb |= (uint32_t)Bt(n, k + 1) << 16;
            }
            As[r][kp] = va;
            Bs[r][kp] = vb;
        }
        __syncthreads();
        uint32_t af[2][4], bfr[4][2];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int row = wm + mt * 16 + g;
            af[mt][0] = As[row][t];
            af[mt][1] = As[row + 8][t];
            af[mt][2] = As[row][t + 4];
            af[mt][3] = As[row + 8][t + 4];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int col = wn + nt * 8 + g;
            bfr[nt][0] = Bs[col][t];
            bfr[nt][1] = Bs[col][t + 4];
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], af[mt], bfr[nt]);
        __syncthreads();
    }
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int r0 = m0 + wm + mt * 16 + g, c0 = n0 + wn + nt * 8 + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = r0 + 8 * h;
                if (r >= M) continue;
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const int c = c0 + q;
                    if (c >= N) continue;
                    float* dst = C + (size_t)blockIdx.z * slice + (size_t)r * ldc + c;
                    if (atomic)
                        atomicAdd(dst, acc[mt][nt][2 * h + q]);
                    else
                        *dst = acc[mt][nt][2 * h + q];
                }
            }
        }
}

template <class LA, class LB>
cudaError_t gemm(LA A, LB Bt, int M, int N, int K, float* C, int ldc, int splits, cudaStream_t st) {
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    splits = max(1, splits);
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + 15) & ~15;
    splits = (K + kchunk - 1) / kchunk;
    const dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64), (unsigned)splits);
    gemm_kernel<<<grid, 128, 0, st>>>(A, Bt, M, N, K, C, ldc, kchunk, splits > 1 ? 1 : 0, (size_t)0);
    return cudaGetLastError();
}

// The forward's GEMMs: K split over enough blocks to fill the GPU when M is
// small (at least 64 of K per split, and no more partial slices than the
// scratch `cap` floats hold), each split storing its own M x N slice of C;
// `used` returns the slice count for the reduction that follows.
template <class LA, class LB>
cudaError_t gemm_sliced(LA A, LB Bt, int M, int N, int K, float* C, size_t cap, int& used, cudaStream_t st) {
    used = 1;
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    const int blocks = ((N + 63) / 64) * ((M + 63) / 64);
    int splits = (2 * 148 + blocks - 1) / blocks;
    splits = min(splits, max(1, K / 64));
    splits = (int)min((size_t)splits, max((size_t)1, cap / ((size_t)M * N)));
    splits = max(1, splits);
    int kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + 15) & ~15;
    splits = (K + kchunk - 1) / kchunk;
    used = splits;
    const dim3 grid((unsigned)((N + 63) / 64), (unsigned)((M + 63) / 64), (unsigned)splits);
    gemm_kernel<<<grid, 128, 0, st>>>(A, Bt, M, N, K, C, N, kchunk, 0, (size_t)M * N);
    return cudaGetLastError();
}

// y[M x C] (the sum of `slices` partial M x C slices, in slice order) +
// bias -> bf16 activation (ReLU) or, with out32, FP32 output.
__global__ void bias_act_kernel(const float* __restrict__ y, const float* __restrict__ bias, int M, int C,
                                uint16_t* act, float* out32, int slices) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)M * C) return;
    float t = y[i];
    for (int z = 1; z < slices; ++z) t = __fadd_rn(t, y[(size_t)z * M * C + i]);
    const float v = __fadd_rn(t, bias[i % C]);
    if (out32)
        out32[i] = v;
    else
        act[i] = to_bf16(fmaxf(v, 0.0f));
}

// d *= (activation > 0): the ReLU's derivative.
__global__ void relu_back_kernel(float* d, const uint16_t* __restrict__ act, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && !(from_bf16(act[i]) > 0.0f)) d[i] = 0.0f;
}

// out[c] += sum over rows of d[m * C + c] (bias gradients): a block per
// (column group of 32, row slice); the block sums its slice and adds once.
__global__ void col_sum_kernel(const float* __restrict__ d, int M, int C, int rows_per_block, float* out) {
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31), ty = threadIdx.x >> 5;
    const int r0 = blockIdx.y * rows_per_block, r1 = min(M, r0 + rows_per_block);
    float s = 0.0f;
    if (c < C)
        for (int r = r0 + ty; r < r1; r += 8) s += d[(size_t)r * C + c];
    part[ty][threadIdx.x & 31] = s;
    __syncthreads();
    if (ty == 0 && c < C) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += part[k][threadIdx.x];
        atomicAdd(&out[c], t);
    }
}

// The adjoint of the 3x3 stride-2 window gather: dx[b, y, x, c] = sum of
// dcol[(b, i, j), (kh, kw, c)] over the windows that read (y, x).
__global__ void col2im_kernel(const float* __restrict__ dcol, int B, int H, int W, int C, float* dx) {
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)B * H * W * C) return;
    const int c = (int)(idx % C);
    size_t r = idx / C;
    const int x = (int)(r % W);
    r /= W;
    const int y = (int)(r % H);
    const int b = (int)(r / H);
    const int Ho = H >> 1, Wo = W >> 1, K = 9 * C;
    float s = 0.0f;
    for (int kh = 0; kh < 3; ++kh) {
        const int yy = y + 1 - kh;
        if (yy < 0 || (yy & 1) || (yy >> 1) >= Ho) continue;
        for (int kw = 0; kw < 3; ++kw) {
            const int xx = x + 1 - kw;
            if (xx < 0 || (xx & 1) || (xx >> 1) >= Wo) continue;
            const size_t m = ((size_t)b * Ho + (yy >> 1)) * Wo + (xx >> 1);
            s += dcol[m * K + (kh * 3 + kw) * C + c];
        }
    }
    dx[idx] = s;
}

// The loss points: a 3x3 grid at -24, 0, 24 patch pixels.
__constant__ float kLossPts[9][2] = {{-24, -24}, {0, -24}, {24, -24}, {-24, 0}, {0, 0},
                                     {24, 0},    {-24, 24}, {0, 24},  {24, 24}};

__global__ void loss_kernel(const float* __restrict__ out, const float* __restrict__ target, int B, float* loss,
                            float* gout) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (b < B) {
        float d[6];
        for (int k = 0; k < 6; ++k) d[k] = out[b * 6 + k] - target[b * 6 + k];
        const float n = (float)(B * 9);
        float g[6] = {0, 0, 0, 0, 0, 0};
        for (int q = 0; q < 9; ++q) {
            const float px = kLossPts[q][0], py = kLossPts[q][1];
            const float ex = d[0] * px + d[1] * py + kPpTScale * d[4];
            const float ey = d[2] * px + d[3] * py + kPpTScale * d[5];
            l += ex * ex + ey * ey;
            g[0] += 2.0f * ex * px;
            g[1] += 2.0f * ex * py;
            g[4] += 2.0f * ex * kPpTScale;
            g[2] += 2.0f * ey * px;
            g[3] += 2.0f * ey * py;
            g[5] += 2.0f * ey * kPpTScale;
        }
        for (int k = 0; k < 6; ++k) gout[b * 6 + k] = g[k] / n;
        l /= n;
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

__global__ void adam_kernel(float* p, const float* __restrict__ g, float* m, float* v, size_t n, float lr, float b1t,
                            float b2t) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / (1.0f - b1t), vh = vi / (1.0f - b2t);
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

// A counter-based generator: uniform [0, 1) from (seed, a, b).
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float uni(uint64_t seed, uint64_t a, uint64_t b) {
    const uint64_t z = mix64(seed ^ mix64(a * 0x100000001b3ull + b));
    return (float)(z >> 40) * (1.0f / 16777216.0f);
}
__device__ __forceinline__ float gauss(uint64_t seed, uint64_t a, uint64_t b) {
    const float u1 = fmaxf(uni(seed, a, 2 * b), 1e-7f), u2 = uni(seed, a, 2 * b + 1);
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

__device__ __forceinline__ float bilinear(const float* S, int W, int H, float x, float y) {
    x = fminf(fmaxf(x, 0.0f), (float)(W - 1));
    y = fminf(fmaxf(y, 0.0f), (float)(H - 1));
    const int x0 = min((int)x, W - 2), y0 = min((int)y, H - 2);
    const float fx = x - (float)x0, fy = y - (float)y0;
    const float* r0 = S + (size_t)y0 * W + x0;
    const float* r1 = r0 + W;
    return (1.0f - fy) * ((1.0f - fx) * r0[0] + fx * r0[1]) + fy * ((1.0f - fx) * r1[0] + fx * r1[1]);
}

// Normalise the block's two 64x64 channels (v[2][4096] in shared memory) to
// zero mean and unit deviation and store them as bf16 NHWC.
__device__ void normalise_store(float (*v)[4096], uint16_t* x) {
    __shared__ float red[2][2][8];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int ch = 0; ch < 2; ++ch) {
        float s = 0.0f, q = 0.0f;
        for (int i = tid; i < 4096; i += 256) {
            s += v[ch][i];
            q += v[ch][i] * v[ch][i];
        }
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
        }
        if (lane == 0) {
            red[ch][0][warp] = s;
            red[ch][1][warp] = q;
        }
    }
    __syncthreads();
    float mean[2], inv[2];
    for (int ch = 0; ch < 2; ++ch) {
        float s = 0.0f, q = 0.0f;
        for (int w = 0; w < 8; ++w) {
            s += red[ch][0][w];
            q += red[ch][1][w];
        }
        mean[ch] = s / 4096.0f;
        const float var = fmaxf(q / 4096.0f - mean[ch] * mean[ch], 0.0f);
        inv[ch] = 1.0f / (sqrtf(var) + 1e-3f);
    }
    for (int i = tid; i < 4096; i += 256) {
        x[2 * i] = to_bf16((v[0][i] - mean[0]) * inv[0]);
        x[2 * i + 1] = to_bf16((v[1][i] - mean[1]) * inv[1]);
    }
}

__global__ void __launch_bounds__(256) synth_kernel(const float* __restrict__ S, int W, int H, PpSynth cfg,
                                                    uint64_t seed, uint16_t* x, float* target) {
    extern __shared__ float vbuf[];
    float(*v)[4096] = reinterpret_cast<float(*)[4096]>(vbuf);
    const int k = blockIdx.x, f = cfg.f;
    const float th = uni(seed, k, 0) * cfg.max_rot;
    const float sx = 1.0f + (2.0f * uni(seed, k, 1) - 1.0f) * cfg.max_stretch;
    const float sy = 1.0f + (2.0f * uni(seed, k, 2) - 1.0f) * cfg.max_stretch;
    const float sh = (2.0f * uni(seed, k, 3) - 1.0f) * cfg.max_shear;
    const float tx = (2.0f * uni(seed, k, 4) - 1.0f) * cfg.max_shift;
    const float ty = (2.0f * uni(seed, k, 5) - 1.0f) * cfg.max_shift;
    const float cs = cosf(th), sn = sinf(th);
    // A = R(th) [[sx, sh], [0, sy]]
    const float a00 = cs * sx, a01 = cs * sh - sn * sy, a10 = sn * sx, a11 = sn * sh + cs * sy;
    const float det = a00 * a11 - a01 * a10;
    const float i00 = a11 / det, i01 = -a01 / det, i10 = -a10 / det, i11 = a00 / det;
    const float reach = 32.0f * f * 1.4143f * (1.0f + cfg.max_stretch + cfg.max_shear) + cfg.max_shift + 4.0f;
    const float cx = floorf(reach + uni(seed, k, 6) * ((float)W - 2.0f * reach));
    const float cy = floorf(reach + uni(seed, k, 7) * ((float)H - 2.0f * reach));
    const float ox = cx - 0.5f, oy = cy - 0.5f;  // the patches' common origin
    const float inv_f2 = 1.0f / (float)(f * f);
    for (int i = threadIdx.x; i < 4096; i += 256) {
        const int u = i & 63, w = i >> 6;
        float r = 0.0f, d = 0.0f;
        for (int sj = 0; sj < f; ++sj)
            for (int si = 0; si < f; ++si) {
                const float px = cx + (float)(f * (u - 32) + si), py = cy + (float)(f * (w - 32) + sj);
                r += S[(size_t)py * W + (size_t)px];
                const float qx = px - ox - tx, qy = py - oy - ty;
                const float X = ox + i00 * qx + i01 * qy, Y = oy + i10 * qx + i11 * qy;
                d += bilinear(S, W, H, X, Y) +
                     cfg.noise * gauss(seed ^ 0x5bd1e995ull, k, (uint64_t)i * 64 + sj * 8 + si);
            }
        v[0][i] = r * inv_f2;
        v[1][i] = d * inv_f2;
    }
    __syncthreads();
    normalise_store(v, x + (size_t)k * 8192);
    if (threadIdx.x == 0) {
        float* t6 = target + (size_t)k * 6;
        t6[0] = a00 - 1.0f;
        t6[1] = a01;
        t6[2] = a10;
        t6[3] = a11 - 1.0f;
        t6[4] = tx / (float)f / kPpTScale;
        t6[5] = ty / (float)f / kPpTScale;
    }
}

__device__ __forceinline__ float px_clamped(const uint8_t* im, int W, int H, int pitch, int x, int y) {
    x = min(max(x, 0), W - 1);
    y = min(max(y, 0), H - 1);
    return (float)im[(size_t)y * pitch + x];
}

__global__ void __launch_bounds__(256) cut_kernel(const uint8_t* __restrict__ ref, const uint8_t* __restrict__ def,
                                                  int W, int H, int pitch, const float* __restrict__ centres, int f,
                                                  uint16_t* x) {
    extern __shared__ float vbuf[];
    float(*v)[4096] = reinterpret_cast<float(*)[4096]>(vbuf);
    const int k = blockIdx.x;
    const int ax = (int)centres[4 * k], ay = (int)centres[4 * k + 1];
    const int bx = (int)centres[4 * k + 2], by = (int)centres[4 * k + 3];
    const float inv_f2 = 1.0f / (float)(f * f);
    for (int i = threadIdx.x; i < 4096; i += 256) {
        const int u = i & 63, w = i >> 6;
        float r = 0.0f, d = 0.0f;
        for (int sj = 0; sj < f; ++sj)
            for (int si = 0; si < f; ++si) {
                const int dx = f * (u - 32) + si, dy = f * (w - 32) + sj;
                r += px_clamped(ref, W, H, pitch, ax + dx, ay + dy);
                d += px_clamped(def, W, H, pitch, bx + dx, by + dy);
            }
        v[0][i] = r * inv_f2;
        v[1][i] = d * inv_f2;
    }
    __syncthreads();
    normalise_store(v, x + (size_t)k * 8192);
}

__device__ __forceinline__ float bilinear_u8(const uint8_t* im, int W, int H, int pitch, float x, float y) {
    x = fminf(fmaxf(x, 0.0f), (float)(W - 1));
    y = fminf(fmaxf(y, 0.0f), (float)(H - 1));
    const int x0 = min((int)x, W - 2), y0 = min((int)y, H - 2);
    const float fx = x - (float)x0, fy = y - (float)y0;
    const uint8_t* r0 = im + (size_t)y0 * pitch + x0;
    const uint8_t* r1 = r0 + pitch;
    return (1.0f - fy) * ((1.0f - fx) * r0[0] + fx * r0[1]) + fy * ((1.0f - fx) * r1[0] + fx * r1[1]);
}

// Pair blockIdx.x's patch pixels blockIdx.y * 256 + threadIdx.x, before
// normalisation, into v32 [B][2][4096].
__global__ void __launch_bounds__(256) cut_warped_kernel(const uint8_t* __restrict__ ref,
                                                         const uint8_t* __restrict__ def, int W, int H, int pitch,
                                                         const float* __restrict__ maps, int f, float* v32) {
    const int k = blockIdx.x;
    const float* m = maps + 8 * k;
    const int ax = (int)m[0], ay = (int)m[1];
    const float inv_f2 = 1.0f / (float)(f * f);
    const int i = blockIdx.y * 256 + threadIdx.x;
    const int u = i & 63, w = i >> 6;
    float r = 0.0f, d = 0.0f;
    for (int sj = 0; sj < f; ++sj)
        for (int si = 0; si < f; ++si) {
            const int X = ax + f * (u - 32) + si, Y = ay + f * (w - 32) + sj;
            r += px_clamped(ref, W, H, pitch, X, Y);
            const float xd = m[2] * (float)X + m[3] * (float)Y + m[6];
            const float yd = m[4] * (float)X + m[5] * (float)Y + m[7];
            d += bilinear_u8(def, W, H, pitch, xd, yd);
        }
    v32[(size_t)k * 8192 + i] = r * inv_f2;
    v32[(size_t)k * 8192 + 4096 + i] = d * inv_f2;
}

// One block per pair: its two channels of v32 normalised into x.
__global__ void __launch_bounds__(256) normalise_kernel(const float* __restrict__ v32, uint16_t* x) {
    const int k = blockIdx.x;
    normalise_store(reinterpret_cast<float(*)[4096]>(const_cast<float*>(v32 + (size_t)k * 8192)),
                    x + (size_t)k * 8192);
}

inline unsigned nblocks(size_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

int dw_splits(int K) { return max(1, min(256, (K + 2047) / 2048)); }

cudaError_t col_sum(const float* d, int M, int C, float* out, cudaStream_t st) {
    const int rows = 1024;
    const dim3 grid((unsigned)((C + 31) / 32), (unsigned)((M + rows - 1) / rows));
    col_sum_kernel<<<grid, 256, 0, st>>>(d, M, C, rows, out);
    return cudaGetLastError();
}

constexpr size_t kActElems[6] = {8192, 16384, 8192, 4096, 2048, 512};  // per pair, per layer
constexpr size_t kScratchElems = 36864;  // per pair: the largest column matrix (layer 2's input gradient)

}  // namespace

size_t pp_work_bytes(int B) {
    size_t b = 0;
    for (int l = 0; l < 6; ++l) b += align256(kActElems[l] * B * 2);
    b += align256((size_t)B * kPpFc1 * 2);
    b += 2 * align256(kScratchElems * B * 4);
    b += 2 * align256((size_t)B * 6 * 4);
    b += align256(4);
    return b;
}

void pp_work_carve(PpWork& w, void* base, int B) {
    char* p = static_cast<char*>(base);
    w.max_batch = B;
    for (int l = 0; l < 6; ++l) {
        w.act[l] = reinterpret_cast<uint16_t*>(p);
        p += align256(kActElems[l] * B * 2);
    }
    w.h = reinterpret_cast<uint16_t*>(p);
    p += align256((size_t)B * kPpFc1 * 2);
    w.y = reinterpret_cast<float*>(p);
    p += align256(kScratchElems * B * 4);
    w.dy = reinterpret_cast<float*>(p);
    p += align256(kScratchElems * B * 4);
    w.out = reinterpret_cast<float*>(p);
    p += align256((size_t)B * 6 * 4);
    w.gout = reinterpret_cast<float*>(p);
    p += align256((size_t)B * 6 * 4);
    w.loss = reinterpret_cast<float*>(p);
}

cudaError_t pp_forward(const float* params, PpWork& w, int B, cudaStream_t st) {
    if (B <= 0 || B > w.max_batch) return cudaErrorInvalidValue;
    const PpLayout L = pp_layout();
    const size_t cap = kScratchElems * (size_t)w.max_batch;
    cudaError_t e;
    int sl = 1;
    for (int l = 0; l < 5; ++l) {
        const int Hs = kPpSide >> l, Ci = kPpChannels[l], Co = kPpChannels[l + 1];
        const int M = B * (Hs / 2) * (Hs / 2), K = 9 * Ci;
        e = gemm_sliced(LdIm2Col<false>{w.act[l], Hs, Hs, Ci}, LdF32Row{params + L.w[l], K}, M, Co, K, w.y, cap, sl,
                        st);
        if (e != cudaSuccess) return e;
        bias_act_kernel<<<nblocks((size_t)M * Co), 256, 0, st>>>(w.y, params + L.b[l], M, Co, w.act[l + 1], nullptr,
                                                                 sl);
    }
    e = gemm_sliced(LdBfRow{w.act[5], kPpFc0}, LdF32Row{params + L.w[5], kPpFc0}, B, kPpFc1, kPpFc0, w.y, cap, sl, st);
    if (e != cudaSuccess) return e;
    bias_act_kernel<<<nblocks((size_t)B * kPpFc1), 256, 0, st>>>(w.y, params + L.b[5], B, kPpFc1, w.h, nullptr, sl);
    e = gemm_sliced(LdBfRow{w.h, kPpFc1}, LdF32Row{params + L.w[6], kPpFc1}, B, kPpOut, kPpFc1, w.y, cap, sl, st);
    if (e != cudaSuccess) return e;
    bias_act_kernel<<<nblocks((size_t)B * kPpOut), 256, 0, st>>>(w.y, params + L.b[6], B, kPpOut, nullptr, w.out, sl);
    return cudaGetLastError();
}

cudaError_t pp_loss(PpWork& w, const float* target, int B, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(w.loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return e;
    loss_kernel<<<nblocks((size_t)B, 128), 128, 0, st>>>(w.out, target, B, w.loss, w.gout);
    return cudaGetLastError();
}

cudaError_t pp_backward(const float* params, PpWork& w, int B, float* grads, cudaStream_t st) {
    if (B <= 0 || B > w.max_batch) return cudaErrorInvalidValue;
    const PpLayout L = pp_layout();
    cudaError_t e = cudaMemsetAsync(grads, 0, L.total * sizeof(float), st);
    if (e != cudaSuccess) return e;
    float* S1 = w.y;
    float* S2 = w.dy;
    // output layer
    e = gemm(LdF32Col{w.gout, kPpOut}, LdBfCol{w.h, kPpFc1}, kPpOut, kPpFc1, B, grads + L.w[6], kPpFc1, dw_splits(B),
             st);
    if (e != cudaSuccess) return e;
    if ((e = col_sum(w.gout, B, kPpOut, grads + L.b[6], st)) != cudaSuccess) return e;
    e = gemm(LdF32Row{w.gout, kPpOut}, LdF32Col{params + L.w[6], kPpFc1}, B, kPpFc1, kPpOut, S1, kPpFc1, 1, st);
    if (e != cudaSuccess) return e;
    relu_back_kernel<<<nblocks((size_t)B * kPpFc1), 256, 0, st>>>(S1, w.h, (size_t)B * kPpFc1);
    if ((e = col_sum(S1, B, kPpFc1, grads + L.b[5], st)) != cudaSuccess) return e;
    e = gemm(LdF32Col{S1, kPpFc1}, LdBfCol{w.act[5], kPpFc0}, kPpFc1, kPpFc0, B, grads + L.w[5], kPpFc0,
             dw_splits(B), st);
    if (e != cudaSuccess) return e;
    e = gemm(LdF32Row{S1, kPpFc1}, LdF32Col{params + L.w[5], kPpFc0}, B, kPpFc0, kPpFc1, S2, kPpFc0, 1, st);
    if (e != cudaSuccess) return e;
    // convolutions, last to first; the gradient w.r.t. a layer's output is in S2
    for (int l = 4; l >= 0; --l) {
        const int Hs = kPpSide >> l, Ci = kPpChannels[l], Co = kPpChannels[l + 1];
        const int M = B * (Hs / 2) * (Hs / 2), K = 9 * Ci;
        relu_back_kernel<<<nblocks((size_t)M * Co), 256, 0, st>>>(S2, w.act[l + 1], (size_t)M * Co);
        if ((e = col_sum(S2, M, Co, grads + L.b[l], st)) != cudaSuccess) return e;
        e = gemm(LdF32Col{S2, Co}, LdIm2Col<true>{w.act[l], Hs, Hs, Ci}, Co, K, M, grads + L.w[l], K, dw_splits(M),
                 st);
        if (e != cudaSuccess) return e;
        if (l == 0) break;
        e = gemm(LdF32Row{S2, Co}, LdF32Col{params + L.w[l], K}, M, K, Co, S1, K, 1, st);
        if (e != cudaSuccess) return e;
        col2im_kernel<<<nblocks((size_t)B * Hs * Hs * Ci), 256, 0, st>>>(S1, B, Hs, Hs, Ci, S2);
    }
    return cudaGetLastError();
}

cudaError_t pp_adam(float* params, const float* grads, float* m, float* v, size_t n, int t, float lr,
                    cudaStream_t st) {
    const float b1t = powf(0.9f, (float)t), b2t = powf(0.999f, (float)t);
    adam_kernel<<<nblocks(n), 256, 0, st>>>(params, grads, m, v, n, lr, b1t, b2t);
    return cudaGetLastError();
}

cudaError_t pp_synth_pairs(const float* S, int W, int H, const PpSynth& cfg, uint64_t seed, int B, uint16_t* x,
                           float* target, cudaStream_t st) {
    if (B <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(synth_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 4096 * 4);
    if (e != cudaSuccess) return e;
    synth_kernel<<<B, 256, 2 * 4096 * 4, st>>>(S, W, H, cfg, seed, x, target);
    return cudaGetLastError();
}

cudaError_t pp_cut_pairs(const uint8_t* ref, const uint8_t* def, int W, int H, int pitch, const float* centres,
                         int B, int f, uint16_t* x, cudaStream_t st) {
    if (B <= 0) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(cut_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 2 * 4096 * 4);
    if (e != cudaSuccess) return e;
    cut_kernel<<<B, 256, 2 * 4096 * 4, st>>>(ref, def, W, H, pitch, centres, f, x);
    return cudaGetLastError();
}

cudaError_t pp_cut_warped(const uint8_t* ref, const uint8_t* def, int W, int H, int pitch, const float* maps, int B,
                          int f, uint16_t* x, float* scratch, cudaStream_t st) {
    if (B <= 0) return cudaSuccess;
    cut_warped_kernel<<<dim3((unsigned)B, 16), 256, 0, st>>>(ref, def, W, H, pitch, maps, f, scratch);
    normalise_kernel<<<B, 256, 0, st>>>(scratch, x);
    return cudaGetLastError();
}

}  // namespace dic
