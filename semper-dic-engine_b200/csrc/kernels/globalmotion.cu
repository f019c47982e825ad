// Global motion by phase correlation (see globalmotion.cuh).
//
// 1. Both ROIs are box-downsampled by f = ceil(max(rw, rh) / N) into an N x N
//    frame (centred), the mean removed and a Hann window applied.
// 2. Rotation and scale: the magnitude spectra (high-pass weighted, centred)
//    are resampled on a log-polar grid (angle over [0, pi), log radius); a
//    rotation of the image is a shift along the angle axis there, a scale a
//    shift along log radius. Phase correlation of the two maps gives both.
// 3. Translation: the deformed ROI resampled through the similarity (for the
//    angle and the angle + pi, which the magnitude spectrum cannot tell
//    apart) is phase-correlated with the reference ROI; the higher peak
//    decides the angle and gives the translation.
// The FFTs are radix-2 Stockham transforms in shared memory (one block per
// row; a 2-D transform is rows, transpose, rows, which leaves a forward
// spectrum transposed and an inverse one in natural order).
#include "globalmotion.cuh"

#include <algorithm>
#include <cmath>
#include <utility>

namespace dic {

namespace {

constexpr int N = GlobalMotion::kN;
constexpr double kPi = 3.14159265358979323846;
constexpr double kMinPeakRotation = 0.05;
constexpr double kMinPeakTranslation = 0.08;
constexpr int kPartials = (N / 128) * N;  // one per block of a 128-wide row slice

// box average of f x f source pixels per output pixel, the region centred in
// the N x N frame; each block leaves the sum of its outputs in partial[] (a
// fixed-order reduction, so the mean is the same on every run)
__global__ void __launch_bounds__(128) downsample_kernel(const uint8_t* __restrict__ img, int W, int rx, int ry,
                                                         int f, int dw, int dh, int ox, int oy,
                                                         float* __restrict__ out, double* __restrict__ partial) {
    __shared__ double ws[4];
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    float v = 0.0f;
    if (x >= ox && x < ox + dw && y >= oy && y < oy + dh) {
        const int sx = rx + (x - ox) * f, sy = ry + (y - oy) * f;
        unsigned acc = 0;
        for (int j = 0; j < f; ++j)
            for (int i = 0; i < f; ++i) acc += img[(size_t)(sy + j) * W + sx + i];
        v = (float)acc / (float)(f * f);
    }
    out[(size_t)y * N + x] = v;
    double s = v;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = ((ws[0] + ws[1]) + ws[2]) + ws[3];
}

// *sum = the count partials added in a fixed order (one block of 256)
__global__ void __launch_bounds__(256) sum_kernel(const double* __restrict__ partial, int count,
                                                  double* __restrict__ sum) {
    __shared__ double ws[8];
    double s = 0.0;
    for (int i = threadIdx.x; i < count; i += 256) s += partial[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += ws[w];
        *sum = t;
    }
}

// mean removed and the Hann window applied inside the region; complex out
__global__ void window_kernel(float* __restrict__ img, const double* __restrict__ sum, int dw, int dh, int ox, int oy,
                              float2* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= N) return;
    float v = 0.0f;
    if (x >= ox && x < ox + dw && y >= oy && y < oy + dh) {
        const float mean = (float)(*sum / ((double)dw * dh));
        const float wx = dw > 1 ? 0.5f - 0.5f * cospif(2.0f * (x - ox) / (float)(dw - 1)) : 1.0f;
        const float wy = dh > 1 ? 0.5f - 0.5f * cospif(2.0f * (y - oy) / (float)(dh - 1)) : 1.0f;
        v = (img[(size_t)y * N + x] - mean) * wx * wy;
    }
    img[(size_t)y * N + x] = v;
    out[(size_t)y * N + x] = make_float2(v, 0.0f);
}

// In-place 1-D transform of each row (one block of N/2 threads per row):
// radix-2 Stockham, log2(N) passes between two shared-memory buffers, each
// thread one butterfly per pass, natural order out; sign -1 forward, +1
// inverse (unnormalised).
__global__ void __launch_bounds__(N / 2) fft_rows_kernel(float2* __restrict__ data, int sign) {
    __shared__ float2 buf[2][N];
    float2* row = data + (size_t)blockIdx.x * N;
    const int j = threadIdx.x;
    buf[0][j] = row[j];
    buf[0][j + N / 2] = row[j + N / 2];
    int src = 0;
    for (int ns = 1; ns < N; ns <<= 1) {
        __syncthreads();
        const float2 a = buf[src][j], b0 = buf[src][j + N / 2];
        const int k = j & (ns - 1);
        float s, c;
        sincospif((float)(sign * k) / (float)ns, &s, &c);
        const float2 b = make_float2(b0.x * c - b0.y * s, b0.x * s + b0.y * c);
        const int d = ((j - k) << 1) + k;
        buf[src ^ 1][d] = make_float2(a.x + b.x, a.y + b.y);
        buf[src ^ 1][d + ns] = make_float2(a.x - b.x, a.y - b.y);
        src ^= 1;
    }
    __syncthreads();
    row[j] = buf[src][j];
    row[j + N / 2] = buf[src][j + N / 2];
}

// out = in^T through a 32 x 32 shared tile
__global__ void transpose_kernel(const float2* __restrict__ in, float2* __restrict__ out) {
    __shared__ float2 tile[32][33];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) tile[r][threadIdx.x] = in[(size_t)(y0 + r) * N + x0 + threadIdx.x];
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) out[(size_t)(x0 + r) * N + y0 + threadIdx.x] = tile[threadIdx.x][r];
}

// centred magnitude spectrum with the high-pass weight (1 - X)(2 - X),
// X = cos(pi kx) cos(pi ky) over the centred frequencies
__global__ void magnitude_kernel(const float2* __restrict__ F, float* __restrict__ mag) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= N) return;
    const int sx = (x + N / 2) % N, sy = (y + N / 2) % N;
    const float2 c = F[(size_t)sx * N + sy];  // the spectrum is stored transposed
    const float kx = (float)(x - N / 2) / N, ky = (float)(y - N / 2) / N;
    const float X = cospif(kx) * cospif(ky);
    mag[(size_t)y * N + x] = sqrtf(c.x * c.x + c.y * c.y) * (1.0f - X) * (2.0f - X);
}

__device__ __forceinline__ float bilinear(const float* __restrict__ m, float X, float Y) {
    int x0 = (int)floorf(X), y0 = (int)floorf(Y);
    const float tx = X - x0, ty = Y - y0;
    x0 = min(max(x0, 0), N - 2);
    y0 = min(max(y0, 0), N - 2);
    const float* p = m + (size_t)y0 * N + x0;
    return p[0] * (1 - tx) * (1 - ty) + p[1] * tx * (1 - ty) + p[N] * (1 - tx) * ty + p[N + 1] * tx * ty;
}

// row a = angle pi a / N, column r = log radius r * lstep (radius 1 .. N/2 - 1)
__global__ void logpolar_kernel(const float* __restrict__ mag, float lstep, float2* __restrict__ out) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x, a = blockIdx.y;
    if (r >= N) return;
    float s, c;
    sincospif((float)a / N, &s, &c);
    const float rho = expf(r * lstep);
    const float v = bilinear(mag, N / 2 + rho * c, N / 2 + rho * s);
    out[(size_t)a * N + r] = make_float2(v, 0.0f);
}

// the deformed ROI sampled through the similarity: b'(x) = b(c + s R (x - c))
__global__ void resample_kernel(const float* __restrict__ b, float cth, float sth, float sc,
                                float2* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= N) return;
    const float dx = x - N / 2.0f, dy = y - N / 2.0f;
    const float X = N / 2.0f + sc * (cth * dx - sth * dy), Y = N / 2.0f + sc * (sth * dx + cth * dy);
    float v = 0.0f;
    if (X >= 0 && Y >= 0 && X <= N - 1 && Y <= N - 1) v = bilinear(b, X, Y);
    out[(size_t)y * N + x] = make_float2(v, 0.0f);
}

// normalised cross power a conj(b)
__global__ void cross_power_kernel(const float2* __restrict__ A, const float2* __restrict__ B,
                                   float2* __restrict__ P) {
    const size_t i = (size_t)blockIdx.y * N + blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x + threadIdx.x >= N) return;
    const float2 a = A[i], b = B[i];
    const float re = a.x * b.x + a.y * b.y, im = a.y * b.x - a.x * b.y;
    const float m = sqrtf(re * re + im * im) + 1e-20f;
    P[i] = make_float2(re / m, im / m);
}

// argmax of the real part: value bits (positive floats order as integers)
// packed above the index; the maximum over each warp first, then one atomic
// per warp (the maximum does not depend on the order)
__global__ void argmax_kernel(const float2* __restrict__ P, unsigned long long* best) {
    const size_t i = (size_t)blockIdx.y * N + blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long key = 0;
    if (blockIdx.x * blockDim.x + threadIdx.x < N) {
        const float v = P[i].x;
        if (v > 0.0f) key = ((unsigned long long)__float_as_uint(v) << 32) | (unsigned long long)i;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, o);
        key = other > key ? other : key;
    }
    if ((threadIdx.x & 31) == 0 && key) atomicMax(best, key);
}

__global__ void neighbourhood_kernel(const float2* __restrict__ P, const unsigned long long* best,
                                     float* __restrict__ out9) {
    const unsigned long long key = *best;
    const int i = (int)(key & 0xffffffffull);
    const int py = i / N, px = i % N;
    const int t = threadIdx.x;
    if (t < 9) {
        const int y = (py + t / 3 - 1 + N) % N, x = (px + t % 3 - 1 + N) % N;
        out9[t] = P[(size_t)y * N + x].x / ((float)N * N);
    }
    if (t == 0) {
        out9[9] = (float)px;
        out9[10] = (float)py;
    }
}

// the peak of P's real part with a parabolic sub-pixel offset on each axis,
// as a shift in (-N/2, N/2]
bool peak(const float* h, double& sx, double& sy, double& height) {
    const double c = h[4];
    if (!(c > 0)) return false;
    auto sub = [](double m, double cc, double p) {
        const double d = m - 2 * cc + p;
        return d == 0 ? 0.0 : 0.5 * (m - p) / d;
    };
    sx = h[9] + sub(h[3], c, h[5]);
    sy = h[10] + sub(h[1], c, h[7]);
    if (sx > N / 2) sx -= N;
    if (sy > N / 2) sy -= N;
    height = c;
    return true;
}

}  // namespace

struct GlobalMotion::Impl {
    float2 *fa = nullptr, *fb = nullptr, *tmp = nullptr, *tmp2 = nullptr, *lpa = nullptr, *lpb = nullptr;
    float *ra = nullptr, *rb = nullptr, *mag = nullptr, *h9 = nullptr;
    double *sums = nullptr, *partial = nullptr;
    unsigned long long* best = nullptr;
    bool ready = false;
    int launches = 0;
    ~Impl() {
        for (void* p : {(void*)fa, (void*)fb, (void*)tmp, (void*)tmp2, (void*)lpa, (void*)lpb, (void*)ra, (void*)rb,
                        (void*)mag, (void*)h9, (void*)sums, (void*)partial, (void*)best})
            if (p) cudaFree(p);
    }
    cudaError_t init() {
        if (ready) return cudaSuccess;
        const size_t nc = (size_t)N * N * sizeof(float2), nf = (size_t)N * N * sizeof(float);
        cudaError_t e;
        for (auto* pp : {&fa, &fb, &tmp, &tmp2, &lpa, &lpb})
            if ((e = cudaMalloc(pp, nc)) != cudaSuccess) return e;
        for (auto* pp : {&ra, &rb, &mag})
            if ((e = cudaMalloc(pp, nf)) != cudaSuccess) return e;
        if ((e = cudaMalloc(&h9, 16 * sizeof(float))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&sums, 2 * sizeof(double))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&partial, kPartials * sizeof(double))) != cudaSuccess) return e;
        if ((e = cudaMalloc(&best, sizeof(unsigned long long))) != cudaSuccess) return e;
        ready = true;
        return cudaSuccess;
    }
    // 2-D transform of `in` into `out` (in is left as scratch): rows,
    // transpose, rows
    void fft2(float2* in, float2* out, int sign, cudaStream_t st) {
        fft_rows_kernel<<<N, N / 2, 0, st>>>(in, sign);
        transpose_kernel<<<dim3(N / 32, N / 32), dim3(32, 8), 0, st>>>(in, out);
        fft_rows_kernel<<<N, N / 2, 0, st>>>(out, sign);
        launches += 3;
    }
    // the peak of the correlation of spectra A and B (a(x) = b(x - s))
    bool correlate(const float2* A, const float2* B, cudaStream_t st, double& sx, double& sy, double& height) {
        const dim3 grid(N / 128, N);
        cross_power_kernel<<<grid, 128, 0, st>>>(A, B, tmp);
        fft2(tmp, tmp2, +1, st);
        cudaMemsetAsync(best, 0, sizeof(unsigned long long), st);
        argmax_kernel<<<grid, 128, 0, st>>>(tmp2, best);
        neighbourhood_kernel<<<1, 32, 0, st>>>(tmp2, best, h9);
        launches += 3;
        float h[16];
        if (cudaMemcpyAsync(h, h9, 11 * sizeof(float), cudaMemcpyDeviceToHost, st) != cudaSuccess) return false;
        if (cudaStreamSynchronize(st) != cudaSuccess) return false;
        return peak(h, sx, sy, height);
    }
};

GlobalMotion::GlobalMotion() : impl_(new Impl()) {}
GlobalMotion::~GlobalMotion() { delete impl_; }

cudaError_t GlobalMotion::estimate(const uint8_t* d_ref, const uint8_t* d_def, int W, int H, int rx, int ry, int rw,
                                   int rh, cudaStream_t st, GlobalSimilarity& out) {
    out = GlobalSimilarity();
    if (rw < 16 || rh < 16 || rx < 0 || ry < 0 || rx + rw > W || ry + rh > H) return cudaSuccess;
    cudaError_t e = impl_->init();
    if (e != cudaSuccess) return e;
    impl_->launches = 0;
    e = estimate_impl(d_ref, d_def, W, rx, ry, rw, rh, st, out);
    out.kernels = impl_->launches;
    if (e != cudaSuccess) out.locked = false;
    return e;
}

cudaError_t GlobalMotion::estimate_impl(const uint8_t* d_ref, const uint8_t* d_def, int W, int rx, int ry, int rw,
                                        int rh, cudaStream_t st, GlobalSimilarity& out) {
    Impl& I = *impl_;
    cudaError_t e;
    const int f = std::max(1, (std::max(rw, rh) + N - 1) / N);
    const int dw = std::min(rw / f, N), dh = std::min(rh / f, N);
    const int ox = (N - dw) / 2, oy = (N - dh) / 2;
    const dim3 grid(N / 128, N);
    downsample_kernel<<<grid, 128, 0, st>>>(d_ref, W, rx, ry, f, dw, dh, ox, oy, I.ra, I.partial);
    sum_kernel<<<1, 256, 0, st>>>(I.partial, kPartials, I.sums);
    downsample_kernel<<<grid, 128, 0, st>>>(d_def, W, rx, ry, f, dw, dh, ox, oy, I.rb, I.partial);
    sum_kernel<<<1, 256, 0, st>>>(I.partial, kPartials, I.sums + 1);
    window_kernel<<<grid, 128, 0, st>>>(I.ra, I.sums, dw, dh, ox, oy, I.fa);
    window_kernel<<<grid, 128, 0, st>>>(I.rb, I.sums + 1, dw, dh, ox, oy, I.fb);
    I.launches += 6;
    I.fft2(I.fa, I.tmp, -1, st);
    std::swap(I.fa, I.tmp);
    I.fft2(I.fb, I.tmp, -1, st);
    std::swap(I.fb, I.tmp);
    // rotation and scale
    const float lstep = (float)(std::log(N / 2.0 - 1.0) / (N - 1));
    magnitude_kernel<<<grid, 128, 0, st>>>(I.fa, I.mag);
    logpolar_kernel<<<grid, 128, 0, st>>>(I.mag, lstep, I.lpa);
    magnitude_kernel<<<grid, 128, 0, st>>>(I.fb, I.mag);
    logpolar_kernel<<<grid, 128, 0, st>>>(I.mag, lstep, I.lpb);
    I.launches += 4;
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    I.fft2(I.lpa, I.tmp, -1, st);
    std::swap(I.lpa, I.tmp);
    I.fft2(I.lpb, I.tmp, -1, st);
    std::swap(I.lpb, I.tmp);
    double sr, sa, hr;
    if (!I.correlate(I.lpb, I.lpa, st, sr, sa, hr)) return cudaGetLastError();
    const double theta0 = sa * kPi / N, scale = std::exp(-sr * lstep);
    // translation, for the angle and the angle + pi
    double best_h = -1, best_t = 0, bsx = 0, bsy = 0;
    for (int k = 0; k < 2; ++k) {
        const double th = theta0 + k * kPi;
        resample_kernel<<<grid, 128, 0, st>>>(I.rb, (float)std::cos(th), (float)std::sin(th), (float)scale, I.tmp);
        ++I.launches;
        I.fft2(I.tmp, I.lpb, -1, st);
        double sx, sy, h;
        if (!I.correlate(I.lpb, I.fa, st, sx, sy, h)) continue;
        if (h > best_h) {
            best_h = h;
            best_t = th;
            bsx = sx;
            bsy = sy;
        }
    }
    if (best_h < 0) return cudaGetLastError();
    // x' = C + s R (X - C) + T in full-resolution pixels; C the ROI centre
    // the downsampled frame's centre stands for
    const double c = std::cos(best_t), s = std::sin(best_t);
    out.theta = std::atan2(s, c);
    out.scale = scale;
    out.tx = f * scale * (c * bsx - s * bsy);
    out.ty = f * scale * (s * bsx + c * bsy);
    out.cx = rx + (N / 2.0 - ox) * f + (f - 1) / 2.0;
    out.cy = ry + (N / 2.0 - oy) * f + (f - 1) / 2.0;
    out.peak_rotation = hr;
    out.peak_translation = best_h;
    out.locked = hr >= kMinPeakRotation && best_h >= kMinPeakTranslation;
    const double a00 = scale * c, a01 = -scale * s, a10 = scale * s, a11 = scale * c;
    out.H[0] = a00;
    out.H[1] = a01;
    out.H[2] = out.cx + out.tx - (a00 * out.cx + a01 * out.cy);
    out.H[3] = a10;
    out.H[4] = a11;
    out.H[5] = out.cy + out.ty - (a10 * out.cx + a11 * out.cy);
    out.H[6] = 0;
    out.H[7] = 0;
    out.H[8] = 1;
    return cudaGetLastError();
}

}  // namespace dic
