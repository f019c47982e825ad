// Seeded synthetic speckle pairs for the benchmark configurations, the tests
// and the proposal network's training data.
//
// The pattern is an analytic sum of Gaussian blobs,
//     g(X) = background + sum_b A_b exp(-|X - c_b|^2 / (2 s_b^2))   (|X - c_b| <= 5 s_b),
// blob centres uniform over the image at a given density, s ~ U[s0, s1],
// A ~ U[a0, a1] (std::mt19937_64 from the pair's seed, in that draw order),
// clipped to 0..255 and rounded as floor(v + 0.5). A deformed frame samples g
// at the exact inverse of the forward map x = X + U(X) (Newton), adds
// N(0, sigma^2) gray-level noise from its own seed, and rounds the same way.
//
// U is a sum of an affine part about a centre, two sinusoids, and Fourier
// modes (a smooth random field):
//   U(X) = t + A (X - c) + [su sin(2 pi Y / Lu), sv sin(2 pi X / Lv)]
//          + sum_k [au_k, av_k] cos(kx_k X + ky_k Y + ph_k)
// The parameter block is documented at synth_warp_params below.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#define SYNTH_API extern "C" __attribute__((visibility("default")))

namespace {

struct Blobs {
    std::vector<float> cx, cy, inv2s2, amp, r2max;
    int bw = 0, bh = 0;
    float cell = 16.0f;
    std::vector<int> start, idx;
};

Blobs make_blobs(int w, int h, uint64_t seed, double density, double s0, double s1, double a0, double a1) {
    Blobs B;
    std::mt19937_64 rng(seed);
    std::uniform_real_distribution<double> ux(0.0, (double)w), uy(0.0, (double)h), us(s0, s1), ua(a0, a1);
    const long n = std::lround(density * (double)w * (double)h);
    for (long i = 0; i < n; ++i) {
        const double x = ux(rng), y = uy(rng), s = us(rng), a = ua(rng);
        B.cx.push_back((float)x);
        B.cy.push_back((float)y);
        B.inv2s2.push_back((float)(1.0 / (2.0 * s * s)));
        B.amp.push_back((float)a);
        B.r2max.push_back((float)(25.0 * s * s));
    }
    B.cell = (float)std::max(8.0, std::ceil(5.0 * s1));
    B.bw = (int)std::ceil(w / B.cell) + 1;
    B.bh = (int)std::ceil(h / B.cell) + 1;
    std::vector<int> cnt((size_t)B.bw * B.bh, 0), cellof(B.cx.size());
    for (size_t i = 0; i < B.cx.size(); ++i) {
        const int bx = std::min(B.bw - 1, std::max(0, (int)(B.cx[i] / B.cell)));
        const int by = std::min(B.bh - 1, std::max(0, (int)(B.cy[i] / B.cell)));
        cellof[i] = by * B.bw + bx;
        cnt[cellof[i]]++;
    }
    B.start.assign(cnt.size() + 1, 0);
    for (size_t c = 0; c < cnt.size(); ++c) B.start[c + 1] = B.start[c] + cnt[c];
    std::vector<int> fill(B.start.begin(), B.start.end() - 1);
    B.idx.assign(B.cx.size(), 0);
    for (size_t i = 0; i < B.cx.size(); ++i) B.idx[fill[cellof[i]]++] = (int)i;
    return B;
}

// g at (x, y); blobs summed in index order within the 3x3 cells around the point.
double eval(const Blobs& B, double bg, double x, double y) {
    const int qx = (int)std::floor(x / B.cell), qy = (int)std::floor(y / B.cell);
    int ids[512];
    int n = 0;
    for (int by = std::max(qy - 1, 0); by <= std::min(qy + 1, B.bh - 1); ++by)
        for (int bx = std::max(qx - 1, 0); bx <= std::min(qx + 1, B.bw - 1); ++bx) {
            const int c = by * B.bw + bx;
            for (int k = B.start[c]; k < B.start[c + 1] && n < 512; ++k) ids[n++] = B.idx[k];
        }
    std::sort(ids, ids + n);
    double v = bg;
    for (int k = 0; k < n; ++k) {
        const int i = ids[k];
        const double dx = x - B.cx[i], dy = y - B.cy[i];
        const double r2 = dx * dx + dy * dy;
        if (r2 <= B.r2max[i]) v += B.amp[i] * std::exp(-r2 * B.inv2s2[i]);
    }
    return v;
}

struct Warp {
    double cx, cy, u0, v0, a00, a01, a10, a11, su, Lu, sv, Lv;
    std::vector<double> modes;  // 5 per mode: kx ky au av ph
    void U(double X, double Y, double& u, double& v, double J[4]) const {
        const double dx = X - cx, dy = Y - cy;
        u = u0 + a00 * dx + a01 * dy;
        v = v0 + a10 * dx + a11 * dy;
        J[0] = a00; J[1] = a01; J[2] = a10; J[3] = a11;
        if (su != 0.0 && Lu != 0.0) {
            const double k = 2.0 * M_PI / Lu;
            u += su * std::sin(k * Y);
            J[1] += su * k * std::cos(k * Y);
        }
        if (sv != 0.0 && Lv != 0.0) {
            const double k = 2.0 * M_PI / Lv;
            v += sv * std::sin(k * X);
            J[2] += sv * k * std::cos(k * X);
        }
        for (size_t m = 0; m + 4 < modes.size(); m += 5) {
            const double kx = modes[m], ky = modes[m + 1], au = modes[m + 2], av = modes[m + 3], ph = modes[m + 4];
            const double arg = kx * X + ky * Y + ph, c = std::cos(arg), s = std::sin(arg);
            u += au * c;
            v += av * c;
            J[0] -= au * s * kx; J[1] -= au * s * ky;
            J[2] -= av * s * kx; J[3] -= av * s * ky;
        }
    }
    // X with X + U(X) = (qx, qy).
    void inverse(double qx, double qy, double& X, double& Y) const {
        double u, v, J[4];
        U(qx, qy, u, v, J);
        X = qx - u;
        Y = qy - v;
        for (int it = 0; it < 20; ++it) {
            U(X, Y, u, v, J);
            const double fx = X + u - qx, fy = Y + v - qy;
            const double j00 = 1.0 + J[0], j01 = J[1], j10 = J[2], j11 = 1.0 + J[3];
            const double det = j00 * j11 - j01 * j10;
            if (!(std::fabs(det) > 1e-12)) break;
            const double dX = (j11 * fx - j01 * fy) / det, dY = (-j10 * fx + j00 * fy) / det;
            X -= dX;
            Y -= dY;
            if (std::fabs(dX) + std::fabs(dY) < 1e-10) break;
        }
    }
};

Warp parse(const double* p) {
    Warp w{};
    if (!p) {
        w.a00 = w.a01 = w.a10 = w.a11 = 0.0;
        return w;
    }
    w.cx = p[0]; w.cy = p[1]; w.u0 = p[2]; w.v0 = p[3];
    w.a00 = p[4]; w.a01 = p[5]; w.a10 = p[6]; w.a11 = p[7];
    w.su = p[8]; w.Lu = p[9]; w.sv = p[10]; w.Lv = p[11];
    const int nm = (int)p[12];
    w.modes.assign(p + 13, p + 13 + 5 * nm);
    return w;
}

uint8_t quant(double v) {
    if (v < 0.0) v = 0.0;
    if (v > 255.0) v = 255.0;
    return (uint8_t)std::floor(v + 0.5);
}

}  // namespace

// Parameter block of a warp (doubles):
//   [0..1] centre cx, cy          [2..3] translation u0, v0
//   [4..7] affine a00 a01 a10 a11 (U = t + A (X - c))
//   [8..11] su, Lu, sv, Lv        (u += su sin(2 pi Y / Lu), v += sv sin(2 pi X / Lv))
//   [12] number of Fourier modes, then 5 doubles each: kx ky au av ph
// A null block is the identity (the reference frame).
//
// Writes one w x h frame of the speckle of (seed, density, sigma range,
// amplitude range, background) under the warp, with N(0, noise^2) noise from
// noise_seed (row r uses its own generator seeded noise_seed * 1000003 + r).
SYNTH_API int synth_speckle(uint8_t* out, int w, int h, uint64_t seed, double density, double s0, double s1,
                            double a0, double a1, double bg, const double* warp, double noise, uint64_t noise_seed) {
    if (!out || w <= 0 || h <= 0) return -1;
    const Blobs B = make_blobs(w, h, seed, density, s0, s1, a0, a1);
    const Warp W = parse(warp);
#pragma omp parallel for schedule(dynamic, 8)
    for (int y = 0; y < h; ++y) {
        std::mt19937_64 rng(noise_seed * 1000003ull + (uint64_t)y);
        std::normal_distribution<double> nd(0.0, noise > 0.0 ? noise : 1.0);
        for (int x = 0; x < w; ++x) {
            double X = x, Y = y;
            if (warp) W.inverse(x, y, X, Y);
            double v = eval(B, bg, X, Y);
            if (noise > 0.0) v += nd(rng);
            out[(size_t)y * w + x] = quant(v);
        }
    }
    return 0;
}

// The displacement U at reference points (X, Y) under a warp (truth for tests).
SYNTH_API void synth_displacement(const double* warp, int n, const double* X, const double* Y, double* u, double* v) {
    const Warp W = parse(warp);
    for (int i = 0; i < n; ++i) {
        double J[4];
        W.U(X[i], Y[i], u[i], v[i], J);
    }
}
