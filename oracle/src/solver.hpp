// ORACLE — test infrastructure only. Never linked into the product library.
//
// The per-subset math restated from the reference:
//   Hessian pool entry   src/math/subset_precomputer.cpp:42-149, src/math/hessian.hpp:40-52
//   subset fill          src/math/subset_precomputer.cpp:159-265
//   IC-GN                src/math/optimization_engine.cpp:272-465
//   ZNSSD / Simplex      src/math/optimization_engine.cpp:467-651
//   coarse search        src/math/optimization_engine.cpp:120-179
//   mode dispatch        src/math/optimization_engine.cpp:55-118
//   solve_node           src/pipeline/full_field_solver.cpp:119-139,
//                        src/pipeline/full_field_internal.hpp:347-365
// Deliberate arithmetic choices (shared with the device kernels, which this
// file models bit for bit):
//   * reductions over the subset use 32 lanes + xor butterfly (arith.hpp);
//   * the 6x6 Hessian is accumulated in FP64 (float products are exact in
//     double), conditioned, factored (Cholesky) and inverted in FP64, and the
//     Gauss-Newton step -H^-1 g is formed in FP64 and rounded to T once;
//   * sample positions are centre + offset (image.hpp, warp_offset).
#pragma once
#include <algorithm>
#include <cmath>
#include <vector>

#include "arith.hpp"
#include "image.hpp"

namespace oracle {

// include/semper/tuning.hpp constants used by the subset solve.
constexpr float kCorrAccept = 0.15f;
constexpr float kCorrSimplexTrigger = 0.4f;
constexpr float kMinValidPixelFraction = 0.90f;
constexpr float kSimplexFailScore = 0.1f;
constexpr float kLmAlpha = 0.05f;
constexpr int kIcgnMaxIter = 50;
constexpr float kGhostRejectFraction = 0.05f;
constexpr float kGhostWallThreshold = -5.0f;
constexpr float kHessianMinRcond = 1e-6f;

enum InitMode { INIT_AUTO_SEARCH = 0, INIT_NO_SEARCH = 1, INIT_NO_SIMPLEX = 2 };

using Mat6 = double[6][6];

// ---------------------------------------------------------------- 6x6 FP64 --

// Cholesky A = L L^T; false unless every pivot is positive and finite.
inline bool cholesky6(const Mat6 A, Mat6 L) {
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) L[i][j] = 0.0;
    for (int j = 0; j < 6; ++j) {
        double s = A[j][j];
        for (int k = 0; k < j; ++k) s = s - L[j][k] * L[j][k];
        if (!(s > 0.0) || !finite_bits(s)) return false;
        const double d = std::sqrt(s);
        L[j][j] = d;
        for (int i = j + 1; i < 6; ++i) {
            double t = A[i][j];
            for (int k = 0; k < j; ++k) t = t - L[i][k] * L[j][k];
            L[i][j] = t / d;
        }
    }
    return true;
}

// Explicit inverse from the Cholesky factor: A^-1 = L^-T L^-1.
inline bool inverse6(const Mat6 A, Mat6 Ainv) {
    Mat6 L;
    if (!cholesky6(A, L)) return false;
    Mat6 Li;
    for (int i = 0; i < 6; ++i)
        for (int j = 0; j < 6; ++j) Li[i][j] = 0.0;
    for (int c = 0; c < 6; ++c) {
        Li[c][c] = 1.0 / L[c][c];
        for (int i = c + 1; i < 6; ++i) {
            double t = 0.0;
            for (int k = c; k < i; ++k) t = t + L[i][k] * Li[k][c];
            Li[i][c] = -t / L[i][i];
        }
    }
    for (int r = 0; r < 6; ++r) {
        for (int c = r; c < 6; ++c) {
            double t = 0.0;
            for (int k = c; k < 6; ++k) t = t + Li[k][r] * Li[k][c];
            Ainv[r][c] = t;
            Ainv[c][r] = t;
        }
    }
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c)
            if (!finite_bits(Ainv[r][c])) return false;
    return true;
}

// hessian::well_conditioned (src/math/hessian.hpp:40-52): scaled 1-norm rcond
// from the explicit inverse, in FP64.
inline bool well_conditioned(const Mat6 H, int half) {
    const double s = half > 1 ? 1.0 / (double)half : 1.0;
    const double d[6] = {1.0, 1.0, s, s, s, s};
    Mat6 Hn, Hi;
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) {
            Hn[r][c] = (d[r] * H[r][c]) * d[c];
            if (!finite_bits(Hn[r][c])) return false;
        }
    if (!inverse6(Hn, Hi)) return false;
    double na = 0.0, ni = 0.0;
    for (int c = 0; c < 6; ++c) {
        double a = 0.0, b = 0.0;
        for (int r = 0; r < 6; ++r) {
            a = a + std::fabs(Hn[r][c]);
            b = b + std::fabs(Hi[r][c]);
        }
        na = std::max(na, a);
        ni = std::max(ni, b);
    }
    return 1.0 / (na * ni) > (double)kHessianMinRcond;
}

// The 2x2 translation-block guard (subset_precomputer.cpp:131-134;
// optimization_engine.cpp:396-401): false when cond > 1e12.
inline bool cond2x2_ok(const Mat6 H) {
    const double det = H[0][0] * H[1][1] - H[1][0] * H[0][1];
    const double nrm = H[0][0] * H[0][0] + H[0][1] * H[0][1] + H[1][0] * H[1][0] + H[1][1] * H[1][1];
    const double cond = std::fabs(det) > 1e-12 ? nrm / std::fabs(det) : 1.0e13;
    return !(cond > 1.0e12);
}

// ------------------------------------------------------------ pool entry --

template <class T>
struct PoolEntry {
    bool valid = false;
    T mean = T(0), std_dev = T(1);
    Mat6 H = {};  // FP64, symmetric
};

inline bool dim_ok(int dim) { return dim >= 3 && dim % 2 == 1; }

template <class T>
inline bool subset_on_image(const Image<T>& im, int cx, int cy, int half) {
    return cx - half >= 0 && cx + half < im.width && cy - half >= 0 && cy + half < im.height;
}

// compute_hessian_only (subset_precomputer.cpp:42-149). Mean and std in T, H in
// FP64; every sum is 32-lane partial + butterfly in the subset's row-major
// pixel order.
template <class T>
PoolEntry<T> compute_hessian_only(const Image<T>& im, int cx, int cy, int dim) {
    PoolEntry<T> e;
    const int half = dim / 2;
    if (!dim_ok(dim) || !subset_on_image(im, cx, cy, half)) return e;
    const int n = dim * dim;
    const int w = im.width;
    auto pix = [&](int i) { return (size_t)(cy - half + i / dim) * w + (cx - half + i % dim); };

    T part[kLanes] = {};
    int count = 0;
    for (int i = 0; i < n; ++i) {
        const T v = im.I[pix(i)];
        if (v < T(kGhostWallThreshold)) continue;
        part[i % kLanes] += v;
        ++count;
    }
    if ((float)count < (float)n * 0.5f) return e;
    const T mean = butterfly(part) / (T)count;

    for (int l = 0; l < kLanes; ++l) part[l] = T(0);
    for (int i = 0; i < n; ++i) {
        const T v = im.I[pix(i)];
        if (v < T(kGhostWallThreshold)) continue;
        const T d = v - mean;
        part[i % kLanes] = fmaT(d, d, part[i % kLanes]);
    }
    T sd = std::sqrt(butterfly(part) / (T)count);
    if (sd < T(1e-5f)) sd = T(1);
    const T inv = T(1) / sd;
    e.mean = mean;
    e.std_dev = sd;

    double hp[21][kLanes] = {};
    for (int i = 0; i < n; ++i) {
        const size_t k = pix(i);
        if (im.I[k] < T(kGhostWallThreshold)) continue;
        const T g0 = im.gx[k] * inv, g1 = im.gy[k] * inv;
        const T fx = (T)(i % dim - half), fy = (T)(i / dim - half);
        const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                             (double)(g1 * fx), (double)(g1 * fy)};
        int q = 0;
        for (int r = 0; r < 6; ++r)
            for (int c = r; c < 6; ++c, ++q) hp[q][i % kLanes] = fmaT(s[r], s[c], hp[q][i % kLanes]);
    }
    int q = 0;
    for (int r = 0; r < 6; ++r)
        for (int c = r; c < 6; ++c, ++q) {
            e.H[r][c] = butterfly(hp[q]);
            e.H[c][r] = e.H[r][c];
        }
    if (!cond2x2_ok(e.H) || !well_conditioned(e.H, half)) return e;
    e.valid = true;
    return e;
}

// ------------------------------------------------------------ the subset --

template <class T>
struct Subset {
    int cx = 0, cy = 0, dim = 0, n = 0;
    std::vector<T> I, gx, gy, rn;    // raw intensity/gradients, normalised ref
    std::vector<T> sd;               // 6 per pixel
    std::vector<unsigned char> ref_valid;
    int invalid_ref = 0;
    Mat6 H = {};
    bool ok = false;
};

// precompute_subset_fast (subset_precomputer.cpp:159-265) from a pool entry.
template <class T>
void fill_subset(Subset<T>& s, const Image<T>& im, int cx, int cy, int dim, const PoolEntry<T>& e) {
    s.cx = cx;
    s.cy = cy;
    s.ok = false;
    if (!dim_ok(dim) || !subset_on_image(im, cx, cy, dim / 2) || !e.valid) return;
    const int half = dim / 2, n = dim * dim;
    s.dim = dim;
    s.n = n;
    s.I.resize(n);
    s.gx.resize(n);
    s.gy.resize(n);
    s.rn.resize(n);
    s.sd.resize((size_t)6 * n);
    s.ref_valid.resize(n);
    const T inv = T(1) / e.std_dev;
    s.invalid_ref = 0;
    for (int i = 0; i < n; ++i) {
        const size_t k = (size_t)(cy - half + i / dim) * im.width + (cx - half + i % dim);
        s.I[i] = im.I[k];
        s.gx[i] = im.gx[k];
        s.gy[i] = im.gy[k];
        s.rn[i] = (s.I[i] - e.mean) * inv;
        const T g0 = s.gx[i] * inv, g1 = s.gy[i] * inv;
        const T fx = (T)(i % dim - half), fy = (T)(i / dim - half);
        T* sp = &s.sd[(size_t)6 * i];
        sp[0] = g0;
        sp[1] = g1;
        sp[2] = g0 * fx;
        sp[3] = g0 * fy;
        sp[4] = g1 * fx;
        sp[5] = g1 * fy;
        s.ref_valid[i] = s.I[i] < T(kGhostWallThreshold) ? 0 : 1;
        if (!s.ref_valid[i]) ++s.invalid_ref;
    }
    for (int r = 0; r < 6; ++r)
        for (int c = 0; c < 6; ++c) s.H[r][c] = e.H[r][c];
    s.ok = true;
}

template <class T>
struct Result {
    T u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0;
    int status = 0;
    T score = 0;
    int iters = 0;
    int invalid_ref = 0;
    int trigger_iters = 0;
};

template <class T>
inline Warp6<T> warp_from(T u, T v, T ux, T uy, T vx, T vy) {
    return Warp6<T>{T(1) + ux, uy, u, vx, T(1) + vy, v};
}

template <class T>
inline Result<T> result_from(const Warp6<T>& W, int status, T score, int iters, int inv_ref) {
    Result<T> r;
    r.u = W.w02;
    r.v = W.w12;
    r.ux = W.w00 - T(1);
    r.uy = W.w01;
    r.vx = W.w10;
    r.vy = W.w11 - T(1);
    r.status = status;
    r.score = score;
    r.iters = iters;
    r.invalid_ref = inv_ref;
    return r;
}

template <class T>
struct Engine {
    bool lm = false;
    bool six = false;
    int simplex_runs = 0;
    std::vector<T> vals;
    std::vector<unsigned char> valid;

    // sample_warped_subset (optimization_engine.cpp:191-269): values, validity,
    // and the lane-reduced sum of the valid values; returns their count.
    int sample(const Subset<T>& s, const Image<T>& def, const Warp6<T>& W, T& sum) {
        vals.assign(s.n, T(0));
        valid.assign(s.n, 0);
        const int half = s.dim / 2;
        T part[kLanes] = {};
        int count = 0;
        for (int i = 0; i < s.n; ++i) {
            const T ox = (T)(i % s.dim - half), oy = (T)(i / s.dim - half);
            T fx, fy;
            warp_offset(W, ox, oy, fx, fy);
            if (!guard_ok(fx, fy, s.cx, s.cy, def.width, def.height)) continue;
            const T val = sample_at(def, s.cx, s.cy, fx, fy, six);
            vals[i] = val;
            if (s.ref_valid[i]) {
                valid[i] = 1;
                part[i % kLanes] += val;
                ++count;
            }
        }
        sum = butterfly(part);
        return count;
    }

    // The step matrix for a whole-subset iteration (optimization_engine.cpp:302-315).
    void step_matrix(const Subset<T>& s, Mat6 Hs) const {
        const int half = s.dim / 2;
        if (lm) {
            Mat6 Hd;
            for (int r = 0; r < 6; ++r)
                for (int c = 0; c < 6; ++c) Hd[r][c] = s.H[r][c];
            Hd[0][0] += (double)kLmAlpha;
            Hd[1][1] += (double)kLmAlpha;
            if (well_conditioned(Hd, half) && inverse6(Hd, Hs)) return;
        }
        inverse6(s.H, Hs);
    }

    Result<T> icgn(const Subset<T>& s, const Image<T>& def, T u0, T v0, T ux0, T uy0, T vx0, T vy0) {
        const int n = s.n, half = s.dim / 2;
        Warp6<T> W = warp_from(u0, v0, ux0, uy0, vx0, vy0);
        Mat6 Href;
        step_matrix(s, Href);
        T final_score = T(1);
        const int min_valid = (int)((float)n * kMinValidPixelFraction);
        auto reject = [&](int it) { return result_from(W, 1, T(2), it, s.invalid_ref); };

        for (int iter = 0; iter < kIcgnMaxIter; ++iter) {
            T sum;
            const int cnt = sample(s, def, W, sum);
            if (cnt < min_valid) return reject(iter);
            const T mean = sum / (T)cnt;

            T part[kLanes] = {};
            for (int i = 0; i < n; ++i) {
                if (!valid[i]) continue;
                const T d = vals[i] - mean;
                part[i % kLanes] = fmaT(d, d, part[i % kLanes]);
            }
            T sdev = std::sqrt(butterfly(part) / (T)cnt);
            if (sdev < T(1e-5f)) sdev = T(1);
            const T inv = T(1) / sdev;

            T ep[kLanes] = {}, gp[6][kLanes] = {};
            const bool full = cnt == n;
            double hp[21][kLanes] = {};
            for (int i = 0; i < n; ++i) {
                if (!valid[i]) continue;
                const T nd = (vals[i] - mean) * inv;
                const T diff = s.rn[i] - nd;
                const int l = i % kLanes;
                ep[l] = fmaT(diff, diff, ep[l]);
                const T* sp = &s.sd[(size_t)6 * i];
                for (int k = 0; k < 6; ++k) gp[k][l] = fmaT(sp[k], diff, gp[k][l]);
                if (!full) {
                    int q = 0;
                    for (int r = 0; r < 6; ++r)
                        for (int c = r; c < 6; ++c, ++q)
                            hp[q][l] = fmaT((double)sp[r], (double)sp[c], hp[q][l]);
                }
            }
            const T err = butterfly(ep);
            T g[6];
            for (int k = 0; k < 6; ++k) g[k] = butterfly(gp[k]);

            Mat6 Hmask;
            const double(*Hstep)[6] = Href;
            if (!full) {
                Mat6 Hd;
                int q = 0;
                for (int r = 0; r < 6; ++r)
                    for (int c = r; c < 6; ++c, ++q) {
                        Hd[r][c] = butterfly(hp[q]);
                        Hd[c][r] = Hd[r][c];
                    }
                if (!cond2x2_ok(Hd)) return reject(iter);
                if (lm) {
                    Hd[0][0] += (double)kLmAlpha;
                    Hd[1][1] += (double)kLmAlpha;
                }
                if (!well_conditioned(Hd, half) || !inverse6(Hd, Hmask)) return reject(iter);
                Hstep = Hmask;
            }
            final_score = err / (T)cnt;

            T dp[6];
            for (int r = 0; r < 6; ++r) {
                double a = 0.0;
                for (int c = 0; c < 6; ++c) a = fmaT(Hstep[r][c], (double)g[c], a);
                dp[r] = (T)(-a);
            }
            // dW = I + [[dp2, dp3, dp0], [dp4, dp5, dp1]]; W <- W dW^-1
            const T a00 = T(1) + dp[2], a01 = dp[3], a10 = dp[4], a11 = T(1) + dp[5];
            const T det = a00 * a11 - a01 * a10;
            bool fin = true;
            for (int k = 0; k < 6; ++k) fin = fin && finite_bits(dp[k]);
            if (!fin || !(std::fabs(det) > T(1e-6f))) return reject(iter + 1);
            const T id = T(1) / det;
            const T i00 = a11 * id, i01 = -a01 * id, i10 = -a10 * id, i11 = a00 * id;
            const T i02 = -(i00 * dp[0] + i01 * dp[1]);
            const T i12 = -(i10 * dp[0] + i11 * dp[1]);
            Warp6<T> Wn;
            Wn.w00 = W.w00 * i00 + W.w01 * i10;
            Wn.w01 = W.w00 * i01 + W.w01 * i11;
            Wn.w02 = (W.w00 * i02 + W.w01 * i12) + W.w02;
            Wn.w10 = W.w10 * i00 + W.w11 * i10;
            Wn.w11 = W.w10 * i01 + W.w11 * i11;
            Wn.w12 = (W.w10 * i02 + W.w11 * i12) + W.w12;
            if (!finite_bits(Wn.w00) || !finite_bits(Wn.w01) || !finite_bits(Wn.w02) ||
                !finite_bits(Wn.w10) || !finite_bits(Wn.w11) || !finite_bits(Wn.w12))
                return reject(iter + 1);
            W = Wn;

            T nn = dp[0] * dp[0];
            for (int k = 1; k < 6; ++k) nn = nn + dp[k] * dp[k];
            if (std::sqrt(nn) < T(0.001f)) {
                // Texture check (optimization_engine.cpp:435-461).
                T sxp[kLanes] = {}, syp[kLanes] = {};
                int surv = 0;
                for (int i = 0; i < n; ++i) {
                    if (!valid[i]) continue;
                    sxp[i % kLanes] = fmaT(s.gx[i], s.gx[i], sxp[i % kLanes]);
                    syp[i % kLanes] = fmaT(s.gy[i], s.gy[i], syp[i % kLanes]);
                    ++surv;
                }
                if (surv == 0) return reject(iter + 1);
                const T sg = std::min(butterfly(sxp), butterfly(syp));
                if (sg <= T(0)) return reject(iter + 1);
                if (!finite_bits(final_score)) return reject(iter + 1);
                return result_from(W, 0, final_score, iter + 1, s.invalid_ref);
            }
        }
        return result_from(W, 1, final_score, kIcgnMaxIter, s.invalid_ref);
    }

    // evaluate_znssd (optimization_engine.cpp:467-528).
    T znssd(const Subset<T>& s, const Image<T>& def, const Warp6<T>& W) {
        T sum;
        const int cnt = sample(s, def, W, sum);
        const int n = s.n;
        if (cnt == 0 || cnt < (int)((float)n * kMinValidPixelFraction)) return T(2);
        const T mean = sum / (T)cnt;
        T part[kLanes] = {};
        for (int i = 0; i < n; ++i) {
            if (!valid[i]) continue;
            const T d = vals[i] - mean;
            part[i % kLanes] = fmaT(d, d, part[i % kLanes]);
        }
        T sdev = std::sqrt(butterfly(part) / (T)cnt);
        if (sdev < T(1e-5f)) sdev = T(1);
        T ep[kLanes] = {};
        if (cnt == n) {
            const T inv = T(1) / sdev;
            for (int i = 0; i < n; ++i) {
                const T diff = s.rn[i] - (vals[i] - mean) * inv;
                ep[i % kLanes] = fmaT(diff, diff, ep[i % kLanes]);
            }
        } else {
            for (int i = 0; i < n; ++i) {
                if (!valid[i]) continue;
                const T diff = s.rn[i] - (vals[i] - mean) / sdev;
                ep[i % kLanes] = fmaT(diff, diff, ep[i % kLanes]);
            }
        }
        const T score = butterfly(ep) / (T)cnt;
        return finite_bits(score) ? score : T(2);
    }

    // solve_simplex (optimization_engine.cpp:531-651).
    Result<T> simplex(const Subset<T>& s, const Image<T>& def, const Result<T>& start, bool trans) {
        ++simplex_runs;
        const int DIM = trans ? 2 : 6, np = DIM + 1;
        T p[7][6] = {};
        T y[7] = {};
        const T scale[6] = {T(2), T(2), T(0.01f), T(0.01f), T(0.01f), T(0.01f)};
        auto eval = [&](const T* pt) {
            if (trans) return znssd(s, def, warp_from(pt[0], pt[1], T(0), T(0), T(0), T(0)));
            return znssd(s, def, warp_from(pt[0], pt[1], pt[2], pt[3], pt[4], pt[5]));
        };
        p[0][0] = start.u;
        p[0][1] = start.v;
        if (!trans) {
            p[0][2] = start.ux;
            p[0][3] = start.uy;
            p[0][4] = start.vx;
            p[0][5] = start.vy;
        }
        y[0] = eval(p[0]);
        for (int i = 1; i < np; ++i) {
            for (int j = 0; j < DIM; ++j) p[i][j] = p[0][j];
            p[i][i - 1] += scale[i - 1];
            y[i] = eval(p[i]);
        }
        const T alpha = T(1), gamma = T(2), rho = T(0.5f), sigma = T(0.5f);
        for (int it = 0; it < 100; ++it) {
            int idx[7] = {0, 1, 2, 3, 4, 5, 6};
            for (int a = 1; a < np; ++a) {
                const int v = idx[a];
                int b = a;
                while (b > 0 && y[v] < y[idx[b - 1]]) {
                    idx[b] = idx[b - 1];
                    --b;
                }
                idx[b] = v;
            }
            if (std::fabs(y[idx[0]] - y[idx[np - 1]]) < T(1e-5f)) break;
            T pb[6] = {};
            for (int i = 0; i < DIM; ++i)
                for (int j = 0; j < DIM; ++j) pb[j] += p[idx[i]][j];
            for (int j = 0; j < DIM; ++j) pb[j] /= (T)DIM;
            T pr[6] = {};
            for (int j = 0; j < DIM; ++j) pr[j] = pb[j] + alpha * (pb[j] - p[idx[np - 1]][j]);
            const T yr = eval(pr);
            if (y[idx[0]] <= yr && yr < y[idx[np - 2]]) {
                for (int j = 0; j < DIM; ++j) p[idx[np - 1]][j] = pr[j];
                y[idx[np - 1]] = yr;
            } else if (yr < y[idx[0]]) {
                T pe[6] = {};
                for (int j = 0; j < DIM; ++j) pe[j] = pb[j] + gamma * (pr[j] - pb[j]);
                const T ye = eval(pe);
                if (ye < yr) {
                    for (int j = 0; j < DIM; ++j) p[idx[np - 1]][j] = pe[j];
                    y[idx[np - 1]] = ye;
                } else {
                    for (int j = 0; j < DIM; ++j) p[idx[np - 1]][j] = pr[j];
                    y[idx[np - 1]] = yr;
                }
            } else {
                T pc[6] = {};
                const bool outside = yr < y[idx[np - 1]];
                const T* bp = outside ? pr : p[idx[np - 1]];
                for (int j = 0; j < DIM; ++j) pc[j] = pb[j] + rho * (bp[j] - pb[j]);
                const T yc = eval(pc);
                if (yc < std::min(yr, y[idx[np - 1]])) {
                    for (int j = 0; j < DIM; ++j) p[idx[np - 1]][j] = pc[j];
                    y[idx[np - 1]] = yc;
                } else {
                    for (int i = 1; i < np; ++i) {
                        for (int j = 0; j < DIM; ++j)
                            p[idx[i]][j] = p[idx[0]][j] + sigma * (p[idx[i]][j] - p[idx[0]][j]);
                        y[idx[i]] = eval(p[idx[i]]);
                    }
                }
            }
        }
        int best = 0;
        for (int k = 1; k < np; ++k)
            if (y[k] < y[best]) best = k;
        Result<T> r;
        r.u = p[best][0];
        r.v = p[best][1];
        if (!trans) {
            r.ux = p[best][2];
            r.uy = p[best][3];
            r.vx = p[best][4];
            r.vy = p[best][5];
        }
        r.status = y[best] > T(kSimplexFailScore) ? -2 : 0;
        r.score = y[best];
        return r;
    }

    // estimate_initial_guess (optimization_engine.cpp:120-179): every 9th
    // subset pixel, offsets +-15 px in steps of 2, zero-mean unit-variance
    // SSD; sequential sums (the device runs one offset per lane).
    void coarse(const Subset<T>& s, const Image<T>& def, T& bu, T& bv) const {
        const int half = s.dim / 2;
        int sampled = 0;
        for (int i = 0; i < s.n; i += 9) ++sampled;
        std::vector<T> r, d;
        T best = T(1e20f);
        for (int v = -15; v <= 15; v += 2) {
            for (int u = -15; u <= 15; u += 2) {
                r.clear();
                d.clear();
                for (int i = 0; i < s.n; i += 9) {
                    if (!s.ref_valid[i]) continue;
                    const int x = s.cx + (i % s.dim - half) + u;
                    const int y = s.cy + (i / s.dim - half) + v;
                    if (x < 4 || x > def.width - 5 || y < 4 || y > def.height - 5) continue;
                    r.push_back(s.I[i]);
                    d.push_back(def.I[(size_t)y * def.width + x]);
                }
                const int m_i = (int)r.size();
                if (m_i < 3 || 2 * m_i < sampled) continue;
                const T m = (T)m_i;
                T mr = T(0), md = T(0);
                for (int k = 0; k < m_i; ++k) {
                    mr = mr + r[k];
                    md = md + d[k];
                }
                mr = mr / m;
                md = md / m;
                T vr = T(0), vd = T(0);
                for (int k = 0; k < m_i; ++k) {
                    vr = vr + (r[k] - mr) * (r[k] - mr);
                    vd = vd + (d[k] - md) * (d[k] - md);
                }
                const T sr = std::sqrt(vr / m), sdv = std::sqrt(vd / m);
                if (!(sr > T(1e-5f)) || !(sdv > T(1e-5f))) continue;
                T score = T(0);
                for (int k = 0; k < m_i; ++k) {
                    const T e = (r[k] - mr) / sr - (d[k] - md) / sdv;
                    score = score + e * e;
                }
                score = score / m;
                if (score < best) {
                    best = score;
                    bu = (T)u;
                    bv = (T)v;
                }
            }
        }
    }

    // calculate_deformation (optimization_engine.cpp:55-118).
    Result<T> solve(const Subset<T>& s, const Image<T>& def, const T g[6], InitMode mode) {
        Result<T> res;
        if (mode == INIT_AUTO_SEARCH) {
            T eu = g[0], ev = g[1];
            if (eu == T(0) && ev == T(0)) coarse(s, def, eu, ev);
            Result<T> start;
            start.u = eu;
            start.v = ev;
            start.score = T(1);
            const Result<T> cr = simplex(s, def, start, true);
            res = icgn(s, def, cr.u, cr.v, T(0), T(0), T(0), T(0));
            res.trigger_iters = res.iters;
        } else {
            res = icgn(s, def, g[0], g[1], g[2], g[3], g[4], g[5]);
            res.trigger_iters = res.iters;
            if ((res.status != 0 || res.score > T(kCorrSimplexTrigger)) && mode != INIT_NO_SIMPLEX) {
                Result<T> start;
                start.u = g[0];
                start.v = g[1];
                start.ux = g[2];
                start.uy = g[3];
                start.vx = g[4];
                start.vy = g[5];
                start.score = T(1);
                const Result<T> rr = simplex(s, def, start, false);
                const int trig = res.iters;
                Result<T> resc = icgn(s, def, rr.u, rr.v, rr.ux, rr.uy, rr.vx, rr.vy);
                resc.trigger_iters = trig;
                const bool first_better =
                    res.status == 0 && (resc.status != 0 || res.score < resc.score);
                if (!first_better) res = resc;
            }
        }
        return res;
    }
};

// solve_node: subset fill, solve, Ghost Wall rejection.
template <class T>
struct NodeSolve {
    bool initialized = false;
    bool rescue = false;
    Result<T> res;
};

template <class T>
NodeSolve<T> solve_node(Engine<T>& eng, Subset<T>& sub, const Image<T>& ref, const Image<T>& def,
                        int x, int y, int dim, const PoolEntry<T>& e, const T g[6], InitMode mode) {
    NodeSolve<T> out;
    fill_subset(sub, ref, x, y, dim, e);
    out.initialized = sub.ok;
    if (!sub.ok) return out;
    const int before = eng.simplex_runs;
    out.res = eng.solve(sub, def, g, mode);
    const float gf = (float)out.res.invalid_ref / (float)(dim * dim);
    if (gf > kGhostRejectFraction) {
        out.res.score = T(2);
        out.res.status = 1;
    }
    out.rescue = eng.simplex_runs > before;
    return out;
}

}  // namespace oracle
