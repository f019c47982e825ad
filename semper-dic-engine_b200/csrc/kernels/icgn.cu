// Batched subset solves: IC-GN with its Simplex rescue and coarse search,
// one warp per subset, a persistent grid pulling tasks from a device queue.
//
// Restates, per task, solve_node (src/pipeline/full_field_solver.cpp:119-139)
// -> calculate_deformation (src/math/optimization_engine.cpp:55-118) ->
// solve_icgn (:272-465) / solve_simplex (:531-651) / estimate_initial_guess
// (:120-179), then reject_if_ghosted (src/pipeline/full_field_internal.hpp:347-353).
//
// Layout per warp (dynamic shared memory, 128-byte aligned): an mbarrier, the
// FP64 step matrices, a tile of the deformed image staged by 2-D TMA around
// the warped subset, and the subset's sampled values, their validity and its
// reference (non-Ghost-Wall) flags. Pixel i of the subset (row-major) belongs
// to lane i % 32. Samples whose 4x4 / 6x6 support lies in the tile read shared
// memory; any other sample reads the image through the read-only cache, with
// the same arithmetic, so the tile only ever changes where the values come from.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "dic_types.h"
#include "icgn.cuh"
#include "tma.cuh"

#include <cstring>

namespace dic {

namespace {

constexpr float kCorrSimplexTrigger = 0.4f;
constexpr float kMinValidPixelFraction = 0.90f;
constexpr float kSimplexFailScore = 0.1f;
constexpr float kLmAlpha = 0.05f;
constexpr int kIcgnMaxIter = 50;
constexpr float kGhostRejectFraction = 0.05f;
constexpr float kGhost = -5.0f;

struct Res {
    float u, v, ux, uy, vx, vy, score;
    int status, iters;
};

__device__ __forceinline__ Res res_from(const float W[6], int status, float score, int iters) {
    Res r;
    r.u = W[2];
    r.v = W[5];
    r.ux = W[0] - 1.0f;
    r.uy = W[1];
    r.vx = W[3];
    r.vy = W[4] - 1.0f;
    r.status = status;
    r.score = score;
    r.iters = iters;
    return r;
}

template <bool SIX>
struct WarpSolver {
    const SolveArgs& a;
    int lane;
    int cx, cy, dim, half, n;
    float mref, iref;
    int min_valid;
    size_t ref_base;  // index of the subset's top-left pixel in the planes
    uint64_t* bar;    // TMA completion barrier
    double* Href;     // [36] step matrix of a whole-subset iteration
    double* Hmask;    // [36] step matrix of a masked iteration
    float* tile;      // [tile_h][tile_w] deformed-image tile
    float* vals;      // [n]
    uint8_t* valid;   // [n]
    uint8_t* refok;   // [n] reference pixel outside the Ghost Wall
    int simplex_runs;
    const CUtensorMap* tmap;
    int tx0, ty0;         // tile origin, image pixels
    bool tile_ok;         // the tile holds the box at (tx0, ty0)
    bool tile_on;         // TMA staging enabled for this warp
    uint32_t phase;       // parity of the next barrier phase

    __device__ WarpSolver(const SolveArgs& args, int ln, unsigned char* sm, const CUtensorMap* map,
                          uint32_t ph)
        : a(args), lane(ln), tmap(map), phase(ph) {
        const SmemLayout L = smem_layout(a.max_n, a.tile_w, a.tile_h);
        bar = reinterpret_cast<uint64_t*>(sm);
        Href = reinterpret_cast<double*>(sm + L.off_h);
        Hmask = Href + 36;
        tile = reinterpret_cast<float*>(sm + L.off_tile);
        vals = reinterpret_cast<float*>(sm + L.off_vals);
        valid = sm + L.off_valid;
        refok = sm + L.off_refok;
        simplex_runs = 0;
        tile_ok = false;
        tile_on = a.tile_w > 0 && a.tile_h > 0;
        tx0 = ty0 = 0;
    }

    // Make the tile cover every sample support of the warped subset, staging
    // a new box with TMA when the warp has left the current one. False when
    // the subset does not fit a box (the samples then read global memory).
    __device__ void ensure_tile(const float W[6]) {
        if (!tile_on) return;
        const float h = (float)half;
        float fx[4], fy[4];
        const float ox[4] = {-h, h, -h, h}, oy[4] = {-h, -h, h, h};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            fx[k] = __fmaf_rn(W[0], ox[k], __fmaf_rn(W[1], oy[k], W[2]));
            fy[k] = __fmaf_rn(W[3], ox[k], __fmaf_rn(W[4], oy[k], W[5]));
        }
        const float mnx = fminf(fminf(fx[0], fx[1]), fminf(fx[2], fx[3]));
        const float mxx = fmaxf(fmaxf(fx[0], fx[1]), fmaxf(fx[2], fx[3]));
        const float mny = fminf(fminf(fy[0], fy[1]), fminf(fy[2], fy[3]));
        const float mxy = fmaxf(fmaxf(fy[0], fy[1]), fmaxf(fy[2], fy[3]));
        if (!(mnx > -1e6f && mxx < 1e6f && mny > -1e6f && mxy < 1e6f)) {
            tile_ok = false;
            return;
        }
        // support of every sample, one pixel of slack for rounding
        const int lo_tap = SIX ? 3 : 2, hi_tap = SIX ? 4 : 3;
        const int x_lo = cx + (int)floorf(mnx) - lo_tap, x_hi = cx + (int)floorf(mxx) + hi_tap;
        const int y_lo = cy + (int)floorf(mny) - lo_tap, y_hi = cy + (int)floorf(mxy) + hi_tap;
        if (tile_ok && x_lo >= tx0 && x_hi < tx0 + a.tile_w && y_lo >= ty0 && y_hi < ty0 + a.tile_h) return;
        const int need_w = x_hi - x_lo + 1, need_h = y_hi - y_lo + 1;
        if (need_w + 3 > a.tile_w || need_h > a.tile_h) {
            tile_ok = false;
            return;
        }
        // centre the support, x start on a 16-byte boundary (a multiple of 4)
        int nx = x_lo - (a.tile_w - 3 - need_w) / 2;
        nx = nx >= 0 ? (nx & ~3) : -((-nx + 3) & ~3);
        const int ny = y_lo - (a.tile_h - need_h) / 2;
        __syncwarp();
        if (lane == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, (uint32_t)(a.tile_w * a.tile_h * 4));
            tma_load_2d(tile, tmap, nx, ny, bar);
        }
        const bool done = mbar_wait_bounded(bar, phase, 1 << 22);
        phase ^= 1u;
        if (!__all_sync(kFull, done)) {
            // A copy that never completed: stop staging for this warp.
            if (lane == 0 && a.err) atomicExch(a.err, 1);
            tile_on = false;
            tile_ok = false;
            return;
        }
        tx0 = nx;
        ty0 = ny;
        tile_ok = true;
    }

    // Walk this lane's pixels i = lane, lane + 32, ...: (row, col) in the subset.
    template <class F>
    __device__ __forceinline__ void for_pixels(F&& f) const {
        int row = lane / dim, col = lane - row * dim;
        const int q = 32 / dim, r = 32 - q * dim;
#pragma unroll 4
        for (int i = lane; i < n; i += 32) {
            f(i, row, col);
            col += r;
            row += q;
            if (col >= dim) {
                col -= dim;
                ++row;
            }
        }
    }

    __device__ __forceinline__ size_t ref_idx(int row, int col) const {
        return ref_base + (size_t)row * a.pitch + col;
    }

    // sample_warped_subset (optimization_engine.cpp:191-269) on centre +
    // offset coordinates; returns the count of valid samples, their sum in `sum`.
    __device__ int sample(const float W[6], float& sum) {
        ensure_tile(W);
        float part = 0.0f;
        int cnt = 0;
        const float lo_x = (float)(4 - cx), hi_x = (float)(a.W - 4 - cx);
        const float lo_y = (float)(4 - cy), hi_y = (float)(a.H - 4 - cy);
        const int lo_tap = SIX ? 2 : 1, hi_tap = SIX ? 3 : 2;
        const bool use_tile = tile_ok;
        for_pixels([&](int i, int row, int col) {
            const float ox = (float)(col - half), oy = (float)(row - half);
            const float fx = __fmaf_rn(W[0], ox, __fmaf_rn(W[1], oy, W[2]));
            const float fy = __fmaf_rn(W[3], ox, __fmaf_rn(W[4], oy, W[5]));
            const float rx = fx + 0.5f, ry = fy + 0.5f;
            float val = 0.0f;
            uint8_t ok = 0;
            if (rx >= lo_x && rx < hi_x && ry >= lo_y && ry < hi_y) {
                const float flx = floorf(fx), fly = floorf(fy);
                const int xi = cx + (int)flx, yi = cy + (int)fly;
                const int lx = xi - tx0, ly = yi - ty0;
                if (use_tile && lx >= lo_tap && lx + hi_tap < a.tile_w && ly >= lo_tap && ly + hi_tap < a.tile_h) {
                    val = SIX ? interp6s(tile, a.tile_w, lx, ly, fx - flx, fy - fly)
                              : interp4s(tile, a.tile_w, lx, ly, fx - flx, fy - fly);
                } else {
                    val = SIX ? interp6(a.defI, a.pitch, xi, yi, fx - flx, fy - fly)
                              : interp4(a.defI, a.pitch, xi, yi, fx - flx, fy - fly);
                }
                if (refok[i]) {
                    ok = 1;
                    part = part + val;
                    ++cnt;
                }
            }
            vals[i] = val;
            valid[i] = ok;
        });
        __syncwarp();
        sum = wsum(part);
        return wsum(cnt);
    }

    __device__ float sum_sq(float mean) const {
        float part = 0.0f;
        for (int i = lane; i < n; i += 32) {
            if (!valid[i]) continue;
            const float d = vals[i] - mean;
            part = __fmaf_rn(d, d, part);
        }
        return wsum(part);
    }

    // The whole-subset step matrix (optimization_engine.cpp:302-315) comes
    // precomputed with the pool entry (FP64, upper triangle): into Href.
    __device__ void step_matrix(const double* Hs21) {
        for (int k = lane; k < 36; k += 32) {
            const int r = k / 6, c = k % 6;
            Href[k] = Hs21[r <= c ? tri21(r, c) : tri21(c, r)];
        }
        __syncwarp();
    }

    __device__ Res icgn(float u0, float v0, float ux0, float uy0, float vx0, float vy0) {
        float W[6] = {1.0f + ux0, uy0, u0, vx0, 1.0f + vy0, v0};
        float final_score = 1.0f;
        for (int iter = 0; iter < kIcgnMaxIter; ++iter) {
            float sum;
            const int cnt = sample(W, sum);
            if (cnt < min_valid) return res_from(W, 1, 2.0f, iter);
            const float mean = sum / (float)cnt;
            float sdev = sqrtf(sum_sq(mean) / (float)cnt);
            if (sdev < 1e-5f) sdev = 1.0f;
            const float inv = 1.0f / sdev;
            const bool full = cnt == n;

            float ep = 0.0f, gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f, gp3 = 0.0f, gp4 = 0.0f, gp5 = 0.0f;
            for_pixels([&](int i, int row, int col) {
                if (!valid[i]) return;
                const size_t k = ref_idx(row, col);
                const float rn = (__ldg(a.refI + k) - mref) * iref;
                const float g0 = __ldg(a.refGx + k) * iref, g1 = __ldg(a.refGy + k) * iref;
                const float fx = (float)(col - half), fy = (float)(row - half);
                const float nd = (vals[i] - mean) * inv;
                const float diff = rn - nd;
                ep = __fmaf_rn(diff, diff, ep);
                gp0 = __fmaf_rn(g0, diff, gp0);
                gp1 = __fmaf_rn(g1, diff, gp1);
                gp2 = __fmaf_rn(g0 * fx, diff, gp2);
                gp3 = __fmaf_rn(g0 * fy, diff, gp3);
                gp4 = __fmaf_rn(g1 * fx, diff, gp4);
                gp5 = __fmaf_rn(g1 * fy, diff, gp5);
            });
            const float err = wsum(ep);
            const float g[6] = {wsum(gp0), wsum(gp1), wsum(gp2), wsum(gp3), wsum(gp4), wsum(gp5)};

            const double* Hstep = Href;
            if (!full) {
                if (!masked_step()) return res_from(W, 1, 2.0f, iter);
                Hstep = Hmask;
            }
            final_score = err / (float)cnt;

            float dpl = 0.0f;
            if (lane < 6) {
                double acc = 0.0;
                for (int c = 0; c < 6; ++c) acc = __fma_rn(Hstep[lane * 6 + c], (double)g[c], acc);
                dpl = (float)(-acc);
            }
            float dp[6];
#pragma unroll
            for (int k = 0; k < 6; ++k) dp[k] = __shfl_sync(kFull, dpl, k);

            const float a00 = 1.0f + dp[2], a01 = dp[3], a10 = dp[4], a11 = 1.0f + dp[5];
            const float det = a00 * a11 - a01 * a10;
            bool fin = true;
#pragma unroll
            for (int k = 0; k < 6; ++k) fin = fin && finite_f(dp[k]);
            if (!fin || !(fabsf(det) > 1e-6f)) return res_from(W, 1, 2.0f, iter + 1);
            const float id = 1.0f / det;
            const float i00 = a11 * id, i01 = -a01 * id, i10 = -a10 * id, i11 = a00 * id;
            const float i02 = -(i00 * dp[0] + i01 * dp[1]);
            const float i12 = -(i10 * dp[0] + i11 * dp[1]);
            float Wn[6];
            Wn[0] = W[0] * i00 + W[1] * i10;
            Wn[1] = W[0] * i01 + W[1] * i11;
            Wn[2] = (W[0] * i02 + W[1] * i12) + W[2];
            Wn[3] = W[3] * i00 + W[4] * i10;
            Wn[4] = W[3] * i01 + W[4] * i11;
            Wn[5] = (W[3] * i02 + W[4] * i12) + W[5];
            bool wfin = true;
#pragma unroll
            for (int k = 0; k < 6; ++k) wfin = wfin && finite_f(Wn[k]);
            if (!wfin) return res_from(W, 1, 2.0f, iter + 1);
#pragma unroll
            for (int k = 0; k < 6; ++k) W[k] = Wn[k];

            float nn = dp[0] * dp[0];
#pragma unroll
            for (int k = 1; k < 6; ++k) nn = nn + dp[k] * dp[k];
            if (sqrtf(nn) < 0.001f) {
                float sx = 0.0f, sy = 0.0f;
                for_pixels([&](int i, int row, int col) {
                    if (!valid[i]) return;
                    const size_t k = ref_idx(row, col);
                    const float gx = __ldg(a.refGx + k), gy = __ldg(a.refGy + k);
                    sx = __fmaf_rn(gx, gx, sx);
                    sy = __fmaf_rn(gy, gy, sy);
                });
                const float tx = wsum(sx), ty = wsum(sy);
                const float sg = ty < tx ? ty : tx;
                if (cnt == 0) return res_from(W, 1, 2.0f, iter + 1);
                if (sg <= 0.0f) return res_from(W, 1, 2.0f, iter + 1);
                if (!finite_f(final_score)) return res_from(W, 1, 2.0f, iter + 1);
                return res_from(W, 0, final_score, iter + 1);
            }
        }
        return res_from(W, 1, final_score, kIcgnMaxIter);
    }

    // The masked iteration's own Hessian (optimization_engine.cpp:373-413),
    // FP64: into Hmask; false to reject.
    __device__ __noinline__ bool masked_step() {
        double hp[21];
#pragma unroll
        for (int q = 0; q < 21; ++q) hp[q] = 0.0;
        for_pixels([&](int i, int row, int col) {
            if (!valid[i]) return;
            const size_t k = ref_idx(row, col);
            const float g0 = __ldg(a.refGx + k) * iref, g1 = __ldg(a.refGy + k) * iref;
            const float fx = (float)(col - half), fy = (float)(row - half);
            const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                                 (double)(g1 * fx), (double)(g1 * fy)};
            int q = 0;
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
                for (int c = r; c < 6; ++c, ++q) hp[q] = __fma_rn(s[r], s[c], hp[q]);
        });
#pragma unroll
        for (int q = 0; q < 21; ++q) hp[q] = wsum(hp[q]);
        int ok = 0;
        if (lane == 0) {
            double Hd[6][6], Hi[6][6];
            for (int r = 0; r < 6; ++r)
                for (int c = r; c < 6; ++c) {
                    Hd[r][c] = hp[tri21(r, c)];
                    Hd[c][r] = Hd[r][c];
                }
            if (cond2x2_ok(Hd)) {
                if (a.lm) {
                    Hd[0][0] += (double)kLmAlpha;
                    Hd[1][1] += (double)kLmAlpha;
                }
                if (well_conditioned(Hd, half) && inverse6(Hd, Hi)) {
                    for (int r = 0; r < 6; ++r)
                        for (int c = 0; c < 6; ++c) Hmask[r * 6 + c] = Hi[r][c];
                    ok = 1;
                }
            }
        }
        ok = __shfl_sync(kFull, ok, 0);
        __syncwarp();
        return ok != 0;
    }

    // evaluate_znssd (optimization_engine.cpp:467-528).
    __device__ float znssd(const float W[6]) {
        float sum;
        const int cnt = sample(W, sum);
        if (cnt == 0 || cnt < min_valid) return 2.0f;
        const float mean = sum / (float)cnt;
        float sdev = sqrtf(sum_sq(mean) / (float)cnt);
        if (sdev < 1e-5f) sdev = 1.0f;
        float ep = 0.0f;
        const bool full = cnt == n;
        const float inv = 1.0f / sdev;
        for_pixels([&](int i, int row, int col) {
            if (!valid[i]) return;
            const float rn = (__ldg(a.refI + ref_idx(row, col)) - mref) * iref;
            const float diff = full ? rn - (vals[i] - mean) * inv : rn - (vals[i] - mean) / sdev;
            ep = __fmaf_rn(diff, diff, ep);
        });
        const float score = wsum(ep) / (float)cnt;
        return finite_f(score) ? score : 2.0f;
    }

    // solve_simplex (optimization_engine.cpp:531-651). Every lane keeps the
    // same simplex; the evaluations are warp-collective.
    __device__ __noinline__ Res simplex(const float start[6], bool trans) {
        ++simplex_runs;
        const int D = trans ? 2 : 6, np = D + 1;
        float p[7][6];
        float y[7];
        for (int i = 0; i < 7; ++i) {
            y[i] = 0.0f;
            for (int j = 0; j < 6; ++j) p[i][j] = 0.0f;
        }
        const float scale[6] = {2.0f, 2.0f, 0.01f, 0.01f, 0.01f, 0.01f};
        auto eval = [&](const float* pt) {
            float W[6];
            if (trans) {
                W[0] = 1.0f; W[1] = 0.0f; W[2] = pt[0]; W[3] = 0.0f; W[4] = 1.0f; W[5] = pt[1];
            } else {
                W[0] = 1.0f + pt[2]; W[1] = pt[3]; W[2] = pt[0]; W[3] = pt[4]; W[4] = 1.0f + pt[5]; W[5] = pt[1];
            }
            return znssd(W);
        };
        p[0][0] = start[0];
        p[0][1] = start[1];
        if (!trans)
            for (int j = 2; j < 6; ++j) p[0][j] = start[j];
        y[0] = eval(p[0]);
        for (int i = 1; i < np; ++i) {
            for (int j = 0; j < D; ++j) p[i][j] = p[0][j];
            p[i][i - 1] += scale[i - 1];
            y[i] = eval(p[i]);
        }
        for (int it = 0; it < 100; ++it) {
            int idx[7] = {0, 1, 2, 3, 4, 5, 6};
            for (int aa = 1; aa < np; ++aa) {
                const int v = idx[aa];
                int b = aa;
                while (b > 0 && y[v] < y[idx[b - 1]]) {
                    idx[b] = idx[b - 1];
                    --b;
                }
                idx[b] = v;
            }
            if (fabsf(y[idx[0]] - y[idx[np - 1]]) < 1e-5f) break;
            float pb[6] = {0, 0, 0, 0, 0, 0};
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) pb[j] += p[idx[i]][j];
            for (int j = 0; j < D; ++j) pb[j] /= (float)D;
            float pr[6] = {0, 0, 0, 0, 0, 0};
            for (int j = 0; j < D; ++j) pr[j] = pb[j] + 1.0f * (pb[j] - p[idx[np - 1]][j]);
            const float yr = eval(pr);
            if (y[idx[0]] <= yr && yr < y[idx[np - 2]]) {
                for (int j = 0; j < D; ++j) p[idx[np - 1]][j] = pr[j];
                y[idx[np - 1]] = yr;
            } else if (yr < y[idx[0]]) {
                float pe[6] = {0, 0, 0, 0, 0, 0};
                for (int j = 0; j < D; ++j) pe[j] = pb[j] + 2.0f * (pr[j] - pb[j]);
                const float ye = eval(pe);
                if (ye < yr) {
                    for (int j = 0; j < D; ++j) p[idx[np - 1]][j] = pe[j];
                    y[idx[np - 1]] = ye;
                } else {
                    for (int j = 0; j < D; ++j) p[idx[np - 1]][j] = pr[j];
                    y[idx[np - 1]] = yr;
                }
            } else {
                float pc[6] = {0, 0, 0, 0, 0, 0};
                const bool outside = yr < y[idx[np - 1]];
                for (int j = 0; j < D; ++j) {
                    const float bj = outside ? pr[j] : p[idx[np - 1]][j];
                    pc[j] = pb[j] + 0.5f * (bj - pb[j]);
                }
                const float yc = eval(pc);
                const float ylast = y[idx[np - 1]];
                if (yc < (ylast < yr ? ylast : yr)) {
                    for (int j = 0; j < D; ++j) p[idx[np - 1]][j] = pc[j];
                    y[idx[np - 1]] = yc;
                } else {
                    for (int i = 1; i < np; ++i) {
                        for (int j = 0; j < D; ++j) p[idx[i]][j] = p[idx[0]][j] + 0.5f * (p[idx[i]][j] - p[idx[0]][j]);
                        y[idx[i]] = eval(p[idx[i]]);
                    }
                }
            }
        }
        int best = 0;
        for (int k = 1; k < np; ++k)
            if (y[k] < y[best]) best = k;
        Res r;
        r.u = p[best][0];
        r.v = p[best][1];
        r.ux = trans ? 0.0f : p[best][2];
        r.uy = trans ? 0.0f : p[best][3];
        r.vx = trans ? 0.0f : p[best][4];
        r.vy = trans ? 0.0f : p[best][5];
        r.status = y[best] > kSimplexFailScore ? -2 : 0;
        r.score = y[best];
        r.iters = 0;
        return r;
    }

    // estimate_initial_guess (optimization_engine.cpp:120-179): one offset per
    // lane at a time (8 each), sequential sums as the reference, then the
    // first minimum in the reference's v-major order.
    __device__ __noinline__ void coarse(float& bu, float& bv) const {
        int sampled = 0;
        for (int i = 0; i < n; i += 9) ++sampled;
        float best = 1e20f;
        int best_idx = 1 << 30;
        for (int j = 0; j < 8; ++j) {
            const int idx = lane * 8 + j;  // increasing per lane: first minimum kept
            const int v = -15 + 2 * (idx / 16), u = -15 + 2 * (idx % 16);
            int m = 0;
            float mr = 0.0f, md = 0.0f;
            auto sample_at = [&](int i, float& r, float& d) {
                const int row = i / dim, col = i - (i / dim) * dim;
                const float rv = __ldg(a.refI + ref_idx(row, col));
                if (rv < kGhost) return false;
                const int x = cx + (col - half) + u, y = cy + (row - half) + v;
                if (x < 4 || x > a.W - 5 || y < 4 || y > a.H - 5) return false;
                r = rv;
                d = __ldg(a.defI + (size_t)y * a.pitch + x);
                return true;
            };
            for (int i = 0; i < n; i += 9) {
                float r, d;
                if (!sample_at(i, r, d)) continue;
                mr = mr + r;
                md = md + d;
                ++m;
            }
            if (m < 3 || 2 * m < sampled) continue;
            const float fm = (float)m;
            mr = mr / fm;
            md = md / fm;
            float vr = 0.0f, vd = 0.0f;
            for (int i = 0; i < n; i += 9) {
                float r, d;
                if (!sample_at(i, r, d)) continue;
                vr = vr + (r - mr) * (r - mr);
                vd = vd + (d - md) * (d - md);
            }
            const float sr = sqrtf(vr / fm), sd = sqrtf(vd / fm);
            if (!(sr > 1e-5f) || !(sd > 1e-5f)) continue;
            float score = 0.0f;
            for (int i = 0; i < n; i += 9) {
                float r, d;
                if (!sample_at(i, r, d)) continue;
                const float e = (r - mr) / sr - (d - md) / sd;
                score = score + e * e;
            }
            score = score / fm;
            if (score < best) {
                best = score;
                best_idx = idx;
            }
        }
        // Warp argmin on (score, idx).
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float os = __shfl_xor_sync(kFull, best, o);
            const int oi = __shfl_xor_sync(kFull, best_idx, o);
            if (os < best || (os == best && oi < best_idx)) {
                best = os;
                best_idx = oi;
            }
        }
        if (best_idx < 256 && best < 1e20f) {
            bv = (float)(-15 + 2 * (best_idx / 16));
            bu = (float)(-15 + 2 * (best_idx % 16));
        }
    }

    // calculate_deformation (optimization_engine.cpp:55-118).
    __device__ Res solve(const float g[6], int mode, int& trigger) {
        Res res;
        if (mode == DIC_INIT_AUTO_SEARCH) {
            float eu = g[0], ev = g[1];
            if (eu == 0.0f && ev == 0.0f) coarse(eu, ev);
            const float st[6] = {eu, ev, 0, 0, 0, 0};
            const Res cr = simplex(st, true);
            res = icgn(cr.u, cr.v, 0.0f, 0.0f, 0.0f, 0.0f);
            trigger = res.iters;
        } else {
            res = icgn(g[0], g[1], g[2], g[3], g[4], g[5]);
            trigger = res.iters;
            if ((res.status != 0 || res.score > kCorrSimplexTrigger) && mode != DIC_INIT_NO_SIMPLEX) {
                const Res rr = simplex(g, false);
                const int trig = res.iters;
                const Res rs = icgn(rr.u, rr.v, rr.ux, rr.uy, rr.vx, rr.vy);
                const bool first_better = res.status == 0 && (rs.status != 0 || res.score < rs.score);
                if (!first_better) {
                    res = rs;
                }
                trigger = trig;
            }
        }
        return res;
    }
};

template <bool SIX>
__global__ void __launch_bounds__(kSolveThreads, 4)
    solve_kernel(const __grid_constant__ CUtensorMap tmap, SolveArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char* my = smem + (size_t)warp * a.smem_per_warp;
    if (lane == 0) mbar_init(reinterpret_cast<uint64_t*>(my), 1);
    fence_proxy_async_smem();
    __syncwarp();
    uint32_t phase = 0;
    bool tile_on = a.tile_w > 0;
    const int ntasks = a.n_tasks_dev ? *a.n_tasks_dev : a.n_tasks;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(a.queue, 1);
        t = __shfl_sync(kFull, t, 0);
        if (t >= ntasks) break;
        if (a.cancel && *(volatile const int*)a.cancel) break;
        const dic_task T = a.tasks[t];
        dic_result out;
        out.u = out.v = out.ux = out.uy = out.vx = out.vy = 0.0f;
        out.score = 0.0f;
        out.status = out.iters = out.trigger_iters = out.invalid_ref = out.flags = 0;

        const int dim = a.dim, half = dim / 2;
        const bool dim_ok = dim >= 3 && (dim & 1) && dim * dim <= a.max_n;
        const bool on_img = T.cx - half >= 0 && T.cx + half < a.W && T.cy - half >= 0 && T.cy + half < a.H;
        if (!dim_ok || !on_img || !a.pool_valid[T.node]) {
            if (lane == 0) a.results[t] = out;
            continue;
        }
        WarpSolver<SIX> s(a, lane, my, &tmap, phase);
        s.tile_on = tile_on;
        s.cx = T.cx;
        s.cy = T.cy;
        s.dim = dim;
        s.half = half;
        s.n = dim * dim;
        const float2 ms = a.pool_ms[T.node];
        s.mref = ms.x;
        s.iref = 1.0f / ms.y;
        s.min_valid = (int)((float)s.n * kMinValidPixelFraction);
        s.ref_base = (size_t)(T.cy - half) * a.pitch + (T.cx - half);

        int ghost = 0;
        s.for_pixels([&](int i, int row, int col) {
            const bool g = __ldg(a.refI + s.ref_idx(row, col)) < kGhost;
            s.refok[i] = g ? 0 : 1;
            if (g) ++ghost;
        });
        ghost = wsum(ghost);
        s.step_matrix(a.pool_Hs + (size_t)T.node * 21);

        int trigger = 0;
        Res r = s.solve(T.g, T.mode, trigger);
        phase = s.phase;
        tile_on = s.tile_on;
        if ((float)ghost / (float)(dim * dim) > kGhostRejectFraction) {
            r.score = 2.0f;
            r.status = 1;
        }
        if (lane == 0) {
            out.u = r.u; out.v = r.v; out.ux = r.ux; out.uy = r.uy; out.vx = r.vx; out.vy = r.vy;
            out.score = r.score;
            out.status = r.status;
            out.iters = r.iters;
            out.trigger_iters = trigger;
            out.invalid_ref = ghost;
            out.flags = DIC_RES_INITIALIZED | (s.simplex_runs > 0 ? DIC_RES_RESCUE : 0);
            a.results[t] = out;
        }
        __syncwarp();
    }
}

}  // namespace

void tile_box(int dim, int six, int& tw, int& th) {
    // the subset's support plus one pixel of rounding slack each side, three
    // columns of alignment slack, and a margin of two pixels for the warp to
    // move in before the tile is staged again
    const int need = dim + (six ? 5 : 3) + 2;
    tw = ((need + 3 + 4) + 3) & ~3;
    th = need + 4;
    if (tw > 256 || th > 256) tw = th = 0;
}

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

}  // namespace

cudaError_t launch_solve(const SolveArgs& a0, int six, int grid_blocks, cudaStream_t st) {
    SolveArgs a = a0;
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    int tw = 0, th = 0;
    tile_box(a.dim, six, tw, th);
    const bool pitch_ok = (a.pitch % 4) == 0 && (reinterpret_cast<uintptr_t>(a.defI) % 16) == 0;
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (tw > 0 && pitch_ok && enc) {
        const cuuint64_t gdim[2] = {(cuuint64_t)a.W, (cuuint64_t)a.H};
        const cuuint64_t gstride[1] = {(cuuint64_t)a.pitch * 4};
        const cuuint32_t box[2] = {(cuuint32_t)tw, (cuuint32_t)th};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = enc(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(a.defI), gdim, gstride,
                               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) tw = th = 0;
    } else {
        tw = th = 0;
    }
    a.tile_w = tw;
    a.tile_h = th;
    a.smem_per_warp = smem_layout(a.max_n, tw, th).bytes;
    const size_t smem = a.smem_per_warp * (kSolveThreads / 32);
    cudaError_t e;
    if (six) {
        e = cudaFuncSetAttribute(solve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        solve_kernel<true><<<grid_blocks, kSolveThreads, smem, st>>>(tmap, a);
    } else {
        e = cudaFuncSetAttribute(solve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        solve_kernel<false><<<grid_blocks, kSolveThreads, smem, st>>>(tmap, a);
    }
    return cudaGetLastError();
}

}  // namespace dic
