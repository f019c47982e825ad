// Batched subset solves: IC-GN with its Simplex rescue and coarse search,
// a persistent grid pulling tasks from a device queue. Three kernels:
// - fast_kernel: one warp per subset, the common case (whole-subset IC-GN);
//   every other task is handed to a list;
// - coop_rescue_kernel: the tasks on that list, with every path, a block of
//   kCoopWarps warps per task (the sampling of each evaluation shared);
// - solve_kernel: every task of a launch whose subsets are too large for the
//   staged solvers (side > 45).
//
// Restates, per task, solve_node (src/pipeline/full_field_solver.cpp:119-139)
// -> calculate_deformation (src/math/optimization_engine.cpp:55-118) ->
// solve_icgn (:272-465) / solve_simplex (:531-651) / estimate_initial_guess
// (:120-179), then reject_if_ghosted (src/pipeline/full_field_internal.hpp:347-353).
//
// Layout per warp (dynamic shared memory, 128-byte aligned): an mbarrier and
// the tile state, the FP64 step matrices, a tile of the deformed image staged
// by 2-D TMA around the warped subset, and the subset's sampled values, their
// validity and its reference (non-Ghost-Wall) flags. Pixel i of the subset
// (row-major) belongs to lane i % 32. Samples whose 4x4 / 6x6 support lies in
// the tile read shared memory; any other sample reads the image through the
// read-only cache with the same arithmetic, so the tile only ever changes where
// the values come from.
//
// The per-subset constants live in a small context passed by value, so the hot
// loops keep them in registers; only the rare paths (Simplex, coarse search,
// masked-iteration Hessian) are out-of-line calls.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <utility>

#include "common.cuh"
#include "dic_types.h"
#include "icgn.cuh"
#include "tma.cuh"

// Unroll factor of the general pass's per-pixel loops.
#ifndef DIC_PIXEL_UNROLL
#define DIC_PIXEL_UNROLL 2
#endif

namespace dic {

namespace {

constexpr int kPixelUnroll = DIC_PIXEL_UNROLL;
constexpr int kArgsBytes = 256;  // shared-memory header: the block's copy of SolveArgs
static_assert(sizeof(SolveArgs) <= kArgsBytes, "SolveArgs header");
constexpr float kCorrSimplexTrigger = 0.4f;
constexpr float kSimplexFailScore = 0.1f;
constexpr float kLmAlpha = 0.05f;
constexpr int kIcgnMaxIter = 50;
constexpr float kGhostRejectFraction = 0.05f;
constexpr float kGhost = -5.0f;
constexpr int kCancelPollTasks = 32;  // a power of two
// Polls of an mbarrier before a TMA completion wait gives up (about 0.1 s),
// unless the launch asks for fewer. A wait that gives up sets the error flag
// and the warp reads global memory from then on; before it exits, the warp
// waits (bounded the same way) for the copy still in flight into its tile.
constexpr int kTmaPolls = 1 << 22;

struct Res {
    float u, v, ux, uy, vx, vy, score;
    int status, iters;
};

// Mutable TMA tile state of a warp, kept in its shared-memory header.
struct TileState {
    int tx0, ty0;    // tile origin, image pixels
    int ok;          // the tile holds the box at (tx0, ty0)
    int on;          // staging enabled (off after a wait ran out)
    unsigned phase;  // parity of the next barrier phase
    int pend;        // a wait ran out: the copy of parity pend_phase may still be in flight
    unsigned pend_phase;
};

// The per-subset values of a solve. Launch constants (plane pointers, image
// and subset sizes, offsets into shared memory) are read where they are used
// from the block's copy of the launch arguments in shared memory, so they take
// no registers. The argument block itself is a plain by-value parameter whose
// address is never taken.
struct Ctx {
    const SolveArgs* a;
    unsigned char* sm;  // the warp's shared memory
    const CUtensorMap* tmap;
    int ref_base;  // index of the subset's top-left pixel in the planes
    int cx, cy, lane;
    float mref, iref;
};

__device__ __forceinline__ uint64_t* bar_of(const Ctx& c) { return reinterpret_cast<uint64_t*>(c.sm); }
__device__ __forceinline__ TileState* state_of(const Ctx& c) { return reinterpret_cast<TileState*>(c.sm + 16); }
__device__ __forceinline__ double* href_of(const Ctx& c) { return reinterpret_cast<double*>(c.sm + 64); }
__device__ __forceinline__ double* hmask_of(const Ctx& c) { return reinterpret_cast<double*>(c.sm + 352); }
__device__ __forceinline__ float* tile_of(const Ctx& c) { return reinterpret_cast<float*>(c.sm + c.a->off_tile); }
__device__ __forceinline__ float* vals_of(const Ctx& c) { return reinterpret_cast<float*>(c.sm + c.a->off_vals); }
__device__ __forceinline__ uint8_t* valid_of(const Ctx& c) { return c.sm + c.a->off_valid; }
__device__ __forceinline__ uint8_t* refok_of(const Ctx& c) { return c.sm + c.a->off_refok; }

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

// Walk this lane's pixels i = lane, lane + 32, ...: (row, col) in the subset.
template <class F>
__device__ __forceinline__ void for_pixels(const Ctx& c, F&& f) {
    int row = c.lane / c.a->dim, col = c.lane - row * c.a->dim;
    const int q = 32 / c.a->dim, r = 32 - q * c.a->dim;
#pragma unroll kPixelUnroll
    for (int i = c.lane; i < c.a->n; i += 32) {
        f(i, row, col);
        col += r;
        row += q;
        if (col >= c.a->dim) {
            col -= c.a->dim;
            ++row;
        }
    }
}

__device__ __forceinline__ int ref_idx(const Ctx& c, int row, int col) {
    return c.ref_base + row * c.a->pitch + col;
}

// Make the tile cover every sample support of the warped subset, staging a
// new box with TMA when the warp has left the current one. The tile is marked
// unusable when the subset does not fit a box (samples then read global memory).
template <bool SIX>
__device__ __forceinline__ void ensure_tile(const Ctx& c, const float W[6]) {
    TileState* ts = state_of(c);
    if (!ts->on) return;
    const float h = (float)c.a->half;
    float mnx = 0.0f, mxx = 0.0f, mny = 0.0f, mxy = 0.0f;
    bool in_range = true;  // every corner finite and within 1e6 px (a NaN fails the comparisons)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float ox = (k & 1) ? h : -h, oy = (k & 2) ? h : -h;
        const float fx = __fmaf_rn(W[0], ox, __fmaf_rn(W[1], oy, W[2]));
        const float fy = __fmaf_rn(W[3], ox, __fmaf_rn(W[4], oy, W[5]));
        in_range = in_range && fx > -1e6f && fx < 1e6f && fy > -1e6f && fy < 1e6f;
        mnx = k ? fminf(mnx, fx) : fx;
        mxx = k ? fmaxf(mxx, fx) : fx;
        mny = k ? fminf(mny, fy) : fy;
        mxy = k ? fmaxf(mxy, fy) : fy;
    }
    if (!in_range) {
        __syncwarp();
        if (c.lane == 0) ts->ok = 0;
        __syncwarp();
        return;
    }
    // support of every sample, one pixel of slack for rounding
    const int lo_tap = SIX ? 3 : 2, hi_tap = SIX ? 4 : 3;
    const int x_lo = c.cx + (int)floorf(mnx) - lo_tap, x_hi = c.cx + (int)floorf(mxx) + hi_tap;
    const int y_lo = c.cy + (int)floorf(mny) - lo_tap, y_hi = c.cy + (int)floorf(mxy) + hi_tap;
    const int tx0 = ts->tx0, ty0 = ts->ty0;
    if (ts->ok && x_lo >= tx0 && x_hi < tx0 + c.a->tile_w && y_lo >= ty0 && y_hi < ty0 + c.a->tile_h) return;
    const int need_w = x_hi - x_lo + 1, need_h = y_hi - y_lo + 1;
    __syncwarp();
    if (need_w + 3 > c.a->tile_w || need_h > c.a->tile_h) {
        if (c.lane == 0) ts->ok = 0;
        __syncwarp();
        return;
    }
    // centre the support, x start on a 16-byte boundary (a multiple of 4)
    int nx = x_lo - (c.a->tile_w - 3 - need_w) / 2;
    nx = nx >= 0 ? (nx & ~3) : -((-nx + 3) & ~3);
    const int ny = y_lo - (c.a->tile_h - need_h) / 2;
    const unsigned phase = ts->phase;
    if (c.lane == 0) {
        fence_proxy_async_smem();
        mbar_arrive_expect_tx(bar_of(c), (uint32_t)(c.a->tile_w * c.a->tile_h * 4));
        tma_load_2d(tile_of(c), c.tmap, nx, ny, bar_of(c));
    }
    const int polls = c.a->tma_max_polls > 0 ? c.a->tma_max_polls : kTmaPolls;
    const bool done = __all_sync(kFull, mbar_wait_bounded(bar_of(c), phase, polls));
    if (c.lane == 0) {
        ts->phase = phase ^ 1u;
        if (done) {
            ts->tx0 = nx;
            ts->ty0 = ny;
            ts->ok = 1;
        } else {
            // a copy that has not completed: stop staging for this warp
            ts->ok = 0;
            ts->on = 0;
            ts->pend = 1;
            ts->pend_phase = phase;
            if (c.a->err) atomicExch(c.a->err, 1);
        }
    }
    __syncwarp();
}

// sample_warped_subset (optimization_engine.cpp:191-269) on centre + offset
// coordinates; returns the count of valid samples, their sum in `sum`.
template <bool SIX>
__device__ __forceinline__ int sample(const Ctx& c, const float W[6], float& sum) {
    ensure_tile<SIX>(c, W);
    const TileState* ts = state_of(c);
    const int use_tile = ts->ok, tx0 = ts->tx0, ty0 = ts->ty0;
    const float* tile = tile_of(c);
    float* vals = vals_of(c);
    uint8_t* valid = valid_of(c);
    const uint8_t* refok = refok_of(c);
    float part = 0.0f;
    int cnt = 0;
    const float lo_x = (float)(4 - c.cx), hi_x = (float)(c.a->W - 4 - c.cx);
    const float lo_y = (float)(4 - c.cy), hi_y = (float)(c.a->H - 4 - c.cy);
    const int lo_tap = SIX ? 2 : 1, hi_tap = SIX ? 3 : 2;
    for_pixels(c, [&](int i, int row, int col) {
        const float ox = (float)(col - c.a->half), oy = (float)(row - c.a->half);
        const float fx = __fmaf_rn(W[0], ox, __fmaf_rn(W[1], oy, W[2]));
        const float fy = __fmaf_rn(W[3], ox, __fmaf_rn(W[4], oy, W[5]));
        const float rx = fx + 0.5f, ry = fy + 0.5f;
        float val = 0.0f;
        uint8_t ok = 0;
        if (rx >= lo_x && rx < hi_x && ry >= lo_y && ry < hi_y) {
            const float flx = floorf(fx), fly = floorf(fy);
            const int xi = c.cx + (int)flx, yi = c.cy + (int)fly;
            const int lx = xi - tx0, ly = yi - ty0;
            if (use_tile && lx >= lo_tap && lx + hi_tap < c.a->tile_w && ly >= lo_tap && ly + hi_tap < c.a->tile_h) {
                val = SIX ? interp6s(tile, c.a->tile_w, lx, ly, fx - flx, fy - fly)
                          : interp4s(tile, c.a->tile_w, lx, ly, fx - flx, fy - fly);
            } else {
                val = SIX ? interp6(c.a->defI, c.a->pitch, xi, yi, fx - flx, fy - fly)
                          : interp4(c.a->defI, c.a->pitch, xi, yi, fx - flx, fy - fly);
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

__device__ __forceinline__ float sum_sq(const Ctx& c, float mean) {
    const float* vals = vals_of(c);
    const uint8_t* valid = valid_of(c);
    float part = 0.0f;
    for (int i = c.lane; i < c.a->n; i += 32) {
        if (!valid[i]) continue;
        const float d = vals[i] - mean;
        part = __fmaf_rn(d, d, part);
    }
    return wsum(part);
}

// The masked iteration's own Hessian (optimization_engine.cpp:373-413),
// FP64, into the Hmask slot; false to reject.
__device__ __noinline__ bool masked_step(Ctx c) {
    const uint8_t* valid = valid_of(c);
    double hp[21];
#pragma unroll
    for (int q = 0; q < 21; ++q) hp[q] = 0.0;
    for_pixels(c, [&](int i, int row, int col) {
        if (!valid[i]) return;
        const int k = ref_idx(c, row, col);
        const float g0 = __ldg(c.a->refGx + k) * c.iref, g1 = __ldg(c.a->refGy + k) * c.iref;
        const float fx = (float)(col - c.a->half), fy = (float)(row - c.a->half);
        const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                             (double)(g1 * fx), (double)(g1 * fy)};
        int q = 0;
#pragma unroll
        for (int a = 0; a < 6; ++a)
#pragma unroll
            for (int b = a; b < 6; ++b, ++q) hp[q] = __fma_rn(s[a], s[b], hp[q]);
    });
#pragma unroll
    for (int q = 0; q < 21; ++q) hp[q] = wsum(hp[q]);
    int ok = 0;
    if (c.lane == 0) {
        double Hd[6][6], Hi[6][6];
        for (int a = 0; a < 6; ++a)
            for (int b = a; b < 6; ++b) {
                Hd[a][b] = hp[tri21(a, b)];
                Hd[b][a] = Hd[a][b];
            }
        if (cond2x2_ok(Hd)) {
            if (c.a->lm) {
                Hd[0][0] += (double)kLmAlpha;
                Hd[1][1] += (double)kLmAlpha;
            }
            if (well_conditioned(Hd, c.a->half) && inverse6(Hd, Hi)) {
                double* Hm = hmask_of(c);
                for (int a = 0; a < 6; ++a)
                    for (int b = 0; b < 6; ++b) Hm[a * 6 + b] = Hi[a][b];
                ok = 1;
            }
        }
    }
    ok = __shfl_sync(kFull, ok, 0);
    __syncwarp();
    return ok != 0;
}

// solve_icgn (optimization_engine.cpp:272-465). The FAST form never takes
// the masked-iteration path: it reports `defer` instead, and the task is
// solved again from the start by the general form.
template <bool SIX, bool FAST>
__device__ __forceinline__ Res icgn(const Ctx& c, const float st[6], bool& defer) {
    float W[6] = {1.0f + st[2], st[3], st[0], st[4], 1.0f + st[5], st[1]};
    float final_score = 1.0f;
    const float* vals = vals_of(c);
    const uint8_t* valid = valid_of(c);
    for (int iter = 0; iter < kIcgnMaxIter; ++iter) {
        float sum;
        const int cnt = sample<SIX>(c, W, sum);
        if (cnt < c.a->min_valid) return res_from(W, 1, 2.0f, iter);
        const float mean = sum / (float)cnt;
        float sdev = sqrtf(sum_sq(c, mean) / (float)cnt);
        if (sdev < 1e-5f) sdev = 1.0f;
        const float inv = 1.0f / sdev;
        const bool full = cnt == c.a->n;

        float ep = 0.0f, gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f, gp3 = 0.0f, gp4 = 0.0f, gp5 = 0.0f;
        for_pixels(c, [&](int i, int row, int col) {
            if (!valid[i]) return;
            const int k = ref_idx(c, row, col);
            const float rn = (__ldg(c.a->refI + k) - c.mref) * c.iref;
            const float g0 = __ldg(c.a->refGx + k) * c.iref, g1 = __ldg(c.a->refGy + k) * c.iref;
            const float fx = (float)(col - c.a->half), fy = (float)(row - c.a->half);
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

        const double* Hstep = href_of(c);
        if (!full) {
            if constexpr (FAST) {
                defer = true;
                return res_from(W, 1, 2.0f, iter);
            } else {
                if (!masked_step(c)) return res_from(W, 1, 2.0f, iter);
                Hstep = hmask_of(c);
            }
        }
        final_score = err / (float)cnt;

        float dpl = 0.0f;
        if (c.lane < 6) {
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) acc = __fma_rn(Hstep[c.lane * 6 + k], (double)g[k], acc);
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
            for_pixels(c, [&](int i, int row, int col) {
                if (!valid[i]) return;
                const int k = ref_idx(c, row, col);
                const float gx = __ldg(c.a->refGx + k), gy = __ldg(c.a->refGy + k);
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

// evaluate_znssd (optimization_engine.cpp:467-528).
template <bool SIX>
__device__ __forceinline__ float znssd(const Ctx& c, const float W[6]) {
    float sum;
    const int cnt = sample<SIX>(c, W, sum);
    if (cnt == 0 || cnt < c.a->min_valid) return 2.0f;
    const float mean = sum / (float)cnt;
    float sdev = sqrtf(sum_sq(c, mean) / (float)cnt);
    if (sdev < 1e-5f) sdev = 1.0f;
    const float* vals = vals_of(c);
    const uint8_t* valid = valid_of(c);
    float ep = 0.0f;
    const bool full = cnt == c.a->n;
    const float inv = 1.0f / sdev;
    for_pixels(c, [&](int i, int row, int col) {
        if (!valid[i]) return;
        const float rn = (__ldg(c.a->refI + ref_idx(c, row, col)) - c.mref) * c.iref;
        const float diff = full ? rn - (vals[i] - mean) * inv : rn - (vals[i] - mean) / sdev;
        ep = __fmaf_rn(diff, diff, ep);
    });
    const float score = wsum(ep) / (float)cnt;
    return finite_f(score) ? score : 2.0f;
}

// solve_simplex (optimization_engine.cpp:531-651). Every lane keeps the same
// simplex; the evaluations are warp-collective.
template <bool SIX>
__device__ __noinline__ Res simplex(Ctx c, float s0, float s1, float s2, float s3, float s4, float s5, bool trans) {
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
        return znssd<SIX>(c, W);
    };
    p[0][0] = s0;
    p[0][1] = s1;
    if (!trans) {
        p[0][2] = s2;
        p[0][3] = s3;
        p[0][4] = s4;
        p[0][5] = s5;
    }
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
// lane at a time (8 each), sequential sums as the reference, then the first
// minimum in the reference's v-major order. Returns (u, v); the guess when no
// offset qualifies.
__device__ __noinline__ float2 coarse(Ctx c, float gu, float gv) {
    int sampled = 0;
    for (int i = 0; i < c.a->n; i += 9) ++sampled;
    float best = 1e20f;
    int best_idx = 1 << 30;
    for (int j = 0; j < 8; ++j) {
        const int idx = c.lane * 8 + j;  // increasing per lane: first minimum kept
        const int v = -15 + 2 * (idx / 16), u = -15 + 2 * (idx % 16);
        auto sample_at = [&](int i, float& r, float& d) {
            const int row = i / c.a->dim, col = i - (i / c.a->dim) * c.a->dim;
            const float rv = __ldg(c.a->refI + ref_idx(c, row, col));
            if (rv < kGhost) return false;
            const int x = c.cx + (col - c.a->half) + u, y = c.cy + (row - c.a->half) + v;
            if (x < 4 || x > c.a->W - 5 || y < 4 || y > c.a->H - 5) return false;
            r = rv;
            d = __ldg(c.a->defI + (size_t)y * c.a->pitch + x);
            return true;
        };
        int m = 0;
        float mr = 0.0f, md = 0.0f;
        for (int i = 0; i < c.a->n; i += 9) {
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
        for (int i = 0; i < c.a->n; i += 9) {
            float r, d;
            if (!sample_at(i, r, d)) continue;
            vr = vr + (r - mr) * (r - mr);
            vd = vd + (d - md) * (d - md);
        }
        const float sr = sqrtf(vr / fm), sd = sqrtf(vd / fm);
        if (!(sr > 1e-5f) || !(sd > 1e-5f)) continue;
        float score = 0.0f;
        for (int i = 0; i < c.a->n; i += 9) {
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
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float os = __shfl_xor_sync(kFull, best, o);
        const int oi = __shfl_xor_sync(kFull, best_idx, o);
        if (os < best || (os == best && oi < best_idx)) {
            best = os;
            best_idx = oi;
        }
    }
    if (best_idx < 256 && best < 1e20f)
        return make_float2((float)(-15 + 2 * (best_idx % 16)), (float)(-15 + 2 * (best_idx / 16)));
    return make_float2(gu, gv);
}

// FAST: the common case only (whole-subset iterations, no Simplex, no coarse
// search), every other task appended to the deferred list. General: the
// deferred tasks, with every path.
template <bool SIX, bool FAST>
__global__ void __launch_bounds__(32, 1)
    solve_kernel(const __grid_constant__ CUtensorMap tmap, const SolveArgs a) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the block's copy of the launch arguments (a by-value copy: the parameter's
    // address is never taken), read by the per-subset code through Ctx::a
    SolveArgs* sa = reinterpret_cast<SolveArgs*>(smem);
    if (threadIdx.x == 0) *sa = a;
    __syncthreads();
    unsigned char* my = smem + kArgsBytes + (size_t)warp * a.smem_per_warp;
    if (lane == 0) {
        mbar_init(reinterpret_cast<uint64_t*>(my), 1);
        TileState* ts = reinterpret_cast<TileState*>(my + 16);
        ts->tx0 = ts->ty0 = 0;
        ts->ok = 0;
        ts->on = a.tile_w > 0 ? 1 : 0;
        ts->phase = 0;
        ts->pend = 0;
        ts->pend_phase = 0;
    }
    fence_proxy_async_smem();
    __syncwarp();
    const int all_tasks = a.n_tasks_dev ? *a.n_tasks_dev : a.n_tasks;
    const int ntasks = (FAST || a.general_all) ? all_tasks : *(volatile const int*)(a.queue + 2);
    int* queue = FAST ? a.queue : a.queue + 1;
    int* const n_deferred = a.queue + 2;
    int* const deferred = a.deferred;
    auto defer_task = [n_deferred, deferred, lane](int t) {
        if (lane == 0) {
            const int slot = atomicAdd(n_deferred, 1);
            deferred[slot] = t;
        }
        __syncwarp();
    };
    int polled = 0;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(queue, 1);
        q = __shfl_sync(kFull, q, 0);
        if (q >= ntasks) break;
        // the cancel flag lives in host memory: a read crosses PCIe, so a warp
        // looks at it once every kCancelPollTasks tasks, not per task
        if (a.cancel && (++polled & (kCancelPollTasks - 1)) == 0 && *(volatile const int*)a.cancel) break;
        const int t = (FAST || a.general_all) ? q : a.deferred[q];
        const dic_task T = a.tasks[t];
        if constexpr (FAST) {
            if (T.mode == DIC_INIT_AUTO_SEARCH) {
                defer_task(t);
                continue;
            }
        }
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
        Ctx c;
        c.a = sa;
        c.sm = my;
        c.tmap = &tmap;
        c.cx = T.cx;
        c.cy = T.cy;
        c.lane = lane;
        const float2 ms = a.pool_ms[T.node];
        c.mref = ms.x;
        c.iref = 1.0f / ms.y;
        c.ref_base = (T.cy - half) * a.pitch + (T.cx - half);

        uint8_t* refok = refok_of(c);
        int ghost = 0;
        for_pixels(c, [&](int i, int row, int col) {
            const bool g = __ldg(c.a->refI + ref_idx(c, row, col)) < kGhost;
            refok[i] = g ? 0 : 1;
            if (g) ++ghost;
        });
        ghost = wsum(ghost);
        // the whole-subset step matrix (optimization_engine.cpp:302-315), from the pool
        {
            const double* Hs21 = a.pool_Hs + (size_t)T.node * 21;
            double* Hr = href_of(c);
            for (int k = lane; k < 36; k += 32) {
                const int r = k / 6, cc = k % 6;
                Hr[k] = Hs21[r <= cc ? tri21(r, cc) : tri21(cc, r)];
            }
        }
        __syncwarp();

        // calculate_deformation (optimization_engine.cpp:55-118)
        const int mode = T.mode;
        float st[6] = {T.g[0], T.g[1], T.g[2], T.g[3], T.g[4], T.g[5]};
        const float* guess = a.tasks[t].g;
        bool rescue = false;
        bool defer = false;
        if constexpr (!FAST) if (mode == DIC_INIT_AUTO_SEARCH) {
            float2 e = make_float2(st[0], st[1]);
            if (e.x == 0.0f && e.y == 0.0f) e = coarse(c, e.x, e.y);
            const Res cr = simplex<SIX>(c, e.x, e.y, 0.0f, 0.0f, 0.0f, 0.0f, true);
            rescue = true;
            st[0] = cr.u; st[1] = cr.v; st[2] = st[3] = st[4] = st[5] = 0.0f;
        }
        Res res;
        int trigger = 0;
        for (int run = 0; run < 2; ++run) {
            const Res r = icgn<SIX, FAST>(c, st, defer);
            if (FAST && defer) break;
            if (run == 0) {
                res = r;
                trigger = r.iters;
                if (mode != DIC_INIT_NO_SEARCH || !(r.status != 0 || r.score > kCorrSimplexTrigger)) break;
                if constexpr (FAST) {
                    defer = true;
                    break;
                } else {
                    const Res rr =
                        simplex<SIX>(c, guess[0], guess[1], guess[2], guess[3], guess[4], guess[5], false);
                    rescue = true;
                    st[0] = rr.u; st[1] = rr.v; st[2] = rr.ux; st[3] = rr.uy; st[4] = rr.vx; st[5] = rr.vy;
                }
            } else {
                const bool first_better = res.status == 0 && (r.status != 0 || res.score < r.score);
                if (!first_better) res = r;
            }
        }
        if (FAST && defer) {
            defer_task(t);
            continue;
        }
        if ((float)ghost / (float)(dim * dim) > kGhostRejectFraction) {
            res.score = 2.0f;
            res.status = 1;
        }
        if (lane == 0) {
            out.u = res.u; out.v = res.v; out.ux = res.ux; out.uy = res.uy; out.vx = res.vx; out.vy = res.vy;
            out.score = res.score;
            out.status = res.status;
            out.iters = res.iters;
            out.trigger_iters = trigger;
            out.invalid_ref = ghost;
            out.flags = DIC_RES_INITIALIZED | (rescue ? DIC_RES_RESCUE : 0);
            a.results[t] = out;
        }
        __syncwarp();
    }
    // a copy whose wait ran out may still be writing into the tile: let it
    // land (bounded) before the block's shared memory is released
    const TileState* ts = reinterpret_cast<const TileState*>(my + 16);
    __syncwarp();
    if (ts->pend) (void)__all_sync(kFull, mbar_wait_bounded(reinterpret_cast<uint64_t*>(my), ts->pend_phase, kTmaPolls));
}

// ---------------------------------------------------------------------------
// The staged solvers: one warp per subset and one warp per block, so that
// shared memory alone sets the occupancy. The deformed image is read from a
// TMA tile in shared memory and the sampled values are kept there. With STAGE
// the warp also stages its reference subset per task ((I - mean) / std, and
// the raw gradients, which the texture check needs as they are), so that the
// iterations read only shared memory (the rescue pass); without it the
// reference is read from the planes, normalised the same way, and a warp
// takes about half the shared memory (the fast pass, where occupancy pays
// more than the staging). Validity and Ghost Wall flags are per-lane bit masks
// (pixel lane + 32k is bit k); the tile state is warp-uniform registers.
// Arithmetic and summation order are those of solve_kernel (and of the CPU
// restatement), so every kernel gives the same bits.
//
// Two kernels share this code. The fast pass runs every task's common case
// (IC-GN with whole-subset iterations) and hands every other task (AUTO
// mode, a masked iteration, a NO_SEARCH rescue) to a list; the rescue pass
// runs those tasks from the start with every path.
//
// Shared memory per warp: the TMA barrier at 0, the whole-subset step matrix
// (36 doubles) at 64, the masked-iteration step matrix at 352, the tile at
// off_tile, then vals[n] and (STAGE) rn[n], gx[n], gy[n].
constexpr int kFastMaxPerLane = 64;  // n <= 2048 (subset <= 45); larger subsets go to solve_kernel
constexpr int kFastMaxSmem = 227 * 1024;

struct StagedLayout {
    int tile_w, tile_h;  // the tile box the layout holds
    int off_tile, off_vals, off_rn, off_gx, off_gy;
    int off_coop;  // the cooperative rescue's request block and guard bits (0: none)
    int bytes;     // per warp (per block for the cooperative rescue), a multiple of 128
};

// The cooperative rescue: warp 0 of a block drives a task, and every warp of
// the block samples a share of the subset for each evaluation; the masked
// iteration's Hessian and its inversion run on the other warps.
constexpr int kCoopWarps = 8;
struct CoopReq {
    // 0: done, 1: sample, 2: coarse search, 3: stage the reference subset,
    // 4: masked-iteration step matrix, 5: ZNSSD residuals
    int op;
    int cx, cy, tile_ok, tx0, ty0;
    float Wp[6];
    float mref, iref;
    float mean, inv, sdev;  // op 5: the warped subset's statistics
    int full;
};
// The request block's layout: request, guard bits (kCoopWarps x 32 masks),
// coarse-search slots, the masked Hessian's 21 sums, its flags, and the
// scratch of the two warps that invert it.
constexpr int kCoopGbits = 128;
static_assert(sizeof(CoopReq) <= kCoopGbits, "request block");
constexpr int kCoopSlots = kCoopGbits + kCoopWarps * 32 * 8;
constexpr int kCoopHsum = kCoopSlots + kCoopWarps * 8;
constexpr int kCoopFlags = kCoopHsum + 176;
constexpr int kCoopScrCond = kCoopFlags + 16;        // 36 + 180 doubles
constexpr int kCoopScrInv = kCoopScrCond + 216 * 8;  // 36 + 72 doubles
constexpr int kCoopBytes = kCoopScrInv + 108 * 8;
static_assert(kCoopHsum % 8 == 0 && kCoopScrCond % 8 == 0, "double alignment");

// stage false: no staged reference subset (the solver reads the planes);
// coop: room for the cooperative rescue's request block
StagedLayout staged_layout(int n, int tw, int th, bool stage = true, bool coop = false) {
    StagedLayout L;
    L.tile_w = tw;
    L.tile_h = th;
    // the block's header (barrier, wait record, step matrix; with coop the
    // masked-iteration matrix too) ahead of the 128-byte aligned tile; 512
    // bytes without coop lets subset 31's fast pass hold 19 warps per SM
    L.off_tile = coop ? 640 : 512;
    int p = L.off_tile + ((tw * th * 4 + 127) & ~127);
    const int arr = (n * 4 + 15) & ~15;
    L.off_vals = p;
    p += arr;
    L.off_rn = L.off_gx = L.off_gy = p;
    if (stage) {
        L.off_rn = p;
        p += arr;
        L.off_gx = p;
        p += arr;
        L.off_gy = p;
        p += arr;
    }
    L.off_coop = 0;
    if (coop) {
        p = (p + 127) & ~127;
        L.off_coop = p;
        p += kCoopBytes;
    }
    L.bytes = (p + 127) & ~127;
    return L;
}

__device__ __forceinline__ void coop_bar() { asm volatile("bar.sync 1, %0;" ::"n"(kCoopWarps * 32) : "memory"); }

template <bool SIX, class Mask = uint64_t, bool STAGE = true, bool COOP = false>
struct WarpSolver {
    // this warp's shared memory
    uint64_t* bar;
    double* Hr;
    double* Hm;
    float* tile;
    float* vals;
    float* srn;
    float* sgx;
    float* sgy;
    const CUtensorMap* tmap;
    // launch constants
    const float* refI;
    const float* refGx;
    const float* refGy;
    const float* defI;
    int* err;
    int n, dim, half, pitch, tw, th, W, H, K, q, r, row0, col0, lane, min_valid, lm;
    int ref_pitch, ref_dx, ref_dy;  // where the reference subset is read (SolveArgs)
    // the TMA tile (warp-uniform)
    int tx0, ty0;
    bool tile_ok, tile_on;
    // every corner of the warped subset inside the 4 px guard with 0.01 px to
    // spare (so every sample is inside it too, rounding included); set by
    // ensure_tile
    bool all_in;
    Mask fullmask;  // bit k set when pixel lane + 32 k exists
    bool no_ghost;  // no reference pixel is a Ghost Wall pixel (launch constant)
    unsigned phase;
    // the task
    int cx, cy, ref_base, ghost;
    float mref, iref, lo_x, hi_x, lo_y, hi_y;
    Mask refok;
    // COOP: the block's request block, guard bits (kCoopWarps x 32) and
    // coarse-search slots, and this warp's index in the block
    CoopReq* req;
    Mask* gbits;
    float2* cslots;
    double* hsum;  // the masked Hessian's upper triangle (21)
    int* mflags;   // [0] 2x2 test, [1] conditioning, [2] inversion
    double* scr_cond;
    double* scr_inv;
    int warp;

    __device__ __forceinline__ void advance(int& row, int& col) const {
        col += r;
        row += q;
        if (col >= dim) {
            col -= dim;
            ++row;
        }
    }

    // The reference subset at pixel i (row, col): from the staged copy, or
    // (STAGE false) from the planes, normalised the same way.
    __device__ __forceinline__ float rn_at(int i, int row, int col) const {
        if constexpr (STAGE)
            return srn[i];
        else
            return (__ldg(refI + ref_base + row * ref_pitch + col) - mref) * iref;
    }
    __device__ __forceinline__ float gx_at(int i, int row, int col) const {
        if constexpr (STAGE)
            return sgx[i];
        else
            return __ldg(refGx + ref_base + row * ref_pitch + col);
    }
    __device__ __forceinline__ float gy_at(int i, int row, int col) const {
        if constexpr (STAGE)
            return sgy[i];
        else
            return __ldg(refGy + ref_base + row * ref_pitch + col);
    }

    // Per task: the step matrix from the pool, the reference subset staged
    // and normalised, the Ghost Wall flags and count.
    __device__ __forceinline__ void begin(const dic_task& T, float2 ms, const double* Hs21) {
        cx = T.cx;
        cy = T.cy;
        mref = ms.x;
        iref = 1.0f / ms.y;
        lo_x = (float)(4 - cx);
        hi_x = (float)(W - 4 - cx);
        lo_y = (float)(4 - cy);
        hi_y = (float)(H - 4 - cy);
        // the whole-subset step matrix (optimization_engine.cpp:302-315), from the pool
        for (int k = lane; k < 36; k += 32) {
            const int rr = k / 6, cc = k % 6;
            Hr[k] = Hs21[rr <= cc ? tri21(rr, cc) : tri21(cc, rr)];
        }
        ref_base = (cy - half + ref_dy) * ref_pitch + (cx - half + ref_dx);
        if constexpr (COOP) {
            // every warp of the block stages a share of the subset
            const int per = (K + kCoopWarps - 1) / kCoopWarps;
            coop_post(3, nullptr);
            int g = 0;
            Mask bits = stage_part(0, min(K, per), g);
            g = wsum(g);
            coop_bar();
#pragma unroll
            for (int w = 1; w < kCoopWarps; ++w) {
                bits |= gbits[w * 32 + lane];
                g += (int)cslots[w].x;
            }
            refok = bits;
            ghost = g;
            __syncwarp();
            return;
        }
        if constexpr (!STAGE) {
            if (no_ghost) {
                // nothing to stage and nothing to count: every pixel is valid reference
                refok = fullmask;
                ghost = 0;
                return;
            }
        }
        int g = 0;
        refok = stage_part(0, K, g);
        ghost = wsum(g);
        __syncwarp();
    }

    // The reference pixels k in [k_lo, k_hi) of this lane: their non-Ghost
    // bits returned, their Ghost count added to g, and (STAGE) the subset
    // staged normalised with its raw gradients.
    __device__ __forceinline__ Mask stage_part(int k_lo, int k_hi, int& g) {
        Mask bits = 0;
        const int i0 = lane + 32 * k_lo;
        int row = i0 / dim, col = i0 - (i0 / dim) * dim;
#pragma unroll 4
        for (int k = k_lo; k < k_hi; ++k) {
            const int i = lane + 32 * k;
            if (i < n) {
                const int idx = ref_base + row * ref_pitch + col;
                const float I = __ldg(refI + idx);
                if (I < kGhost)
                    ++g;
                else
                    bits |= Mask(1) << k;
                if constexpr (STAGE) {
                    srn[i] = (I - mref) * iref;
                    sgx[i] = __ldg(refGx + idx);
                    sgy[i] = __ldg(refGy + idx);
                }
            }
            advance(row, col);
        }
        return bits;
    }

    // The tile must cover every sample support of the warped subset: stage a
    // new box with TMA when the warp has left the current one.
    __device__ __forceinline__ void ensure_tile(const float Wp[6]) {
        all_in = false;
        if (!tile_on) return;
        const float h = (float)half;
        float mnx = 0.0f, mxx = 0.0f, mny = 0.0f, mxy = 0.0f;
        bool in_range = true;  // every corner finite and within 1e6 px (a NaN fails the comparisons)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float ox = (k & 1) ? h : -h, oy = (k & 2) ? h : -h;
            const float fx = __fmaf_rn(Wp[0], ox, __fmaf_rn(Wp[1], oy, Wp[2]));
            const float fy = __fmaf_rn(Wp[3], ox, __fmaf_rn(Wp[4], oy, Wp[5]));
            in_range = in_range && fx > -1e6f && fx < 1e6f && fy > -1e6f && fy < 1e6f;
            mnx = k ? fminf(mnx, fx) : fx;
            mxx = k ? fmaxf(mxx, fx) : fx;
            mny = k ? fminf(mny, fy) : fy;
            mxy = k ? fmaxf(mxy, fy) : fy;
        }
        if (!in_range) {
            tile_ok = false;
            return;
        }
        all_in = mnx + 0.5f >= lo_x + 0.01f && mxx + 0.5f < hi_x - 0.01f && mny + 0.5f >= lo_y + 0.01f &&
                 mxy + 0.5f < hi_y - 0.01f;
        const int lo_tap = SIX ? 3 : 2, hi_tap = SIX ? 4 : 3;
        const int x_lo = cx + (int)floorf(mnx) - lo_tap, x_hi = cx + (int)floorf(mxx) + hi_tap;
        const int y_lo = cy + (int)floorf(mny) - lo_tap, y_hi = cy + (int)floorf(mxy) + hi_tap;
        if (tile_ok && x_lo >= tx0 && x_hi < tx0 + tw && y_lo >= ty0 && y_hi < ty0 + th) return;
        const int need_w = x_hi - x_lo + 1, need_h = y_hi - y_lo + 1;
        if (need_w + 3 > tw || need_h > th) {
            tile_ok = false;
            return;
        }
        // centre the support, x start on a 16-byte boundary (a multiple of 4)
        int nx = x_lo - (tw - 3 - need_w) / 2;
        nx = nx >= 0 ? (nx & ~3) : -((-nx + 3) & ~3);
        const int ny = y_lo - (th - need_h) / 2;
        __syncwarp();  // every lane is done with the old tile
        if (lane == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, (uint32_t)(tw * th * 4));
            tma_load_2d(tile, tmap, nx, ny, bar);
        }
        int* const aux = reinterpret_cast<int*>(bar + 1);  // [max polls, pending, pending parity]
        const bool done = __all_sync(kFull, mbar_wait_bounded(bar, phase, aux[0]));
        if (done) {
            tx0 = nx;
            ty0 = ny;
            tile_ok = true;
        } else {
            // a copy that has not completed: stop staging for this warp
            tile_ok = false;
            tile_on = false;
            if (lane == 0) {
                aux[1] = 1;
                aux[2] = (int)phase;
                if (err) atomicExch(err, 1);
            }
            __syncwarp();
        }
        phase ^= 1u;
    }

    // Before the warp exits: a copy whose wait ran out may still be writing
    // into the tile; wait for it (bounded) so that it lands before the block's
    // shared memory is released.
    __device__ __forceinline__ void drain() {
        const int* const aux = reinterpret_cast<const int*>(bar + 1);
        __syncwarp();
        if (aux[1]) (void)__all_sync(kFull, mbar_wait_bounded(bar, (unsigned)aux[2], kTmaPolls));
    }

    // The pixels k in [k_lo, k_hi) of this lane (i = lane + 32 k): their
    // values into vals and the guard bits (inside the 4 px guard) returned.
    // Four pixels' loads are issued before their stores.
    __device__ __forceinline__ Mask sample_part(const float Wp[6], int k_lo, int k_hi) {
        Mask g = 0;
        const int i0 = lane + 32 * k_lo;
        int row = i0 / dim, col = i0 - (i0 / dim) * dim;
        for (int k0 = k_lo; k0 < k_hi; k0 += 4) {
            float v[4];
            int ii[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u;
                ii[u] = lane + 32 * k;
                v[u] = 0.0f;
                if (k < k_hi && ii[u] < n) {
                    const float ox = (float)(col - half), oy = (float)(row - half);
                    const float fx = __fmaf_rn(Wp[0], ox, __fmaf_rn(Wp[1], oy, Wp[2]));
                    const float fy = __fmaf_rn(Wp[3], ox, __fmaf_rn(Wp[4], oy, Wp[5]));
                    const float rx = fx + 0.5f, ry = fy + 0.5f;
                    if (rx >= lo_x && rx < hi_x && ry >= lo_y && ry < hi_y) {
                        const float flx = floorf(fx), fly = floorf(fy);
                        const int xi = cx + (int)flx, yi = cy + (int)fly;
                        const int lx = xi - tx0, ly = yi - ty0;
                        if (tile_ok)
                            v[u] = SIX ? interp6s(tile, tw, lx, ly, fx - flx, fy - fly)
                                       : interp4s(tile, tw, lx, ly, fx - flx, fy - fly);
                        else
                            v[u] = SIX ? interp6(defI, pitch, xi, yi, fx - flx, fy - fly)
                                       : interp4(defI, pitch, xi, yi, fx - flx, fy - fly);
                        g |= Mask(1) << k;
                    }
                }
                advance(row, col);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u < k_hi && ii[u] < n) vals[ii[u]] = v[u];
        }
        return g;
    }

    // COOP, warps 1..: serve the driver's requests until it is done.
    __device__ void coop_serve() {
        const int per = (K + kCoopWarps - 1) / kCoopWarps;
        for (;;) {
            coop_bar();  // a request is posted
            const int op = req->op;
            if (op == 0) break;
            cx = req->cx;
            cy = req->cy;
            lo_x = (float)(4 - cx);
            hi_x = (float)(W - 4 - cx);
            lo_y = (float)(4 - cy);
            hi_y = (float)(H - 4 - cy);
            ref_base = (cy - half + ref_dy) * ref_pitch + (cx - half + ref_dx);
            if (op == 5) {
                const int lo = warp * per, hi = min(K, lo + per);
                residual_part(lo, hi, gbits[lane], req->mean, req->inv, req->sdev, req->full != 0);
            } else if (op == 4) {
                masked_serve();
            } else if (op == 3) {
                mref = req->mref;
                iref = req->iref;
                const int lo = warp * per, hi = min(K, lo + per);
                int g = 0;
                gbits[warp * 32 + lane] = lo < hi ? stage_part(lo, hi, g) : Mask(0);
                g = wsum(g);
                if (lane == 0) cslots[warp] = make_float2((float)g, 0.0f);
            } else if (op == 1) {
                tile_ok = req->tile_ok != 0;
                tx0 = req->tx0;
                ty0 = req->ty0;
                float Wp[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) Wp[k] = req->Wp[k];
                const int lo = warp * per, hi = min(K, lo + per);
                gbits[warp * 32 + lane] = lo < hi ? sample_part(Wp, lo, hi) : Mask(0);
            } else {
                coarse_warp(warp * 32 + lane);
            }
            coop_bar();  // results in shared memory
        }
    }

    // COOP, the driver: post a request; the caller's own share follows.
    __device__ __forceinline__ void coop_post(int op, const float* Wp) {
        if (lane == 0) {
            req->op = op;
            req->cx = cx;
            req->cy = cy;
            req->tile_ok = tile_ok ? 1 : 0;
            req->tx0 = tx0;
            req->ty0 = ty0;
            req->mref = mref;
            req->iref = iref;
            if (Wp)
                for (int k = 0; k < 6; ++k) req->Wp[k] = Wp[k];
        }
        __syncwarp();
        coop_bar();
    }

    // sample_warped_subset (optimization_engine.cpp:191-269): every pixel's
    // value into vals, the valid ones (inside the guard, outside the Ghost
    // Wall) flagged in `valid` and summed in pixel order; returns their count.
    __device__ __forceinline__ int sample(const float Wp[6], float& sum, Mask& valid) {
        ensure_tile(Wp);
        if constexpr (COOP) {
            const int per = (K + kCoopWarps - 1) / kCoopWarps;
            coop_post(1, Wp);
            Mask g = sample_part(Wp, 0, min(K, per));
            coop_bar();
#pragma unroll
            for (int w = 1; w < kCoopWarps; ++w) g |= gbits[w * 32 + lane];
            valid = g & refok;
            const float part = vals_chain(valid, 0.0f, [](float v, float a) { return a + v; });
            sum = wsum(part);
            return wsum(__popcll((unsigned long long)valid));
        }
        if constexpr (!STAGE && !COOP) {
            // the fast pass's common case: every sample inside the guard and
            // the tile, no Ghost Wall pixel, so every pixel is valid and the
            // per-pixel tests are skipped (same values, same order of sums)
            if (all_in && tile_ok && ghost == 0) {
                float part = 0.0f;
                int row = row0, col = col0;
                if (!SIX && dim == 31) {
                    // Subset 31: lane c samples column c of every row (lane 31
                    // idle), two rows per paired FP32 instruction, so the taps
                    // of a warp lie on one tile row and hit 31 distinct banks
                    // (the sums' layout puts a 32nd pixel on the next row,
                    // which the tile's 16-byte row pitch makes collide). The
                    // values go to vals; the ordered sum then reads them in
                    // the sums' layout.
                    const float2 W0 = f2(Wp[0]), W1 = f2(Wp[1]), W2 = f2(Wp[2]);
                    const float2 W3 = f2(Wp[3]), W4 = f2(Wp[4]), W5 = f2(Wp[5]);
                    const int bx = cx - tx0, by = cy - ty0;
                    const bool act = lane < 31;
                    const float2 OX = f2((float)((act ? lane : half) - half));
#pragma unroll 2
                    for (int r0 = 0; r0 < 31; r0 += 2) {
                        const int r1 = r0 + 1 < 31 ? r0 + 1 : r0;
                        const float2 OY = make_float2((float)(r0 - half), (float)(r1 - half));
                        const float2 FX = __ffma2_rn(W0, OX, __ffma2_rn(W1, OY, W2));
                        const float2 FY = __ffma2_rn(W3, OX, __ffma2_rn(W4, OY, W5));
                        const float2 FLX = make_float2(floorf(FX.x), floorf(FX.y));
                        const float2 FLY = make_float2(floorf(FY.x), floorf(FY.y));
                        const float2 V = interp4s_x2(tile, tw, bx + (int)FLX.x, by + (int)FLY.x, bx + (int)FLX.y,
                                                     by + (int)FLY.y, __ffma2_rn(FLX, f2(-1.0f), FX),
                                                     __ffma2_rn(FLY, f2(-1.0f), FY));
                        if (act) {
                            vals[r0 * 31 + lane] = V.x;
                            if (r1 != r0) vals[r1 * 31 + lane] = V.y;
                        }
                    }
                    __syncwarp();
#pragma unroll 8
                    for (int k = 0; k < K; ++k) {
                        const int i = lane + 32 * k;
                        if (i < n) part = part + vals[i];
                    }
                } else if constexpr (!SIX) {
                    // two pixels per paired FP32 instruction; a pixel past
                    // the subset samples the centre (inside the tile) and is
                    // dropped
                    const float2 W0 = f2(Wp[0]), W1 = f2(Wp[1]), W2 = f2(Wp[2]);
                    const float2 W3 = f2(Wp[3]), W4 = f2(Wp[4]), W5 = f2(Wp[5]);
                    const int bx = cx - tx0, by = cy - ty0;
                    constexpr int PG = 8;  // pixels in flight per lane
                    for (int k0 = 0; k0 < K; k0 += PG) {
                        float v[PG], ox[PG], oy[PG];
                        int ii[PG];
                        bool ok[PG];
#pragma unroll
                        for (int u = 0; u < PG; ++u) {
                            const int k = k0 + u;
                            ii[u] = lane + 32 * k;
                            ok[u] = k < K && ii[u] < n;
                            ox[u] = ok[u] ? (float)(col - half) : 0.0f;
                            oy[u] = ok[u] ? (float)(row - half) : 0.0f;
                            advance(row, col);
                        }
#pragma unroll
                        for (int u = 0; u < PG; u += 2) {
                            const float2 OX = make_float2(ox[u], ox[u + 1]), OY = make_float2(oy[u], oy[u + 1]);
                            const float2 FX = __ffma2_rn(W0, OX, __ffma2_rn(W1, OY, W2));
                            const float2 FY = __ffma2_rn(W3, OX, __ffma2_rn(W4, OY, W5));
                            const float2 FLX = make_float2(floorf(FX.x), floorf(FX.y));
                            const float2 FLY = make_float2(floorf(FY.x), floorf(FY.y));
                            // fx - floor(fx) as one rounding: fma(floor, -1, fx)
                            const float2 V = interp4s_x2(tile, tw, bx + (int)FLX.x, by + (int)FLY.x, bx + (int)FLX.y,
                                                         by + (int)FLY.y, __ffma2_rn(FLX, f2(-1.0f), FX),
                                                         __ffma2_rn(FLY, f2(-1.0f), FY));
                            v[u] = V.x;
                            v[u + 1] = V.y;
                        }
#pragma unroll
                        for (int u = 0; u < PG; ++u)
                            if (ok[u]) {
                                part = part + v[u];
                                vals[ii[u]] = v[u];
                            }
                    }
                } else {
                    for (int k0 = 0; k0 < K; k0 += 4) {
                        float v[4];
                        int ii[4];
#pragma unroll
                        for (int u = 0; u < 4; ++u) {
                            const int k = k0 + u;
                            ii[u] = lane + 32 * k;
                            v[u] = 0.0f;
                            if (k < K && ii[u] < n) {
                                const float ox = (float)(col - half), oy = (float)(row - half);
                                const float fx = __fmaf_rn(Wp[0], ox, __fmaf_rn(Wp[1], oy, Wp[2]));
                                const float fy = __fmaf_rn(Wp[3], ox, __fmaf_rn(Wp[4], oy, Wp[5]));
                                const float flx = floorf(fx), fly = floorf(fy);
                                const int lx = cx + (int)flx - tx0, ly = cy + (int)fly - ty0;
                                v[u] = interp6s(tile, tw, lx, ly, fx - flx, fy - fly);
                                part = part + v[u];
                            }
                            advance(row, col);
                        }
#pragma unroll
                        for (int u = 0; u < 4; ++u)
                            if (k0 + u < K && ii[u] < n) vals[ii[u]] = v[u];
                    }
                }
                __syncwarp();
                valid = fullmask;
                sum = wsum(part);
                return n;
            }
        }

        float part = 0.0f;
        int cnt = 0;
        valid = 0;
        int row = row0, col = col0;
        for (int k0 = 0; k0 < K; k0 += 4) {
            float v[4];
            int ii[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + u;
                ii[u] = lane + 32 * k;
                v[u] = 0.0f;
                if (k < K && ii[u] < n) {
                    const float ox = (float)(col - half), oy = (float)(row - half);
                    const float fx = __fmaf_rn(Wp[0], ox, __fmaf_rn(Wp[1], oy, Wp[2]));
                    const float fy = __fmaf_rn(Wp[3], ox, __fmaf_rn(Wp[4], oy, Wp[5]));
                    const float rx = fx + 0.5f, ry = fy + 0.5f;
                    if (rx >= lo_x && rx < hi_x && ry >= lo_y && ry < hi_y) {
                        const float flx = floorf(fx), fly = floorf(fy);
                        const int xi = cx + (int)flx, yi = cy + (int)fly;
                        const int lx = xi - tx0, ly = yi - ty0;
                        // a staged tile covers every sample support: ensure_tile sized it from
                        // the warped corners, which bound every interior sample, with a pixel
                        // of slack each side for the rounding of the corner positions
                        if (tile_ok)
                            v[u] = SIX ? interp6s(tile, tw, lx, ly, fx - flx, fy - fly)
                                       : interp4s(tile, tw, lx, ly, fx - flx, fy - fly);
                        else
                            v[u] = SIX ? interp6(defI, pitch, xi, yi, fx - flx, fy - fly)
                                       : interp4(defI, pitch, xi, yi, fx - flx, fy - fly);
                        if ((refok >> k) & 1u) {
                            valid |= Mask(1) << k;
                            part = part + v[u];
                            ++cnt;
                        }
                    }
                }
                advance(row, col);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (k0 + u < K && ii[u] < n) vals[ii[u]] = v[u];
        }
        __syncwarp();
        sum = wsum(part);
        return wsum(cnt);
    }

    // COOP: this lane's ordered chain over vals, acc = f(vals[lane + 32 k],
    // acc) for the valid pixels in increasing k, eight values loaded ahead of
    // their eight steps so that the loads do not wait on the chain.
    template <class F>
    __device__ __forceinline__ float vals_chain(Mask valid, float acc, F&& f) const {
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 8) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int i = lane + 32 * (k0 + u);
                v[u] = k0 + u < K ? vals[i < n ? i : n - 1] : 0.0f;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (k0 + u < K && ((valid >> (k0 + u)) & 1u)) acc = f(v[u], acc);
        }
        return acc;
    }

    __device__ __forceinline__ float sum_sq(float mean, Mask valid) const {
        float sq = 0.0f;
        if constexpr (COOP) {
            sq = vals_chain(valid, 0.0f, [&](float v, float a) {
                const float d = v - mean;
                return __fmaf_rn(d, d, a);
            });
        } else {
#pragma unroll 4
            for (int k = 0; k < K; ++k) {
                if (!((valid >> k) & 1u)) continue;
                const float d = vals[lane + 32 * k] - mean;
                sq = __fmaf_rn(d, d, sq);
            }
        }
        return wsum(sq);
    }

    // The masked iteration's own Hessian (optimization_engine.cpp:373-413),
    // FP64, into Hm; false to reject.
    __device__ __forceinline__ bool masked_step(Mask valid) {
        double hp[21];
#pragma unroll
        for (int k = 0; k < 21; ++k) hp[k] = 0.0;
        int row = row0, col = col0;
        for (int k = 0; k < K; ++k) {
            if ((valid >> k) & 1u) {
                const int i = lane + 32 * k;
                const float g0 = gx_at(i, row, col) * iref, g1 = gy_at(i, row, col) * iref;
                const float fx = (float)(col - half), fy = (float)(row - half);
                const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                                     (double)(g1 * fx), (double)(g1 * fy)};
                int m = 0;
#pragma unroll
                for (int aa = 0; aa < 6; ++aa)
#pragma unroll
                    for (int bb = aa; bb < 6; ++bb, ++m) hp[m] = __fma_rn(s[aa], s[bb], hp[m]);
            }
            advance(row, col);
        }
#pragma unroll
        for (int k = 0; k < 21; ++k) hp[k] = wsum(hp[k]);
        int ok = 0;
        if (lane == 0) {
            double Hd[6][6], Hi[6][6];
            for (int aa = 0; aa < 6; ++aa)
                for (int bb = aa; bb < 6; ++bb) {
                    Hd[aa][bb] = hp[tri21(aa, bb)];
                    Hd[bb][aa] = Hd[aa][bb];
                }
            if (cond2x2_ok(Hd)) {
                if (lm) {
                    Hd[0][0] += (double)kLmAlpha;
                    Hd[1][1] += (double)kLmAlpha;
                }
                if (well_conditioned(Hd, half) && inverse6(Hd, Hi)) {
                    for (int aa = 0; aa < 6; ++aa)
                        for (int bb = 0; bb < 6; ++bb) Hm[aa * 6 + bb] = Hi[aa][bb];
                    ok = 1;
                }
            }
        }
        ok = __shfl_sync(kFull, ok, 0);
        __syncwarp();
        return ok != 0;
    }

    // COOP, warps 1..7: three of the masked Hessian's 21 sums (upper-triangle
    // entries M0..M0+2), each with the operations and order of masked_step.
    template <int M0>
    __device__ __forceinline__ void masked_sums3(Mask valid) {
        constexpr int a0 = tri_row(M0), b0 = tri_col(M0), a1 = tri_row(M0 + 1), b1 = tri_col(M0 + 1);
        constexpr int a2 = tri_row(M0 + 2), b2 = tri_col(M0 + 2);
        double h0 = 0.0, h1 = 0.0, h2 = 0.0;
        int row = row0, col = col0;
#pragma unroll 4
        for (int k = 0; k < K; ++k) {
            if ((valid >> k) & 1u) {
                const int i = lane + 32 * k;
                const float g0 = gx_at(i, row, col) * iref, g1 = gy_at(i, row, col) * iref;
                const float fx = (float)(col - half), fy = (float)(row - half);
                const double s[6] = {(double)g0, (double)g1, (double)(g0 * fx), (double)(g0 * fy),
                                     (double)(g1 * fx), (double)(g1 * fy)};
                h0 = __fma_rn(s[a0], s[b0], h0);
                h1 = __fma_rn(s[a1], s[b1], h1);
                h2 = __fma_rn(s[a2], s[b2], h2);
            }
            advance(row, col);
        }
        h0 = wsum(h0);
        h1 = wsum(h1);
        h2 = wsum(h2);
        if (lane == 0) {
            hsum[M0] = h0;
            hsum[M0 + 1] = h1;
            hsum[M0 + 2] = h2;
        }
    }

    // COOP, warps 1..7: the masked iteration's step matrix (masked_step's
    // Hessian, tests and inverse) into Hm, its verdicts into mflags. Warp 1
    // runs the 2x2 test and the conditioning, warp 2 the inversion, at the
    // same time.
    __device__ void masked_serve() {
        const Mask valid = gbits[lane];
        switch (warp) {
            case 1: masked_sums3<0>(valid); break;
            case 2: masked_sums3<3>(valid); break;
            case 3: masked_sums3<6>(valid); break;
            case 4: masked_sums3<9>(valid); break;
            case 5: masked_sums3<12>(valid); break;
            case 6: masked_sums3<15>(valid); break;
            default: masked_sums3<18>(valid); break;
        }
        asm volatile("bar.sync 2, %0;" ::"n"((kCoopWarps - 1) * 32) : "memory");
        if (warp != 1 && warp != 2) return;
        double* Hd = warp == 1 ? scr_cond : scr_inv;
        for (int e = lane; e < 36; e += 32) {
            const int rr = e / 6, cc = e - (e / 6) * 6;
            double h = hsum[rr <= cc ? tri21(rr, cc) : tri21(cc, rr)];
            if (lm && rr == cc && rr < 2) h += (double)kLmAlpha;
            Hd[e] = h;
        }
        __syncwarp();
        if (warp == 1) {
            if (lane == 0) {
                double H2[6][6];
                H2[0][0] = hsum[tri21(0, 0)];
                H2[0][1] = H2[1][0] = hsum[tri21(0, 1)];
                H2[1][1] = hsum[tri21(1, 1)];
                mflags[0] = cond2x2_ok(H2) ? 1 : 0;
            }
            const bool wc = well_conditioned_warp(Hd, half, scr_cond + 36);
            if (lane == 0) mflags[1] = wc ? 1 : 0;
        } else {
            bool factored;
            const bool ok = inverse6_warp(Hd, Hm, scr_inv + 36, factored);
            if (lane == 0) mflags[2] = ok ? 1 : 0;
        }
    }

    // solve_icgn (optimization_engine.cpp:272-465). With GENERAL false a
    // masked iteration is not taken: `defer` is set instead.
    template <bool GENERAL>
    __device__ __forceinline__ Res icgn(const float st[6], bool& defer) {
        float Wp[6] = {1.0f + st[2], st[3], st[0], st[4], 1.0f + st[5], st[1]};
        float final_score = 1.0f;
        for (int iter = 0; iter < kIcgnMaxIter; ++iter) {
            float sum;
            Mask valid;
            const int cnt = sample(Wp, sum, valid);
            if (cnt < min_valid) return res_from(Wp, 1, 2.0f, iter);
            const bool full = cnt == n;
            if constexpr (!GENERAL) {
                if (!full) {
                    defer = true;
                    return res_from(Wp, 1, 2.0f, iter);
                }
            }
            if constexpr (GENERAL && COOP) {
                // the other warps form the masked iteration's step matrix
                // while this one forms the residual sums
                if (!full) {
                    gbits[lane] = valid;
                    coop_post(4, nullptr);
                }
            }
            const float mean = sum / (float)cnt;
            float sdev = sqrtf(sum_sq(mean, valid) / (float)cnt);
            if (sdev < 1e-5f) sdev = 1.0f;
            const float inv = 1.0f / sdev;

            float ep = 0.0f, gp0 = 0.0f, gp1 = 0.0f, gp2 = 0.0f, gp3 = 0.0f, gp4 = 0.0f, gp5 = 0.0f;
            // the texture check's sums of the raw gradients over the same valid
            // pixels in the same order, taken here where the gradients are
            // loaded anyway (reference read from the planes)
            float tsx = 0.0f, tsy = 0.0f;
            if constexpr (STAGE) {
                int row = row0, col = col0;
#pragma unroll 4
                for (int k = 0; k < K; ++k) {
                    if ((valid >> k) & 1u) {
                        const int i = lane + 32 * k;
                        const float diff = srn[i] - (vals[i] - mean) * inv;
                        const float g0 = sgx[i] * iref, g1 = sgy[i] * iref;
                        const float fx = (float)(col - half), fy = (float)(row - half);
                        ep = __fmaf_rn(diff, diff, ep);
                        gp0 = __fmaf_rn(g0, diff, gp0);
                        gp1 = __fmaf_rn(g1, diff, gp1);
                        gp2 = __fmaf_rn(g0 * fx, diff, gp2);
                        gp3 = __fmaf_rn(g0 * fy, diff, gp3);
                        gp4 = __fmaf_rn(g1 * fx, diff, gp4);
                        gp5 = __fmaf_rn(g1 * fy, diff, gp5);
                    }
                    advance(row, col);
                }
            } else {
                // The reference comes from the planes (L2): the loads of the
                // next four pixels are issued before the current four are
                // summed, so their latency overlaps the arithmetic.
                constexpr int G = 4;
                float nI[G], nX[G], nY[G], nfx[G], nfy[G];
                int lr = row0, lc = col0;
                auto fetch = [&](int k0) {
#pragma unroll
                    for (int u = 0; u < G; ++u) {
                        const int k = k0 + u;
                        nI[u] = nX[u] = nY[u] = 0.0f;
                        nfx[u] = (float)(lc - half);
                        nfy[u] = (float)(lr - half);
                        if (k < K && lane + 32 * k < n) {
                            const int idx = ref_base + lr * ref_pitch + lc;
                            nI[u] = __ldg(refI + idx);
                            nX[u] = __ldg(refGx + idx);
                            nY[u] = __ldg(refGy + idx);
                        }
                        advance(lr, lc);
                    }
                };
                // One pixel's share of the residual and steepest-descent sums,
                // independent sums in pairs on the paired FP32 instructions:
                // (tsx, tsy), (gp0, gp1), (gp2, gp4), (gp3, gp5). Per sum:
                // ts += g g; rn = (I - mref) iref; nd = (v - mean) inv;
                // diff = rn - nd; ep += diff^2; gp0 += g0 diff, gp1 += g1 diff,
                // gp2 += (g0 fx) diff, gp3 += (g0 fy) diff, gp4 += (g1 fx)
                // diff, gp5 += (g1 fy) diff, with g0 = gx iref, g1 = gy iref.
                float2 TS = f2(0.0f), GP01 = f2(0.0f), GP24 = f2(0.0f), GP35 = f2(0.0f);
                const float2 NEG = make_float2(-mref, -mean), SCL = make_float2(iref, inv);
                auto accumulate2 = [&](int i, float I, float gx, float gy, float fx, float fy) {
                    const float2 GXY = make_float2(gx, gy);
                    TS = __ffma2_rn(GXY, GXY, TS);
                    // (rn, nd) = ((I - mref) * iref, (vals[i] - mean) * inv)
                    const float2 RN = __fmul2_rn(__fadd2_rn(make_float2(I, vals[i]), NEG), SCL);
                    const float diff = RN.x - RN.y;
                    const float2 G01 = __fmul2_rn(GXY, f2(iref));  // (g0, g1)
                    const float2 D = f2(diff);
                    ep = __fmaf_rn(diff, diff, ep);
                    GP01 = __ffma2_rn(G01, D, GP01);
                    GP24 = __ffma2_rn(__fmul2_rn(G01, f2(fx)), D, GP24);  // (g0 fx, g1 fx)
                    GP35 = __ffma2_rn(__fmul2_rn(G01, f2(fy)), D, GP35);  // (g0 fy, g1 fy)
                };
                fetch(0);
                for (int k0 = 0; k0 < K; k0 += G) {
                    float cI[G], cX[G], cY[G], cfx[G], cfy[G];
#pragma unroll
                    for (int u = 0; u < G; ++u) {
                        cI[u] = nI[u];
                        cX[u] = nX[u];
                        cY[u] = nY[u];
                        cfx[u] = nfx[u];
                        cfy[u] = nfy[u];
                    }
                    if (k0 + G < K) fetch(k0 + G);
#pragma unroll
                    for (int u = 0; u < G; ++u) {
                        const int k = k0 + u;
                        if (k < K && ((valid >> k) & 1u)) accumulate2(lane + 32 * k, cI[u], cX[u], cY[u], cfx[u], cfy[u]);
                    }
                }
                tsx = TS.x;
                tsy = TS.y;
                gp0 = GP01.x;
                gp1 = GP01.y;
                gp2 = GP24.x;
                gp4 = GP24.y;
                gp3 = GP35.x;
                gp5 = GP35.y;
            }
            const float err2 = wsum(ep);
            const float g[6] = {wsum(gp0), wsum(gp1), wsum(gp2), wsum(gp3), wsum(gp4), wsum(gp5)};

            const double* Hstep = Hr;
            if constexpr (GENERAL) {
                if (!full) {
                    if constexpr (COOP) {
                        coop_bar();  // the step matrix is formed
                        if (!(mflags[0] && mflags[1] && mflags[2])) return res_from(Wp, 1, 2.0f, iter);
                    } else {
                        if (!masked_step(valid)) return res_from(Wp, 1, 2.0f, iter);
                    }
                    Hstep = Hm;
                }
            }
            final_score = err2 / (float)cnt;

            float dpl = 0.0f;
            if (lane < 6) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < 6; ++k) acc = __fma_rn(Hstep[lane * 6 + k], (double)g[k], acc);
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
            if (!fin || !(fabsf(det) > 1e-6f)) return res_from(Wp, 1, 2.0f, iter + 1);
            const float id = 1.0f / det;
            const float i00 = a11 * id, i01 = -a01 * id, i10 = -a10 * id, i11 = a00 * id;
            const float i02 = -(i00 * dp[0] + i01 * dp[1]);
            const float i12 = -(i10 * dp[0] + i11 * dp[1]);
            float Wn[6];
            Wn[0] = Wp[0] * i00 + Wp[1] * i10;
            Wn[1] = Wp[0] * i01 + Wp[1] * i11;
            Wn[2] = (Wp[0] * i02 + Wp[1] * i12) + Wp[2];
            Wn[3] = Wp[3] * i00 + Wp[4] * i10;
            Wn[4] = Wp[3] * i01 + Wp[4] * i11;
            Wn[5] = (Wp[3] * i02 + Wp[4] * i12) + Wp[5];
            bool wfin = true;
#pragma unroll
            for (int k = 0; k < 6; ++k) wfin = wfin && finite_f(Wn[k]);
            if (!wfin) return res_from(Wp, 1, 2.0f, iter + 1);
#pragma unroll
            for (int k = 0; k < 6; ++k) Wp[k] = Wn[k];

            float nn = dp[0] * dp[0];
#pragma unroll
            for (int k = 1; k < 6; ++k) nn = nn + dp[k] * dp[k];
            if (sqrtf(nn) < 0.001f) {
                // texture check on the raw reference gradients (optimization_engine.cpp:435-461)
                float sx = 0.0f, sy = 0.0f;
                if constexpr (STAGE) {
                    int row = row0, col = col0;
#pragma unroll 4
                    for (int k = 0; k < K; ++k) {
                        if ((valid >> k) & 1u) {
                            const int i = lane + 32 * k;
                            const float gx = sgx[i], gy = sgy[i];
                            sx = __fmaf_rn(gx, gx, sx);
                            sy = __fmaf_rn(gy, gy, sy);
                        }
                        advance(row, col);
                    }
                } else {
                    sx = tsx;  // this iteration's residual pass summed them
                    sy = tsy;
                }
                const float tx = wsum(sx), ty = wsum(sy);
                const float sg = ty < tx ? ty : tx;
                if (sg <= 0.0f || !finite_f(final_score)) return res_from(Wp, 1, 2.0f, iter + 1);
                return res_from(Wp, 0, final_score, iter + 1);
            }
        }
        return res_from(Wp, 1, final_score, kIcgnMaxIter);
    }

    // COOP: the ZNSSD residuals of pixels k in [k_lo, k_hi) of this lane, in
    // place of their values (evaluate_znssd's per-pixel difference).
    __device__ __forceinline__ void residual_part(int k_lo, int k_hi, Mask valid, float mean, float inv, float sdev,
                                                  bool full) {
        for (int k = k_lo; k < k_hi; ++k) {
            if ((valid >> k) & 1u) {
                const int i = lane + 32 * k;
                const float rn = srn[i];
                vals[i] = full ? rn - (vals[i] - mean) * inv : rn - (vals[i] - mean) / sdev;
            }
        }
    }

    // evaluate_znssd (optimization_engine.cpp:467-528).
    __device__ __forceinline__ float znssd(const float Wp[6]) {
        float sum;
        Mask valid;
        const int cnt = sample(Wp, sum, valid);
        if (cnt == 0 || cnt < min_valid) return 2.0f;
        const float mean = sum / (float)cnt;
        float sdev = sqrtf(sum_sq(mean, valid) / (float)cnt);
        if (sdev < 1e-5f) sdev = 1.0f;
        const bool full = cnt == n;
        const float inv = 1.0f / sdev;
        float ep = 0.0f;
        if constexpr (COOP) {
            // every warp forms the residuals of its share (each with its own
            // division), then this warp sums their squares in pixel order
            const int per = (K + kCoopWarps - 1) / kCoopWarps;
            gbits[lane] = valid;
            if (lane == 0) {
                req->mean = mean;
                req->inv = inv;
                req->sdev = sdev;
                req->full = full ? 1 : 0;
            }
            coop_post(5, nullptr);
            residual_part(0, min(K, per), valid, mean, inv, sdev, full);
            coop_bar();
            ep = vals_chain(valid, 0.0f, [](float d, float a) { return __fmaf_rn(d, d, a); });
            const float score = wsum(ep) / (float)cnt;
            return finite_f(score) ? score : 2.0f;
        }
        int row = row0, col = col0;
#pragma unroll 4
        for (int k = 0; k < K; ++k) {
            if ((valid >> k) & 1u) {
                const int i = lane + 32 * k;
                const float rn = rn_at(i, row, col);
                const float diff = full ? rn - (vals[i] - mean) * inv : rn - (vals[i] - mean) / sdev;
                ep = __fmaf_rn(diff, diff, ep);
            }
            advance(row, col);
        }
        const float score = wsum(ep) / (float)cnt;
        return finite_f(score) ? score : 2.0f;
    }

    // solve_simplex (optimization_engine.cpp:531-651). Every lane keeps the
    // same simplex; the evaluations are warp-collective.
    __device__ __forceinline__ Res simplex(float s0, float s1, float s2, float s3, float s4, float s5, bool trans) {
        const int D = trans ? 2 : 6, np = D + 1;
        float p[7][6];
        float y[7];
        for (int i = 0; i < 7; ++i) {
            y[i] = 0.0f;
            for (int j = 0; j < 6; ++j) p[i][j] = 0.0f;
        }
        const float scale[6] = {2.0f, 2.0f, 0.01f, 0.01f, 0.01f, 0.01f};
        auto eval = [&](const float* pt) {
            float Wq[6];
            if (trans) {
                Wq[0] = 1.0f; Wq[1] = 0.0f; Wq[2] = pt[0]; Wq[3] = 0.0f; Wq[4] = 1.0f; Wq[5] = pt[1];
            } else {
                Wq[0] = 1.0f + pt[2]; Wq[1] = pt[3]; Wq[2] = pt[0]; Wq[3] = pt[4]; Wq[4] = 1.0f + pt[5]; Wq[5] = pt[1];
            }
            return znssd(Wq);
        };
        p[0][0] = s0;
        p[0][1] = s1;
        if (!trans) {
            p[0][2] = s2;
            p[0][3] = s3;
            p[0][4] = s4;
            p[0][5] = s5;
        }
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
        Res res;
        res.u = p[best][0];
        res.v = p[best][1];
        res.ux = trans ? 0.0f : p[best][2];
        res.uy = trans ? 0.0f : p[best][3];
        res.vx = trans ? 0.0f : p[best][4];
        res.vy = trans ? 0.0f : p[best][5];
        res.status = y[best] > kSimplexFailScore ? -2 : 0;
        res.score = y[best];
        res.iters = 0;
        return res;
    }

    // estimate_initial_guess (optimization_engine.cpp:120-179) for one offset
    // (idx: v-major over the 16 x 16 grid of +-15 px in steps of 2) with the
    // reference's sequential sums over every 9th subset pixel; 1e20 when the
    // offset does not qualify.
    __device__ __forceinline__ float coarse_score(int idx, int sampled) const {
        const int v = -15 + 2 * (idx / 16), u = -15 + 2 * (idx % 16);
        auto sample_at = [&](int i, float& rr, float& dd) {
            const int row = i / dim, col = i - (i / dim) * dim;
            const float rv = __ldg(refI + ref_base + row * ref_pitch + col);
            if (rv < kGhost) return false;
            const int x = cx + (col - half) + u, y = cy + (row - half) + v;
            if (x < 4 || x > W - 5 || y < 4 || y > H - 5) return false;
            rr = rv;
            dd = __ldg(defI + (size_t)y * pitch + x);
            return true;
        };
        int m = 0;
        float mr = 0.0f, md = 0.0f;
        for (int i = 0; i < n; i += 9) {
            float rr, dd;
            if (!sample_at(i, rr, dd)) continue;
            mr = mr + rr;
            md = md + dd;
            ++m;
        }
        if (m < 3 || 2 * m < sampled) return 1e20f;
        const float fm = (float)m;
        mr = mr / fm;
        md = md / fm;
        float vr = 0.0f, vd = 0.0f;
        for (int i = 0; i < n; i += 9) {
            float rr, dd;
            if (!sample_at(i, rr, dd)) continue;
            vr = vr + (rr - mr) * (rr - mr);
            vd = vd + (dd - md) * (dd - md);
        }
        const float sr = sqrtf(vr / fm), sd = sqrtf(vd / fm);
        if (!(sr > 1e-5f) || !(sd > 1e-5f)) return 1e20f;
        float score = 0.0f;
        for (int i = 0; i < n; i += 9) {
            float rr, dd;
            if (!sample_at(i, rr, dd)) continue;
            const float e = (rr - mr) / sr - (dd - md) / sd;
            score = score + e * e;
        }
        return score / fm;
    }

    // The warp's minimum over (best, idx): the lowest score, ties to the lower
    // offset index (the reference's first minimum).
    __device__ __forceinline__ static void argmin_warp(float& best, int& best_idx) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float os = __shfl_xor_sync(kFull, best, o);
            const int oi = __shfl_xor_sync(kFull, best_idx, o);
            if (os < best || (os == best && oi < best_idx)) {
                best = os;
                best_idx = oi;
            }
        }
    }

    // COOP: offset idx on this thread; the warp's minimum into its slot.
    __device__ __forceinline__ void coarse_warp(int idx) {
        int sampled = 0;
        for (int i = 0; i < n; i += 9) ++sampled;
        float best = coarse_score(idx, sampled);
        int best_idx = best < 1e20f ? idx : (1 << 30);
        argmin_warp(best, best_idx);
        if (lane == 0) cslots[warp] = make_float2(best, __int_as_float(best_idx));
    }

    // estimate_initial_guess: the first minimum in the reference's v-major
    // order. One offset per lane at a time (8 each); with COOP one per thread
    // of the block. Returns (u, v); the guess when no offset qualifies.
    __device__ __forceinline__ float2 coarse(float gu, float gv) {
        float best = 1e20f;
        int best_idx = 1 << 30;
        if constexpr (COOP) {
            coop_post(2, nullptr);
            coarse_warp(lane);
            coop_bar();
            for (int w = 0; w < kCoopWarps; ++w) {
                const float2 c = cslots[w];
                const int ci = __float_as_int(c.y);
                if (c.x < best || (c.x == best && ci < best_idx)) {
                    best = c.x;
                    best_idx = ci;
                }
            }
        } else {
            int sampled = 0;
            for (int i = 0; i < n; i += 9) ++sampled;
            for (int j = 0; j < 8; ++j) {
                const int idx = lane * 8 + j;  // increasing per lane: first minimum kept
                const float score = coarse_score(idx, sampled);
                if (score < best) {
                    best = score;
                    best_idx = idx;
                }
            }
            argmin_warp(best, best_idx);
        }
        if (best_idx < 256 && best < 1e20f)
            return make_float2((float)(-15 + 2 * (best_idx % 16)), (float)(-15 + 2 * (best_idx / 16)));
        return make_float2(gu, gv);
    }
};

// Set a warp's solver up for a launch: shared-memory arrays, launch
// constants (copied out of the by-value argument block), tile state, barrier.
template <bool SIX, class Mask, bool STAGE, bool COOP>
__device__ __forceinline__ void solver_setup(WarpSolver<SIX, Mask, STAGE, COOP>& s, unsigned char* smem, const StagedLayout& L,
                                             const CUtensorMap* tmap, const float* refI, const float* refGx,
                                             const float* refGy, const float* defI, int* err, int n, int dim,
                                             int pitch, int tw, int th, int W, int H, int min_valid, int lm,
                                             int ref_pitch, int ref_dx, int ref_dy, int max_polls) {
    const int lane = threadIdx.x & 31;
    s.bar = reinterpret_cast<uint64_t*>(smem);
    s.Hr = reinterpret_cast<double*>(smem + 64);
    s.Hm = reinterpret_cast<double*>(smem + 352);
    s.tile = reinterpret_cast<float*>(smem + L.off_tile);
    s.vals = reinterpret_cast<float*>(smem + L.off_vals);
    s.srn = reinterpret_cast<float*>(smem + L.off_rn);
    s.sgx = reinterpret_cast<float*>(smem + L.off_gx);
    s.sgy = reinterpret_cast<float*>(smem + L.off_gy);
    s.tmap = tmap;
    s.refI = refI;
    s.refGx = refGx;
    s.refGy = refGy;
    s.defI = defI;
    s.err = err;
    s.n = n;
    s.dim = dim;
    s.half = dim / 2;
    s.pitch = pitch;
    s.ref_pitch = ref_pitch > 0 ? ref_pitch : pitch;
    s.ref_dx = ref_dx;
    s.ref_dy = ref_dy;
    s.tw = tw;
    s.th = th;
    s.W = W;
    s.H = H;
    s.K = (n + 31) >> 5;
    s.q = 32 / dim;
    s.r = 32 - s.q * dim;
    s.row0 = lane / dim;
    s.col0 = lane - s.row0 * dim;
    s.lane = lane;
    s.min_valid = min_valid;
    s.lm = lm;
    s.tx0 = s.ty0 = 0;
    s.tile_ok = false;
    s.tile_on = tw > 0;
    s.all_in = false;
    s.no_ghost = false;
    s.fullmask = 0;
    for (int k = 0; k < s.K; ++k)
        if (lane + 32 * k < n) s.fullmask |= Mask(1) << k;
    s.phase = 0;
    s.warp = (int)(threadIdx.x >> 5);
    s.req = reinterpret_cast<CoopReq*>(smem + L.off_coop);
    s.gbits = reinterpret_cast<Mask*>(smem + L.off_coop + kCoopGbits);
    s.cslots = reinterpret_cast<float2*>(smem + L.off_coop + kCoopSlots);
    s.hsum = reinterpret_cast<double*>(smem + L.off_coop + kCoopHsum);
    s.mflags = reinterpret_cast<int*>(smem + L.off_coop + kCoopFlags);
    s.scr_cond = reinterpret_cast<double*>(smem + L.off_coop + kCoopScrCond);
    s.scr_inv = reinterpret_cast<double*>(smem + L.off_coop + kCoopScrInv);
    // one barrier per block, set up by its first warp (the driver, with COOP),
    // and beside it the wait limit and the record of a wait that ran out
    if (threadIdx.x == 0) {
        mbar_init(s.bar, 1);
        int* const aux = reinterpret_cast<int*>(s.bar + 1);
        aux[0] = max_polls > 0 ? max_polls : kTmaPolls;
        aux[1] = 0;
        aux[2] = 0;
    }
    fence_proxy_async_smem();
    __syncwarp();
}

// The fast pass over every task: the common case, everything else deferred.
// DIMC > 0: the subset size, the tile box and the pixels per lane known at
// compile time (the launch checks they match), so the per-pixel loop
// bookkeeping folds away; 32-bit validity masks up to 32 pixels per lane.
// Subset 41's tile and sampled values (18.7 KB a warp) leave room for 12
// warps per SM, so its registers are capped for 12 (no spills), the others'
// for 18. RT: the tile box taken from the launch (a box sized for a rotated
// or stretched subset) with the subset size still known at compile time.
template <bool SIX, int DIMC, bool STAGE, bool RT = false>
__global__ void __launch_bounds__(32, (DIMC == 41 ? 12 : 18)) fast_kernel(const __grid_constant__ CUtensorMap tmap, const SolveArgs a,
                                                  const StagedLayout L) {
    extern __shared__ __align__(128) unsigned char smem[];
    using Mask = std::conditional_t<(DIMC > 0 && DIMC * DIMC <= 1024), uint32_t, uint64_t>;
    constexpr int kTw = DIMC > 0 ? ((DIMC + (SIX ? 5 : 3) + 2 + 7 + 3) & ~3) : 0;
    constexpr int kTh = DIMC > 0 ? DIMC + (SIX ? 5 : 3) + 2 + 2 : 0;
    WarpSolver<SIX, Mask, STAGE> s;
    solver_setup(s, smem, L, &tmap, a.refI, a.refGx, a.refGy, a.defI, a.err, DIMC > 0 ? DIMC * DIMC : a.n,
                 DIMC > 0 ? DIMC : a.dim, a.pitch, (DIMC > 0 && !RT) ? kTw : a.tile_w,
                 (DIMC > 0 && !RT) ? kTh : a.tile_h, a.W, a.H,
                 a.min_valid, a.lm, a.ref_pitch, a.ref_dx, a.ref_dy, a.tma_max_polls);
    if (DIMC > 0) s.tile_on = a.tile_w > 0;
    s.no_ghost = a.ref_no_ghost != 0;
    const int lane = s.lane, dim = s.dim, half = s.half;
    const int ntasks = a.n_tasks_dev ? *a.n_tasks_dev : a.n_tasks;
    int* const n_deferred = a.queue + 2;
    int* const deferred = a.deferred;
    int polled = 0;
    // One task of lookahead: the next task is claimed, and its record loaded
    // (word i of the 10 by lane i: one register a lane) while the current one
    // is solved. The record passes through shared memory where the
    // masked-iteration matrix of the rescue pass would be (unused here).
    static_assert(sizeof(dic_task) == 40, "task record of 10 words");
    int* const tn_s = reinterpret_cast<int*>(smem + 352);
    int tw = 0;
    auto fetch_task = [&](int tt) {
        if (tt < ntasks && lane < 10) tw = reinterpret_cast<const int*>(a.tasks + tt)[lane];
    };
    int t_next = 0;
    if (lane == 0) t_next = atomicAdd(a.queue, 1);
    t_next = __shfl_sync(kFull, t_next, 0);
    fetch_task(t_next);
    for (;;) {
        const int t = t_next;
        if (t >= ntasks) break;
        // the cancel flag lives in host memory: a read crosses PCIe, so a warp
        // looks at it once every kCancelPollTasks tasks, not per task
        if (a.cancel && (++polled & (kCancelPollTasks - 1)) == 0 && *(volatile const int*)a.cancel) break;
        __syncwarp();
        if (lane < 10) tn_s[lane] = tw;
        __syncwarp();
        const dic_task T = *reinterpret_cast<const dic_task*>(tn_s);
        if (lane == 0) t_next = atomicAdd(a.queue, 1);
        t_next = __shfl_sync(kFull, t_next, 0);
        fetch_task(t_next);
        if (T.mode == DIC_INIT_AUTO_SEARCH || s.K > kFastMaxPerLane) {
            if (lane == 0) deferred[atomicAdd(n_deferred, 1)] = t;
            __syncwarp();
            continue;
        }
        dic_result out;
        out.u = out.v = out.ux = out.uy = out.vx = out.vy = 0.0f;
        out.score = 0.0f;
        out.status = out.iters = out.trigger_iters = out.invalid_ref = out.flags = 0;
        const bool dim_ok = dim >= 3 && (dim & 1) && dim * dim <= a.max_n;
        const bool on_img = T.cx - half >= 0 && T.cx + half < a.W && T.cy - half >= 0 && T.cy + half < a.H;
        if (!dim_ok || !on_img || !a.pool_valid[T.node]) {
            if (lane == 0) a.results[t] = out;
            continue;
        }
        s.begin(T, a.pool_ms[T.node], a.pool_Hs + (size_t)T.node * 21);
        // calculate_deformation (optimization_engine.cpp:55-118), IC-GN only
        bool defer = false;
        Res res = s.template icgn<false>(T.g, defer);
        // a NO_SEARCH task that would take the Simplex rescue goes to the rescue pass
        if (!defer && T.mode == DIC_INIT_NO_SEARCH && (res.status != 0 || res.score > kCorrSimplexTrigger))
            defer = true;
        if (defer) {
            if (lane == 0) deferred[atomicAdd(n_deferred, 1)] = t;
            __syncwarp();
            continue;
        }
        if ((float)s.ghost / (float)(dim * dim) > kGhostRejectFraction) {
            res.score = 2.0f;
            res.status = 1;
        }
        if (lane == 0) {
            out.u = res.u; out.v = res.v; out.ux = res.ux; out.uy = res.uy; out.vx = res.vx; out.vy = res.vy;
            out.score = res.score;
            out.status = res.status;
            out.iters = res.iters;
            out.trigger_iters = res.iters;
            out.invalid_ref = s.ghost;
            out.flags = DIC_RES_INITIALIZED;
            a.results[t] = out;
        }
        __syncwarp();
    }
    s.drain();
}

// The rescue pass over the tasks the fast pass handed on, with every path of
// calculate_deformation (optimization_engine.cpp:55-118): the coarse search
// and 2-DOF Simplex of AUTO_SEARCH, masked iterations, and the 6-DOF Simplex
// rescue of NO_SEARCH, keeping the better run. A block of kCoopWarps warps
// per task: warp 0 runs the task, and every evaluation's sampling (and the
// coarse search's 256 offsets) is shared by all warps of the block. The
// ordered reductions stay on warp 0, so the results are those of a single
// warp. Every exit of the driver's loop posts "done", which is what ends the
// other warps' loop. DIMC > 0: the subset size known at compile time (the
// launch checks it), so warp 0's ordered per-lane chains unroll with their
// loads ahead, and subsets of at most 1024 pixels use 32-bit validity masks.
template <bool SIX, int DIMC>
__global__ void __launch_bounds__(kCoopWarps * 32, 1) coop_rescue_kernel(const __grid_constant__ CUtensorMap tmap,
                                                                         const SolveArgs a, const StagedLayout L) {
    extern __shared__ __align__(128) unsigned char smem[];
    using Mask = std::conditional_t<(DIMC > 0 && DIMC * DIMC <= 1024), uint32_t, uint64_t>;
    WarpSolver<SIX, Mask, true, true> s;
    solver_setup(s, smem, L, &tmap, a.refI, a.refGx, a.refGy, a.defI, a.err, DIMC > 0 ? DIMC * DIMC : a.n,
                 DIMC > 0 ? DIMC : a.dim, a.pitch, L.tile_w, L.tile_h, a.W, a.H, a.min_valid, a.lm, a.ref_pitch,
                 a.ref_dx, a.ref_dy, a.tma_max_polls);
    if (s.warp != 0) {
        s.coop_serve();
        return;
    }
    const int lane = s.lane, dim = s.dim, half = s.half;
    // the tasks the fast pass handed on, or (rescue_all) every task
    const int ntasks = a.rescue_all ? a.n_tasks : *(volatile const int*)(a.queue + 2);
    int* const queue = a.queue + 1;
    int polled = 0;
    for (;;) {
        int q = 0;
        if (lane == 0) q = atomicAdd(queue, 1);
        q = __shfl_sync(kFull, q, 0);
        if (q >= ntasks) break;
        if (a.cancel && (++polled & (kCancelPollTasks - 1)) == 0 && *(volatile const int*)a.cancel) break;
        const int t = a.rescue_all ? q : a.deferred[q];
        const dic_task T = a.tasks[t];
        dic_result out;
        out.u = out.v = out.ux = out.uy = out.vx = out.vy = 0.0f;
        out.score = 0.0f;
        out.status = out.iters = out.trigger_iters = out.invalid_ref = out.flags = 0;
        const bool dim_ok = dim >= 3 && (dim & 1) && dim * dim <= a.max_n;
        const bool on_img = T.cx - half >= 0 && T.cx + half < a.W && T.cy - half >= 0 && T.cy + half < a.H;
        if (!dim_ok || !on_img || !a.pool_valid[T.node]) {
            if (lane == 0) a.results[t] = out;
            continue;
        }
        s.begin(T, a.pool_ms[T.node], a.pool_Hs + (size_t)T.node * 21);
        const int mode = T.mode;
        float st[6] = {T.g[0], T.g[1], T.g[2], T.g[3], T.g[4], T.g[5]};
        bool rescue = false;
        if (mode == DIC_INIT_AUTO_SEARCH) {
            float2 e = make_float2(st[0], st[1]);
            if (e.x == 0.0f && e.y == 0.0f) e = s.coarse(e.x, e.y);
            const Res cr = s.simplex(e.x, e.y, 0.0f, 0.0f, 0.0f, 0.0f, true);
            rescue = true;
            st[0] = cr.u; st[1] = cr.v; st[2] = st[3] = st[4] = st[5] = 0.0f;
        }
        Res res;
        int trigger = 0;
        bool unused = false;
        for (int run = 0; run < 2; ++run) {
            const Res r = s.template icgn<true>(st, unused);
            if (run == 0) {
                res = r;
                trigger = r.iters;
                if (mode != DIC_INIT_NO_SEARCH || !(r.status != 0 || r.score > kCorrSimplexTrigger)) break;
                const Res rr = s.simplex(T.g[0], T.g[1], T.g[2], T.g[3], T.g[4], T.g[5], false);
                rescue = true;
                st[0] = rr.u; st[1] = rr.v; st[2] = rr.ux; st[3] = rr.uy; st[4] = rr.vx; st[5] = rr.vy;
            } else {
                const bool first_better = res.status == 0 && (r.status != 0 || res.score < r.score);
                if (!first_better) res = r;
            }
        }
        if ((float)s.ghost / (float)(dim * dim) > kGhostRejectFraction) {
            res.score = 2.0f;
            res.status = 1;
        }
        if (lane == 0) {
            out.u = res.u; out.v = res.v; out.ux = res.ux; out.uy = res.uy; out.vx = res.vx; out.vy = res.vy;
            out.score = res.score;
            out.status = res.status;
            out.iters = res.iters;
            out.trigger_iters = trigger;
            out.invalid_ref = s.ghost;
            out.flags = DIC_RES_INITIALIZED | (rescue ? DIC_RES_RESCUE : 0);
            a.results[t] = out;
        }
        __syncwarp();
    }
    s.coop_post(0, nullptr);  // done: the other warps leave their loop
    s.drain();
}

// The dynamic shared-memory limit of a kernel, always set to the device's
// opt-in maximum. The attribute belongs to the function for the whole
// process, so a per-launch value would race between engines solving on other
// threads: one thread's smaller setting would make another thread's larger
// launch invalid. The occupancy still follows each launch's own size.
// Launch facts that do not change during the process (per device and
// kernel): the opt-in attribute set, and each (kernel, threads, bytes)
// occupancy. Looked up once, so that the many small solves of Path B rounds
// pay no runtime queries.
struct LaunchCache {
    std::mutex m;
    std::map<std::pair<int, const void*>, bool> smem_set;
    std::map<std::tuple<int, const void*, int, size_t>, int> occupancy;
    std::map<int, int> sms;
};
LaunchCache& launch_cache() {
    static LaunchCache c;
    return c;
}

template <class K>
cudaError_t allow_max_smem(K kernel) {
    int dev = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    LaunchCache& c = launch_cache();
    {
        std::lock_guard<std::mutex> g(c.m);
        if (c.smem_set.count({dev, (const void*)kernel})) return cudaSuccess;
    }
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    cudaFuncAttributes fa;
    e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(c.m);
    c.smem_set[{dev, (const void*)kernel}] = true;
    return cudaSuccess;
}
template <class K>
cudaError_t one_wave(K kernel, size_t smem, long cap, long tasks, long& blocks, int threads = 32) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    LaunchCache& c = launch_cache();
    const auto key = std::make_tuple(dev, (const void*)kernel, threads, smem);
    bool have = false;
    {
        std::lock_guard<std::mutex> g(c.m);
        const auto it = c.occupancy.find(key);
        const auto is = c.sms.find(dev);
        if (it != c.occupancy.end() && is != c.sms.end()) {
            per_sm = it->second;
            sms = is->second;
            have = true;
        }
    }
    if (!have) {
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> g(c.m);
        c.occupancy[key] = per_sm;
        c.sms[dev] = sms;
    }
    blocks = (long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    if (cap > 0 && blocks > cap) blocks = cap;
    if (blocks > tasks) blocks = tasks > 0 ? tasks : 1;
    return cudaSuccess;
}

// The fast pass and then the rescue pass over what it handed on; subsets the
// staged solvers do not take go to solve_kernel, which takes every task.
template <bool SIX>
cudaError_t launch_passes(const CUtensorMap& tmap, const CUtensorMap& tmap_r, int tw_r, int th_r, const SolveArgs& a,
                          const StagedLayout& SL, bool staged_ok, int grid_blocks, size_t smem, cudaStream_t st) {
    // the caller's hint counts units of kSolveThreads / 32 subsets
    const long cap = grid_blocks > 0 ? (long)grid_blocks * (kSolveThreads / 32) : 0;
    long blocks = 1;
    cudaError_t e;
    if (staged_ok) {
        // subset sizes with a compile-time kernel (the tile box must be the one it assumes)
        int tw = 0, th = 0;
        tile_box(a.dim, SIX ? 1 : 0, tw, th);
        const bool box_ok = a.tile_w == 0 || (a.tile_w == tw && a.tile_h == th);
        // the fast pass reads the reference subset from the planes (about
        // half the shared memory per warp, twice the resident warps) or
        // stages it per task (fast_stage): the caller's autotuner times both
        const bool stage = a.fast_stage != 0;
        auto fast = stage ? fast_kernel<SIX, 0, true> : fast_kernel<SIX, 0, false>;
        if (box_ok && a.dim == 21) fast = stage ? fast_kernel<SIX, 21, true> : fast_kernel<SIX, 21, false>;
        if (box_ok && a.dim == 31) fast = stage ? fast_kernel<SIX, 31, true> : fast_kernel<SIX, 31, false>;
        if (box_ok && a.dim == 41) fast = stage ? fast_kernel<SIX, 41, true> : fast_kernel<SIX, 41, false>;
        // a box sized for a rotated subset (the seeding model's spread): the
        // compile-time subset size with the launch's box
        if (!box_ok && !stage && a.tile_w > 0) {
            if (a.dim == 21) fast = fast_kernel<SIX, 21, false, true>;
            if (a.dim == 31) fast = fast_kernel<SIX, 31, false, true>;
            if (a.dim == 41) fast = fast_kernel<SIX, 41, false, true>;
        }
        const StagedLayout FL = staged_layout(a.n, a.tile_w, a.tile_h, stage);
        if (!a.rescue_all) {
            e = allow_max_smem(fast);
            if (e != cudaSuccess) return e;
            e = one_wave(fast, FL.bytes, 0, a.n_tasks, blocks);
            if (e != cudaSuccess) return e;
            fast<<<(unsigned)blocks, 32, FL.bytes, st>>>(tmap, a, FL);
        }
        // the rescue pass: a block of kCoopWarps warps per task, with its own
        // larger tile (one block per SM leaves the shared memory for it)
        const StagedLayout RL = staged_layout(a.n, tw_r, th_r, true, true);
        auto coop = coop_rescue_kernel<SIX, 0>;
        if (a.dim == 21) coop = coop_rescue_kernel<SIX, 21>;
        if (a.dim == 31) coop = coop_rescue_kernel<SIX, 31>;
        if (a.dim == 41) coop = coop_rescue_kernel<SIX, 41>;
        e = allow_max_smem(coop);
        if (e != cudaSuccess) return e;
        e = one_wave(coop, RL.bytes, cap, a.n_tasks, blocks, kCoopWarps * 32);
        if (e != cudaSuccess) return e;
        coop<<<(unsigned)blocks, kCoopWarps * 32, RL.bytes, st>>>(tw_r > 0 ? tmap_r : tmap, a, RL);
        return cudaGetLastError();
    }
    e = allow_max_smem(solve_kernel<SIX, false>);
    if (e != cudaSuccess) return e;
    e = one_wave(solve_kernel<SIX, false>, smem, cap, a.n_tasks, blocks);
    if (e != cudaSuccess) return e;
    solve_kernel<SIX, false><<<(unsigned)blocks, 32, smem, st>>>(tmap, a);
    return cudaGetLastError();
}

// The driver's tensor-map encoder, looked up once per process (a function
// static: thread-safe initialisation, engines may run on several threads).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    }();
    return fn;
}

}  // namespace

// The support a warped subset needs: the subset's side, grown by `spread`
// when it is above 1, plus the interpolation taps and a pixel of rounding
// slack each side.
static int support_of(int dim, int six, float spread) {
    // at most 1.5 (any rotation): larger spreads keep the tiles of 1.5, so
    // that both passes' tiles fit shared memory and the TMA box limit
    spread = std::min(spread, 1.5f);
    const int side = spread > 1.0f ? (int)std::ceil((double)dim * spread) : dim;
    return side + (six ? 5 : 3) + 2;
}

void tile_box(int dim, int six, int& tw, int& th, float spread) {
    // the warped subset's support, three columns of alignment slack, and a
    // margin for the warp to move in before the tile is staged again: two
    // pixels each way across, one up and down (two rows fewer of shared
    // memory: subset 41's fast pass holds 12 warps per SM instead of 11)
    const int need = support_of(dim, six, spread);
    tw = ((need + 3 + 4) + 3) & ~3;
    th = need + 2;
    if (tw > 256 || th > 256) tw = th = 0;
}

// The rescue pass's tile: twice the support each way (capped by the TMA box
// limit), so the wide warps of Simplex probes and diverging iterations keep
// reading shared memory; 0 when the fast pass's box is unavailable.
void rescue_tile_box(int dim, int six, int& tw, int& th, float spread = 0.0f) {
    int fw = 0, fh = 0;
    tile_box(dim, six, fw, fh, spread);
    if (fw == 0) {
        tw = th = 0;
        return;
    }
    const int need = support_of(dim, six, spread);
    tw = std::min(((2 * need + 7) + 3) & ~3, 256);
    th = std::min(2 * need, 256);
}

cudaError_t launch_solve(const SolveArgs& a0, int six, int grid_blocks, cudaStream_t st) {
    SolveArgs a = a0;
    CUtensorMap tmap;
    std::memset(&tmap, 0, sizeof(tmap));
    int tw = 0, th = 0;
    tile_box(a.dim, six, tw, th, a.tile_spread);
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
    CUtensorMap tmap_r;
    std::memset(&tmap_r, 0, sizeof(tmap_r));
    int tw_r = 0, th_r = 0;
    if (tw > 0) {
        rescue_tile_box(a.dim, six, tw_r, th_r, a.tile_spread);
        const cuuint64_t gdim[2] = {(cuuint64_t)a.W, (cuuint64_t)a.H};
        const cuuint64_t gstride[1] = {(cuuint64_t)a.pitch * 4};
        const cuuint32_t box[2] = {(cuuint32_t)tw_r, (cuuint32_t)th_r};
        const cuuint32_t estr[2] = {1, 1};
        const CUresult r = enc(&tmap_r, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(a.defI), gdim, gstride,
                               box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            // the rescue pass then uses the fast pass's box
            tw_r = tw;
            th_r = th;
            tmap_r = tmap;
        }
    }
    const SmemLayout L = smem_layout(a.max_n, tw, th);
    a.smem_per_warp = L.bytes;
    a.half = a.dim / 2;
    a.n = a.dim * a.dim;
    a.min_valid = (int)((float)a.n * 0.90f);
    a.off_tile = (int)L.off_tile;
    a.off_vals = (int)L.off_vals;
    a.off_valid = (int)L.off_valid;
    a.off_refok = (int)L.off_refok;
    const size_t smem = kArgsBytes + a.smem_per_warp;
    // queue[0]: fast pass, queue[1]: general pass, queue[2]: deferred count
    cudaError_t e = cudaMemsetAsync(a.queue, 0, 3 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    // the fast pass takes subsets up to kFastMaxPerLane pixels per lane whose
    // shared memory fits one block; otherwise the general pass takes every task
    const StagedLayout SL = staged_layout(a.n, tw, th);
    const bool staged_ok = ((a.n + 31) >> 5) <= kFastMaxPerLane && SL.bytes <= kFastMaxSmem;
    a.general_all = staged_ok ? 0 : 1;
    // A launch of a few tasks per SM (Path B rounds, the anchor lattice, patch
    // solves) is bound by each task's latency: every task then goes to the
    // rescue pass, whose 8 warps per task sample each evaluation together.
    // Both passes give the same result for a task.
    int sms = 0, dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
        a.rescue_all = staged_ok && a.n_tasks <= 4 * sms ? 1 : 0;
    else
        a.rescue_all = 0;
    // reference planes of another frame are read by the staged solver only
    const bool own_ref = (a.ref_pitch > 0 && a.ref_pitch != a.pitch) || a.ref_dx != 0 || a.ref_dy != 0;
    if (own_ref && !staged_ok) return cudaErrorInvalidValue;
    return six ? launch_passes<true>(tmap, tmap_r, tw_r, th_r, a, SL, staged_ok, grid_blocks, smem, st)
               : launch_passes<false>(tmap, tmap_r, tw_r, th_r, a, SL, staged_ok, grid_blocks, smem, st);
}

}  // namespace dic
