// Per-node kernels of the incremental session (incnode.cuh).
//
// One thread per node. The arithmetic of each per-node rule is written out
// operation by operation as the reference evaluates it (float where it uses
// float, double where it uses double; built without FP contraction), because
// the totals it produces are compared bit for bit with the CPU restatement:
//   increment sampling       src/pipeline/incremental_math.cpp:59-119
//   coasting plane fit       incremental_math.cpp:121-186
//   anchor need              incremental_math.cpp:188-221
//   fill of invalid nodes    incremental_math.cpp:281-322
//   local stretch            incremental_math.cpp:371-447
//   the session's node step  src/pipeline/incremental_session.cpp:323-462
// The reference finds the anchor need from two exact distance transforms of
// the whole grid. Here each node searches its own window instead: a gap or
// hole decides only whether one lies within a fixed radius, and a window one
// cell wider than that radius holds every position that can decide it, so the
// decisions are the same.
#include "incnode.cuh"

#include <climits>

namespace dic {

namespace {

// include/semper/tuning.hpp values the node step uses.
constexpr float kTaylorMaxCells = 1.5f;
constexpr int kCoastMinNodes = 6;
constexpr float kCorrInvalid = -1.0f;

constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ bool in_grid(const IncField& f, int i, int j) {
    return i >= 0 && i < f.gw && j >= 0 && j < f.gh;
}

// solved, with a result, kept by the median test (node_field_from_capture,
// incremental_math.cpp:19-57)
__device__ __forceinline__ bool usable(const IncField& f, int k) {
    return f.solved[k] && f.corr[k] >= 0.0f && f.ok[k];
}

__device__ __forceinline__ float node_xf(int rect, int i, int step) { return (float)(rect + i * step); }

// Warp-aggregated add to a counter.
__device__ __forceinline__ void count_add(int* c, int v) {
    const int s = __reduce_add_sync(kAll, v);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(c, s);
}

// Order-preserving int key of a float (min and max by signed compare).
__device__ __forceinline__ int fkey(float x) {
    const int b = __float_as_int(x);
    return b >= 0 ? b : b ^ 0x7fffffff;
}

struct Sample {
    bool ok, taylor;
    float u, v, corr;
};

// sample_increment: the node's value on a node, bilinear in a cell with four
// usable corners, else the first-order expansion from the nearest usable node
// of the 4x4 block within kTaylorMaxCells cells.
__device__ Sample sample_increment(const IncField& f, float x, float y) {
    Sample s{false, false, 0.0f, 0.0f, 0.0f};
    if (f.gw <= 0 || f.gh <= 0 || f.step <= 0) return s;
    const float gx = __fdiv_rn(__fsub_rn(x, (float)f.rect_x), (float)f.step);
    const float gy = __fdiv_rn(__fsub_rn(y, (float)f.rect_y), (float)f.step);
    const int i0 = (int)floorf(gx), j0 = (int)floorf(gy);
    const float fx = __fsub_rn(gx, (float)i0), fy = __fsub_rn(gy, (float)j0);
    if (fx == 0.0f && fy == 0.0f && in_grid(f, i0, j0) && usable(f, j0 * f.gw + i0)) {
        const int k = j0 * f.gw + i0;
        s.ok = true;
        s.u = f.u[k];
        s.v = f.v[k];
        s.corr = f.corr[k];
        return s;
    }
    if (in_grid(f, i0, j0) && in_grid(f, i0 + 1, j0 + 1)) {
        const int a = j0 * f.gw + i0, b = a + 1, c = a + f.gw, d = c + 1;
        if (usable(f, a) && usable(f, b) && usable(f, c) && usable(f, d)) {
            const float ex = __fsub_rn(1.0f, fx), ey = __fsub_rn(1.0f, fy);
            const float wa = __fmul_rn(ex, ey), wb = __fmul_rn(fx, ey);
            const float wc = __fmul_rn(ex, fy), wd = __fmul_rn(fx, fy);
            s.ok = true;
            s.u = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(wa, f.u[a]), __fmul_rn(wb, f.u[b])), __fmul_rn(wc, f.u[c])),
                            __fmul_rn(wd, f.u[d]));
            s.v = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(wa, f.v[a]), __fmul_rn(wb, f.v[b])), __fmul_rn(wc, f.v[c])),
                            __fmul_rn(wd, f.v[d]));
            s.corr = fmaxf(fmaxf(f.corr[a], f.corr[b]), fmaxf(f.corr[c], f.corr[d]));
            return s;
        }
    }
    const float max_d = __fmul_rn(kTaylorMaxCells, (float)f.step);
    float best = __int_as_float(0x7f800000);
    int bi = -1, bj = -1;
    for (int j = j0 - 1; j <= j0 + 2; ++j)
        for (int i = i0 - 1; i <= i0 + 2; ++i) {
            if (!in_grid(f, i, j) || !usable(f, j * f.gw + i)) continue;
            const float dx = __fsub_rn(x, node_xf(f.rect_x, i, f.step));
            const float dy = __fsub_rn(y, node_xf(f.rect_y, j, f.step));
            const float d2 = __fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy));
            if (d2 < best) {
                best = d2;
                bi = i;
                bj = j;
            }
        }
    if (bi < 0 || best > __fmul_rn(max_d, max_d)) return s;
    const int k = bj * f.gw + bi;
    const float dx = __fsub_rn(x, node_xf(f.rect_x, bi, f.step));
    const float dy = __fsub_rn(y, node_xf(f.rect_y, bj, f.step));
    s.ok = true;
    s.taylor = true;
    s.u = __fadd_rn(__fadd_rn(f.u[k], __fmul_rn(f.ux[k], dx)), __fmul_rn(f.uy[k], dy));
    s.v = __fadd_rn(__fadd_rn(f.v[k], __fmul_rn(f.vx[k], dx)), __fmul_rn(f.vy[k], dy));
    s.corr = f.corr[k];
    return s;
}

__device__ __forceinline__ double det3(const double m[3][3]) {
    const double a = __dsub_rn(__dmul_rn(m[1][1], m[2][2]), __dmul_rn(m[1][2], m[2][1]));
    const double b = __dsub_rn(__dmul_rn(m[1][0], m[2][2]), __dmul_rn(m[1][2], m[2][0]));
    const double c = __dsub_rn(__dmul_rn(m[1][0], m[2][1]), __dmul_rn(m[1][1], m[2][0]));
    return __dadd_rn(__dsub_rn(__dmul_rn(m[0][0], a), __dmul_rn(m[0][1], b)), __dmul_rn(m[0][2], c));
}

// fit_increment: the weighted plane through the usable nodes within radius
// (weights 1 / (1 + (d/step)^2)), its value at (x, y) by Cramer's rule; needs
// kCoastMinNodes nodes spread at least one step along both principal axes.
__device__ Sample fit_increment(const IncField& f, float x, float y, float radius) {
    Sample s{false, false, 0.0f, 0.0f, 0.0f};
    if (f.gw <= 0 || f.gh <= 0 || f.step <= 0 || radius <= 0.0f) return s;
    const double step = (double)f.step;
    const int r = (int)ceil(__ddiv_rn((double)radius, step));
    const int ic = (int)llround(__ddiv_rn((double)__fsub_rn(x, (float)f.rect_x), step));
    const int jc = (int)llround(__ddiv_rn((double)__fsub_rn(y, (float)f.rect_y), step));
    const double r2max = __dmul_rn((double)radius, (double)radius);
    const double step2 = __dmul_rn(step, step);
    double S[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
    double bu[3] = {0.0, 0.0, 0.0}, bv[3] = {0.0, 0.0, 0.0};
    int n = 0;
    float worst = 0.0f;
    const int j_lo = max(0, jc - r), j_hi = min(f.gh - 1, jc + r);
    const int i_lo = max(0, ic - r), i_hi = min(f.gw - 1, ic + r);
    for (int j = j_lo; j <= j_hi; ++j)
        for (int i = i_lo; i <= i_hi; ++i) {
            const int k = j * f.gw + i;
            if (!usable(f, k)) continue;
            const double dx = (double)__fsub_rn(node_xf(f.rect_x, i, f.step), x);
            const double dy = (double)__fsub_rn(node_xf(f.rect_y, j, f.step), y);
            const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
            if (d2 > r2max) continue;
            const double w = __ddiv_rn(1.0, __dadd_rn(1.0, __ddiv_rn(d2, step2)));
            const double p[3] = {1.0, __ddiv_rn(dx, step), __ddiv_rn(dy, step)};
            const double uk = (double)f.u[k], vk = (double)f.v[k];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const double wp = __dmul_rn(w, p[a]);
#pragma unroll
                for (int b = 0; b < 3; ++b) S[a][b] = __dadd_rn(S[a][b], __dmul_rn(wp, p[b]));
                bu[a] = __dadd_rn(bu[a], __dmul_rn(wp, uk));
                bv[a] = __dadd_rn(bv[a], __dmul_rn(wp, vk));
            }
            worst = fmaxf(worst, f.corr[k]);
            ++n;
        }
    if (n < kCoastMinNodes) return s;
    const double W = S[0][0];
    const double mx = __ddiv_rn(S[0][1], W), my = __ddiv_rn(S[0][2], W);
    const double cxx = __dsub_rn(__ddiv_rn(S[1][1], W), __dmul_rn(mx, mx));
    const double cyy = __dsub_rn(__ddiv_rn(S[2][2], W), __dmul_rn(my, my));
    const double cxy = __dsub_rn(__ddiv_rn(S[1][2], W), __dmul_rn(mx, my));
    const double tr = __dadd_rn(cxx, cyy);
    const double det2 = __dsub_rn(__dmul_rn(cxx, cyy), __dmul_rn(cxy, cxy));
    const double disc = fmax(0.0, __dsub_rn(__dmul_rn(tr, tr), __dmul_rn(4.0, det2)));
    const double lmin = __dmul_rn(0.5, __dsub_rn(tr, __dsqrt_rn(disc)));
    if (lmin < 1.0) return s;
    const double D = det3(S);
    if (fabs(D) < 1e-12) return s;
    double M[3][3];
    for (int a = 0; a < 3; ++a) {
        M[a][1] = S[a][1];
        M[a][2] = S[a][2];
    }
    for (int a = 0; a < 3; ++a) M[a][0] = bu[a];
    const double cu = __ddiv_rn(det3(M), D);
    for (int a = 0; a < 3; ++a) M[a][0] = bv[a];
    const double cv = __ddiv_rn(det3(M), D);
    s.ok = true;
    s.u = (float)cu;
    s.v = (float)cv;
    s.corr = worst;
    return s;
}

// The distance, in px, that a squared distance of d2 cells gives on a grid
// of this step, rounded as the reference's distance transform rounds it
// (the root to float, then the product with the step in double to float).
__device__ __forceinline__ float cells_to_px(int d2, int step) {
    const float d = (float)__dsqrt_rn((double)d2);
    return (float)__dmul_rn((double)d, (double)step);
}

// The anchor need of one node of the increment field: its subset is clean
// when no unusable node lies within half a subset plus a step (keep
// otherwise); a gap is within reach when an unusable node or an off-grid
// position (the one-node ring around the grid) lies within two subsets plus
// two steps (refresh), else drop.
__global__ void need_kernel(IncField f, int subset, uint8_t* __restrict__ need) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= f.gw * f.gh) return;
    const int i = k % f.gw, j = k / f.gw;
    const float hole_thr = (float)(subset / 2 + f.step);
    const float gap_thr = (float)(2 * subset + 2 * f.step);
    // windows one cell wider than the radii in cells
    const int rh = (int)ceilf(hole_thr / (float)f.step) + 1;
    const int rg = (int)ceilf(gap_thr / (float)f.step) + 1;
    int hole_d2 = INT_MAX, gap_d2 = INT_MAX;
    for (int dj = -rg; dj <= rg; ++dj) {
        const int jj = j + dj;
        if (jj < -1 || jj > f.gh) continue;
        for (int di = -rg; di <= rg; ++di) {
            const int ii = i + di;
            if (ii < -1 || ii > f.gw) continue;
            const int d2 = di * di + dj * dj;
            const bool on = ii >= 0 && ii < f.gw && jj >= 0 && jj < f.gh;
            if (on && usable(f, jj * f.gw + ii)) continue;
            // an unusable node, or the off-grid ring
            if (d2 < gap_d2) gap_d2 = d2;
            if (on && d2 < hole_d2 && di >= -rh && di <= rh && dj >= -rh && dj <= rh) hole_d2 = d2;
        }
    }
    uint8_t out = 0;  // drop
    if (hole_d2 != INT_MAX && cells_to_px(hole_d2, f.step) <= hole_thr)
        out = 2;  // keep
    else if (gap_d2 != INT_MAX && cells_to_px(gap_d2, f.step) <= gap_thr)
        out = 1;  // refresh
    need[k] = out;
}

// anchor_need at (x, y): the need of the nearest node of the field.
__device__ __forceinline__ uint8_t need_at(const IncField& f, const uint8_t* need, float x, float y) {
    if (f.gw <= 0 || f.gh <= 0) return 2;
    const int i = min(f.gw - 1, max(0, (int)lroundf(__fdiv_rn(__fsub_rn(x, (float)f.rect_x), (float)f.step))));
    const int j = min(f.gh - 1, max(0, (int)lroundf(__fdiv_rn(__fsub_rn(y, (float)f.rect_y), (float)f.step))));
    return need[j * f.gw + i];
}

__global__ void first_kernel(IncField f, const uint8_t* __restrict__ need, IncFrame fr) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= f.gw * f.gh) return;
    const bool result = f.solved[k] && f.corr[k] >= 0.0f;
    const bool ok = result && f.ok[k];
    fr.U[k] = result ? f.u[k] : 0.0f;
    fr.V[k] = result ? f.v[k] : 0.0f;
    fr.corr[k] = result ? f.corr[k] : kCorrInvalid;
    fr.cstep[k] = 0.0f;
    uint8_t nd = 2;
    if (ok) nd = need_at(f, need, node_xf(f.rect_x, k % f.gw, f.step), node_xf(f.rect_y, k / f.gw, f.step));
    fr.flags[k] = (uint8_t)((ok ? (kIncCarried | kIncValid) : 0) | (nd << kIncNeedShift));
}

// The correctly rounded length of (a, b): the root of the exact double sum of
// squares, to float.
__device__ __forceinline__ float length2(float a, float b) {
    const double s = __dadd_rn(__dmul_rn((double)a, (double)a), __dmul_rn((double)b, (double)b));
    return (float)__dsqrt_rn(s);
}

// One frame-0 node against the increment field of an updated reference.
__global__ void step_kernel(IncGrid g, IncState s, IncField f, const uint8_t* __restrict__ need, IncStepArgs a,
                            IncFrame fr, int* counters, int* match_list, float* match_info) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.gw * g.gh;
    if (k >= n) return;
    float U = 0.0f, V = 0.0f, corr = 0.0f, cstep = 0.0f;
    uint8_t flags = (uint8_t)(2 << kIncNeedShift);
    if (s.alive[k]) {
        const float x = node_xf(g.rect_x, k % g.gw, g.step), y = node_xf(g.rect_y, k / g.gw, g.step);
        const float ub = s.ubase[k], vb = s.vbase[k];
        const float px = __fadd_rn(x, ub), py = __fadd_rn(y, vb);
        const Sample smp = sample_increment(f, px, py);
        if (!smp.ok) {
            // coast on the plane fitted through the neighbours, inside the frame only
            if (!(px < 0.0f || py < 0.0f || px > (float)(a.width - 1) || py > (float)(a.height - 1))) {
                const Sample fit = fit_increment(f, px, py, a.coast_radius);
                if (fit.ok) {
                    const float travel = length2(fit.u, fit.v);
                    if (!(__fadd_rn(s.travel[k], travel) > a.max_travel)) {
                        U = __fadd_rn(ub, fit.u);
                        V = __fadd_rn(vb, fit.v);
                        cstep = travel;
                        flags |= kIncCarried;
                    }
                }
            }
        } else {
            U = __fadd_rn(ub, smp.u);
            V = __fadd_rn(vb, smp.v);
            corr = smp.corr;
            const uint8_t nd = need_at(f, need, px, py);
            flags = (uint8_t)((nd << kIncNeedShift) | (smp.taylor ? kIncTaylor : 0));
            if (s.travel[k] > a.trusted_travel) {
                // confirmed only by a direct match of its subset from where it was last clean
                if (nd == 2 || !s.anchored[k]) {
                    flags |= kIncCarried;
                } else {
                    flags |= kIncMatch;
                    const int slot = atomicAdd(&counters[2], 1);
                    match_list[slot] = k;
                    match_info[3 * slot] = U;
                    match_info[3 * slot + 1] = V;
                    match_info[3 * slot + 2] = s.travel[k];
                }
            } else {
                flags |= kIncCarried | kIncValid;
            }
        }
    }
    fr.U[k] = U;
    fr.V[k] = V;
    fr.corr[k] = corr;
    fr.cstep[k] = cstep;
    fr.flags[k] = flags;
}

}  // namespace

namespace {

// The host's anchor matches written back: a confirmed node is measured
// (valid) at the matched position, an unconfirmed one keeps its sample as a
// carried total.
__global__ void apply_matches_kernel(int m, const IncMatch* __restrict__ rec, IncFrame fr) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m) return;
    const IncMatch r = rec[t];
    uint8_t fl = (uint8_t)(fr.flags[r.node] & ~kIncMatch);
    if (r.ok) {
        fr.U[r.node] = r.U;
        fr.V[r.node] = r.V;
        fr.corr[r.node] = r.corr;
        fl |= kIncCarried | kIncValid;
    } else {
        fl |= kIncCarried;
    }
    fr.flags[r.node] = fl;
}

__global__ void finish_kernel(int n, IncFrame fr, float* gu, float* gv, float* gcorr, uint8_t* gsolved,
                              int* counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const uint8_t fl = k < n ? fr.flags[k] : 0;
    const bool valid = (fl & kIncValid) != 0;
    if (k < n && gu) {
        gu[k] = valid ? fr.U[k] : 0.0f;
        gv[k] = valid ? fr.V[k] : 0.0f;
        gcorr[k] = valid ? fr.corr[k] : kCorrInvalid;
        gsolved[k] = valid ? 1 : 0;
    }
    count_add(&counters[0], (fl & kIncCarried) ? 1 : 0);
    count_add(&counters[1], (valid && (fl & kIncTaylor)) ? 1 : 0);
}

__global__ void update_kernel(IncGrid g, IncState s, IncFrame fr, float* travel_next, uint8_t* alive_next,
                              int* counters, int* refresh_list, float* refresh_xy, int* drop_list) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = g.gw * g.gh;
    bool carried = false;
    if (k < n) {
        const uint8_t fl = fr.flags[k];
        carried = (fl & kIncCarried) != 0;
        const bool valid = (fl & kIncValid) != 0;
        const int nd = (fl >> kIncNeedShift) & 3;
        travel_next[k] = (carried && !valid) ? __fadd_rn(s.travel[k], fr.cstep[k]) : 0.0f;
        alive_next[k] = carried ? 1 : 0;
        const float x = __fadd_rn(node_xf(g.rect_x, k % g.gw, g.step), fr.U[k]);
        const float y = __fadd_rn(node_xf(g.rect_y, k / g.gw, g.step), fr.V[k]);
        if (!carried || (valid && nd == 0)) {
            if (s.anchored[k]) drop_list[atomicAdd(&counters[4], 1)] = k;
        } else if (valid && nd == 1) {
            const int slot = atomicAdd(&counters[3], 1);
            refresh_list[slot] = k;
            refresh_xy[2 * slot] = x;
            refresh_xy[2 * slot + 1] = y;
        }
        if (carried) {
            atomicMin(&counters[6], fkey(x));
            atomicMin(&counters[7], fkey(y));
            atomicMax(&counters[8], fkey(x));
            atomicMax(&counters[9], fkey(y));
        }
    }
    count_add(&counters[5], carried ? 1 : 0);
}

__global__ void fill_init_kernel(int n, const float* __restrict__ U, const float* __restrict__ V,
                                 const uint8_t* __restrict__ valid, float* fu, float* fv, uint8_t* filled,
                                 int* counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = k < n && valid[k];
    if (k < n) {
        fu[k] = ok ? U[k] : 0.0f;
        fv[k] = ok ? V[k] : 0.0f;
        filled[k] = ok ? 1 : 0;
    }
    if (__any_sync(kAll, ok) && (threadIdx.x & 31) == 0) atomicOr(&counters[13], 1);
}

__global__ void fill_pass_kernel(int gw, int gh, const float* __restrict__ fu, const float* __restrict__ fv,
                                 const uint8_t* __restrict__ filled, float* nu, float* nv, uint8_t* nfilled,
                                 int* counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= gw * gh) return;
    if (filled[k]) {
        nu[k] = fu[k];
        nv[k] = fv[k];
        nfilled[k] = 1;
        return;
    }
    const int x = k % gw, y = k / gw;
    const int nx[4] = {x - 1, x + 1, x, x};
    const int ny[4] = {y, y, y - 1, y + 1};
    float su = 0.0f, sv = 0.0f;
    int cnt = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        if (nx[t] < 0 || nx[t] >= gw || ny[t] < 0 || ny[t] >= gh) continue;
        const int j = ny[t] * gw + nx[t];
        if (!filled[j]) continue;
        su = __fadd_rn(su, fu[j]);
        sv = __fadd_rn(sv, fv[j]);
        ++cnt;
    }
    if (cnt == 0) {
        nu[k] = fu[k];
        nv[k] = fv[k];
        nfilled[k] = 0;
        return;
    }
    nu[k] = __fdiv_rn(su, (float)cnt);
    nv[k] = __fdiv_rn(sv, (float)cnt);
    nfilled[k] = 1;
    counters[12] = 1;
}

__global__ void stretch_kernel(int gw, int gh, int step, const float* __restrict__ fu, const float* __restrict__ fv,
                               int* counters) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= gw * gh) return;
    const int x = k % gw, y = k / gw;
    const int ix = x + 1 < gw ? k + 1 : k, iy = y + 1 < gh ? k + gw : k;
    const double ux = (double)__fdiv_rn(__fsub_rn(fu[ix], fu[k]), (float)step);
    const double uy = (double)__fdiv_rn(__fsub_rn(fu[iy], fu[k]), (float)step);
    const double vx = (double)__fdiv_rn(__fsub_rn(fv[ix], fv[k]), (float)step);
    const double vy = (double)__fdiv_rn(__fsub_rn(fv[iy], fv[k]), (float)step);
    const double a = __dadd_rn(fabs(__dadd_rn(1.0, ux)), fabs(uy));
    const double b = __dadd_rn(fabs(vx), fabs(__dadd_rn(1.0, vy)));
    const double m = fmax(a, b);
    // non-negative doubles order as their bit patterns
    atomicMax(reinterpret_cast<unsigned long long*>(&counters[10]), (unsigned long long)__double_as_longlong(m));
}

inline unsigned blocks_for(int n) { return (unsigned)((n + 255) / 256); }

}  // namespace

cudaError_t launch_inc_need(const IncField& f, int subset, uint8_t* need, cudaStream_t st) {
    const int n = f.gw * f.gh;
    if (n <= 0) return cudaSuccess;
    need_kernel<<<blocks_for(n), 256, 0, st>>>(f, subset, need);
    return cudaGetLastError();
}

cudaError_t launch_inc_first(const IncField& f, const uint8_t* need, const IncFrame& fr, cudaStream_t st) {
    const int n = f.gw * f.gh;
    if (n <= 0) return cudaSuccess;
    first_kernel<<<blocks_for(n), 256, 0, st>>>(f, need, fr);
    return cudaGetLastError();
}

cudaError_t launch_inc_step(const IncGrid& g, const IncState& s, const IncField& f, const uint8_t* need,
                            const IncStepArgs& a, const IncFrame& fr, int* counters, int* match_list,
                            float* match_info, cudaStream_t st) {
    const int n = g.gw * g.gh;
    if (n <= 0) return cudaSuccess;
    step_kernel<<<blocks_for(n), 256, 0, st>>>(g, s, f, need, a, fr, counters, match_list, match_info);
    return cudaGetLastError();
}

cudaError_t launch_inc_apply_matches(int m, const IncMatch* rec, const IncFrame& fr, cudaStream_t st) {
    if (m <= 0) return cudaSuccess;
    apply_matches_kernel<<<blocks_for(m), 256, 0, st>>>(m, rec, fr);
    return cudaGetLastError();
}

cudaError_t launch_inc_finish(int n, const IncFrame& fr, float* gu, float* gv, float* gcorr, uint8_t* gsolved,
                              int* counters, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    finish_kernel<<<blocks_for(n), 256, 0, st>>>(n, fr, gu, gv, gcorr, gsolved, counters);
    return cudaGetLastError();
}

cudaError_t launch_inc_update(const IncGrid& g, const IncState& s, const IncFrame& fr, float* travel_next,
                              uint8_t* alive_next, int* counters, int* refresh_list, float* refresh_xy,
                              int* drop_list, cudaStream_t st) {
    const int n = g.gw * g.gh;
    if (n <= 0) return cudaSuccess;
    update_kernel<<<blocks_for(n), 256, 0, st>>>(g, s, fr, travel_next, alive_next, counters, refresh_list,
                                                 refresh_xy, drop_list);
    return cudaGetLastError();
}

cudaError_t launch_inc_fill_init(int n, const float* U, const float* V, const uint8_t* valid, float* fu, float* fv,
                                 uint8_t* filled, int* counters, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    fill_init_kernel<<<blocks_for(n), 256, 0, st>>>(n, U, V, valid, fu, fv, filled, counters);
    return cudaGetLastError();
}

cudaError_t launch_inc_fill_pass(int gw, int gh, const float* fu, const float* fv, const uint8_t* filled, float* nu,
                                 float* nv, uint8_t* nfilled, int* counters, cudaStream_t st) {
    const int n = gw * gh;
    if (n <= 0) return cudaSuccess;
    fill_pass_kernel<<<blocks_for(n), 256, 0, st>>>(gw, gh, fu, fv, filled, nu, nv, nfilled, counters);
    return cudaGetLastError();
}

cudaError_t launch_inc_stretch(int gw, int gh, int step, const float* fu, const float* fv, int* counters,
                               cudaStream_t st) {
    const int n = gw * gh;
    if (n <= 0) return cudaSuccess;
    stretch_kernel<<<blocks_for(n), 256, 0, st>>>(gw, gh, step, fu, fv, counters);
    return cudaGetLastError();
}

}  // namespace dic
