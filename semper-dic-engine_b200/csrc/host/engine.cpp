// run_full_field on the device: see engine.hpp.
//
// Stage map (reference file:line -> what runs where):
//   prepare_data of the deformed frame (full_field_solver.cpp:199-201)      image kernel
//   grid scan (full_field_solver.cpp:266-318)                               scan kernel
//   Hessian pre-pass (full_field_solver.cpp:380-428)                        pool kernel (FP64)
//   anchor lattice solves (full_field_anchors.cpp:355-452)                  solve kernel, one batch
//   median test / routing / refit (full_field_anchors.cpp:122-168,455-561)  host
//   Delaunay + affine per triangle (full_field_mesh.cpp:66-137)             host (geometry.hpp)
//   guess assignment / extrapolation / homography / smoothing (:168-280)    mesh kernels
//   Path C (full_field_path_c.cpp:27-156)                                   solve kernel, one batch
//   Path A (full_field_path_a.cpp:28-114)                                   task + solve + commit kernels
//   Path B rounds (full_field_path_b.cpp:148-412)                           host claims, batched solves
//   median test, VSG, packing (full_field_solver_stats.cpp:21-91)           strain kernels
//   metrics (full_field_solver_stats.cpp:182-280)                           host
#include "engine.hpp"
#include "proposal.hpp"

#include <algorithm>
#include <limits>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <map>
#include <deque>
#include <mutex>
#include <queue>
#include <thread>

#include "../kernels/icgn.cuh"
#include "../kernels/mesh.cuh"
#include "../kernels/prep.cuh"
#include "../kernels/incmask.cuh"
#include "../kernels/strain.cuh"
#include "geometry.hpp"

namespace semper_b200 {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

namespace {

// include/semper/tuning.hpp
constexpr float kCorrAccept = 0.15f;
constexpr float kAnchorSparseCoverage = 0.05f;
constexpr int kAnchorTarget = 256;
constexpr float kAnchorAcceptScore = 0.40f;
constexpr float kAnchorMedianTol = 1.0f;
constexpr float kAnchorFullFraction = 0.60f;
constexpr int kAnchorFullMinVertices = 10;
constexpr float kAnchorFullCoverage = 0.30f;
constexpr double kAnchorRefitRansacPx = 1.0;
constexpr int kAnchorRefitMinPoints = 8;
constexpr float kSimilarityMinCornerPx = 4.0f;
constexpr float kSimilarityKeepFraction = 0.90f;
constexpr int kPathCMaxCandidates = 9;
constexpr int kPathBBatchNodes = 32;
constexpr int kMetricsLen = 24;

enum class Quality { NONE, SPARSE, FULL };

int metrics_prefix_len(int len) { return len < 16 ? 0 : len >= kMetricsLen ? kMetricsLen : len == 18 ? 17 : len; }

bool clip_axis(int& lo, int& len, int step, int extent) {
    int64_t a = lo;
    const int64_t b = std::min<int64_t>((int64_t)lo + (int64_t)len, extent);
    if (a < 0) a += ((-a + step - 1) / step) * (int64_t)step;
    if (b <= a) return false;
    lo = (int)a;
    len = (int)(b - a);
    return true;
}

int64_t max_strain_window(const Params& p) {
    if (p.step <= 0) return 0;
    const int64_t gmin = std::min(p.rect_w / p.step, p.rect_h / p.step);
    return 2 * (gmin + 1) * (int64_t)p.step;
}

// validate_params (full_field_solver.cpp:97-111).
int validate_params(Params& p, int width, int height) {
    if (width <= 0 || height <= 0) return -3;
    if ((int64_t)width * (int64_t)height > (int64_t)INT32_MAX) return -3;
    if (p.step <= 0) return -2;
    if (p.subset_size < 3 || p.subset_size % 2 == 0) return -3;
    if (p.rect_w <= 0 || p.rect_h <= 0) return -2;
    if (!clip_axis(p.rect_x, p.rect_w, p.step, width)) return -2;
    if (!clip_axis(p.rect_y, p.rect_h, p.step, height)) return -2;
    if (p.rect_w / p.step <= 0 || p.rect_h / p.step <= 0) return -2;
    if ((int64_t)p.strain_window > max_strain_window(p)) return -3;
    return 0;
}

// StrainCalculator::vsg_window_node_count (strain_calculator.cpp:12-25).
int vsg_window_node_count(int step, int window) {
    if (step <= 0) return 0;
    const float radius = window / 2.0f;
    const int grid_rad = (int)std::ceil(radius / (float)step);
    const double r2 = (double)(radius * radius) + 1.0e-5;
    int count = 0;
    for (int dy = -grid_rad; dy <= grid_rad; ++dy)
        for (int dx = -grid_rad; dx <= grid_rad; ++dx) {
            const double px = (double)(dx * step), py = (double)(dy * step);
            if (px * px + py * py <= r2) ++count;
        }
    return count;
}

int lattice_count(int n, int stride) {
    if (n <= 0 || stride <= 0) return 0;
    int c = (n + stride - 1) / stride;
    if ((c - 1) * stride != n - 1) c++;
    return c;
}

// plan_anchor_lattice (full_field_anchors.cpp:73-120).
void plan_lattice(int gw, int gh, int& sx, int& sy) {
    int stride = (int)std::lround(std::sqrt((double)(gw * gh) / (double)kAnchorTarget));
    stride = std::max(1, stride);
    const int budget = lattice_count(gw, stride) * lattice_count(gh, stride);
    sx = stride;
    sy = stride;
    while (sx > 1 && lattice_count(gw, sx) < 3) --sx;
    while (sy > 1 && lattice_count(gh, sy) < 3) --sy;
    while (lattice_count(gw, sx) * lattice_count(gh, sy) > budget) {
        const bool gx = lattice_count(gw, sx + 1) >= 3, gy = lattice_count(gh, sy + 1) >= 3;
        if (!gx && !gy) break;
        if (gx && (!gy || lattice_count(gw, sx) >= lattice_count(gh, sy))) ++sx;
        else ++sy;
    }
}

// util::median_inplace (src/util/median.hpp:21-30) on finite values.
float median_of(std::vector<float> v) {
    if (v.empty()) return 0.0f;
    std::sort(v.begin(), v.end());
    const size_t n = v.size(), mid = n / 2;
    if (n % 2 == 1) return v[mid];
    return 0.5f * (v[mid - 1] + v[mid]);
}

struct Anchor {
    int gx = 0, gy = 0;
    float rx = 0, ry = 0, u = 0, v = 0, ux = 0, uy = 0, vx = 0, vy = 0, corr = 0;
    bool used_simplex = false, vertex = false, output = false, kept = false;
};

struct HostStats {
    long long icgn_iters = 0;
    int points = 0, simp_calls = 0, simp_saved = 0, simp_dead = 0;
    void record(const dic_result& r) {
        icgn_iters += r.iters;
        if (r.flags & DIC_RES_RESCUE) {
            simp_calls++;
            if (r.status == 0 && r.score <= kCorrAccept) simp_saved++;
            else simp_dead++;
        }
    }
};

// Progress ticker: percentages from a thread the solve owns, the final 100 on
// the caller's thread (full_field_solver.cpp:334-373, 537-544).
class Ticker {
public:
    explicit Ticker(Progress cb) : cb_(std::move(cb)) {
        if (cb_) th_ = std::thread([this] { loop(); });
    }
    ~Ticker() { stop(); }
    void set(int pct) { pct_.store(pct, std::memory_order_relaxed); }
    void stop() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        if (th_.joinable()) th_.join();
    }

private:
    void loop() {
        std::unique_lock<std::mutex> lk(m_);
        while (!stop_) {
            const int p = pct_.load(std::memory_order_relaxed);
            lk.unlock();
            try {
                cb_(p);
            } catch (...) {
            }
            lk.lock();
            cv_.wait_for(lk, std::chrono::milliseconds(100), [this] { return stop_; });
        }
    }
    Progress cb_;
    std::thread th_;
    std::mutex m_;
    std::condition_variable cv_;
    bool stop_ = false;
    std::atomic<int> pct_{10};
};

struct Cancelled {};

}  // namespace

struct Engine::Impl {
    Engine& E;
    explicit Impl(Engine& e) : E(e) {}

    DevBuf<float> rI, rGx, rGy;      // reference planes
    DevBuf<uint8_t> dGray;           // deformed frame bytes
    DevBuf<uint8_t> rGray;           // reference frame bytes (global motion)
    bool ref_gray = false;           // rGray holds the current reference
    bool ref_ghost = false;          // the reference planes may hold Ghost Wall pixels (a mask was given)
    const uint8_t* last_def = nullptr;
    dic::GlobalMotion gm;
    DevBuf<float> dI, dGx, dGy;      // deformed planes (gradients kept for adoption)
    DevBuf<uint8_t> dMask;

    // grid scan + pool cache (RefPrecompute, full_field_internal.hpp:214-242)
    bool grid_valid = false;
    Params key;
    std::vector<uint8_t> mask_key;
    int gridW = 0, gridH = 0, total_valid = 0;
    DevBuf<uint8_t> skip;
    std::vector<uint8_t> h_skip;
    DevBuf<uint8_t> pool_valid;
    DevBuf<float2> pool_ms;
    DevBuf<double> pool_Hs;

    // per-solve field
    DevBuf<float> fu, fv, fux, fuy, fvx, fvy, fcorr;
    DevBuf<uint8_t> fsolved, ftag;
    DevBuf<int> fiters;
    DevBuf<float> gu, gv, gux, guy, gvx, gvy, gtmp;
    DevBuf<uint8_t> in_mesh;
    DevBuf<dic_task> tasks;
    DevBuf<dic_result> results;
    DevBuf<int> counters;  // [1] n_tasks [2] n_valid [3] n_fail [4] n_drop [5..6] emit [7] n_boundary [9] TMA error
    DevBuf<int> solve_q;   // the solve's work counters
    DevBuf<int> deferred;  // tasks the fast solve pass leaves to the general one
    DevBuf<dic::PathStats> pstats;
    DevBuf<dic::BoundarySeed> bseeds;
    DevBuf<dic::ScatterRec> scat;
    DevBuf<dic::MeshTri> tris;
    DevBuf<uint8_t> valid, fail;
    DeviceField last_field;  // the field of the last run (device pointers)
    DevBuf<float> exx, eyy, exy;
    DevBuf<unsigned char> pack_scratch;
    DevBuf<float> d_out;

    int sm_count = 0;
    cudaEvent_t ev[10];

    // Path B keeps two rounds in flight (full_field_path_b.cpp:148-412). Each
    // in-flight round has its own slot: a stream, scratch and host staging, so
    // the second round's solves run on the device while the first round is
    // committed on the host. A round's tasks and results stay in mapped pinned
    // host memory that the kernels read and write directly (a round is at most
    // a few hundred tasks): no copies to wait for between the rounds' kernels.
    struct Slot {
        DevBuf<int> q, deferred;
        dic_task* h_tasks = nullptr;  // mapped pinned
        dic_result* h_results = nullptr;
        dic_task* d_tasks = nullptr;  // their device addresses
        dic_result* d_results = nullptr;
        size_t h_n = 0, n = 0;
        cudaStream_t s = nullptr;
        cudaEvent_t done = nullptr;
    };
    Slot slots[2];

    ~Impl() {
        for (Slot& S : slots) {
            if (S.h_tasks) cudaFreeHost(S.h_tasks);
            if (S.h_results) cudaFreeHost(S.h_results);
            if (S.done) cudaEventDestroy(S.done);
            if (S.s) cudaStreamDestroy(S.s);
        }
    }

    // Enqueue one round's solves on slot k, after the work already on the
    // engine stream (event `after`); results land in the slot's mapped buffer.
    void launch_round(int k, const std::vector<dic_task>& tk, const Params& p, cudaEvent_t after) {
        Slot& S = slots[k];
        if (!S.s) {
            check(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking), "slot stream");
            check(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming), "slot event");
            S.q.ensure(8);
        }
        S.n = tk.size();
        check(cudaStreamWaitEvent(S.s, after, 0), "slot wait");
        if (S.n > 0) {
            if (S.h_n < S.n) {
                if (S.h_tasks) cudaFreeHost(S.h_tasks);
                if (S.h_results) cudaFreeHost(S.h_results);
                S.h_tasks = nullptr;
                S.h_results = nullptr;
                S.h_n = 0;
                const size_t want = std::max<size_t>(S.n, 256);
                check(cudaHostAlloc(&S.h_tasks, want * sizeof(dic_task), cudaHostAllocMapped), "mapped tasks");
                check(cudaHostAlloc(&S.h_results, want * sizeof(dic_result), cudaHostAllocMapped), "mapped results");
                check(cudaHostGetDevicePointer(&S.d_tasks, S.h_tasks, 0), "mapped tasks address");
                check(cudaHostGetDevicePointer(&S.d_results, S.h_results, 0), "mapped results address");
                S.h_n = want;
            }
            S.deferred.ensure(std::max(S.deferred.n, S.n));
            std::memcpy(S.h_tasks, tk.data(), S.n * sizeof(dic_task));
            dic::SolveArgs a = solve_args(p.subset_size, p.six);
            a.tasks = S.d_tasks;
            a.n_tasks = (int)S.n;
            a.n_tasks_dev = nullptr;
            a.results = S.d_results;
            a.queue = S.q.p;
            a.deferred = S.deferred.p;
            launched(2, dic::launch_solve(a, p.six ? 1 : 0, solve_grid((int)S.n), S.s), "round solve");
        }
        check(cudaEventRecord(S.done, S.s), "slot record");
    }

    const dic_result* wait_round(int k) {
        check(cudaEventSynchronize(slots[k].done), "slot sync");
        poll_cancel();
        return slots[k].h_results;
    }

    dic::FieldGrid field() {
        return dic::FieldGrid{fu.p, fv.p, fux.p, fuy.p, fvx.p, fvy.p, fcorr.p, fsolved.p, fiters.p};
    }
    dic::MeshGrid mesh() { return dic::MeshGrid{gu.p, gv.p, gux.p, guy.p, gvx.p, gvy.p, in_mesh.p}; }

    void sync() { check(cudaStreamSynchronize(E.stream_), "stream sync"); }
    void launched(int kernels, cudaError_t e, const char* what) {
        check(e, what);
        E.times_.launches += kernels;
    }
    void poll_cancel() {
        if (E.h_cancel_[0]) throw Cancelled{};
    }

    // Autotuner of the fast pass's shape, per (subset size, interpolator): the
    // first four large Path A launches alternate between reading the
    // reference subset from the planes and staging it in shared memory; the
    // shape with the lower of its two times per subset pixel-iteration is kept
    // from then on (two trials each, so that the first frame's cold caches do
    // not decide). Both shapes give the same results, so the choice changes
    // the time only.
    static constexpr int kTuneTrials = 4;
    struct Tune {
        int trials = 0, best = -1;
        double t[2] = {0.0, 0.0};
    };
    std::map<std::pair<int, int>, Tune> tune;
    int tune_pick(int dim, int six) {
        const Tune& t = tune[{dim, six}];
        return t.best >= 0 ? t.best : t.trials % 2;
    }
    void tune_record(int dim, int six, int variant, double ms_per_pixel_iter) {
        Tune& t = tune[{dim, six}];
        if (t.best >= 0 || !(ms_per_pixel_iter > 0.0)) return;
        if (t.t[variant] == 0.0 || ms_per_pixel_iter < t.t[variant]) t.t[variant] = ms_per_pixel_iter;
        if (++t.trials >= kTuneTrials) t.best = t.t[1] < t.t[0] ? 1 : 0;
    }

    // The learned proposal of the global model, from the network's
    // predictions on patch pairs (64 x 64 patches box-averaged by f):
    // 1. the rotation about the ROI centre, four rounds at f = 4, 4, 4, 2 over
    //    nine pairs (the centre and eight at 48 px around it): each round
    //    samples the deformed patches through the current estimate, the
    //    network predicts what is left of the motion, every pair's map takes
    //    its prediction on, and the estimate becomes the rotation by the
    //    pairs' circular median angle that lands the centre on their median
    //    landing (a pure rotation, so that no stray shear or scale carries
    //    the next round outside the motions the network was trained on);
    // 2. a 6 x 6 grid of pairs over the central 70 % of the ROI, started from
    //    that rotation, three rounds at f = 4, 2, 1, each pair's own affine
    //    map refined by the network's prediction;
    // 3. a homography fitted to where the pairs' origins land (DLT with an
    //    inlier refit at 6 px). False when the fit fails or keeps fewer than
    //    8 pairs.
    struct Affine {
        double a00 = 1, a01 = 0, a10 = 0, a11 = 1, bx = 0, by = 0;
    };
    // T o E, with E the network's output for a pair whose patches share the
    // origin (ox, oy): E(X) = o + f t + A_r (X - o).
    static Affine compose(const Affine& T, const float* o6, double ox, double oy, int f) {
        const double r00 = 1.0 + o6[0], r01 = o6[1], r10 = o6[2], r11 = 1.0 + o6[3];
        const double ex = ox + f * dic::kPpTScale * o6[4] - (r00 * ox + r01 * oy);
        const double ey = oy + f * dic::kPpTScale * o6[5] - (r10 * ox + r11 * oy);
        Affine C;
        C.a00 = T.a00 * r00 + T.a01 * r10;
        C.a01 = T.a00 * r01 + T.a01 * r11;
        C.a10 = T.a10 * r00 + T.a11 * r10;
        C.a11 = T.a10 * r01 + T.a11 * r11;
        C.bx = T.a00 * ex + T.a01 * ey + T.bx;
        C.by = T.a10 * ex + T.a11 * ey + T.by;
        return C;
    }
    static void map_of(const Affine& T, float cx, float cy, float* m) {
        m[0] = cx;
        m[1] = cy;
        m[2] = (float)T.a00;
        m[3] = (float)T.a01;
        m[4] = (float)T.a10;
        m[5] = (float)T.a11;
        m[6] = (float)T.bx;
        m[7] = (float)T.by;
    }

    static Affine rotation_landing(const std::vector<Affine>& C, double ox, double oy) {
        const size_t n = C.size();
        std::vector<double> th(n), lx(n), ly(n);
        for (size_t k = 0; k < n; ++k) {
            th[k] = std::atan2(C[k].a10 - C[k].a01, C[k].a00 + C[k].a11);
            lx[k] = C[k].a00 * ox + C[k].a01 * oy + C[k].bx;
            ly[k] = C[k].a10 * ox + C[k].a11 * oy + C[k].by;
        }
        // circular median: the angle with the least summed distance to the others
        size_t best = 0;
        double best_d = 0.0;
        for (size_t k = 0; k < n; ++k) {
            double d = 0.0;
            for (size_t j = 0; j < n; ++j) d += std::fabs(std::remainder(th[k] - th[j], 2.0 * M_PI));
            if (k == 0 || d < best_d) {
                best = k;
                best_d = d;
            }
        }
        std::nth_element(lx.begin(), lx.begin() + n / 2, lx.end());
        std::nth_element(ly.begin(), ly.begin() + n / 2, ly.end());
        const double c = std::cos(th[best]), s = std::sin(th[best]);
        Affine T;
        T.a00 = c;
        T.a01 = -s;
        T.a10 = s;
        T.a11 = c;
        T.bx = lx[n / 2] - (c * ox - s * oy);
        T.by = ly[n / 2] - (s * ox + c * oy);
        return T;
    }

    bool learned_model(const Params& params, const uint8_t* d_def, double H[9]) {
        LearnedSeed& L = E.last_learned_;
        L = LearnedSeed{};
        L.ran = true;
        ProposalNet& net = *E.proposal_;
        cudaStream_t st = E.stream_;
        const int W = E.W_, Hh = E.H_;
        cudaEvent_t e0, e1;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        check(cudaEventRecord(e0, st), "event");
        const int cx = params.rect_x + params.rect_w / 2, cy = params.rect_y + params.rect_h / 2;
        const double ox = cx - 0.5, oy = cy - 0.5;
        constexpr int kRing = 9, G = 6;
        int px[G * G], py[G * G];
        px[0] = cx;
        py[0] = cy;
        for (int k = 1; k < kRing; ++k) {
            const double a = (k - 1) * (M_PI / 4.0);
            px[k] = cx + (int)std::lround(48.0 * std::cos(a));
            py[k] = cy + (int)std::lround(48.0 * std::sin(a));
        }
        float maps[G * G * 8], o6[G * G * 6];
        Affine T;
        std::vector<Affine> C(kRing);
        for (const int f : {4, 4, 4, 2}) {
            for (int k = 0; k < kRing; ++k) map_of(T, (float)px[k], (float)py[k], maps + 8 * k);
            net.predict_warped(rGray.p, d_def, W, Hh, W, maps, kRing, f, o6, st);
            for (int k = 0; k < kRing; ++k) C[k] = compose(T, o6 + 6 * k, px[k] - 0.5, py[k] - 0.5, f);
            T = rotation_landing(C, ox, oy);
            L.pairs += kRing;
        }
        constexpr int K = G * G;
        std::vector<Affine> Tg(K, T);
        for (int j = 0; j < G; ++j)
            for (int i = 0; i < G; ++i) {
                px[j * G + i] = params.rect_x + (int)(params.rect_w * (0.15 + 0.7 * (i + 0.5) / G));
                py[j * G + i] = params.rect_y + (int)(params.rect_h * (0.15 + 0.7 * (j + 0.5) / G));
            }
        for (const int f : {4, 2, 1}) {
            for (int k = 0; k < K; ++k) map_of(Tg[k], (float)px[k], (float)py[k], maps + 8 * k);
            net.predict_warped(rGray.p, d_def, W, Hh, W, maps, K, f, o6, st);
            for (int k = 0; k < K; ++k) Tg[k] = compose(Tg[k], o6 + 6 * k, px[k] - 0.5, py[k] - 0.5, f);
            L.pairs += K;
        }
        std::vector<semper_geom::Pt> rp, dp;
        for (int k = 0; k < K; ++k) {
            const double x = px[k] - 0.5, y = py[k] - 0.5;
            const double X = Tg[k].a00 * x + Tg[k].a01 * y + Tg[k].bx, Y = Tg[k].a10 * x + Tg[k].a11 * y + Tg[k].by;
            if (!std::isfinite(X) || !std::isfinite(Y)) continue;
            rp.push_back({x, y});
            dp.push_back({X, Y});
        }
        bool ok = rp.size() >= 8 && semper_geom::fit_homography(rp, dp, 6.0, H);
        if (ok) {
            for (size_t k = 0; k < rp.size(); ++k) {
                double X, Y, J[4];
                if (semper_geom::homography_at(H, rp[k].x, rp[k].y, X, Y, J) &&
                    std::hypot(X - dp[k].x, Y - dp[k].y) <= 6.0)
                    L.inliers++;
            }
            ok = L.inliers >= 8;
        }
        check(cudaEventRecord(e1, st), "event");
        check(cudaEventSynchronize(e1), "event");
        cudaEventElapsedTime(&L.ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        E.times_.launches += 7 * 14;
        L.proposed = ok;
        if (ok) std::copy(H, H + 9, L.H);
        return ok;
    }

    // Each anchor's displacement under the proposed model H, refined by the
    // network: the map starts as H's local affine at the anchor, two rounds
    // at f = 2 and 1 move it by the network's predictions, and the guess is
    // where the anchor's pixel lands (the gradients stay H's). One entry per
    // lattice node, NaN for nodes that are not attempted.
    std::vector<float> learned_anchor_guesses(const uint8_t* d_def, const double* H, const Params& params,
                                              const std::vector<int>& lat_x, const std::vector<int>& lat_y,
                                              const std::vector<uint8_t>& solved, int gW) {
        ProposalNet& net = *E.proposal_;
        const int LW = (int)lat_x.size(), LH = (int)lat_y.size(), N = LW * LH;
        std::vector<float> uv((size_t)2 * N, std::numeric_limits<float>::quiet_NaN());
        std::vector<int> idx, px, py;
        std::vector<Affine> Tk;
        for (int i = 0; i < N; ++i) {
            const int gx = lat_x[i % LW], gy = lat_y[i / LW];
            if (solved[(size_t)gy * gW + gx]) continue;
            const int x = params.rect_x + gx * params.step, y = params.rect_y + gy * params.step;
            double X, Y, J[4];
            if (!semper_geom::homography_at(H, x, y, X, Y, J)) continue;
            Affine T;
            T.a00 = J[0];
            T.a01 = J[1];
            T.a10 = J[2];
            T.a11 = J[3];
            T.bx = X - (J[0] * x + J[1] * y);
            T.by = Y - (J[2] * x + J[3] * y);
            idx.push_back(i);
            px.push_back(x);
            py.push_back(y);
            Tk.push_back(T);
        }
        const int K = (int)idx.size(), B = net.max_batch();
        std::vector<float> maps((size_t)B * 8), o6((size_t)B * 6);
        for (const int f : {2, 1}) {
            for (int k0 = 0; k0 < K; k0 += B) {
                const int nb = std::min(B, K - k0);
                for (int k = 0; k < nb; ++k) map_of(Tk[k0 + k], (float)px[k0 + k], (float)py[k0 + k], &maps[8 * k]);
                net.predict_warped(rGray.p, d_def, E.W_, E.H_, E.W_, maps.data(), nb, f, o6.data(), E.stream_);
                for (int k = 0; k < nb; ++k)
                    Tk[k0 + k] = compose(Tk[k0 + k], &o6[6 * k], px[k0 + k] - 0.5, py[k0 + k] - 0.5, f);
                E.times_.launches += 14;
                E.last_learned_.pairs += nb;
            }
        }
        for (int k = 0; k < K; ++k) {
            const double x = px[k], y = py[k];
            const double X = Tk[k].a00 * x + Tk[k].a01 * y + Tk[k].bx, Y = Tk[k].a10 * x + Tk[k].a11 * y + Tk[k].by;
            if (!std::isfinite(X) || !std::isfinite(Y)) continue;
            uv[2 * (size_t)idx[k]] = (float)(X - x);
            uv[2 * (size_t)idx[k] + 1] = (float)(Y - y);
        }
        return uv;
    }

    dic::SolveArgs solve_args(int dim, int six) {
        dic::SolveArgs a{};
        a.refI = rI.p;
        a.refGx = rGx.p;
        a.refGy = rGy.p;
        a.defI = dI.p;
        a.W = E.W_;
        a.H = E.H_;
        a.pitch = pitch();
        a.err = counters.p + 9;
        a.tma_max_polls = E.tma_polls_;
        a.pool_valid = pool_valid.p;
        a.pool_ms = pool_ms.p;
        a.pool_Hs = pool_Hs.p;
        a.dim = dim;
        a.max_n = dim * dim;
        a.lm = 1;
        a.cancel = E.d_cancel_;
        a.queue = solve_q.p;
        a.ref_no_ghost = ref_ghost ? 0 : 1;
        a.tile_spread = tile_spread;
        (void)six;
        return a;
    }

    // The solves' TMA tiles follow the seeding model: a rotated or stretched
    // subset's bounding box outgrows the subset by max(|J00| + |J01|,
    // |J10| + |J11|) (J the model's local linear map at the ROI centre), and
    // the tiles grow with it, 4 % beyond for the field's own variation.
    // Below 1.03 the tiles of an unrotated subset serve; the spread is capped
    // at 1.5 (any rotation), so a model that stretches further (a zoom) keeps
    // tiles that fit shared memory, its outer samples read global memory.
    // the last Delaunay triangulation of the mesh guess and its points
    std::vector<semper_geom::Pt> dl_pts;
    std::vector<semper_geom::Tri> dl_tris;

    float tile_spread = 0.f;
    void set_tile_spread(const double* H, const Params& p) {
        tile_spread = 0.f;
        if (!H) return;
        double X, Y, J[4];
        if (!semper_geom::homography_at(H, p.rect_x + 0.5 * p.rect_w, p.rect_y + 0.5 * p.rect_h, X, Y, J)) return;
        const double g = std::max(std::fabs(J[0]) + std::fabs(J[1]), std::fabs(J[2]) + std::fabs(J[3]));
        if (std::isfinite(g) && g > 1.03) tile_spread = (float)std::min(1.04 * g, 1.5);
    }

    int solve_grid(int ntasks) {
        if (E.solve_blocks_ > 0) return E.solve_blocks_;
        const int per_block = dic::kSolveThreads / 32;
        const int need = (ntasks + per_block - 1) / per_block;
        return std::max(1, std::min(need, sm_count * 4));
    }

    // One batch of subset solves (host tasks in, host results out).
    std::vector<dic_result> solve_batch(const std::vector<dic_task>& tk, const Params& p) {
        std::vector<dic_result> out(tk.size());
        if (tk.empty()) return out;
        tasks.ensure(std::max(tasks.n, tk.size()));
        results.ensure(std::max(results.n, tk.size()));
        deferred.ensure(std::max(deferred.n, tk.size()));
        check(cudaMemcpyAsync(tasks.p, tk.data(), tk.size() * sizeof(dic_task), cudaMemcpyHostToDevice, E.stream_),
              "H2D tasks");
        dic::SolveArgs a = solve_args(p.subset_size, p.six);
        a.tasks = tasks.p;
        a.n_tasks = (int)tk.size();
        a.n_tasks_dev = nullptr;
        a.results = results.p;
        a.deferred = deferred.p;
        launched(2, dic::launch_solve(a, p.six ? 1 : 0, solve_grid((int)tk.size()), E.stream_), "solve");
        check(cudaMemcpyAsync(out.data(), results.p, tk.size() * sizeof(dic_result), cudaMemcpyDeviceToHost,
                              E.stream_),
              "D2H results");
        sync();
        poll_cancel();
        return out;
    }

    int pitch() const { return (E.W_ + 3) & ~3; }

    // pack_full_field_output (full_field_solver_stats.cpp:21-91) over the
    // field buffers: the displacement median test, VSG strain and packing on
    // the device, into d_out_p (capacity floats). Returns the points written;
    // records ev[8] after the packing.
    int strain_pack(int gW, int gH, int rect_x, int rect_y, int step, int window, float* d_out_p, int capacity,
                    int& dropped_outlier, int& dropped_post) {
        cudaStream_t st = E.stream_;
        const size_t NG = (size_t)gW * gH;
        valid.ensure(NG); fail.ensure(NG); exx.ensure(NG); eyy.ensure(NG); exy.ensure(NG);
        launched(1, dic::launch_valid((int)NG, field(), valid.p, st), "valid");
        dropped_outlier = 0;
        for (int pass = 0; pass < 5; ++pass) {
            check(cudaMemsetAsync(counters.p + 3, 0, sizeof(int), st), "memset");
            launched(1, dic::launch_median_pass(gW, gH, fu.p, fv.p, valid.p, fail.p, counters.p + 3, st), "median");
            int nf = 0;
            check(cudaMemcpyAsync(&nf, counters.p + 3, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H fail");
            sync();
            if (nf == 0) break;
            launched(1, dic::launch_clear_failed((int)NG, valid.p, fail.p, st), "clear");
            dropped_outlier += nf;
        }
        launched(1, dic::launch_vsg(gW, gH, step, window, fu.p, fv.p, valid.p, exx.p, eyy.p, exy.p, st), "vsg");
        const size_t scr = dic::pack_scratch_bytes((int)NG);
        pack_scratch.ensure(std::max(pack_scratch.n, scr));
        check(cudaMemsetAsync(counters.p + 4, 0, 3 * sizeof(int), st), "memset");
        const int max_pts = capacity / 8;
        launched(4, dic::launch_pack(gW, gH, rect_x, rect_y, step, max_pts, valid.p, fu.p, fv.p, fcorr.p, exx.p, eyy.p,
                                     exy.p, d_out_p, counters.p + 4, counters.p + 5, pack_scratch.p, pack_scratch.n, st),
                 "pack");
        // the packing counts [4..6] and, in the same copy, the run's TMA-wait flag [9]
        int cnts[6] = {0, 0, 0, 0, 0, 0};
        check(cudaMemcpyAsync(cnts, counters.p + 4, 6 * sizeof(int), cudaMemcpyDeviceToHost, st), "D2H pack");
        check(cudaEventRecord(ev[8], st), "event");
        sync();
        E.last_tma_timeout_ = cnts[5];
        dropped_post = cnts[0];
        return std::min(cnts[1] + cnts[2], max_pts);
    }

    // The patch reference of an anchor match: its gray bytes, prepared planes,
    // pool entry, task and result.
    DevBuf<uint8_t> aGray, aSkip, aValid;
    DevBuf<float> aI, aGx, aGy, aMs;
    DevBuf<double> aHs;
    DevBuf<dic_task> aTask;
    DevBuf<dic_result> aRes;
    DevBuf<int> aQ;

    // the material-mask warp of incremental DIC
    DevBuf<uint8_t> mMask0, mOut, mTmp;
    size_t mMask0_px = 0;  // pixels of the material mask last uploaded to mMask0
    DevBuf<float> mU, mV;
    DevBuf<int> mBox;

    void prepare_deformed(const uint8_t* d_def) {
        const size_t n = (size_t)pitch() * E.H_;
        dI.ensure(n);
        dGx.ensure(n);
        dGy.ensure(n);
        launched(1, dic::launch_image_prep(d_def, nullptr, E.W_, E.H_, pitch(), dI.p, dGx.p, dGy.p, E.stream_),
                 "image prep");
    }

    int run(const uint8_t* d_def, const uint8_t* mask, Params params, float* d_out_p, int capacity,
            float* metrics, int metrics_len, const double* model_H, Progress progress, Capture* capture);
};

Engine::Engine() : impl_(new Impl(*this)) {
    check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "stream");
    int* h = nullptr;
    check(cudaHostAlloc(&h, sizeof(int), cudaHostAllocMapped), "cancel flag");
    h_cancel_ = h;
    h_cancel_[0] = 0;
    check(cudaHostGetDevicePointer(&d_cancel_, h, 0), "cancel flag device pointer");
    int dev = 0;
    check(cudaGetDevice(&dev), "device");
    check(cudaDeviceGetAttribute(&impl_->sm_count, cudaDevAttrMultiProcessorCount, dev), "SM count");
    for (auto& e : impl_->ev) check(cudaEventCreate(&e), "event");
    impl_->counters.ensure(16);
    impl_->solve_q.ensure(4);
    impl_->pstats.ensure(1);
}

Engine::~Engine() {
    if (impl_)
        for (auto& e : impl_->ev) cudaEventDestroy(e);
    impl_.reset();
    if (h_cancel_) cudaFreeHost((void*)h_cancel_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::reset() {
    has_ref_ = false;
    W_ = H_ = 0;
    impl_->grid_valid = false;
    impl_->ref_gray = false;
    impl_->ref_ghost = false;
    impl_->last_def = nullptr;
    last_global_ = dic::GlobalSimilarity();
}

int Engine::fast_pass_shape(int subset_size, bool six) const {
    const auto it = impl_->tune.find({subset_size, six ? 1 : 0});
    return it == impl_->tune.end() ? -1 : it->second.best;
}

int Engine::set_reference(const uint8_t* gray, int w, int h, const uint8_t* mask) {
    reset();
    if (!gray || w <= 0 || h <= 0) return -3;
    if ((int64_t)w * h > (int64_t)INT32_MAX) return -3;
    const size_t n = (size_t)w * h;
    const size_t np = (size_t)((w + 3) & ~3) * h;  // planes: rows padded to 16 bytes (TMA)
    Impl& I = *impl_;
    I.dGray.ensure(n);
    I.rI.ensure(np);
    I.rGx.ensure(np);
    I.rGy.ensure(np);
    check(cudaMemcpyAsync(I.dGray.p, gray, n, cudaMemcpyHostToDevice, stream_), "H2D reference");
    const uint8_t* dm = nullptr;
    if (mask) {
        I.dMask.ensure(n);
        check(cudaMemcpyAsync(I.dMask.p, mask, n, cudaMemcpyHostToDevice, stream_), "H2D mask");
        dm = I.dMask.p;
    }
    check(dic::launch_image_prep(I.dGray.p, dm, w, h, (w + 3) & ~3, I.rI.p, I.rGx.p, I.rGy.p, stream_),
          "reference prep");
    check(cudaStreamSynchronize(stream_), "reference sync");
    std::swap(I.rGray.p, I.dGray.p);  // the reference bytes stay for the global motion estimate
    std::swap(I.rGray.n, I.dGray.n);
    I.ref_gray = true;
    I.ref_ghost = mask != nullptr;
    W_ = w;
    H_ = h;
    has_ref_ = true;
    I.grid_valid = false;
    return 0;
}

int Engine::adopt_last_deformed(const uint8_t* mask, bool mask_on_device) {
    Impl& I = *impl_;
    if (!has_ref_ || !I.dI.p) return -3;
    std::swap(I.rI.p, I.dI.p);
    std::swap(I.rI.n, I.dI.n);
    std::swap(I.rGx.p, I.dGx.p);
    std::swap(I.rGx.n, I.dGx.n);
    std::swap(I.rGy.p, I.dGy.p);
    std::swap(I.rGy.n, I.dGy.n);
    // the adopted frame's bytes, when the last run's frame was the engine's own copy
    I.ref_gray = I.last_def != nullptr && I.last_def == I.dGray.p;
    if (I.ref_gray) {
        std::swap(I.rGray.p, I.dGray.p);
        std::swap(I.rGray.n, I.dGray.n);
    }
    I.last_def = nullptr;
    I.ref_ghost = mask != nullptr;
    if (mask) {
        // Ghost Wall on the adopted frame: the gradients stay those of the
        // real intensities (stamp after prepare, reference_cache.cpp:95-96).
        const size_t n = (size_t)W_ * H_;
        if (!(mask_on_device && I.mOut.p && I.mOut.n >= n)) {
            I.mOut.ensure(std::max(I.mOut.n, n));
            check(cudaMemcpyAsync(I.mOut.p, mask, n, cudaMemcpyHostToDevice, stream_), "H2D mask");
        }
        I.launched(1, dic::launch_stamp_ghost(I.rI.p, W_, H_, (W_ + 3) & ~3, I.mOut.p, stream_), "ghost stamp");
        check(cudaStreamSynchronize(stream_), "sync");
    }
    I.grid_valid = false;
    return 0;
}

int Engine::run(const uint8_t* def_gray, const uint8_t* mask, Params p, float* out, int capacity, float* metrics,
                int metrics_len, const double* model_H, Progress progress, Capture* capture) {
    if (!out || !has_ref_ || !def_gray) return -3;
    Impl& I = *impl_;
    const size_t n = (size_t)W_ * H_;
    I.dGray.ensure(n);
    check(cudaMemcpyAsync(I.dGray.p, def_gray, n, cudaMemcpyHostToDevice, stream_), "H2D deformed");
    const int cap = std::max(capacity, 0);
    I.d_out.ensure((size_t)std::max(cap, 8));
    const int rc = I.run(I.dGray.p, mask, p, I.d_out.p, cap, metrics, metrics_len, model_H, progress, capture);
    if (rc > 0) {
        check(cudaMemcpyAsync(out, I.d_out.p, (size_t)rc * 8 * sizeof(float), cudaMemcpyDeviceToHost, stream_),
              "D2H output");
        check(cudaStreamSynchronize(stream_), "output sync");
    }
    return rc;
}

int check_params(Params& p, int width, int height) { return validate_params(p, width, height); }

int Engine::warp_mask(const uint8_t* mask0, int W, int H, int gridW, int gridH, int rect_x, int rect_y, int step,
                      const float* U, const float* V, int X0, int X1, int Y0, int Y1, int per_px, uint8_t* out,
                      int box[4], bool mask0_resident) {
    Impl& I = *impl_;
    if (!mask0 || !U || !V || !out || W <= 0 || H <= 0 || gridW <= 0 || gridH <= 0 || step <= 0) return -3;
    cudaStream_t st = stream_;
    const size_t n = (size_t)W * H, ng = (size_t)gridW * gridH;
    // the material mask of frame 0 stays on the device between calls
    mask0_resident = mask0_resident && I.mMask0.p && I.mMask0_px == n;
    I.mMask0.ensure(std::max(I.mMask0.n, n));
    I.mOut.ensure(std::max(I.mOut.n, n));
    I.mTmp.ensure(std::max(I.mTmp.n, n));
    I.mU.ensure(std::max(I.mU.n, ng));
    I.mV.ensure(std::max(I.mV.n, ng));
    I.mBox.ensure(4);
    if (!mask0_resident) {
        check(cudaMemcpyAsync(I.mMask0.p, mask0, n, cudaMemcpyHostToDevice, st), "H2D material mask");
        I.mMask0_px = n;
    }
    check(cudaMemcpyAsync(I.mU.p, U, ng * 4, cudaMemcpyDefault, st), "copy U");
    check(cudaMemcpyAsync(I.mV.p, V, ng * 4, cudaMemcpyDefault, st), "copy V");
    const dic::MaskField f{gridW, gridH, rect_x, rect_y, step, I.mU.p, I.mV.p};
    I.launched(1, dic::launch_warp_mask(I.mMask0.p, W, H, X0, X1, Y0, Y1, per_px, f, I.mOut.p, st), "mask warp");
    I.launched(2, dic::launch_close3x3(I.mOut.p, I.mTmp.p, W, H, st), "mask close");
    I.launched(2, dic::launch_mask_bbox(I.mOut.p, W, H, I.mBox.p, st), "mask box");
    int b[4] = {0, 0, 0, 0};
    check(cudaMemcpyAsync(out, I.mOut.p, n, cudaMemcpyDeviceToHost, st), "D2H mask");
    check(cudaMemcpyAsync(b, I.mBox.p, sizeof(b), cudaMemcpyDeviceToHost, st), "D2H box");
    check(cudaStreamSynchronize(st), "sync");
    if (b[2] < 0) {
        box[0] = box[1] = box[2] = box[3] = 0;
    } else {
        box[0] = b[0];
        box[1] = b[1];
        box[2] = b[2] - b[0] + 1;
        box[3] = b[3] - b[1] + 1;
    }
    return 0;
}
int vsg_window_nodes(int step, int window) { return vsg_window_node_count(step, window); }

DeviceField Engine::last_field() const { return impl_->last_field; }

int Engine::pack_field(int gW, int gH, int rect_x, int rect_y, int step, int window, const float* u, const float* v,
                       const float* corr, const uint8_t* solved, float* out, int capacity) {
    Impl& I = *impl_;
    if (gW <= 0 || gH <= 0 || step <= 0 || !u || !v || !corr || !solved || !out) return -3;
    const size_t NG = (size_t)gW * gH;
    for (DevBuf<float>* b : {&I.fu, &I.fv, &I.fux, &I.fuy, &I.fvx, &I.fvy, &I.fcorr}) b->ensure(std::max(b->n, NG));
    I.fsolved.ensure(std::max(I.fsolved.n, NG));
    I.fiters.ensure(std::max(I.fiters.n, NG));
    // host or device inputs (unified addressing tells them apart)
    check(cudaMemcpyAsync(I.fu.p, u, NG * 4, cudaMemcpyDefault, stream_), "copy u");
    check(cudaMemcpyAsync(I.fv.p, v, NG * 4, cudaMemcpyDefault, stream_), "copy v");
    check(cudaMemcpyAsync(I.fcorr.p, corr, NG * 4, cudaMemcpyDefault, stream_), "copy corr");
    check(cudaMemcpyAsync(I.fsolved.p, solved, NG, cudaMemcpyDefault, stream_), "copy solved");
    I.last_field = DeviceField{};
    const int cap = std::max(capacity, 0);
    I.d_out.ensure(std::max<size_t>(I.d_out.n, (size_t)std::max(cap, 8)));
    int dropped_outlier = 0, dropped_post = 0;
    const int n = I.strain_pack(gW, gH, rect_x, rect_y, step, window, I.d_out.p, cap, dropped_outlier, dropped_post);
    if (n > 0) {
        check(cudaMemcpyAsync(out, I.d_out.p, (size_t)n * 8 * sizeof(float), cudaMemcpyDeviceToHost, stream_),
              "D2H packed");
        check(cudaStreamSynchronize(stream_), "sync");
    }
    return n;
}

PatchSolve Engine::solve_patch(const uint8_t* patch, int size, int ax, int ay, float gu, float gv, int subset,
                               bool six) {
    Impl& I = *impl_;
    PatchSolve r;
    if (!has_ref_ || !I.dI.p || !patch || size < subset || subset < 3 || (subset & 1) == 0) return r;
    cudaStream_t st = stream_;
    const int pp = (size + 3) & ~3, c = size / 2;
    const size_t n = (size_t)size * size, planes = (size_t)pp * size;
    I.aGray.ensure(std::max(I.aGray.n, n));
    for (DevBuf<float>* b : {&I.aI, &I.aGx, &I.aGy}) b->ensure(std::max(b->n, planes));
    I.aSkip.ensure(1);
    I.aValid.ensure(1);
    I.aMs.ensure(2);
    I.aHs.ensure(21);
    I.aTask.ensure(1);
    I.aRes.ensure(1);
    I.aQ.ensure(16);
    check(cudaMemcpyAsync(I.aGray.p, patch, n, cudaMemcpyHostToDevice, st), "H2D patch");
    I.launched(1, dic::launch_image_prep(I.aGray.p, nullptr, size, size, pp, I.aI.p, I.aGx.p, I.aGy.p, st),
               "patch prep");
    check(cudaMemsetAsync(I.aSkip.p, 0, 1, st), "memset");
    I.launched(2, dic::launch_pool(I.aI.p, I.aGx.p, I.aGy.p, size, size, pp, I.aSkip.p, 1, 1, c, c, 1, subset, 1,
                                   I.aValid.p, reinterpret_cast<float2*>(I.aMs.p), nullptr, I.aHs.p, st),
               "patch pool");
    dic_task t{};
    t.node = 0;
    t.cx = ax;
    t.cy = ay;
    t.mode = DIC_INIT_NO_SEARCH;
    t.g[0] = gu;
    t.g[1] = gv;
    check(cudaMemcpyAsync(I.aTask.p, &t, sizeof(t), cudaMemcpyHostToDevice, st), "H2D patch task");
    dic::SolveArgs a = I.solve_args(subset, six ? 1 : 0);
    a.ref_no_ghost = 0;  // the patch planes, not the reference's
    a.refI = I.aI.p;
    a.refGx = I.aGx.p;
    a.refGy = I.aGy.p;
    a.ref_pitch = pp;
    a.ref_dx = c - ax;
    a.ref_dy = c - ay;
    a.pool_valid = I.aValid.p;
    a.pool_ms = reinterpret_cast<const float2*>(I.aMs.p);
    a.pool_Hs = I.aHs.p;
    a.tasks = I.aTask.p;
    a.n_tasks = 1;
    a.n_tasks_dev = nullptr;
    a.results = I.aRes.p;
    a.queue = I.aQ.p;
    a.deferred = I.aQ.p + 8;
    I.launched(2, dic::launch_solve(a, six ? 1 : 0, 1, st), "patch solve");
    dic_result res{};
    check(cudaMemcpyAsync(&res, I.aRes.p, sizeof(res), cudaMemcpyDeviceToHost, st), "D2H patch result");
    check(cudaStreamSynchronize(st), "sync");
    r.initialized = (res.flags & DIC_RES_INITIALIZED) != 0;
    r.status = res.status;
    r.score = res.score;
    r.u = res.u;
    r.v = res.v;
    r.ux = res.ux;
    r.uy = res.uy;
    r.vx = res.vx;
    r.vy = res.vy;
    return r;
}

int Engine::run_device(const uint8_t* d_def, const uint8_t* mask, Params p, float* d_out, int capacity,
                       float* metrics, int metrics_len, const double* model_H, Progress progress,
                       Capture* capture) {
    if (!d_out || !has_ref_ || !d_def) return -3;
    return impl_->run(d_def, mask, p, d_out, std::max(capacity, 0), metrics, metrics_len, model_H, progress,
                      capture);
}

int Engine::Impl::run(const uint8_t* d_def, const uint8_t* mask, Params params, float* d_out_p, int capacity,
                      float* metrics, int metrics_len, const double* model_H, Progress progress,
                      Capture* capture) {
    using clk = std::chrono::high_resolution_clock;
    auto ms_since = [](clk::time_point t) { return std::chrono::duration<double, std::milli>(clk::now() - t).count(); };
    const auto t_total = clk::now();
    cudaStream_t st = E.stream_;
    const int W = E.W_, H = E.H_;
    const int prc = validate_params(params, W, H);
    if (prc != 0) return prc;
    E.times_ = PhaseTimes{};
    E.last_global_ = dic::GlobalSimilarity();
    last_def = d_def;
    last_field = DeviceField{};
    try {
        poll_cancel();
        check(cudaEventRecord(ev[0], st), "event");
        check(cudaMemsetAsync(counters.p + 9, 0, sizeof(int), st), "memset");
        E.last_tma_timeout_ = 0;
        prepare_deformed(d_def);
        check(cudaEventRecord(ev[1], st), "event");

        const int gW = params.rect_w / params.step, gH = params.rect_h / params.step;
        if (vsg_window_node_count(params.step, params.strain_window) < 3) return -4;
        const size_t NG = (size_t)gW * gH;
        const int dim = params.subset_size;

        // ---------------------------------------------------------------- grid + pool
        const auto t_prepass = clk::now();
        // the cached grid and pool hold for this mask (compared in place: no copy on a hit)
        const size_t mask_n = mask ? (size_t)W * H : 0;
        // the mask compared last, and only when everything else matches (a
        // reference just adopted rebuilds the grid without comparing)
        const bool cached = grid_valid && key.rect_x == params.rect_x && key.rect_y == params.rect_y &&
                            key.rect_w == params.rect_w && key.rect_h == params.rect_h && key.step == params.step &&
                            key.subset_size == params.subset_size && gridW == gW && gridH == gH &&
                            mask_key.size() == mask_n &&
                            (mask_n == 0 || std::memcmp(mask_key.data(), mask, mask_n) == 0);
        if (!cached) {
            grid_valid = false;
            skip.ensure(NG);
            const uint8_t* dm = nullptr;
            if (mask) {
                dMask.ensure((size_t)W * H);
                check(cudaMemcpyAsync(dMask.p, mask, (size_t)W * H, cudaMemcpyHostToDevice, st), "H2D mask");
                dm = dMask.p;
            }
            check(cudaMemsetAsync(counters.p + 2, 0, sizeof(int), st), "memset");
            launched(1, dic::launch_grid_scan(dm, W, H, gW, gH, params.rect_x, params.rect_y, params.step, dim, skip.p,
                                        counters.p + 2, st),
                  "grid scan");
            int nv = 0;
            check(cudaMemcpyAsync(&nv, counters.p + 2, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H count");
            sync();
            if (nv == 0) return -2;
            pool_valid.ensure(NG);
            pool_ms.ensure(NG);
            pool_Hs.ensure(NG * 21);
            launched(2, dic::launch_pool(rI.p, rGx.p, rGy.p, W, H, pitch(), skip.p, gW, gH, params.rect_x, params.rect_y,
                                   params.step, dim, 1, pool_valid.p, pool_ms.p, nullptr, pool_Hs.p, st),
                  "pool");
            h_skip.resize(NG);
            check(cudaMemcpyAsync(h_skip.data(), skip.p, NG, cudaMemcpyDeviceToHost, st), "D2H skip");
            sync();
            poll_cancel();
            key = params;
            mask_key.assign(mask, mask + mask_n);
            gridW = gW;
            gridH = gH;
            total_valid = nv;
            grid_valid = true;
        }
        check(cudaEventRecord(ev[2], st), "event");
        const double ms_prepass = ms_since(t_prepass);
        Ticker ticker(progress);
        ticker.set(10);

        // field init: skipped nodes count as solved (never attempted)
        fu.ensure(NG); fv.ensure(NG); fux.ensure(NG); fuy.ensure(NG); fvx.ensure(NG); fvy.ensure(NG);
        fcorr.ensure(NG); fsolved.ensure(NG); ftag.ensure(NG); fiters.ensure(NG);
        gu.ensure(NG); gv.ensure(NG); gux.ensure(NG); guy.ensure(NG); gvx.ensure(NG); gvy.ensure(NG);
        gtmp.ensure(NG); in_mesh.ensure(NG);
        check(cudaMemcpyAsync(fsolved.p, skip.p, NG, cudaMemcpyDeviceToDevice, st), "init solved");
        check(cudaMemsetAsync(ftag.p, 0, NG, st), "init tag");
        launched(1, dic::launch_fill(fcorr.p, (int)NG, -1.0f, st), "init corr");
        std::vector<uint8_t> solved = h_skip;  // host mirror of the solved flags
        const int total = total_valid;

        // ---------------------------------------------------------------- global model
        const auto t_seed = clk::now();
        E.last_learned_ = LearnedSeed{};
        // the tiles follow this run's model only (solves outside a run, such
        // as an incremental session's anchor matches, take the unrotated box)
        tile_spread = 0.f;
        struct SpreadReset {
            float& v;
            ~SpreadReset() { v = 0.f; }
        } spread_reset{tile_spread};
        double learned_H[9];
        // the caller's model, if any, rules out both front ends
        const bool caller_model = model_H != nullptr;
        bool learned = !caller_model && ref_gray && E.learned_ && !E.learned_rescue_ && E.proposal_ &&
                       learned_model(params, d_def, learned_H);
        if (learned) model_H = learned_H;
        auto plain_estimate = [&]() {
            if (!model_H && E.global_motion_ && ref_gray) {
                dic::GlobalSimilarity& g = E.last_global_;
                check(gm.estimate(rGray.p, d_def, W, H, params.rect_x, params.rect_y, params.rect_w, params.rect_h,
                                  st, g),
                      "global motion");
                E.times_.launches += g.kernels;
                if (g.locked) model_H = g.H;
            }
        };
        plain_estimate();

        // ---------------------------------------------------------------- anchor lattice
        HostStats st_anchor, st_a, st_b;
        float globalU = 0, globalV = 0;
        bool have_model = false, model_full = false, model_rejected = false;
        double t_u = 0, t_v = 0;
        Quality quality = Quality::NONE;
        float coverage = 0.f;
        int accepted = 0, attempted = 0, anchors_solved = 0;
        std::vector<Anchor> anchors;
        std::vector<semper_geom::Pt> ref_pts, def_pts;
        auto model_at = [&](double x, double y, float g6[6]) {
            double X, Y, J[4];
            if (!semper_geom::homography_at(model_H, x, y, X, Y, J)) return false;
            g6[0] = (float)(X - x); g6[1] = (float)(Y - y);
            g6[2] = (float)(J[0] - 1.0); g6[3] = (float)J[1];
            g6[4] = (float)J[2]; g6[5] = (float)(J[3] - 1.0);
            return true;
        };
        bool locked = false;
        std::vector<double> homography;
        // The model's guesses and its reach over the ROI (full_field_anchors.cpp:204-279).
        auto setup_model = [&]() {
        have_model = model_H != nullptr;
        model_full = model_rejected = false;
        t_u = t_v = 0;
        if (have_model) {
            const double gcx = params.rect_x + 0.5 * params.rect_w, gcy = params.rect_y + 0.5 * params.rect_h;
            float g6[6];
            if (!model_at(gcx, gcy, g6)) {
                have_model = false;
            } else {
                t_u = g6[0];
                t_v = g6[1];
                const double xs[2] = {(double)params.rect_x, (double)(params.rect_x + params.rect_w)};
                const double ys[2] = {(double)params.rect_y, (double)(params.rect_y + params.rect_h)};
                for (double x : xs)
                    for (double y : ys)
                        if (!model_at(x, y, g6) || std::hypot(g6[0] - t_u, g6[1] - t_v) > kSimilarityMinCornerPx)
                            model_full = true;
            }
        }
        locked = have_model;
        homography.clear();
        if (have_model) homography.assign(model_H, model_H + 9);
        set_tile_spread(have_model ? model_H : nullptr, params);
        };
        setup_model();

        int sx, sy;
        plan_lattice(gW, gH, sx, sy);
        std::vector<int> lat_x, lat_y;
        for (int gx = 0; gx < gW; gx += sx) lat_x.push_back(gx);
        if (lat_x.back() != gW - 1) lat_x.push_back(gW - 1);
        for (int gy = 0; gy < gH; gy += sy) lat_y.push_back(gy);
        if (lat_y.back() != gH - 1) lat_y.push_back(gH - 1);
        const int LW = (int)lat_x.size(), LH = (int)lat_y.size();
        // learned seeding: the network's guess per anchor under its model
        std::vector<float> anchor_uv;
        bool guided = false;
        auto learned_guesses = [&]() {
            const auto t_g = clk::now();
            anchor_uv = learned_anchor_guesses(d_def, model_H, params, lat_x, lat_y, solved, gW);
            // the model refitted to where the anchors land under the guesses,
            // so that what the keep rule measures against it is the field's own
            // departure from a homography, not the coarse estimate's error
            std::vector<semper_geom::Pt> rp, dp;
            for (int i = 0; i < LW * LH; ++i) {
                if (!std::isfinite(anchor_uv[2 * (size_t)i]) || !std::isfinite(anchor_uv[2 * (size_t)i + 1])) continue;
                const double x = params.rect_x + lat_x[i % LW] * params.step;
                const double y = params.rect_y + lat_y[i / LW] * params.step;
                rp.push_back({x, y});
                dp.push_back({x + anchor_uv[2 * (size_t)i], y + anchor_uv[2 * (size_t)i + 1]});
            }
            double Hr[9];
            if (rp.size() >= 8 && semper_geom::fit_homography(rp, dp, 6.0, Hr)) {
                std::copy(Hr, Hr + 9, learned_H);
                std::copy(Hr, Hr + 9, E.last_learned_.H);
                setup_model();
            }
            E.last_learned_.ms += (float)ms_since(t_g);
            E.last_learned_.anchor_uv = anchor_uv;
            guided = true;
        };
        if (learned) learned_guesses();

        auto solve_lattice = [&](bool sim) -> float {
            quality = Quality::NONE;
            coverage = 0.f;
            accepted = attempted = anchors_solved = 0;
            globalU = (float)t_u;
            globalV = (float)t_v;
            ref_pts.clear();
            def_pts.clear();
            anchors.assign((size_t)LW * LH, Anchor{});
            const int mode = have_model ? DIC_INIT_NO_SIMPLEX : DIC_INIT_AUTO_SEARCH;
            std::vector<dic_task> tk;
            std::vector<int> slot;
            for (int i = 0; i < LW * LH; ++i) {
                const int gx = lat_x[i % LW], gy = lat_y[i / LW];
                if (solved[(size_t)gy * gW + gx]) continue;
                ++attempted;
                dic_task t;
                t.node = gy * gW + gx;
                t.cx = params.rect_x + gx * params.step;
                t.cy = params.rect_y + gy * params.step;
                t.mode = mode;
                float gs[6] = {globalU, globalV, 0, 0, 0, 0};
                if (sim && !model_at(t.cx, t.cy, gs)) {
                    gs[0] = globalU; gs[1] = globalV; gs[2] = gs[3] = gs[4] = gs[5] = 0;
                }
                // the learned seeding's own guess for this anchor under its model
                if (sim && guided && std::isfinite(anchor_uv[2 * (size_t)i]) &&
                    std::isfinite(anchor_uv[2 * (size_t)i + 1])) {
                    gs[0] = anchor_uv[2 * (size_t)i];
                    gs[1] = anchor_uv[2 * (size_t)i + 1];
                }
                for (int k = 0; k < 6; ++k) t.g[k] = gs[k];
                tk.push_back(t);
                slot.push_back(i);
            }
            const std::vector<dic_result> rs = solve_batch(tk, params);
            for (size_t k = 0; k < tk.size(); ++k) {
                const dic_result& r = rs[k];
                if (!(r.flags & DIC_RES_INITIALIZED)) continue;
                st_anchor.record(r);
                if (r.status != 0) continue;
                Anchor& a = anchors[slot[k]];
                a.gx = lat_x[slot[k] % LW];
                a.gy = lat_y[slot[k] / LW];
                a.rx = (float)(params.rect_x + a.gx * params.step);
                a.ry = (float)(params.rect_y + a.gy * params.step);
                a.u = r.u; a.v = r.v; a.ux = r.ux; a.uy = r.uy; a.vx = r.vx; a.vy = r.vy;
                a.corr = r.score;
                a.used_simplex = (r.flags & DIC_RES_RESCUE) != 0;
                a.vertex = r.score <= kAnchorAcceptScore;
                a.output = r.score <= kCorrAccept;
            }
            // mark_kept_anchors (full_field_anchors.cpp:122-168) on the residual from the model
            std::vector<float> ru(anchors.size(), 0.f), rv(anchors.size(), 0.f);
            for (size_t i = 0; i < anchors.size(); ++i) {
                const Anchor& a = anchors[i];
                if (!a.vertex) continue;
                float g[6] = {0, 0, 0, 0, 0, 0};
                if (sim && !model_at(a.rx, a.ry, g)) { g[0] = globalU; g[1] = globalV; }
                ru[i] = a.u - g[0];
                rv[i] = a.v - g[1];
            }
            for (int lj = 0; lj < LH; ++lj)
                for (int li = 0; li < LW; ++li) {
                    const size_t idx = (size_t)lj * LW + li;
                    anchors[idx].kept = false;
                    if (!anchors[idx].vertex) continue;
                    std::vector<float> nu, nv;
                    for (int dj = -1; dj <= 1; ++dj)
                        for (int di = -1; di <= 1; ++di) {
                            if (di == 0 && dj == 0) continue;
                            const int nj = lj + dj, ni = li + di;
                            if (ni < 0 || ni >= LW || nj < 0 || nj >= LH) continue;
                            const size_t k = (size_t)nj * LW + ni;
                            if (!anchors[k].vertex) continue;
                            nu.push_back(ru[k]);
                            nv.push_back(rv[k]);
                        }
                    if (nu.size() < 3) continue;
                    const float mu = median_of(nu), mv = median_of(nv);
                    if (std::fabs(ru[idx] - mu) > kAnchorMedianTol || std::fabs(rv[idx] - mv) > kAnchorMedianTol)
                        continue;
                    anchors[idx].kept = true;
                }
            std::vector<float> us, vs;
            for (const Anchor& a : anchors) {
                if (!a.kept) continue;
                ref_pts.push_back({(double)a.rx, (double)a.ry});
                def_pts.push_back({(double)(a.rx + a.u), (double)(a.ry + a.v)});
                us.push_back(a.u);
                vs.push_back(a.v);
                if (a.output) anchors_solved++;
            }
            accepted = (int)ref_pts.size();
            if (accepted >= 3) {
                globalU = median_of(us);
                globalV = median_of(vs);
                const float roi_area = (float)(params.rect_w * params.rect_h);
                coverage = roi_area > 0.f ? (float)semper_geom::hull_area(ref_pts) / roi_area : 0.f;
            }
            const float frac = attempted > 0 ? (float)accepted / (float)attempted : 0.f;
            if (accepted >= kAnchorFullMinVertices && frac >= kAnchorFullFraction && coverage >= kAnchorFullCoverage)
                quality = Quality::FULL;
            else if (accepted >= 3 && coverage >= kAnchorSparseCoverage)
                quality = Quality::SPARSE;
            else
                quality = Quality::NONE;
            return frac;
        };

        auto seed_lattice = [&]() {
        if (LW >= 2 && LH >= 2) {
            if (!model_full) {
                solve_lattice(false);
            } else {
                const float kept = solve_lattice(true);
                if (quality != Quality::FULL || kept < kSimilarityKeepFraction) {
                    solve_lattice(false);
                    model_rejected = true;
                }
            }
            bool refitted = false;
            if (accepted >= kAnchorRefitMinPoints) {
                double Hf[9];
                if (semper_geom::fit_homography(ref_pts, def_pts, kAnchorRefitRansacPx, Hf)) {
                    homography.assign(Hf, Hf + 9);
                    refitted = true;
                }
            }
            if (model_rejected && !refitted) homography.clear();
        } else {
            globalU = (float)t_u;
            globalV = (float)t_v;
        }
        };
        seed_lattice();
        // the lattice judges the proposal: its error against the anchors
        // solved under it, and whether the keep rule held
        auto judge_learned = [&]() {
            LearnedSeed& Ls = E.last_learned_;
            double se = 0.0;
            for (const Anchor& a : anchors) {
                if (!a.vertex) continue;
                float g6[6];
                if (!model_at(a.rx, a.ry, g6)) continue;
                const float e = std::hypot(a.u - g6[0], a.v - g6[1]);
                se += e;
                Ls.err_max = std::max(Ls.err_max, e);
                Ls.anchors++;
            }
            Ls.err_mean = Ls.anchors ? (float)(se / Ls.anchors) : 0.f;
            Ls.kept = have_model && !model_rejected;
            return Ls.kept;
        };
        // seed again from the global-motion estimate alone, the anchors'
        // statistics counted for that seeding only
        auto reseed_plain = [&]() {
            st_anchor = HostStats();
            model_H = nullptr;
            guided = false;
            plain_estimate();
            setup_model();
            seed_lattice();
        };
        if (learned) {
            if (!judge_learned()) reseed_plain();
        } else if (!caller_model && ref_gray && E.learned_rescue_ && E.proposal_ &&
                   (model_rejected || (!have_model && quality != Quality::FULL))) {
            // rescue order: the lattice rejected the estimate's model, or the
            // estimate did not lock and the plain lattice fell short of full
            // quality, so the proposal is tried, its seeding judged the same
            // way; a rejected proposal leaves the run as the estimate seeded it
            if (learned_model(params, d_def, learned_H)) {
                learned = true;
                st_anchor = HostStats();
                model_H = learned_H;
                setup_model();
                learned_guesses();
                seed_lattice();
                if (!judge_learned()) reseed_plain();
            }
        }
        // publish_anchor_results (full_field_anchors.cpp:576-607)
        {
            std::vector<dic::ScatterRec> recs;
            for (const Anchor& a : anchors) {
                if (!a.output || !a.kept) continue;
                dic::ScatterRec r;
                r.node = a.gy * gW + a.gx;
                r.solved = 1;
                r.write_values = 1;
                r.v[0] = a.u; r.v[1] = a.v; r.v[2] = a.ux; r.v[3] = a.uy; r.v[4] = a.vx; r.v[5] = a.vy;
                r.v[6] = a.corr;
                recs.push_back(r);
                solved[r.node] = 1;
                st_anchor.points++;
            }
            if (!recs.empty()) {
                scat.ensure(std::max(scat.n, recs.size()));
                check(cudaMemcpyAsync(scat.p, recs.data(), recs.size() * sizeof(dic::ScatterRec),
                                      cudaMemcpyHostToDevice, st),
                      "H2D anchors");
                launched(1, dic::launch_scatter((int)recs.size(), scat.p, field(), st), "scatter anchors");
                check(cudaMemsetAsync(ftag.p, 0, NG, st), "tag");
            }
        }
        check(cudaEventRecord(ev[3], st), "event");
        const double ms_seed = ms_since(t_seed);
        ticker.set(20);
        poll_cancel();

        const bool have_seed = anchors_solved > 0 || accepted >= 3;
        const bool exec_c = quality == Quality::NONE && !have_seed;

        // ---------------------------------------------------------------- mesh guesses
        const auto t_mesh = clk::now();
        launched(1, dic::launch_init_guess((int)NG, globalU, globalV, mesh(), st), "init guess");
        std::vector<dic::MeshTri> htris;
        {
            std::vector<semper_geom::Pt> ins;
            std::vector<int> ins_of;
            for (size_t i = 0; i < ref_pts.size(); ++i)
                if (ref_pts[i].x > 0 && ref_pts[i].x < W && ref_pts[i].y > 0 && ref_pts[i].y < H) {
                    ins.push_back(ref_pts[i]);
                    ins_of.push_back((int)i);
                }
            // the triangulation depends on the points alone: a frame whose
            // kept anchors sit where the last one's did (a fixed reference,
            // an incremental sequence's lattice) reuses it
            if (ins.size() != dl_pts.size() ||
                !std::equal(ins.begin(), ins.end(), dl_pts.begin(), [](const semper_geom::Pt& a, const semper_geom::Pt& b) {
                    return a.x == b.x && a.y == b.y;
                })) {
                dl_tris = semper_geom::delaunay(ins);
                dl_pts = ins;
            }
            for (const semper_geom::Tri& t : dl_tris) {
                dic::MeshTri mt;
                semper_geom::Pt src[3], dst[3];
                const int vi[3] = {t.a, t.b, t.c};
                for (int k = 0; k < 3; ++k) {
                    src[k] = ins[vi[k]];
                    dst[k] = def_pts[ins_of[vi[k]]];
                    mt.px[k] = src[k].x;
                    mt.py[k] = src[k].y;
                    mt.X[k] = std::llround(src[k].x);
                    mt.Y[k] = std::llround(src[k].y);
                }
                double M[6];
                if (!semper_geom::affine3(src, dst, M)) continue;
                const double detF = M[0] * M[4] - M[1] * M[3];
                if (!std::isfinite(detF) || std::fabs(detF) <= 1e-3) continue;
                mt.ux = M[0] - 1.0; mt.uy = M[1]; mt.vx = M[3]; mt.vy = M[4] - 1.0; mt.u = M[2]; mt.v = M[5];
                const float mnx = (float)std::min({src[0].x, src[1].x, src[2].x});
                const float mxx = (float)std::max({src[0].x, src[1].x, src[2].x});
                const float mny = (float)std::min({src[0].y, src[1].y, src[2].y});
                const float mxy = (float)std::max({src[0].y, src[1].y, src[2].y});
                mt.bx = mnx - 15.0f; mt.by = mny - 15.0f; mt.bw = (mxx - mnx) + 30.0f; mt.bh = (mxy - mny) + 30.0f;
                htris.push_back(mt);
            }
        }
        if (!htris.empty()) {
            tris.ensure(std::max(tris.n, htris.size()));
            check(cudaMemcpyAsync(tris.p, htris.data(), htris.size() * sizeof(dic::MeshTri), cudaMemcpyHostToDevice,
                                  st),
                  "H2D triangles");
        }
        // The assignment kernels skip solved nodes; the device's solved flags
        // hold skip + published anchors.
        dic::Homog hg;
        const bool use_h = homography.size() == 9;
        if (use_h)
            for (int k = 0; k < 9; ++k) hg.h[k] = homography[k];
        launched((htris.empty() ? 0 : (quality == Quality::FULL ? 2 : 1)) + (use_h ? 1 : 0), dic::launch_mesh_assign(gW, gH, params.rect_x, params.rect_y, params.step, tris.p, (int)htris.size(),
                                      quality == Quality::FULL ? 1 : 0, use_h ? &hg : nullptr, fsolved.p, ftag.p,
                                      mesh(), st),
              "mesh assign");
        launched(6, dic::launch_smooth(gW, gH, params.step, mesh(), gtmp.p, st), "smooth");
        check(cudaEventRecord(ev[4], st), "event");
        sync();
        const double ms_mesh = ms_since(t_mesh);

        // ---------------------------------------------------------------- Path C
        int pc_x = gW / 2, pc_y = gH / 2;
        if (exec_c) {
            std::vector<int> cand;
            if (!ref_pts.empty()) {
                const float gcx2 = params.rect_x + (gW / 2.f) * params.step, gcy2 = params.rect_y + (gH / 2.f) * params.step;
                float md = 1e9f;
                int bi = -1;
                for (size_t i = 0; i < ref_pts.size(); ++i) {
                    const float dx = (float)ref_pts[i].x - gcx2, dy = (float)ref_pts[i].y - gcy2;
                    const float d = dx * dx + dy * dy;
                    if (d < md) { md = d; bi = (int)i; }
                }
                if (bi >= 0) {
                    const int gx = std::max(0, std::min(gW - 1, (int)std::round(((float)ref_pts[bi].x - params.rect_x) / params.step)));
                    const int gy = std::max(0, std::min(gH - 1, (int)std::round(((float)ref_pts[bi].y - params.rect_y) / params.step)));
                    if (!solved[(size_t)gy * gW + gx]) cand.push_back(gy * gW + gx);
                }
            }
            {
                const float cxg = gW / 2.0f, cyg = gH / 2.0f;
                std::vector<std::pair<float, int>> fr;
                for (int y = 0; y < gH; ++y)
                    for (int x = 0; x < gW; ++x) {
                        if (solved[(size_t)y * gW + x]) continue;
                        const float dx = x - cxg, dy = y - cyg;
                        fr.emplace_back(dx * dx + dy * dy, y * gW + x);
                    }
                std::stable_sort(fr.begin(), fr.end(), [](const std::pair<float, int>& a, const std::pair<float, int>& b) {
                    return a.first < b.first;
                });
                for (const auto& f : fr) {
                    if ((int)cand.size() >= kPathCMaxCandidates) break;
                    if (!cand.empty() && cand.front() == f.second) continue;
                    cand.push_back(f.second);
                }
            }
            if (cand.empty() && !locked) return -2;
            std::vector<dic_task> tk;
            for (int fi : cand) {
                dic_task t;
                t.node = fi;
                t.cx = params.rect_x + (fi % gW) * params.step;
                t.cy = params.rect_y + (fi / gW) * params.step;
                t.mode = DIC_INIT_AUTO_SEARCH;
                t.g[0] = globalU; t.g[1] = globalV; t.g[2] = t.g[3] = t.g[4] = t.g[5] = 0.f;
                tk.push_back(t);
            }
            const std::vector<dic_result> rs = solve_batch(tk, params);
            bool ok = false;
            for (size_t k = 0; k < tk.size(); ++k) {
                const dic_result& r = rs[k];
                if (!(r.flags & DIC_RES_INITIALIZED)) continue;
                if (r.status == 0 && r.score <= kCorrAccept) {
                    pc_x = tk[k].node % gW;
                    pc_y = tk[k].node / gW;
                    globalU = r.u;
                    globalV = r.v;
                    ok = true;
                    break;
                }
            }
            if (!ok && !cand.empty()) {
                pc_x = cand.front() % gW;
                pc_y = cand.front() / gW;
                if (!locked) return -5;
            }
        }
        poll_cancel();

        // ---------------------------------------------------------------- Path A
        const auto t_a = clk::now();
        int tune_variant = 0;
        tasks.ensure(std::max(tasks.n, NG));
        results.ensure(std::max(results.n, NG));
        deferred.ensure(std::max(deferred.n, NG));
        check(cudaMemsetAsync(counters.p, 0, 2 * sizeof(int), st), "counters");
        check(cudaMemsetAsync(pstats.p, 0, sizeof(dic::PathStats), st), "stats");
        launched(1, dic::launch_path_a_tasks(gW, gH, params.rect_x, params.rect_y, params.step, fsolved.p, ftag.p, mesh(),
                                       tasks.p, counters.p + 1, st),
              "path A tasks");
        int n_a = 0;
        check(cudaMemcpyAsync(&n_a, counters.p + 1, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H n_a");
        sync();
        if (n_a > 0) {
            dic::SolveArgs a = solve_args(dim, params.six);
            a.tasks = tasks.p;
            a.n_tasks_dev = counters.p + 1;
            a.n_tasks = n_a;
            tune_variant = tune_pick(dim, params.six ? 1 : 0);
            a.fast_stage = tune_variant;
            a.results = results.p;
            a.deferred = deferred.p;
            check(cudaEventRecord(ev[5], st), "event");
            launched(2, dic::launch_solve(a, params.six ? 1 : 0, solve_grid(n_a), st), "path A solve");
            check(cudaEventRecord(ev[6], st), "event");
            launched(1, dic::launch_commit(tasks.p, counters.p + 1, n_a, results.p, field(), pstats.p, st), "path A commit");
        }
        dic::PathStats ps{};
        check(cudaMemcpyAsync(&ps, pstats.p, sizeof(ps), cudaMemcpyDeviceToHost, st), "D2H stats");
        sync();
        poll_cancel();
        if (n_a > 0) {
            float ms = 0.f;
            check(cudaEventElapsedTime(&ms, ev[5], ev[6]), "elapsed");
            E.times_.path_a = ms;
            // launches small enough to go straight to the rescue pass run no fast pass
            if (n_a > 4 * sm_count && ps.icgn_iters > 0)
                tune_record(dim, params.six ? 1 : 0, tune_variant, ms / ((double)dim * dim * ps.icgn_iters));
        }
        E.times_.path_a_tasks = n_a;
        st_a.icgn_iters = (long long)ps.icgn_iters;
        st_a.points = ps.points;
        st_a.simp_calls = ps.simp_calls;
        st_a.simp_saved = ps.simp_saved;
        st_a.simp_dead = ps.simp_dead;
        E.times_.path_a_pixel_iters = (long long)dim * dim * st_a.icgn_iters;
        const double ms_a = ms_since(t_a);
        ticker.set(90);

        // ---------------------------------------------------------------- Path B
        const auto t_b = clk::now();
        {
            check(cudaMemcpyAsync(solved.data(), fsolved.p, NG, cudaMemcpyDeviceToHost, st), "D2H solved");
            bseeds.ensure(std::max<size_t>(bseeds.n, NG));
            check(cudaMemsetAsync(counters.p + 7, 0, sizeof(int), st), "memset");
            launched(1, dic::launch_boundary(gW, gH, field(), bseeds.p, counters.p + 7, st), "boundary");
            int nb = 0;
            check(cudaMemcpyAsync(&nb, counters.p + 7, sizeof(int), cudaMemcpyDeviceToHost, st), "D2H nb");
            sync();
            std::vector<dic::BoundarySeed> hb((size_t)nb);
            if (nb > 0) {
                check(cudaMemcpyAsync(hb.data(), bseeds.p, (size_t)nb * sizeof(dic::BoundarySeed),
                                      cudaMemcpyDeviceToHost, st),
                      "D2H boundary");
                sync();
            }
            struct Seed {
                int x, y;
                float u, v, ux, uy, vx, vy, c;
            };
            struct Order {
                bool operator()(const Seed& a, const Seed& b) const {
                    if (a.c != b.c) return a.c > b.c;
                    if (a.y != b.y) return a.y > b.y;
                    return a.x > b.x;
                }
            };
            std::priority_queue<Seed, std::vector<Seed>, Order> q;
            std::vector<uint8_t> claimed = solved;
            const int dx4[] = {1, -1, 0, 0}, dy4[] = {0, 0, 1, -1};
            std::vector<Seed> gseeds;
            const Seed pcs{pc_x, pc_y, globalU, globalV, 0, 0, 0, 0, 0};
            bool pcs_queued = false;
            for (const auto& b : hb)
                q.push({b.node % gW, b.node / gW, b.v[0], b.v[1], b.v[2], b.v[3], b.v[4], b.v[5], b.v[6]});
            if (hb.empty()) {
                struct Cand {
                    int ix, iy;
                    float u, v, dc, mag;
                };
                std::vector<Cand> cands;
                const float gcx2 = params.rect_x + (gW / 2.f) * params.step, gcy2 = params.rect_y + (gH / 2.f) * params.step;
                for (size_t fi = 0; fi < ref_pts.size(); ++fi) {
                    const float fx = (float)ref_pts[fi].x, fy = (float)ref_pts[fi].y;
                    const int ix = (int)std::round((fx - params.rect_x) / (float)params.step);
                    const int iy = (int)std::round((fy - params.rect_y) / (float)params.step);
                    if (ix < 0 || ix >= gW || iy < 0 || iy >= gH || solved[(size_t)iy * gW + ix]) continue;
                    const float du = (float)def_pts[fi].x - fx, dv = (float)def_pts[fi].y - fy;
                    const float wx = (float)(params.rect_x + ix * params.step), wy = (float)(params.rect_y + iy * params.step);
                    const float dc = std::sqrt((wx - gcx2) * (wx - gcx2) + (wy - gcy2) * (wy - gcy2));
                    cands.push_back({ix, iy, du, dv, dc, std::sqrt(du * du + dv * dv)});
                }
                if (cands.empty()) {
                    gseeds.push_back(pcs);
                    pcs_queued = true;
                } else {
                    std::sort(cands.begin(), cands.end(), [](const Cand& a, const Cand& b) {
                        const float ma = std::floor(a.mag), mb = std::floor(b.mag);
                        if (ma != mb) return ma < mb;
                        if (a.dc != b.dc) return a.dc < b.dc;
                        if (a.iy != b.iy) return a.iy < b.iy;
                        return a.ix < b.ix;
                    });
                    for (size_t k = 0; k < cands.size() && k < 5; ++k)
                        gseeds.push_back({cands[k].ix, cands[k].iy, cands[k].u, cands[k].v, 0, 0, 0, 0, 0});
                }
            }
            std::vector<dic::ScatterRec> recs;  // every claimed node's final state
            auto make_task = [&](int x, int y, const float g[6]) {
                dic_task t;
                t.node = y * gW + x;
                t.cx = params.rect_x + x * params.step;
                t.cy = params.rect_y + y * params.step;
                t.mode = DIC_INIT_NO_SEARCH;
                for (int k = 0; k < 6; ++k) t.g[k] = g[k];
                return t;
            };
            // A claimed cell stays marked solved whatever its solve gave; a
            // seed solved before the rounds is solved only if it passes
            // (full_field_path_b.cpp:120-145, 313-318).
            auto commit = [&](const dic_task& t, const dic_result& r, bool claimed_cell) {
                dic::ScatterRec rec;
                rec.node = t.node;
                rec.solved = claimed_cell ? 1 : 0;
                rec.write_values = 0;
                rec.v[6] = -1.0f;
                if (r.flags & DIC_RES_INITIALIZED) {
                    st_b.record(r);
                    if (r.status == 0 && r.score <= kCorrAccept) {
                        rec.write_values = 1;
                        rec.solved = 1;
                        rec.v[0] = r.u; rec.v[1] = r.v; rec.v[2] = r.ux; rec.v[3] = r.uy; rec.v[4] = r.vx;
                        rec.v[5] = r.vy; rec.v[6] = r.score;
                        st_b.points++;
                        q.push({t.node % gW, t.node / gW, r.u, r.v, r.ux, r.uy, r.vx, r.vy, r.score});
                    }
                }
                recs.push_back(rec);
            };
            for (const Seed& s : gseeds) {
                const size_t f = (size_t)s.y * gW + s.x;
                if (claimed[f]) continue;
                claimed[f] = 1;
                const float g[6] = {s.u, s.v, 0, 0, 0, 0};
                const std::vector<dic_task> tk{make_task(s.x, s.y, g)};
                const std::vector<dic_result> rs = solve_batch(tk, params);
                commit(tk[0], rs[0], false);
            }
            if (q.empty() && !gseeds.empty() && !pcs_queued) {
                const size_t f = (size_t)pcs.y * gW + pcs.x;
                if (pcs.x >= 0 && pcs.x < gW && pcs.y >= 0 && pcs.y < gH && !claimed[f]) {
                    claimed[f] = 1;
                    const float g[6] = {pcs.u, pcs.v, 0, 0, 0, 0};
                    const std::vector<dic_task> tk{make_task(pcs.x, pcs.y, g)};
                    const std::vector<dic_result> rs = solve_batch(tk, params);
                    commit(tk[0], rs[0], false);
                }
            }
            // Rounds: a claim sees the commits of every round but the one
            // still in flight (two rounds in flight, committed in order).
            std::deque<std::vector<dic_task>> rounds;
            auto claim = [&]() -> bool {
                if (q.empty()) return false;
                std::vector<dic_task> r;
                int popped = 0;
                while (!q.empty() && popped < kPathBBatchNodes) {
                    const Seed c = q.top();
                    q.pop();
                    ++popped;
                    for (int k = 0; k < 4; ++k) {
                        const int nx = c.x + dx4[k], ny = c.y + dy4[k];
                        if (nx < 0 || nx >= gW || ny < 0 || ny >= gH) continue;
                        const size_t f = (size_t)ny * gW + nx;
                        if (claimed[f]) continue;
                        claimed[f] = 1;
                        const float ddx = (float)((nx - c.x) * params.step), ddy = (float)((ny - c.y) * params.step);
                        const float g[6] = {c.u + c.ux * ddx + c.uy * ddy, c.v + c.vx * ddx + c.vy * ddy,
                                            c.ux, c.uy, c.vx, c.vy};
                        r.push_back(make_task(nx, ny, g));
                    }
                }
                rounds.push_back(std::move(r));
                return true;
            };
            // Round k runs on slot k % 2; its solves start as soon as it is
            // claimed, so two rounds run on the device at once. A slot's host
            // buffers are rewritten only once its previous work is done (an
            // earlier run that ended early may have left some queued).
            for (const Slot& S : slots)
                if (S.s) check(cudaStreamSynchronize(S.s), "slot drain");
            check(cudaEventRecord(ev[9], st), "event");
            int launched_rounds = 0, done_rounds = 0;
            auto claim_launch = [&]() -> bool {
                if (!claim()) return false;
                launch_round(launched_rounds % 2, rounds.back(), params, ev[9]);
                ++launched_rounds;
                return true;
            };
            while (rounds.size() < 2 && claim_launch()) {}
            while (!rounds.empty()) {
                const std::vector<dic_task> r = std::move(rounds.front());
                rounds.pop_front();
                const dic_result* rs = wait_round(done_rounds % 2);
                ++done_rounds;
                for (size_t k = 0; k < r.size(); ++k) commit(r[k], rs[k], true);
                while (rounds.size() < 2 && claim_launch()) {}
            }
            if (!recs.empty()) {
                scat.ensure(std::max(scat.n, recs.size()));
                check(cudaMemcpyAsync(scat.p, recs.data(), recs.size() * sizeof(dic::ScatterRec),
                                      cudaMemcpyHostToDevice, st),
                      "H2D path B");
                launched(1, dic::launch_scatter((int)recs.size(), scat.p, field(), st), "scatter path B");
            }
        }
        check(cudaEventRecord(ev[7], st), "event");
        const double ms_b = ms_since(t_b);
        E.times_.path_b = ms_b;
        poll_cancel();

        if (capture) {
            capture->gridW = gW; capture->gridH = gH;
            capture->rect_x = params.rect_x; capture->rect_y = params.rect_y;
            capture->step = params.step; capture->attempted = total;
            auto grab = [&](std::vector<float>& h, const DevBuf<float>& d) {
                h.resize(NG);
                check(cudaMemcpyAsync(h.data(), d.p, NG * 4, cudaMemcpyDeviceToHost, st), "D2H capture");
            };
            grab(capture->u, fu); grab(capture->v, fv); grab(capture->ux, fux); grab(capture->uy, fuy);
            grab(capture->vx, fvx); grab(capture->vy, fvy); grab(capture->corr, fcorr);
            capture->solved.resize(NG);
            check(cudaMemcpyAsync(capture->solved.data(), fsolved.p, NG, cudaMemcpyDeviceToHost, st), "D2H capture");
            sync();
        }

        // ---------------------------------------------------------------- pack + strain
        const auto t_strain = clk::now();
        int dropped_outlier = 0, dropped_post = 0;
        const int valid_count = strain_pack(gW, gH, params.rect_x, params.rect_y, params.step, params.strain_window,
                                            d_out_p, capacity, dropped_outlier, dropped_post);
        last_field = DeviceField{gW, gH, params.rect_x, params.rect_y, params.step, total, fu.p, fv.p, fux.p, fuy.p,
                                 fvx.p, fvy.p, fcorr.p, fsolved.p, valid.p};
        if (capture) {
            capture->median_valid.resize(NG);
            check(cudaMemcpyAsync(capture->median_valid.data(), valid.p, NG, cudaMemcpyDeviceToHost, st),
                  "D2H median flags");
            capture->median_rejected = dropped_outlier;
            sync();
        }
        const double ms_strain = ms_since(t_strain);
        ticker.stop();
        if (progress) {
            try {
                progress(100);
            } catch (...) {
            }
        }
        const double ms_total = ms_since(t_total);

        {
            float v = 0.f;
            cudaEventElapsedTime(&v, ev[0], ev[1]); E.times_.prep = v;
            cudaEventElapsedTime(&v, ev[1], ev[2]); E.times_.pool = v;
            cudaEventElapsedTime(&v, ev[2], ev[3]); E.times_.seed = v;
            cudaEventElapsedTime(&v, ev[3], ev[4]); E.times_.mesh = v;
            cudaEventElapsedTime(&v, ev[7], ev[8]); E.times_.strain = v;
            cudaEventElapsedTime(&v, ev[0], ev[8]); E.times_.total = v;
            E.times_.icgn_iters = st_a.icgn_iters + st_b.icgn_iters + st_anchor.icgn_iters;
            E.times_.pixel_iters = (long long)dim * dim * E.times_.icgn_iters;
        }

        const int ncopy = metrics_prefix_len(metrics_len);
        if (metrics && ncopy > 0) {
            const long long iters = st_a.icgn_iters + st_b.icgn_iters + st_anchor.icgn_iters;
            float m[kMetricsLen];
            m[0] = (float)total;
            m[1] = (float)valid_count;
            m[2] = (float)(total - valid_count);
            m[3] = (float)st_a.points;
            m[4] = (float)st_b.points;
            m[5] = (float)(st_a.simp_calls + st_b.simp_calls + st_anchor.simp_calls);
            m[6] = (float)(st_a.simp_saved + st_b.simp_saved + st_anchor.simp_saved);
            m[7] = (float)(st_a.simp_dead + st_b.simp_dead + st_anchor.simp_dead);
            m[8] = valid_count > 0 ? (float)iters / (float)valid_count : 0.f;
            m[9] = (float)ms_total;
            m[10] = (float)ms_seed;
            m[11] = (float)ms_prepass;
            m[12] = (float)ms_mesh;
            m[13] = (float)ms_strain;
            m[14] = ms_total > 0 ? (float)(valid_count / ms_total) : 0.f;
            m[15] = total > 0 ? ((float)valid_count / total) * 100.0f : 0.f;
            m[16] = quality == Quality::FULL ? 2.f : quality == Quality::SPARSE ? 1.f : 0.f;
            m[17] = 0.f;
            m[18] = (float)(ms_a + ms_b);
            m[19] = (float)st_anchor.points;
            m[20] = (float)dropped_post;
            m[21] = locked ? 1.f : 0.f;
            m[22] = coverage;
            m[23] = (float)dropped_outlier;
            for (int i = 0; i < ncopy; ++i) metrics[i] = m[i];
        }
        return valid_count;
    } catch (const Cancelled&) {
        // work still queued (Path B rounds on their slot streams included) ends
        // before the next run reuses the buffers it reads and writes
        cudaStreamSynchronize(st);
        for (const Slot& S : slots)
            if (S.s) cudaStreamSynchronize(S.s);
        return -99;
    }
}

}  // namespace semper_b200
