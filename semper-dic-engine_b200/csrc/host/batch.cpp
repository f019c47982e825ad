// Batched full-field solves: many independent (reference, deformed) pairs
// with their own sizes, masks and settings, solved concurrently on one GPU.
//
// Each worker owns an Engine (its own stream, device buffers and staging) and
// a host thread; jobs are taken largest first from a shared counter. The
// engines may sit on several GPUs (semper_b200_batch_create_on): jobs then
// spread over the devices as the workers take them. The
// engines' persistent solve kernels, image passes and copies then overlap on
// the device, and one job's host-side steps (lattice routing, Delaunay,
// Path B claims) run while the others' kernels execute. Every job is solved
// exactly as a lone semper_set_reference + semper_run on a fresh handle would
// solve it (an engine's state is reset per job), so results do not depend on
// the batch, its order or the worker count.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <exception>
#include <memory>
#include <mutex>
#include <numeric>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../../include/semper_b200_ext.h"
#include "engine.hpp"

using semper_b200::Engine;
using semper_b200::Params;

struct semper_b200_batch {
    int device = 0;                 // the caller's device at creation
    std::vector<int> dev_of;        // each engine's device
    std::vector<std::unique_ptr<Engine>> engines;
    std::atomic<bool> busy{false};
    std::mutex err_mu;
    std::string last_error;  // the first failure of the last run, if any
};

namespace {

Params job_params(const semper_params& p) {
    Params q;
    q.rect_x = p.rect_x;
    q.rect_y = p.rect_y;
    q.rect_w = p.rect_w;
    q.rect_h = p.rect_h;
    q.step = p.step;
    q.subset_size = p.subset_size;
    q.strain_window = p.strain_window;
    q.six = p.use_6x6_interpolator != 0;
    return q;
}

// One job on one engine: semper_set_reference then semper_run, raw 8-bit
// frames (and mask) of width x height.
int run_job(Engine& e, semper_b200_job& j) {
    if (!j.reference || !j.deformed || !j.out || j.width <= 0 || j.height <= 0 || j.out_capacity < 0)
        return SEMPER_ERR_INIT;
    if ((int64_t)j.width * j.height > (int64_t)INT32_MAX) return SEMPER_ERR_INIT;
    e.reset();
    if (e.set_reference(j.reference, j.width, j.height, j.mask) != 0) return SEMPER_ERR_INIT;
    return e.run(j.deformed, j.mask, job_params(j.params), j.out, j.out_capacity, j.metrics, j.metrics_len);
}

}  // namespace

extern "C" {

SEMPER_C_API semper_b200_batch* semper_b200_batch_create_on(int32_t workers, const int32_t* devices,
                                                             int32_t n_devices) {
    if (n_devices < 0 || (n_devices > 0 && devices == nullptr)) return nullptr;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return nullptr;
    std::unique_ptr<semper_b200_batch> b(new semper_b200_batch());
    b->device = cur;
    try {
        if (workers <= 0) workers = 8;
        for (int i = 0; i < workers; ++i) {
            const int dev = n_devices > 0 ? devices[i % n_devices] : cur;
            if (cudaSetDevice(dev) != cudaSuccess) throw std::runtime_error("device");
            b->engines.emplace_back(new Engine());  // its stream and buffers on `dev`
            b->dev_of.push_back(dev);
        }
    } catch (...) {
        semper_b200_batch_destroy(b.release());
        cudaSetDevice(cur);
        return nullptr;
    }
    cudaSetDevice(cur);
    return b.release();
}

SEMPER_C_API semper_b200_batch* semper_b200_batch_create(int32_t workers) {
    return semper_b200_batch_create_on(workers, nullptr, 0);
}

SEMPER_C_API void semper_b200_batch_destroy(semper_b200_batch* b) {
    if (b == nullptr) return;
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    for (size_t i = 0; i < b->engines.size(); ++i) {
        if (i < b->dev_of.size()) cudaSetDevice(b->dev_of[i]);
        b->engines[i].reset();  // freed with its own device current
    }
    if (have) cudaSetDevice(cur);
    delete b;
}

SEMPER_C_API int semper_b200_batch_run(semper_b200_batch* b, semper_b200_job* jobs, int32_t n_jobs) {
    if (b == nullptr || (jobs == nullptr && n_jobs > 0) || n_jobs < 0) return SEMPER_ERR_INIT;
    if (b->busy.exchange(true, std::memory_order_acquire)) return SEMPER_ERR_INIT;
    // largest first, so the last jobs to start are the short ones
    std::vector<int> order((size_t)n_jobs);
    std::iota(order.begin(), order.end(), 0);
    auto area = [&](int i) {
        const semper_params& p = jobs[i].params;
        return (int64_t)p.rect_w * p.rect_h / std::max(1, p.step * p.step);
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return area(x) > area(y); });
    {
        std::lock_guard<std::mutex> g(b->err_mu);
        b->last_error.clear();
    }
    std::atomic<int> next{0};
    auto work = [&](size_t w) {
        Engine& e = *b->engines[w];
        cudaSetDevice(b->dev_of[w]);
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= n_jobs) break;
            semper_b200_job& j = jobs[order[(size_t)k]];
            std::string why;
            try {
                j.result = run_job(e, j);
            } catch (const std::exception& ex) {
                j.result = SEMPER_ERR_INIT;
                why = ex.what();
            } catch (...) {
                j.result = SEMPER_ERR_INIT;
                why = "unknown exception";
            }
            if (!why.empty()) {
                std::lock_guard<std::mutex> g(b->err_mu);
                if (b->last_error.empty()) b->last_error = "job " + std::to_string(order[(size_t)k]) + ": " + why;
            }
        }
    };
    const size_t nw = std::min(b->engines.size(), (size_t)std::max(n_jobs, 1));
    std::vector<std::thread> threads;
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    for (size_t w = 1; w < nw; ++w) threads.emplace_back(work, w);
    work(0);
    for (auto& t : threads) t.join();
    if (have) cudaSetDevice(cur);
    b->busy.store(false, std::memory_order_release);
    return 0;
}

SEMPER_C_API const char* semper_b200_batch_last_error(semper_b200_batch* b) {
    if (b == nullptr) return "";
    std::lock_guard<std::mutex> g(b->err_mu);
    return b->last_error.c_str();
}

}  // extern "C"
