// dic_cuda_solve_noalloc: the batched subset solve of dic_cuda_solve for
// callers that cannot allocate device memory.
//
// Some hosts own every device allocation themselves: a plugin running inside
// another application's memory pool, a process under a fixed device-memory
// budget, or code that must not call cudaMalloc in the middle of its work
// (cudaMalloc can synchronise the device and can fail late). Such a caller
// can pass the solve its inputs and outputs, but not a scratch buffer. This
// entry point keeps the solve's scratch (three work counters and the list of
// tasks the fast pass hands on) in a fixed array that is part of the
// library's device image, so a call allocates nothing.
//
// The cost is a fixed 4 MiB array on every GPU where the library's device code
// is loaded (under lazy module loading, from its first use there), held until
// the process exits, and a limit of DIC_CUDA_SOLVE_NOALLOC_MAX_TASKS tasks per
// call.
#include <cuda_runtime.h>

#include <mutex>

#include "../../../include/semper_dic_cuda.h"
#include "icgn.cuh"

namespace {

constexpr int kCounters = 8;  // the solve's work counters: 3 used, padded to 32 bytes
constexpr int kMaxTasks = DIC_CUDA_SOLVE_NOALLOC_MAX_TASKS;
constexpr int kMaxDevices = 64;

// The shared scratch: counters, then the deferred-task list. In host code
// this name is only a stand-in for the device symbol; the device address
// comes from cudaGetSymbolAddress below.
static __device__ __align__(256) int g_solve_scratch[kCounters + kMaxTasks];

std::mutex g_mu;
int* g_scratch[kMaxDevices] = {};

// The scratch's device address on the current device, looked up once per
// device (with that device current) and cached. A reset of the device's
// primary context reloads the module and moves the array, so the entry is not
// for use across cudaDeviceReset (the header says so).
cudaError_t scratch_on_current_device(int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_solve_scratch);
        if (e != cudaSuccess) return e;
        g_scratch[dev] = static_cast<int*>(p);
    }
    *out = g_scratch[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" __attribute__((visibility("default"))) int dic_cuda_solve_noalloc(
    const float* d_ref_I, const float* d_ref_gx, const float* d_ref_gy, const float* d_def_I, int width, int height,
    int pitch, const uint8_t* d_pool_valid, const float* d_pool_mean_std, const double* d_pool_Hs21, int subset, int lm,
    int six, const dic_task* d_tasks, int n_tasks, dic_result* d_results, int blocks, void* stream) {
    if (n_tasks <= 0) return 0;
    if (n_tasks > kMaxTasks) return (int)cudaErrorInvalidValue;  // too many tasks for the fixed scratch
    int* scratch = nullptr;
    const cudaError_t e = scratch_on_current_device(&scratch);
    if (e != cudaSuccess) return (int)e;
    dic::SolveArgs a{};
    a.refI = d_ref_I;
    a.refGx = d_ref_gx;
    a.refGy = d_ref_gy;
    a.defI = d_def_I;
    a.W = width;
    a.H = height;
    a.pitch = pitch;
    a.err = nullptr;
    a.pool_valid = d_pool_valid;
    a.pool_ms = reinterpret_cast<const float2*>(d_pool_mean_std);
    a.pool_Hs = d_pool_Hs21;
    a.dim = subset;
    a.max_n = subset * subset;
    a.lm = lm;
    a.tasks = d_tasks;
    a.n_tasks = n_tasks;
    a.results = d_results;
    // launch_solve zeroes the counters on `stream` before its launches; the
    // deferred list is written before it is read and needs no clearing
    a.queue = scratch;
    a.deferred = scratch + kCounters;
    if (blocks <= 0) {
        int dev = 0, sms = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int need = (n_tasks + dic::kSolveThreads / 32 - 1) / (dic::kSolveThreads / 32);
        blocks = need < sms * 4 ? need : sms * 4;
    }
    return (int)dic::launch_solve(a, six, blocks, static_cast<cudaStream_t>(stream));
}
