// Batched incremental sequences: several frame sequences, each tracked by its
// own incremental session (one engine, one stream, its own device state). A
// process call advances every listed sequence by one frame, each on
// its own host thread, so the sessions' kernels and copies interleave on the
// device while one session's host steps (anchor matches, update schedule,
// packing) overlap the others' solves. A sequence is solved exactly as a lone
// semper_incremental handle solves it: the sessions share nothing. The
// sessions may sit on several GPUs (semper_b200_inc_batch_create_on).
#include <atomic>
#include <cstdint>
#include <memory>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../../include/semper_b200_ext.h"

struct semper_b200_inc_batch {
    int device = 0;
    struct Seq {
        semper_incremental* h = nullptr;
        int device = 0;  // the session's device
        int width = 0, height = 0;
    };
    std::vector<Seq> seqs;
    std::atomic<bool> busy{false};
    ~semper_b200_inc_batch() {
        int cur = 0;
        const bool have = cudaGetDevice(&cur) == cudaSuccess;
        for (Seq& s : seqs)
            if (s.h) {
                cudaSetDevice(s.device);
                semper_incremental_destroy(s.h);
            }
        if (have) cudaSetDevice(cur);
    }
};

namespace {

struct BusyGuard {
    std::atomic<bool>& flag;
    bool owned;
    explicit BusyGuard(std::atomic<bool>& f) : flag(f), owned(!f.exchange(true, std::memory_order_acquire)) {}
    ~BusyGuard() {
        if (owned) flag.store(false, std::memory_order_release);
    }
};

}  // namespace

extern "C" {

SEMPER_C_API semper_b200_inc_batch* semper_b200_inc_batch_create_on(int32_t sequences, const int32_t* devices,
                                                                     int32_t n_devices) {
    if (sequences <= 0 || n_devices < 0 || (n_devices > 0 && devices == nullptr)) return nullptr;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return nullptr;
    semper_b200_inc_batch* out = nullptr;
    try {
        std::unique_ptr<semper_b200_inc_batch> b(new semper_b200_inc_batch());
        b->device = cur;
        b->seqs.resize((size_t)sequences);
        bool ok = true;
        for (size_t q = 0; q < b->seqs.size() && ok; ++q) {
            auto& s = b->seqs[q];
            s.device = n_devices > 0 ? devices[q % (size_t)n_devices] : cur;
            ok = cudaSetDevice(s.device) == cudaSuccess;
            if (ok) s.h = semper_incremental_create();  // its engine and stream on s.device
            ok = ok && s.h != nullptr;
        }
        if (ok) out = b.release();
    } catch (...) {
        out = nullptr;
    }
    cudaSetDevice(cur);
    return out;
}

SEMPER_C_API semper_b200_inc_batch* semper_b200_inc_batch_create(int32_t sequences) {
    return semper_b200_inc_batch_create_on(sequences, nullptr, 0);
}

SEMPER_C_API void semper_b200_inc_batch_destroy(semper_b200_inc_batch* b) { delete b; }

SEMPER_C_API int semper_b200_inc_batch_init(semper_b200_inc_batch* b, int32_t sequence, const uint8_t* reference,
                                            const uint8_t* mask, int32_t width, int32_t height,
                                            const semper_params* params, int32_t update_interval) {
    if (b == nullptr || sequence < 0 || sequence >= (int32_t)b->seqs.size()) return SEMPER_ERR_INIT;
    if (reference == nullptr || width <= 0 || height <= 0) return SEMPER_ERR_INIT;
    BusyGuard g(b->busy);
    if (!g.owned) return SEMPER_ERR_INIT;
    auto& s = b->seqs[(size_t)sequence];
    const size_t len = (size_t)width * (size_t)height;
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    cudaSetDevice(s.device);
    const int rc = semper_incremental_init(s.h, reference, len, mask, mask ? len : 0, width, height, params,
                                           update_interval);
    if (have) cudaSetDevice(cur);
    s.width = rc == 0 ? width : 0;
    s.height = rc == 0 ? height : 0;
    return rc;
}

SEMPER_C_API int semper_b200_inc_batch_process(semper_b200_inc_batch* b, semper_b200_inc_frame* frames, int32_t n) {
    if (b == nullptr || n < 0 || (frames == nullptr && n > 0)) return SEMPER_ERR_INIT;
    BusyGuard g(b->busy);
    if (!g.owned) return SEMPER_ERR_INIT;
    std::vector<char> named(b->seqs.size(), 0);
    for (int32_t i = 0; i < n; ++i) {
        const int32_t q = frames[i].sequence;
        if (q < 0 || q >= (int32_t)b->seqs.size() || named[(size_t)q]) return SEMPER_ERR_INIT;
        named[(size_t)q] = 1;
    }
    int cur = 0;
    const bool have = cudaGetDevice(&cur) == cudaSuccess;
    auto one = [b](semper_b200_inc_frame& f) {
        auto& s = b->seqs[(size_t)f.sequence];
        cudaSetDevice(s.device);
        f.info = semper_incremental_info{};
        if (s.width <= 0 || f.frame == nullptr) {
            f.result = SEMPER_ERR_INIT;
            return;
        }
        f.result = semper_incremental_process(s.h, f.frame, (size_t)s.width * (size_t)s.height, f.out,
                                              f.out_capacity, f.metrics, f.metrics_len, &f.info, nullptr, nullptr);
    };
    std::vector<std::thread> threads;
    try {
        for (int32_t i = 1; i < n; ++i) threads.emplace_back(one, std::ref(frames[i]));
    } catch (...) {
        // no thread to spare: the rest run on this one
        for (int32_t i = 1 + (int32_t)threads.size(); i < n; ++i) one(frames[i]);
    }
    if (n > 0) one(frames[0]);
    for (auto& t : threads) t.join();
    if (have) cudaSetDevice(cur);
    return 0;
}

}  // extern "C"
