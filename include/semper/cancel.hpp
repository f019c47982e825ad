/*
 * semper/cancel.hpp — cancellation and result codes of the C++ API of this
 * B200 build. Same names, values and behaviour as the reference's
 * include/semper/cancel.hpp:1-140, so that C++ callers of
 * Semper::pipeline::run_full_field build against this library unchanged.
 */
#ifndef SEMPER_CANCEL_HPP
#define SEMPER_CANCEL_HPP

#include <atomic>

#ifndef SEMPER_CXX_API
#define SEMPER_CXX_API __attribute__((visibility("default")))
#endif

namespace Semper {
namespace pipeline {

constexpr int kCancelled = -99;       // the solve was cancelled (cancel.hpp:10)
constexpr int kBadStrainWindow = -4;  // strain_window too small for step (cancel.hpp:22)
constexpr int kSeedFailed = -5;       // nothing could seed the solve (cancel.hpp:31)

/* A cancel flag owned by one caller (cancel.hpp:33-80): request() from any
   thread stops the solve that polls it. A solve clears its token when it
   starts, unless the caller opened the window first (begin(), or a
   CancelScope), in which case requests made since then stop it. */
class CancelToken {
public:
    CancelToken() = default;
    CancelToken(const CancelToken&) = delete;
    CancelToken& operator=(const CancelToken&) = delete;

    void request() noexcept { requested_.store(true, std::memory_order_relaxed); }
    void clear() noexcept { requested_.store(false, std::memory_order_relaxed); }
    bool requested() const noexcept { return requested_.load(std::memory_order_relaxed); }

    /* Open the window: forget earlier requests, keep the ones from now on. */
    void begin() noexcept {
        clear();
        open_.store(true, std::memory_order_release);
    }
    /* Close a window no solve entered. */
    void end() noexcept { open_.store(false, std::memory_order_release); }
    /* Called by a solve as it starts. */
    void enter() noexcept {
        if (!open_.exchange(false, std::memory_order_acq_rel)) clear();
    }

private:
    std::atomic<bool> requested_{false};
    std::atomic<bool> open_{false};
};

/* begin() for the lifetime of one call, end() when it returns. */
class CancelScope {
public:
    explicit CancelScope(CancelToken& t) noexcept : t_(t) { t_.begin(); }
    ~CancelScope() { t_.end(); }
    CancelScope(const CancelScope&) = delete;
    CancelScope& operator=(const CancelScope&) = delete;

private:
    CancelToken& t_;
};

/* The process-wide token that the overloads without a token poll
   (cancel.hpp:112-140). */
SEMPER_CXX_API void request_cancel();
SEMPER_CXX_API void clear_cancel();
SEMPER_CXX_API bool cancel_requested();

namespace detail {
SEMPER_CXX_API CancelToken& global_cancel_token() noexcept;
}  // namespace detail

}  // namespace pipeline
}  // namespace Semper

#endif
