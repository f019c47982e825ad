// ORACLE — test infrastructure only. Never linked into the product library.
//
// Arithmetic primitives of the CPU restatement. The reference sums its subset
// reductions in SIMD lanes (include/semper/simd.hpp:30-150: per-lane partial
// sums over i = lane (mod lanes), then a horizontal reduce); the lane width is a
// property of the build target (4 on x86-64 SSE, 8 on AVX, 4 on NEON). This
// restatement fixes it at 32 lanes — one warp — and the horizontal reduce at an
// xor butterfly, so that a device kernel which accumulates pixel i in lane
// i % 32 and reduces with __shfl_xor_sync produces the same bits. Products and
// sums that the device fuses are fused here with std::fma; everything else is
// a separately rounded IEEE operation (built with -ffp-contract=off).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

namespace oracle {

constexpr int kLanes = 32;

#ifdef ORACLE_REFERENCE_FLAGS
// The timing build (the CPU baseline), compiled with the reference's own flags
// (CMakeLists.txt:80: -O3 -ffast-math -fno-finite-math-only -ffp-contract=off):
// every multiply-add is a separate multiply and add, as the reference computes
// it, not a library fma call on a target without the instruction. Its bits
// differ from the device contract; it is timed, never compared bit for bit.
inline float fmaT(float a, float b, float c) { return a * b + c; }
inline double fmaT(double a, double b, double c) { return a * b + c; }
#else
inline float fmaT(float a, float b, float c) { return std::fmaf(a, b, c); }
inline double fmaT(double a, double b, double c) { return std::fma(a, b, c); }
#endif

// Warp xor-butterfly: after the step with offset o, lane l holds
// v[l] + v[l ^ o]. IEEE addition is commutative, so every lane ends with the
// same bits; this returns that value.
template <class T>
inline T butterfly(const T in[kLanes]) {
    T v[kLanes];
    for (int l = 0; l < kLanes; ++l) v[l] = in[l];
    for (int o = kLanes / 2; o > 0; o >>= 1) {
        T t[kLanes];
        for (int l = 0; l < kLanes; ++l) t[l] = v[l] + v[l ^ o];
        for (int l = 0; l < kLanes; ++l) v[l] = t[l];
    }
    return v[0];
}

// True unless f is Inf or NaN, read from the bits (src/util/finite.hpp:18-28).
inline bool finite_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, sizeof u);
    return (u & 0x7f800000u) != 0x7f800000u;
}
inline bool finite_bits(double d) {
    uint64_t u;
    std::memcpy(&u, &d, sizeof u);
    return (u & 0x7ff0000000000000ull) != 0x7ff0000000000000ull;
}

}  // namespace oracle
