// Shared definitions of the hrnn_b200 library: status codes, errors, CUDA checks
// and the exact-order FP32 L2 kernels used by every phase.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

#include "../../include/hrnn_capi.h"

namespace hrnn {

// Error carried from any layer to the C ABI, where it becomes a status code and
// the thread-local message returned by hrnn_last_error().
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void fail(int code, const std::string& msg) { throw Error(code, msg); }

inline void cuda_check(cudaError_t e, const char* what, const char* file, int line) {
    if (e != cudaSuccess) {
        char buf[512];
        std::snprintf(buf, sizeof(buf), "%s: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
        fail(e == cudaErrorMemoryAllocation ? HRNN_ERR_NOMEM : HRNN_ERR_CUDA, buf);
    }
}
// Number of kernels this library has launched (every launch site ends with
// CUDA_LAUNCH_CHECK); per-call deltas are reported in the search statistics.
inline std::atomic<unsigned long long>& launch_counter() {
    static std::atomic<unsigned long long> c{0};
    return c;
}

#define CUDA_CHECK(x) ::hrnn::cuda_check((x), #x, __FILE__, __LINE__)
#define CUDA_LAUNCH_CHECK()                                                              \
    do {                                                                                 \
        ::hrnn::launch_counter().fetch_add(1, std::memory_order_relaxed);                \
        ::hrnn::cuda_check(cudaGetLastError(), "kernel launch", __FILE__, __LINE__);     \
    } while (0)

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kExpanded = 0x80000000u;   // flag bit in beam-list ids (ids < 2^31)
constexpr uint32_t kIdMask = 0x7FFFFFFFu;

// FP32 summation order of the reference's L2Space on the host it was built for
// (space_l2.h:214-238): element e accumulates into lane e % lanes; the lanes are
// then summed left to right.  fused bit 0: the SIMD multiply-add is one FMA;
// bit 1: the scalar tail loop (dims not a multiple of 16/4) is fused.
struct L2Order {
    int lanes = 16;
    int fused = 2;
};

__host__ __device__ inline uint32_t div_up(uint32_t a, uint32_t b) { return (a + b - 1) / b; }

// ----------------------------------------------------------------------------
// Exact-order L2 on the device
// ----------------------------------------------------------------------------

__device__ __forceinline__ float sq_step(float acc, float t, bool fused) {
    // Written with round-to-nearest intrinsics so the compiler never contracts
    // or reassociates: the rounding sequence is exactly the reference's.
    return fused ? __fmaf_rn(t, t, acc) : __fadd_rn(acc, __fmul_rn(t, t));
}

// One thread, any dim: restates the dispatch of space_l2.h:214-238.
__device__ inline float l2_thread(const float* __restrict__ a, const float* __restrict__ b,
                                  uint32_t d, int lanes, int fused) {
    auto simd = [&](uint32_t len, int L) {
        float acc[16];
#pragma unroll
        for (int l = 0; l < 16; ++l) acc[l] = 0.f;
        for (uint32_t e = 0; e < len; ++e) {
            int l = (int)(e % (uint32_t)L);
            acc[l] = sq_step(acc[l], a[e] - b[e], fused & 1);
        }
        float r = acc[0];
        for (int l = 1; l < L; ++l) r = __fadd_rn(r, acc[l]);
        return r;
    };
    auto scalar = [&](uint32_t off, uint32_t len) {
        float r = 0.f;
        for (uint32_t e = 0; e < len; ++e) r = sq_step(r, a[off + e] - b[off + e], (fused & 2) != 0);
        return r;
    };
    if (d % 16 == 0) return simd(d, lanes);
    if (d % 4 == 0) return simd(d, 4);
    if (d > 16) {
        uint32_t d16 = d & ~15u;
        return __fadd_rn(simd(d16, lanes), scalar(d16, d - d16));
    }
    if (d > 4) {
        uint32_t d4 = d & ~3u;
        return __fadd_rn(simd(d4, 4), scalar(d4, d - d4));
    }
    return scalar(0, d);
}

// Half-warp form for d % 16 == 0 and 16 lanes: lane l (0..15 of its half) owns
// accumulator l, i.e. elements l, l+16, l+32, ... -- the AVX-512 register lanes.
// q is read from shared memory, x from global memory (64 contiguous bytes per
// half-warp per step).  Returns the distance in every lane of the half.
template <bool FUSED>
__device__ __forceinline__ float l2_half16(const float* __restrict__ q_smem,
                                           const float* __restrict__ x, uint32_t nb, int l) {
    float acc = 0.f;
    uint32_t i = 0;
    for (; i + 4 <= nb; i += 4) {
        float x0 = __ldg(x + 16 * (i + 0) + l);
        float x1 = __ldg(x + 16 * (i + 1) + l);
        float x2 = __ldg(x + 16 * (i + 2) + l);
        float x3 = __ldg(x + 16 * (i + 3) + l);
        acc = sq_step(acc, q_smem[16 * (i + 0) + l] - x0, FUSED);
        acc = sq_step(acc, q_smem[16 * (i + 1) + l] - x1, FUSED);
        acc = sq_step(acc, q_smem[16 * (i + 2) + l] - x2, FUSED);
        acc = sq_step(acc, q_smem[16 * (i + 3) + l] - x3, FUSED);
    }
    for (; i < nb; ++i) acc = sq_step(acc, q_smem[16 * i + l] - __ldg(x + 16 * i + l), FUSED);
    // TmpRes[0] + TmpRes[1] + ... + TmpRes[15], left to right.
    float s = __shfl_sync(0xFFFFFFFFu, acc, 0, 16);
#pragma unroll
    for (int k = 1; k < 16; ++k) s = __fadd_rn(s, __shfl_sync(0xFFFFFFFFu, acc, k, 16));
    return s;
}

}  // namespace hrnn
