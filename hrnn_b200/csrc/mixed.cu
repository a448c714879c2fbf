// BF16 copies of the stored vectors for the mixed-precision search, with the
// per-vector rounding error e(x) = ||x - bf16(x)||_2 (computed in FP64, rounded
// up to FP32) that makes the verification screen's bound rigorous:
// | ||q - x|| - ||q - bf16(x)|| | <= e(x).  INT8 copies (per-vector scale) for the
// INT8 beam search.
#include <cuda_bf16.h>

#include <algorithm>

#include "index.hpp"

namespace hrnn {

namespace {

__global__ void k_to_bf16(const float* __restrict__ vec, size_t n, uint32_t dim, uint16_t* __restrict__ out,
                          float* __restrict__ err) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        double e2 = 0.0;
        for (uint32_t j = lane; j < dim; j += 32) {
            float x = vec[i * dim + j];
            __nv_bfloat16 b = __float2bfloat16_rn(x);
            out[i * dim + j] = __bfloat16_as_ushort(b);
            double dlt = (double)x - (double)__bfloat162float(b);
            e2 += dlt * dlt;
        }
        for (int o = 16; o; o >>= 1) e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
        if (lane == 0) err[i] = __double2float_ru(sqrt(e2) * (1.0 + 1e-12));
    }
}

// INT8 copies: per row s = max|x| / 127 (1 for a zero row), c = round(x / s) in
// [-127, 127], meta = (s, ||x - s c||_2 in FP64 rounded up, sum c^2, 0).
__global__ void k_to_i8(const float* __restrict__ vec, size_t n, uint32_t dim, int8_t* __restrict__ out,
                        float4* __restrict__ meta) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        float mx = 0.f;
        for (uint32_t j = lane; j < dim; j += 32) mx = fmaxf(mx, fabsf(vec[i * dim + j]));
        for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
        const float sc = mx > 0.f ? mx / 127.f : 1.f;
        double e2 = 0.0;
        int c2 = 0;
        for (uint32_t j = lane; j < dim; j += 32) {
            const float x = vec[i * dim + j];
            const int c = max(-127, min(127, __float2int_rn(x / sc)));
            out[i * dim + j] = (int8_t)c;
            const double dlt = (double)x - (double)sc * (double)c;
            e2 += dlt * dlt;
            c2 += c * c;
        }
        for (int o = 16; o; o >>= 1) {
            e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
            c2 += __shfl_xor_sync(0xFFFFFFFFu, c2, o);
        }
        if (lane == 0) meta[i] = make_float4(sc, __double2float_ru(sqrt(e2) * (1.0 + 1e-12)), (float)c2, 0.f);
    }
}

}  // namespace

void ensure_i8(Index& ix) {
    if (ix.i8_valid) return;
    const size_t cap = std::max<size_t>(ix.max_elements, 1);
    if (ix.vec_i8.bytes < cap * ix.dim) ix.vec_i8.alloc(cap * ix.dim);
    if (ix.i8_meta.bytes < cap * 16) ix.i8_meta.alloc(cap * 16);
    if (ix.cur) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ix.device);
        k_to_i8<<<nsm * 16, 256, 0, ix.stream>>>(ix.vec.as<float>(), ix.cur, (uint32_t)ix.dim,
                                                 ix.vec_i8.as<int8_t>(), ix.i8_meta.as<float4>());
        CUDA_LAUNCH_CHECK();
        CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    }
    ix.i8_valid = true;
}

void ensure_bf16(Index& ix) {
    if (ix.bf16_valid) return;
    const size_t cap = std::max<size_t>(ix.max_elements, 1);
    if (ix.vec_bf16.bytes < cap * ix.dim * 2) ix.vec_bf16.alloc(cap * ix.dim * 2);
    if (ix.vec_norm.bytes < cap * 4) ix.vec_norm.alloc(cap * 4);
    if (ix.cur) {
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ix.device);
        k_to_bf16<<<nsm * 16, 256, 0, ix.stream>>>(ix.vec.as<float>(), ix.cur, (uint32_t)ix.dim,
                                                   ix.vec_bf16.as<uint16_t>(), ix.vec_norm.as<float>());
        CUDA_LAUNCH_CHECK();
        CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    }
    ix.bf16_valid = true;
}

}  // namespace hrnn
