// Tensor-core (tcgen05) forward layer of the budget MLP:
//
//   out = act( norm(A) W^T + b ),   A [M x 256] FP32, W [256 x 256] FP32 masters,
//
// with both operands rounded to BF16 as they are staged into shared memory (the
// same rounding as the CUDA-core GEMM of mlp.cu) and the products accumulated in
// FP32 in tensor memory.  One CTA of 128 threads per 128-row tile:
//
//   1. warp 0 allocates 256 TMEM columns (a 128 x 256 FP32 accumulator);
//   2. all threads stage A's tile (128 x 256) and W (256 x 256) as BF16 in the
//      canonical K-major, no-swizzle layout: 8-row x 16-byte core matrices, the
//      16 core matrices of a 128-byte K slab adjacent (leading byte offset 128),
//      8-row groups 4096 bytes apart (stride byte offset);
//   3. one thread issues the 16 tcgen05.mma (M=128, N=256, K=16 each) and
//      commits them to an mbarrier; every thread waits on it (bounded);
//   4. warp w reads TMEM lanes 32w..32w+31 (its 32 rows) 16 columns at a time
//      with tcgen05.ld, adds the bias, applies GELU and writes the outputs;
//   5. warp 0 frees the TMEM columns.
//
// Shared memory 192 KB: one CTA per SM, so the allocation never waits on
// another CTA's columns.
#include <cuda_bf16.h>

#include <cstdint>

#include "index.hpp"
#include "mlp.hpp"

namespace hrnn {

namespace {

constexpr int kTM = 128, kTN = 256, kTK = 256;
constexpr uint32_t kSBO = (kTK / 8) * 128;  // bytes between 8-row core-matrix groups
constexpr uint32_t kLBO = 128;              // bytes between K-adjacent core matrices
constexpr size_t kSmemA = (size_t)kTM * kTK * 2, kSmemB = (size_t)kTN * kTK * 2;
constexpr size_t kSmemTC = kSmemA + kSmemB + 64;
constexpr uint32_t kWaitLimit = 1u << 26;   // mbarrier polls before giving up

// K-major, no-swizzle shared-memory matrix descriptor (tcgen05 "matrix
// descriptor": start address, leading / stride byte offsets >> 4, version 1).
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(kLBO >> 4) << 16) | ((uint64_t)(kSBO >> 4) << 32) |
           (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

// Byte offset of element (r, k) of a K-major tile in the core-matrix layout.
__device__ __forceinline__ uint32_t cm_off(uint32_t r, uint32_t k) {
    return (r >> 3) * kSBO + (k >> 3) * kLBO + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__device__ __forceinline__ float gelu_f(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678f)); }

// Stages rows [r0, r0 + R) x 256 of an FP32 matrix (row stride 256) as BF16; rows
// at or beyond `rows` are zero.  With `nrm`, x -> (x - mean) * inv first (the
// input normalisation, plain IEEE subtract and multiply).
__device__ __forceinline__ void stage(char* smem, const float* __restrict__ src, int r0, int R, int rows,
                                      const float* __restrict__ nrm) {
    // thread -> (row, 8-element chunk): 32 chunks per row
    for (int i = threadIdx.x; i < R * (kTK / 8); i += blockDim.x) {
        const int r = i >> 5, c = i & 31;
        const int gr = r0 + r;
        float v[8];
        if (gr < rows) {
            const float4* p = reinterpret_cast<const float4*>(src + (size_t)gr * kTK + c * 8);
            const float4 a = __ldg(p), b = __ldg(p + 1);
            v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
            if (nrm) {
#pragma unroll
                for (int j = 0; j < 8; ++j) v[j] = __fmul_rn(__fsub_rn(v[j], nrm[c * 8 + j]), nrm[kTK + c * 8 + j]);
            }
        } else {
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = 0.f;
        }
        uint4 w;
        w.x = pack_bf16(v[0], v[1]);
        w.y = pack_bf16(v[2], v[3]);
        w.z = pack_bf16(v[4], v[5]);
        w.w = pack_bf16(v[6], v[7]);
        *reinterpret_cast<uint4*>(smem + cm_off((uint32_t)r, (uint32_t)c * 8)) = w;
    }
}

__global__ void __launch_bounds__(128, 1) k_mlp_layer_tc(const float* __restrict__ A, int M,
                                                         const float* __restrict__ W,
                                                         const float* __restrict__ bias,
                                                         const float* __restrict__ nrm, float* __restrict__ z_out,
                                                         float* __restrict__ a_out, int act,
                                                         int* __restrict__ err) {
    extern __shared__ __align__(1024) char smem[];
    char* sA = smem;
    char* sB = smem + kSmemA;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kSmemA + kSmemB);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(smem + kSmemA + kSmemB + 16);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r0 = blockIdx.x * kTM;

    const uint32_t mbar_a = (uint32_t)__cvta_generic_to_shared(mbar);
    if (warp == 0) {
        const uint32_t slot_a = (uint32_t)__cvta_generic_to_shared(tslot);
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_a), "r"(kTN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar_a));
    stage(sA, A, r0, kTM, M, nrm);
    stage(sB, W, 0, kTN, kTN, nullptr);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic stores -> tensor-core reads
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        const uint32_t a0 = (uint32_t)__cvta_generic_to_shared(sA), b0 = (uint32_t)__cvta_generic_to_shared(sB);
#pragma unroll 1
        for (int s = 0; s < kTK / 16; ++s) {
            const uint64_t da = smem_desc(a0 + (uint32_t)s * 2 * kLBO), db = smem_desc(b0 + (uint32_t)s * 2 * kLBO);
            const uint32_t accum = s > 0 ? 1u : 0u;
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
                "l"(da), "l"(db), "r"(kIdesc), "r"(accum));
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar_a)
                     : "memory");
    }
    // bounded wait for the accumulator (phase 0 of the mbarrier)
    uint32_t done = 0;
    for (uint32_t it = 0; it < kWaitLimit && !done; ++it) {
        asm volatile(
            "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], 0;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
            : "=r"(done)
            : "r"(mbar_a)
            : "memory");
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!done) {
        if (lane == 0) atomicExch(err, 1);
    } else {
        const int row = r0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < kTN; c0 += 16) {
            uint32_t v[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < M) {
                float z[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) z[j] = __uint_as_float(v[j]) + bias[c0 + j];
                if (z_out) {
                    float4* o = reinterpret_cast<float4*>(z_out + (size_t)row * kTN + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) o[j] = make_float4(z[4 * j], z[4 * j + 1], z[4 * j + 2], z[4 * j + 3]);
                }
                if (a_out) {
                    float4* o = reinterpret_cast<float4*>(a_out + (size_t)row * kTN + c0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        float4 t = make_float4(z[4 * j], z[4 * j + 1], z[4 * j + 2], z[4 * j + 3]);
                        if (act) t = make_float4(gelu_f(t.x), gelu_f(t.y), gelu_f(t.z), gelu_f(t.w));
                        o[j] = t;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTN));
}

}  // namespace

void mlp_layer_tc_prepare() {
    CUDA_CHECK(cudaFuncSetAttribute(k_mlp_layer_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemTC));
}

// out_z / out_a (either may be null): [M x 256] FP32.  nrm: input normalisation
// (mean[256], inv[256]) or null.  err: device int set to 1 if a wait ran out.
void mlp_layer_tc(const float* A, int M, const float* W, const float* bias, const float* nrm, float* out_z,
                  float* out_a, bool gelu, int* err, cudaStream_t s) {
    if (M <= 0) return;
    // a stream being recorded into a graph gets the launch alone (mlp_layer_tc_prepare ran before the capture)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_CHECK(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone) mlp_layer_tc_prepare();
    k_mlp_layer_tc<<<(unsigned)((M + kTM - 1) / kTM), 128, kSmemTC, s>>>(A, M, W, bias, nrm, out_z, out_a,
                                                                          gelu ? 1 : 0, err);
    CUDA_LAUNCH_CHECK();
}

}  // namespace hrnn
