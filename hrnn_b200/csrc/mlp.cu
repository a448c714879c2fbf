// Learned search budget: a 256 -> 256 -> 256 -> 2 MLP (GELU) with BF16 weights,
// trained and run on the device with the kernels below.
//
//   GEMMs: Y = X W^T + b (forward), dX = dY W, dW = dY^T X (backward); both
//   operands are rounded to BF16 (round to nearest) as they are staged, products
//   are accumulated in FP32.  The two 256 x 256 forward layers run on the tensor
//   cores (tcgen05, mlp_tc.cu, GELU in the epilogue); the 2-output layer and the
//   backward GEMMs on the CUDA cores (k_gemm, shared-memory tiles).  Master
//   weights and Adam state are FP32.  Loss: binary cross-entropy with logits on
//   both outputs.
//
// The two outputs are the logits of "the query's answer is complete with budget
// level 0" and "... with level 1" (the levels are set by hrnn_set_budget); the
// search takes the cheapest level whose probability reaches the confidence
// cutoff and falls back to the caller's (m, ef) otherwise.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "index.hpp"
#include "mlp.hpp"

namespace hrnn {

namespace {

constexpr int TB = 32;  // GEMM tile

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// C[M x N] = alpha * sum_k A(m, k) B(k, n) (+ bias[n]) (+ beta * C), with
// A(m, k) = TA ? A[k * lda + m] : A[m * lda + k] and B(k, n) = TB_ ? B[n * ldb + k] : B[k * ldb + n].
template <bool TA, bool TBT>
__global__ void k_gemm(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ Cm,
                       const float* __restrict__ bias, int M, int N, int K, int lda, int ldb, float beta) {
    __shared__ float As[TB][TB + 1];
    __shared__ float Bs[TB][TB + 1];
    const int tx = threadIdx.x % TB, ty = threadIdx.x / TB;  // 32 x 8 threads, 4 rows each
    const int m0 = blockIdx.y * TB, n0 = blockIdx.x * TB;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = 0; k0 < K; k0 += TB) {
        for (int r = ty; r < TB; r += 8) {
            const int m = m0 + r, k = k0 + tx;
            float a = 0.f;
            if (m < M && k < K) a = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
            As[r][tx] = bf16r(a);
            const int kk = k0 + r, n = n0 + tx;
            float b = 0.f;
            if (kk < K && n < N) b = TBT ? B[(size_t)n * ldb + kk] : B[(size_t)kk * ldb + n];
            Bs[r][tx] = bf16r(b);
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < TB; ++k) {
            const float b = Bs[k][tx];
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = fmaf(As[ty + 8 * i][k], b, acc[i]);
        }
        __syncthreads();
    }
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + ty + 8 * i, n = n0 + tx;
        if (m < M && n < N) {
            float v = acc[i] + (bias ? bias[n] : 0.f);
            if (beta != 0.f) v += beta * Cm[(size_t)m * N + n];
            Cm[(size_t)m * N + n] = v;
        }
    }
}

__device__ __forceinline__ float gelu_d(float x) {
    return 0.5f * (1.f + erff(x * 0.70710678f)) + x * 0.39894228f * expf(-0.5f * x * x);
}

// xn = (x - mean) * inv, per input feature (plain IEEE FP32 subtract and multiply).
__global__ void k_normalize(const float* __restrict__ x, const float* __restrict__ nrm, float* __restrict__ xn,
                            size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int f = (int)(i % kMlpIn);
        xn[i] = __fmul_rn(__fsub_rn(x[i], nrm[f]), nrm[kMlpIn + f]);
    }
}

__global__ void k_gelu_back(const float* __restrict__ z, float* __restrict__ g, size_t n) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g[i] *= gelu_d(z[i]);
}

// dZ3 = (sigmoid(z) - y) / B for both outputs; loss accumulated in *loss.
__global__ void k_bce(const float* __restrict__ z, const uint8_t* __restrict__ y, float* __restrict__ dz, int B,
                      float* __restrict__ loss) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * 2) return;
    const float t = y[i] ? 1.f : 0.f, x = z[i];
    const float s = 1.f / (1.f + expf(-x));
    dz[i] = (s - t) / (float)B;
    const float l = fmaxf(x, 0.f) - x * t + log1pf(expf(-fabsf(x)));
    atomicAdd(loss, l / (float)B);
}

// db[n] = sum_m dY[m, n]
__global__ void k_colsum(const float* __restrict__ dy, float* __restrict__ db, int M, int N) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (int m = 0; m < M; ++m) s += dy[(size_t)m * N + n];
    db[n] = s;
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, size_t n, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       float wd) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i] + wd * w[i];
    m1[i] = b1 * m1[i] + (1.f - b1) * gi;
    m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
    w[i] -= lr * (m1[i] / bc1) / (sqrtf(m2[i] / bc2) + eps);
}

__global__ void k_gather_rows(const float* __restrict__ X, const uint8_t* __restrict__ Y, const uint32_t* __restrict__ idx,
                              int B, int D, float* __restrict__ xb, uint8_t* __restrict__ yb) {
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < B * D) xb[t] = X[(size_t)idx[t / D] * D + (t % D)];
    if (t < B * 2) yb[t] = Y[(size_t)idx[t / 2] * 2 + (t % 2)];
}

void gemm(bool ta, bool tb, const float* A, const float* B, float* C, const float* bias, int M, int N, int K, int lda,
          int ldb, float beta, cudaStream_t s) {
    dim3 grid((N + TB - 1) / TB, (M + TB - 1) / TB);
    if (!ta && !tb) k_gemm<false, false><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, beta);
    else if (!ta && tb) k_gemm<false, true><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, beta);
    else if (ta && !tb) k_gemm<true, false><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, beta);
    else k_gemm<true, true><<<grid, 256, 0, s>>>(A, B, C, bias, M, N, K, lda, ldb, beta);
    CUDA_LAUNCH_CHECK();
}

unsigned blocks(size_t n) { return (unsigned)((n + 255) / 256); }

}  // namespace

Mlp::Mlp() {
    const size_t sz[6] = {(size_t)kMlpH * kMlpIn, kMlpH, (size_t)kMlpH * kMlpH, kMlpH, (size_t)kMlpOut * kMlpH, kMlpOut};
    for (int i = 0; i < 6; ++i) n[i] = sz[i];
}

void Mlp::init(uint64_t seed, cudaStream_t s) {
    std::mt19937_64 g(seed);
    const int fan_in[6] = {kMlpIn, kMlpIn, kMlpH, kMlpH, kMlpH, kMlpH};
    for (int i = 0; i < 6; ++i) {
        std::vector<float> h(n[i], 0.f);
        if (i % 2 == 0) {  // weights: U(-1/sqrt(fan_in), 1/sqrt(fan_in)); biases 0
            std::uniform_real_distribution<float> U(-1.f / std::sqrt((float)fan_in[i]), 1.f / std::sqrt((float)fan_in[i]));
            for (auto& x : h) x = U(g);
        }
        p[i].alloc(n[i] * 4);
        gr[i].alloc(n[i] * 4);
        m1[i].alloc(n[i] * 4);
        m2[i].alloc(n[i] * 4);
        CUDA_CHECK(cudaMemcpyAsync(p[i].p, h.data(), n[i] * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemsetAsync(m1[i].p, 0, n[i] * 4, s));
        CUDA_CHECK(cudaMemsetAsync(m2[i].p, 0, n[i] * 4, s));
    }
    std::vector<float> nr(2 * kMlpIn, 0.f);
    for (int f = 0; f < kMlpIn; ++f) nr[kMlpIn + f] = 1.f;
    norm.alloc(nr.size() * 4);
    CUDA_CHECK(cudaMemcpyAsync(norm.p, nr.data(), nr.size() * 4, cudaMemcpyHostToDevice, s));
    tc_err.alloc(16);
    CUDA_CHECK(cudaMemsetAsync(tc_err.p, 0, 16, s));
    step = 0;
    ready = true;
    CUDA_CHECK(cudaStreamSynchronize(s));
}

void Mlp::ensure_work(int B) {
    if (cap >= B) return;
    cap = B;
    const size_t b = (size_t)B;
    xn.alloc(b * kMlpIn * 4);
    z1.alloc(b * kMlpH * 4);
    a1.alloc(b * kMlpH * 4);
    z2.alloc(b * kMlpH * 4);
    a2.alloc(b * kMlpH * 4);
    z3.alloc(b * kMlpOut * 4);
    g1.alloc(b * kMlpH * 4);
    g2.alloc(b * kMlpH * 4);
    g3.alloc(b * kMlpOut * 4);
}

void Mlp::forward(const float* X, int B, cudaStream_t s) {
    ensure_work(B);
    forward_into(X, B, xn.as<float>(), z1.as<float>(), a1.as<float>(), z2.as<float>(), a2.as<float>(), z3.as<float>(),
                 s);
}

void Mlp::forward_into(const float* X, int B, float* xn_, float* z1_, float* a1_, float* z2_, float* a2_, float* z3_,
                       cudaStream_t s) const {
    k_normalize<<<blocks((size_t)B * kMlpIn), 256, 0, s>>>(X, norm.as<float>(), xn_, (size_t)B * kMlpIn);
    CUDA_LAUNCH_CHECK();
    // the two 256 x 256 layers on the tensor cores (GELU in the epilogue), the
    // 2-output layer on the CUDA cores
    mlp_layer_tc(xn_, B, w(0), b(0), nullptr, z1_, a1_, true, tc_err.as<int>(), s);
    mlp_layer_tc(a1_, B, w(1), b(1), nullptr, z2_, a2_, true, tc_err.as<int>(), s);
    gemm(false, true, a2_, w(2), z3_, b(2), B, kMlpOut, kMlpH, kMlpH, kMlpH, 0.f, s);
}

// Gradients of the mean BCE over the batch into gr[] (forward must have run on X;
// layer 1 reads the normalised copy it left in xn).
void Mlp::backward(const float* X, const uint8_t* Y, int B, float* loss, cudaStream_t s) {
    (void)X;
    k_bce<<<blocks((size_t)B * 2), 256, 0, s>>>(z3.as<float>(), Y, g3.as<float>(), B, loss);
    CUDA_LAUNCH_CHECK();
    // layer 3: dW3 = g3^T a2, db3 = colsum g3, g2 = g3 W3 * gelu'(z2)
    gemm(true, false, g3.as<float>(), a2.as<float>(), gr[4].as<float>(), nullptr, kMlpOut, kMlpH, B, kMlpOut, kMlpH,
         0.f, s);
    k_colsum<<<1, 256, 0, s>>>(g3.as<float>(), gr[5].as<float>(), B, kMlpOut);
    CUDA_LAUNCH_CHECK();
    gemm(false, false, g3.as<float>(), w(2), g2.as<float>(), nullptr, B, kMlpH, kMlpOut, kMlpOut, kMlpH, 0.f, s);
    k_gelu_back<<<blocks((size_t)B * kMlpH), 256, 0, s>>>(z2.as<float>(), g2.as<float>(), (size_t)B * kMlpH);
    CUDA_LAUNCH_CHECK();
    // layer 2
    gemm(true, false, g2.as<float>(), a1.as<float>(), gr[2].as<float>(), nullptr, kMlpH, kMlpH, B, kMlpH, kMlpH, 0.f,
         s);
    k_colsum<<<1, 256, 0, s>>>(g2.as<float>(), gr[3].as<float>(), B, kMlpH);
    CUDA_LAUNCH_CHECK();
    gemm(false, false, g2.as<float>(), w(1), g1.as<float>(), nullptr, B, kMlpH, kMlpH, kMlpH, kMlpH, 0.f, s);
    k_gelu_back<<<blocks((size_t)B * kMlpH), 256, 0, s>>>(z1.as<float>(), g1.as<float>(), (size_t)B * kMlpH);
    CUDA_LAUNCH_CHECK();
    // layer 1
    gemm(true, false, g1.as<float>(), xn.as<float>(), gr[0].as<float>(), nullptr, kMlpH, kMlpIn, B, kMlpH, kMlpIn,
         0.f, s);
    k_colsum<<<1, 256, 0, s>>>(g1.as<float>(), gr[1].as<float>(), B, kMlpH);
    CUDA_LAUNCH_CHECK();
}

void Mlp::check_tc() {
    int e = 0;
    CUDA_CHECK(cudaMemcpy(&e, tc_err.p, 4, cudaMemcpyDeviceToHost));
    if (e) fail(HRNN_ERR_TIMEOUT, "budget MLP: a tensor-core wait ran out");
}

void Mlp::adam(float lr, float wd, cudaStream_t s) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float bc1 = 1.f - std::pow(b1, (float)step), bc2 = 1.f - std::pow(b2, (float)step);
    for (int i = 0; i < 6; ++i) {
        k_adam<<<blocks(n[i]), 256, 0, s>>>(p[i].as<float>(), gr[i].as<float>(), m1[i].as<float>(), m2[i].as<float>(),
                                            n[i], lr, b1, b2, 1e-8f, bc1, bc2, (i % 2 == 0) ? wd : 0.f);
        CUDA_LAUNCH_CHECK();
    }
}

float Mlp::train(const float* d_X, const uint8_t* d_Y, size_t N, int epochs, int batch, float lr, uint64_t seed,
                 cudaStream_t s) {
    if (!ready) fail(HRNN_ERR_STATE, "budget: model not initialised");
    DevMem idx, xb, yb, loss;
    idx.alloc(N * 4);
    xb.alloc((size_t)batch * kMlpIn * 4);
    yb.alloc((size_t)batch * 2);
    loss.alloc(4);
    std::vector<uint32_t> perm(N);
    for (size_t i = 0; i < N; ++i) perm[i] = (uint32_t)i;
    std::mt19937_64 g(seed ^ 0x9E3779B97F4A7C15ull);
    float last = 0.f;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), g);
        CUDA_CHECK(cudaMemcpyAsync(idx.p, perm.data(), N * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemsetAsync(loss.p, 0, 4, s));
        int nb = 0;
        for (size_t b0 = 0; b0 + (size_t)batch <= N; b0 += batch, ++nb) {
            k_gather_rows<<<blocks((size_t)batch * kMlpIn), 256, 0, s>>>(d_X, d_Y, idx.as<uint32_t>() + b0, batch,
                                                                        kMlpIn, xb.as<float>(), yb.as<uint8_t>());
            CUDA_LAUNCH_CHECK();
            forward(xb.as<float>(), batch, s);
            backward(xb.as<float>(), yb.as<uint8_t>(), batch, loss.as<float>(), s);
            adam(lr, 1e-4f, s);
        }
        float l = 0.f;
        CUDA_CHECK(cudaMemcpyAsync(&l, loss.p, 4, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        check_tc();
        last = nb ? l / nb : 0.f;
    }
    return last;
}

}  // namespace hrnn
