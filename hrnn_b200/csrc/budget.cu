// Learned search budget: features of a query and its first beam frontier, the
// MLP decision, and the host entry points for training and serving.
//
// Frontier pass: the beam search (the caller's, or the level ef in two-pass mode)
// returning its kFrontier nearest entries.  Features (256 per query): 128 values of a fixed Gaussian
// projection of the query (/ sqrt(dim)); for each of the 32 frontier entries
// log(1 + d), log(1 + kdist(p, k-1)), d / kdist (clipped to [0, 4]) and the
// reverse in-degree log(1 + |R(p)|) / 8 (missing entries: 0).
// Decision: level 0 when sigmoid(z0) >= confidence, else level 1 when
// sigmoid(z1) >= confidence, else the caller's m.  Levels take the first m0 / m1
// entries of the frontier (the proxies the plain search finds with that m).
// Single-pass mode (level ef 0): the frontier is the caller's own beam, so the
// budget only trims proxies.  Two-pass mode: the frontier beam is the level ef
// and the fallback queries are searched again with the caller's (m, ef).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <random>
#include <vector>

#include "beam.cuh"
#include "index.hpp"
#include "mlp.hpp"

namespace hrnn {

__global__ void k_budget_features(DevView v, const float* __restrict__ Q, uint32_t nq,
                                  const uint32_t* __restrict__ prox, const float* __restrict__ proxd,
                                  const uint32_t* __restrict__ nprox, uint32_t stride,
                                  const float* __restrict__ kcol, const float* __restrict__ proj,
                                  float* __restrict__ feat) {
    const int lane = threadIdx.x & 31;
    const uint32_t qi = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (qi >= nq) return;
    const float* q = Q + (size_t)qi * v.dim;
    float* f = feat + (size_t)qi * kMlpIn;
    const float sc = rsqrtf((float)v.dim);
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t i = 0; i < v.dim; ++i) {
        const float x = q[i];
#pragma unroll
        for (int t = 0; t < 4; ++t) acc[t] = fmaf(x, proj[(size_t)i * 128 + lane + 32 * t], acc[t]);
    }
#pragma unroll
    for (int t = 0; t < 4; ++t) f[lane + 32 * t] = acc[t] * sc;
    const uint32_t np_ = nprox[qi];
    float f0 = 0.f, f1 = 0.f, f2 = 0.f, f3 = 0.f;
    if ((uint32_t)lane < np_) {
        const uint32_t id = prox[(size_t)qi * stride + lane];
        const float d = proxd[(size_t)qi * stride + lane];
        const float kd = kcol[id];
        f0 = log1pf(d);
        f1 = kd >= FLT_MAX ? 20.f : log1pf(kd);
        f2 = kd >= FLT_MAX ? 0.f : fminf(d / fmaxf(kd, 1e-30f), 4.f);
        f3 = log1pf((float)(v.csr_off[id + 1] - v.csr_off[id])) * 0.125f;
    }
    f[128 + lane] = f0;
    f[160 + lane] = f1;
    f[192 + lane] = f2;
    f[224 + lane] = f3;
}

// Per query: budget level from the logits; nprox trimmed for levels 0/1.
// Fallback queries keep the caller's m (single pass) or are listed for a second
// search (rerun).
// grp (may be null): 1 for the queries listed for the second search, else 0.
__global__ void k_budget_decide(const float* __restrict__ z, uint32_t nq, float conf, uint32_t m0, uint32_t m1,
                                const uint32_t* __restrict__ qm, int rerun, uint32_t* __restrict__ nprox,
                                uint32_t* __restrict__ fb_list,
                                uint32_t* __restrict__ fb_count, unsigned long long* __restrict__ levels,
                                uint8_t* __restrict__ grp) {
    const uint32_t qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    const float p0 = 1.f / (1.f + expf(-z[2 * qi])), p1 = 1.f / (1.f + expf(-z[2 * qi + 1]));
    uint8_t g = 0;
    if (p0 >= conf) {
        nprox[qi] = min(nprox[qi], min(m0, qm[qi]));
        atomicAdd(&levels[0], 1ull);
    } else if (p1 >= conf) {
        nprox[qi] = min(nprox[qi], min(m1, qm[qi]));
        atomicAdd(&levels[1], 1ull);
    } else {
        if (rerun) {
            fb_list[atomicAdd(fb_count, 1u)] = qi;
            g = 1;
        } else {
            nprox[qi] = min(nprox[qi], qm[qi]);
        }
        atomicAdd(&levels[2], 1ull);
    }
    if (grp) grp[qi] = g;
}

void ensure_projection(Index& ix, Budget& b) {
    if (b.proj_dim == ix.dim) return;
    std::mt19937_64 g(0x5EEDBA5Eull);
    std::normal_distribution<float> N(0.f, 1.f);
    std::vector<float> h(ix.dim * 128);
    for (auto& x : h) x = N(g);
    b.proj.alloc(h.size() * 4);
    CUDA_CHECK(cudaMemcpy(b.proj.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    b.proj_dim = (uint32_t)ix.dim;
}

void budget_set(Index& ix, bool enable, uint32_t m0, uint32_t m1, uint32_t ef, float confidence) {
    Budget& b = budget_of(ix);
    if (enable && !b.mlp.ready) fail(HRNN_ERR_STATE, "budget: train the model or set its weights first");
    if (m0 == 0 || m1 < m0 || m1 > (uint32_t)kFrontier) fail(HRNN_ERR_ARG, "budget: need 1 <= m0 <= m1 <= 32");
    if (ef != 0 && (ef < m1 || ef > (1u << 16))) fail(HRNN_ERR_ARG, "budget: ef must be 0 or in [m1, 65536]");
    if (!(confidence > 0.5f && confidence <= 1.f)) fail(HRNN_ERR_ARG, "budget: confidence must be in (0.5, 1]");
    if (ix.dim % 4 != 0) fail(HRNN_ERR_ARG, "budget: dim must be a multiple of 4");
    b.m[0] = m0;
    b.m[1] = m1;
    b.ef = ef;
    b.confidence = confidence;
    b.enabled = enable;
}

namespace {

void upload(DevMem& d, const void* h, size_t bytes, cudaStream_t s) {
    d.alloc(bytes);
    CUDA_CHECK(cudaMemcpyAsync(d.p, h, bytes, cudaMemcpyHostToDevice, s));
}

}  // namespace

float budget_train(Index& ix, const float* feat, const uint8_t* labels, size_t n, int epochs, int batch, float lr,
                   uint64_t seed) {
    if (n == 0 || epochs <= 0 || batch <= 0 || !(lr > 0.f)) fail(HRNN_ERR_ARG, "budget_train: bad arguments");
    if ((size_t)batch > n) batch = (int)n;
    if (n > 0xFFFFFFFFull) fail(HRNN_ERR_ARG, "budget_train: too many samples");
    Budget& b = budget_of(ix);
    cudaStream_t s = ix.stream;
    if (!b.mlp.ready) {
        // Fresh model: random weights and the training features' per-feature mean
        // and 1/std (0 for constant features) as the input normalisation.
        b.mlp.init(seed, s);
        std::vector<double> mu(kMlpIn, 0.0), var(kMlpIn, 0.0);
        for (size_t i = 0; i < n; ++i)
            for (int f = 0; f < kMlpIn; ++f) mu[f] += feat[i * kMlpIn + f];
        for (int f = 0; f < kMlpIn; ++f) mu[f] /= (double)n;
        for (size_t i = 0; i < n; ++i)
            for (int f = 0; f < kMlpIn; ++f) {
                const double d = feat[i * kMlpIn + f] - mu[f];
                var[f] += d * d;
            }
        std::vector<float> nr(2 * kMlpIn);
        for (int f = 0; f < kMlpIn; ++f) {
            const double sd = std::sqrt(var[f] / (double)n);
            nr[f] = (float)mu[f];
            nr[kMlpIn + f] = sd > 1e-12 ? (float)(1.0 / sd) : 0.f;
        }
        CUDA_CHECK(cudaMemcpyAsync(b.mlp.norm.p, nr.data(), nr.size() * 4, cudaMemcpyHostToDevice, s));
    }
    DevMem X, Y;
    upload(X, feat, n * kMlpIn * 4, s);
    upload(Y, labels, n * 2, s);
    return b.mlp.train(X.as<float>(), Y.as<uint8_t>(), n, epochs, batch, lr, seed, s);
}

void budget_predict(Index& ix, const float* feat, size_t n, float* logits) {
    Budget& b = budget_of(ix);
    if (!b.mlp.ready) fail(HRNN_ERR_STATE, "budget: the model has no weights");
    cudaStream_t s = ix.stream;
    const size_t chunk = 16384;
    DevMem X;
    X.alloc(std::min(n, chunk) * kMlpIn * 4);
    for (size_t i0 = 0; i0 < n; i0 += chunk) {
        const size_t c = std::min(chunk, n - i0);
        CUDA_CHECK(cudaMemcpyAsync(X.p, feat + i0 * kMlpIn, c * kMlpIn * 4, cudaMemcpyHostToDevice, s));
        b.mlp.forward(X.as<float>(), (int)c, s);
        CUDA_CHECK(cudaMemcpyAsync(logits + i0 * kMlpOut, b.mlp.z3.p, c * kMlpOut * 4, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        b.mlp.check_tc();
    }
}

float budget_gradients(Index& ix, const float* feat, const uint8_t* labels, size_t n, float* grads) {
    Budget& b = budget_of(ix);
    if (!b.mlp.ready) fail(HRNN_ERR_STATE, "budget: the model has no weights");
    if (n == 0 || n > (1u << 20)) fail(HRNN_ERR_ARG, "budget_gradients: n must be in [1, 2^20]");
    cudaStream_t s = ix.stream;
    DevMem X, Y, L;
    upload(X, feat, n * kMlpIn * 4, s);
    upload(Y, labels, n * 2, s);
    L.alloc(4);
    CUDA_CHECK(cudaMemsetAsync(L.p, 0, 4, s));
    b.mlp.forward(X.as<float>(), (int)n, s);
    b.mlp.backward(X.as<float>(), Y.as<uint8_t>(), (int)n, L.as<float>(), s);
    size_t off = 0;
    for (int i = 0; i < 6; ++i) {
        CUDA_CHECK(cudaMemcpyAsync(grads + off, b.mlp.gr[i].p, b.mlp.n[i] * 4, cudaMemcpyDeviceToHost, s));
        off += b.mlp.n[i];
    }
    std::fill(grads + off, grads + off + 2 * kMlpIn, 0.f);
    float loss = 0.f;
    CUDA_CHECK(cudaMemcpyAsync(&loss, L.p, 4, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    b.mlp.check_tc();
    return loss;
}

void budget_get_weights(Index& ix, float* params) {
    Budget& b = budget_of(ix);
    if (!b.mlp.ready) fail(HRNN_ERR_STATE, "budget: the model has no weights");
    size_t off = 0;
    for (int i = 0; i < 6; ++i) {
        CUDA_CHECK(cudaMemcpy(params + off, b.mlp.p[i].p, b.mlp.n[i] * 4, cudaMemcpyDeviceToHost));
        off += b.mlp.n[i];
    }
    CUDA_CHECK(cudaMemcpy(params + off, b.mlp.norm.p, 2 * kMlpIn * 4, cudaMemcpyDeviceToHost));
}

void budget_set_weights(Index& ix, const float* params) {
    Budget& b = budget_of(ix);
    if (!b.mlp.ready) b.mlp.init(0, ix.stream);
    size_t off = 0;
    for (int i = 0; i < 6; ++i) {
        CUDA_CHECK(cudaMemcpy(b.mlp.p[i].p, params + off, b.mlp.n[i] * 4, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemset(b.mlp.m1[i].p, 0, b.mlp.n[i] * 4));
        CUDA_CHECK(cudaMemset(b.mlp.m2[i].p, 0, b.mlp.n[i] * 4));
        off += b.mlp.n[i];
    }
    CUDA_CHECK(cudaMemcpy(b.mlp.norm.p, params + off, 2 * kMlpIn * 4, cudaMemcpyHostToDevice));
    b.mlp.step = 0;
}

}  // namespace hrnn
