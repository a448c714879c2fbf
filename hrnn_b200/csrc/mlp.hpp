// The budget MLP (mlp.cu) and its serving parameters (budget.cu).
#pragma once

#include <cstdint>

#include "index.hpp"

namespace hrnn {

constexpr int kMlpIn = 256, kMlpH = 256, kMlpOut = 2;
constexpr int kFrontier = 32;  // beam entries the features read

struct Mlp {
    // parameters: W1 [H x In], b1, W2 [H x H], b2, W3 [Out x H], b3 (FP32 masters)
    DevMem p[6], gr[6], m1[6], m2[6];
    size_t n[6];
    DevMem norm;  // input normalisation: mean[In], 1/std[In] (x -> (x - mean) * inv)
    DevMem tc_err;  // set by the tensor-core layers when a bounded wait runs out
    DevMem xn, z1, a1, z2, a2, z3, g1, g2, g3;  // normalised input, activations / gradients of one batch
    int cap = 0;
    long step = 0;
    bool ready = false;

    Mlp();
    float* w(int l) const { return p[2 * l].as<float>(); }
    float* b(int l) const { return p[2 * l + 1].as<float>(); }
    void init(uint64_t seed, cudaStream_t s);  // random weights, identity normalisation
    void ensure_work(int B);
    void forward(const float* X, int B, cudaStream_t s);  // logits in z3
    // The same into caller buffers (xn [B x In], z1 a1 z2 a2 [B x H], z3 [B x Out]):
    // no allocation, so it can be recorded in a graph that outlives the members'.
    void forward_into(const float* X, int B, float* xn_, float* z1_, float* a1_, float* z2_, float* a2_, float* z3_,
                      cudaStream_t s) const;
    void backward(const float* X, const uint8_t* Y, int B, float* loss, cudaStream_t s);
    void adam(float lr, float wd, cudaStream_t s);
    void check_tc();  // after a synchronisation: fails if a tensor-core wait ran out
    float train(const float* d_X, const uint8_t* d_Y, size_t N, int epochs, int batch, float lr, uint64_t seed,
                cudaStream_t s);  // d_X raw features; the model must be initialised
};

struct Budget {
    Mlp mlp;
    bool enabled = false;
    uint32_t m[2] = {1, 3};       // proxies of budget levels 0 and 1
    uint32_t ef = 0;              // level beam (two-pass mode); 0: the caller's beam
    float confidence = 0.9f;      // probability cutoff for taking a level
    DevMem proj;                  // [dim x 128] fixed random projection of the query
    uint32_t proj_dim = 0;
    DevMem feat, decided, fallback_list, proxd;  // per-call work buffers
    DevMem saved;                 // two-pass mode: the frontier beams the fallback resumes
    unsigned long long n_level[3] = {0, 0, 0};  // queries served at level 0 / 1 / fallback (last call)
};

// mlp_tc.cu: tcgen05 layer out = act(norm(A) W^T + b), A [M x 256], W [256 x 256]
void mlp_layer_tc(const float* A, int M, const float* W, const float* bias, const float* nrm, float* out_z,
                  float* out_a, bool gelu, int* err, cudaStream_t s);
// The layer kernel's launch attributes on the current device (before a stream
// capture that records the layer).
void mlp_layer_tc_prepare();

// search_plain.cu
Budget& budget_of(Index& ix);
void budget_features(Index& ix, const float* d_q, size_t nq, uint32_t k, uint32_t m, uint32_t ef, float* d_feat);

// budget.cu: host entry points (host buffers unless named d_*)
void budget_set(Index& ix, bool enable, uint32_t m0, uint32_t m1, uint32_t ef, float confidence);
float budget_train(Index& ix, const float* feat, const uint8_t* labels, size_t n, int epochs, int batch, float lr,
                   uint64_t seed);
void budget_predict(Index& ix, const float* feat, size_t n, float* logits);
float budget_gradients(Index& ix, const float* feat, const uint8_t* labels, size_t n, float* grads);
void budget_get_weights(Index& ix, float* params);
void budget_set_weights(Index& ix, const float* params);
// Parameter layout of get/set weights: W1 b1 W2 b2 W3 b3, then mean and 1/std of
// the input normalisation.
constexpr size_t kBudgetParams = (size_t)kMlpH * kMlpIn + kMlpH + (size_t)kMlpH * kMlpH + kMlpH +
                                 (size_t)kMlpOut * kMlpH + kMlpOut + 2 * (size_t)kMlpIn;

}  // namespace hrnn
