// extern "C" boundary: handle management, status codes and the thread-local
// error message.  Every entry point maps one HRNN<float> member (see
// include/hrnn_capi.h for the citations) onto the device implementation.
#include <cuda_runtime.h>

#include <cstring>
#include <algorithm>
#include <random>
#include <numeric>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "index.hpp"
#include "plan.hpp"
#include "mlp.hpp"

static_assert(hrnn::kBudgetParams == HRNN_BUDGET_PARAMS, "budget parameter layout");

struct hrnn_index {
    hrnn::Index ix;
};

struct hrnn_search_plan {
    hrnn_index* h;
    hrnn::SearchPlan p;
};

namespace {

thread_local std::string g_last_error;

template <class F>
hrnn_status guard(F&& f) {
    try {
        g_last_error.clear();
        f();
        return HRNN_OK;
    } catch (const hrnn::Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "Not enough memory";
        return HRNN_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return HRNN_ERR_STATE;
    }
}

void need(const void* p, const char* what) {
    if (!p) hrnn::fail(HRNN_ERR_ARG, std::string(what) + " is NULL");
}

void set_device(hrnn_index* h) { CUDA_CHECK(cudaSetDevice(h->ix.device)); }

}  // namespace

namespace hrnn {
void set_last_error(const std::string& m) { g_last_error = m; }
}  // namespace hrnn

extern "C" {

const char* hrnn_last_error(void) { return g_last_error.c_str(); }

int hrnn_version(void) { return 10000; }

hrnn_status hrnn_create(hrnn_index** out, size_t dim, size_t max_elements, size_t M, size_t efc,
                        size_t seed, size_t K, int device) {
    return guard([&] {
        need(out, "out");
        *out = nullptr;
        if (M < 2) hrnn::fail(HRNN_ERR_ARG, "M must be >= 2");
        auto h = std::make_unique<hrnn_index>();
        h->ix.device = device;
        h->ix.order = hrnn::detect_l2_order();
        hrnn::init_layout(h->ix, dim, max_elements, M, efc, seed, K);
        hrnn::alloc_device(h->ix, max_elements);
        *out = h.release();
    });
}

hrnn_status hrnn_load(hrnn_index** out, const char* path, size_t dim, size_t max_elements, int device) {
    return guard([&] {
        need(out, "out");
        need(path, "path");
        *out = nullptr;
        auto h = std::make_unique<hrnn_index>();
        h->ix.device = device;
        h->ix.order = hrnn::detect_l2_order();
        hrnn::load_idx(h->ix, path, dim, max_elements);  // file checks come before any CUDA call
        *out = h.release();
    });
}

hrnn_status hrnn_save(hrnn_index* h, const char* path) {
    return guard([&] {
        need(h, "index");
        need(path, "path");
        set_device(h);
        hrnn::save_idx(h->ix, path);
    });
}

void hrnn_destroy(hrnn_index* h) {
    if (!h) return;
    cudaSetDevice(h->ix.device);
    delete h;
}

hrnn_status hrnn_add_points(hrnn_index* h, const float* data, const uint64_t* labels, size_t n) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        if (n) need(data, "data");
        set_device(h);
        hrnn::add_points(h->ix, data, labels, n);
    });
}

hrnn_status hrnn_refine_knng(hrnn_index* h, int iters, int sample) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        set_device(h);
        hrnn::refine_knng(h->ix, iters, sample);
    });
}

hrnn_status hrnn_build_rknng(hrnn_index* h) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        set_device(h);
        hrnn::build_rknng(h->ix);
    });
}

hrnn_status hrnn_build_rknng_mutable(hrnn_index* h) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        set_device(h);
        hrnn::build_rknng_mutable(h->ix);
    });
}

hrnn_status hrnn_search_rknn_batch_device(hrnn_index* h, const float* d_q, size_t nq, const uint32_t* d_m,
                                          const uint32_t* d_Kp, const uint32_t* d_ef, float threshold,
                                          uint32_t k, uint64_t* d_out_offsets, uint64_t* d_out_labels,
                                          size_t cap, uint64_t* out_total, void* stream) {
    return guard([&] {
        need(h, "index");
        if (nq) {
            need(d_q, "queries");
            need(d_m, "m");
            need(d_Kp, "K_prime");
            need(d_ef, "ef_search");
        }
        need(d_out_offsets, "out_offsets");
        set_device(h);
        hrnn::SearchArgs a{d_q, nq, d_m, d_Kp, d_ef, threshold, k, d_out_offsets, d_out_labels, cap,
                           (cudaStream_t)stream};
        uint64_t total = hrnn::search_batch(h->ix, a);
        if (out_total) *out_total = total;
        if (total > cap) hrnn::fail(HRNN_ERR_CAPACITY, "searchRknn: output capacity too small");
    });
}

hrnn_status hrnn_search_rknn_batch(hrnn_index* h, const float* q, size_t nq, const uint32_t* m,
                                   const uint32_t* Kp, const uint32_t* ef, float threshold, uint32_t k,
                                   uint64_t* out_offsets, uint64_t* out_labels, size_t cap) {
    return guard([&] {
        need(h, "index");
        need(out_offsets, "out_offsets");
        if (nq) {
            need(q, "queries");
            need(m, "m");
            need(Kp, "K_prime");
            need(ef, "ef_search");
        }
        set_device(h);
        hrnn::Index& ix = h->ix;
        cudaStream_t s = ix.stream;
        // Inputs and outputs staged through one device block: queries, m, K', ef,
        // offsets, labels.
        size_t qb = nq * ix.dim * 4, ib = nq * 4, ob = (nq + 1) * 8, lb = std::max<size_t>(cap, 1) * 8;
        auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
        size_t need_b = al(qb) + 3 * al(ib) + al(ob) + al(lb);
        hrnn::DevMem& io = ix.io;
        io.ensure(need_b);
        char* base = io.as<char>();
        float* dq = (float*)base;
        uint32_t* dm = (uint32_t*)(base + al(qb));
        uint32_t* dkp = (uint32_t*)((char*)dm + al(ib));
        uint32_t* def = (uint32_t*)((char*)dkp + al(ib));
        uint64_t* doff = (uint64_t*)((char*)def + al(ib));
        uint64_t* dlab = (uint64_t*)((char*)doff + al(ob));
        if (nq) {
            CUDA_CHECK(cudaMemcpyAsync(dq, q, qb, cudaMemcpyHostToDevice, s));
            CUDA_CHECK(cudaMemcpyAsync(dm, m, ib, cudaMemcpyHostToDevice, s));
            CUDA_CHECK(cudaMemcpyAsync(dkp, Kp, ib, cudaMemcpyHostToDevice, s));
            CUDA_CHECK(cudaMemcpyAsync(def, ef, ib, cudaMemcpyHostToDevice, s));
        }
        hrnn::SearchArgs a{dq, nq, dm, dkp, def, threshold, k, doff, dlab, cap, s};
        for (size_t i = 0; i < nq; ++i) {  // the maxima from the host arrays: no read-back
            a.h_mmax = std::max(a.h_mmax, m[i]);
            a.h_efmax = std::max(a.h_efmax, std::max(ef[i], m[i]));
        }
        uint64_t total = hrnn::search_batch(ix, a);
        CUDA_CHECK(cudaMemcpyAsync(out_offsets, doff, ob, cudaMemcpyDeviceToHost, s));
        if (total <= cap && total && out_labels)
            CUDA_CHECK(cudaMemcpyAsync(out_labels, dlab, total * 8, cudaMemcpyDeviceToHost, s));
        CUDA_CHECK(cudaStreamSynchronize(s));
        if (total > cap) hrnn::fail(HRNN_ERR_CAPACITY, "searchRknn: output capacity too small");
    });
}

hrnn_status hrnn_search_rknn(hrnn_index* h, const float* query, size_t m, float threshold, size_t k,
                             size_t K_prime, size_t ef_search, uint64_t* out_labels, size_t cap,
                             size_t* out_count) {
    uint32_t mm = (uint32_t)m, kp = (uint32_t)std::min<size_t>(K_prime, 0xFFFFFFFFu),
             ee = (uint32_t)ef_search;
    uint64_t off[2] = {0, 0};
    hrnn_status st = hrnn_search_rknn_batch(h, query, 1, &mm, &kp, &ee, threshold, (uint32_t)k, off,
                                            out_labels, cap);
    if (out_count) *out_count = (size_t)off[1];
    return st;
}

hrnn_status hrnn_search_plan_create(hrnn_index* h, const float* d_queries, size_t nq, const uint32_t* d_m,
                                    const uint32_t* d_K_prime, const uint32_t* d_ef_search, uint32_t m_max,
                                    uint32_t ef_max, float threshold, uint32_t k, uint64_t* d_out_offsets,
                                    uint64_t* d_out_labels, size_t cap, void* stream, hrnn_search_plan** out) {
    return guard([&] {
        need(h, "index");
        need(out, "out");
        need(d_queries, "queries");
        need(d_m, "m");
        need(d_K_prime, "K_prime");
        need(d_ef_search, "ef_search");
        need(d_out_offsets, "out_offsets");
        if (cap > 0) need(d_out_labels, "out_labels");
        set_device(h);
        auto* pl = new hrnn_search_plan{h, {}};
        try {
            hrnn::SearchPlan& p = pl->p;
            p.ix = &h->ix;
            p.nq = nq;
            p.cap = cap;
            p.m_max = m_max;
            p.ef_max = ef_max;
            p.k = k;
            p.threshold = threshold;
            p.d_q = d_queries;
            p.d_m = d_m;
            p.d_kp = d_K_prime;
            p.d_ef = d_ef_search;
            p.d_out_off = d_out_offsets;
            p.d_out_lab = d_out_labels;
            hrnn::plan_create(p, stream ? (cudaStream_t)stream : h->ix.stream);
        } catch (...) {
            delete pl;
            throw;
        }
        *out = pl;
    });
}

hrnn_status hrnn_search_plan_run(hrnn_search_plan* plan, void* stream) {
    return guard([&] {
        need(plan, "plan");
        set_device(plan->h);
        hrnn::plan_run(plan->p, stream ? (cudaStream_t)stream : plan->h->ix.stream);
    });
}

hrnn_status hrnn_search_plan_result(hrnn_search_plan* plan, void* stream, uint64_t* total, int* clamped) {
    return guard([&] {
        need(plan, "plan");
        set_device(plan->h);
        const uint64_t t = hrnn::plan_result(plan->p, stream ? (cudaStream_t)stream : plan->h->ix.stream, clamped);
        if (total) *total = t;
        if (t > plan->p.cap) hrnn::fail(HRNN_ERR_CAPACITY, "search plan: results exceed the capacity; labels not written");
    });
}

hrnn_status hrnn_search_plan_run_host(hrnn_search_plan* plan, const float* queries, const uint32_t* m,
                                      const uint32_t* K_prime, const uint32_t* ef_search, uint64_t* out_offsets,
                                      uint64_t* out_labels, size_t cap, uint64_t* total, int* clamped, void* stream) {
    return guard([&] {
        need(plan, "plan");
        need(queries, "queries");
        need(m, "m");
        need(K_prime, "K_prime");
        need(ef_search, "ef_search");
        need(out_offsets, "out_offsets");
        set_device(plan->h);
        hrnn::SearchPlan& p = plan->p;
        cudaStream_t s = stream ? (cudaStream_t)stream : plan->h->ix.stream;
        const size_t nq = p.nq;
        // the host batch into the plan's input buffers, the graph, the outputs back
        CUDA_CHECK(cudaMemcpyAsync(const_cast<float*>(p.d_q), queries, nq * plan->h->ix.dim * 4,
                                   cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(p.d_m), m, nq * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(p.d_kp), K_prime, nq * 4, cudaMemcpyHostToDevice, s));
        CUDA_CHECK(cudaMemcpyAsync(const_cast<uint32_t*>(p.d_ef), ef_search, nq * 4, cudaMemcpyHostToDevice, s));
        hrnn::plan_run(p, s);
        const uint64_t t = hrnn::plan_result(p, s, clamped);
        if (total) *total = t;
        if (t > cap || t > p.cap)
            hrnn::fail(HRNN_ERR_CAPACITY, "search plan: results exceed the capacity; labels not written");
        CUDA_CHECK(cudaMemcpyAsync(out_offsets, p.d_out_off, (nq + 1) * 8, cudaMemcpyDeviceToHost, s));
        if (t) {
            need(out_labels, "out_labels");
            CUDA_CHECK(cudaMemcpyAsync(out_labels, p.d_out_lab, t * 8, cudaMemcpyDeviceToHost, s));
        }
        CUDA_CHECK(cudaStreamSynchronize(s));
    });
}

hrnn_status hrnn_search_plan_kernels(hrnn_search_plan* plan, size_t* n) {
    return guard([&] {
        need(plan, "plan");
        need(n, "n");
        *n = plan->p.kernel_nodes;
    });
}

void hrnn_search_plan_destroy(hrnn_search_plan* plan) {
    if (!plan) return;
    cudaSetDevice(plan->h->ix.device);
    delete plan;
}

hrnn_status hrnn_compact_for_serving(hrnn_index* h, size_t mks) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        set_device(h);
        hrnn::compact_for_serving(h->ix, mks);
    });
}

hrnn_status hrnn_get_rknng_mutable(hrnn_index* h, uint64_t* lens, uint32_t* flat) {
    return guard([&] {
        need(h, "index");
        set_device(h);
        hrnn::mutable_get(h->ix, lens, flat);
    });
}

hrnn_status hrnn_get_kdist(hrnn_index* h, uint32_t k, float* out) {
    return guard([&] {
        need(h, "index");
        need(out, "out");
        set_device(h);
        hrnn::kdist_column(h->ix, k, out);
    });
}

hrnn_status hrnn_insert_dynamic(hrnn_index* h, const float* data, const uint64_t* labels, size_t n,
                                unsigned m_update, int bidirectional) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        if (n) need(data, "data");
        set_device(h);
        hrnn::insert_dynamic(h->ix, data, labels, n, m_update, bidirectional != 0);
    });
}

hrnn_status hrnn_set_ef(hrnn_index* h, size_t ef) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        h->ix.ef = ef;
    });
}

hrnn_status hrnn_get_info(hrnn_index* h, hrnn_info* info) {
    return guard([&] {
        need(h, "index");
        need(info, "info");
        const hrnn::Index& ix = h->ix;
        hrnn_info o{};
        o.dim = ix.dim;
        o.max_elements = ix.max_elements;
        o.cur_element_count = ix.cur;
        o.M = ix.M;
        o.maxM = ix.maxM;
        o.maxM0 = ix.maxM0;
        o.ef_construction = ix.ef_construction;
        o.ef = ix.ef;
        o.K_knng = ix.K;
        o.maxlevel = ix.maxlevel;
        o.enterpoint = ix.enterpoint;
        o.knng_built = ix.knng_built;
        o.rknng_built = ix.rknng_built;
        o.rknng_wide = ix.wide;
        o.rank_bits = ix.rank_bits;
        o.rknng_entries = ix.csr_entries;
        o.serve_mode = ix.serve_mode;
        o.max_k_serve = ix.max_k_serve;
        o.l2_lanes = ix.order.lanes;
        o.l2_fused = ix.order.fused;
        o.device_bytes = ix.device_bytes();
        *info = o;
    });
}

hrnn_status hrnn_get_search_stats(hrnn_index* h, hrnn_search_stats* st) {
    return guard([&] {
        need(h, "index");
        need(st, "stats");
        *st = h->ix.last_stats;
    });
}

hrnn_status hrnn_set_precision(hrnn_index* h, int precision) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        if (precision != HRNN_PREC_FP32_EXACT && precision != HRNN_PREC_BF16 && precision != HRNN_PREC_INT8)
            hrnn::fail(HRNN_ERR_ARG, "set_precision: unknown precision");
        if (precision == HRNN_PREC_INT8 && (h->ix.dim % 16 != 0 || h->ix.dim > 256))
            hrnn::fail(HRNN_ERR_ARG, "set_precision: INT8 needs dim a multiple of 16, at most 256");
        h->ix.precision = precision;
    });
}

hrnn_status hrnn_set_autotune(hrnn_index* h, int enable) {
    return guard([&] {
        need(h, "index");
        h->ix.autotune = enable != 0;
    });
}

hrnn_status hrnn_set_join_mode(hrnn_index* h, int mode) {
    return guard([&] {
        need(h, "index");
        if (mode != HRNN_JOIN_EXACT && mode != HRNN_JOIN_TENSOR && mode != HRNN_JOIN_AUDIT)
            hrnn::fail(HRNN_ERR_ARG, "set_join_mode: unknown join mode");
        h->ix.join_mode = mode;
    });
}

hrnn_status hrnn_set_budget(hrnn_index* h, int enable, uint32_t m0, uint32_t m1, uint32_t ef,
                            float confidence) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;  // captured plans record the budget's settings
        set_device(h);
        hrnn::budget_set(h->ix, enable != 0, m0, m1, ef, confidence);
    });
}

hrnn_status hrnn_budget_features(hrnn_index* h, const float* queries, size_t nq, uint32_t k, uint32_t m,
                                 uint32_t ef_search, float* feat) {
    return guard([&] {
        need(h, "index");
        need(queries, "queries");
        need(feat, "feat");
        if (k == 0) hrnn::fail(HRNN_ERR_ARG, "budget_features: k must be >= 1");
        set_device(h);
        auto& ix = h->ix;
        if (ix.serve_mode ? k > ix.max_k_serve : k > ix.K)
            hrnn::fail(HRNN_ERR_ARG, "budget_features: k larger than the stored neighbour lists");
        if (nq == 0) return;
        hrnn::DevMem q, f;
        q.alloc(nq * ix.dim * 4);
        f.alloc(nq * hrnn::kMlpIn * 4);
        CUDA_CHECK(cudaMemcpyAsync(q.p, queries, nq * ix.dim * 4, cudaMemcpyHostToDevice, ix.stream));
        hrnn::budget_features(ix, q.as<float>(), nq, k, m, ef_search, f.as<float>());
        CUDA_CHECK(cudaMemcpy(feat, f.p, nq * hrnn::kMlpIn * 4, cudaMemcpyDeviceToHost));
    });
}

hrnn_status hrnn_budget_train(hrnn_index* h, const float* feat, const uint8_t* labels, size_t n, int epochs,
                              int batch, float lr, uint64_t seed, float* final_loss) {
    return guard([&] {
        need(h, "index");
        need(feat, "feat");
        need(labels, "labels");
        h->ix.generation++;  // new weights: captured plans record the old ones
        set_device(h);
        const float l = hrnn::budget_train(h->ix, feat, labels, n, epochs, batch, lr, seed);
        if (final_loss) *final_loss = l;
    });
}

hrnn_status hrnn_budget_predict(hrnn_index* h, const float* feat, size_t n, float* logits) {
    return guard([&] {
        need(h, "index");
        need(feat, "feat");
        need(logits, "logits");
        set_device(h);
        hrnn::budget_predict(h->ix, feat, n, logits);
    });
}

hrnn_status hrnn_budget_gradients(hrnn_index* h, const float* feat, const uint8_t* labels, size_t n,
                                  float* grads, float* loss) {
    return guard([&] {
        need(h, "index");
        need(feat, "feat");
        need(labels, "labels");
        need(grads, "grads");
        set_device(h);
        const float l = hrnn::budget_gradients(h->ix, feat, labels, n, grads);
        if (loss) *loss = l;
    });
}

hrnn_status hrnn_budget_get_weights(hrnn_index* h, float* params) {
    return guard([&] {
        need(h, "index");
        need(params, "params");
        set_device(h);
        hrnn::budget_get_weights(h->ix, params);
    });
}

hrnn_status hrnn_budget_set_weights(hrnn_index* h, const float* params) {
    return guard([&] {
        need(h, "index");
        need(params, "params");
        h->ix.generation++;  // new weights: captured plans record the old ones
        set_device(h);
        hrnn::budget_set_weights(h->ix, params);
    });
}

hrnn_status hrnn_get_dynamic_stats(hrnn_index* h, hrnn_dynamic_stats* st) {
    return guard([&] {
        need(h, "index");
        need(st, "stats");
        *st = h->ix.dyn_stats;
    });
}

hrnn_status hrnn_get_refine_stats(hrnn_index* h, hrnn_refine_stats* st) {
    return guard([&] {
        need(h, "index");
        need(st, "stats");
        *st = h->ix.refine_stats;
    });
}

hrnn_status hrnn_set_l2_order(hrnn_index* h, int lanes, int fused) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        if (lanes != 16 && lanes != 8 && lanes != 4) hrnn::fail(HRNN_ERR_ARG, "lanes must be 16, 8 or 4");
        if (fused < 0 || fused > 3) hrnn::fail(HRNN_ERR_ARG, "fused must be in [0, 3]");
        h->ix.order.lanes = lanes;
        h->ix.order.fused = fused;
    });
}

hrnn_status hrnn_dynamic_split(uint64_t n, uint32_t seed, uint32_t* perm) {
    return guard([&] {
        need(perm, "perm");
        if (n > 0xFFFFFFFFull) hrnn::fail(HRNN_ERR_ARG, "dynamic_split: n must fit 32-bit ids");
        std::iota(perm, perm + n, 0u);
        std::mt19937 rng(seed);
        std::shuffle(perm, perm + n, rng);
    });
}

hrnn_status hrnn_detect_l2_order(int* lanes, int* fused) {
    return guard([&] {
        need(lanes, "lanes");
        need(fused, "fused");
        hrnn::L2Order o = hrnn::detect_l2_order();
        *lanes = o.lanes;
        *fused = o.fused;
    });
}

hrnn_status hrnn_get_knng(hrnn_index* h, uint32_t* ids, float* dists, uint32_t* cnt) {
    return guard([&] {
        need(h, "index");
        if (h->ix.serve_mode) hrnn::fail(HRNN_ERR_STATE, "KNN graph slot removed by compactForServing");
        set_device(h);
        hrnn::get_knng(h->ix, ids, dists, cnt);
    });
}

hrnn_status hrnn_set_knng(hrnn_index* h, const uint32_t* ids, const float* dists, const uint32_t* cnt) {
    return guard([&] {
        need(h, "index");
        h->ix.generation++;
        need(ids, "ids");
        need(dists, "dists");
        need(cnt, "cnt");
        if (h->ix.serve_mode) hrnn::fail(HRNN_ERR_STATE, "KNN graph slot removed by compactForServing");
        set_device(h);
        hrnn::set_knng(h->ix, ids, dists, cnt);
    });
}

hrnn_status hrnn_get_rknng(hrnn_index* h, uint64_t* n_offsets, uint64_t* n_entries, uint32_t* entry_bytes,
                           uint32_t* rank_bits, uint64_t* offsets, void* entries, int reference_order) {
    return guard([&] {
        need(h, "index");
        hrnn::Index& ix = h->ix;
        if (!ix.rknng_built) hrnn::fail(HRNN_ERR_STATE, "searchRknn: RKNNG not built");
        set_device(h);
        hrnn::ensure_flat_rknng(ix);
        if (n_offsets) *n_offsets = ix.cur + 1;
        if (n_entries) *n_entries = ix.csr_entries;
        if (entry_bytes) *entry_bytes = ix.wide ? 8 : 4;
        if (rank_bits) *rank_bits = ix.rank_bits;
        if (!offsets && !entries) return;
        need(offsets, "offsets");
        need(entries, "entries");
        if (reference_order) {
            hrnn::rknng_reference_order(ix, offsets, entries);
        } else {
            CUDA_CHECK(cudaStreamSynchronize(ix.stream));
            CUDA_CHECK(cudaMemcpy(offsets, ix.csr_off.p, (ix.cur + 1) * 8, cudaMemcpyDeviceToHost));
            if (ix.csr_entries)
                CUDA_CHECK(cudaMemcpy(entries, ix.csr_ent.p, ix.csr_entries * (ix.wide ? 8 : 4),
                                      cudaMemcpyDeviceToHost));
        }
    });
}

hrnn_status hrnn_l2_batch(const float* a, const float* b, size_t n, size_t dim, int lanes, int fused, float* out) {
    return guard([&] {
        need(a, "a");
        need(b, "b");
        need(out, "out");
        if (lanes != 16 && lanes != 8 && lanes != 4) hrnn::fail(HRNN_ERR_ARG, "lanes must be 16, 8 or 4");
        hrnn::DevMem da, db, dout;
        da.alloc(n * dim * 4);
        db.alloc(n * dim * 4);
        dout.alloc(n * 4);
        CUDA_CHECK(cudaMemcpy(da.p, a, n * dim * 4, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(db.p, b, n * dim * 4, cudaMemcpyHostToDevice));
        hrnn::L2Order o;
        o.lanes = lanes;
        o.fused = fused;
        hrnn::l2_batch_device(da.as<float>(), db.as<float>(), n, dim, o, dout.as<float>(), nullptr);
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaMemcpy(out, dout.p, n * 4, cudaMemcpyDeviceToHost));
    });
}

}  // extern "C"
