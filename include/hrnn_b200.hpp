// C++ face of the C ABI with the member names of the reference's
// hnswlib::HRNN<float> (include/hnswlib/hrnn.h), so that code written against the
// reference -- its three drivers in particular -- compiles against this library
// unchanged: the same constructors, addPoint / refineKNNG / buildRKNNG /
// buildRKNNG_mutable / saveIndex / searchRknn / insertPointDynamic /
// compactForServing / setEf / getCurrentElementCount, and the public fields
// K_knng_, knng_built_ and rknng_built_.  Failures throw std::runtime_error with
// the reference's message.
//
// The GPU wants batches: addPoint and insertPointDynamic queue their points
// (thread-safe, so an OpenMP insert loop works as written) and the queue goes to
// the device as one batch on the next call of any other member, or when it
// reaches kQueueLimit points.  The ids these calls return are the internal ids
// the points receive (insertion order of the queue).  searchRknnBatch is the
// batched form of searchRknn (one call for many queries, uneven parameters).
#ifndef HRNN_B200_HPP
#define HRNN_B200_HPP

#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "hrnn_capi.h"

namespace hrnn_b200 {

inline void check(hrnn_status s) {
    if (s != HRNN_OK) throw std::runtime_error(hrnn_last_error());
}

}  // namespace hrnn_b200

namespace hnswlib {

typedef size_t labeltype;      // hnswlib.h:125
typedef unsigned int tableint;

template <typename dist_t>
class SpaceInterface {
public:
    virtual ~SpaceInterface() = default;
    virtual size_t get_data_size() = 0;
    virtual void* get_dist_func_param() = 0;
};

// Squared L2 over float vectors (space_l2.h); the device computes it.
class L2Space : public SpaceInterface<float> {
    size_t dim_;

public:
    explicit L2Space(size_t dim) : dim_(dim) {}
    size_t get_data_size() override { return dim_ * sizeof(float); }
    void* get_dist_func_param() override { return &dim_; }
    size_t dim() const { return dim_; }
};

template <typename dist_t>
class HRNN {
    static_assert(sizeof(dist_t) == 4, "the device index stores float distances");

public:
    static constexpr size_t kQueueLimit = 1u << 20;

    // Public fields of the reference (hrnn.h:83-91), refreshed after every call.
    mutable size_t K_knng_ = 0;
    mutable bool knng_built_ = false;
    mutable bool rknng_built_ = false;

    // HRNN(space, max_elements, M, ef_construction, random_seed,
    //      allow_replace_deleted, K_knng) -- hrnn.h:128
    HRNN(SpaceInterface<dist_t>* s, size_t max_elements, size_t M = 16, size_t ef_construction = 200,
         size_t random_seed = 100, bool allow_replace_deleted = false, size_t K_knng = 0, int device = 0)
        : dim_(*static_cast<size_t*>(s->get_dist_func_param())) {
        if (allow_replace_deleted) throw std::runtime_error("HRNN: replacement of deleted elements is not supported");
        hrnn_b200::check(hrnn_create(&h_, dim_, max_elements, M, ef_construction, random_seed, K_knng, device));
        refresh();
    }

    // HRNN(space, location, nmslib, max_elements) -- hrnn.h:117 (loadIndex)
    HRNN(SpaceInterface<dist_t>* s, const std::string& location, bool nmslib = false, size_t max_elements = 0,
         int device = 0)
        : dim_(*static_cast<size_t*>(s->get_dist_func_param())) {
        if (nmslib) throw std::runtime_error("HRNN: nmslib-format indices are not supported");
        hrnn_b200::check(hrnn_load(&h_, location.c_str(), dim_, max_elements, device));
        refresh();
    }

    ~HRNN() { hrnn_destroy(h_); }
    HRNN(const HRNN&) = delete;
    HRNN& operator=(const HRNN&) = delete;

    // addPoint(data_point, label) -- hrnn.h:1179 (queued)
    tableint addPoint(const void* data_point, labeltype label, int level = -1) {
        if (level != -1) throw std::runtime_error("addPoint: an explicit level is not supported");
        std::lock_guard<std::mutex> lk(mu_);
        if (!dyn_lab_.empty()) flush_locked();
        const tableint id = (tableint)(count_locked() + add_lab_.size());
        push(add_data_, add_lab_, data_point, label);
        if (add_lab_.size() >= kQueueLimit) flush_locked();
        return id;
    }

    // insertPointDynamic(data_point, label, m_update, bidirectional) -- hrnn.h:2360 (queued)
    tableint insertPointDynamic(const void* data_point, labeltype label, unsigned m_update = 0,
                                bool bidirectional = false) {
        std::lock_guard<std::mutex> lk(mu_);
        if (!add_lab_.empty() || (!dyn_lab_.empty() && (m_update != dyn_m_ || bidirectional != dyn_bidir_)))
            flush_locked();
        dyn_m_ = m_update;
        dyn_bidir_ = bidirectional;
        const tableint id = (tableint)(count_locked() + dyn_lab_.size());
        push(dyn_data_, dyn_lab_, data_point, label);
        if (dyn_lab_.size() >= kQueueLimit) flush_locked();
        return id;
    }

    void refineKNNG(int num_iters = 3, int sample_size = 20) { call([&] { return hrnn_refine_knng(h_, num_iters, sample_size); }); }
    void buildRKNNG() { call([&] { return hrnn_build_rknng(h_); }); }
    void buildRKNNG_mutable() { call([&] { return hrnn_build_rknng_mutable(h_); }); }
    void saveIndex(const std::string& location) { call([&] { return hrnn_save(h_, location.c_str()); }); }
    void compactForServing(size_t max_k_serve) { call([&] { return hrnn_compact_for_serving(h_, max_k_serve); }); }
    void setEf(size_t ef) { call([&] { return hrnn_set_ef(h_, ef); }); }

    size_t getCurrentElementCount() const {
        std::lock_guard<std::mutex> lk(mu_);
        flush_locked();
        return count_locked();
    }

    // searchRknn(query, m, threshold, k, K_prime, ef_search) -- hrnn.h:1966; labels in
    // ascending internal-id order, as the reference returns them.
    std::vector<labeltype> searchRknn(const void* query, size_t m, float threshold, size_t k, size_t K_prime,
                                      size_t ef_search) const {
        const uint32_t mm = (uint32_t)m, kp = (uint32_t)K_prime, ee = (uint32_t)ef_search;
        return searchRknnBatch(static_cast<const float*>(query), 1, &mm, &kp, &ee, threshold, k, true).at(0);
    }

    // Batched searchRknn: nq queries, one (m, K', ef_search) per query (`uniform`:
    // the first entry for all).  Host buffers in and out.
    std::vector<std::vector<labeltype>> searchRknnBatch(const float* queries, size_t nq, const uint32_t* m,
                                                        const uint32_t* K_prime, const uint32_t* ef_search,
                                                        float threshold, size_t k, bool uniform = false) const {
        {
            std::lock_guard<std::mutex> lk(mu_);
            flush_locked();
        }
        std::vector<uint32_t> mv, kv, ev;
        if (uniform) {
            mv.assign(nq, m[0]);
            kv.assign(nq, K_prime[0]);
            ev.assign(nq, ef_search[0]);
            m = mv.data();
            K_prime = kv.data();
            ef_search = ev.data();
        }
        std::vector<uint64_t> off(nq + 1, 0), lab;
        size_t cap = 64 * nq + 64;
        lab.resize(cap);
        hrnn_status st = hrnn_search_rknn_batch(h_, queries, nq, m, K_prime, ef_search, threshold, (uint32_t)k,
                                                off.data(), lab.data(), cap);
        if (st == HRNN_ERR_CAPACITY) {
            cap = (size_t)off[nq];
            lab.resize(cap);
            st = hrnn_search_rknn_batch(h_, queries, nq, m, K_prime, ef_search, threshold, (uint32_t)k, off.data(),
                                        lab.data(), cap);
        }
        hrnn_b200::check(st);
        std::vector<std::vector<labeltype>> out(nq);
        for (size_t i = 0; i < nq; ++i) out[i].assign(lab.begin() + (ptrdiff_t)off[i], lab.begin() + (ptrdiff_t)off[i + 1]);
        return out;
    }

    // Precision of the search (HRNN_PREC_FP32_EXACT: the reference's answers;
    // HRNN_PREC_BF16: the mixed-precision form with exact decisions).
    void setPrecision(int precision) { call([&] { return hrnn_set_precision(h_, precision); }); }
    // Local join of refineKNNG (HRNN_JOIN_EXACT, HRNN_JOIN_TENSOR, HRNN_JOIN_AUDIT).
    void setJoinMode(int mode) { call([&] { return hrnn_set_join_mode(h_, mode); }); }
    // Launch-shape autotuning of the batch search (on by default).
    void setAutotune(bool enable) { call([&] { return hrnn_set_autotune(h_, enable ? 1 : 0); }); }

    hrnn_index* handle() {
        std::lock_guard<std::mutex> lk(mu_);
        flush_locked();
        return h_;
    }

private:
    template <class F>
    void call(F&& f) {
        std::lock_guard<std::mutex> lk(mu_);
        flush_locked();
        hrnn_b200::check(f());
        refresh();
    }

    void push(std::vector<float>& data, std::vector<uint64_t>& lab, const void* x, labeltype label) {
        const float* v = static_cast<const float*>(x);
        data.insert(data.end(), v, v + dim_);
        lab.push_back((uint64_t)label);
    }

    size_t count_locked() const {
        hrnn_info inf;
        hrnn_b200::check(hrnn_get_info(h_, &inf));
        return (size_t)inf.cur_element_count;
    }

    void flush_locked() const {
        if (!add_lab_.empty()) {
            hrnn_status st = hrnn_add_points(h_, add_data_.data(), add_lab_.data(), add_lab_.size());
            add_data_.clear();
            add_lab_.clear();
            hrnn_b200::check(st);
        }
        if (!dyn_lab_.empty()) {
            hrnn_status st = hrnn_insert_dynamic(h_, dyn_data_.data(), dyn_lab_.data(), dyn_lab_.size(), dyn_m_,
                                                 dyn_bidir_ ? 1 : 0);
            dyn_data_.clear();
            dyn_lab_.clear();
            hrnn_b200::check(st);
        }
        refresh();
    }

    void refresh() const {
        hrnn_info inf;
        if (hrnn_get_info(h_, &inf) != HRNN_OK) return;
        K_knng_ = (size_t)inf.K_knng;
        knng_built_ = inf.knng_built != 0;
        rknng_built_ = inf.rknng_built != 0;
    }

    size_t dim_;
    hrnn_index* h_ = nullptr;
    mutable std::mutex mu_;
    mutable std::vector<float> add_data_, dyn_data_;
    mutable std::vector<uint64_t> add_lab_, dyn_lab_;
    mutable unsigned dyn_m_ = 0;
    mutable bool dyn_bidir_ = false;
};

}  // namespace hnswlib

#endif  // HRNN_B200_HPP
