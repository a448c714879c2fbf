// Test-infrastructure harness around the REFERENCE implementation.
//
// This file is part of the oracle (a checker), never of the product path.
// It is compiled by oracle/Makefile together with the reference's own header
// `include/hnswlib/hrnn.h` (read in place from the reference tree) into
// oracle/_ref/libhrnn_ref.so, and exposes a flat extern "C" surface so that the
// tests and the CPU-baseline leg of bench.py can drive the reference's code:
//
//   ref_create        -> HRNN(space, max_elements, M, ef_c, seed, false, K)  hrnn.h:128
//   ref_add_points    -> addPoint loop as in src/hrnn_build.cpp:75-88
//   ref_refine        -> refineKNNG(iters, sample)                           hrnn.h:1725
//   ref_build_rknng   -> buildRKNNG()                                        hrnn.h:1869
//   ref_build_mutable -> buildRKNNG_mutable()                                hrnn.h:1942
//   ref_insert_dynamic-> insertPointDynamic(x, label, m_update, bidir)       hrnn.h:2360
//   ref_save / ref_load -> saveIndex / HRNN(space, path, false, max_elems)   hrnn.h:861, 117
//   ref_search_batch  -> searchRknn per query (src/hrnn_search.cpp:168-180)  hrnn.h:1966
//   ref_compact       -> compactForServing(max_k_serve)                      hrnn.h:299
//   ref_l2            -> L2Space(d).get_dist_func()                          space_l2.h:214
//
// No code of the reference is copied here; the header is #included.
#include "hnswlib/hrnn.h"

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct RefHandle {
    std::unique_ptr<hnswlib::L2Space> space;
    std::unique_ptr<hnswlib::HRNN<float>> index;
    size_t dim = 0;
    std::string err;
};

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

void* ref_create(size_t dim, size_t max_elements, size_t M, size_t ef_c, size_t seed, size_t K) {
    auto* h = new RefHandle();
    h->dim = dim;
    h->space.reset(new hnswlib::L2Space(dim));
    h->index.reset(new hnswlib::HRNN<float>(h->space.get(), max_elements, M, ef_c, seed, false, K));
    return h;
}

void* ref_load(const char* path, size_t dim, size_t max_elements) {
    auto* h = new RefHandle();
    h->dim = dim;
    h->space.reset(new hnswlib::L2Space(dim));
    int rc = guard([&] {
        h->index.reset(new hnswlib::HRNN<float>(h->space.get(), std::string(path), false, max_elements));
    });
    if (rc) {
        delete h;
        return nullptr;
    }
    return h;
}

void ref_free(void* p) { delete static_cast<RefHandle*>(p); }

// Inserts n points.  threads == 1 gives the deterministic serial build; threads > 1
// mirrors the driver's `omp parallel for schedule(dynamic, 512)` loop.
int ref_add_points(void* p, const float* X, size_t n, const uint64_t* labels, int threads) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] {
        if (threads <= 1) {
            for (size_t i = 0; i < n; ++i)
                h->index->addPoint(X + i * h->dim, (hnswlib::labeltype)labels[i]);
            return;
        }
        set_threads(threads);
        std::string first_err;
#pragma omp parallel for schedule(dynamic, 512)
        for (long long i = 0; i < (long long)n; ++i) {
            try {
                h->index->addPoint(X + (size_t)i * h->dim, (hnswlib::labeltype)labels[i]);
            } catch (const std::exception& e) {
#pragma omp critical
                first_err = e.what();
            }
        }
        if (!first_err.empty()) throw std::runtime_error(first_err);
    });
}

int ref_refine(void* p, int iters, int sample, int threads) {
    auto* h = static_cast<RefHandle*>(p);
    set_threads(threads);
    return guard([&] { h->index->refineKNNG(iters, sample); });
}

int ref_build_rknng(void* p) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] { h->index->buildRKNNG(); });
}

int ref_build_mutable(void* p) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] { h->index->buildRKNNG_mutable(); });
}

int ref_insert_dynamic(void* p, const float* X, size_t n, const uint64_t* labels,
                       unsigned m_update, int bidirectional, int threads) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] {
        set_threads(threads);
        std::string first_err;
#pragma omp parallel for schedule(dynamic, 64) if (threads > 1)
        for (long long i = 0; i < (long long)n; ++i) {
            try {
                h->index->insertPointDynamic(X + (size_t)i * h->dim, (hnswlib::labeltype)labels[i],
                                             m_update, bidirectional != 0);
            } catch (const std::exception& e) {
#pragma omp critical
                first_err = e.what();
            }
        }
        if (!first_err.empty()) throw std::runtime_error(first_err);
    });
}

int ref_save(void* p, const char* path) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] { h->index->saveIndex(std::string(path)); });
}

int ref_compact(void* p, size_t max_k_serve) {
    auto* h = static_cast<RefHandle*>(p);
    return guard([&] { h->index->compactForServing(max_k_serve); });
}

size_t ref_count(void* p) { return static_cast<RefHandle*>(p)->index->getCurrentElementCount(); }

// Runs searchRknn for nq queries with per-query (m, K', ef).  Results go to
// out_labels in query order; out_offsets has nq+1 entries.  Returns 0 on success,
// 2 if the output capacity is too small (out_offsets[nq] then holds the need).
// threads > 1 runs queries in parallel (searchRknn is const and thread-safe);
// *seconds receives the wall time of the query loop.
int ref_search_batch(void* p, const float* Q, size_t nq, const uint32_t* m, const uint32_t* Kp,
                     const uint32_t* ef, float threshold, uint32_t k, uint64_t* out_offsets,
                     uint64_t* out_labels, size_t cap, int threads, double* seconds) {
    auto* h = static_cast<RefHandle*>(p);
    std::vector<std::vector<hnswlib::labeltype>> res(nq);
    int rc = guard([&] {
        set_threads(threads);
        auto t0 = std::chrono::steady_clock::now();
        std::string first_err;
#pragma omp parallel for schedule(dynamic, 16) if (threads > 1)
        for (long long q = 0; q < (long long)nq; ++q) {
            try {
                res[q] = h->index->searchRknn(Q + (size_t)q * h->dim, m[q], threshold, k, Kp[q], ef[q]);
            } catch (const std::exception& e) {
#pragma omp critical
                first_err = e.what();
            }
        }
        auto t1 = std::chrono::steady_clock::now();
        if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
        if (!first_err.empty()) throw std::runtime_error(first_err);
    });
    if (rc) return rc;
    uint64_t total = 0;
    out_offsets[0] = 0;
    for (size_t q = 0; q < nq; ++q) {
        total += res[q].size();
        out_offsets[q + 1] = total;
    }
    if (total > cap) return 2;
    for (size_t q = 0; q < nq; ++q)
        std::memcpy(out_labels + out_offsets[q], res[q].data(), res[q].size() * sizeof(uint64_t));
    return 0;
}

float ref_l2(const float* a, const float* b, size_t dim) {
    hnswlib::L2Space sp(dim);
    auto f = sp.get_dist_func();
    return f(a, b, sp.get_dist_func_param());
}

// Batch of distances a[i] vs b[i] (n pairs of dim floats each).
void ref_l2_batch(const float* a, const float* b, size_t n, size_t dim, float* out) {
    hnswlib::L2Space sp(dim);
    auto f = sp.get_dist_func();
    for (size_t i = 0; i < n; ++i) out[i] = f(a + i * dim, b + i * dim, sp.get_dist_func_param());
}

// Copies the KNN-graph slot of every element: ids/dists are n x K, cnt is n.
void ref_get_knng(void* p, uint32_t* ids, float* dists, uint32_t* cnt) {
    auto* h = static_cast<RefHandle*>(p);
    auto& ix = *h->index;
    size_t n = ix.getCurrentElementCount();
    size_t K = ix.K_knng_;
    for (size_t i = 0; i < n; ++i) {
        unsigned c = ix.getListCount(ix.get_knng_linklist((hnswlib::tableint)i));
        cnt[i] = c;
        for (size_t j = 0; j < K; ++j) {
            ids[i * K + j] = ix.get_knng_neighbor((hnswlib::tableint)i, (unsigned)j);
            dists[i * K + j] = ix.get_knng_dist((hnswlib::tableint)i, (unsigned)j);
        }
    }
}

// Overwrites the KNN-graph slot of every element (used to start the reference's
// refinement from a given graph).
void ref_set_knng(void* p, const uint32_t* ids, const float* dists, const uint32_t* cnt) {
    auto* h = static_cast<RefHandle*>(p);
    auto& ix = *h->index;
    size_t n = ix.getCurrentElementCount();
    size_t K = ix.K_knng_;
    for (size_t i = 0; i < n; ++i) {
        auto* ll = ix.get_knng_linklist((hnswlib::tableint)i);
        ix.setListCount(ll, (unsigned short)cnt[i]);
        char* base = (char*)(ll + 1);
        for (size_t j = 0; j < K; ++j) {
            std::memcpy(base + j * 8, &ids[i * K + j], 4);
            std::memcpy(base + j * 8 + 4, &dists[i * K + j], 4);
        }
    }
}

// CSR of the reverse KNN graph: sizes first (call with null arrays), then data.
int ref_get_csr(void* p, uint64_t* n_offsets, uint64_t* n_entries, uint32_t* entry_bytes,
                uint32_t* rank_bits, uint64_t* offsets, void* entries) {
    auto* h = static_cast<RefHandle*>(p);
    auto& ix = *h->index;
    if (!ix.rknng_built_) return 1;
    *n_offsets = ix.rknng_offsets_.size();
    *entry_bytes = ix.rknng_wide_ ? 8 : 4;
    *rank_bits = ix.rknng_rank_bits_;
    *n_entries = ix.rknng_wide_ ? ix.rknng_entries_64_.size() : ix.rknng_entries_32_.size();
    if (offsets) std::memcpy(offsets, ix.rknng_offsets_.data(), *n_offsets * 8);
    if (entries) {
        if (ix.rknng_wide_)
            std::memcpy(entries, ix.rknng_entries_64_.data(), *n_entries * 8);
        else
            std::memcpy(entries, ix.rknng_entries_32_.data(), *n_entries * 4);
    }
    return 0;
}

// Mutable reverse lists (buildRKNNG_mutable / insertPointDynamic): lengths, then data.
void ref_get_mutable(void* p, uint64_t* lens, uint32_t* flat) {
    auto* h = static_cast<RefHandle*>(p);
    auto& L = h->index->rknng_lists_;
    size_t n = h->index->getCurrentElementCount();
    size_t pos = 0;
    for (size_t i = 0; i < n; ++i) {
        lens[i] = i < L.size() ? L[i].size() : 0;
        if (flat && i < L.size()) {
            std::memcpy(flat + pos, L[i].data(), L[i].size() * 4);
            pos += L[i].size();
        }
    }
}

}  // extern "C"
