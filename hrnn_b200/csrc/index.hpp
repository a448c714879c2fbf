// Index state of the B200-native HRNN: header fields with the reference's names
// (include/hnswlib/hrnn.h:31-112) and the device structure-of-arrays that the
// kernels read.  The reference keeps one AoS record per element
// ([links0 | KNN slot | vector | label], hrnn.h:160-177); here each field is its
// own HBM array so that vectors are 16-byte aligned rows and neighbour lists are
// contiguous.  The .idx reader/writer converts between the two byte-exactly.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace hrnn {

struct Budget;  // mlp.hpp

// Owning device allocation.
struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    void alloc(size_t n) {
        release();
        if (n == 0) n = 16;
        CUDA_CHECK(cudaMalloc(&p, n));
        bytes = n;
    }
    // Grows to at least n bytes; content is not preserved.
    void ensure(size_t n) {
        if (bytes < n) alloc(n);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Per-search counters accumulated on the device (see hrnn_search_stats).
struct SearchCounters {
    unsigned long long n_dist, n_expanded, n_posting, n_cand, n_verified, n_result;
    unsigned long long n_lowp, n_fp32, n_fp64, n_flip, overflow;
};

// Device mutable reverse lists (rknng_mutable.cu): element i's owners in
// ent[off[i] .. off[i] + len[i]), cap[i] slots.
struct MutableLists {
    DevMem off, len, cap, ent;
    DevMem ops, ctl;                          // pending edits; ctl: edit count (u64), flags
    DevMem ocnt, ocur, ooff, grouped, tmp;    // grouping work space
    unsigned long long ops_cap = 0;
    uint32_t slack_shift = 0;                 // capacities doubled after an overflow
    bool valid = false;
    uint64_t rebuilds = 0, applied = 0;
};

// Work space of the streaming INT8 verification (verify_stream.cu), reserved
// for a batch shape.
struct StreamBufs {
    DevMem qq, qmeta;      // the queries' INT8 copies and their scalars
    DevMem cnt, coff;      // chunks per (query, proxy) pair and their prefix sum
    DevMem chunks;         // work items
    DevMem acc_cnt;        // acceptances per query
    DevMem ctl;            // work counter
    DevMem tmp;            // scan scratch
    size_t npairs = 0;
    void reserve(uint32_t nq, uint32_t dim, size_t npairs, size_t max_chunks);
};

struct Index {
    // ---- device / stream -------------------------------------------------
    int device = 0;
    cudaStream_t stream = nullptr;
    L2Order order;
    int precision = HRNN_PREC_FP32_EXACT;
    bool autotune = true;                                   // hrnn_set_autotune
    std::unordered_map<uint64_t, std::pair<uint32_t, uint32_t>> a_shape;  // (mode, beam) -> (warps/block, slots)
    uint64_t generation = 0;  // bumped by every call that changes the index (captured plans check it)
    int join_mode = 0;  // refineKNNG local join (HRNN_JOIN_EXACT; HRNN_JOIN_TENSOR screens on the tensor cores)

    // ---- header (hrnn.h names) -------------------------------------------
    size_t dim = 0, max_elements = 0, cur = 0;
    size_t M = 0, maxM = 0, maxM0 = 0, ef_construction = 0, ef = 10, K = 0;
    size_t size_links_level0 = 0, size_links_per_element = 0, size_knng_slot = 0;
    size_t offsetKNNG = 0, offsetData = 0, label_offset = 0, size_data_per_element = 0;
    size_t offsetLevel0 = 0;
    double mult = 0.0;
    int maxlevel = -1;
    uint32_t enterpoint = kInvalid;
    bool knng_built = false, rknng_built = false;
    std::default_random_engine level_generator;
    std::unordered_map<uint64_t, uint32_t> label_lookup;

    // ---- element levels and upper layers (host-authoritative, mirrored) --
    std::vector<int32_t> levels;          // per element
    std::vector<uint64_t> upper_off;      // word offset of level-1 block
    std::vector<uint32_t> upper;          // flat (1+maxM)-word blocks
    bool upper_dirty = true;              // host copy newer than the device one

    // ---- device arrays (capacity max_elements) ---------------------------
    DevMem vec;        // f32 [cap][dim]
    DevMem vec_bf16;   // bf16 [cap][dim] (mixed-precision search), built on demand
    DevMem vec_norm;   // f32 [cap]: ||x||, mixed-precision error bounds
    bool bf16_valid = false;
    DevMem vec_i8;     // int8 [cap][dim]: round(x / s), s = max|x| / 127 (INT8 beam), built on demand
    DevMem i8_meta;    // float4 [cap]: s, ||x - s c||_2 rounded up, sum c^2, 0
    bool i8_valid = false;
    DevMem adj0;       // u32 [cap][1+maxM0]: raw level-0 link words
    DevMem knn_hdr;    // u32 [cap]: raw KNN-slot count word (count in low 16 bits)
    DevMem knn_ids;    // u32 [cap][K]
    DevMem knn_dist;   // f32 [cap][K]
    DevMem labels;     // u64 [cap]
    DevMem d_upper;    // u32 mirror of `upper`
    DevMem d_upper_off;// u64 mirror of `upper_off`

    // ---- reverse CSR ------------------------------------------------------
    DevMem csr_off;    // u64 [n+1]
    DevMem csr_ent;    // u32 or u64 [entries]
    size_t csr_entries = 0;
    uint32_t rank_bits = 0;
    bool wide = false;
    bool csr_in_reference_order = false;  // loaded from a reference .idx

    // ---- buildRKNNG_mutable / insertPointDynamic: the reverse lists are the
    // CSR above, rebuilt after each batch of inserts (so they are exact).
    bool rknng_mutable = false;
    MutableLists mr;          // the reverse lists insertPointDynamic reads and edits
    bool csr_stale = false;   // the flat CSR predates inserts: rebuilt before its next use
    hrnn_dynamic_stats dyn_stats{};

    // ---- serve mode (compactForServing, hrnn.h:299-364) -------------------
    bool serve_mode = false;
    size_t max_k_serve = 0;
    DevMem kdist_serve;  // f32 [n][max_k_serve]

    // ---- scratch reused across calls ---------------------------------------
    DevMem scratch[10];
    // a second stream and two events: the learned budget's second search runs
    // beside the verification of the queries it does not concern
    cudaStream_t aux = nullptr;
    cudaEvent_t aux_ev[2] = {nullptr, nullptr};
    DevMem io;           // host-buffer entry points stage their inputs/outputs here
    DevMem counters;     // SearchCounters
    DevMem kcol;         // f32 [n]: kdist(p, k-1) of the current search call
    StreamBufs sb;       // streaming verification of the INT8 form
    hrnn_search_stats last_stats{};
    hrnn_refine_stats refine_stats{};
    std::unique_ptr<Budget> budget;  // learned search budget (hrnn_set_budget)

    Index();
    ~Index();

    size_t n() const { return cur; }
    void sync_upper_to_device();
    size_t device_bytes() const;
};

// index.cpp
void init_layout(Index& ix, size_t dim, size_t max_elements, size_t M, size_t efc,
                 size_t seed, size_t K);
void alloc_device(Index& ix, size_t capacity);
void load_idx(Index& ix, const std::string& path, size_t dim, size_t max_elements);
void save_idx(Index& ix, const std::string& path);
void get_knng(Index& ix, uint32_t* ids, float* dists, uint32_t* cnt);
void set_knng(Index& ix, const uint32_t* ids, const float* dists, const uint32_t* cnt);
void compact_for_serving(Index& ix, size_t max_k_serve);
L2Order detect_l2_order();

// csr.cu
void build_rknng(Index& ix);
void rknng_reference_order(Index& ix, uint64_t* offsets, void* entries);
void build_rknng_mutable(Index& ix);
void ensure_flat_rknng(Index& ix);  // rebuilds the flat CSR when inserts made it stale

// rknng_mutable.cu
void mutable_build(Index& ix);
void mutable_ops_reserve(Index& ix, unsigned long long cap);
void mutable_register(Index& ix, uint32_t x0, uint32_t nx);
void mutable_apply(Index& ix);
void mutable_get(Index& ix, uint64_t* lens, uint32_t* flat);

// search.cu
struct SearchArgs {
    const float* d_q;
    size_t nq;
    const uint32_t* d_m;
    const uint32_t* d_Kp;
    const uint32_t* d_ef;
    float threshold;
    uint32_t k;
    uint64_t* d_out_offsets;
    uint64_t* d_out_labels;
    size_t cap;
    cudaStream_t stream;
    // the batch's largest m and max(ef, m) when the caller knows them (host
    // inputs); 0: read back from d_m / d_ef
    uint32_t h_mmax = 0, h_efmax = 0;
};
uint64_t search_batch(Index& ix, const SearchArgs& a);  // returns total results
void kdist_column(Index& ix, uint32_t k, float* host_out);  // kdist(p, k-1) of every element
void l2_batch_device(const float* a, const float* b, size_t n, size_t dim, L2Order o, float* out,
                     cudaStream_t s);

// nndescent.cu
void refine_knng(Index& ix, int iters, int sample);

// hnsw_build.cu
void add_points(Index& ix, const float* data, const uint64_t* labels, size_t n);

// dynamic.cu
void insert_dynamic(Index& ix, const float* data, const uint64_t* labels, size_t n,
                    unsigned m_update, bool bidirectional);

// scan.cu: exclusive prefix sums on the device
void exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t s,
                        DevMem& tmp);
void exclusive_scan_u32_to_u64(const uint32_t* in, uint64_t* out, size_t n, cudaStream_t s,
                               DevMem& tmp);

}  // namespace hrnn
