/* hrnn_b200 -- C ABI of the B200-native HRNN hot path.
 *
 * This is the drop-in boundary.  Every entry point replaces one member of the
 * reference's `hnswlib::HRNN<float>` (include/hnswlib/hrnn.h) that the three
 * reference drivers call (src/hrnn_build.cpp:67-109, src/hrnn_search.cpp:137-178,
 * src/hrnn_dynamic_test.cpp:224-393); the citation is on each declaration.
 *
 * Conventions
 *  - Plain pointers and sizes only; no exceptions cross this boundary.
 *  - Every call returns an hrnn_status (0 = HRNN_OK).  On failure the message of
 *    the reference's std::runtime_error for the same condition (for example
 *    "searchRknn: RKNNG not built", "Not an HRNN index file (bad magic)") is
 *    available from hrnn_last_error() on the calling thread.
 *  - Pointers named `d_*` are device pointers; all others are host pointers.
 *  - `stream` is a cudaStream_t passed as void* (NULL = the handle's stream).
 *    Calls on one handle must not overlap; use one handle per stream.
 *  - Internal ids are assigned in insertion order; labels are the caller's u64
 *    labels (labeltype = size_t, hnswlib.h:125).
 */
#ifndef HRNN_CAPI_H
#define HRNN_CAPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int hrnn_status;
#define HRNN_OK 0
#define HRNN_ERR_ARG 1      /* invalid argument                                   */
#define HRNN_ERR_STATE 2    /* call not valid in the index's state                */
#define HRNN_ERR_IO 3       /* file cannot be opened / read / written             */
#define HRNN_ERR_FORMAT 4   /* not an HRNN .idx file, or a truncated one          */
#define HRNN_ERR_CUDA 5     /* CUDA runtime error                                 */
#define HRNN_ERR_NOMEM 6    /* device or host allocation failed                   */
#define HRNN_ERR_CAPACITY 7 /* caller's output buffer too small (size reported)   */
#define HRNN_ERR_LIMIT 8    /* element count exceeds max_elements                 */
#define HRNN_ERR_TIMEOUT 9  /* a bounded device-side wait expired                 */

typedef struct hrnn_index hrnn_index;

/* Summary of an index (public fields and getters of HRNN<float>). */
typedef struct {
    uint64_t dim, max_elements, cur_element_count;   /* getCurrentElementCount hrnn.h:393 */
    uint64_t M, maxM, maxM0, ef_construction, ef;    /* hrnn.h:38-42, setEf hrnn.h:226     */
    uint64_t K_knng;                                 /* K_knng_ hrnn.h:83                  */
    int32_t maxlevel;
    uint32_t enterpoint;
    int32_t knng_built, rknng_built, rknng_wide;    /* hrnn.h:86-87, 91                   */
    uint32_t rank_bits;                              /* hrnn.h:93                          */
    uint64_t rknng_entries;
    int32_t serve_mode;                              /* compactForServing hrnn.h:109       */
    uint64_t max_k_serve;
    int32_t l2_lanes, l2_fused;                      /* FP32 summation order in use        */
    uint64_t device_bytes;                           /* HBM held by the index              */
} hrnn_info;

/* Per-call counters of the last search (RknnProfile, hrnn.h:2077-2084, plus the
 * work counts the roofline is computed from). */
typedef struct {
    uint64_t n_queries;
    uint64_t n_dist;        /* FP32 distance evaluations, phase A              */
    uint64_t n_expanded;    /* base-layer nodes expanded, phase A              */
    uint64_t n_posting;     /* reverse-list entries read, phase B              */
    uint64_t n_cand;        /* distinct candidates after phase B               */
    uint64_t n_verified;    /* candidates passing the score threshold          */
    uint64_t n_result;      /* accepted points                                 */
    uint64_t n_lowp_decided;/* mixed precision: decided by the low-precision bound */
    uint64_t n_fp32_decided;/* mixed precision: re-decided in exact FP32        */
    uint64_t n_fp64_decided;/* mixed precision: re-decided in FP64 (tie band)   */
    uint64_t n_fp64_flipped;/* ... of which FP64 decided against FP32           */
    uint64_t n_launches;    /* kernels this call launched                       */
    uint64_t n_budget[3];   /* learned budget: queries at level 0, 1, fallback */
    double phase_a_ms, phase_b_ms, phase_c_ms;   /* device time of each phase   */
    uint32_t a_warps_per_block, a_visit_slots;   /* phase-A launch shape used (autotuned) */
} hrnn_search_stats;

/* Per-iteration counters of the last refineKNNG call (the reference prints the
 * updates and distance counts per iteration, hrnn.h:1855-1859). */
#define HRNN_MAX_ITERS 64
typedef struct {
    int32_t iters;
    uint64_t join_dists[HRNN_MAX_ITERS];     /* pair distances of the local join     */
    uint64_t updates[HRNN_MAX_ITERS];        /* entries inserted into lists          */
    uint64_t proposals[HRNN_MAX_ITERS];      /* proposals that passed the bound      */
    uint64_t sample_entries[HRNN_MAX_ITERS]; /* sum over nodes of |new| + |old|      */
    double ms[HRNN_MAX_ITERS];               /* device time of the iteration         */
    double sample_ms[HRNN_MAX_ITERS];        /* ... of which sampling (phase 1)      */
    double join_ms[HRNN_MAX_ITERS];          /* ... local joins                      */
    double bucket_ms[HRNN_MAX_ITERS];        /* ... grouping proposals by target     */
    double merge_ms[HRNN_MAX_ITERS];         /* ... list merges                      */
    uint64_t screen_survivors[HRNN_MAX_ITERS];   /* tensor-core join: pairs given exact FP32 */
    uint64_t screen_dense_nodes[HRNN_MAX_ITERS]; /* ... nodes joined densely (list overflow) */
    uint64_t screen_misses[HRNN_MAX_ITERS];      /* ... audit mode: proposals the screen
                                                    would have dropped (0 when the bound holds) */
    int32_t join_mode;                           /* join mode the last call ran          */
} hrnn_refine_stats;

/* The split of src/hrnn_dynamic_test.cpp:200-203: perm[0..n) = 0..n-1 shuffled by
 * std::shuffle with std::mt19937(seed) (seed 42 there) -- the first split*n
 * entries build the index, the rest are inserted.  std::shuffle's draw sequence
 * belongs to the C++ standard library, so the permutation is made by this
 * library's own libstdc++ rather than restated. */
hrnn_status hrnn_dynamic_split(uint64_t n, uint32_t seed, uint32_t* perm);

/* The mutable reverse lists of buildRKNNG_mutable (rknng_lists_, hrnn.h:1942-1959),
 * as insertPointDynamic maintains them on the device: lens[cur_element_count]
 * receives each list's length, flat the lists one after another (owner ids, in
 * no particular order, as the reference's per-node vectors).  Either may be NULL. */
hrnn_status hrnn_get_rknng_mutable(hrnn_index* h, uint64_t* lens, uint32_t* flat);

/* Counters of the last hrnn_insert_dynamic call. */
typedef struct {
    uint64_t n_inserted;     /* points added                                    */
    uint64_t n_batches;      /* insertion batches                               */
    uint64_t n_dist;         /* exact FP32 distances of the self-queries        */
    uint64_t n_proposals;    /* list updates proposed                           */
    uint64_t n_updates;      /* list entries inserted                           */
    double insert_ms;        /* HNSW insertion and KNN-graph seeds              */
    double rknng_ms;         /* reverse-list rebuilds                           */
    double maintain_ms;      /* self-queries and list merges                    */
} hrnn_dynamic_stats;

/* Thread-local message of the last failing call on this thread ("" if none). */
const char* hrnn_last_error(void);
/* ABI version (major*10000 + minor*100 + patch). */
int hrnn_version(void);

/* HRNN(space, max_elements, M, ef_construction, random_seed, false, K_knng)
 * -- hrnn.h:128-195.  device: CUDA ordinal. */
hrnn_status hrnn_create(hrnn_index** out, size_t dim, size_t max_elements, size_t M,
                        size_t ef_construction, size_t random_seed, size_t K_knng, int device);

/* HRNN(space, path, false, max_elements) -> loadIndex -- hrnn.h:117-124, 930-1047.
 * max_elements below the stored count keeps the stored capacity (hrnn.h:948-951). */
hrnn_status hrnn_load(hrnn_index** out, const char* path, size_t dim, size_t max_elements,
                      int device);

/* saveIndex -- hrnn.h:861-927.  Byte layout identical to the reference's. */
hrnn_status hrnn_save(hrnn_index* h, const char* path);

/* ~HRNN -- hrnn.h:198-214. */
void hrnn_destroy(hrnn_index* h);

/* The addPoint loop of src/hrnn_build.cpp:75-88 (addPoint hrnn.h:1179, 1378-1517):
 * HNSW insertion with the KNN-graph seed of hrnn.h:1479-1501, batched on the GPU.
 * data: n x dim host floats; labels: n host labels (NULL = 0..n-1 offset by the
 * current count). */
hrnn_status hrnn_add_points(hrnn_index* h, const float* data, const uint64_t* labels, size_t n);

/* refineKNNG(num_iters, sample_size) -- hrnn.h:1725-1862. */
hrnn_status hrnn_refine_knng(hrnn_index* h, int num_iters, int sample_size);

/* buildRKNNG() -- hrnn.h:1869-1935. */
hrnn_status hrnn_build_rknng(hrnn_index* h);

/* buildRKNNG_mutable() -- hrnn.h:1942-1959. */
hrnn_status hrnn_build_rknng_mutable(hrnn_index* h);

/* searchRknn(q, m, threshold, k, K_prime, ef_search) -- hrnn.h:1966-2071, one query,
 * host buffers.  Labels are written in ascending internal-id order, as the
 * reference returns them.  *out_count receives the result size; if it exceeds
 * cap, HRNN_ERR_CAPACITY is returned and nothing past cap is written. */
hrnn_status hrnn_search_rknn(hrnn_index* h, const float* query, size_t m, float threshold,
                             size_t k, size_t K_prime, size_t ef_search, uint64_t* out_labels,
                             size_t cap, size_t* out_count);

/* A batch of searchRknn calls (the query loop of src/hrnn_search.cpp:168-180) with
 * one (m, K', ef_search) per query, HOST buffers (copied in and out inside the
 * call).  out_offsets: nq+1 entries; query i's labels are
 * out_labels[out_offsets[i] .. out_offsets[i+1]).  On HRNN_ERR_CAPACITY,
 * out_offsets is filled and out_offsets[nq] is the capacity needed. */
hrnn_status hrnn_search_rknn_batch(hrnn_index* h, const float* queries, size_t nq,
                                   const uint32_t* m, const uint32_t* K_prime,
                                   const uint32_t* ef_search, float threshold, uint32_t k,
                                   uint64_t* out_offsets, uint64_t* out_labels, size_t cap);

/* Same with DEVICE buffers, stream-ordered (no host synchronisation except to
 * size scratch).  d_out_offsets: nq+1 device u64; *out_total (host) receives the
 * total result count. */
hrnn_status hrnn_search_rknn_batch_device(hrnn_index* h, const float* d_queries, size_t nq,
                                          const uint32_t* d_m, const uint32_t* d_K_prime,
                                          const uint32_t* d_ef_search, float threshold,
                                          uint32_t k, uint64_t* d_out_offsets,
                                          uint64_t* d_out_labels, size_t cap,
                                          uint64_t* out_total, void* stream);

/* Captured search plan (new; the reference answers one query per call).  The batch
 * search of hrnn_search_rknn_batch_device for one batch shape -- nq queries in
 * d_queries, per-query m / K' / ef_search in d_m / d_K_prime / d_ef_search, results
 * to d_out_offsets (nq + 1) and d_out_labels (cap) -- recorded once as a CUDA graph
 * and replayed by hrnn_search_plan_run with no host synchronisation inside: fill
 * the same input buffers, run, read the outputs.  The bounds a plan is made for:
 * m <= m_max and ef_search <= ef_max (larger values run clamped to them and are
 * reported by hrnn_search_plan_result), threshold and k fixed.  Staging is sized
 * for nq * m_max * (the index's longest reverse list) postings (HRNN_ERR_NOMEM
 * when that exceeds half the free device memory).  The precision form is the
 * index's at creation, and so is the learned budget when it is enabled (its
 * frontier pass, MLP, levels and second search are recorded with the budget's
 * settings and weights).  A plan is bound to the index as it was: any later call
 * that changes the index or those settings (add, refine, build, insert, compact,
 * set_knng, set_l2_order, set_precision, set_ef, set_budget, budget_train,
 * budget_set_weights) makes run fail with HRNN_ERR_STATE.  Answers equal
 * hrnn_search_rknn_batch_device's.
 *   hrnn_search_plan_result: waits for `stream`; *total = out_offsets[nq];
 *     *clamped = 1 if some query's m or ef_search was above the maxima;
 *     HRNN_ERR_CAPACITY when total > cap (labels then not written). */
typedef struct hrnn_search_plan hrnn_search_plan;
hrnn_status hrnn_search_plan_create(hrnn_index* h, const float* d_queries, size_t nq, const uint32_t* d_m,
                                    const uint32_t* d_K_prime, const uint32_t* d_ef_search, uint32_t m_max,
                                    uint32_t ef_max, float threshold, uint32_t k, uint64_t* d_out_offsets,
                                    uint64_t* d_out_labels, size_t cap, void* stream, hrnn_search_plan** out);
hrnn_status hrnn_search_plan_run(hrnn_search_plan* plan, void* stream);
hrnn_status hrnn_search_plan_result(hrnn_search_plan* plan, void* stream, uint64_t* total, int* clamped);
/* One run of a plan on a host batch: copies the nq queries and their m / K' /
 * ef_search from host memory into the plan's input buffers (the device buffers
 * given at creation), replays the graph, waits, and copies out_offsets (nq + 1)
 * and the labels (at most cap; HRNN_ERR_CAPACITY beyond, labels not written) back
 * to host memory.  The serving call of hrnn_search_rknn_batch for a fixed batch
 * shape; *clamped as hrnn_search_plan_result. */
hrnn_status hrnn_search_plan_run_host(hrnn_search_plan* plan, const float* queries, const uint32_t* m,
                                      const uint32_t* K_prime, const uint32_t* ef_search, uint64_t* out_offsets,
                                      uint64_t* out_labels, size_t cap, uint64_t* total, int* clamped, void* stream);
/* Kernel launches one run of the plan makes (the graph's kernel nodes). */
hrnn_status hrnn_search_plan_kernels(hrnn_search_plan* plan, size_t* n);
void hrnn_search_plan_destroy(hrnn_search_plan* plan);

/* compactForServing(max_k_serve) -- hrnn.h:299-364: dense kdist[n x max_k_serve]. */
hrnn_status hrnn_compact_for_serving(hrnn_index* h, size_t max_k_serve);

/* The radius every verification compares against, kdist(p, k-1) of
 * hrnn.h:286-293 (FLT_MAX where the KNN list is shorter than k; the serve-mode
 * matrix after compactForServing), for every element: out[cur_element_count]. */
hrnn_status hrnn_get_kdist(hrnn_index* h, uint32_t k, float* out);

/* insertPointDynamic(x, label, m_update, bidirectional) for n points --
 * hrnn.h:2360-2534, as the insert loop of src/hrnn_dynamic_test.cpp:310-331. */
hrnn_status hrnn_insert_dynamic(hrnn_index* h, const float* data, const uint64_t* labels, size_t n,
                                unsigned m_update, int bidirectional);

/* Counters of the last hrnn_insert_dynamic call. */
hrnn_status hrnn_get_dynamic_stats(hrnn_index* h, hrnn_dynamic_stats* st);

/* setEf -- hrnn.h:226-228. */
hrnn_status hrnn_set_ef(hrnn_index* h, size_t ef);

/* Public fields / getters (K_knng_, knng_built_, rknng_built_, getCurrentElementCount). */
hrnn_status hrnn_get_info(hrnn_index* h, hrnn_info* info);

/* Counters of the last search call. */
hrnn_status hrnn_get_search_stats(hrnn_index* h, hrnn_search_stats* st);

/* Counters of the last refineKNNG call. */
hrnn_status hrnn_get_refine_stats(hrnn_index* h, hrnn_refine_stats* st);

/* Precision of the search (new; the reference has FP32 only).
 *  HRNN_PREC_FP32_EXACT (default): every distance is the reference's FP32 value;
 *      answers are bit-identical to searchRknn.
 *  HRNN_PREC_BF16: the beam search ranks with BF16 copies of the vectors and the
 *      verification screens with them under a rigorous per-vector error bound;
 *      every undecided accept/reject is re-decided with the reference's exact
 *      FP32 distance, and within 16 ulps of the radius in FP64 against the
 *      FP64 distance to the k-th neighbour.  Proxies may differ from the
 *      reference's (recall, not membership); counts in hrnn_search_stats.
 *  HRNN_PREC_INT8: as HRNN_PREC_BF16, but the beam search ranks with INT8 copies
 *      of the vectors (per-vector scale) against an INT8 copy of the query
 *      (integer dot products): the proxies are approximate, the decisions are
 *      made as in HRNN_PREC_BF16.  Needs dim a multiple of 16, at most 256. */
#define HRNN_PREC_FP32_EXACT 0
#define HRNN_PREC_BF16 1
#define HRNN_PREC_INT8 2
hrnn_status hrnn_set_precision(hrnn_index* h, int precision);

/* Launch-shape autotuning of the beam search (new).  With it on (the default), the
 * first batch of at least 1024 queries for a given distance mode and beam size
 * times the beam-search kernel at warps-per-block {2, 4} x visited-cache slots
 * {256, 512, 1024} on that batch and keeps the fastest for the index; answers do
 * not depend on the shape (a visited-cache miss only re-scores a node, which the
 * beam bound rejects again).  Off: 4 warps per block (fewer when the beam does not
 * fit), 512 slots. */
hrnn_status hrnn_set_autotune(hrnn_index* h, int enable);

/* Local join of refineKNNG (new; the reference computes every sample pair's FP32
 * distance, hrnn.h:1823-1853).  Every mode yields the same proposals, hence the
 * same lists:
 *  HRNN_JOIN_EXACT (default):  exact FP32 distance of every pair on the CUDA cores.
 *  HRNN_JOIN_TENSOR: a BF16 Gram matrix of each node's sample rows on
 *      the tensor cores bounds every pair's FP32 distance from below; pairs whose
 *      bound reaches both ends' farthest entries are dropped, the rest get the
 *      exact FP32 distance.  Used for dim a multiple of 16 up to 128 and sample
 *      sizes up to 64 (16-lane L2 order); otherwise the exact join runs.
 *  HRNN_JOIN_AUDIT:  the screen's decisions recorded, then every pair exact;
 *      proposals the screen would have dropped are counted in
 *      hrnn_refine_stats.screen_misses. */
#define HRNN_JOIN_EXACT 0
#define HRNN_JOIN_TENSOR 1
#define HRNN_JOIN_AUDIT 2
hrnn_status hrnn_set_join_mode(hrnn_index* h, int mode);

/* Learned search budget (new; no counterpart in the reference).  A 256-256-256-2
 * MLP with GELU and BF16 weights reads a query and its beam frontier (the 32
 * nearest beam entries) and outputs two logits: "the answer with m = m0 proxies
 * is complete" and "... with m = m1".  The batch search then uses the cheapest
 * level whose probability reaches `confidence`, and the caller's m otherwise.
 * Verification still decides every returned point: the budget changes work,
 * never membership.
 *   ef = 0 (single pass): the frontier is the caller's own beam (ef_search), so a
 *     level's answer equals the plain search with (m_l, ef_search).
 *   ef > 0 (two pass): the frontier beam is ef; a level's answer equals the plain
 *     search with (m_l, ef); the other queries are searched again with the
 *     caller's (m, ef_search).
 *   hrnn_set_budget: stores (m0, m1, ef, confidence) with 1 <= m0 <= m1 <= 32,
 *     ef = 0 or m1 <= ef, 0.5 < confidence <= 1, also when disabling; enabling
 *     needs weights.
 *   hrnn_budget_features: the 256 features of nq host queries (host out, nq x 256)
 *     for result size k, from the frontier of a search with (m, ef_search) --
 *     (m1, ef) in two-pass mode.
 *   hrnn_budget_train: trains on the device with the library's BF16 kernels
 *     (labels: nq x 2 bytes, 1 = complete at that level); returns the last
 *     epoch's mean loss.  A model without weights is first initialised from
 *     `seed`, with the training features' per-feature mean and 1/std as its
 *     input normalisation (x -> (x - mean) * inv, applied before layer 1).
 *   hrnn_budget_predict / hrnn_budget_gradients: forward logits / gradients of
 *     the mean binary cross-entropy (summed over both outputs) with respect to
 *     W1 b1 W2 b2 W3 b3, FP32 (the normalisation entries are left untouched).
 *   hrnn_budget_get_weights / _set_weights: W1 [256x256] b1 W2 [256x256] b2
 *     W3 [2x256] b3, then mean[256] and inv[256] (HRNN_BUDGET_PARAMS floats). */
#define HRNN_BUDGET_PARAMS (256 * 256 + 256 + 256 * 256 + 256 + 2 * 256 + 2 + 2 * 256)
hrnn_status hrnn_set_budget(hrnn_index* h, int enable, uint32_t m0, uint32_t m1, uint32_t ef,
                            float confidence);
hrnn_status hrnn_budget_features(hrnn_index* h, const float* queries, size_t nq, uint32_t k, uint32_t m,
                                 uint32_t ef_search, float* feat);
hrnn_status hrnn_budget_train(hrnn_index* h, const float* feat, const uint8_t* labels, size_t n,
                              int epochs, int batch, float lr, uint64_t seed, float* final_loss);
hrnn_status hrnn_budget_predict(hrnn_index* h, const float* feat, size_t n, float* logits);
hrnn_status hrnn_budget_gradients(hrnn_index* h, const float* feat, const uint8_t* labels, size_t n,
                                  float* grads, float* loss);
hrnn_status hrnn_budget_get_weights(hrnn_index* h, float* params);
hrnn_status hrnn_budget_set_weights(hrnn_index* h, const float* params);

/* FP32 summation order of the L2 kernel (space_l2.h:214-238 picks it per host):
 * lanes in {16, 8, 4}; fused bit 0 = SIMD multiply-add contracted, bit 1 = scalar
 * tail contracted.  hrnn_detect_l2_order reports what the reference compiled with
 * -march=native would use on this host (AVX-512 -> 16, AVX -> 8, else 4). */
hrnn_status hrnn_set_l2_order(hrnn_index* h, int lanes, int fused);
hrnn_status hrnn_detect_l2_order(int* lanes, int* fused);

/* Read access to the KNN graph slot (get_knng_linklist hrnn.h:262-281):
 * ids, dists: n x K_knng host arrays; cnt: n host counts.  Any may be NULL. */
hrnn_status hrnn_get_knng(hrnn_index* h, uint32_t* ids, float* dists, uint32_t* cnt);
/* Replace the KNN graph slot (e.g. to refine a graph produced elsewhere). */
hrnn_status hrnn_set_knng(hrnn_index* h, const uint32_t* ids, const float* dists,
                          const uint32_t* cnt);

/* Reverse CSR (rknng_offsets_ / rknng_entries_*, hrnn.h:89-101).  Call with NULL
 * arrays to get the sizes.  reference_order = 1 returns the entries in the exact
 * byte order the reference's buildRKNNG_fill produces (its std::sort call is
 * applied to the owner-ordered scatter on the host); 0 returns the device's
 * canonical (rank, owner) order. */
hrnn_status hrnn_get_rknng(hrnn_index* h, uint64_t* n_offsets, uint64_t* n_entries,
                           uint32_t* entry_bytes, uint32_t* rank_bits, uint64_t* offsets,
                           void* entries, int reference_order);

/* Reverse-KNN CSR of a KNN graph the caller owns, with NO device allocation.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc (an arena that owns every device byte, or a serving loop that must
 * not synchronise the device), and takes all buffers from the caller:
 *   d_knn_ids  n x K u32 neighbour ids; d_knn_cnt n counts (low 16 bits used);
 *   d_offsets  n+1 u64 out; d_entries entries_cap entries out -- u32 when
 *              node_bits + rank_bits <= 32 (*wide = 0), else u64;
 *   *n_entries receives the entry count (also on HRNN_ERR_CAPACITY).
 * Same output as hrnn_build_rknng + hrnn_get_rknng(..., reference_order = 0).
 * The graph is checked on the device first: a count above K or a neighbour id
 * >= n returns HRNN_ERR_ARG and nothing is scattered.
 * Its scratch is a fixed 32 MiB __device__ array in the library, held by every
 * GPU that loads it: n is limited to 2,097,152 (HRNN_ERR_LIMIT beyond).  The
 * counters take 12 (n+1) bytes of it and the rest stages the sort of reverse
 * lists longer than 16,384 entries, so one reverse list may hold at most the
 * largest power of two <= (33,554,432 - 12 (n+1) - 8 ceil((n+1)/4096) - 1280) / 8
 * entries: 524,288 at n = 2,097,152; every possible list (< n) at
 * n <= 1,048,576.  A longer list returns HRNN_ERR_LIMIT.  The first call on a
 * device looks up the array's address (again after the device's context was
 * re-created); make it before any stream capture.  Calls share the array:
 * calls that overlap on the GPU race; issue them one after another.
 * Runs on `stream` (cudaStream_t) on the current device and returns after it
 * finishes. */
hrnn_status hrnn_build_rknng_noalloc(const uint32_t* d_knn_ids, const uint32_t* d_knn_cnt, size_t n,
                                     size_t K, uint64_t* d_offsets, void* d_entries,
                                     size_t entries_cap, uint32_t* rank_bits, int* wide,
                                     uint64_t* n_entries, void* stream);

/* Squared L2 of n pairs (a[i], b[i]) of dim floats on the device, in the order set by
 * hrnn_set_l2_order.  Host arrays.  (L2Space::get_dist_func, space_l2.h:240-248.) */
hrnn_status hrnn_l2_batch(const float* a, const float* b, size_t n, size_t dim, int lanes,
                          int fused, float* out);

#ifdef __cplusplus
}
#endif
#endif /* HRNN_CAPI_H */
