/* CPU restatement of the reference's hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This is the oracle: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg may load it, and only as a checker.  The product library
 * (hrnn_b200/) never links or calls it.  Each function restates one piece of
 * the reference (include/hnswlib/hrnn.h and space_l2.h) and cites the lines it
 * follows.  Parity is pinned by tests/test_oracle_pin.py against the reference
 * itself compiled from its sources (oracle/_ref/libhrnn_ref.so) and against the
 * committed fixtures under tests/golden/.
 */
#ifndef HRNN_ORACLE_H
#define HRNN_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Squared L2 with the reference's FP32 summation order.
 * lanes: width of the SIMD accumulator the reference's L2Space picked
 *        (16 = AVX-512, 8 = AVX, 4 = SSE).
 * fused: bit 0 set when the compiler contracted the SIMD multiply-add into an
 *        FMA, bit 1 set when it contracted the scalar tail loop.  GCC 13 with
 *        -march=native on a Sapphire Rapids host (the GPU hosts of this project)
 *        keeps the SIMD chain unfused and fuses the scalar tail: fused = 2.
 * space_l2.h:6-20 (scalar), :25-54 (AVX-512), :61-91 (AVX), :97-143 (SSE),
 * :148-159 (16 + residual), :163-200 (4-wide), :214-238 (dispatch by dim). */
float orc_l2(const float* a, const float* b, size_t d, int lanes, int fused);
void orc_l2_batch(const float* a, const float* b, size_t n, size_t d, int lanes, int fused,
                  float* out);

/* Device-independent view of an HRNN index in structure-of-arrays form. */
typedef struct {
    size_t n, d, maxM0, maxM, K;
    const float* vec;          /* n*d */
    const uint32_t* adj0;      /* n*(1+maxM0); word 0 = count in its low 16 bits */
    const int32_t* level;      /* n */
    const uint64_t* upper_off; /* n; word offset of level-1 block in `upper` */
    const uint32_t* upper;     /* per element: level blocks of (1+maxM) words */
    uint32_t enterpoint;
    int32_t maxlevel;
    const uint32_t* knn_cnt;   /* n (count of the KNN-graph slot) */
    const float* knn_dist;     /* n*K */
    const float* kdist_serve;  /* serve mode: n*max_k_serve, else NULL */
    size_t max_k_serve;
    const uint64_t* csr_off;   /* n+1 */
    const void* csr_ent;       /* u32 or u64 entries */
    int entry_bytes;           /* 4 or 8 */
    uint32_t rank_bits;
    const uint64_t* labels;    /* n */
    int lanes, fused;
} orc_index;

typedef struct {
    uint64_t n_dist;       /* distance evaluations in phase A */
    uint64_t n_expanded;   /* base-layer nodes expanded */
    uint64_t n_posting;    /* reverse-list entries read in phase B */
    uint64_t n_cand;       /* distinct candidates after phase B */
    uint64_t n_verified;   /* candidates passing the score threshold */
    uint64_t n_result;
} orc_stats;

/* searchRknn (hrnn.h:1966-2071).  score_buf: n floats, all zero on entry and on
 * return.  Writes at most cap labels; returns the result count.  proxies_out
 * (optional, m entries) receives the proxy ids in ascending distance order. */
size_t orc_search_rknn(const orc_index* ix, const float* q, size_t m, float threshold,
                       size_t k, size_t Kp, size_t ef, uint64_t* out, size_t cap,
                       float* score_buf, orc_stats* st, uint32_t* proxies_out,
                       size_t* n_proxies);

/* Batch form with one (m, K', ef) per query; out_offsets has nq+1 entries.
 * Returns 0, or 2 when cap is too small (out_offsets[nq] then holds the need). */
int orc_search_rknn_batch(const orc_index* ix, const float* Q, size_t nq, const uint32_t* m,
                          const uint32_t* Kp, const uint32_t* ef, float threshold, uint32_t k,
                          uint64_t* out_offsets, uint64_t* out_labels, size_t cap, int threads);

/* buildRKNNG (hrnn.h:1869-1935) without the final per-segment sort:
 * offsets (n+1), and the owner-ascending "scatter" array the reference sorts.
 * Returns rank_bits; *wide = 1 when node_bits + rank_bits > 32. */
uint32_t orc_rknng_params(size_t n, size_t K, int* wide);
void orc_rknng_presort(size_t n, size_t K, const uint32_t* knn_ids, const uint32_t* knn_cnt,
                       uint32_t rank_bits, int wide, uint64_t* offsets, void* entries);
/* Canonical order: each segment stably sorted by rank, i.e. (rank, owner). */
void orc_rknng_canonical(size_t n, uint32_t rank_bits, int wide, const uint64_t* offsets,
                         void* entries);

/* refineKNNG (hrnn.h:1725-1862) as the reference runs it on ONE thread.
 * ids/dists: n*K, cnt: n, is_new: n*K flags (1 = new); all updated in place.
 * vec: n*d.  Per-iteration counters are written to updates/dists (iters each,
 * may be NULL). */
void orc_refine_knng(size_t n, size_t d, size_t K, const float* vec, int lanes, int fused,
                     uint32_t* ids, float* dists, uint32_t* cnt, uint8_t* is_new, int iters,
                     int sample, uint64_t* updates, uint64_t* join_dists);

#ifdef __cplusplus
}
#endif
#endif
