/* CPU restatement of the reference's hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * The oracle is a checker: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg load it; the product library never does.  Every function
 * restates the reference's algorithm in plain C, citing the lines of
 * include/hnswlib/hrnn.h / space_l2.h it follows.  It is pinned against the
 * reference compiled from its own sources (oracle/_ref) and the committed
 * fixtures under tests/golden/ by tests/test_oracle_pin.py.
 *
 * Compiled with -ffp-contract=off: every fused multiply-add below is an
 * explicit fmaf(), so the restated summation order is exactly what is written.
 */
#include "hrnn_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* L2 distance                                                               */
/* ------------------------------------------------------------------------- */

static inline float sq_acc(float acc, float t, int fused) {
    return fused ? fmaf(t, t, acc) : acc + t * t;
}

/* space_l2.h:6-20: res += t*t, left to right. */
static float l2_scalar(const float* a, const float* b, size_t d, int fused) {
    float res = 0.0f;
    for (size_t i = 0; i < d; ++i) res = sq_acc(res, a[i] - b[i], fused & 2);
    return res;
}

/* space_l2.h:25-54 (16 lanes), :61-91 (8 lanes), :97-143 (4 lanes): element e
 * accumulates into lane e % lanes in increasing e; the lanes are then summed
 * left to right (TmpRes[0] + TmpRes[1] + ...). d must be a multiple of 16. */
static float l2_simd(const float* a, const float* b, size_t d, int lanes, int fused) {
    float acc[16];
    for (int l = 0; l < lanes; ++l) acc[l] = 0.0f;
    for (size_t e = 0; e < d; ++e)
        acc[e % (size_t)lanes] = sq_acc(acc[e % (size_t)lanes], a[e] - b[e], fused & 1);
    float res = acc[0];
    for (int l = 1; l < lanes; ++l) res = res + acc[l];
    return res;
}

/* space_l2.h:214-238 dispatch by dim. */
float orc_l2(const float* a, const float* b, size_t d, int lanes, int fused) {
    if (d % 16 == 0) return l2_simd(a, b, d, lanes, fused);
    if (d % 4 == 0) return l2_simd(a, b, d, 4, fused);              /* :163-183 */
    if (d > 16) {                                                    /* :148-159 */
        size_t d16 = d >> 4 << 4;
        float r = l2_simd(a, b, d16, lanes, fused);
        float t = l2_scalar(a + d16, b + d16, d - d16, fused);
        return r + t;
    }
    if (d > 4) {                                                     /* :185-200 */
        size_t d4 = d >> 2 << 2;
        float r = l2_simd(a, b, d4, 4, fused);
        float t = l2_scalar(a + d4, b + d4, d - d4, fused);
        return r + t;
    }
    return l2_scalar(a, b, d, fused);
}

void orc_l2_batch(const float* a, const float* b, size_t n, size_t d, int lanes, int fused,
                  float* out) {
    for (size_t i = 0; i < n; ++i) out[i] = orc_l2(a + i * d, b + i * d, d, lanes, fused);
}

/* ------------------------------------------------------------------------- */
/* Binary heaps of (dist, id) -- the two std::priority_queue of hrnn.h:491-492 */
/* ------------------------------------------------------------------------- */

typedef struct { float d; uint32_t id; } pr;
typedef struct { pr* a; size_t n, cap; int max_heap; } heap;

static int heap_before(const heap* h, pr x, pr y) { /* x above y in the heap */
    return h->max_heap ? (x.d > y.d) : (x.d < y.d);
}
static void heap_push(heap* h, float d, uint32_t id) {
    if (h->n == h->cap) {
        h->cap = h->cap ? h->cap * 2 : 64;
        h->a = (pr*)realloc(h->a, h->cap * sizeof(pr));
    }
    size_t i = h->n++;
    pr x = {d, id};
    while (i > 0) {
        size_t p = (i - 1) / 2;
        if (!heap_before(h, x, h->a[p])) break;
        h->a[i] = h->a[p];
        i = p;
    }
    h->a[i] = x;
}
static pr heap_pop(heap* h) {
    pr top = h->a[0];
    pr x = h->a[--h->n];
    size_t i = 0;
    for (;;) {
        size_t c = 2 * i + 1;
        if (c >= h->n) break;
        if (c + 1 < h->n && heap_before(h, h->a[c + 1], h->a[c])) ++c;
        if (!heap_before(h, h->a[c], x)) break;
        h->a[i] = h->a[c];
        i = c;
    }
    if (h->n) h->a[i] = x;
    return top;
}

/* ------------------------------------------------------------------------- */
/* searchRknn                                                                */
/* ------------------------------------------------------------------------- */

static const float* vec_of(const orc_index* ix, uint32_t id) { return ix->vec + (size_t)id * ix->d; }

static float l2q(const orc_index* ix, const float* q, uint32_t id) {
    return orc_l2(q, vec_of(ix, id), ix->d, ix->lanes, ix->fused);
}

/* searchBaseLayerST<bare_bone_search=true> (hrnn.h:484-616). */
static void base_layer_search(const orc_index* ix, uint32_t ep, const float* q, size_t ef,
                              uint8_t* visited, heap* top, orc_stats* st) {
    heap cand = {0};
    cand.max_heap = 0;
    float d0 = l2q(ix, q, ep);
    if (st) st->n_dist++;
    float lower = d0;
    heap_push(top, d0, ep);
    heap_push(&cand, d0, ep);
    visited[ep] = 1;
    while (cand.n) {
        pr c = cand.a[0];
        if (c.d > lower) break;                                 /* :521-523, :532 */
        heap_pop(&cand);
        const uint32_t* list = ix->adj0 + (size_t)c.id * (1 + ix->maxM0);
        unsigned size = list[0] & 0xFFFFu;                      /* getListCount: u16 */
        if (st) st->n_expanded++;
        for (unsigned j = 1; j <= size; ++j) {
            uint32_t cid = list[j];
            if (visited[cid]) continue;
            visited[cid] = 1;
            float d = l2q(ix, q, cid);
            if (st) st->n_dist++;
            if (top->n < ef || lower > d) {                     /* :572 */
                heap_push(&cand, d, cid);
                heap_push(top, d, cid);
                while (top->n > ef) heap_pop(top);
                if (top->n) lower = top->a[0].d;
            }
        }
    }
    free(cand.a);
}

static float verify_kdist(const orc_index* ix, uint32_t id, unsigned k_idx) {
    /* getVerifyKdistSq (hrnn.h:286-293) */
    if (ix->kdist_serve) return ix->kdist_serve[(size_t)id * ix->max_k_serve + k_idx];
    unsigned cnt = ix->knn_cnt[id] & 0xFFFFu;
    if (k_idx >= cnt) return FLT_MAX;
    return ix->knn_dist[(size_t)id * ix->K + k_idx];
}

static int cmp_u32(const void* x, const void* y) {
    uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
    return (a > b) - (a < b);
}

size_t orc_search_rknn(const orc_index* ix, const float* q, size_t m, float threshold,
                       size_t k, size_t Kp, size_t ef, uint64_t* out, size_t cap,
                       float* score_buf, orc_stats* st, uint32_t* proxies_out,
                       size_t* n_proxies) {
    if (n_proxies) *n_proxies = 0;
    if (ix->n == 0) return 0;                                   /* :1987 */
    /* Phase A: greedy descent over the upper layers (hrnn.h:1992-2013). */
    uint32_t cur = ix->enterpoint;
    float curdist = l2q(ix, q, cur);
    if (st) st->n_dist++;
    for (int level = ix->maxlevel; level > 0; --level) {
        int changed = 1;
        while (changed) {
            changed = 0;
            const uint32_t* data = ix->upper + ix->upper_off[cur] + (size_t)(level - 1) * (1 + ix->maxM);
            unsigned size = data[0] & 0xFFFFu;
            for (unsigned i = 0; i < size; ++i) {
                uint32_t c = data[1 + i];
                float d = l2q(ix, q, c);
                if (st) st->n_dist++;
                if (d < curdist) {
                    curdist = d;
                    cur = c;
                    changed = 1;
                }
            }
        }
    }
    /* Base layer with ef = max(ef_search, m), then trim to m (hrnn.h:2016-2019). */
    uint8_t* visited = (uint8_t*)calloc(ix->n, 1);
    heap top = {0};
    top.max_heap = 1;
    base_layer_search(ix, cur, q, ef > m ? ef : m, visited, &top, st);
    free(visited);
    while (top.n > m) heap_pop(&top);

    /* Phase B: reverse-list prefix scan, farthest proxy first (hrnn.h:2021-2037). */
    size_t np = top.n;
    uint32_t* prox = (uint32_t*)malloc((np ? np : 1) * sizeof(uint32_t));
    for (size_t i = 0; i < np; ++i) prox[np - 1 - i] = heap_pop(&top).id;
    free(top.a);
    if (proxies_out) memcpy(proxies_out, prox, np * sizeof(uint32_t));
    if (n_proxies) *n_proxies = np;
    uint64_t rmask = (1ull << ix->rank_bits) - 1ull;
    size_t ncap = 1024, nc = 0;
    uint32_t* cands = (uint32_t*)malloc(ncap * sizeof(uint32_t));
    for (size_t pi = np; pi-- > 0;) {                           /* farthest first */
        uint32_t p = prox[pi];
        for (uint64_t e = ix->csr_off[p]; e < ix->csr_off[p + 1]; ++e) {
            uint64_t packed = ix->entry_bytes == 8 ? ((const uint64_t*)ix->csr_ent)[e]
                                                   : ((const uint32_t*)ix->csr_ent)[e];
            uint32_t rank = (uint32_t)(packed & rmask);
            if (rank >= Kp) break;
            uint32_t c = (uint32_t)(packed >> ix->rank_bits);
            if (st) st->n_posting++;
            if (score_buf[c] == 0.0f) {
                if (nc == ncap) {
                    ncap *= 2;
                    cands = (uint32_t*)realloc(cands, ncap * sizeof(uint32_t));
                }
                cands[nc++] = c;
            }
            score_buf[c] += 1.0f;
        }
    }
    free(prox);
    if (st) st->n_cand += nc;
    /* Phase C.1: threshold filter + reset (hrnn.h:2043-2052). */
    size_t w = 0;
    for (size_t i = 0; i < nc; ++i) {
        uint32_t c = cands[i];
        int keep = score_buf[c] >= threshold;
        score_buf[c] = 0.0f;
        if (keep) cands[w++] = c;
    }
    nc = w;
    if (st) st->n_verified += nc;
    /* Phase C.2: id order, then exact verification (hrnn.h:2055-2069). */
    qsort(cands, nc, sizeof(uint32_t), cmp_u32);
    unsigned k_idx = (unsigned)(k - 1);
    size_t nr = 0;
    for (size_t i = 0; i < nc; ++i) {
        uint32_t c = cands[i];
        float d = l2q(ix, q, c);
        float kd = verify_kdist(ix, c, k_idx);
        if (d <= kd) {
            if (nr < cap) out[nr] = ix->labels[c];
            nr++;
        }
    }
    free(cands);
    if (st) st->n_result += nr;
    return nr;
}

int orc_search_rknn_batch(const orc_index* ix, const float* Q, size_t nq, const uint32_t* m,
                          const uint32_t* Kp, const uint32_t* ef, float threshold, uint32_t k,
                          uint64_t* out_offsets, uint64_t* out_labels, size_t cap, int threads) {
    uint64_t** res = (uint64_t**)calloc(nq ? nq : 1, sizeof(uint64_t*));
    size_t* cnt = (size_t*)calloc(nq ? nq : 1, sizeof(size_t));
#pragma omp parallel num_threads(threads > 0 ? threads : 1)
    {
        float* score = (float*)calloc(ix->n ? ix->n : 1, sizeof(float));
#pragma omp for schedule(dynamic, 8)
        for (long long qi = 0; qi < (long long)nq; ++qi) {
            size_t mcap = (size_t)m[qi] * (Kp[qi] ? Kp[qi] : 1) + 64;
            uint64_t* buf = (uint64_t*)malloc(mcap * sizeof(uint64_t));
            size_t r = orc_search_rknn(ix, Q + (size_t)qi * ix->d, m[qi], threshold, k, Kp[qi],
                                       ef[qi], buf, mcap, score, NULL, NULL, NULL);
            if (r > mcap) { /* hub-heavy case: rerun with the exact size */
                free(buf);
                buf = (uint64_t*)malloc(r * sizeof(uint64_t));
                orc_search_rknn(ix, Q + (size_t)qi * ix->d, m[qi], threshold, k, Kp[qi], ef[qi], buf,
                                r, score, NULL, NULL, NULL);
            }
            res[qi] = buf;
            cnt[qi] = r;
        }
        free(score);
    }
    uint64_t total = 0;
    out_offsets[0] = 0;
    for (size_t qi = 0; qi < nq; ++qi) {
        total += cnt[qi];
        out_offsets[qi + 1] = total;
    }
    int rc = total > cap ? 2 : 0;
    for (size_t qi = 0; qi < nq; ++qi) {
        if (!rc) memcpy(out_labels + out_offsets[qi], res[qi], cnt[qi] * sizeof(uint64_t));
        free(res[qi]);
    }
    free(res);
    free(cnt);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* Reverse KNN graph (CSR transpose)                                         */
/* ------------------------------------------------------------------------- */

uint32_t orc_rknng_params(size_t n, size_t K, int* wide) {
    uint32_t rb = 0, nb = 0;                                    /* hrnn.h:1876-1880 */
    while ((1ull << rb) < K) rb++;
    while ((1ull << nb) < n) nb++;
    *wide = (nb + rb) > 32;
    return rb;
}

void orc_rknng_presort(size_t n, size_t K, const uint32_t* knn_ids, const uint32_t* knn_cnt,
                       uint32_t rank_bits, int wide, uint64_t* offsets, void* entries) {
    memset(offsets, 0, (n + 1) * sizeof(uint64_t));             /* hrnn.h:1891-1900 */
    for (size_t i = 0; i < n; ++i) {
        unsigned c = knn_cnt[i] & 0xFFFFu;
        for (unsigned j = 0; j < c; ++j) offsets[knn_ids[i * K + j] + 1]++;
    }
    for (size_t i = 1; i <= n; ++i) offsets[i] += offsets[i - 1];
    uint64_t* pos = (uint64_t*)malloc((n + 1) * sizeof(uint64_t));
    memcpy(pos, offsets, (n + 1) * sizeof(uint64_t));
    for (size_t i = 0; i < n; ++i) {                            /* hrnn.h:1919-1925 */
        unsigned c = knn_cnt[i] & 0xFFFFu;
        for (unsigned j = 0; j < c; ++j) {
            uint32_t nbr = knn_ids[i * K + j];
            uint64_t v = ((uint64_t)i << rank_bits) | j;
            if (wide) ((uint64_t*)entries)[pos[nbr]++] = v;
            else ((uint32_t*)entries)[pos[nbr]++] = (uint32_t)v;
        }
    }
    free(pos);
}

static uint32_t g_rb;
static int cmp_rank_owner32(const void* x, const void* y) {
    uint32_t a = *(const uint32_t*)x, b = *(const uint32_t*)y;
    uint32_t m = (uint32_t)((1ull << g_rb) - 1);
    uint32_t ra = a & m, rbv = b & m;
    if (ra != rbv) return ra < rbv ? -1 : 1;
    return (a > b) - (a < b);
}
static int cmp_rank_owner64(const void* x, const void* y) {
    uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    uint64_t m = (1ull << g_rb) - 1;
    uint64_t ra = a & m, rbv = b & m;
    if (ra != rbv) return ra < rbv ? -1 : 1;
    return (a > b) - (a < b);
}

void orc_rknng_canonical(size_t n, uint32_t rank_bits, int wide, const uint64_t* offsets,
                         void* entries) {
    g_rb = rank_bits;
    for (size_t b = 0; b < n; ++b) {
        size_t len = offsets[b + 1] - offsets[b];
        if (wide) qsort((uint64_t*)entries + offsets[b], len, 8, cmp_rank_owner64);
        else qsort((uint32_t*)entries + offsets[b], len, 4, cmp_rank_owner32);
    }
}

/* ------------------------------------------------------------------------- */
/* NNDescent refinement, one thread                                          */
/* ------------------------------------------------------------------------- */

typedef struct { uint32_t* a; size_t n, cap; } vec_u32;
static void vpush(vec_u32* v, uint32_t x) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 16;
        v->a = (uint32_t*)realloc(v->a, v->cap * sizeof(uint32_t));
    }
    v->a[v->n++] = x;
}

/* try_update_knng_nnd (hrnn.h:1660-1722). */
static int try_update(size_t K, uint32_t* ids, float* dists, uint32_t* cnt, uint8_t* is_new,
                      uint32_t u, uint32_t w, float d) {
    uint32_t* I = ids + (size_t)u * K;
    float* D = dists + (size_t)u * K;
    uint8_t* F = is_new + (size_t)u * K;
    unsigned c = cnt[u] & 0xFFFFu;
    if (c >= K && d >= D[c - 1]) return 0;
    for (unsigned i = 0; i < c; ++i)
        if (I[i] == w) return 0;
    unsigned at;
    if (c < K) {
        at = c;
        cnt[u] = c + 1;
    } else {
        at = c - 1;
    }
    I[at] = w;
    D[at] = d;
    F[at] = 1;
    for (unsigned i = at; i > 0; --i) {
        if (D[i] < D[i - 1]) {
            uint32_t ti = I[i]; I[i] = I[i - 1]; I[i - 1] = ti;
            float td = D[i]; D[i] = D[i - 1]; D[i - 1] = td;
            uint8_t tf = F[i]; F[i] = F[i - 1]; F[i - 1] = tf;
        } else {
            break;
        }
    }
    return 1;
}

void orc_refine_knng(size_t n, size_t d, size_t K, const float* vec, int lanes, int fused,
                     uint32_t* ids, float* dists, uint32_t* cnt, uint8_t* is_new, int iters,
                     int sample, uint64_t* updates, uint64_t* join_dists) {
    unsigned S = (unsigned)sample, R = S;                       /* hrnn.h:1727-1728 */
    vec_u32* nn_new = (vec_u32*)calloc(n, sizeof(vec_u32));
    vec_u32* nn_old = (vec_u32*)calloc(n, sizeof(vec_u32));
    vec_u32* rnn_new = (vec_u32*)calloc(n, sizeof(vec_u32));
    vec_u32* rnn_old = (vec_u32*)calloc(n, sizeof(vec_u32));
    for (int it = 0; it < iters; ++it) {
        uint64_t upd = 0, jd = 0;
        for (size_t i = 0; i < n; ++i) nn_new[i].n = nn_old[i].n = rnn_new[i].n = rnn_old[i].n = 0;
        /* Phase 1 (hrnn.h:1757-1810), in the order a single thread visits it. */
        for (size_t i = 0; i < n; ++i) {
            unsigned c = cnt[i] & 0xFFFFu;
            for (unsigned j = 0; j < c; ++j) {
                uint32_t nbr = ids[i * K + j];
                float dij = dists[i * K + j];
                int entry_new = is_new[i * K + j];
                unsigned cn = cnt[nbr] & 0xFFFFu;
                float worst = cn >= K ? dists[(size_t)nbr * K + cn - 1] : FLT_MAX;
                if (entry_new) {
                    if (nn_new[i].n < S) vpush(&nn_new[i], nbr);
                    is_new[i * K + j] = 0;
                    if (cn > 0 && dij > worst && rnn_new[nbr].n < R) vpush(&rnn_new[nbr], (uint32_t)i);
                } else {
                    if (nn_old[i].n < S) vpush(&nn_old[i], nbr);
                    if (cn > 0 && dij > worst && rnn_old[nbr].n < R) vpush(&rnn_old[nbr], (uint32_t)i);
                }
            }
        }
        /* Merge (hrnn.h:1813-1819). */
        for (size_t i = 0; i < n; ++i) {
            for (size_t r = 0; r < rnn_new[i].n; ++r) vpush(&nn_new[i], rnn_new[i].a[r]);
            for (size_t r = 0; r < rnn_old[i].n; ++r) vpush(&nn_old[i], rnn_old[i].a[r]);
            if (nn_old[i].n > 2 * R) nn_old[i].n = 2 * R;
        }
        /* Phase 2: local join (hrnn.h:1823-1853). */
        for (size_t node = 0; node < n; ++node) {
            vec_u32* nw = &nn_new[node];
            vec_u32* ol = &nn_old[node];
            for (size_t i = 0; i < nw->n; ++i) {
                for (size_t j = i + 1; j < nw->n; ++j) {
                    uint32_t a = nw->a[i], b = nw->a[j];
                    if (a == b) continue;
                    float dd = orc_l2(vec + (size_t)a * d, vec + (size_t)b * d, d, lanes, fused);
                    jd++;
                    upd += try_update(K, ids, dists, cnt, is_new, a, b, dd);
                    upd += try_update(K, ids, dists, cnt, is_new, b, a, dd);
                }
            }
            for (size_t i = 0; i < nw->n; ++i) {
                for (size_t j = 0; j < ol->n; ++j) {
                    uint32_t a = nw->a[i], b = ol->a[j];
                    if (a == b) continue;
                    float dd = orc_l2(vec + (size_t)a * d, vec + (size_t)b * d, d, lanes, fused);
                    jd++;
                    upd += try_update(K, ids, dists, cnt, is_new, a, b, dd);
                    upd += try_update(K, ids, dists, cnt, is_new, b, a, dd);
                }
            }
        }
        if (updates) updates[it] = upd;
        if (join_dists) join_dists[it] = jd;
    }
    for (size_t i = 0; i < n; ++i) {
        free(nn_new[i].a); free(nn_old[i].a); free(rnn_new[i].a); free(rnn_old[i].a);
    }
    free(nn_new); free(nn_old); free(rnn_new); free(rnn_old);
}
