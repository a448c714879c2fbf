// Host side of the index: construction parameters (hrnn.h:128-195), the .idx
// reader/writer (hrnn.h:861-1047, byte-identical), KNN-slot access and the
// serve-mode kdist matrix (hrnn.h:299-364).
#include <cpuid.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <fstream>

#include "index.hpp"
#include "mlp.hpp"

namespace hrnn {

Index::Index() = default;

Index::~Index() {
    for (auto& e : aux_ev)
        if (e) cudaEventDestroy(e);
    if (aux) cudaStreamDestroy(aux);
    if (stream) cudaStreamDestroy(stream);
}

size_t Index::device_bytes() const {
    size_t s = 0;
    for (const DevMem* m : {&vec, &vec_bf16, &vec_norm, &vec_i8, &i8_meta, &adj0, &knn_hdr, &knn_ids, &knn_dist, &labels,
                            &d_upper, &d_upper_off, &csr_off, &csr_ent, &kdist_serve, &counters, &io})
        s += m->bytes;
    for (const auto& m : scratch) s += m.bytes;
    return s;
}

void Index::sync_upper_to_device() {
    if (!upper_dirty) return;
    size_t words = std::max<size_t>(upper.size(), 1);
    if (d_upper.bytes < words * 4) d_upper.alloc(words * 4 + (words * 4) / 4);
    if (!upper.empty())
        CUDA_CHECK(cudaMemcpyAsync(d_upper.p, upper.data(), upper.size() * 4, cudaMemcpyHostToDevice, stream));
    size_t cap = std::max<size_t>(max_elements, 1);
    if (d_upper_off.bytes < cap * 8) d_upper_off.alloc(cap * 8);
    if (!upper_off.empty())
        CUDA_CHECK(cudaMemcpyAsync(d_upper_off.p, upper_off.data(), upper_off.size() * 8,
                                   cudaMemcpyHostToDevice, stream));
    CUDA_CHECK(cudaStreamSynchronize(stream));
    upper_dirty = false;
}

void init_layout(Index& ix, size_t dim, size_t max_elements, size_t M, size_t efc, size_t seed,
                 size_t K) {
    if (dim == 0) fail(HRNN_ERR_ARG, "dim must be > 0");
    ix.dim = dim;
    ix.max_elements = max_elements;
    ix.M = M <= 10000 ? M : 10000;                       // hrnn.h:143-150
    ix.maxM = ix.M;
    ix.maxM0 = ix.M * 2;
    ix.ef_construction = std::max(efc, ix.M);
    ix.ef = 10;
    ix.level_generator.seed((unsigned)seed);             // hrnn.h:157
    ix.size_links_level0 = ix.maxM0 * 4 + 4;             // hrnn.h:160
    ix.K = K;
    if (K > 0) {                                          // hrnn.h:163-172
        ix.size_knng_slot = 4 + K * 8;
        ix.offsetKNNG = ix.size_links_level0;
        ix.offsetData = ix.offsetKNNG + ix.size_knng_slot;
    } else {
        ix.size_knng_slot = 0;
        ix.offsetKNNG = 0;
        ix.offsetData = ix.size_links_level0;
    }
    ix.label_offset = ix.offsetData + dim * 4;
    ix.size_data_per_element = ix.label_offset + 8;
    ix.offsetLevel0 = 0;
    ix.size_links_per_element = ix.maxM * 4 + 4;          // hrnn.h:191
    ix.mult = 1 / std::log(1.0 * ix.M);
    ix.maxlevel = -1;
    ix.enterpoint = kInvalid;
}

void alloc_device(Index& ix, size_t cap) {
    CUDA_CHECK(cudaSetDevice(ix.device));
    if (!ix.stream) CUDA_CHECK(cudaStreamCreateWithFlags(&ix.stream, cudaStreamNonBlocking));
    cap = std::max<size_t>(cap, 1);
    size_t K = std::max<size_t>(ix.K, 1);
    ix.vec.alloc(cap * ix.dim * 4);
    ix.adj0.alloc(cap * (1 + ix.maxM0) * 4);
    ix.knn_hdr.alloc(cap * 4);
    ix.knn_ids.alloc(cap * K * 4);
    ix.knn_dist.alloc(cap * K * 4);
    ix.labels.alloc(cap * 8);
    CUDA_CHECK(cudaMemsetAsync(ix.adj0.p, 0, ix.adj0.bytes, ix.stream));
    CUDA_CHECK(cudaMemsetAsync(ix.knn_hdr.p, 0, ix.knn_hdr.bytes, ix.stream));
    CUDA_CHECK(cudaMemsetAsync(ix.knn_ids.p, 0, ix.knn_ids.bytes, ix.stream));
    CUDA_CHECK(cudaMemsetAsync(ix.knn_dist.p, 0, ix.knn_dist.bytes, ix.stream));
    ix.counters.alloc(sizeof(SearchCounters));
    ix.levels.assign(cap, 0);
    ix.upper_off.assign(cap, 0);
    ix.upper_dirty = true;
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
}

// ---------------------------------------------------------------------------
// .idx reader (loadIndex, hrnn.h:930-1047)
// ---------------------------------------------------------------------------

namespace {

struct Reader {
    std::ifstream in;
    template <class T>
    void pod(T& v) {
        in.read(reinterpret_cast<char*>(&v), sizeof(T));
        if (!in) fail(HRNN_ERR_FORMAT, "loadIndex: truncated index file");
    }
    void bytes(void* p, size_t n) {
        in.read(static_cast<char*>(p), (std::streamsize)n);
        if (!in) fail(HRNN_ERR_FORMAT, "loadIndex: truncated index file");
    }
};

struct Writer {
    std::ofstream out;
    template <class T>
    void pod(const T& v) { out.write(reinterpret_cast<const char*>(&v), sizeof(T)); }
    void bytes(const void* p, size_t n) { out.write(static_cast<const char*>(p), (std::streamsize)n); }
};

constexpr uint32_t kMagic = 0x4E4E5248;  // "HRNN", hrnn.h:865
constexpr size_t kChunk = 1 << 16;       // elements per staging chunk

}  // namespace

void load_idx(Index& ix, const std::string& path, size_t dim, size_t max_elements_i) {
    Reader r;
    r.in.open(path, std::ios::binary);
    if (!r.in.is_open()) fail(HRNN_ERR_IO, "Cannot open file");
    uint32_t magic = 0;
    r.in.read(reinterpret_cast<char*>(&magic), 4);
    if (!r.in || magic != kMagic) fail(HRNN_ERR_FORMAT, "Not an HRNN index file (bad magic)");
    size_t stored_max, cur;
    r.pod(ix.offsetLevel0);
    r.pod(stored_max);
    r.pod(cur);
    size_t max_elements = max_elements_i;                 // hrnn.h:946-951
    if (max_elements < cur) max_elements = stored_max;
    r.pod(ix.size_data_per_element);
    r.pod(ix.label_offset);
    r.pod(ix.offsetData);
    r.pod(ix.maxlevel);
    r.pod(ix.enterpoint);
    r.pod(ix.maxM);
    r.pod(ix.maxM0);
    r.pod(ix.M);
    r.pod(ix.mult);
    r.pod(ix.ef_construction);
    r.pod(ix.K);
    r.pod(ix.size_knng_slot);
    r.pod(ix.offsetKNNG);
    r.pod(ix.knng_built);
    r.pod(ix.rknng_built);
    if (ix.label_offset < ix.offsetData || (ix.label_offset - ix.offsetData) != dim * 4)
        fail(HRNN_ERR_FORMAT, "loadIndex: vector size in file does not match dim");
    if (ix.size_data_per_element != ix.label_offset + 8 || ix.maxM0 > 4096 || ix.maxM > 4096 ||
        (ix.K > 0 && ix.size_knng_slot != 4 + ix.K * 8) || ix.K > 0xFFFF ||
        ix.offsetLevel0 + (1 + ix.maxM0) * 4 > ix.size_data_per_element ||
        (ix.K > 0 && ix.offsetKNNG + ix.size_knng_slot > ix.size_data_per_element))
        fail(HRNN_ERR_FORMAT, "loadIndex: inconsistent element layout");
    // Every id the device kernels follow is range-checked below before it is
    // uploaded: a corrupt file is rejected here instead of becoming out-of-bounds
    // device reads in the search and refinement kernels.
    if (cur > 0xFFFFFFFEull) fail(HRNN_ERR_FORMAT, "loadIndex: element count beyond 32-bit ids");
    if (cur > 0 && (ix.enterpoint >= cur || ix.maxlevel < 0))
        fail(HRNN_ERR_FORMAT, "loadIndex: entry point out of range");
    if (cur == 0 && ix.maxlevel >= 0) fail(HRNN_ERR_FORMAT, "loadIndex: entry point out of range");
    ix.dim = dim;
    ix.max_elements = max_elements;
    ix.cur = cur;
    ix.size_links_level0 = ix.maxM0 * 4 + 4;
    ix.size_links_per_element = ix.maxM * 4 + 4;
    ix.ef = 10;
    alloc_device(ix, max_elements);

    // Level-0 records, split into the SoA arrays chunk by chunk.
    const size_t S = ix.size_data_per_element, W = 1 + ix.maxM0, K = ix.K;
    std::vector<char> blob(std::min(cur, kChunk) * S + 1);
    std::vector<uint32_t> a0, kh, kid;
    std::vector<float> kd, vv;
    std::vector<uint64_t> lb;
    for (size_t base = 0; base < cur; base += kChunk) {
        size_t c = std::min(kChunk, cur - base);
        r.bytes(blob.data(), c * S);
        a0.resize(c * W);
        kh.resize(c);
        kid.resize(c * std::max<size_t>(K, 1));
        kd.resize(c * std::max<size_t>(K, 1));
        vv.resize(c * dim);
        lb.resize(c);
        int bad_links = 0, bad_knn = 0;
#pragma omp parallel for schedule(static) reduction(| : bad_links, bad_knn)
        for (long long e = 0; e < (long long)c; ++e) {
            const char* rec = blob.data() + (size_t)e * S;
            std::memcpy(&a0[e * W], rec + ix.offsetLevel0, W * 4);
            // level-0 links: count (low 16 bits) <= maxM0, ids < cur
            const uint32_t lc = a0[e * W] & 0xFFFFu;
            if (lc > ix.maxM0) bad_links = 1;
            else
                for (uint32_t j = 0; j < lc; ++j) bad_links |= a0[e * W + 1 + j] >= cur;
            if (K > 0) {
                std::memcpy(&kh[e], rec + ix.offsetKNNG, 4);
                const char* p = rec + ix.offsetKNNG + 4;
                for (size_t j = 0; j < K; ++j) {
                    std::memcpy(&kid[e * K + j], p + j * 8, 4);
                    std::memcpy(&kd[e * K + j], p + j * 8 + 4, 4);
                }
                // KNN slot: count <= K, ids < cur
                const uint32_t kc = kh[e] & 0xFFFFu;
                if (kc > K) bad_knn = 1;
                else
                    for (uint32_t j = 0; j < kc; ++j) bad_knn |= kid[e * K + j] >= cur;
            }
            std::memcpy(&vv[e * dim], rec + ix.offsetData, dim * 4);
            std::memcpy(&lb[e], rec + ix.label_offset, 8);
        }
        if (bad_links) fail(HRNN_ERR_FORMAT, "loadIndex: level-0 link count or id out of range");
        if (bad_knn) fail(HRNN_ERR_FORMAT, "loadIndex: KNN-graph count or id out of range");
        CUDA_CHECK(cudaMemcpy(ix.adj0.as<uint32_t>() + base * W, a0.data(), c * W * 4, cudaMemcpyHostToDevice));
        if (K > 0) {
            CUDA_CHECK(cudaMemcpy(ix.knn_hdr.as<uint32_t>() + base, kh.data(), c * 4, cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMemcpy(ix.knn_ids.as<uint32_t>() + base * K, kid.data(), c * K * 4, cudaMemcpyHostToDevice));
            CUDA_CHECK(cudaMemcpy(ix.knn_dist.as<float>() + base * K, kd.data(), c * K * 4, cudaMemcpyHostToDevice));
        }
        CUDA_CHECK(cudaMemcpy(ix.vec.as<float>() + base * dim, vv.data(), c * dim * 4, cudaMemcpyHostToDevice));
        CUDA_CHECK(cudaMemcpy(ix.labels.as<uint64_t>() + base, lb.data(), c * 8, cudaMemcpyHostToDevice));
        for (size_t e = 0; e < c; ++e) ix.label_lookup[lb[e]] = (uint32_t)(base + e);
    }
    // Upper layers: (u32 size, blob) per element (hrnn.h:1008-1021).
    ix.upper.clear();
    for (size_t i = 0; i < cur; ++i) {
        uint32_t sz;
        r.pod(sz);
        ix.upper_off[i] = ix.upper.size();
        if (sz == 0) {
            ix.levels[i] = 0;
            continue;
        }
        if (sz % 4 != 0 || sz % ix.size_links_per_element != 0)
            fail(HRNN_ERR_FORMAT, "loadIndex: bad upper-layer record");
        ix.levels[i] = (int32_t)(sz / ix.size_links_per_element);
        size_t w0 = ix.upper.size();
        ix.upper.resize(w0 + sz / 4);
        r.bytes(ix.upper.data() + w0, sz);
    }
    // Upper layers: the entry point reaches maxlevel, and a link at level l leads
    // to an element that has level l (the descent then reads that element's
    // level-l block, which must exist).
    if (cur > 0 && ix.levels[ix.enterpoint] < ix.maxlevel)
        fail(HRNN_ERR_FORMAT, "loadIndex: entry point below maxlevel");
    {
        const size_t WU = 1 + ix.maxM;
        int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
        for (long long i = 0; i < (long long)cur; ++i) {
            for (int32_t l = 1; l <= ix.levels[i]; ++l) {
                const uint32_t* blk = ix.upper.data() + ix.upper_off[i] + (size_t)(l - 1) * WU;
                const uint32_t c = blk[0] & 0xFFFFu;
                if (c > ix.maxM) {
                    bad = 1;
                    break;
                }
                for (uint32_t j = 0; j < c; ++j) {
                    const uint32_t id = blk[1 + j];
                    bad |= id >= cur || ix.levels[id] < l;
                }
            }
        }
        if (bad) fail(HRNN_ERR_FORMAT, "loadIndex: upper-layer link count or id out of range");
    }
    ix.upper_dirty = true;
    ix.sync_upper_to_device();
    // Reverse CSR (hrnn.h:1024-1047).
    if (ix.rknng_built) {
        uint8_t eb;
        r.pod(eb);
        ix.wide = (eb == 8);
        r.pod(ix.rank_bits);
        size_t no;
        r.pod(no);
        std::vector<uint64_t> off(no);
        r.bytes(off.data(), no * 8);
        size_t ne;
        r.pod(ne);
        size_t esz = ix.wide ? 8 : 4;
        std::vector<char> ent(ne * esz + 1);
        r.bytes(ent.data(), ne * esz);
        uint64_t mask = 0;
        if (ix.wide) r.pod(mask);
        else {
            uint32_t m32;
            r.pod(m32);
        }
        if (no != cur + 1 || (no && off[no - 1] != ne))
            fail(HRNN_ERR_FORMAT, "loadIndex: inconsistent reverse CSR");
        // Offsets ascend from 0; every entry's owner is an element and its rank a
        // KNN-slot position (owner << rank_bits | rank, hrnn.h:1876-1880, 1910-1918).
        const uint32_t eb_bits = ix.wide ? 64u : 32u;
        if (ix.rank_bits >= eb_bits || (ix.K > 0 && ix.K > (1ull << ix.rank_bits)) || (no && off[0] != 0))
            fail(HRNN_ERR_FORMAT, "loadIndex: inconsistent reverse CSR");
        {
            int bad = 0;
            const uint64_t rmask = (1ull << ix.rank_bits) - 1;
#pragma omp parallel for schedule(static) reduction(| : bad)
            for (long long i = 1; i < (long long)no; ++i) bad |= off[i] < off[i - 1];
            if (!bad) {
#pragma omp parallel for schedule(static) reduction(| : bad)
                for (long long e = 0; e < (long long)ne; ++e) {
                    uint64_t x;
                    if (ix.wide) std::memcpy(&x, ent.data() + (size_t)e * 8, 8);
                    else {
                        uint32_t x32;
                        std::memcpy(&x32, ent.data() + (size_t)e * 4, 4);
                        x = x32;
                    }
                    bad |= (x >> ix.rank_bits) >= cur || (x & rmask) >= std::max<size_t>(ix.K, 1);
                }
            }
            if (bad) fail(HRNN_ERR_FORMAT, "loadIndex: reverse CSR offset, owner or rank out of range");
        }
        ix.csr_off.alloc(no * 8);
        ix.csr_ent.alloc(ne * esz);
        CUDA_CHECK(cudaMemcpy(ix.csr_off.p, off.data(), no * 8, cudaMemcpyHostToDevice));
        if (ne) CUDA_CHECK(cudaMemcpy(ix.csr_ent.p, ent.data(), ne * esz, cudaMemcpyHostToDevice));
        ix.csr_entries = ne;
        ix.csr_in_reference_order = true;
    }
}

// ---------------------------------------------------------------------------
// .idx writer (saveIndex, hrnn.h:861-927)
// ---------------------------------------------------------------------------

void save_idx(Index& ix, const std::string& path) {
    if (ix.serve_mode) fail(HRNN_ERR_STATE, "saveIndex: index is in serve mode");
    ensure_flat_rknng(ix);
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    Writer w;
    w.out.open(path, std::ios::binary);
    if (!w.out.is_open()) fail(HRNN_ERR_IO, "Cannot open file");
    const size_t cur = ix.cur;
    w.pod(kMagic);
    w.pod(ix.offsetLevel0);
    w.pod(ix.max_elements);
    w.pod(cur);
    w.pod(ix.size_data_per_element);
    w.pod(ix.label_offset);
    w.pod(ix.offsetData);
    w.pod(ix.maxlevel);
    w.pod(ix.enterpoint);
    w.pod(ix.maxM);
    w.pod(ix.maxM0);
    w.pod(ix.M);
    w.pod(ix.mult);
    w.pod(ix.ef_construction);
    w.pod(ix.K);
    w.pod(ix.size_knng_slot);
    w.pod(ix.offsetKNNG);
    w.pod(ix.knng_built);
    w.pod(ix.rknng_built);
    const size_t S = ix.size_data_per_element, W = 1 + ix.maxM0, K = ix.K, dim = ix.dim;
    std::vector<char> blob(std::min(cur, kChunk) * S + 1);
    std::vector<uint32_t> a0, kh, kid;
    std::vector<float> kd, vv;
    std::vector<uint64_t> lb;
    for (size_t base = 0; base < cur; base += kChunk) {
        size_t c = std::min(kChunk, cur - base);
        a0.resize(c * W);
        kh.resize(c);
        kid.resize(c * std::max<size_t>(K, 1));
        kd.resize(c * std::max<size_t>(K, 1));
        vv.resize(c * dim);
        lb.resize(c);
        CUDA_CHECK(cudaMemcpy(a0.data(), ix.adj0.as<uint32_t>() + base * W, c * W * 4, cudaMemcpyDeviceToHost));
        if (K > 0) {
            CUDA_CHECK(cudaMemcpy(kh.data(), ix.knn_hdr.as<uint32_t>() + base, c * 4, cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(kid.data(), ix.knn_ids.as<uint32_t>() + base * K, c * K * 4, cudaMemcpyDeviceToHost));
            CUDA_CHECK(cudaMemcpy(kd.data(), ix.knn_dist.as<float>() + base * K, c * K * 4, cudaMemcpyDeviceToHost));
        }
        CUDA_CHECK(cudaMemcpy(vv.data(), ix.vec.as<float>() + base * dim, c * dim * 4, cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(lb.data(), ix.labels.as<uint64_t>() + base, c * 8, cudaMemcpyDeviceToHost));
        std::memset(blob.data(), 0, c * S);
#pragma omp parallel for schedule(static)
        for (long long e = 0; e < (long long)c; ++e) {
            char* rec = blob.data() + (size_t)e * S;
            std::memcpy(rec + ix.offsetLevel0, &a0[e * W], W * 4);
            if (K > 0) {
                std::memcpy(rec + ix.offsetKNNG, &kh[e], 4);
                char* p = rec + ix.offsetKNNG + 4;
                for (size_t j = 0; j < K; ++j) {
                    std::memcpy(p + j * 8, &kid[e * K + j], 4);
                    std::memcpy(p + j * 8 + 4, &kd[e * K + j], 4);
                }
            }
            std::memcpy(rec + ix.offsetData, &vv[e * dim], dim * 4);
            std::memcpy(rec + ix.label_offset, &lb[e], 8);
        }
        w.bytes(blob.data(), c * S);
    }
    for (size_t i = 0; i < cur; ++i) {
        uint32_t sz = ix.levels[i] > 0 ? (uint32_t)(ix.size_links_per_element * ix.levels[i]) : 0;
        w.pod(sz);
        if (sz) w.bytes(ix.upper.data() + ix.upper_off[i], sz);
    }
    if (ix.rknng_built) {
        uint8_t eb = ix.wide ? 8 : 4;
        w.pod(eb);
        w.pod(ix.rank_bits);
        size_t no = ix.cur + 1, ne = ix.csr_entries;
        std::vector<uint64_t> off(no);
        std::vector<char> ent(ne * eb + 1);
        rknng_reference_order(ix, off.data(), ent.data());
        w.pod(no);
        w.bytes(off.data(), no * 8);
        w.pod(ne);
        w.bytes(ent.data(), ne * eb);
        if (ix.wide) w.pod((uint64_t)((1ull << ix.rank_bits) - 1));
        else w.pod((uint32_t)((1ull << ix.rank_bits) - 1));
    }
    w.out.close();
    if (!w.out) fail(HRNN_ERR_IO, "saveIndex: write failed");
}

// ---------------------------------------------------------------------------
// KNN slot access, serve mode, L2 order detection
// ---------------------------------------------------------------------------

void get_knng(Index& ix, uint32_t* ids, float* dists, uint32_t* cnt) {
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    size_t n = ix.cur, K = ix.K;
    if (ids && K) CUDA_CHECK(cudaMemcpy(ids, ix.knn_ids.p, n * K * 4, cudaMemcpyDeviceToHost));
    if (dists && K) CUDA_CHECK(cudaMemcpy(dists, ix.knn_dist.p, n * K * 4, cudaMemcpyDeviceToHost));
    if (cnt) {
        CUDA_CHECK(cudaMemcpy(cnt, ix.knn_hdr.p, n * 4, cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < n; ++i) cnt[i] &= 0xFFFFu;
    }
}

void set_knng(Index& ix, const uint32_t* ids, const float* dists, const uint32_t* cnt) {
    size_t n = ix.cur, K = ix.K;
    if (!K) fail(HRNN_ERR_STATE, "set_knng: index has no KNN graph slot (K_knng = 0)");
    for (size_t i = 0; i < n; ++i)
        if (cnt[i] > K) fail(HRNN_ERR_ARG, "set_knng: count exceeds K_knng");
    CUDA_CHECK(cudaStreamSynchronize(ix.stream));
    CUDA_CHECK(cudaMemcpy(ix.knn_ids.p, ids, n * K * 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(ix.knn_dist.p, dists, n * K * 4, cudaMemcpyHostToDevice));
    CUDA_CHECK(cudaMemcpy(ix.knn_hdr.p, cnt, n * 4, cudaMemcpyHostToDevice));
}

L2Order detect_l2_order() {
    // L2Space picks AVX-512 / AVX / SSE at run time (space_l2.h:217-234,
    // hnswlib.h:62-117).  GCC 13 at -march=native on the AVX-512 hosts of this
    // project keeps the SIMD chain unfused and contracts the scalar tail.
    unsigned a, b, c, d;
    L2Order o;
    bool avx = false, avx512 = false, fma = false;
    if (__get_cpuid(1, &a, &b, &c, &d)) {
        avx = (c >> 28) & 1;
        fma = (c >> 12) & 1;
    }
    if (__get_cpuid_count(7, 0, &a, &b, &c, &d)) avx512 = (b >> 16) & 1;
    o.lanes = avx512 ? 16 : (avx ? 8 : 4);
    o.fused = fma ? 2 : 0;
    return o;
}

}  // namespace hrnn
