// hrnn_build_rknng_noalloc: the reverse-KNN CSR transpose of a KNN graph that
// the caller owns, for callers that cannot allocate device memory -- for
// example code that manages every device byte through its own arena, or a
// serving loop that must not call cudaMalloc (which can synchronise the device).
// The caller passes the graph and the output buffers; the scratch the transpose
// needs (in-degree counters, scatter cursors, the prefix-sum partials, the list
// of long segments and their sort staging) lives in one file-scope __device__
// array of kScratchBytes.
//
// Host code cannot use that array's name as a device address: the device
// address is obtained once per device with cudaGetSymbolAddress, on the first
// call with that device current (and again if the device's context was
// re-created since, e.g. by cudaDeviceReset).  Make that first call before any
// stream capture.  All calls share the array, so calls that overlap on the GPU (two
// streams, two threads) race; run them one after the other.  The array keeps the
// last call's contents; every region that must start at zero is cleared here.
//
// Output: offsets (n+1, u64) and entries ((owner << rank_bits) | rank; u32 when
// node_bits + rank_bits <= 32, else u64), every segment in (rank, owner) order --
// the same bytes as hrnn_get_rknng(..., reference_order = 0) after
// hrnn_build_rknng on the same graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "index.hpp"

namespace hrnn {
namespace {

constexpr size_t kScratchBytes = 32ull << 20;  // 32 MiB, held by every device that loads the library
constexpr size_t kMaxN = 1ull << 21;           // 2,097,152 elements
constexpr int kNaWarpSegMax = 1024;
constexpr int kNaSmemKeys = 16384;
constexpr int kScanT = 512, kScanPer = 8, kScanTile = kScanT * kScanPer;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
struct ScratchSlot {
    void* ctx = nullptr;   // the device context the address belongs to
    void* addr = nullptr;
};
ScratchSlot g_slot[64];
using CtxGetCurrent = int (*)(void**);  // cuCtxGetCurrent(CUcontext*), fetched through the runtime

void* current_context() {
    static CtxGetCurrent fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrent>(f);
    }();
    void* ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// Device address of g_scratch on `dev` (current).  Looked up with
// cudaGetSymbolAddress on the first call on a device, and again when the
// device's context is not the one the cached address was taken in (after a
// cudaDeviceReset the module is loaded anew and the array may move).
void* scratch_address(int dev) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (dev < 0 || dev >= 64) fail(HRNN_ERR_ARG, "build_rknng_noalloc: device ordinal out of range");
    CUDA_CHECK(cudaSetDevice(dev));  // binds (and, after a reset, creates) the device's primary context
    void* ctx = current_context();
    ScratchSlot& sl = g_slot[dev];
    if (!sl.addr || !ctx || ctx != sl.ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p)
            fail(HRNN_ERR_CUDA, std::string("build_rknng_noalloc: cudaGetSymbolAddress failed: ") +
                                    cudaGetErrorString(e));
        sl.addr = p;
        sl.ctx = ctx ? ctx : current_context();
    }
    return sl.addr;
}

// In-degree histogram of the caller's graph, which is checked on the way: a count
// above K or an id >= n is not followed but flagged in bad[0] / bad[1], and the
// transpose stops with HRNN_ERR_ARG before anything is scattered.
__global__ void na_degree(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cnt, size_t n, uint32_t K,
                          uint32_t* __restrict__ deg, uint32_t* __restrict__ bad) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = cnt[i] & 0xFFFFu;
        if (c > K) {
            if (lane == 0) atomicAdd(&bad[0], 1u);
            continue;
        }
        for (uint32_t j = lane; j < c; j += 32) {
            const uint32_t id = ids[i * K + j];
            if (id < n) atomicAdd(&deg[id], 1u);
            else atomicAdd(&bad[1], 1u);
        }
    }
}

// Exclusive scan of deg[0..n] (deg[n] = 0) into off, tile partials in part.
__global__ void na_scan_tiles(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, size_t n,
                              uint64_t* __restrict__ part) {
    __shared__ uint64_t wt[kScanT / 32];
    size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
    uint64_t v[kScanPer], s = 0;
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t inc = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wt[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint64_t t = lane < kScanT / 32 ? wt[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kScanT / 32) wt[lane] = t;
    }
    __syncthreads();
    uint64_t run = inc - s + (w ? wt[w - 1] : 0);
#pragma unroll
    for (int k = 0; k < kScanPer; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanT - 1) part[blockIdx.x] = wt[kScanT / 32 - 1];
}

// Serial exclusive scan of the (at most kMaxN / kScanTile + 1 = 513) tile partials.
__global__ void na_scan_parts(uint64_t* part, size_t tiles) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        uint64_t run = 0;
        for (size_t i = 0; i < tiles; ++i) {
            uint64_t v = part[i];
            part[i] = run;
            run += v;
        }
    }
}

__global__ void na_scan_add(uint64_t* __restrict__ out, size_t n, const uint64_t* __restrict__ part) {
    size_t base = (size_t)blockIdx.x * kScanTile;
    for (int k = threadIdx.x; k < kScanTile; k += kScanT)
        if (base + k < n) out[base + k] += part[blockIdx.x];
}

template <class E>
__global__ void na_scatter(const uint32_t* __restrict__ ids, const uint32_t* __restrict__ cnt, size_t n, uint32_t K,
                           const uint64_t* __restrict__ off, uint32_t* __restrict__ cursor, E* __restrict__ ent,
                           uint32_t rb) {
    size_t warp = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    size_t nw = ((size_t)gridDim.x * blockDim.x) >> 5;
    for (size_t i = warp; i < n; i += nw) {
        uint32_t c = cnt[i] & 0xFFFFu;
        for (uint32_t j = lane; j < c; j += 32) {
            uint32_t nbr = ids[i * K + j];
            ent[off[nbr] + atomicAdd(&cursor[nbr], 1u)] = (E)(((uint64_t)i << rb) | j);
        }
    }
}

template <class E>
__device__ __forceinline__ uint64_t na_key(E e, uint32_t rb) {
    uint64_t v = (uint64_t)e;
    return ((v & ((1ull << rb) - 1)) << 32) | (v >> rb);
}
template <class E>
__device__ __forceinline__ E na_entry(uint64_t k, uint32_t rb) {
    return (E)(((k & 0xFFFFFFFFull) << rb) | (k >> 32));
}

template <class Sync>
__device__ void na_bitonic(uint64_t* s, uint32_t P, uint32_t t, uint32_t nt, Sync sync) {
    for (uint32_t k = 2; k <= P; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = t; i < P; i += nt) {
                uint32_t p = i ^ j;
                if (p > i) {
                    uint64_t a = s[i], b = s[p];
                    if ((a > b) == ((i & k) == 0)) {
                        s[i] = b;
                        s[p] = a;
                    }
                }
            }
            sync();
        }
}

// Segments up to 1024 entries, one warp each; longer ones are listed in `big`
// and their largest power-of-two size is tracked in *maxP.
template <class E>
__global__ void na_sort_small(const uint64_t* __restrict__ off, size_t n, E* __restrict__ ent, uint32_t rb,
                              uint32_t* __restrict__ big, uint32_t* __restrict__ nbig, uint32_t* __restrict__ maxP) {
    __shared__ uint64_t sm[4][kNaWarpSegMax];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (size_t seg = (size_t)blockIdx.x * 4 + w; seg < n; seg += (size_t)gridDim.x * 4) {
        uint64_t b = off[seg];
        uint32_t len = (uint32_t)(off[seg + 1] - b);
        if (len <= 1) continue;
        uint32_t P = 32;
        while (P < len) P <<= 1;
        if (len > kNaWarpSegMax) {
            if (lane == 0) {
                big[atomicAdd(nbig, 1u)] = (uint32_t)seg;
                atomicMax(maxP, P);
            }
            continue;
        }
        uint64_t* s = sm[w];
        for (uint32_t i = lane; i < P; i += 32) s[i] = i < len ? na_key<E>(ent[b + i], rb) : ~0ull;
        __syncwarp();
        na_bitonic(s, P, lane, 32, [] { __syncwarp(); });
        for (uint32_t i = lane; i < len; i += 32) ent[b + i] = na_entry<E>(s[i], rb);
        __syncwarp();
    }
}

// One block per long segment; keys in dynamic shared memory when they fit,
// otherwise in the staging area (stride words per block).
template <class E>
__global__ void na_sort_big(const uint64_t* __restrict__ off, const uint32_t* __restrict__ big, uint32_t first,
                            E* __restrict__ ent, uint32_t rb, uint64_t* __restrict__ stage, size_t stride) {
    extern __shared__ uint64_t dyn[];
    uint32_t seg = big[first + blockIdx.x];
    uint64_t b = off[seg];
    uint32_t len = (uint32_t)(off[seg + 1] - b);
    uint32_t P = 32;
    while (P < len) P <<= 1;
    uint64_t* s = P <= (uint32_t)kNaSmemKeys ? dyn : stage + (size_t)blockIdx.x * stride;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) s[i] = i < len ? na_key<E>(ent[b + i], rb) : ~0ull;
    __syncthreads();
    na_bitonic(s, P, threadIdx.x, blockDim.x, [] { __syncthreads(); });
    for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) ent[b + i] = na_entry<E>(s[i], rb);
}

size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

template <class E>
uint64_t transpose(const uint32_t* ids, const uint32_t* cnt, size_t n, uint32_t K, uint32_t rb, uint64_t* off,
                   void* entries, size_t cap, char* base, cudaStream_t s, int nsm) {
    // scratch layout
    const size_t tiles = (n + 1 + kScanTile - 1) / kScanTile;
    uint32_t* deg = (uint32_t*)base;
    uint32_t* cursor = (uint32_t*)(base + al256((n + 1) * 4));
    uint32_t* big = (uint32_t*)((char*)cursor + al256((n + 1) * 4));
    uint64_t* part = (uint64_t*)((char*)big + al256((n + 1) * 4));
    // ctl: [0] n_big, [1] max P, [2] counts above K, [3] ids >= n
    uint32_t* ctl = (uint32_t*)((char*)part + al256(tiles * 8));
    uint64_t* stage = (uint64_t*)((char*)ctl + 256);
    const size_t used = (size_t)((char*)stage - base);
    const size_t stage_words = (kScratchBytes - used) / 8;
    CUDA_CHECK(cudaMemsetAsync(deg, 0, (n + 1) * 4, s));
    CUDA_CHECK(cudaMemsetAsync(cursor, 0, (n + 1) * 4, s));
    CUDA_CHECK(cudaMemsetAsync(ctl, 0, 16, s));
    const int grid = nsm * 8;
    na_degree<<<grid, 256, 0, s>>>(ids, cnt, n, K, deg, ctl + 2);
    CUDA_LAUNCH_CHECK();
    na_scan_tiles<<<(unsigned)tiles, kScanT, 0, s>>>(deg, off, n + 1, part);
    CUDA_LAUNCH_CHECK();
    na_scan_parts<<<1, 32, 0, s>>>(part, tiles);
    CUDA_LAUNCH_CHECK();
    na_scan_add<<<(unsigned)tiles, kScanT, 0, s>>>(off, n + 1, part);
    CUDA_LAUNCH_CHECK();
    uint64_t total = 0;
    uint32_t badc[2] = {0, 0};
    CUDA_CHECK(cudaMemcpyAsync(&total, off + n, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaMemcpyAsync(badc, ctl + 2, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    if (badc[0] || badc[1])
        fail(HRNN_ERR_ARG, "build_rknng_noalloc: the graph has " + std::to_string(badc[0]) +
                               " count(s) above K and " + std::to_string(badc[1]) + " neighbour id(s) >= n");
    if (total > cap) return total;  // caller's entry buffer too small: report the need
    E* ent = static_cast<E*>(entries);
    na_scatter<E><<<grid, 256, 0, s>>>(ids, cnt, n, K, off, cursor, ent, rb);
    CUDA_LAUNCH_CHECK();
    unsigned blocks = (unsigned)std::min<size_t>((n + 3) / 4, (size_t)nsm * 32);
    na_sort_small<E><<<blocks ? blocks : 1, 128, 0, s>>>(off, n, ent, rb, big, ctl, ctl + 1);
    CUDA_LAUNCH_CHECK();
    uint32_t hc[2] = {0, 0};
    CUDA_CHECK(cudaMemcpyAsync(hc, ctl, 8, cudaMemcpyDeviceToHost, s));
    CUDA_CHECK(cudaStreamSynchronize(s));
    if (hc[0]) {
        const uint32_t P = hc[1];
        const size_t stride = P > (uint32_t)kNaSmemKeys ? P : 0;
        if (stride && stride > stage_words)
            fail(HRNN_ERR_LIMIT, "build_rknng_noalloc: a reverse list longer than the scratch staging allows (" +
                                     std::to_string(stage_words) + " entries)");
        const uint32_t per_launch = stride ? (uint32_t)std::min<size_t>(stage_words / stride, 65535) : 65535;
        const size_t smem = (size_t)kNaSmemKeys * 8;
        CUDA_CHECK(cudaFuncSetAttribute(na_sort_big<E>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        for (uint32_t first = 0; first < hc[0]; first += per_launch) {
            uint32_t cnt_b = std::min(per_launch, hc[0] - first);
            na_sort_big<E><<<cnt_b, 512, smem, s>>>(off, big, first, ent, rb, stage, stride);
            CUDA_LAUNCH_CHECK();
        }
    }
    CUDA_CHECK(cudaStreamSynchronize(s));
    return total;
}

}  // namespace
}  // namespace hrnn

namespace hrnn {
void set_last_error(const std::string& m);  // capi.cpp: the message hrnn_last_error() returns
}

hrnn_status hrnn_build_rknng_noalloc(const uint32_t* d_knn_ids, const uint32_t* d_knn_cnt, size_t n, size_t K,
                                     uint64_t* d_offsets, void* d_entries, size_t entries_cap, uint32_t* rank_bits,
                                     int* wide, uint64_t* n_entries, void* stream) {
    try {
        hrnn::set_last_error("");
        if (!d_knn_ids || !d_knn_cnt || !d_offsets || !d_entries)
            hrnn::fail(HRNN_ERR_ARG, "build_rknng_noalloc: a buffer pointer is NULL");
        if (n == 0 || K == 0) hrnn::fail(HRNN_ERR_ARG, "build_rknng_noalloc: n and K must be > 0");
        if (n > hrnn::kMaxN)
            hrnn::fail(HRNN_ERR_LIMIT, "build_rknng_noalloc: n = " + std::to_string(n) +
                                           " exceeds the limit of 2097152 elements of its fixed scratch");
        if (K > 0xFFFF) hrnn::fail(HRNN_ERR_ARG, "build_rknng_noalloc: K must be < 65536");
        uint32_t rb = 0, nb = 0;                      // the bit split of buildRKNNG, hrnn.h:1876-1880
        while ((1ull << rb) < K) rb++;
        while ((1ull << nb) < n) nb++;
        const bool w = nb + rb > 32;
        int dev = 0;
        CUDA_CHECK(cudaGetDevice(&dev));
        int nsm = 148;
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        char* base = static_cast<char*>(hrnn::scratch_address(dev));
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        uint64_t total = w ? hrnn::transpose<uint64_t>(d_knn_ids, d_knn_cnt, n, (uint32_t)K, rb, d_offsets, d_entries,
                                                       entries_cap, base, s, nsm)
                           : hrnn::transpose<uint32_t>(d_knn_ids, d_knn_cnt, n, (uint32_t)K, rb, d_offsets, d_entries,
                                                       entries_cap, base, s, nsm);
        if (rank_bits) *rank_bits = rb;
        if (wide) *wide = w;
        if (n_entries) *n_entries = total;
        if (total > entries_cap)
            hrnn::fail(HRNN_ERR_CAPACITY, "build_rknng_noalloc: entries buffer too small (need " +
                                              std::to_string(total) + " entries)");
        return HRNN_OK;
    } catch (const hrnn::Error& e) {
        hrnn::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        hrnn::set_last_error(e.what());
        return HRNN_ERR_STATE;
    }
}
