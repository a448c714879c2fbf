// Exclusive prefix sums (u64 and u32 -> u64) on the device: per-tile scan with
// a recursive pass over the tile totals.  Used for CSR offsets and for packing
// per-query results.
#include "index.hpp"

namespace hrnn {

namespace {

constexpr int kScanThreads = 512;
constexpr int kPerThread = 8;
constexpr int kTile = kScanThreads * kPerThread;

template <class In>
__global__ void scan_tiles(const In* __restrict__ in, uint64_t* __restrict__ out, size_t n,
                           uint64_t* __restrict__ tile_sums) {
    __shared__ uint64_t warp_tot[kScanThreads / 32];
    size_t base = (size_t)blockIdx.x * kTile + (size_t)threadIdx.x * kPerThread;
    uint64_t v[kPerThread];
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        v[k] = (base + k < n) ? (uint64_t)in[base + k] : 0;
        s += v[k];
    }
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint64_t incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        uint64_t t = lane < kScanThreads / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < kScanThreads / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    uint64_t run = incl - s + (w ? warp_tot[w - 1] : 0);
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
    if (threadIdx.x == kScanThreads - 1 && tile_sums) tile_sums[blockIdx.x] = warp_tot[kScanThreads / 32 - 1];
}

__global__ void add_tile_offsets(uint64_t* __restrict__ out, size_t n, const uint64_t* __restrict__ offs) {
    size_t base = (size_t)blockIdx.x * kTile;
    uint64_t add = offs[blockIdx.x];
    for (int k = threadIdx.x; k < kTile; k += kScanThreads)
        if (base + k < n) out[base + k] += add;
}

template <class In>
void scan_impl(const In* in, uint64_t* out, size_t n, cudaStream_t s, DevMem& tmp, size_t tmp_off) {
    if (n == 0) return;
    size_t tiles = (n + kTile - 1) / kTile;
    if (tiles == 1) {
        scan_tiles<In><<<1, kScanThreads, 0, s>>>(in, out, n, nullptr);
        CUDA_LAUNCH_CHECK();
        return;
    }
    // tmp layout: [tile sums | tile offsets] per recursion level
    size_t need = (tmp_off + 2 * tiles) * 8;
    if (tmp.bytes < need) fail(HRNN_ERR_NOMEM, "scan: scratch too small");
    uint64_t* sums = tmp.as<uint64_t>() + tmp_off;
    uint64_t* offs = sums + tiles;
    scan_tiles<In><<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, n, sums);
    CUDA_LAUNCH_CHECK();
    scan_impl<uint64_t>(sums, offs, tiles, s, tmp, tmp_off + 2 * tiles);
    add_tile_offsets<<<(unsigned)tiles, kScanThreads, 0, s>>>(out, n, offs);
    CUDA_LAUNCH_CHECK();
}

size_t scan_tmp_words(size_t n) {
    size_t w = 0;
    while (n > (size_t)kTile) {
        size_t tiles = (n + kTile - 1) / kTile;
        w += 2 * tiles;
        n = tiles;
    }
    return w + 16;
}

}  // namespace

void exclusive_scan_u64(const uint64_t* in, uint64_t* out, size_t n, cudaStream_t s, DevMem& tmp) {
    tmp.ensure(scan_tmp_words(n) * 8);
    scan_impl<uint64_t>(in, out, n, s, tmp, 0);
}

void exclusive_scan_u32_to_u64(const uint32_t* in, uint64_t* out, size_t n, cudaStream_t s,
                               DevMem& tmp) {
    tmp.ensure(scan_tmp_words(n) * 8);
    scan_impl<uint32_t>(in, out, n, s, tmp, 0);
}

}  // namespace hrnn
