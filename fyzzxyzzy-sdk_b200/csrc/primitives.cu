// Data-parallel primitives used by the step: exclusive scan and a stable
// LSD radix sort of (u32 key, u32 value) pairs.
//
// The radix sort processes 8-bit digits.  Each pass is three launches:
//   histogram  per 2048-key tile, 256 bins in shared memory
//   scan       exclusive scan of the digit-major histogram (tile order
//              inside a digit preserves stability)
//   scatter    per tile: warp-level multi-split ranking with __match_any_sync
//              (ranks within a warp round), per-warp running digit counts in
//              shared memory, then an exclusive scan across the 8 warps.
// Counts may live in device memory (n_dev) so the sort can follow a
// data-dependent producer inside one captured CUDA graph.
#include "state.h"

namespace fyzz::b200 {
namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive block scan of one value per thread; returns the block total.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t& excl, uint32_t* smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inc = warp_incl_scan(v);
    if (lane == 31) smem[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < THREADS / 32 ? smem[lane] : 0u;
        const uint32_t wi = warp_incl_scan(w);
        if (lane < THREADS / 32) smem[lane] = wi - w;
        if (lane == THREADS / 32 - 1) smem[THREADS / 32] = wi;
    }
    __syncthreads();
    excl = inc - v + smem[warp];
    const uint32_t total = smem[THREADS / 32];
    __syncthreads();
    return total;
}

__global__ void k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n, const uint32_t* n_dev,
                              uint32_t* __restrict__ sums) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < lim) s += in[base + i];
    uint32_t excl;
    const uint32_t total = block_excl_scan<kScanThreads>(s, excl, sm);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void k_scan_sums(uint32_t* sums, uint32_t nb, uint32_t* total) {
    __shared__ uint32_t sm[1024 / 32 + 1];
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < nb; base += 1024) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < nb ? sums[i] : 0u;
        uint32_t excl;
        const uint32_t t = block_excl_scan<1024>(v, excl, sm);
        if (i < nb) sums[i] = excl + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += t;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void k_scan_apply(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t n,
                             const uint32_t* n_dev, const uint32_t* __restrict__ sums) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const uint32_t base = blockIdx.x * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < lim ? in[base + i] : 0u;
        s += v[i];
    }
    uint32_t excl;
    block_excl_scan<kScanThreads>(s, excl, sm);
    uint32_t run = excl + sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < lim) out[base + i] = run;
        run += v[i];
    }
}

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

__global__ void k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, const uint32_t* n_dev,
                             int shift, uint32_t* __restrict__ hist, uint32_t ntiles) {
    __shared__ uint32_t h[256];
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        const uint32_t idx = base + i;
        if (idx < lim) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void k_radix_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                uint32_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                uint32_t n, const uint32_t* n_dev, int shift,
                                const uint32_t* __restrict__ offs, uint32_t ntiles) {
    __shared__ uint32_t wcount[kSortWarps][257];
    __shared__ uint32_t wofs[kSortWarps][257];
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kSortWarps * 257; i += kSortThreads) (&wcount[0][0])[i] = 0;
    __syncthreads();
    const uint32_t wbase = blockIdx.x * kSortTile + warp * 32 * kSortItems;
    uint32_t key[kSortItems], val[kSortItems], dig[kSortItems], rank[kSortItems];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        const bool valid = idx < lim;
        key[r] = valid ? kin[idx] : 0u;
        val[r] = valid ? vin[idx] : 0u;
        dig[r] = valid ? ((key[r] >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
        const int leader = __ffs(peers) - 1;
        const uint32_t base = wcount[warp][dig[r]];
        __syncwarp();
        if (lane == leader) wcount[warp][dig[r]] = base + __popc(peers);
        __syncwarp();
        rank[r] = base + __popc(peers & lt);
    }
    __syncthreads();
    {
        uint32_t s = 0;
        for (int w = 0; w < kSortWarps; ++w) {
            wofs[w][threadIdx.x] = s;
            s += wcount[w][threadIdx.x];
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        if (dig[r] < 256u) {
            const uint32_t pos = offs[dig[r] * ntiles + blockIdx.x] + wofs[warp][dig[r]] + rank[r];
            kout[pos] = key[r];
            vout[pos] = val[r];
        }
    }
}

}  // namespace

size_t scan_tmp_words_for(uint32_t n_cap) {
    return (n_cap + kScanTile - 1) / kScanTile + 1;
}

void scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, const uint32_t* n_dev,
                    uint32_t* total, uint32_t* tmp, size_t tmp_words, cudaStream_t st) {
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) {
        if (total) cudaMemsetAsync(total, 0, 4, st);
        return;
    }
    (void)tmp_words;
    k_scan_reduce<<<nb, kScanThreads, 0, st>>>(in, n, n_dev, tmp);
    k_scan_sums<<<1, 1024, 0, st>>>(tmp, nb, total);
    k_scan_apply<<<nb, kScanThreads, 0, st>>>(in, out, n, n_dev, tmp);
}

size_t radix_hist_words(uint32_t n_cap) {
    const uint32_t ntiles = (n_cap + kSortTile - 1) / kSortTile;
    return size_t(256) * ntiles + 1;
}

// Sorts bits [begin_bit, end_bit) of the keys; the result ends in keys/vals.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      uint32_t n_cap, const uint32_t* n_dev, int begin_bit, int end_bit,
                      uint32_t* hist, size_t hist_words, uint32_t* scan_tmp, size_t scan_words,
                      cudaStream_t st) {
    const uint32_t ntiles = (n_cap + kSortTile - 1) / kSortTile;
    if (ntiles == 0) return;
    (void)hist_words;
    uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += 8, ++passes) {
        k_radix_hist<<<ntiles, kSortThreads, 0, st>>>(ki, n_cap, n_dev, shift, hist, ntiles);
        scan_exclusive(hist, hist, 256u * ntiles, nullptr, nullptr, scan_tmp, scan_words, st);
        k_radix_scatter<<<ntiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n_cap, n_dev, shift, hist, ntiles);
        uint32_t* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    if (passes & 1) {
        cudaMemcpyAsync(keys, ki, size_t(n_cap) * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, vi, size_t(n_cap) * 4, cudaMemcpyDeviceToDevice, st);
    }
}

}  // namespace fyzz::b200
