// Decoupled look-back building blocks (Merrill and Garland, "Single-pass
// Parallel Prefix Scan with Decoupled Look-back", 2016), shared by the
// scans and sorts (primitives.cu) and the step's single-pass compactions
// (solver.cu).  Tiles take ids in the order their blocks start, publish
// their sum, then walk back one warp-width of predecessors at a time until
// an inclusive prefix is found, and publish their own.  Tile states carry
// the launch's epoch, so they need no reset between passes; every wait is
// bounded and reports kErrLogic instead of hanging.
#pragma once
#include "state.h"

namespace fyzz::b200 {

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

// Scan scratch: [0] epoch, [1] tile ticket, [2] finished blocks, [3] pad,
// then one 64-bit state per tile: epoch (30 bits) | status (2 bits: 1 sum
// of the tile, 2 inclusive prefix) | value (32 bits).
constexpr uint32_t kScanHeader = 4;
constexpr uint32_t kLookbackSpin = 1u << 18;
__device__ __forceinline__ unsigned long long scan_state_load(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void scan_state_store(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Warp 0 of a block (all 32 lanes): publishes tile `tile`'s sum `agg`,
// finds the exclusive prefix of the tiles before it, publishes its
// inclusive prefix and returns the exclusive one (on every lane).  Sets
// `failed` when a bounded wait gave up (the prefix is then unknown).
__device__ __forceinline__ uint32_t tile_lookback(unsigned long long* state, uint32_t tile, uint32_t agg,
                                                  uint32_t epoch, bool& failed) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned long long tag = (unsigned long long)epoch << 34;
    if (lane == 0) scan_state_store(&state[tile], tag | ((tile == 0 ? 2ull : 1ull) << 32) | agg);
    uint32_t prefix = 0;
    int64_t look = int64_t(tile) - 1;
    bool gave_up = false;
    while (look >= 0) {
        const int64_t idx = look - int64_t(lane);
        uint32_t status = 2u, value = 0u;     // before tile 0: an empty prefix
        if (idx >= 0) {
            uint32_t spins = 0;
            for (;;) {
                const unsigned long long st = scan_state_load(&state[idx]);
                status = uint32_t(st >> 32) & 3u;
                if ((st >> 34) == epoch && status != 0u) { value = uint32_t(st); break; }
                if (++spins == kLookbackSpin) { gave_up = true; status = 2u; value = 0u; break; }
            }
        }
        const uint32_t pmask = __ballot_sync(0xffffffffu, status == 2u);
        const int stop = pmask ? __ffs(pmask) - 1 : 31;
        uint32_t part = int(lane) <= stop ? value : 0u;
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
        prefix += part;
        if (pmask) break;
        look -= 32;
    }
    failed = __any_sync(0xffffffffu, gave_up);
    if (lane == 0 && tile != 0) scan_state_store(&state[tile], tag | (2ull << 32) | (prefix + agg));
    return prefix;
}

// Single-pass stable compaction over [0, lim) by a resident grid of
// kScanThreads-thread blocks: tiles of kScanTile elements are taken in
// ticket order; count(i) (0 or 1, with any side effects) for each of a
// thread's kScanItems consecutive elements, the block's scan, the tile's
// look-back, then emit(i, position) for every counted element, and
// last(total) once, by the block of the last tile (or with total 0 when
// lim is 0).  tmp is the scan scratch.
template <class Count, class Emit, class Last>
__device__ __forceinline__ void compact_tiles(uint32_t lim, uint32_t* tmp, uint32_t* err, Count count, Emit emit,
                                              Last last) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    __shared__ uint32_t s_tile, s_prefix;
    unsigned long long* state = reinterpret_cast<unsigned long long*>(tmp + kScanHeader);
    const uint32_t epoch = *reinterpret_cast<volatile uint32_t*>(&tmp[0]) & 0x3fffffffu;
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&tmp[1], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        __syncthreads();
        if (uint64_t(tile) * kScanTile >= lim) {
            if (tile == 0 && threadIdx.x == 0) last(0u);
            break;
        }
        const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
        uint32_t bits = 0, sum = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i)
            if (base + i < lim && count(base + i)) { bits |= 1u << i; ++sum; }
        uint32_t excl;
        const uint32_t agg = block_excl_scan<kScanThreads>(sum, excl, sm);
        if (threadIdx.x < 32) {
            bool failed = false;
            const uint32_t prefix = tile_lookback(state, tile, agg, epoch, failed);
            if (threadIdx.x == 0) {
                if (failed && err) atomicOr(err, kErrLogic);
                s_prefix = prefix;
                if (uint64_t(tile + 1) * kScanTile >= lim) last(prefix + agg);
            }
        }
        __syncthreads();
        uint32_t at = excl + s_prefix;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i)
            if (bits & (1u << i)) emit(base + i, at++);
    }
    // the last block to finish opens the next epoch and resets the ticket
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&tmp[2], 1u) == gridDim.x - 1) {
            tmp[0] = (epoch + 1u) & 0x3fffffffu;
            tmp[1] = 0u;
            tmp[2] = 0u;
            __threadfence();
        }
    }
}

// Resident grid of a compaction / scan over n elements: two blocks per SM
// at most.
inline uint32_t lookback_grid(uint32_t n) {
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    return nb == 0 ? 1u : nb < 296u ? nb : 296u;
}

}  // namespace fyzz::b200
