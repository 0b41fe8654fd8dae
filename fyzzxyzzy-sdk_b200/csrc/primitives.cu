// Data-parallel primitives used by the step: exclusive scan and a stable
// LSD radix sort of (u32 key, u32 value) pairs.
//
// The scan is one launch with decoupled look-back (Merrill and Garland,
// "Single-pass Parallel Prefix Scan with Decoupled Look-back", 2016): tiles
// take ids in the order their blocks start, publish their sum, then walk back
// one warp-width of predecessors at a time until an inclusive prefix is
// found, and publish their own.  Tile states carry the launch's epoch, so
// they need no reset between scans; every wait is bounded and reports
// kErrLogic instead of hanging.
//
// The radix sort with 8-bit digits (the default) is a one-sweep LSD sort
// (Adinets and Merrill, "Onesweep: A Faster Least Significant Digit Radix
// Sort for GPUs", 2022), in 8- or 9-bit digits, whichever needs fewer
// passes: one launch counts the digits of every pass at once, then
// each pass is one launch whose tiles (taken in ticket order) rank their
// keys, publish their digit counts and find the counts of the tiles before
// them by the same bounded, epoch-tagged look-back as the scan.  Other
// digit widths (9 to 11 bits: fewer passes, larger histograms) run three
// launches per pass:
//   histogram  per 2048-key tile, 2^B bins in shared memory
//   scan       exclusive scan of the digit-major histogram (tile order
//              inside a digit preserves stability)
//   scatter    per tile: warp-level multi-split ranking with __match_any_sync
//              (ranks within a warp round), per-warp running digit counts in
//              shared memory, then an exclusive scan across the 8 warps.
// Counts may live in device memory (n_dev) so the sort can follow a
// data-dependent producer inside one captured CUDA graph.
#include "lookback.cuh"

namespace fyzz::b200 {
namespace {

// A one-sweep digit state carries all its data in the word: no ordering
// against other stores is needed.
__device__ __forceinline__ void os_state_store(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__global__ void __launch_bounds__(kScanThreads) k_scan_lookback(const uint32_t* in, uint32_t* out, uint32_t n,
                                                               const uint32_t* n_dev, uint32_t* total,
                                                               uint32_t* tmp, uint32_t* err) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    __shared__ uint32_t s_tile, s_prefix;
    unsigned long long* state = reinterpret_cast<unsigned long long*>(tmp + kScanHeader);
    const uint32_t epoch = *reinterpret_cast<volatile uint32_t*>(&tmp[0]) & 0x3fffffffu;
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const unsigned long long tag = (unsigned long long)epoch << 34;
    // A resident grid takes tiles in ticket order until the input ends, so
    // every tile a block waits on belongs to a running block.
    for (;;) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&tmp[1], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        __syncthreads();
        if (uint64_t(tile) * kScanTile >= lim) {
            if (tile == 0 && threadIdx.x == 0 && total) *total = 0u;
            break;
        }
        const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        uint32_t sum = 0;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            v[i] = base + i < lim ? in[base + i] : 0u;
            sum += v[i];
        }
        uint32_t excl;
        const uint32_t agg = block_excl_scan<kScanThreads>(sum, excl, sm);
        if (threadIdx.x < 32) {
            const uint32_t lane = threadIdx.x;
            if (lane == 0) scan_state_store(&state[tile], tag | ((tile == 0 ? 2ull : 1ull) << 32) | agg);
            uint32_t prefix = 0;
            int64_t look = int64_t(tile) - 1;
            bool failed = false;
            while (look >= 0) {
                const int64_t idx = look - int64_t(lane);
                uint32_t status = 2u, value = 0u;     // before tile 0: an empty prefix
                if (idx >= 0) {
                    uint32_t spins = 0;
                    for (;;) {
                        const unsigned long long st = scan_state_load(&state[idx]);
                        status = uint32_t(st >> 32) & 3u;
                        if ((st >> 34) == epoch && status != 0u) { value = uint32_t(st); break; }
                        if (++spins == kLookbackSpin) { failed = true; status = 2u; value = 0u; break; }
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
            if (__any_sync(0xffffffffu, failed) && lane == 0 && err) atomicOr(err, kErrLogic);
            if (lane == 0) {
                if (tile != 0) scan_state_store(&state[tile], tag | (2ull << 32) | (prefix + agg));
                s_prefix = prefix;
                if (total && uint64_t(tile + 1) * kScanTile >= lim) *total = prefix + agg;
            }
        }
        __syncthreads();
        uint32_t run = excl + s_prefix;
#pragma unroll
        for (int i = 0; i < kScanItems; ++i) {
            if (base + i < lim) out[base + i] = run;
            run += v[i];
        }
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

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;
constexpr int kSortWarps = kSortThreads / 32;

template <int B>
__global__ void __launch_bounds__(kSortThreads) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n,
                                                            const uint32_t* n_dev, int shift,
                                                            uint32_t* __restrict__ hist, uint32_t ntiles) {
    constexpr uint32_t R = 1u << B;
    __shared__ uint32_t h[R];
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    for (uint32_t d = threadIdx.x; d < R; d += kSortThreads) h[d] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    for (int i = threadIdx.x; i < kSortTile; i += kSortThreads) {
        const uint32_t idx = base + i;
        if (idx < lim) atomicAdd(&h[(keys[idx] >> shift) & (R - 1u)], 1u);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < R; d += kSortThreads) hist[d * ntiles + blockIdx.x] = h[d];
}

// Shared memory of k_radix_scatter<B>: running digit counts of each warp
// and their exclusive scan across warps (one invalid-key bin each).
template <int B> constexpr size_t scatter_smem() { return 2 * size_t(kSortWarps) * ((1u << B) + 1) * 4; }

template <int B>
__global__ void __launch_bounds__(kSortThreads) k_radix_scatter(const uint32_t* __restrict__ kin,
                                                               const uint32_t* __restrict__ vin,
                                                               uint32_t* __restrict__ kout,
                                                               uint32_t* __restrict__ vout, uint32_t n,
                                                               const uint32_t* n_dev, int shift,
                                                               const uint32_t* __restrict__ offs, uint32_t ntiles) {
    constexpr uint32_t R = 1u << B;
    extern __shared__ uint32_t sm[];
    uint32_t* wcount = sm;                         // [warp][R + 1]
    uint32_t* wofs = sm + kSortWarps * (R + 1);    // [warp][R + 1]
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t i = threadIdx.x; i < kSortWarps * (R + 1); i += kSortThreads) wcount[i] = 0;
    __syncthreads();
    const uint32_t wbase = blockIdx.x * kSortTile + warp * 32 * kSortItems;
    uint32_t key[kSortItems], val[kSortItems], dig[kSortItems], rank[kSortItems];
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t* wc = wcount + warp * (R + 1);
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        const uint32_t idx = wbase + r * 32 + lane;
        const bool valid = idx < lim;
        key[r] = valid ? kin[idx] : 0u;
        val[r] = valid ? vin[idx] : 0u;
        dig[r] = valid ? ((key[r] >> shift) & (R - 1u)) : R;
        const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
        const int leader = __ffs(peers) - 1;
        const uint32_t base = wc[dig[r]];
        __syncwarp();
        if (lane == leader) wc[dig[r]] = base + __popc(peers);
        __syncwarp();
        rank[r] = base + __popc(peers & lt);
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < R; d += kSortThreads) {
        uint32_t s = 0;
        for (int w = 0; w < kSortWarps; ++w) {
            wofs[w * (R + 1) + d] = s;
            s += wcount[w * (R + 1) + d];
        }
    }
    __syncthreads();
    const uint32_t* wo = wofs + warp * (R + 1);
    // offsets from a scan that gave up a wait are unknown: nothing lands
    // outside the output (the scan reported the error)
#pragma unroll
    for (int r = 0; r < kSortItems; ++r) {
        if (dig[r] < R) {
            const uint32_t pos = offs[dig[r] * ntiles + blockIdx.x] + wo[dig[r]] + rank[r];
            if (pos < lim) {
                kout[pos] = key[r];
                vout[pos] = val[r];
            }
        }
    }
}

// ---- one-sweep passes (8- or 9-bit digits) ----
// Scratch (zeroed when allocated): [0] epoch, [1] tile ticket, [2] finished
// blocks, [3] pad, then kOsMaxPasses x 512 digit totals, then one 64-bit
// state per tile and digit (512 a tile): epoch (30 bits) | status (2 bits:
// 1 count of the tile, 2 inclusive count) | value (32 bits).
constexpr int kOsMaxPasses = 4, kOsMaxDigits = 512;
constexpr uint32_t kOsHeader = 4, kOsHist = kOsMaxPasses * kOsMaxDigits;
constexpr int kOsLook = 8;   // predecessors read together in the look-back

// Digit totals of every pass (ghist must be zero).
template <int B>
__global__ void __launch_bounds__(kSortThreads) k_os_hist(const uint32_t* __restrict__ keys, uint32_t n,
                                                         const uint32_t* n_dev, int begin_bit, int passes,
                                                         uint32_t* ghist) {
    constexpr uint32_t R = 1u << B;
    __shared__ uint32_t h[kOsMaxPasses * R];
    for (int i = threadIdx.x; i < passes * int(R); i += kSortThreads) h[i] = 0u;
    __syncthreads();
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    for (uint32_t idx = blockIdx.x * kSortThreads + threadIdx.x; idx < lim; idx += gridDim.x * kSortThreads) {
        const uint32_t k = keys[idx];
        for (int p = 0; p < passes; ++p) atomicAdd(&h[p * R + ((k >> (begin_bit + B * p)) & (R - 1u))], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * int(R); i += kSortThreads)
        if (h[i]) atomicAdd(&ghist[i], h[i]);
}

// One pass: ranks a tile's keys by digit (stable), then places them at the
// digit's global offset + the counts of the digit in earlier tiles + the
// rank.  Thread t looks after digits t, t + 256, ...
template <int B>
__global__ void __launch_bounds__(kSortThreads) k_os_scatter(const uint32_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin,
                                                            uint32_t* __restrict__ kout,
                                                            uint32_t* __restrict__ vout, uint32_t n,
                                                            const uint32_t* n_dev, int shift,
                                                            const uint32_t* __restrict__ ghist, uint32_t* ctl,
                                                            unsigned long long* state, uint32_t* err) {
    constexpr uint32_t R = 1u << B, DPT = R / kSortThreads;   // digits a thread looks after
    __shared__ uint32_t wcount[kSortWarps][R + 1];
    __shared__ uint32_t wofs[kSortWarps][R + 1];
    __shared__ uint32_t base_d[R];
    __shared__ uint32_t sm_scan[kSortThreads / 32 + 1];
    __shared__ uint32_t s_tile;
    // blocks beyond the live tiles leave before taking a ticket
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    const uint32_t live = uint32_t((uint64_t(lim) + kSortTile - 1) / kSortTile);
    if (blockIdx.x >= live) return;
    const uint32_t epoch = *reinterpret_cast<volatile uint32_t*>(&ctl[0]) & 0x3fffffffu;
    const unsigned long long tag = (unsigned long long)epoch << 34;
    if (threadIdx.x == 0) s_tile = atomicAdd(&ctl[1], 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (uint32_t i = threadIdx.x; i < kSortWarps * (R + 1); i += kSortThreads) (&wcount[0][0])[i] = 0u;
        __syncthreads();
        const uint32_t wbase = tile * kSortTile + warp * 32 * kSortItems;
        uint32_t key[kSortItems], val[kSortItems], dig[kSortItems], rank[kSortItems];
        const uint32_t lt = (1u << lane) - 1u;
        uint32_t* wc = wcount[warp];
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) {
            const uint32_t idx = wbase + r * 32 + lane;
            const bool valid = idx < lim;
            key[r] = valid ? kin[idx] : 0u;
            val[r] = valid ? vin[idx] : 0u;
            dig[r] = valid ? ((key[r] >> shift) & (R - 1u)) : R;
            const uint32_t peers = __match_any_sync(0xffffffffu, dig[r]);
            const int leader = __ffs(peers) - 1;
            const uint32_t base = wc[dig[r]];
            __syncwarp();
            if (lane == leader) wc[dig[r]] = base + __popc(peers);
            __syncwarp();
            rank[r] = base + __popc(peers & lt);
        }
        __syncthreads();
        // thread t: digits t * DPT .. t * DPT + DPT - 1 (consecutive, so the
        // block scan of their totals gives each its global offset)
        uint32_t cnt[DPT], gtot = 0, gsum[DPT];
#pragma unroll
        for (uint32_t e = 0; e < DPT; ++e) {
            const uint32_t d = threadIdx.x * DPT + e;
            uint32_t c = 0;
            for (int w = 0; w < kSortWarps; ++w) {
                wofs[w][d] = c;
                c += wcount[w][d];
            }
            cnt[e] = c;
            gsum[e] = gtot;
            gtot += ghist[d];
        }
        uint32_t gx;
        block_excl_scan<kSortThreads>(gtot, gx, sm_scan);
        bool failed = false;
#pragma unroll
        for (uint32_t e = 0; e < DPT; ++e) {
            const uint32_t d = threadIdx.x * DPT + e;
            unsigned long long* my = state + size_t(tile) * R + d;
            os_state_store(my, tag | ((tile == 0 ? 2ull : 1ull) << 32) | cnt[e]);
        }
#pragma unroll
        for (uint32_t e = 0; e < DPT; ++e) {
            const uint32_t d = threadIdx.x * DPT + e;
            // look-back over kOsLook predecessors at a time (their loads in
            // flight together): sum tile counts until an inclusive count
            uint32_t prefix = 0;
            bool found = tile == 0;
            for (int64_t look = int64_t(tile) - 1; !found && !failed; look -= kOsLook) {
                unsigned long long st[kOsLook];
#pragma unroll
                for (int k = 0; k < kOsLook; ++k)
                    st[k] = look - k >= 0 ? scan_state_load(state + size_t(look - k) * R + d) : (tag | (2ull << 32));
#pragma unroll
                for (int k = 0; k < kOsLook; ++k) {
                    if (found || failed) break;
                    uint32_t spins = 0;
                    while (!((st[k] >> 34) == epoch && ((st[k] >> 32) & 3u) != 0u)) {
                        if (++spins == kLookbackSpin) { failed = true; break; }
                        st[k] = scan_state_load(state + size_t(look - k) * R + d);
                    }
                    if (failed) break;
                    prefix += uint32_t(st[k]);
                    found = ((st[k] >> 32) & 3u) == 2u;
                }
            }
            if (tile != 0) os_state_store(state + size_t(tile) * R + d, tag | (2ull << 32) | (prefix + cnt[e]));
            base_d[d] = gx + gsum[e] + prefix;
        }
        if (failed && err) atomicOr(err, kErrLogic);
        __syncthreads();
        // a look-back that gave up leaves the offsets unknown: the step
        // reports the error and nothing lands outside the output
#pragma unroll
        for (int r = 0; r < kSortItems; ++r) {
            if (dig[r] < R) {
                const uint32_t pos = base_d[dig[r]] + wofs[warp][dig[r]] + rank[r];
                if (pos < lim) {
                    kout[pos] = key[r];
                    vout[pos] = val[r];
                } else if (err) {
                    atomicOr(err, kErrLogic);
                }
            }
        }
    }
    // the last live block to finish opens the next epoch and resets the ticket
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctl[2], 1u) == live - 1) {
            ctl[0] = (epoch + 1u) & 0x3fffffffu;
            ctl[1] = 0u;
            ctl[2] = 0u;
            __threadfence();
        }
    }
}

// The live entries of a sort that ended in the alternate buffers, copied
// back.
__global__ void k_copy_live(const uint32_t* __restrict__ ks, const uint32_t* __restrict__ vs, uint32_t* kd,
                            uint32_t* vd, uint32_t n, const uint32_t* n_dev) {
    const uint32_t lim = n_dev ? min(n, *n_dev) : n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < lim; i += gridDim.x * blockDim.x) {
        kd[i] = ks[i];
        vd[i] = vs[i];
    }
}

template <int B>
void onesweep_sort(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint32_t n_cap,
                   const uint32_t* n_dev, int begin_bit, int passes, uint32_t ntiles, uint32_t* os_scratch,
                   cudaStream_t st, uint32_t* err) {
    uint32_t* ghist = os_scratch + kOsHeader;
    auto* state = reinterpret_cast<unsigned long long*>(os_scratch + kOsHeader + kOsHist);
    cudaMemsetAsync(ghist, 0, size_t(passes) * (1u << B) * 4, st);
    k_os_hist<B><<<ntiles < 296u ? ntiles : 296u, kSortThreads, 0, st>>>(keys, n_cap, n_dev, begin_bit, passes,
                                                                         ghist);
    uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    for (int p = 0; p < passes; ++p) {
        k_os_scatter<B><<<ntiles, kSortThreads, 0, st>>>(ki, vi, ko, vo, n_cap, n_dev, begin_bit + B * p,
                                                          ghist + (1u << B) * p, os_scratch, state, err);
        uint32_t* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    if (passes & 1) {
        const uint32_t nb = (n_cap + 255) / 256;
        k_copy_live<<<nb < 1184u ? nb : 1184u, 256, 0, st>>>(ki, vi, keys, vals, n_cap, n_dev);
    }
}

template <int B>
void radix_pass(const uint32_t* ki, const uint32_t* vi, uint32_t* ko, uint32_t* vo, uint32_t n_cap,
                const uint32_t* n_dev, int shift, uint32_t* hist, uint32_t ntiles, uint32_t* scan_tmp,
                size_t scan_words, cudaStream_t st, uint32_t* err) {
    k_radix_hist<B><<<ntiles, kSortThreads, 0, st>>>(ki, n_cap, n_dev, shift, hist, ntiles);
    scan_exclusive(hist, hist, (1u << B) * ntiles, nullptr, nullptr, scan_tmp, scan_words, st, err);
    k_radix_scatter<B><<<ntiles, kSortThreads, scatter_smem<B>(), st>>>(ki, vi, ko, vo, n_cap, n_dev, shift, hist,
                                                                         ntiles);
}

}  // namespace

size_t scan_tmp_words_for(uint32_t n_cap) {
    return kScanHeader + 2 * (size_t((n_cap + kScanTile - 1) / kScanTile) + 1);
}

// The scratch must be zero when first used (world allocation clears it).
void scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, const uint32_t* n_dev,
                    uint32_t* total, uint32_t* tmp, size_t tmp_words, cudaStream_t st, uint32_t* err) {
    const uint32_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) {
        if (total) cudaMemsetAsync(total, 0, 4, st);
        return;
    }
    if (scan_tmp_words_for(n) > tmp_words) {   // never: callers size the scratch for their largest scan
        if (err) cudaMemsetAsync(err, 0xff, 4, st);
        return;
    }
    // two blocks per SM at most: the whole grid is resident
    k_scan_lookback<<<nb < 296u ? nb : 296u, kScanThreads, 0, st>>>(in, out, n, n_dev, total, tmp, err);
}

size_t onesweep_words(uint32_t n_cap) {
    const size_t ntiles = (size_t(n_cap) + kSortTile - 1) / kSortTile;
    return kOsHeader + kOsHist + 2 * size_t(kOsMaxDigits) * ntiles;
}

size_t radix_hist_words(uint32_t n_cap) {
    const uint32_t ntiles = (n_cap + kSortTile - 1) / kSortTile;
    return (size_t(1) << kRadixMaxBits) * ntiles + 1;
}

void init_primitive_kernels() {
    cudaFuncSetAttribute(k_radix_scatter<10>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(scatter_smem<10>()));
    cudaFuncSetAttribute(k_radix_scatter<11>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(scatter_smem<11>()));
}

// Sorts bits [begin_bit, end_bit) of the keys (the other bits must be equal
// across keys or zero) in passes of digit_bits (8..11) bits; the result
// ends in keys/vals.
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      uint32_t n_cap, const uint32_t* n_dev, int begin_bit, int end_bit,
                      uint32_t* hist, size_t hist_words, uint32_t* scan_tmp, size_t scan_words,
                      cudaStream_t st, uint32_t* err, int digit_bits, uint32_t* os_scratch, size_t os_words) {
    const uint32_t ntiles = (n_cap + kSortTile - 1) / kSortTile;
    if (ntiles == 0) return;
    const int B = digit_bits >= 8 && digit_bits <= kRadixMaxBits ? digit_bits : 8;
    // one-sweep passes: 8- or 9-bit digits, whichever needs fewer passes
    const int width = end_bit - begin_bit;
    const int os_b = (width + 8) / 9 < (width + 7) / 8 ? 9 : 8;
    const int os_passes = (width + os_b - 1) / os_b;
    if (B == 8 && os_scratch && os_passes <= kOsMaxPasses) {
        if (onesweep_words(n_cap) > os_words) {   // never: the world sizes the scratch for its largest sort
            if (err) cudaMemsetAsync(err, 0xff, 4, st);
            return;
        }
        if (os_b == 9) onesweep_sort<9>(keys, vals, keys_alt, vals_alt, n_cap, n_dev, begin_bit, os_passes, ntiles,
                                        os_scratch, st, err);
        else onesweep_sort<8>(keys, vals, keys_alt, vals_alt, n_cap, n_dev, begin_bit, os_passes, ntiles,
                              os_scratch, st, err);
        return;
    }
    uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    int passes = 0;
    for (int shift = begin_bit; shift < end_bit; shift += B, ++passes) {
        switch (B) {
            case 9: radix_pass<9>(ki, vi, ko, vo, n_cap, n_dev, shift, hist, ntiles, scan_tmp, scan_words, st, err); break;
            case 10: radix_pass<10>(ki, vi, ko, vo, n_cap, n_dev, shift, hist, ntiles, scan_tmp, scan_words, st, err); break;
            case 11: radix_pass<11>(ki, vi, ko, vo, n_cap, n_dev, shift, hist, ntiles, scan_tmp, scan_words, st, err); break;
            default: radix_pass<8>(ki, vi, ko, vo, n_cap, n_dev, shift, hist, ntiles, scan_tmp, scan_words, st, err); break;
        }
        uint32_t* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
    }
    if (passes & 1) {
        cudaMemcpyAsync(keys, ki, size_t(n_cap) * 4, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, vi, size_t(n_cap) * 4, cudaMemcpyDeviceToDevice, st);
    }
}

}  // namespace fyzz::b200
