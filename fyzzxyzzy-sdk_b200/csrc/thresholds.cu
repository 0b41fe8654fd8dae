// Force-threshold stream of a step, published on the device.
//
// Reference behaviour (src/native/scene.cpp, Scene::update_threshold_stream
// 9391-9508, after the solver's force writeback 9293-9330):
//   * every touching contact manager that the step solved -- at least one
//     body dynamic and awake (dormant managers get no rows and write zero
//     impulses, 7804-7820) -- contributes one row keyed by its body pair:
//     a pair with the static world uses the key (dynamic body, world), any
//     other pair (actor0 < actor1), kinematic bodies keeping their own id;
//   * the row's threshold is the dynamic body's report threshold against
//     the world, else the smaller of the two; FLT_MAX (the default)
//     disables the row;
//   * the row's impulse is the sum, in double precision, of the manager's
//     final per-contact normal impulses; rows summing to zero are dropped
//     and a non-finite sum is an overflow error;
//   * rows are sorted by key (actor0, static world, actor1) and equal keys
//     aggregated (impulses added, thresholds min); a key exceeds when its
//     impulse is strictly greater than threshold * dt;
//   * the exceeded keys are merged with the previous step's in key order:
//     Found (new key: this step's impulse and threshold), Persists (the
//     PREVIOUS step's impulse and threshold), Lost (impulse zero, the
//     previous threshold).
//
// B200 mapping: one thread per touching manager builds the rows; the keys
// (split into two 32-bit halves) go through two stable LSD radix sorts, so
// equal keys keep the managers' canonical pair order and their impulses are
// added in that order; run heads aggregate their (short) runs; the merge
// finds each record's slot in the union of both sorted generations from two
// binary searches and two scans of the "also in the other list" flags.  The
// generations ping-pong with the contact-manager generations.
#include <cfloat>
#include "state.h"

namespace fyzz::b200 {
namespace {

__device__ __forceinline__ uint64_t th_key(uint32_t hi, uint32_t lo) { return (uint64_t(hi) << 32) | lo; }

__device__ __forceinline__ bool th_awake_dynamic(const DevState& s, uint32_t body) {
    return (s.b_flags[body] & kBodyDynamic) && !(s.sleep && (s.b_sleep[body] & kSleeping));
}

// Rows of the touching managers (one thread per manager slot).
__global__ void k_th_rows(DevState s, uint32_t* flags) {
    const uint32_t nm = s.counters[kCntMan];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < s.pair_cap; m += stride) {
        uint32_t ok = 0u;
        if (m < nm) {
            const uint32_t k = s.man_list[m];
            const uint64_t pk = s.cur.key[k];
            const uint32_t b0 = s.s_body[uint32_t(pk >> 32)], b1 = s.s_body[uint32_t(pk)];
            const uint32_t pa = b0 < b1 ? b0 : b1, pb = b0 < b1 ? b1 : b0;
            const uint32_t fa = s.b_flags[pa], fb = s.b_flags[pb];
            const bool dyn_a = (fa & kBodyDynamic) != 0u, dyn_b = (fb & kBodyDynamic) != 0u;
            if ((dyn_a || dyn_b) && (th_awake_dynamic(s, pa) || th_awake_dynamic(s, pb))) {
                const bool world = !(fa & (kBodyDynamic | kBodyKinematic)) || !(fb & (kBodyDynamic | kBodyKinematic));
                const uint32_t a0 = world ? (dyn_a ? pa : pb) : pa;
                const uint32_t a1 = world ? 0u : pb;
                const float ta = s.b_thresh[pa], tb = s.b_thresh[pb];
                const float thr = world ? s.b_thresh[a0] : (tb < ta ? tb : ta);   // std::min
                if (thr != FLT_MAX) {
                    const uint32_t count = s.cur.count[k];
                    double sum = 0.0;
                    for (uint32_t j = 0; j < count && j < 4u; ++j) sum += double(s.nrow[4 * size_t(m) + j].applied);
                    if (!isfinite(sum)) {
                        atomicOr(s.err, kErrNonFinite);
                    } else if (sum != 0.0) {
                        ok = 1u;
                        s.th_hi[m] = (a0 << 1) | (world ? 1u : 0u);
                        s.th_lo[m] = a1;
                        s.th_sum[m] = sum;
                        s.th_thr[m] = thr;
                    }
                }
            }
        }
        flags[m] = ok;
    }
}
// Compacted rows: low key half and the manager index, in manager order.
__global__ void k_th_compact(DevState s, const uint32_t* flags, const uint32_t* pos) {
    const uint32_t nm = s.counters[kCntMan];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += stride)
        if (flags[m]) {
            s.th_k[pos[m]] = s.th_lo[m];
            s.th_v[pos[m]] = m;
        }
}
// After the sort by the low half: the high halves in that order.
__global__ void k_th_gather_hi(DevState s) {
    const uint32_t n = s.counters[kCntThRows];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) s.th_k[i] = s.th_hi[s.th_v[i]];
}
// Run heads of equal keys aggregate their run in sorted (= pair) order and
// flag the keys whose impulse exceeds threshold * dt.
__global__ void k_th_aggregate(DevState s, uint32_t* flags) {
    const uint32_t n = s.counters[kCntThRows];
    const uint32_t stride = gridDim.x * blockDim.x;
    const double dt = double(s.dt);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.pair_cap; i += stride) {
        uint32_t ok = 0u;
        if (i < n) {
            const uint32_t m = s.th_v[i];
            const uint64_t key = th_key(s.th_hi[m], s.th_lo[m]);
            const bool head = i == 0 || th_key(s.th_hi[s.th_v[i - 1]], s.th_lo[s.th_v[i - 1]]) != key;
            if (head) {
                double sum = s.th_sum[m];
                float thr = s.th_thr[m];
                for (uint32_t j = i + 1; j < n; ++j) {
                    const uint32_t mj = s.th_v[j];
                    if (th_key(s.th_hi[mj], s.th_lo[mj]) != key) break;
                    sum += s.th_sum[mj];
                    const float t = s.th_thr[mj];
                    thr = t < thr ? t : thr;
                }
                ok = sum > double(thr) * dt ? 1u : 0u;
                s.th_run_sum[i] = sum;
                s.th_run_thr[i] = thr;
            }
        }
        flags[i] = ok;
    }
}
__global__ void k_th_emit(DevState s, const uint32_t* flags, const uint32_t* pos) {
    const uint32_t n = s.counters[kCntThRows];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        if (flags[i]) {
            const uint32_t m = s.th_v[i], p = pos[i];
            s.th_cur.key[p] = (uint64_t(s.th_hi[m]) << 32) | s.th_lo[m];
            s.th_cur.impulse[p] = s.th_run_sum[i];
            s.th_cur.thr[p] = s.th_run_thr[i];
        }
}
__device__ __forceinline__ uint32_t th_rank(const uint64_t* keys, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// Per record of each generation: is its key also in the other generation.
__global__ void k_th_common(DevState s) {
    const uint32_t np = *s.th_prev.n, nc = *s.th_cur.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < s.pair_cap; i += stride) {
        uint32_t in_cur = 0u, in_prev = 0u;
        if (i < np) {
            const uint32_t r = th_rank(s.th_cur.key, nc, s.th_prev.key[i]);
            in_cur = (r < nc && s.th_cur.key[r] == s.th_prev.key[i]) ? 1u : 0u;
        }
        if (i < nc) {
            const uint32_t r = th_rank(s.th_prev.key, np, s.th_cur.key[i]);
            in_prev = (r < np && s.th_prev.key[r] == s.th_cur.key[i]) ? 1u : 0u;
        }
        s.th_f0[i] = in_cur;
        s.th_f1[i] = in_prev;
    }
}
__device__ __forceinline__ ForceThresholdRecord th_record(uint64_t key, uint32_t change, double impulse, float thr) {
    ForceThresholdRecord r;
    r.actor0 = uint32_t(key >> 33);
    r.static_world = uint32_t(key >> 32) & 1u;
    r.actor1 = uint32_t(key);
    r.change = change;
    r.normal_impulse = impulse;
    r.threshold = thr;
    r.pad = 0u;
    return r;
}
// The merged change list in key order.  A record's slot is its index in
// its own generation plus the keys of the other generation below it that
// the own generation lacks (keys below it in the other list, minus the
// common keys below it, which the exclusive scans of the flags count).
__global__ void k_th_changes(DevState s) {
    const uint32_t np = *s.th_prev.n, nc = *s.th_cur.n;
    ForceThresholdRecord* out = static_cast<ForceThresholdRecord*>(s.th_changes);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < np || i < nc; i += stride) {
        if (i < np) {
            const uint64_t key = s.th_prev.key[i];
            const uint32_t r = th_rank(s.th_cur.key, nc, key);
            const uint32_t slot = i + r - s.th_p0[i];
            out[slot] = s.th_f0[i] ? th_record(key, 1u, s.th_prev.impulse[i], s.th_prev.thr[i])
                                   : th_record(key, 2u, 0.0, s.th_prev.thr[i]);
        }
        if (i < nc && !s.th_f1[i]) {
            const uint64_t key = s.th_cur.key[i];
            const uint32_t r = th_rank(s.th_prev.key, np, key);
            out[i + r - s.th_p1[i]] = th_record(key, 0u, s.th_cur.impulse[i], s.th_cur.thr[i]);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) s.counters[kCntThChanges] = np + nc - s.counters[kCntThCommon];
}
__global__ void k_th_copy_set(ThresholdSet dst, ThresholdSet src, uint32_t cap) {
    const uint32_t n = min(*src.n, cap);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        dst.key[i] = src.key[i];
        dst.impulse[i] = src.impulse[i];
        dst.thr[i] = src.thr[i];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *dst.n = min(*src.n, cap);
}

inline uint32_t th_blocks(uint32_t n, uint32_t t) {
    const uint32_t g = (n + t - 1) / t;
    return g == 0 ? 1 : (g < 148u * 8u ? g : 148u * 8u);
}
inline int th_bits(uint64_t max_value) {
    int bits = 1;
    while ((1ull << bits) <= max_value) ++bits;
    return bits;
}

}  // namespace

void enqueue_thresholds(const DevState& s, cudaStream_t st) {
    const uint32_t T = 256;
    const uint32_t g = th_blocks(s.pair_cap, T);
    k_th_rows<<<g, T, 0, st>>>(s, s.th_f0);
    scan_exclusive(s.th_f0, s.th_p0, s.pair_cap, s.counters + kCntMan, s.counters + kCntThRows, s.scan_tmp,
                   s.scan_tmp_words, st, s.err);
    k_th_compact<<<g, T, 0, st>>>(s, s.th_f0, s.th_p0);
    // stable LSD sorts: by actor1, then by (actor0, static world)
    radix_sort_pairs(s.th_k, s.th_v, s.th_k2, s.th_v2, s.pair_cap, s.counters + kCntThRows, 0,
                     th_bits(s.n_bodies), s.sort_hist, s.sort_hist_words, s.scan_tmp, s.scan_tmp_words, st, s.err,
                     s.radix_bits, s.sort_os, s.sort_os_words);
    k_th_gather_hi<<<g, T, 0, st>>>(s);
    radix_sort_pairs(s.th_k, s.th_v, s.th_k2, s.th_v2, s.pair_cap, s.counters + kCntThRows, 0,
                     th_bits(2ull * s.n_bodies + 1), s.sort_hist, s.sort_hist_words, s.scan_tmp, s.scan_tmp_words,
                     st, s.err, s.radix_bits, s.sort_os, s.sort_os_words);
    k_th_aggregate<<<g, T, 0, st>>>(s, s.th_f0);
    scan_exclusive(s.th_f0, s.th_p0, s.pair_cap, s.counters + kCntThRows, s.th_cur.n, s.scan_tmp,
                   s.scan_tmp_words, st, s.err);
    k_th_emit<<<g, T, 0, st>>>(s, s.th_f0, s.th_p0);
    // merge with the previous generation
    k_th_common<<<g, T, 0, st>>>(s);
    scan_exclusive(s.th_f0, s.th_p0, s.pair_cap, s.th_prev.n, s.counters + kCntThCommon, s.scan_tmp,
                   s.scan_tmp_words, st, s.err);
    scan_exclusive(s.th_f1, s.th_p1, s.pair_cap, s.th_cur.n, nullptr, s.scan_tmp, s.scan_tmp_words, st, s.err);
    k_th_changes<<<g, T, 0, st>>>(s);
}

void enqueue_copy_threshold_set(const ThresholdSet& dst, const ThresholdSet& src, uint32_t cap, cudaStream_t st) {
    k_th_copy_set<<<th_blocks(cap, 256), 256, 0, st>>>(dst, src, cap);
}

}  // namespace fyzz::b200
