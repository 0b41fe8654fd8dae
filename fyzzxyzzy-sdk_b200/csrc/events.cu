// Contact events of a step, published on the device.
//
// Reference behaviour (src/native/scene.cpp):
//   touch transitions        Scene::update_contacts 4655-4700: a pair starts
//                            touching when its manifold has contacts and had
//                            none the step before; a previously touching pair
//                            stops touching when it has no contacts or left
//                            the broadphase
//   Scene::publish_contact_events 9149-9264: every touching manager in pair
//                            order reports Found or Persists with its points;
//                            lost touches are merged in pair order with no
//                            points; event bodies ordered body0 < body1; point
//                            normals flipped when the manager's solver
//                            orientation (gu_order_reversed, 3276-3287)
//                            disagrees with body order; impulses are the final
//                            normal impulses of the solver rows, summed in
//                            double precision; a persisting touch is
//                            reported only while one of its bodies is an
//                            awake dynamic body (9201-9216)
//
// B200 mapping: both streams are already sorted by pair key, so each event
// finds its slot in the merged list with one binary search in the other
// stream; point windows come from a scan of the managers' contact counts.
#include "state.h"

namespace fyzz::b200 {
namespace {

__device__ __forceinline__ int32_t find_pair(const uint64_t* keys, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return (lo < n && keys[lo] == key) ? int32_t(lo) : -1;
}
// Number of entries of a sorted key stream below key.
template <class KeyAt>
__device__ __forceinline__ uint32_t rank_below(KeyAt key_at, uint32_t n, uint64_t key) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key_at(mid) < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ void fill_bodies(const DevState& s, uint64_t key, EventRecord& e) {
    const uint32_t a = uint32_t(key >> 32), b = uint32_t(key);
    const uint32_t ba = s.s_body[a], bb = s.s_body[b];
    const bool rev = ba > bb;
    e.body0 = rev ? bb : ba;
    e.body1 = rev ? ba : bb;
    e.shape0 = rev ? b : a;
    e.shape1 = rev ? a : b;
}

__global__ void k_ev_lost_flags(DevState s, uint32_t* flags) {
    const uint32_t np = *s.prev.n, nc = *s.cur.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < s.pair_cap; j += stride) {
        uint32_t lost = 0u;
        if (j < np && s.prev.count[j] > 0u) {
            const int32_t k = find_pair(s.cur.key, nc, s.prev.key[j]);
            lost = (k < 0 || s.cur.count[k] == 0u) ? 1u : 0u;
        }
        flags[j] = lost;
    }
}
__global__ void k_ev_lost_scatter(DevState s, const uint32_t* flags, const uint32_t* pos) {
    const uint32_t np = *s.prev.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += stride)
        if (flags[j]) s.ev_lost_key[pos[j]] = s.prev.key[j];
}
// Sc's active actor (scene.cpp:9207-9216): an awake dynamic body, or a
// kinematic body moving to its target or settling after it.
__device__ __forceinline__ bool awake_dynamic(const DevState& s, uint32_t body) {
    if (s.b_flags[body] & kBodyKinematic) return (s.b_sleep[body] & (kKinPending | kKinSettling)) != 0u;
    return (s.b_flags[body] & kBodyDynamic) && !(s.sleep && (s.b_sleep[body] & kSleeping));
}
// Touching managers with an event (rep, scanned into rep_pos) and their
// point counts.
__global__ void k_ev_counts(DevState s, uint32_t* rep) {
    const uint32_t nm = s.counters[kCntMan];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < s.pair_cap; m += stride) {
        bool on = false;
        uint32_t count = 0u;
        if (m < nm) {
            const uint32_t k = s.man_list[m];
            const uint64_t key = s.cur.key[k];
            const int32_t pj = s.prev_idx[k];
            const bool fresh = pj < 0 || s.prev.count[pj] == 0u;
            on = fresh || awake_dynamic(s, s.s_body[uint32_t(key >> 32)]) || awake_dynamic(s, s.s_body[uint32_t(key)]);
            count = on ? s.cur.count[k] : 0u;
        }
        rep[m] = on ? 1u : 0u;
        s.ev_cnt[m] = count;
    }
}
__global__ void k_ev_managers(DevState s, const uint32_t* rep, const uint32_t* rep_pos) {
    const uint32_t nm = s.counters[kCntMan], nl = s.counters[kCntLost];
    EventRecord* ev = static_cast<EventRecord*>(s.ev);
    EventPoint* pts = static_cast<EventPoint*>(s.ev_pts);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += stride) {
        if (!rep[m]) continue;
        const uint32_t k = s.man_list[m];
        const uint64_t key = s.cur.key[k];
        const uint32_t slot = rep_pos[m] + rank_below([&](uint32_t i) { return s.ev_lost_key[i]; }, nl, key);
        const int32_t pj = s.prev_idx[k];
        EventRecord e;
        fill_bodies(s, key, e);
        e.kind = (pj < 0 || s.prev.count[pj] == 0u) ? 0u : 1u;
        e.count = s.cur.count[k];
        e.point_offset = s.ev_pt_off[m];
        // solver orientation of the manager against body order
        const uint32_t a = uint32_t(key >> 32), b = uint32_t(key);
        const uint32_t ba = s.s_body[a], bb = s.s_body[b];
        const bool da = (s.b_flags[ba] & kBodyDynamic) != 0u, db = (s.b_flags[bb] & kBodyDynamic) != 0u;
        const bool reversed = !da || (da && db && ba < bb);
        const bool flip = reversed != (ba > bb);
        double total = 0.0;
        for (uint32_t j = 0; j < e.count; ++j) {
            const ContactPt& c = s.pts[4 * size_t(k) + j];
            EventPoint p;
            p.position[0] = c.p[0]; p.position[1] = c.p[1]; p.position[2] = c.p[2];
            p.normal[0] = flip ? -c.n[0] : c.n[0];
            p.normal[1] = flip ? -c.n[1] : c.n[1];
            p.normal[2] = flip ? -c.n[2] : c.n[2];
            p.separation = c.sep;
            p.pad = 0u;
            p.normal_impulse = double(s.nrow[4 * size_t(m) + j].applied);
            total += p.normal_impulse;
            pts[e.point_offset + j] = p;
        }
        e.normal_impulse = total;
        ev[slot] = e;
    }
}
__global__ void k_ev_lost(DevState s, const uint32_t* rep_pos) {
    const uint32_t nm = s.counters[kCntMan], nl = s.counters[kCntLost];
    const uint32_t total_pts = s.counters[kCntEvPts], total_rep = s.counters[kCntReported];
    EventRecord* ev = static_cast<EventRecord*>(s.ev);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += stride) {
        const uint64_t key = s.ev_lost_key[l];
        const uint32_t before = rank_below([&](uint32_t i) { return s.cur.key[s.man_list[i]]; }, nm, key);
        EventRecord e;
        fill_bodies(s, key, e);
        e.kind = 2u;
        e.count = 0u;
        e.point_offset = before < nm ? s.ev_pt_off[before] : total_pts;
        e.normal_impulse = 0.0;
        ev[l + (before < nm ? rep_pos[before] : total_rep)] = e;
    }
}

inline uint32_t blocks_for(uint32_t n, uint32_t t) {
    const uint32_t g = (n + t - 1) / t;
    return g == 0 ? 1 : (g < 148u * 8u ? g : 148u * 8u);
}

}  // namespace

void enqueue_events(const DevState& s, cudaStream_t st) {
    const uint32_t T = 256;
    k_ev_lost_flags<<<blocks_for(s.pair_cap, T), T, 0, st>>>(s, s.tmp_flags);
    scan_exclusive(s.tmp_flags, s.tmp_pos, s.pair_cap, s.prev.n, s.counters + kCntLost, s.scan_tmp,
                   s.scan_tmp_words, st, s.err);
    k_ev_lost_scatter<<<blocks_for(s.pair_cap, T), T, 0, st>>>(s, s.tmp_flags, s.tmp_pos);
    // the lost-touch flags are consumed: tmp_flags / tmp_pos now hold the
    // reported managers
    k_ev_counts<<<blocks_for(s.pair_cap, T), T, 0, st>>>(s, s.tmp_flags);
    scan_exclusive(s.tmp_flags, s.tmp_pos, s.pair_cap, s.counters + kCntMan, s.counters + kCntReported,
                   s.scan_tmp, s.scan_tmp_words, st, s.err);
    scan_exclusive(s.ev_cnt, s.ev_pt_off, s.pair_cap, s.counters + kCntMan, s.counters + kCntEvPts,
                   s.scan_tmp, s.scan_tmp_words, st, s.err);
    k_ev_managers<<<blocks_for(s.pair_cap, T), T, 0, st>>>(s, s.tmp_flags, s.tmp_pos);
    k_ev_lost<<<blocks_for(s.pair_cap, T), T, 0, st>>>(s, s.tmp_pos);
}

}  // namespace fyzz::b200
