// Dy: unconstrained velocities, solver bodies, islands, conflict-free
// partitions, contact / friction / distance row preparation, PGS and pose
// integration.
//
// Reference routines (src/native/scene.cpp):
//   prepare_unconstrained_velocities  10383-10507
//   prepare_solver_bodies             6940-7110 (sqrt inverse inertia in world)
//   partition_constraints             7113-7488 (greedy first-fit 32-bit masks,
//                                       overflow waves, statics after the body's
//                                       last dynamic partition)
//   prepare_constraints               7490-8510 (distance rows, material
//                                       combine, friction correlation and anchor
//                                       growth, contact and tangent rows)
//   solve_constraint_task             8853-9148 (4 biased + 1 velocity pass,
//                                       friction on the last three position passes)
//   publish_solver_bodies / integrate 9509-9548, 10508-10707
//
// B200 mapping.  Descriptors are the distance joints (constraint slot
// descending) followed by the touching managers in pair order.  A lock-free
// union-find groups them into islands; a stable radix sort by island root
// keeps each island's descriptors in that order, so the per-island greedy
// partition is exactly the reference's per-task greedy (islands share no
// dynamic body).  PGS runs one warp (small islands) or one CTA (large
// islands) per island, sweeping its partitions in order with warp / block
// barriers only: no grid-wide synchronisation and no host round trip.
#include "solver_common.cuh"
#include "lookback.cuh"
#include <cfloat>
#include <type_traits>

namespace fyzz::b200 {

namespace {
constexpr uint32_t kInvalid = 0xffffffffu;
constexpr int kMaxLevels = 256;
constexpr uint32_t kSerialIsland = 32;   // partitioned by one thread

__global__ void k_frame_begin(DevState s) {
    if (threadIdx.x == 0 && blockIdx.x == 0) s.counters[kCntFrame] += 1u;
}

__device__ __forceinline__ bool is_asleep(const DevState& s, uint32_t b) {
    return s.sleep && (s.b_sleep[b] & kSleeping);
}

// Per-step resets of the body tables; counts the bodies asleep at the start
// of the step.
__global__ void k_bodies_begin(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool on = b < s.n_bodies;
    const bool dyn = on && is_dyn(s, b);
    const bool asleep = dyn && is_asleep(s, b);
    const bool ready = dyn && s.sleep && (s.b_sleep[b] & kReady);
    const uint32_t am = __activemask();
    const uint32_t votes = __ballot_sync(am, asleep), ready_votes = __ballot_sync(am, ready);
    if ((threadIdx.x & 31u) == uint32_t(__ffs(am) - 1)) {
        if (votes) atomicAdd(&s.counters[kCntSleeping], __popc(votes));
        if (ready_votes) atomicAdd(&s.counters[kCntReady], __popc(ready_votes));
    }
    if (!on) return;
    s.uf_parent[b] = b;
    s.sb_mask[b] = 0u;
    s.sb_maxdyn[b] = 0u;
    s.sb_static[b] = 0u;
    const float4 z = make_float4(0, 0, 0, 0);
    s.sb_dv[b] = z; s.sb_dw[b] = z; s.sb_mdv[b] = z; s.sb_mdw[b] = z;
    if (s.sleep) {
        s.sl_act[b] = 0u;
        s.sl_spec[b] = b;
        s.sl_root[b] = 0u;
        s.b_counted[b] = s.b_jcount[b];
    }
}

// Unconstrained velocity + solver-body data for every awake dynamic body
// (scene.cpp:10383 prepare_unconstrained_velocities skips sleeping actors).
__global__ void k_bodies_velocity(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b)) return;
    if (is_asleep(s, b)) {
        const float4 z = make_float4(0, 0, 0, 0);
        s.sb_v[b] = z;
        s.sb_w[b] = z;
        return;
    }
    const float dt = s.dt;
    const float gravity = -9.81f;
    const float4 d0 = s.b_dyn0[b];
    v3 v = ld3(s.b_v[b]);
    float vx = v.x, vy = v.y + gravity * dt, vz = v.z;
    const float lm = smax(1.0f - d0.x * dt, 0.0f);
    vx *= lm; vy *= lm; vz *= lm;
    v3 w = ld3(s.b_w[b]);
    const float am = smax(1.0f - d0.y * dt, 0.0f);
    w.x *= am; w.y *= am; w.z *= am;
    const float s2 = vx * vx + vy * vy + vz * vz;
    const float ml2 = d0.z * d0.z, ma2 = d0.w * d0.w;
    if (s2 > ml2) {
        const float f = sqrtf(ml2 / s2);
        vx *= f; vy *= f; vz *= f;
    }
    const float w2 = w.x * w.x + w.y * w.y + w.z * w.z;
    if (w2 > ma2) {
        const float f = sqrtf(ma2 / w2);
        w.x *= f; w.y *= f; w.z *= f;
    }
    if (!(isfinite(vx) && isfinite(vy) && isfinite(vz) && vfinite(w))) atomicOr(s.err, kErrNonFinite);
    s.b_v[b] = make_float4(vx, vy, vz, 0.0f);
    s.b_w[b] = st4(w, 0.0f);
    s.sb_v[b] = make_float4(vx, vy, vz, 0.0f);
    s.sb_w[b] = st4(w, 0.0f);
    const float4 inv = s.b_inv[b];
    const v3 l = {sqrtf(inv.x), sqrtf(inv.y), sqrtf(inv.z)};
    const qt q = mass_orientation(s, b);
    float4* si = s.sb_sqrt_i + 3 * size_t(b);
    if (q.x == 0.0f && q.y == 0.0f && q.z == 0.0f && q.w == 1.0f) {
        si[0] = make_float4(l.x, 0, 0, 0); si[1] = make_float4(0, l.y, 0, 0); si[2] = make_float4(0, 0, l.z, 0);
        return;
    }
    const v3 rx = rot_sc(q, {1, 0, 0}), ry = rot_sc(q, {0, 1, 0}), rz = rot_sc(q, {0, 0, 1});
    const float xx = l.x * rx.x * rx.x + l.y * ry.x * ry.x + l.z * rz.x * rz.x;
    const float yy = l.x * rx.y * rx.y + l.y * ry.y * ry.y + l.z * rz.y * rz.y;
    const float zz = l.x * rx.z * rx.z + l.y * ry.z * ry.z + l.z * rz.z * rz.z;
    const float xy = l.x * rx.x * rx.y + l.y * ry.x * ry.y + l.z * rz.x * rz.y;
    const float xz = l.x * rx.x * rx.z + l.y * ry.x * ry.z + l.z * rz.x * rz.z;
    const float yz = l.x * rx.y * rx.z + l.y * ry.y * ry.z + l.z * rz.y * rz.z;
    si[0] = make_float4(xx, xy, xz, 0); si[1] = make_float4(xy, yy, yz, 0); si[2] = make_float4(xz, yz, zz, 0);
}

__device__ void sleep_pair(const DevState& s, uint32_t k, bool touch);
// Touching managers in canonical pair order, in one pass: each tile flags
// its pairs as touching (with sleeping on, also each pair's counted
// interactions and activations, sleep_pair), scans the flags and writes the
// touching pairs' indices; the last tile sets the manager and descriptor
// counts.
__global__ void __launch_bounds__(kScanThreads) k_touch_compact(DevState s) {
    const uint32_t n = min(*s.cur.n, s.pair_cap);
    compact_tiles(
        n, s.scan_tmp, s.err,
        [&](uint32_t k) {
            const bool touch = s.cur.count[k] > 0u;
            if (s.sleep) sleep_pair(s, k, touch);
            return touch;
        },
        [&](uint32_t k, uint32_t at) { s.man_list[at] = k; },
        [&](uint32_t total) {
            s.counters[kCntMan] = total;
            s.counters[kCntDesc] = s.n_joints + total;
        });
}

// Lock-free union-find after ECL-CC (Jaiganesh and Burtscher, "A
// high-performance connected components implementation for GPUs", HPDC
// 2018): a root is hooked under the smaller root, so every parent index is
// at most its child's and the root of a set is its smallest member; finds
// shorten the path they walk (intermediate pointer jumping, plain stores:
// a node that is not a root only ever gets an ancestor written); a failed
// hook continues from the value it found instead of finding both roots
// again.  Loads go through L1: a stale parent is still an ancestor (sets
// only merge), a stale root fails its hook and the hook continues from the
// value the atomic returns, and the root of a large set is then read from
// each SM's L1 instead of by every thread from one L2 line.
__device__ uint32_t uf_find(uint32_t* parent, uint32_t x) {
    uint32_t cur = parent[x];
    if (cur == x) return x;
    uint32_t prev = x, next;
    for (int it = 0; it < (1 << 24) && cur > (next = parent[cur]); ++it) {
        parent[prev] = next;
        prev = cur;
        cur = next;
    }
    return cur;
}
__device__ void uf_union(const DevState& s, uint32_t* parent, uint32_t a, uint32_t b) {
    uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
    // every failed hook moves one root strictly down, so this ends
    for (int it = 0; it < (1 << 24); ++it) {
        if (ra == rb) return;
        if (ra < rb) {
            const uint32_t r = atomicCAS(&parent[rb], rb, ra);
            if (r == rb) return;
            rb = r;
        } else {
            const uint32_t r = atomicCAS(&parent[ra], ra, rb);
            if (r == ra) return;
            ra = r;
        }
    }
    atomicOr(s.err, kErrUnionFind);
}
// Descriptor endpoints: joints use the ordered edge pair (scene.cpp:3154),
// managers the Gu order.  -1 marks the static world body.  Resolved once per
// step into d_bod by k_desc_bodies; every later stage reads that array.
__device__ __forceinline__ void resolve_desc_bodies(const DevState& s, uint32_t d, int32_t& b0, int32_t& b1) {
    if (d < s.n_joints) {
        b0 = int32_t(s.j_a[d]);
        b1 = int32_t(s.j_b[d]);
    } else {
        uint32_t sh0, sh1;
        manager_bodies(s, s.man_list[d - s.n_joints], sh0, sh1);
        b0 = int32_t(s.s_body[sh0]);
        b1 = int32_t(s.s_body[sh1]);
    }
    if (!is_dyn(s, uint32_t(b0))) b0 = -1;
    if (!is_dyn(s, uint32_t(b1))) b1 = -1;
}
__device__ __forceinline__ void desc_bodies(const DevState& s, uint32_t d, int32_t& b0, int32_t& b1) {
    const int2 b = s.d_bod[d];
    b0 = b.x;
    b1 = b.y;
}
__global__ void k_desc_bodies(DevState s) {
    const uint32_t n = s.counters[kCntDesc];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        int32_t b0, b1;
        resolve_desc_bodies(s, d, b0, b1);
        s.d_bod[d] = make_int2(b0, b1);
    }
}
__global__ void k_union(DevState s) {
    const uint32_t n = s.counters[kCntDesc];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        int32_t b0, b1;
        desc_bodies(s, d, b0, b1);
        if (b0 >= 0 && b1 >= 0) uf_union(s, s.uf_parent, uint32_t(b0), uint32_t(b1));
    }
}
// Island key of every descriptor: the union-find root of its bodies.  The
// descriptors of sleeping islands (every island is either awake or asleep
// once the step's sleep decisions are made) take the key n_bodies, which
// sorts them after every awake island; kCntAwake counts the others.
__global__ void k_desc_keys(DevState s) {
    const uint32_t n = s.counters[kCntDesc];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        int32_t b0, b1;
        desc_bodies(s, d, b0, b1);
        const uint32_t body = b0 >= 0 ? uint32_t(b0) : uint32_t(b1);
        const bool asleep = is_asleep(s, body);
        s.d_key[d] = asleep ? s.n_bodies : uf_find(s.uf_parent, body);
        s.d_val[d] = d;
        s.d_level[d] = kInvalid;
        const uint32_t am = __activemask();
        const uint32_t votes = __ballot_sync(am, !asleep);
        if ((threadIdx.x & 31u) == uint32_t(__ffs(am) - 1)) atomicAdd(&s.counters[kCntAwake], __popc(votes));
    }
}

// Replayed order (one step): descriptors are first sorted by their rank in
// the given order -- joints by rp_jrank, then the listed touching managers
// by their position in the list, then unlisted managers in pair order --
// while d_level holds each descriptor's island key; the stable sort by
// island key that follows keeps that order inside every island.
__device__ __forceinline__ uint32_t replay_rank(const DevState& s, uint32_t d) {
    if (d < s.n_joints) return s.rp_jrank[d];
    const uint32_t m = d - s.n_joints;
    const uint64_t key = s.cur.key[s.man_list[m]];
    uint32_t lo = 0, hi = s.rp_n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s.rp_keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return s.n_joints + ((lo < s.rp_n && s.rp_keys[lo] == key) ? s.rp_pos[lo] : s.rp_n + m);
}
__global__ void k_replay_keys(DevState s) {
    const uint32_t n = s.counters[kCntDesc];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += stride) {
        s.d_level[d] = s.d_key[d];
        s.d_key[d] = replay_rank(s, d);
    }
}
__global__ void k_replay_rekey(DevState s) {
    const uint32_t n = s.counters[kCntDesc];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const uint32_t d = s.d_val[p];
        s.d_key[p] = s.d_level[d];
        s.d_level[d] = kInvalid;
    }
}

// ---------------- sleep ----------------
// Reference behaviour (src/native/scene.cpp), per step:
//   activate_published_islands 6148-6250: a newly found overlap pair of two
//     dynamic bodies, at least one awake, marks both activating; a newly
//     found touch marks its dynamic bodies activating and not ready for
//     sleep; every sleeping body in the overlap-graph island of an
//     activating body wakes (wake counter >= 0.4 s, sleep filters cleared)
//   deactivate_ready_accurate_islands 6465-6530: an island of the touch and
//     constraint graph whose bodies are all ready for sleep and not all
//     asleep falls asleep (velocities and filters cleared, counter 0)
//   integrate_solver_task 10640-10705: sleepCheck of every awake body after
//     integration sets its wake counter and readiness for the next step
//   change_counted_interactions 2728-2749: a body's counted interactions are
//     its overlap pairs plus its constraints
// Activation sees the overlap graph's islands as the previous step left
// them: the previous step's pairs and the constraints (this step's lost
// pairs split them only afterwards, in the third pass).  They are rebuilt
// here only when some body is asleep, on top of the touch graph's islands
// of this step (its touching pairs and constraints): the touching pairs
// that are new this step join two activating bodies, whose islands wake
// either way, so adding them changes no wake.  What remains to join are the
// previous step's pairs that do not touch now: the kept ones and the lost
// ones, each joining the two touch-graph roots of its bodies.

// Counted interactions and activations of current pair k.
// sl_act bits: activating this step; linked to a kinematic body whose
// target is pending (its island may not sleep, mark_kinematic_awake,
// scene.cpp:6430-6463); linked to a kinematic body given a new target (its
// sleeping or sleep-ready partners wake, scene.cpp:893-911).
constexpr uint32_t kActActivating = 1u, kActKinematic = 2u, kActKinWake = 4u;
__device__ __forceinline__ void kinematic_link(const DevState& s, uint32_t a, uint32_t b) {
    const bool ka = s.b_flags[a] & kBodyKinematic, kb = s.b_flags[b] & kBodyKinematic;
    if (ka == kb) return;
    const uint32_t kin = ka ? a : b, dyn = ka ? b : a;
    if (!is_dyn(s, dyn)) return;
    const uint32_t f = s.b_sleep[kin];
    if (f & kKinPending) atomicOr(&s.sl_act[dyn], kActKinematic);
    if (f & kKinNew) {
        atomicOr(&s.sl_act[dyn], kActKinWake | kActActivating);
        atomicOr(&s.counters[kCntActivating], 1u);
    }
}
__device__ void sleep_pair(const DevState& s, uint32_t k, bool touch) {
    const uint64_t key = s.cur.key[k];
    const uint32_t ba = s.s_body[uint32_t(key >> 32)], bb = s.s_body[uint32_t(key)];
    const bool da = is_dyn(s, ba), db = is_dyn(s, bb);
    if (da) atomicAdd(&s.b_counted[ba], 1u);
    if (db) atomicAdd(&s.b_counted[bb], 1u);
    const int32_t pj = s.prev_idx[k];
    const bool found = pj < 0;
    const bool touched = !found && s.prev.count[pj] > 0u;
    if (found && da && db && (!is_asleep(s, ba) || !is_asleep(s, bb))) {
        atomicOr(&s.sl_act[ba], kActActivating);
        atomicOr(&s.sl_act[bb], kActActivating);
        atomicOr(&s.counters[kCntActivating], 1u);
    }
    if (touch && !touched) {
        if (da) { atomicOr(&s.sl_act[ba], kActActivating); atomicAnd(&s.b_sleep[ba], ~kReady); }
        if (db) { atomicOr(&s.sl_act[bb], kActActivating); atomicAnd(&s.b_sleep[bb], ~kReady); }
        if (da || db) atomicOr(&s.counters[kCntActivating], 1u);
    }
    if (touch && s.n_kinematic) kinematic_link(s, ba, bb);
}
// Joints linking a dynamic body to a kinematic one act on sleep as touches do.
__global__ void k_sleep_kinematic_joints(DevState s) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < s.n_joints) kinematic_link(s, s.j_a[j], s.j_b[j]);
}
// The overlap graph's union-find runs over touch-graph island roots: a
// body's overlap-graph island is that of its touch-graph root.
// Remaining pair i of the previous step (kept and not touching, or lost):
// the touch-graph roots of its two dynamic bodies, or false.
__device__ __forceinline__ bool spec_pair(const DevState& s, uint32_t i, uint32_t n, uint32_t& ra, uint32_t& rb) {
    uint64_t key;
    if (i < n) {
        if (s.prev_idx[i] < 0 || s.cur.count[i] > 0u) return false;   // new, or joined already
        key = s.cur.key[i];
    } else {
        if (!s.lost_flag[i - n]) return false;
        key = s.prev.key[i - n];
    }
    const uint32_t ba = s.s_body[uint32_t(key >> 32)], bb = s.s_body[uint32_t(key)];
    if (!is_dyn(s, ba) || !is_dyn(s, bb)) return false;
    ra = uf_find(s.uf_parent, ba);
    rb = uf_find(s.uf_parent, bb);
    return ra != rb;
}
// Only an activating body can wake a sleeping island, so without one the
// overlap graph is not needed this step.
__global__ void k_sleep_spec(DevState s) {
    if (s.counters[kCntSleeping] == 0u || s.counters[kCntActivating] == 0u) return;
    const uint32_t n = *s.cur.n, np = *s.prev.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n + np; i += stride) {
        uint32_t ra, rb;
        if (spec_pair(s, i, n, ra, rb)) uf_union(s, s.sl_spec, ra, rb);
    }
}
__device__ __forceinline__ uint32_t spec_root(const DevState& s, uint32_t acc_root) {
    return uf_find(s.sl_spec, acc_root);
}
constexpr uint32_t kRootWake = 1u, kRootUnready = 2u, kRootAwake = 4u;
__global__ void k_sleep_wake_roots(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || s.counters[kCntSleeping] == 0u || !(s.sl_act[b] & kActActivating)) return;
    atomicOr(&s.sl_root[spec_root(s, uf_find(s.uf_parent, b))], kRootWake);
}
// Wakes the sleeping bodies of marked overlap-graph islands, then adds each
// body's readiness and wakefulness to its touch-graph island's root (only
// when some body could fall asleep: a body was ready at the step's start).
__global__ void k_sleep_wake_flags(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b)) return;
    uint32_t f = s.b_sleep[b];
    const uint32_t root = uf_find(s.uf_parent, b);
    const uint32_t act = s.sl_act[b];
    if (((f & kSleeping) && s.counters[kCntSleeping] != 0u && (s.sl_root[spec_root(s, root)] & kRootWake)) ||
        ((act & kActKinWake) && (f & (kSleeping | kReady)))) {
        f = 0u;
        s.b_sleep[b] = 0u;
        s.b_wake[b] = smax(s.b_wake[b], 0.4f);
        const float4 z = make_float4(0, 0, 0, 0);
        s.b_sacc[2 * size_t(b)] = z;
        s.b_sacc[2 * size_t(b) + 1] = z;
    }
    if (s.counters[kCntReady] == 0u) return;
    const uint32_t bits = ((f & kReady) && !(act & kActKinematic) ? 0u : kRootUnready) |
                          ((f & kSleeping) ? 0u : kRootAwake);
    // the bits only accumulate: once a root holds them, the thousands of
    // bodies of a large island skip the atomic on its one word
    if (bits && (*reinterpret_cast<volatile uint32_t*>(&s.sl_root[root]) & bits) != bits)
        atomicOr(&s.sl_root[root], bits);
}
__global__ void k_sleep_decide(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || s.counters[kCntReady] == 0u || !is_dyn(s, b) || (s.b_sleep[b] & kSleeping)) return;
    const uint32_t f = s.sl_root[uf_find(s.uf_parent, b)];
    if ((f & kRootUnready) || !(f & kRootAwake)) return;
    s.b_sleep[b] = kSleeping | kReady;
    s.b_wake[b] = 0.0f;
    const float4 z = make_float4(0, 0, 0, 0);
    s.b_v[b] = z;
    s.b_w[b] = z;
    s.b_sacc[2 * size_t(b)] = z;
    s.b_sacc[2 * size_t(b) + 1] = z;
}
// Island starts in one pass: a descriptor whose key differs from its
// predecessor's opens an island (descriptors sorted by island root); the
// last tile sets the island count, the end sentinel, and clears the
// island-class list counters that k_island_classes fills next.
__global__ void __launch_bounds__(kScanThreads) k_island_compact(DevState s) {
    const uint32_t n = min(s.counters[kCntAwake], s.desc_cap);
    compact_tiles(
        n, s.scan_tmp, s.err, [&](uint32_t i) { return i == 0 || s.d_key[i] != s.d_key[i - 1]; },
        [&](uint32_t i, uint32_t at) { s.isl_begin[at] = i; },
        [&](uint32_t total) {
            *s.n_isl = total;
            s.isl_begin[total] = n;
            for (int c = 0; c < 4; ++c) s.counters[kCntList + c] = 0u;
            for (int c = 0; c < 5; ++c) s.counters[kCntList4 + c] = 0u;   // lists 4-5, work-queue tickets
        });
}

// Size classes of the islands (lists consumed by the partition and PGS
// kernels of each class).
__global__ void k_island_classes(DevState s) {
    const uint32_t ni = *s.n_isl;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < ni; isl += stride) {
        const uint32_t n = s.isl_begin[isl + 1] - s.isl_begin[isl];
        auto push = [&](int c) { s.isl_list[c][atomicAdd(&s.counters[list_counter(c)], 1u)] = isl; };
        // partitions
        if (n > kSerialIsland && n <= kMidIsland) push(0);
        else if (n > kMidIsland && n <= kBigIsland) push(2);
        else if (n > kBigIsland) push(3);
        // PGS
        if (n > s.isl_thread && n <= s.isl_warp) push(5);
        else if (n > s.isl_warp && n <= s.isl_mid) push(1);
        else if (n > s.isl_mid && n <= kBigIsland) push(4);
    }
}

// Partitioning.  The reference assigns each dynamic/dynamic descriptor, in
// order, the lowest partition bit free on both bodies (32-bit masks, overflow
// waves), then gives each static descriptor the partition after its body's
// last dynamic one plus the number of earlier statics on that body
// (scene.cpp:7367-7437).
//
// Small islands: one warp, whose lane 0 replays that sequential loop.
// Larger islands: one CTA reproduces it exactly in rounds.  A descriptor that
// is the earliest undecided one on both of its bodies has every earlier
// descriptor touching those bodies already decided, so it sees exactly the
// masks the sequential loop would; all such descriptors share no body and are
// decided together.  Each round decides at least the earliest undecided
// descriptor of the island.  Waves and the static pass use the same rule.
constexpr uint32_t kDeferred = 0xfffffffeu;

__global__ void __launch_bounds__(256) k_partition_large(DevState s, uint32_t* lvl_bound) {
    __shared__ uint32_t cursor[kMaxLevels + 1];
    __shared__ uint32_t nlev_s;
    const uint32_t n_list = s.counters[kCntList + 3];
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    for (uint32_t k = blockIdx.x; k < n_list; k += gridDim.x) {
        const uint32_t isl = s.isl_list[3][k];
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        if (tid == 0) nlev_s = 0;
        uint32_t nlev = 0;
        bool ok = true;
        for (uint32_t wave = 0; ok; wave += 32) {
            if (wave) {
                for (uint32_t i = begin + tid; i < end; i += nt) {
                    const uint32_t d = s.d_val[i];
                    if (s.d_level[d] != kDeferred) continue;
                    const int2 b = s.d_bod[d];
                    s.sb_mask[b.x] = 0u;
                    s.sb_mask[b.y] = 0u;
                }
                __syncthreads();
                for (uint32_t i = begin + tid; i < end; i += nt) {
                    const uint32_t d = s.d_val[i];
                    if (s.d_level[d] == kDeferred) s.d_level[d] = kInvalid;
                }
                __syncthreads();
            }
            for (uint32_t round = 0; round <= end - begin; ++round) {
                bool any = false;
                for (uint32_t i = begin + tid; i < end; i += nt) {
                    const uint32_t d = s.d_val[i];
                    const int2 b = s.d_bod[d];
                    if (b.x < 0 || b.y < 0 || s.d_level[d] != kInvalid) continue;
                    s.sb_earliest[b.x] = kInvalid;
                    s.sb_earliest[b.y] = kInvalid;
                    any = true;
                }
                if (!__syncthreads_or(any)) break;
                for (uint32_t i = begin + tid; i < end; i += nt) {
                    const uint32_t d = s.d_val[i];
                    const int2 b = s.d_bod[d];
                    if (b.x < 0 || b.y < 0 || s.d_level[d] != kInvalid) continue;
                    atomicMin(&s.sb_earliest[b.x], i);
                    atomicMin(&s.sb_earliest[b.y], i);
                }
                __syncthreads();
                for (uint32_t i = begin + tid; i < end; i += nt) {
                    const uint32_t d = s.d_val[i];
                    const int2 b = s.d_bod[d];
                    if (b.x < 0 || b.y < 0 || s.d_level[d] != kInvalid) continue;
                    if (s.sb_earliest[b.x] != i || s.sb_earliest[b.y] != i) continue;
                    const uint32_t avail = ~(s.sb_mask[b.x] | s.sb_mask[b.y]);
                    if (!avail) { s.d_level[d] = kDeferred; continue; }
                    const uint32_t bit = __ffs(avail) - 1;
                    s.sb_mask[b.x] |= 1u << bit;
                    s.sb_mask[b.y] |= 1u << bit;
                    const uint32_t lp = wave + bit;
                    s.sb_maxdyn[b.x] = max(s.sb_maxdyn[b.x], lp + 1);
                    s.sb_maxdyn[b.y] = max(s.sb_maxdyn[b.y], lp + 1);
                    s.d_level[d] = lp;
                    nlev = max(nlev, lp + 1);
                }
                __syncthreads();
            }
            bool deferred = false;
            for (uint32_t i = begin + tid; i < end; i += nt)
                deferred |= s.d_level[s.d_val[i]] == kDeferred;
            if (!__syncthreads_or(deferred)) break;
            if (wave + 32 >= kMaxLevels) {
                if (tid == 0) atomicOr(s.err, kErrLevelRange);
                ok = false;
            }
        }
        // statics, in descriptor order per body
        for (uint32_t round = 0; round <= end - begin; ++round) {
            bool any = false;
            for (uint32_t i = begin + tid; i < end; i += nt) {
                const uint32_t d = s.d_val[i];
                const int2 b = s.d_bod[d];
                if ((b.x < 0) == (b.y < 0) || s.d_level[d] != kInvalid) continue;
                s.sb_earliest[b.x >= 0 ? b.x : b.y] = kInvalid;
                any = true;
            }
            if (!__syncthreads_or(any)) break;
            for (uint32_t i = begin + tid; i < end; i += nt) {
                const uint32_t d = s.d_val[i];
                const int2 b = s.d_bod[d];
                if ((b.x < 0) == (b.y < 0) || s.d_level[d] != kInvalid) continue;
                atomicMin(&s.sb_earliest[b.x >= 0 ? b.x : b.y], i);
            }
            __syncthreads();
            for (uint32_t i = begin + tid; i < end; i += nt) {
                const uint32_t d = s.d_val[i];
                const int2 b = s.d_bod[d];
                if ((b.x < 0) == (b.y < 0) || s.d_level[d] != kInvalid) continue;
                const int32_t act = b.x >= 0 ? b.x : b.y;
                if (s.sb_earliest[act] != i) continue;
                const uint32_t lp = s.sb_maxdyn[act] + s.sb_static[act]++;
                s.d_level[d] = lp;
                nlev = max(nlev, lp + 1);
            }
            __syncthreads();
        }
        atomicMax(&nlev_s, nlev);
        __syncthreads();
        nlev = max(nlev_s, 1u);
        if (nlev > kMaxLevels || nlev > end - begin) {
            if (tid == 0) atomicOr(s.err, kErrLevelRange);
            nlev = min(min(nlev, uint32_t(kMaxLevels)), end - begin);
        }
        // partition starts and placement (order inside a partition is free:
        // its descriptors share no dynamic body)
        for (uint32_t l = tid; l <= nlev; l += nt) cursor[l] = 0u;
        __syncthreads();
        for (uint32_t i = begin + tid; i < end; i += nt)
            atomicAdd(&cursor[min(s.d_level[s.d_val[i]], nlev - 1)], 1u);
        __syncthreads();
        if (tid == 0) {
            uint32_t* bound = lvl_bound + begin + isl;
            uint32_t run = begin;
            for (uint32_t l = 0; l < nlev; ++l) {
                const uint32_t c = cursor[l];
                bound[l] = run;
                cursor[l] = run;
                run += c;
            }
            bound[nlev] = end;
            s.isl_end[isl] = nlev;
        }
        __syncthreads();
        for (uint32_t i = begin + tid; i < end; i += nt) {
            const uint32_t d = s.d_val[i];
            s.d_val2[atomicAdd(&cursor[min(s.d_level[d], nlev - 1)], 1u)] = d;
        }
        __syncthreads();
    }
}

// Island-local numbers of the bodies of up to 32 descriptors held one per
// lane (bx, by; -1 for the static world): bodies are numbered in the order
// of their first appearance in x0, y0, x1, y1, ..., so an entry's number is
// the count of first appearances before the entry's own first appearance.  lx / ly
// receive the numbers (0xffff for the static world), nb the body count and
// fx / fy the entry index of the body's first appearance.
__device__ __forceinline__ void warp_local_slots(int32_t bx, int32_t by, uint32_t n, uint32_t& lx, uint32_t& ly,
                                                 uint32_t& nb, uint32_t& fx, uint32_t& fy) {
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31u;
    fx = 2u * lane;
    fy = 2u * lane + 1u;
    for (uint32_t j = 0; j < n; ++j) {
        const int32_t ox = __shfl_sync(full, bx, int(j)), oy = __shfl_sync(full, by, int(j));
        const uint32_t ex = 2u * j, ey = ex + 1u;
        if (ox == bx && ex < fx) fx = ex;
        if (oy == bx && ey < fx) fx = ey;
        if (ox == by && ex < fy) fy = ex;
        if (oy == by && ey < fy) fy = ey;
    }
    const bool on = lane < n;
    const uint32_t mx = __ballot_sync(full, on && bx >= 0 && fx == 2u * lane);
    const uint32_t my = __ballot_sync(full, on && by >= 0 && fy == 2u * lane + 1u);
    auto number = [&](uint32_t f) {
        const uint32_t j = f >> 1, below = (1u << j) - 1u;
        return uint32_t(__popc(mx & below) + __popc(my & below)) + ((f & 1u) ? ((mx >> j) & 1u) : 0u);
    };
    lx = bx >= 0 ? number(fx) : 0xffffu;
    ly = by >= 0 ? number(fy) : 0xffffu;
    nb = uint32_t(__popc(mx) + __popc(my));
}

// One warp per small island: lane i holds the island's i-th descriptor.
// Lane 0 replays the sequential loop over island-local body masks kept in
// shared memory; the placement by level and the island-local body numbering
// of the placed order are spread over the lanes.
constexpr int kPartWarps = 4;
__global__ void __launch_bounds__(kPartWarps * 32) k_partition(DevState s, uint32_t* lvl_bound) {
    __shared__ uint32_t smask[kPartWarps][2 * kSerialIsland], smaxd[kPartWarps][2 * kSerialIsland];
    __shared__ uint32_t sstat[kPartWarps][2 * kSerialIsland], spair[kPartWarps][kSerialIsland];
    __shared__ uint32_t slev[kPartWarps][kSerialIsland], snlev[kPartWarps];
    __shared__ int2 sbod[kPartWarps][kSerialIsland];
    const uint32_t full = 0xffffffffu, lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    uint32_t* mask = smask[wib];
    uint32_t* maxd = smaxd[wib];
    uint32_t* stat = sstat[wib];
    uint32_t* pr = spair[wib];
    uint32_t* lv = slev[wib];
    const uint32_t ni = *s.n_isl;
    for (uint32_t isl = blockIdx.x * kPartWarps + wib; isl < ni; isl += gridDim.x * kPartWarps) {
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        const uint32_t n = end - begin;
        if (n > kSerialIsland) continue;
        const bool on = lane < n;
        const uint32_t d = on ? s.d_val[begin + lane] : 0u;
        const int2 b = on ? s.d_bod[d] : make_int2(-1, -1);
        uint32_t lx, ly, nb, fx, fy;
        warp_local_slots(b.x, b.y, n, lx, ly, nb, fx, fy);
        mask[lane] = mask[lane + 32] = 0u;
        maxd[lane] = maxd[lane + 32] = 0u;
        stat[lane] = stat[lane + 32] = 0u;
        pr[lane] = lx | (ly << 16);
        lv[lane] = kInvalid;
        __syncwarp();
        if (lane == 0) {
            uint32_t nlev = 0;
            bool pending = true;
            for (uint32_t wave = 0; pending; wave += 32) {
                if (wave >= kMaxLevels) { atomicOr(s.err, kErrLevelRange); break; }
                pending = false;
                if (wave)
                    for (uint32_t i = 0; i < n; ++i) {
                        const uint32_t x = pr[i] & 0xffffu, y = pr[i] >> 16;
                        if (lv[i] != kInvalid || x == 0xffffu || y == 0xffffu) continue;
                        mask[x] = 0u;
                        mask[y] = 0u;
                    }
                bool progress = false;
                for (uint32_t i = 0; i < n; ++i) {
                    const uint32_t x = pr[i] & 0xffffu, y = pr[i] >> 16;
                    if (lv[i] != kInvalid || x == 0xffffu || y == 0xffffu) continue;
                    const uint32_t avail = ~(mask[x] | mask[y]);
                    if (!avail) { pending = true; continue; }
                    const uint32_t bit = __ffs(avail) - 1;
                    mask[x] |= 1u << bit;
                    mask[y] |= 1u << bit;
                    const uint32_t lp = wave + bit;
                    maxd[x] = max(maxd[x], lp + 1);
                    maxd[y] = max(maxd[y], lp + 1);
                    lv[i] = lp;
                    nlev = max(nlev, lp + 1);
                    progress = true;
                }
                if (pending && !progress) { atomicOr(s.err, kErrPartition); break; }
            }
            for (uint32_t i = 0; i < n; ++i) {
                if (lv[i] != kInvalid) continue;
                const uint32_t x = pr[i] & 0xffffu, y = pr[i] >> 16;
                const uint32_t act = x != 0xffffu ? x : y;
                if (act == 0xffffu) continue;
                const uint32_t lp = maxd[act] + stat[act]++;
                lv[i] = lp;
                nlev = max(nlev, lp + 1);
            }
            if (nlev > kMaxLevels) { atomicOr(s.err, kErrLevelRange); nlev = kMaxLevels; }
            if (nlev > n) { atomicOr(s.err, kErrLevelRange); nlev = n; }
            snlev[wib] = nlev;
        }
        __syncwarp();
        const uint32_t nlev = snlev[wib];
        const uint32_t level = lv[lane];
        if (on) s.d_level[d] = level;
        // placement by level, stable in island order
        const uint32_t l = on ? min(level, nlev ? nlev - 1u : 0u) : 0xffffffffu;
        uint32_t before = 0, rank = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t o = __shfl_sync(full, l, int(j));
            before += o < lane ? 1u : 0u;
            rank += (o < l || (o == l && j < lane)) ? 1u : 0u;
        }
        uint32_t* bound = lvl_bound + begin + isl;   // nlev + 1 entries
        if (lane < nlev) bound[lane] = begin + before;
        if (lane == 0) {
            bound[nlev] = end;
            s.isl_end[isl] = nlev;
        }
        if (on) {
            s.d_val2[begin + rank] = d;
            sbod[wib][rank] = b;
        }
        __syncwarp();
        // island-local body numbering, in placed order
        const int2 pb = on ? sbod[wib][lane] : make_int2(-1, -1);
        __syncwarp();
        warp_local_slots(pb.x, pb.y, n, lx, ly, nb, fx, fy);
        if (on) {
            s.d_lbod[begin + lane] = lx | (ly << 16);
            int32_t* ib = s.isl_bod + begin + isl;
            if (pb.x >= 0 && fx == 2u * lane) ib[lx] = pb.x;
            if (pb.y >= 0 && fy == 2u * lane + 1u) ib[ly] = pb.y;
        }
        if (lane == 0) s.isl_nbod[isl] = nb;
        __syncwarp();
    }
}

// Block-wide exclusive scan of one value per thread; *total receives the sum.
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t incl = v;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += t;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    uint32_t pre = 0, tot = 0;
    for (uint32_t k = 0; k < nw; ++k) {
        const uint32_t t = warp_tot[k];
        if (k < w) pre += t;
        tot += t;
    }
    if (threadIdx.x == 0) *total = tot;
    __syncthreads();
    return pre + incl - v;
}

__host__ __device__ constexpr uint32_t pow2_at_least(uint32_t x) {
    uint32_t p = 1;
    while (p < x) p <<= 1;
    return p;
}
// Shared memory of k_partition_smem<MAXN>: a body hash table of at least
// 1.5x the island's bodies (<= descriptors + 1) with its dense numbering,
// and per-descriptor local bodies and partitions.
template <uint32_t MAXN> struct PartSmem {
    static constexpr uint32_t kTable = pow2_at_least(3 * (MAXN + 1) / 2 + 1);
    static constexpr size_t kBytes = (2 * size_t(kTable) + 2 * size_t(MAXN)) * 4;
};

__device__ __forceinline__ uint32_t body_hash(int32_t b, uint32_t lg) {
    return (uint32_t(b) * 0x9E3779B1u) >> (32u - lg);
}
__device__ __forceinline__ uint32_t find_local(const uint32_t* key, const uint32_t* slot, uint32_t T,
                                               uint32_t lg, int32_t b) {
    if (b < 0) return 0xffffu;
    uint32_t h = body_hash(b, lg);
    for (uint32_t probe = 0; probe < T; ++probe) {
        if (key[h] == uint32_t(b)) return slot[h];
        h = (h + 1) & (T - 1);
    }
    return 0xffffu;   // unreachable: every body was inserted
}

// Islands of one size class (at most MAXN descriptors): the rounds of k_partition_large on
// island-local body slots in shared memory.  The island's dynamic bodies
// are numbered through a shared-memory hash (open addressing), compacted to
// 0..nb-1 (written to isl_bod for the solver), and the per-body partition
// state lives in shared memory.  A round needs two passes: every undecided
// descriptor offers its index to its bodies (atomicMin), then the ones that
// won on both bodies are decided and clear their bodies' minimum.
template <uint32_t MAXN>
__global__ void __launch_bounds__(256) k_partition_smem(DevState s, uint32_t* lvl_bound, int list_class) {
    constexpr uint32_t TMAX = PartSmem<MAXN>::kTable;
    extern __shared__ uint32_t sm[];
    uint32_t* key = sm;              // [T] hashed body ids
    uint32_t* slot = sm + TMAX;      // [T] dense number of an occupied entry
    uint32_t* lid = sm + 2 * TMAX;   // [n] local a | local b << 16
    uint32_t* lvl = lid + MAXN;      // [n] partition, kInvalid undecided, kDeferred
    // After numbering, the body state reuses the table (3 nb <= 2 T):
    uint32_t* mask = sm;             // [nb] partition bits of the current wave
    uint32_t* mds = sm;              // [nb] last dynamic partition + 1 | statics << 16 (set below)
    uint32_t* earliest = sm;         // [nb]
    __shared__ uint32_t cursor[kMaxLevels + 1];
    __shared__ uint32_t warp_tot[32];
    __shared__ uint32_t nb_s, nlev_s;
    const uint32_t tid = threadIdx.x, nt = blockDim.x;
    const uint32_t n_list = s.counters[kCntList + list_class];
    const uint32_t* list = s.isl_list[list_class];
    for (uint32_t k = blockIdx.x; k < n_list; k += gridDim.x) {
        const uint32_t isl = list[k];
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        const uint32_t n = end - begin;
        const uint32_t T = pow2_at_least(3 * (n + 1) / 2 + 1);
        uint32_t lg = 0;
        while ((1u << lg) < T) ++lg;
        for (uint32_t h = tid; h < T; h += nt) key[h] = kInvalid;
        __syncthreads();
        for (uint32_t i = tid; i < n; i += nt) {
            const int2 b = s.d_bod[s.d_val[begin + i]];
            for (int k = 0; k < 2; ++k) {
                const int32_t body = k ? b.y : b.x;
                if (body < 0) continue;
                uint32_t h = body_hash(body, lg);
                for (uint32_t probe = 0; probe < T; ++probe) {
                    const uint32_t prev = atomicCAS(&key[h], kInvalid, uint32_t(body));
                    if (prev == kInvalid || prev == uint32_t(body)) break;
                    h = (h + 1) & (T - 1);
                }
            }
        }
        __syncthreads();
        {
            const uint32_t per = (T + nt - 1) / nt;
            const uint32_t h0 = min(tid * per, T), h1 = min(h0 + per, T);
            uint32_t c = 0;
            for (uint32_t h = h0; h < h1; ++h) c += key[h] != kInvalid ? 1u : 0u;
            uint32_t at = block_excl_scan(c, warp_tot, &nb_s);
            for (uint32_t h = h0; h < h1; ++h)
                if (key[h] != kInvalid) {
                    slot[h] = at;
                    s.isl_bod[begin + isl + at] = int32_t(key[h]);
                    ++at;
                }
        }
        __syncthreads();
        const uint32_t nb = nb_s;
        for (uint32_t i = tid; i < n; i += nt) {
            const int2 b = s.d_bod[s.d_val[begin + i]];
            lid[i] = find_local(key, slot, T, lg, b.x) | (find_local(key, slot, T, lg, b.y) << 16);
            lvl[i] = kInvalid;
        }
        __syncthreads();
        mask = sm;
        mds = sm + nb;
        earliest = sm + 2 * nb;
        for (uint32_t l = tid; l < nb; l += nt) { mask[l] = 0u; mds[l] = 0u; }
        __syncthreads();
        uint32_t nlev = 0;
        for (uint32_t wave = 0;; wave += 32) {
            if (wave) {
                for (uint32_t i = tid; i < n; i += nt)
                    if (lvl[i] == kDeferred) { mask[lid[i] & 0xffffu] = 0u; mask[lid[i] >> 16] = 0u; }
                __syncthreads();
                for (uint32_t i = tid; i < n; i += nt)
                    if (lvl[i] == kDeferred) lvl[i] = kInvalid;
            }
            for (uint32_t l = tid; l < nb; l += nt) earliest[l] = kInvalid;
            __syncthreads();
            for (uint32_t round = 0; round <= n; ++round) {
                for (uint32_t i = tid; i < n; i += nt) {
                    const uint32_t la = lid[i] & 0xffffu, lb = lid[i] >> 16;
                    if (la == 0xffffu || lb == 0xffffu || lvl[i] != kInvalid) continue;
                    atomicMin(&earliest[la], i);
                    atomicMin(&earliest[lb], i);
                }
                __syncthreads();
                bool left = false;
                for (uint32_t i = tid; i < n; i += nt) {
                    const uint32_t la = lid[i] & 0xffffu, lb = lid[i] >> 16;
                    if (la == 0xffffu || lb == 0xffffu || lvl[i] != kInvalid) continue;
                    if (earliest[la] != i || earliest[lb] != i) { left = true; continue; }
                    earliest[la] = kInvalid;
                    earliest[lb] = kInvalid;
                    const uint32_t avail = ~(mask[la] | mask[lb]);
                    if (!avail) { lvl[i] = kDeferred; continue; }
                    const uint32_t bit = __ffs(avail) - 1;
                    mask[la] |= 1u << bit;
                    mask[lb] |= 1u << bit;
                    const uint32_t lp = wave + bit;
                    mds[la] = max(mds[la], lp + 1);
                    mds[lb] = max(mds[lb], lp + 1);
                    lvl[i] = lp;
                    nlev = max(nlev, lp + 1);
                }
                if (!__syncthreads_or(left)) break;
            }
            bool deferred = false;
            for (uint32_t i = tid; i < n; i += nt) deferred |= lvl[i] == kDeferred;
            if (!__syncthreads_or(deferred)) break;
            if (wave + 32 >= kMaxLevels) {
                if (tid == 0) atomicOr(s.err, kErrLevelRange);
                break;
            }
        }
        // statics, in descriptor order per body, after its last dynamic partition
        for (uint32_t l = tid; l < nb; l += nt) earliest[l] = kInvalid;
        __syncthreads();
        for (uint32_t round = 0; round <= n; ++round) {
            for (uint32_t i = tid; i < n; i += nt) {
                const uint32_t la = lid[i] & 0xffffu, lb = lid[i] >> 16;
                if ((la == 0xffffu) == (lb == 0xffffu) || lvl[i] != kInvalid) continue;
                atomicMin(&earliest[la != 0xffffu ? la : lb], i);
            }
            __syncthreads();
            bool left = false;
            for (uint32_t i = tid; i < n; i += nt) {
                const uint32_t la = lid[i] & 0xffffu, lb = lid[i] >> 16;
                if ((la == 0xffffu) == (lb == 0xffffu) || lvl[i] != kInvalid) continue;
                const uint32_t act = la != 0xffffu ? la : lb;
                if (earliest[act] != i) { left = true; continue; }
                earliest[act] = kInvalid;
                const uint32_t m = mds[act];
                const uint32_t lp = (m & 0xffffu) + (m >> 16);
                mds[act] = m + 0x10000u;
                lvl[i] = lp;
                nlev = max(nlev, lp + 1);
            }
            if (!__syncthreads_or(left)) break;
        }
        if (tid == 0) nlev_s = 0;
        __syncthreads();
        atomicMax(&nlev_s, nlev);
        __syncthreads();
        nlev = max(nlev_s, 1u);
        if (nlev > uint32_t(kMaxLevels) || nlev > n) {
            if (tid == 0) atomicOr(s.err, kErrLevelRange);
            nlev = min(min(nlev, uint32_t(kMaxLevels)), n);
        }
        for (uint32_t l = tid; l <= nlev; l += nt) cursor[l] = 0u;
        __syncthreads();
        for (uint32_t i = tid; i < n; i += nt) atomicAdd(&cursor[min(lvl[i], nlev - 1)], 1u);
        __syncthreads();
        if (tid == 0) {
            uint32_t* bound = lvl_bound + begin + isl;
            uint32_t run = begin;
            for (uint32_t l = 0; l < nlev; ++l) {
                const uint32_t c = cursor[l];
                bound[l] = run;
                cursor[l] = run;
                run += c;
            }
            bound[nlev] = end;
            s.isl_end[isl] = nlev;
            s.isl_nbod[isl] = nb;
        }
        __syncthreads();
        for (uint32_t i = tid; i < n; i += nt) {
            const uint32_t d = s.d_val[begin + i];
            const uint32_t at = atomicAdd(&cursor[min(lvl[i], nlev - 1)], 1u);
            s.d_val2[at] = d;
            s.d_lbod[at] = lid[i];
            s.d_level[d] = lvl[i];
        }
        __syncthreads();
    }
}

// ---------------- row preparation ----------------
// Joint rows (scene.cpp:7615-7767): one thread per joint.  Distance kinds
// give one row along the anchor separation; the others lock translation
// along frame A's axes (prismatic: not X) and rotation through the relative
// quaternion's vector part (spherical: none; revolute: not X), the rows
// orthogonalised in the inverse-mass metric in order.
__device__ __forceinline__ uint32_t joint_row_count(uint32_t kind) {
    return kind <= kJointAnchored ? 1u : kind == kJointSpherical ? 3u : kind == kJointFixed ? 6u : 5u;
}
__global__ void k_prep_joints(DevState s) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= s.n_joints) return;
    const uint32_t a = s.j_a[j], b = s.j_b[j], kind = s.j_kind[j];
    const bool da = is_dyn(s, a), db = is_dyn(s, b);
    if (s.sleep && ((da && (s.b_sleep[a] & kSleeping)) || (db && (s.b_sleep[b] & kSleeping)))) return;
    const float inv_dt = 1.0f / s.dt;
    const qt qa0 = ldq(s.b_q[a]), qb0 = ldq(s.b_q[b]);
    const v3 world0 = vadd(ld3(s.b_p[a]), rot_sc(qa0, ld3(s.j_la[j])));
    const v3 world1 = vadd(ld3(s.b_p[b]), rot_sc(qb0, ld3(s.j_lb[j])));
    const v3 c0 = mass_position(s, a), c1 = mass_position(s, b);
    const v3 ra = vsub(world0, c0), rb = vsub(world1, c1);
    const float m0 = da ? s.b_inv[a].w : 0.0f, m1 = db ? s.b_inv[b].w : 0.0f;
    const v3 rel = vsub(ld3(s.b_v[a]), ld3(s.b_v[b]));
    const v3 wa = ld3(s.b_w[a]), wb = ld3(s.b_w[b]);
    const SBody A = load_sbody_any(s, a, da ? int32_t(a) : -1), B = load_sbody_any(s, b, db ? int32_t(b) : -1);
    JointRow* out = s.jrow + s.j_row[j];
    uint32_t emitted = 0;
    auto emit = [&](v3 axis, v3 a0, v3 a1, v3 ja, v3 jb, float error, float response) {
        if (!(response > 0.0f) || !isfinite(response)) atomicOr(s.err, kErrLogic);
        const float rcp = 1.0f / response;
        JointRow r;
        r.axis[0] = axis.x; r.axis[1] = axis.y; r.axis[2] = axis.z;
        r.ang_a[0] = ja.x; r.ang_a[1] = ja.y; r.ang_a[2] = ja.z;
        r.ang_b[0] = jb.x; r.ang_b[1] = jb.y; r.ang_b[2] = jb.z;
        r.ima = m0; r.imb = m1;
        r.vel_mult = -rcp;
        const float speed = vdot(axis, rel) + vdot(a0, wa) - vdot(a1, wb);
        r.constant = -rcp * (error * inv_dt + speed);
        r.unbiased = -rcp * speed;
        r.applied = 0.0f;
        r.pad = 0.0f;
        if (!isfinite(r.constant) || !isfinite(r.unbiased)) atomicOr(s.err, kErrNonFinite);
        out[emitted++] = r;
    };
    if (kind <= kJointAnchored) {
        const v3 off = {c0.x + ra.x - c1.x - rb.x, c0.y + ra.y - c1.y - rb.y, c0.z + ra.z - c1.z - rb.z};
        const float dist = sqrtf(vdot(off, off));
        const v3 axis = dist < 1.192092896e-07f ? v3{1, 0, 0} : v3{off.x / dist, off.y / dist, off.z / dist};
        const v3 an0 = vcross(ra, axis), an1 = vcross(rb, axis);
        const v3 ja = da ? xform(A, an0) : v3{0, 0, 0};
        const v3 jb = db ? xform(B, an1) : v3{0, 0, 0};
        emit(axis, an0, an1, ja, jb, dist - s.j_len[j], m0 + m1 + vdot(ja, ja) + vdot(jb, jb));
        return;
    }
    const qt qa = qmul(qa0, ldq(s.j_qa[j]));
    const v3 error_p = rotinv_sc(qa, vsub(world0, world1));
    v3 ea = {0, 0, 0}, va = {0, 0, 0}, vb = {0, 0, 0}, c = {0, 0, 0};
    float dd = 0.0f, overlap = 0.0f;
    if (kind != kJointSpherical) {
        qt qb = qmul(qb0, ldq(s.j_qb[j]));
        if (qa.x * qb.x + qa.y * qb.y + qa.z * qb.z + qa.w * qb.w < 0.0f) qb = {-qb.x, -qb.y, -qb.z, -qb.w};
        const qt eq = qmul(qconj(qa), qb);
        ea = {eq.x, eq.y, eq.z};
        va = {qa.x, qa.y, qa.z};
        vb = {qb.x, qb.y, qb.z};
        dd = qa.w * qb.w - vdot(va, vb);
        overlap = qa.w * qb.w + vdot(va, vb);
        c = {qa.w * vb.x + qb.w * va.x, qa.w * vb.y + qb.w * va.y, qa.w * vb.z + qb.w * va.z};
    }
    const float errors[6] = {error_p.x, error_p.y, error_p.z, -ea.x, -ea.y, -ea.z};
    const float avc[3] = {va.x, va.y, va.z}, bvc[3] = {vb.x, vb.y, vb.z};
    const v3 diag[3] = {{dd, c.z, -c.y}, {-c.z, dd, c.x}, {c.y, -c.x, dd}};
    struct Eq { v3 lin, a0, a1, ja, jb; float err, inv; };
    Eq er[6];
    const uint32_t count = joint_row_count(kind);
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t comp = k + (kind == kJointPrismatic ? 1u : 0u) + (kind == kJointRevolute && k >= 3u ? 1u : 0u);
        Eq e;
        e.err = errors[comp];
        if (comp < 3u) {
            const v3 basis = {comp == 0u ? 1.0f : 0.0f, comp == 1u ? 1.0f : 0.0f, comp == 2u ? 1.0f : 0.0f};
            e.lin = rot_sc(qa, basis);
            const v3 arm = kind == kJointPrismatic ? vsub(world1, c0) : ra;
            e.a0 = vcross(arm, e.lin);
            e.a1 = vcross(rb, e.lin);
        } else {
            const uint32_t q = comp - 3u;
            const v3 v = diag[q];
            e.lin = {0, 0, 0};
            e.a0 = {0.5f * (va.x * bvc[q] + vb.x * avc[q] + v.x), 0.5f * (va.y * bvc[q] + vb.y * avc[q] + v.y),
                    0.5f * (va.z * bvc[q] + vb.z * avc[q] + v.z)};
            if (overlap == 0.0f) {
                // the relative quaternion's Jacobian is singular at 180 degrees
                const float t = -FLT_EPSILON;
                const v3 basis = {q == 0u ? 1.0f : 0.0f, q == 1u ? 1.0f : 0.0f, q == 2u ? 1.0f : 0.0f};
                e.a0 = {e.a0.x - basis.x * t, e.a0.y - basis.y * t, e.a0.z - basis.z * t};
            }
            e.a1 = e.a0;
        }
        e.ja = da ? xform(A, e.a0) : v3{0, 0, 0};
        e.jb = db ? xform(B, e.a1) : v3{0, 0, 0};
        for (uint32_t p = 0; p < k; ++p) {
            const Eq& f = er[p];
            const float t = ((m0 + m1) * vdot(e.lin, f.lin) + vdot(e.ja, f.ja) + vdot(e.jb, f.jb)) * f.inv;
            e.lin = {e.lin.x - f.lin.x * t, e.lin.y - f.lin.y * t, e.lin.z - f.lin.z * t};
            e.a0 = {e.a0.x - f.a0.x * t, e.a0.y - f.a0.y * t, e.a0.z - f.a0.z * t};
            e.a1 = {e.a1.x - f.a1.x * t, e.a1.y - f.a1.y * t, e.a1.z - f.a1.z * t};
            e.ja = {e.ja.x - f.ja.x * t, e.ja.y - f.ja.y * t, e.ja.z - f.ja.z * t};
            e.jb = {e.jb.x - f.jb.x * t, e.jb.y - f.jb.y * t, e.jb.z - f.jb.z * t};
            e.err -= f.err * t;
        }
        const float response = (m0 + m1) * vdot(e.lin, e.lin) + vdot(e.ja, e.ja) + vdot(e.jb, e.jb);
        e.inv = response > 0.0f ? 1.0f / response : 0.0f;
        er[k] = e;
        emit(e.lin, e.a0, e.a1, e.ja, e.jb, e.err, response);
    }
}

__global__ void k_prep_contacts(DevState s) {
    const uint32_t nm = s.counters[kCntMan];
    const uint32_t frame = s.counters[kCntFrame];
    const float inv_dt = 1.0f / s.dt;
    const float bias_coeff = 0.8f, bounce = -2.0f, same_normal = 0.999f, fr_thr = 0.04f;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < nm; m += stride) {
        const uint32_t pair = s.man_list[m];
        uint32_t sh0, sh1;
        manager_bodies(s, pair, sh0, sh1);
        const uint32_t a0 = s.s_body[sh0], a1 = s.s_body[sh1];
        const int32_t b0 = is_dyn(s, a0) ? int32_t(a0) : -1;
        const int32_t b1 = is_dyn(s, a1) ? int32_t(a1) : -1;
        // managers of sleeping islands are not solved (their history stays)
        if (is_asleep(s, uint32_t(b0 >= 0 ? b0 : b1))) continue;
        const SBody A = load_sbody_any(s, a0, b0), B = load_sbody_any(s, a1, b1);
        const float4 m0 = s.s_mat[sh0], m1 = s.s_mat[sh1];
        const float4 d0 = s.b_dyn1[a0], d1 = s.b_dyn1[a1];
        const float rest_d = m0.w + m1.w;
        const float maximp = smin(d0.y, d1.y);
        const float maxpen = -smin(d0.x, d1.x);
        const float restitution = 0.5f * (m0.z + m1.z);
        const float damping = 0.0f;
        const float dfr = smax(0.0f, 0.5f * (m0.y + m1.y));
        const float sfr = smax(dfr, 0.5f * (m0.x + m1.x));
        const uint32_t count = s.cur.count[pair];
        const ContactPt* pts = s.pts + 4 * size_t(pair);
        const v3 n = lv(pts[0].n);
        v3 bmin = lv(pts[0].p), bmax = bmin;
        for (uint32_t j = 1; j < count; ++j) {
            const v3 p = lv(pts[j].p);
            bmin = {smin(bmin.x, p.x), smin(bmin.y, p.y), smin(bmin.z, p.z)};
            bmax = {smax(bmax.x, p.x), smax(bmax.y, p.y), smax(bmax.z, p.z)};
        }
        const qt q0 = mass_orientation(s, a0), q1 = mass_orientation(s, a1);
        const v3 p0 = mass_position(s, a0), p1 = mass_position(s, a1);
        // correlatePatches: a valid previous anchor patch comes first
        // (cached_friction_patch_valid, scene.cpp:3981-4011).  The history
        // is the manager's record in the previous generation; it counts only
        // when that step prepared it.
        FrictionHist h;
        const int32_t pj = s.prev_idx[pair];
        if (pj >= 0) h = s.prev.fric[pj];
        else h.epoch = 0u;
        bool have_old = false;
        if (h.epoch != 0u && h.epoch + 1u == frame && (h.meta & 512u)) {
            bool valid = !((h.meta >> 8) & 1u) && (h.meta & 255u) != 0u;
            if (valid) {
                const v3 on = rotinv_sc(q0, rot_sc(q1, lv(h.n1)));
                if (vdot(lv(h.n0), on) <= same_normal) valid = false;
                for (uint32_t k = 0; valid && k < (h.meta & 255u); ++k) {
                    const v3 lc = rot_sc(q1, lv(h.a1[k]));
                    const v3 wld = {lc.x + p1.x, lc.y + p1.y, lc.z + p1.z};
                    const v3 in0 = rotinv_sc(q0, {wld.x - p0.x, wld.y - p0.y, wld.z - p0.z});
                    const v3 dl = {h.a0[k][0] - in0.x, h.a0[k][1] - in0.y, h.a0[k][2] - in0.z};
                    if (fabsf(vdot(dl, lv(h.n0))) >= 0.025f) valid = false;
                }
            }
            if (valid) {
                const v3 pn = rot_sc(q0, lv(h.n0));
                have_old = vdot(pn, n) >= same_normal && h.rest == restitution && h.damping == damping &&
                           h.sf == sfr && h.df == dfr;
            }
        }
        uint32_t anchors = 0;
        v3 a0l[2], a1l[2];
        v3 patch_n0, patch_n1;
        if (have_old) {
            anchors = h.meta & 255u;
            a0l[0] = lv(h.a0[0]); a0l[1] = lv(h.a0[1]);
            a1l[0] = lv(h.a1[0]); a1l[1] = lv(h.a1[1]);
            patch_n0 = lv(h.n0);
            patch_n1 = lv(h.n1);
        } else {
            a0l[0] = a0l[1] = a1l[0] = a1l[1] = {0, 0, 0};
            patch_n0 = rotinv_sc(q0, n);
            patch_n1 = rotinv_sc(q1, n);
        }
        // contact rows in Gu point order (one patch, one run)
        NormalRow* rows = s.nrow + 4 * size_t(m);
        for (uint32_t j = 0; j < count; ++j) {
            const v3 pos = lv(pts[j].p);
            const v3 raxn = vcross(vsub(pos, A.p), n);
            const v3 rbxn = vcross(vsub(pos, B.p), n);
            const float lin_vrel = vdot(n, vsub(A.v, B.v));
            const v3 ra = xform(A, raxn), rb = xform(B, rbxn);
            const float ang_vrel = vdot(raxn, A.w) - vdot(rbxn, B.w);
            const float vrel = lin_vrel + ang_vrel;
            const float response = (A.inv_mass + vdot(ra, ra)) + (B.inv_mass + vdot(rb, rb));
            const float vm = response > 0.0f ? 1.0f / response : 0.0f;
            const float pen = pts[j].sep - rest_d;
            const float pen_dt = pen * inv_dt;
            const bool separated = pen >= 0.0f;
            const bool closing = -vrel > pen_dt;
            const bool bouncing = restitution > 0.0f && bounce > vrel && closing;
            const float tv = bouncing ? -vrel * restitution : 0.0f;
            NormalRow r;
            sv(r.n, n); sv(r.ra, ra); sv(r.rb, rb);
            r.max_impulse = maximp;
            r.applied = 0.0f;
            r.pad = 0.0f;
            const float target = tv - vrel;
            if (restitution < 0.0f) {
                // compliant spring (scene.cpp:8251-8272)
                const float en_damp = separated && !closing ? 0.0f : damping;
                const float nrdt = s.dt * restitution;
                const float a_coeff = s.dt * (en_damp - nrdt);
                const float x = 1.0f / (1.0f + a_coeff * response);
                const float bias = x * (-nrdt * pen);
                r.vel_mult = x * a_coeff;
                r.imp_mult = 1.0f - x;
                r.biased = target * r.vel_mult - bias;
                r.unbiased = r.biased;
            } else {
                const float pds = separated ? pen_dt : pen * (inv_dt * bias_coeff);
                const float sb_ = bouncing ? 0.0f : vm * smax(maxpen, pds);
                r.vel_mult = vm;
                r.imp_mult = 1.0f;
                r.biased = target * vm - sb_;
                r.unbiased = target * vm - (bouncing ? 0.0f : smax(sb_, 0.0f));
            }
            if (!isfinite(response) || !isfinite(r.biased) || !isfinite(r.unbiased)) atomicOr(s.err, kErrNonFinite);
            rows[j] = r;
        }
        // growPatches (scene.cpp:8296-8380)
        const v3 ext = vsub(bmax, bmin);
        const float dsq = vlen2(ext);
        bool keep_pair = false;
        uint32_t fresh_bits = 0;   // anchors taken from this step's points: bit k, source point at 2 + 2k
        if (anchors == 2) {
            keep_pair = vlen2(vsub(a0l[0], a0l[1])) * 4.0f >= dsq;
            if (!keep_pair) anchors = 0;
        }
        if (!keep_pair) {
            v3 anch[2] = {{0, 0, 0}, {0, 0, 0}};
            bool changed[2] = {false, false};
            uint32_t src[2] = {0, 0};
            uint32_t cnt = anchors;
            if (cnt == 1) anch[0] = vadd(rot_sc(q0, a0l[0]), p0);
            float pd2 = 0.0f;
            for (uint32_t j = 0; j < count; ++j) {
                if (pts[j].sep >= fr_thr + rest_d) continue;
                const v3 w = lv(pts[j].p);
                if (cnt == 0) { anch[0] = w; changed[0] = true; src[0] = j; ++cnt; }
                else if (cnt == 1) {
                    const float dd = vlen2(vsub(w, anch[0]));
                    if (dd > 1.0e-8f) { anch[1] = w; changed[1] = true; src[1] = j; pd2 = dd; ++cnt; }
                } else {
                    const float e0 = vlen2(vsub(w, anch[0]));
                    const float e1 = vlen2(vsub(w, anch[1]));
                    if (e0 > e1 && e0 > pd2) { anch[1] = w; changed[1] = true; src[1] = j; pd2 = e0; }
                    else if (e1 >= e0 && e1 > pd2) { anch[0] = w; changed[0] = true; src[0] = j; pd2 = e1; }
                }
            }
            for (uint32_t k = 0; k < 2; ++k)
                if (changed[k]) fresh_bits |= (1u << k) | (src[k] << (2 + 2 * k));
            for (uint32_t k = 0; k < cnt; ++k) {
                if (!changed[k]) continue;
                a0l[k] = rotinv_sc(q0, {anch[k].x - p0.x, anch[k].y - p0.y, anch[k].z - p0.z});
                a1l[k] = rotinv_sc(q1, {anch[k].x - p1.x, anch[k].y - p1.y, anch[k].z - p1.z});
            }
            if (cnt == 0) { a0l[0] = {0, 0, 0}; a1l[0] = {0, 0, 0}; }
            anchors = cnt;
        }
        // tangent rows (scene.cpp:8400-8450)
        FrictionRow* fr = s.frow + 4 * size_t(m);
        if (anchors) {
            const v3 rel = vsub(A.v, B.v);
            v3 t0 = vsub(rel, {n.x * vdot(rel, n), n.y * vdot(rel, n), n.z * vdot(rel, n)});
            if (vlen2(t0) <= 0.0001f) t0 = fabsf(n.x) < 0.70710678f ? v3{0.0f, -n.z, n.y} : v3{-n.y, n.x, 0.0f};
            const float il = 1.0f / sqrtf(vlen2(t0));
            t0 = {t0.x * il, t0.y * il, t0.z * il};
            const v3 t1 = vcross(n, t0);
            for (uint32_t k = 0; k < anchors; ++k) {
                const v3 ra = rot_sc(q0, a0l[k]);
                const v3 rb = rot_sc(q1, a1l[k]);
                const v3 err = vsub({ra.x + p0.x, ra.y + p0.y, ra.z + p0.z}, {rb.x + p1.x, rb.y + p1.y, rb.z + p1.z});
                for (int t = 0; t < 2; ++t) {
                    const v3 tg = t == 0 ? t0 : t1;
                    const v3 ax0 = vcross(ra, tg), ax1 = vcross(rb, tg);
                    const v3 j0 = xform(A, ax0), j1 = xform(B, ax1);
                    const float resp = (A.inv_mass + vdot(j0, j0)) + (B.inv_mass + vdot(j1, j1));
                    FrictionRow f;
                    sv(f.t, tg); sv(f.ra, j0); sv(f.rb, j1);
                    f.vel_mult = resp > 0.0f ? bias_coeff / resp : 0.0f;
                    f.bias = vdot(tg, err) * inv_dt;
                    f.target = -(vdot(tg, rel) + vdot(ax0, A.w) - vdot(ax1, B.w));
                    f.applied = 0.0f;
                    f.pad[0] = f.pad[1] = f.pad[2] = 0.0f;
                    fr[2 * k + t] = f;
                }
            }
        }
        ManagerHeader hd;
        hd.b0 = b0; hd.b1 = b1; hd.count = count; hd.anchors = anchors;
        hd.sf = sfr; hd.df = dfr; hd.ima = A.inv_mass; hd.imb = B.inv_mass;
        s.mh[m] = hd;
        // the new history replaces the old one (friction_by_edge_ swap)
        FrictionHist nh;
        sv(nh.n0, patch_n0); sv(nh.n1, patch_n1);
        sv(nh.a0[0], a0l[0]); sv(nh.a0[1], a0l[1]);
        sv(nh.a1[0], a1l[0]); sv(nh.a1[1], a1l[1]);
        nh.sf = sfr; nh.df = dfr; nh.rest = restitution; nh.damping = damping;
        nh.meta = anchors | 512u | (fresh_bits << 10);   // broken bit written by the last PGS pass
        nh.epoch = frame;
        s.cur.fric[pair] = nh;
    }
}

// ---------------- PGS ----------------
// Velocity deltas of the solver bodies, addressed either by global body
// (islands too large for shared memory) or by island-local slot in shared
// memory.  Handle -1 is the static world (zero delta, never written).
struct GlobalDeltas {
    static constexpr bool kLocal = false;
    const DevState& s;
    __device__ __forceinline__ void load(int32_t b, v3& dv, v3& dw) const {
        if (b < 0) { dv = dw = {0, 0, 0}; return; }
        dv = ld3(s.sb_dv[b]);
        dw = ld3(s.sb_dw[b]);
    }
    __device__ __forceinline__ void store(int32_t b, v3 dv, v3 dw) const {
        if (b < 0) return;
        s.sb_dv[b] = st4(dv, 0.0f);
        s.sb_dw[b] = st4(dw, 0.0f);
    }
};
struct LocalDeltas {
    static constexpr bool kLocal = true;
    float4* dv_;
    float4* dw_;
    __device__ __forceinline__ void load(int32_t l, v3& dv, v3& dw) const {
        if (l < 0) { dv = dw = {0, 0, 0}; return; }
        dv = ld3(dv_[l]);
        dw = ld3(dw_[l]);
    }
    __device__ __forceinline__ void store(int32_t l, v3 dv, v3 dw) const {
        if (l < 0) return;
        dv_[l] = st4(dv, 0.0f);
        dw_[l] = st4(dw, 0.0f);
    }
};
__device__ __forceinline__ int32_t unpack_local(uint32_t v) { return v == 0xffffu ? -1 : int32_t(v); }

// 32 bytes per thread in one load (sm_100's 256-bit global loads): a solver
// row is two loads instead of four 128-bit ones.  Scattered rows (one
// manager per thread) cost one L1 wavefront per thread and load instruction,
// so halving the instructions halves the L1 work of the row loads, which is
// what bounds the CTA solvers.  The rows are written by this kernel in an
// earlier pass, so the load is ordered against memory (no caching across
// the asm).
__device__ __forceinline__ void ldg256(const void* p, float4& a, float4& b) {
    asm volatile("ld.global.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
                 : "l"(p)
                 : "memory");
}

// A joint's rows in order (scene.cpp:8905-8945) between bodies b0 / b1
// (-1: the static world).
template <class D>
__device__ __forceinline__ void solve_joint(const DevState& s, uint32_t d, int32_t b0, int32_t b1, int it, int pos,
                                            const D& D_) {
    v3 av, aw, bv, bw;
    D_.load(b0, av, aw);
    D_.load(b1, bv, bw);
    const uint32_t r0 = s.j_row[d], nr = joint_row_count(s.j_kind[d]);
    for (uint32_t q = 0; q < nr; ++q) {
        JointRow& r = s.jrow[r0 + q];
        const v3 ax = lv(r.axis), ja = lv(r.ang_a), jb = lv(r.ang_b);
        const float nd = ax.x * (av.x - bv.x) + ax.y * (av.y - bv.y) + ax.z * (av.z - bv.z) + vdot(ja, aw) -
                         vdot(jb, bw);
        const float cst = it < pos ? r.constant : r.unbiased;
        const float nx = sclamp(r.applied + nd * r.vel_mult + cst, -FLT_MAX, FLT_MAX);
        const float imp = nx - r.applied;
        const float ia = imp * r.ima, ib = imp * r.imb;
        av = {av.x + ia * ax.x, av.y + ia * ax.y, av.z + ia * ax.z};
        bv = {bv.x - ib * ax.x, bv.y - ib * ax.y, bv.z - ib * ax.z};
        aw = {aw.x + imp * ja.x, aw.y + imp * ja.y, aw.z + imp * ja.z};
        bw = {bw.x - imp * jb.x, bw.y - imp * jb.y, bw.z - imp * jb.z};
        r.applied = nx;
        if (s.tape_j) s.tape_j[size_t(it) * s.n_jrows + r0 + q] = nx;
    }
    D_.store(b0, av, aw);
    D_.store(b1, bv, bw);
}

// One descriptor's rows for pass `it` (scene.cpp:8853-9148), read from the
// per-manager arrays prep writes.  lid carries the island-local bodies when
// D addresses shared memory.
// kEagerFriction issues the friction-row loads together with the normal
// rows (lowest latency); otherwise they are issued after the normal rows
// are solved (fewer registers).
template <class D, bool kEagerFriction = true>
__device__ void solve_desc(const DevState& s, uint32_t d, uint32_t lid, int it, int pos, int vel, const D& D_) {
    if (d < s.n_joints) {
        int32_t b0, b1;
        if constexpr (D::kLocal) {
            b0 = unpack_local(lid & 0xffffu);
            b1 = unpack_local(lid >> 16);
        } else {
            b0 = is_dyn(s, s.j_a[d]) ? int32_t(s.j_a[d]) : -1;
            b1 = is_dyn(s, s.j_b[d]) ? int32_t(s.j_b[d]) : -1;
        }
        solve_joint(s, d, b0, b1, it, pos, D_);
        return;
    }
    const uint32_t m = d - s.n_joints;
    // All of a manager's rows are loaded up front (issued together) before
    // the sequential Gauss-Seidel updates run on registers.
    // NormalRow float4s: {n.xyz, ra.x} {ra.yz, rb.xy} {rb.z, vel_mult,
    // imp_mult, biased} {unbiased, applied, max_impulse, -}; FrictionRow:
    // {t.xyz, ra.x} {ra.yz, rb.xy} {rb.z, vel_mult, bias, target} {applied}.
    ManagerHeader hd;
    {
        float4 h0, h1;
        ldg256(s.mh + m, h0, h1);
        hd.b0 = __float_as_int(h0.x); hd.b1 = __float_as_int(h0.y);
        hd.count = __float_as_uint(h0.z); hd.anchors = __float_as_uint(h0.w);
        hd.sf = h1.x; hd.df = h1.y; hd.ima = h1.z; hd.imb = h1.w;
    }
    const float ima = hd.ima, imb = hd.imb;   // 0 for the static world
    const bool friction = (it >= pos || pos - it <= 3) && hd.anchors;
    const float4* nr = reinterpret_cast<const float4*>(s.nrow + 4 * size_t(m));
    const float4* fq = reinterpret_cast<const float4*>(s.frow + 4 * size_t(m));
    float4 n0[4], n1[4], n2[4], n3[4], f0[4], f1[4], f2[4];
    float fa[4];
    if constexpr (kEagerFriction) {
        // All four row slots of the manager are read without waiting for
        // the header (unused slots are never consumed), so the row loads and
        // the header load are in flight together.
        const bool friction_pass = it >= pos || pos - it <= 3;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            ldg256(nr + 4 * j, n0[j], n1[j]);
            ldg256(nr + 4 * j + 2, n2[j], n3[j]);
            if (friction_pass) {
                float4 f3;
                ldg256(fq + 4 * j, f0[j], f1[j]);
                ldg256(fq + 4 * j + 2, f2[j], f3);
                fa[j] = f3.x;
            }
        }
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (uint32_t(j) < hd.count) {
                ldg256(nr + 4 * j, n0[j], n1[j]);
                ldg256(nr + 4 * j + 2, n2[j], n3[j]);
            }
    }
    int32_t h0, h1;
    if constexpr (D::kLocal) {
        h0 = unpack_local(lid & 0xffffu);
        h1 = unpack_local(lid >> 16);
    } else {
        h0 = hd.b0;
        h1 = hd.b1;
    }
    v3 av, aw, bv, bw;
    D_.load(h0, av, aw);
    D_.load(h1, bv, bw);
    float nsum = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (uint32_t(j) >= hd.count) break;
        const v3 n = {n0[j].x, n0[j].y, n0[j].z};
        const v3 ra = {n0[j].w, n1[j].x, n1[j].y};
        const v3 rb = {n1[j].z, n1[j].w, n2[j].x};
        const float vel_mult = n2[j].y, imp_mult = n2[j].z;
        const float applied = n3[j].y, max_impulse = n3[j].z;
        const float nvel = vdot(n, av) - vdot(n, bv) + vdot(aw, ra) - vdot(bw, rb);
        const float err = it < pos ? n2[j].w : n3[j].x;
        const float dc = smax(-nvel * vel_mult + err, -applied);
        const float ni = smin(max_impulse, imp_mult * applied + dc);
        const float dl = ni - applied;
        const float da = dl * ima, db = dl * imb;
        av = {av.x + n.x * da, av.y + n.y * da, av.z + n.z * da};
        bv = {bv.x - n.x * db, bv.y - n.y * db, bv.z - n.z * db};
        aw = {aw.x + ra.x * dl, aw.y + ra.y * dl, aw.z + ra.z * dl};
        bw = {bw.x - rb.x * dl, bw.y - rb.y * dl, bw.z - rb.z * dl};
        s.nrow[4 * size_t(m) + j].applied = ni;
        if (s.tape_n) s.tape_n[(size_t(it) * s.pair_cap + m) * 4 + j] = ni;
        nsum += ni;
    }
    if (friction) {
        if constexpr (!kEagerFriction) {
#pragma unroll
            for (int j = 0; j < 4; ++j)
                if (uint32_t(j) < 2 * hd.anchors) {
                    float4 f3;
                    ldg256(fq + 4 * j, f0[j], f1[j]);
                    ldg256(fq + 4 * j + 2, f2[j], f3);
                    fa[j] = f3.x;
                }
        }
        const float coeff = hd.anchors == 2 ? 0.5f : 1.0f;
        const float ms = hd.sf * coeff * nsum;
        const float md = hd.df * coeff * nsum;
        bool broken = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (uint32_t(k) >= 2 * hd.anchors) break;
            const v3 n = {f0[k].x, f0[k].y, f0[k].z};
            const v3 ra = {f0[k].w, f1[k].x, f1[k].y};
            const v3 rb = {f1[k].z, f1[k].w, f2[k].x};
            const float vel_mult = f2[k].y, target = f2[k].w, applied = fa[k];
            const float td = vdot(n, av) - vdot(n, bv) + vdot(aw, ra) - vdot(bw, rb);
            const float bias = it < pos ? f2[k].z : 0.0f;
            const float cand = applied + (target - bias - td) * vel_mult;
            const bool clamped = fabsf(cand) > ms;
            const float nx = clamped ? smin(md, smax(-md, cand)) : cand;
            const float dl = nx - applied;
            const float da = dl * ima, db = dl * imb;
            av = {av.x + n.x * da, av.y + n.y * da, av.z + n.z * da};
            bv = {bv.x - n.x * db, bv.y - n.y * db, bv.z - n.z * db};
            aw = {aw.x + ra.x * dl, aw.y + ra.y * dl, aw.z + ra.z * dl};
            bw = {bw.x - rb.x * dl, bw.y - rb.y * dl, bw.z - rb.z * dl};
            s.frow[4 * size_t(m) + k].applied = nx;
            if (s.tape_f) s.tape_f[(size_t(it) * s.pair_cap + m) * 4 + k] = nx;
            broken |= clamped;
        }
        if (it + 1 == pos + vel) {
            FrictionHist& h = s.cur.fric[s.man_list[m]];
            h.meta = (h.meta & ~256u) | (broken ? 256u : 0u);
        }
    }
    D_.store(h0, av, aw);
    D_.store(h1, bv, bw);
}

// ---- placed-order planes (DevState::slot_rows) ----
// The island solvers copy each manager's rows once per step into planes
// indexed by placed slot, keeping only what the passes read.  Slots come in
// blocks of 32; a block holds kSlotVecPlanes float4 planes of 32 records --
// 0: {sf, df, ima, imb}; normal row j at 1 + 3j: {n.xyz, ra.x} {ra.yz,
// rb.xy} {rb.z, vel_mult, imp_mult, max_impulse}; friction row k at
// 13 + 3k: {t.xyz, ra.x} {ra.yz, rb.xy} {rb.z, vel_mult, bias, target} --
// and, after all blocks' vector planes, kSlotScalarPlanes float planes of
// 32 records -- biased j (0 + j), unbiased j (4 + j), normal applied j
// (8 + j), friction applied k (12 + k).  Lanes solving consecutive slots
// read consecutive records, a plane is a constant offset from the slot's
// first record, and only the rows a manager has are read (its point and
// anchor counts travel with its island-local bodies).
struct SlotPtr {
    float4* v;   // plane 0 record of the slot; plane p at v + 32 p
    float* f;    // scalar plane 0 record; plane p at f + 32 p
    __device__ __forceinline__ SlotPtr(const DevState& s, uint32_t slot) {
        const size_t blk = slot >> 5, lane = slot & 31u;
        v = s.slot_rows + blk * (32u * kSlotVecPlanes) + lane;
        const size_t nblk = (size_t(s.desc_cap) + 31u) >> 5;
        f = reinterpret_cast<float*>(s.slot_rows + nblk * (32u * kSlotVecPlanes)) + blk * (32u * kSlotScalarPlanes) +
            lane;
    }
    __device__ __forceinline__ float4& vec(uint32_t p) const { return v[32 * p]; }
    __device__ __forceinline__ float& sca(uint32_t p) const { return f[32 * p]; }
};
// Island-local bodies in 13 bits each (0x1fff: the static world), the
// manager's point count in bits 13-15 and anchor count in bits 29-31.
__device__ __forceinline__ uint32_t pack_slot_meta(uint32_t lid, uint32_t count, uint32_t anchors) {
    const uint32_t lo = lid & 0xffffu, hi = lid >> 16;
    const uint32_t lo13 = lo == 0xffffu ? 0x1fffu : lo, hi13 = hi == 0xffffu ? 0x1fffu : hi;
    return lo13 | (count << 13) | (hi13 << 16) | (anchors << 29);
}
__device__ __forceinline__ int32_t unpack_local13(uint32_t v) {
    v &= 0x1fffu;
    return v == 0x1fffu ? -1 : int32_t(v);
}
// Copies manager m's rows to slot `slot` and returns its island-local
// bodies with the counts (pack_slot_meta).
__device__ __forceinline__ uint32_t stage_slot_rows(const DevState& s, uint32_t m, uint32_t slot, uint32_t lid) {
    const float4* nr = reinterpret_cast<const float4*>(s.nrow + 4 * size_t(m));
    const float4* fq = reinterpret_cast<const float4*>(s.frow + 4 * size_t(m));
    const SlotPtr P(s, slot);
    float4 h0, h1, q[2][4];
    // rows 0-1 travel with the header; the rest once the counts are known
    ldg256(s.mh + m, h0, h1);
    ldg256(nr, q[0][0], q[0][1]);
    ldg256(nr + 2, q[0][2], q[0][3]);
    ldg256(nr + 4, q[1][0], q[1][1]);
    ldg256(nr + 6, q[1][2], q[1][3]);
    const uint32_t count = min(__float_as_uint(h0.z), 4u), anchors = min(__float_as_uint(h0.w), 2u);
    P.vec(0) = h1;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (uint32_t(j) >= count) break;
        if (j == 2) {
            ldg256(nr + 8, q[0][0], q[0][1]);
            ldg256(nr + 10, q[0][2], q[0][3]);
            if (count > 3) {
                ldg256(nr + 12, q[1][0], q[1][1]);
                ldg256(nr + 14, q[1][2], q[1][3]);
            }
        }
        const float4* r = q[j & 1];
        P.vec(1 + 3 * j) = r[0];
        P.vec(2 + 3 * j) = r[1];
        P.vec(3 + 3 * j) = make_float4(r[2].x, r[2].y, r[2].z, r[3].z);
        P.sca(0 + j) = r[2].w;
        P.sca(4 + j) = r[3].x;
        P.sca(8 + j) = r[3].y;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (uint32_t(k) >= 2 * anchors) break;
        float4 f0, f1, f2, f3;
        ldg256(fq + 4 * k, f0, f1);
        ldg256(fq + 4 * k + 2, f2, f3);
        P.vec(13 + 3 * k) = f0;
        P.vec(14 + 3 * k) = f1;
        P.vec(15 + 3 * k) = f2;
        P.sca(12 + k) = f3.x;
    }
    return pack_slot_meta(lid, count, anchors);
}

// solve_desc on the placed-order planes: descriptor d in slot `slot`, its
// island-local bodies and counts in meta (pack_slot_meta).  The same
// arithmetic in the same order; the impulses of the last pass also go back
// to the per-manager rows, where the events, the force thresholds and the
// rollouts read them.
template <class D, bool kEagerFriction = true>
__device__ void solve_slot(const DevState& s, uint32_t d, uint32_t meta, int it, int pos, int vel, const D& D_,
                           uint32_t slot) {
    const int32_t h0 = unpack_local13(meta), h1 = unpack_local13(meta >> 16);
    if (d < s.n_joints) {
        solve_joint(s, d, h0, h1, it, pos, D_);
        return;
    }
    const uint32_t m = d - s.n_joints;
    const uint32_t count = (meta >> 13) & 7u, anchors = meta >> 29;
    const bool last = it + 1 == pos + vel;
    const bool friction = (it >= pos || pos - it <= 3) && anchors;
    const SlotPtr P(s, slot);
    const float4 hd = P.vec(0);   // {sf, df, ima, imb}
    const float ima = hd.z, imb = hd.w;        // 0 for the static world
    float4 n0[4], n1[4], n2[4], f0[4], f1[4], f2[4];
    float ne[4], na[4], fa[4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (uint32_t(j) < count) {
            n0[j] = P.vec(1 + 3 * j);
            n1[j] = P.vec(2 + 3 * j);
            n2[j] = P.vec(3 + 3 * j);
            ne[j] = P.sca((it < pos ? 0 : 4) + j);
            na[j] = P.sca(8 + j);
        }
    if constexpr (kEagerFriction) {
        if (friction) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (uint32_t(k) < 2 * anchors) {
                    f0[k] = P.vec(13 + 3 * k);
                    f1[k] = P.vec(14 + 3 * k);
                    f2[k] = P.vec(15 + 3 * k);
                    fa[k] = P.sca(12 + k);
                }
        }
    }
    v3 av, aw, bv, bw;
    D_.load(h0, av, aw);
    D_.load(h1, bv, bw);
    float nsum = 0.0f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        if (uint32_t(j) >= count) break;
        const v3 n = {n0[j].x, n0[j].y, n0[j].z};
        const v3 ra = {n0[j].w, n1[j].x, n1[j].y};
        const v3 rb = {n1[j].z, n1[j].w, n2[j].x};
        const float vel_mult = n2[j].y, imp_mult = n2[j].z, max_impulse = n2[j].w;
        const float applied = na[j];
        const float nvel = vdot(n, av) - vdot(n, bv) + vdot(aw, ra) - vdot(bw, rb);
        const float dc = smax(-nvel * vel_mult + ne[j], -applied);
        const float ni = smin(max_impulse, imp_mult * applied + dc);
        const float dl = ni - applied;
        const float da = dl * ima, db = dl * imb;
        av = {av.x + n.x * da, av.y + n.y * da, av.z + n.z * da};
        bv = {bv.x - n.x * db, bv.y - n.y * db, bv.z - n.z * db};
        aw = {aw.x + ra.x * dl, aw.y + ra.y * dl, aw.z + ra.z * dl};
        bw = {bw.x - rb.x * dl, bw.y - rb.y * dl, bw.z - rb.z * dl};
        P.sca(8 + j) = ni;
        if (last) s.nrow[4 * size_t(m) + j].applied = ni;
        if (s.tape_n) s.tape_n[(size_t(it) * s.pair_cap + m) * 4 + j] = ni;
        nsum += ni;
    }
    if (friction) {
        if constexpr (!kEagerFriction) {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (uint32_t(k) < 2 * anchors) {
                    f0[k] = P.vec(13 + 3 * k);
                    f1[k] = P.vec(14 + 3 * k);
                    f2[k] = P.vec(15 + 3 * k);
                    fa[k] = P.sca(12 + k);
                }
        }
        const float coeff = anchors == 2 ? 0.5f : 1.0f;
        const float ms = hd.x * coeff * nsum;
        const float md = hd.y * coeff * nsum;
        bool broken = false;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (uint32_t(k) >= 2 * anchors) break;
            const v3 n = {f0[k].x, f0[k].y, f0[k].z};
            const v3 ra = {f0[k].w, f1[k].x, f1[k].y};
            const v3 rb = {f1[k].z, f1[k].w, f2[k].x};
            const float vel_mult = f2[k].y, target = f2[k].w, applied = fa[k];
            const float td = vdot(n, av) - vdot(n, bv) + vdot(aw, ra) - vdot(bw, rb);
            const float bias = it < pos ? f2[k].z : 0.0f;
            const float cand = applied + (target - bias - td) * vel_mult;
            const bool clamped = fabsf(cand) > ms;
            const float nx = clamped ? smin(md, smax(-md, cand)) : cand;
            const float dl = nx - applied;
            const float da = dl * ima, db = dl * imb;
            av = {av.x + n.x * da, av.y + n.y * da, av.z + n.z * da};
            bv = {bv.x - n.x * db, bv.y - n.y * db, bv.z - n.z * db};
            aw = {aw.x + ra.x * dl, aw.y + ra.y * dl, aw.z + ra.z * dl};
            bw = {bw.x - rb.x * dl, bw.y - rb.y * dl, bw.z - rb.z * dl};
            P.sca(12 + k) = nx;
            if (last) s.frow[4 * size_t(m) + k].applied = nx;
            if (s.tape_f) s.tape_f[(size_t(it) * s.pair_cap + m) * 4 + k] = nx;
            broken |= clamped;
        }
        if (last) {
            FrictionHist& h = s.cur.fric[s.man_list[m]];
            h.meta = (h.meta & ~256u) | (broken ? 256u : 0u);
        }
    }
    D_.store(h0, av, aw);
    D_.store(h1, bv, bw);
}
__device__ __forceinline__ void save_motion(const DevState& s, uint32_t d) {
    int32_t b0, b1;
    if (d < s.n_joints) {
        b0 = is_dyn(s, s.j_a[d]) ? int32_t(s.j_a[d]) : -1;
        b1 = is_dyn(s, s.j_b[d]) ? int32_t(s.j_b[d]) : -1;
    } else {
        const ManagerHeader hd = s.mh[d - s.n_joints];
        b0 = hd.b0; b1 = hd.b1;
    }
    if (b0 >= 0) { s.sb_mdv[b0] = s.sb_dv[b0]; s.sb_mdw[b0] = s.sb_dw[b0]; }
    if (b1 >= 0) { s.sb_mdv[b1] = s.sb_dv[b1]; s.sb_mdw[b1] = s.sb_dw[b1]; }
}

// Copies of an island's shared-memory deltas to the solver bodies.
__device__ __forceinline__ void island_deltas_out(float4* dst_v, float4* dst_w, const int32_t* ib, uint32_t nb,
                                                  const float4* sdv, const float4* sdw, uint32_t t0,
                                                  uint32_t nt) {
    for (uint32_t l = t0; l < nb; l += nt) {
        const int32_t g = ib[l];
        dst_v[g] = sdv[l];
        dst_w[g] = sdw[l];
    }
}

// One thread per tiny island (<= kTinyIsland descriptors): the island's
// placed descriptors are solved in order (level by level, the order the
// wider kernels use, since a level's descriptors share no body) with the
// deltas in the thread's slice of shared memory.  Tiny islands (a body
// resting alone, a short chain) are most islands of a spread-out scene; a
// warp each would leave 31 lanes idle for all five passes.
constexpr uint32_t kTinyIsland = 8;
constexpr uint32_t kPgsThreadBlock = 128;
__global__ void __launch_bounds__(kPgsThreadBlock) k_pgs_thread(DevState s) {
    __shared__ float4 sh[kPgsThreadBlock][2][kTinyIsland + 1];
    const uint32_t ni = *s.n_isl;
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    float4* sdv = sh[threadIdx.x][0];
    float4* sdw = sh[threadIdx.x][1];
    const LocalDeltas D{sdv, sdw};
    const float4 zero = make_float4(0, 0, 0, 0);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t isl = blockIdx.x * blockDim.x + threadIdx.x; isl < ni; isl += stride) {
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        if (end - begin > s.isl_thread) continue;
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        for (uint32_t l = 0; l < nb; ++l) { sdv[l] = zero; sdw[l] = zero; }
        for (int it = 0; it < pos + vel; ++it) {
            for (uint32_t i = begin; i < end; ++i)
                solve_desc<LocalDeltas>(s, s.d_val2[i], s.d_lbod[i], it, pos, vel, D);
            if (it + 1 == pos) island_deltas_out(s.sb_mdv, s.sb_mdw, ib, nb, sdv, sdw, 0u, 1u);
        }
        island_deltas_out(s.sb_dv, s.sb_dw, ib, nb, sdv, sdw, 0u, 1u);
    }
}

// One warp per small island (kTinyIsland < descriptors <= kSmallIsland, so
// <= 97 bodies): the island's deltas live in this warp's slice of shared
// memory.
constexpr uint32_t kWarpBodies = kSmallIsland + 1;
constexpr uint32_t kPgsWarpsPerBlock = 4;
__global__ void __launch_bounds__(kPgsWarpsPerBlock * 32, 3) k_pgs_warp(DevState s, const uint32_t* lvl_bound) {
    __shared__ float4 sh[kPgsWarpsPerBlock][2][kWarpBodies];
    __shared__ uint32_t sdesc[kPgsWarpsPerBlock][2][kSmallIsland];   // descriptor, local bodies per slot
    __shared__ uint32_t sbound[kPgsWarpsPerBlock][kSmallIsland + 1];
    const uint32_t n_list = s.counters[list_counter(5)];
    const uint32_t* list = s.isl_list[5];
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    float4* sdv = sh[wib][0];
    float4* sdw = sh[wib][1];
    const LocalDeltas D{sdv, sdw};
    const float4 zero = make_float4(0, 0, 0, 0);
    for (uint32_t k = warp;;) {
        if (s.work_queue) {
            uint32_t t = 0;
            if (lane == 0) t = atomicAdd(&s.counters[kCntQueue], 1u);
            k = __shfl_sync(0xffffffffu, t, 0);
        }
        if (k >= n_list) break;
        const uint32_t isl = list[k];
        if (!s.work_queue) k += nwarps;
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        const uint32_t* bound = lvl_bound + begin + isl;
        uint32_t* sd = sdesc[wib][0];
        uint32_t* sl = sdesc[wib][1];
        uint32_t* sb = sbound[wib];
        for (uint32_t l = lane; l < nb; l += 32) { sdv[l] = zero; sdw[l] = zero; }
        for (uint32_t i = lane; i < end - begin; i += 32) {
            const uint32_t d = s.d_val2[begin + i], lid = s.d_lbod[begin + i];
            sd[i] = d;
            sl[i] = d >= s.n_joints ? stage_slot_rows(s, d - s.n_joints, begin + i, lid) : pack_slot_meta(lid, 0u, 0u);
        }
        for (uint32_t l = lane; l <= nlev; l += 32) sb[l] = bound[l] - begin;
        __syncwarp();
        for (int it = 0; it < pos + vel; ++it) {
            for (uint32_t l = 0; l < nlev; ++l) {
                const uint32_t lb = sb[l], le = sb[l + 1];
                for (uint32_t i = lb + lane; i < le; i += 32)
                    solve_slot<LocalDeltas>(s, sd[i], sl[i], it, pos, vel, D, begin + i);
                __syncwarp();
            }
            if (it + 1 == pos) {
                island_deltas_out(s.sb_mdv, s.sb_mdw, ib, nb, sdv, sdw, lane, 32);
                __syncwarp();
            }
        }
        island_deltas_out(s.sb_dv, s.sb_dw, ib, nb, sdv, sdw, lane, 32);
        __syncwarp();
    }
}

// One CTA of NT threads per island of a size class (at most MAXN
// descriptors), with the island's deltas in shared memory
// (2 x (MAXN + 1) float4).
// Shared memory of k_pgs_block_smem<MAXN>: deltas, then the island's
// placed descriptors and local bodies, then its partition bounds.
template <uint32_t MAXN> struct PgsSmem {
    static constexpr size_t kBytes = 2 * size_t(MAXN + 1) * sizeof(float4) + 2 * size_t(MAXN) * 4 +
                                     size_t(kMaxLevels + 1) * 4;
};
// Threads of the CTA that solves an island of (kMidIsland, kBigIsland]
// descriptors: 12 warps, the most the register budget of the solver (about
// 160 registers a thread) allows on one SM; a level of such an island holds
// a few hundred descriptors, so more threads mean fewer rounds per level.
constexpr uint32_t kBigPgsThreads = 384;
template <uint32_t MAXN, uint32_t NT>
__global__ void __launch_bounds__(NT) k_pgs_block_smem(DevState s, const uint32_t* lvl_bound, int list_class) {
    extern __shared__ float4 shb[];
    float4* sdv = shb;
    float4* sdw = shb + (MAXN + 1);
    uint32_t* sd = reinterpret_cast<uint32_t*>(shb + 2 * (MAXN + 1));   // descriptor per placed slot
    uint32_t* sl = sd + MAXN;                                             // local bodies per placed slot
    uint32_t* sb = sl + MAXN;                                             // partition bounds (island-relative)
    const LocalDeltas D{sdv, sdw};
    const uint32_t n_list = s.counters[list_counter(list_class)];
    const uint32_t* list = s.isl_list[list_class];
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    const float4 zero = make_float4(0, 0, 0, 0);
    uint32_t* ticket = s.counters + kCntQueue + (list_class == 1 ? 1 : 2);
    __shared__ uint32_t s_next;
    for (uint32_t k = blockIdx.x;;) {
        if (s.work_queue) {
            if (threadIdx.x == 0) s_next = atomicAdd(ticket, 1u);
            __syncthreads();
            k = s_next;
        }
        if (k >= n_list) break;
        const uint32_t isl = list[k];
        if (!s.work_queue) k += gridDim.x;
        const uint32_t begin = s.isl_begin[isl];
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t nb = s.isl_nbod[isl];
        const int32_t* ib = s.isl_bod + begin + isl;
        const uint32_t* bound = lvl_bound + begin + isl;
        const uint32_t n = s.isl_begin[isl + 1] - begin;
        for (uint32_t l = threadIdx.x; l < nb; l += blockDim.x) { sdv[l] = zero; sdw[l] = zero; }
        for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t d = s.d_val2[begin + i], lid = s.d_lbod[begin + i];
            sd[i] = d;
            sl[i] = d >= s.n_joints ? stage_slot_rows(s, d - s.n_joints, begin + i, lid) : pack_slot_meta(lid, 0u, 0u);
        }
        for (uint32_t l = threadIdx.x; l <= nlev; l += blockDim.x) sb[l] = bound[l] - begin;
        __syncthreads();
        for (int it = 0; it < pos + vel; ++it) {
            for (uint32_t l = 0; l < nlev; ++l) {
                const uint32_t lb = sb[l], le = sb[l + 1];
                for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x)
                    solve_slot<LocalDeltas>(s, sd[i], sl[i], it, pos, vel, D, begin + i);
                __syncthreads();
            }
            if (it + 1 == pos) {
                island_deltas_out(s.sb_mdv, s.sb_mdw, ib, nb, sdv, sdw, threadIdx.x, blockDim.x);
                __syncthreads();
            }
        }
        island_deltas_out(s.sb_dv, s.sb_dw, ib, nb, sdv, sdw, threadIdx.x, blockDim.x);
        __syncthreads();
    }
}

// One CTA per island beyond kBigIsland descriptors: deltas in global memory.
__global__ void __launch_bounds__(256) k_pgs_block(DevState s, const uint32_t* lvl_bound) {
    const uint32_t n_list = s.counters[kCntList + 3];
    const int pos = s.pos_iters, vel = s.vel_iters < 1 ? 1 : s.vel_iters;
    const GlobalDeltas D{s};
    for (uint32_t k = blockIdx.x; k < n_list; k += gridDim.x) {
        const uint32_t isl = s.isl_list[3][k];
        const uint32_t begin = s.isl_begin[isl], end = s.isl_begin[isl + 1];
        const uint32_t nlev = s.isl_end[isl];
        const uint32_t* bound = lvl_bound + begin + isl;
        for (int it = 0; it < pos + vel; ++it) {
            for (uint32_t l = 0; l < nlev; ++l) {
                const uint32_t lb = bound[l], le = bound[l + 1];
                for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x)
                    solve_desc(s, s.d_val2[i], 0u, it, pos, vel, D);
                __syncthreads();
            }
            if (it + 1 == pos) {
                for (uint32_t i = begin + threadIdx.x; i < end; i += blockDim.x) save_motion(s, s.d_val2[i]);
                __syncthreads();
            }
        }
    }
}

// Dy sleepCheck without stabilization (DySleep.cpp updateWakeCounter as the
// reference restates it, scene.cpp:10640-10705): the motion velocities of
// the step accumulate while the wake counter is low; enough accumulated
// energy (scaled by the body's counted interactions) resets the counter,
// otherwise it runs down; a body whose counter reached 0 is ready to sleep.
__device__ void sleep_check(const DevState& s, uint32_t b, qt q, v3 ml, v3 mw) {
    constexpr float kWakeReset = 20.0f * 0.02f;
    constexpr float kEnergy = 5.0e-5f * 10.0f * 10.0f;
    const float dt = s.dt;
    float wc = s.b_wake[b];
    float4* acc = s.b_sacc + 2 * size_t(b);
    v3 lin = ld3(acc[0]), ang = ld3(acc[1]);
    if (wc < kWakeReset * 0.5f || wc < dt) {
        const v3 la = rotinv_sc(q, mw);
        const v3 lacc = {lin.x + ml.x, lin.y + ml.y, lin.z + ml.z};
        const v3 aacc = {ang.x + la.x, ang.y + la.y, ang.z + la.z};
        if (!(vfinite(lacc) && vfinite(aacc))) atomicOr(s.err, kErrNonFinite);
        const float4 inv = s.b_inv[b];
        const v3 inertia = {inv.x > 0.0f ? 1.0f / inv.x : 1.0f, inv.y > 0.0f ? 1.0f / inv.y : 1.0f,
                            inv.z > 0.0f ? 1.0f / inv.z : 1.0f};
        const float angular = (aacc.x * aacc.x * inertia.x + aacc.y * aacc.y * inertia.y +
                               aacc.z * aacc.z * inertia.z) * inv.w;
        const float linear = lacc.x * lacc.x + lacc.y * lacc.y + lacc.z * lacc.z;
        const float energy = 0.5f * (angular + linear);
        const float cluster = 1.0f + float(s.b_counted[b]);
        const float threshold = cluster * kEnergy;
        if (energy >= threshold) {
            lin = {0, 0, 0};
            ang = {0, 0, 0};
            const float factor = threshold == 0.0f ? 2.0f : smin(energy / threshold, 2.0f);
            wc = factor * 0.5f * kWakeReset + dt * (cluster - 1.0f);
        } else {
            lin = lacc;
            ang = aacc;
            wc = smax(wc - dt, 0.0f);
        }
    } else {
        wc = smax(wc - dt, 0.0f);
    }
    const bool ready = wc == 0.0f;
    if (ready) { lin = {0, 0, 0}; ang = {0, 0, 0}; }
    s.b_wake[b] = wc;
    s.b_sleep[b] = ready ? kReady : 0u;
    acc[0] = st4(lin, 0.0f);
    acc[1] = st4(ang, 0.0f);
}

__global__ void k_integrate(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b) || is_asleep(s, b)) return;
    const float dt = s.dt;
    const v3 v = ld3(s.sb_v[b]), w = ld3(s.sb_w[b]);
    const float4* si = s.sb_sqrt_i + 3 * size_t(b);
    const v3 c0 = ld3(si[0]), c1 = ld3(si[1]), c2 = ld3(si[2]);
    const v3 mdv = ld3(s.sb_mdv[b]), mdw = ld3(s.sb_mdw[b]);
    const v3 fdv = ld3(s.sb_dv[b]), fdw = ld3(s.sb_dw[b]);
    const v3 ml = {v.x + mdv.x, v.y + mdv.y, v.z + mdv.z};
    const v3 mw = {w.x + c0.x * mdw.x + c1.x * mdw.y + c2.x * mdw.z,
                   w.y + c0.y * mdw.x + c1.y * mdw.y + c2.y * mdw.z,
                   w.z + c0.z * mdw.x + c1.z * mdw.y + c2.z * mdw.z};
    const v3 fv = {v.x + fdv.x, v.y + fdv.y, v.z + fdv.z};
    const v3 fw = {w.x + c0.x * fdw.x + c1.x * fdw.y + c2.x * fdw.z,
                   w.y + c0.y * fdw.x + c1.y * fdw.y + c2.y * fdw.z,
                   w.z + c0.z * fdw.x + c1.z * fdw.y + c2.z * fdw.z};
    const v3 center = mass_position(s, b);
    v3 p = {center.x + ml.x * dt, center.y + ml.y * dt, center.z + ml.z * dt};
    const qt mlq = ldq(s.b_ml_q[b]);
    qt q = integrate_q(mass_orientation(s, b), mw, dt);
    q = qmul(q, qconj(mlq));
    const v3 off = rot_sc(q, ld3(s.b_ml_p[b]));
    p = {p.x - off.x, p.y - off.y, p.z - off.z};
    if (!(vfinite(p) && isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w) && vfinite(fv) && vfinite(fw)))
        atomicOr(s.err, kErrNonFinite);
    s.b_p[b] = make_float4(p.x, p.y, p.z, s.b_p[b].w);
    s.b_q[b] = stq(q);
    s.b_v[b] = st4(fv, 0.0f);
    s.b_w[b] = st4(fw, 0.0f);
    if (s.sleep) sleep_check(s, b, q, ml, mw);
}

// An authored velocity wakes every dynamic body it is written to
// (scene.cpp:728-783): a sleeping body restarts with cleared filters.
__global__ void k_wake_bodies(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !is_dyn(s, b)) return;
    if (s.b_sleep[b] & kSleeping) {
        const float4 z = make_float4(0, 0, 0, 0);
        s.b_sacc[2 * size_t(b)] = z;
        s.b_sacc[2 * size_t(b) + 1] = z;
    }
    s.b_wake[b] = smax(s.b_wake[b], 0.4f);
    s.b_sleep[b] = 0u;
}

inline uint32_t grid_for(uint32_t n, uint32_t t, uint32_t cap) {
    const uint32_t g = (n + t - 1) / t;
    return g == 0 ? 1 : (g < cap ? g : cap);
}

}  // namespace

// The largest islands set the critical path of the partition and PGS
// stages: their one-CTA-per-island kernels launch with the device's highest
// priority so their CTAs take SMs before the many small-island blocks of
// the concurrent branches (graphs are instantiated with node priorities).
static int g_high_priority = 0;
template <class... KArgs, class... Args>
static void launch_high(void (*kernel)(KArgs...), uint32_t grid, uint32_t block, size_t smem, cudaStream_t st,
                        Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = g_high_priority;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Fork n side branches off st (or run everything on st without branches).
static void fork_branches(const Branches* br, cudaStream_t st, int n) {
    if (!br) return;
    cudaEventRecord(br->fork, st);
    for (int i = 0; i < n; ++i) cudaStreamWaitEvent(br->st[i], br->fork, 0);
}
static void join_branches(const Branches* br, cudaStream_t st, int n) {
    if (!br) return;
    for (int i = 0; i < n; ++i) {
        cudaEventRecord(br->join[i], br->st[i]);
        cudaStreamWaitEvent(st, br->join[i], 0);
    }
}

// Kinematic target velocities (scene.cpp:2005-2043): the velocities that
// carry the body's mass centre and orientation to its target in one step;
// zero without a pending target.
__global__ void k_kinematic_velocities(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !(s.b_flags[b] & kBodyKinematic)) return;
    const float4 z = make_float4(0, 0, 0, 0);
    if (!(s.b_sleep[b] & kKinPending)) { s.b_v[b] = z; s.b_w[b] = z; return; }
    const float inv_dt = 1.0f / s.dt;
    const v3 tp = ld3(s.b_ktarget[2 * size_t(b)]);
    const qt tq = ldq(s.b_ktarget[2 * size_t(b) + 1]);
    const v3 off = rot_sc(tq, ld3(s.b_ml_p[b]));
    const v3 target = {tp.x + off.x, tp.y + off.y, tp.z + off.z};
    const v3 center = mass_position(s, b);
    const v3 v = {(target.x - center.x) * inv_dt, (target.y - center.y) * inv_dt, (target.z - center.z) * inv_dt};
    qt rel = qmul(tq, qconj(ldq(s.b_q[b])));
    if (rel.w < 0.0f) rel = {-rel.x, -rel.y, -rel.z, -rel.w};
    const float len = sqrtf(rel.x * rel.x + rel.y * rel.y + rel.z * rel.z);
    v3 w = {0, 0, 0};
    if (len > 0.0f) {
        const float angle = 2.0f * atan2f(len, rel.w);
        const float scale = angle * inv_dt / len;
        w = {rel.x * scale, rel.y * scale, rel.z * scale};
    }
    if (!(vfinite(v) && vfinite(w))) atomicOr(s.err, kErrNonFinite);
    s.b_v[b] = st4(v, 0.0f);
    s.b_w[b] = st4(w, 0.0f);
}
// After the solve (scene.cpp:2045-2065): a kinematic body with a pending
// target takes it and is ready for sleep; the step after (settling), its
// velocity is zero (scene.cpp:10992-11005).
__global__ void k_kinematic_publish(DevState s) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies || !(s.b_flags[b] & kBodyKinematic)) return;
    uint32_t f = s.b_sleep[b];
    if (f & kKinPending) {
        const float4 tp = s.b_ktarget[2 * size_t(b)];
        s.b_p[b] = make_float4(tp.x, tp.y, tp.z, s.b_p[b].w);
        s.b_q[b] = s.b_ktarget[2 * size_t(b) + 1];
        f = (f & ~(kKinPending | kKinNew)) | kReady | kKinSettling;
    } else {
        f &= ~kKinSettling;
    }
    s.b_sleep[b] = f & ~kKinNew;
}

// Host-buffer transfers: the 14-float body records of read_bodies packed
// on the device (one D2H), and write_velocities' 6-float records unpacked
// on the device (one H2D) into the velocities, waking every dynamic body.
__global__ void k_pack_bodies(DevState s, float* out) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies) return;
    const float4 p = s.b_p[b], v = s.b_v[b], q = s.b_q[b], w = s.b_w[b];
    float* o = out + 14 * size_t(b);
    o[0] = p.x; o[1] = p.y; o[2] = p.z;
    o[3] = v.x; o[4] = v.y; o[5] = v.z;
    o[6] = q.x; o[7] = q.y; o[8] = q.z; o[9] = q.w;
    o[10] = w.x; o[11] = w.y; o[12] = w.z;
    o[13] = (s.b_sleep[b] & kSleeping) ? 1.0f : 0.0f;
}
// Velocities from host records of `stride` floats: linear at lin, angular
// at ang (6-float records: 0 / 3; the 14-float body records: 3 / 10).
__global__ void k_unpack_velocities(DevState s, const float* rec, uint32_t stride, uint32_t lin, uint32_t ang) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= s.n_bodies) return;
    const bool dyn = is_dyn(s, b);
    const float* r = rec + stride * size_t(b);
    s.b_v[b] = dyn ? make_float4(r[lin], r[lin + 1], r[lin + 2], 0.0f) : make_float4(0, 0, 0, 0);
    s.b_w[b] = dyn ? make_float4(r[ang], r[ang + 1], r[ang + 2], 0.0f) : make_float4(0, 0, 0, 0);
}
void enqueue_pack_bodies(const DevState& s, float* out, cudaStream_t st) {
    if (s.n_bodies) k_pack_bodies<<<grid_for(s.n_bodies, 256, 1u << 30), 256, 0, st>>>(s, out);
}
void enqueue_unpack_velocities(const DevState& s, const float* rec, uint32_t stride, uint32_t lin, uint32_t ang,
                               cudaStream_t st) {
    if (!s.n_bodies) return;
    k_unpack_velocities<<<grid_for(s.n_bodies, 256, 1u << 30), 256, 0, st>>>(s, rec, stride, lin, ang);
    k_wake_bodies<<<grid_for(s.n_bodies, 256, 1u << 30), 256, 0, st>>>(s);
}

void enqueue_wake_bodies(const DevState& s, cudaStream_t st) {
    if (s.n_bodies) k_wake_bodies<<<grid_for(s.n_bodies, 256, 1u << 30), 256, 0, st>>>(s);
}

void init_solver_kernels() {
    init_primitive_kernels();
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) g_high_priority = greatest;
    cudaFuncSetAttribute(k_partition_smem<kBigIsland>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(PartSmem<kBigIsland>::kBytes));
    cudaFuncSetAttribute(k_pgs_block_smem<kBigIsland, kBigPgsThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(PgsSmem<kBigIsland>::kBytes));
}

void enqueue_solver(const DevState& s, cudaStream_t st, const StageHook& hook, const Branches* br) {
    uint32_t* lvl_bound = s.lvl_bound;
    const uint32_t T = s.elem_block;   // elementwise kernels (at most 56 registers, no launch bounds)
    const uint32_t cap_blocks = 148u * 8u;
    auto side = [&](int i) { return br ? br->st[i] : st; };
    hook(kStIslands, st);
    k_frame_begin<<<1, 32, 0, st>>>(s);
    cudaMemsetAsync(s.counters + kCntAwake, 0, 2 * sizeof(uint32_t), st);
    cudaMemsetAsync(s.counters + kCntReady, 0, sizeof(uint32_t), st);
    cudaMemsetAsync(s.counters + kCntActivating, 0, sizeof(uint32_t), st);
    k_bodies_begin<<<grid_for(s.n_bodies, T, 1u << 30), T, 0, st>>>(s);
    // touching managers in canonical pair order
    k_touch_compact<<<lookback_grid(s.pair_cap), kScanThreads, 0, st>>>(s);
    // islands
    k_desc_bodies<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
    k_union<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
    if (s.sleep) {
        const uint32_t bb = grid_for(s.n_bodies, T, 1u << 30);
        if (s.n_kinematic && s.n_joints)
            k_sleep_kinematic_joints<<<grid_for(s.n_joints, T, 1u << 30), T, 0, st>>>(s);
        k_sleep_spec<<<grid_for(2u * s.pair_cap, T, cap_blocks), T, 0, st>>>(s);
        k_sleep_wake_roots<<<bb, T, 0, st>>>(s);
        k_sleep_wake_flags<<<bb, T, 0, st>>>(s);
        k_sleep_decide<<<bb, T, 0, st>>>(s);
    }
    if (s.n_kinematic) k_kinematic_velocities<<<grid_for(s.n_bodies, T, 1u << 30), T, 0, st>>>(s);
    k_bodies_velocity<<<grid_for(s.n_bodies, T, 1u << 30), T, 0, st>>>(s);
    k_desc_keys<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
    if (s.replay) {
        int rbits = 1;
        while ((1ull << rbits) < uint64_t(s.n_joints) + 2ull * s.pair_cap + 1u) ++rbits;
        k_replay_keys<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
        radix_sort_pairs(s.d_key, s.d_val, s.d_key2, s.d_val2, s.desc_cap, s.counters + kCntDesc, 0, rbits,
                         s.sort_hist, s.sort_hist_words, s.scan_tmp, s.scan_tmp_words, st, s.err, s.radix_bits, s.sort_os, s.sort_os_words);
        k_replay_rekey<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
    }
    // keys are island roots < n_bodies, or n_bodies for sleeping islands
    int bits = 1;
    while ((1ull << bits) < uint64_t(s.n_bodies) + 1u) ++bits;
    radix_sort_pairs(s.d_key, s.d_val, s.d_key2, s.d_val2, s.desc_cap, s.counters + kCntDesc, 0, bits,
                     s.sort_hist, s.sort_hist_words, s.scan_tmp, s.scan_tmp_words, st, s.err, s.radix_bits, s.sort_os, s.sort_os_words);
    k_island_compact<<<lookback_grid(s.desc_cap), kScanThreads, 0, st>>>(s);
    k_island_classes<<<grid_for(s.desc_cap, T, cap_blocks), T, 0, st>>>(s);
    // partitions by island size class, and row preparation: independent
    hook(kStPrep, st);
    fork_branches(br, st, 3);
    launch_high(k_partition_smem<kBigIsland>, grid_for(s.desc_cap, kMidIsland + 1, 148u * 2u), 256u,
                PartSmem<kBigIsland>::kBytes, side(1), s, lvl_bound, 2);
    launch_high(k_partition_large, grid_for(s.desc_cap, kBigIsland + 1, 148u), 256u, size_t(0), side(1), s,
                lvl_bound);
    k_partition<<<grid_for(s.desc_cap, kPartWarps, 148u * 16u), kPartWarps * 32, 0, st>>>(s, lvl_bound);
    k_partition_smem<kMidIsland><<<grid_for(s.desc_cap, kSerialIsland + 1, 148u * 8u), 256,
                                   PartSmem<kMidIsland>::kBytes, side(0)>>>(s, lvl_bound, 0);
    if (s.n_joints) k_prep_joints<<<grid_for(s.n_joints, 128, 1u << 30), 128, 0, side(2)>>>(s);   // ~150 registers
    k_prep_contacts<<<grid_for(s.desc_cap, 128, cap_blocks), 128, 0, side(2)>>>(s);
    join_branches(br, st, 3);
    // PGS: islands by size class, independent
    hook(kStPgs, st);
    fork_branches(br, st, 3);
    launch_high(k_pgs_block_smem<kBigIsland, kBigPgsThreads>, grid_for(s.desc_cap, s.isl_mid + 1, 148u),
                kBigPgsThreads, PgsSmem<kBigIsland>::kBytes, side(1), s, lvl_bound, 4);
    launch_high(k_pgs_block, grid_for(s.desc_cap, kBigIsland + 1, 148u), 256u, size_t(0), side(1), s, lvl_bound);
    k_pgs_warp<<<grid_for(s.desc_cap * 32u, kPgsWarpsPerBlock * 32u, 148u * 3u), kPgsWarpsPerBlock * 32u, 0, st>>>(
        s, lvl_bound);
    k_pgs_block_smem<kMidIsland, 128><<<grid_for(s.desc_cap, s.isl_warp + 1, 148u * 3u), 128,
                                        PgsSmem<kMidIsland>::kBytes, side(0)>>>(s, lvl_bound, 1);
    k_pgs_thread<<<grid_for(s.desc_cap, kPgsThreadBlock, 148u * 8u), kPgsThreadBlock, 0, side(2)>>>(s);
    join_branches(br, st, 3);
    hook(kStIntegrate, st);
    k_integrate<<<grid_for(s.n_bodies, T, 1u << 30), T, 0, st>>>(s);
    if (s.n_kinematic) k_kinematic_publish<<<grid_for(s.n_bodies, T, 1u << 30), T, 0, st>>>(s);
    if (s.thresholds) enqueue_thresholds(s, st);
    if (s.events) enqueue_events(s, st);
    hook(kStEnd, st);
}

}  // namespace fyzz::b200
