// Broadphase: shape poses, integer-encoded AABBs, the sorted x-axis sweep
// and canonical overlap-pair publication (found / lost against the
// previous generation).
//
// Reference behaviour (src/native/scene.cpp):
//   encode_float/min/max             26-35
//   Scene::update_shape_bounds       1233-1316   (box basis extent, sphere r,
//                                                 plus contact offset)
//   Scene::update_bounds endpoint order 1341-1345 (value, min-before-max, id)
//   Scene::update_pairs full sweep   2635-2704   (y/z test, different bodies,
//                                                 at least one dynamic; planes
//                                                 pair with every dynamic volume)
//   Scene::publish_pairs             3230-3304   (sorted merge -> found / lost)
//
// B200 layout: min-x keys are sorted per scene (one CTA per scene when the
// scene fits in shared memory, otherwise the device-wide radix sort); the
// sweep then reads y/z bounds gathered into sorted order so the candidate
// scan is a contiguous read.  Pairs are emitted into per-owner buckets
// (owner = lower shape id) so the published list is already in canonical
// (a, b) order after a per-bucket sort, without a device-wide pair sort.
#include "state.h"

namespace fyzz::b200 {
namespace {

__device__ __forceinline__ uint32_t encode_float(float v) {
    const uint32_t bits = __float_as_uint(v);
    return (bits & 0x80000000u) ? ~bits : (bits | 0x80000000u);
}
__device__ __forceinline__ uint32_t encode_min(float v) { return ((encode_float(v) >> 4) - 1u) << 4; }
__device__ __forceinline__ uint32_t encode_max(float v) { return (((encode_float(v) >> 4) + 1u) << 4) | 4u; }

__global__ void k_shape_bounds(DevState s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_shapes) return;
    const uint32_t b = s.s_body[i];
    const v3 bp = ld3(s.b_p[b]);
    const qt bq = ldq(s.b_q[b]);
    const float4 lp = s.s_lp[i];
    const v3 wp = vadd(bp, rot_sc(bq, ld3(lp)));           // scene.cpp:366-371
    const qt wq = qmul(bq, ldq(s.s_lq[i]));
    s.s_wp[i] = st4(wp, 0.0f);
    s.s_wq[i] = stq(wq);
    const uint32_t type = s.s_type[i];
    if (type == kPlane) return;
    const float4 g = s.s_geom[i];
    const v3 h = {g.x, g.y, g.z};
    v3 e = type == kSphere ? v3{g.w, g.w, g.w} : h;
    v3 c = wp;
    if (type == kBox && (wq.x != 0.0f || wq.y != 0.0f || wq.z != 0.0f || wq.w != 1.0f)) {
        const v3 x = rot_sc(wq, {1, 0, 0}), y = rot_sc(wq, {0, 1, 0}), z = rot_sc(wq, {0, 0, 1});
        e = {fabsf(x.x) * h.x + fabsf(y.x) * h.y + fabsf(z.x) * h.z,
             fabsf(x.y) * h.x + fabsf(y.y) * h.y + fabsf(z.y) * h.z,
             fabsf(x.z) * h.x + fabsf(y.z) * h.y + fabsf(z.z) * h.z};
    } else if (type == kConvex) {
        // the rotated hull's vertex bounds, centred where the hull is
        // (scene.cpp:1258-1298)
        const uint4 mt = s.m_tab[s.s_mesh[i]];
        v3 vlo = {INFINITY, INFINITY, INFINITY}, vhi = {-INFINITY, -INFINITY, -INFINITY};
        for (uint32_t v = 0; v < mt.y; ++v) {
            const v3 r = rot_sc(wq, ld3(s.hv[mt.x + v]));
            vlo = {smin(vlo.x, r.x), smin(vlo.y, r.y), smin(vlo.z, r.z)};
            vhi = {smax(vhi.x, r.x), smax(vhi.y, r.y), smax(vhi.z, r.z)};
        }
        c = {wp.x + (vhi.x + vlo.x) * 0.5f, wp.y + (vhi.y + vlo.y) * 0.5f, wp.z + (vhi.z + vlo.z) * 0.5f};
        e = {(vhi.x - vlo.x) * 0.5f, (vhi.y - vlo.y) * 0.5f, (vhi.z - vlo.z) * 0.5f};
    }
    const float co = lp.w;
    e.x += co; e.y += co; e.z += co;
    const float lo[3] = {c.x - e.x, c.y - e.y, c.z - e.z};
    const float hi[3] = {c.x + e.x, c.y + e.y, c.z + e.z};
    if (!(isfinite(lo[0]) && isfinite(lo[1]) && isfinite(lo[2]) &&
          isfinite(hi[0]) && isfinite(hi[1]) && isfinite(hi[2])))
        atomicOr(s.err, kErrNonFinite);
    const uint4 elo = make_uint4(encode_min(lo[0]), encode_min(lo[1]), encode_min(lo[2]), 0u);
    const uint4 ehi = make_uint4(encode_max(hi[0]), encode_max(hi[1]), encode_max(hi[2]), 0u);
    s.s_lo[i] = elo;
    s.s_hi[i] = ehi;
    const int32_t f = s.s_frank[i];
    s.srt_key[f] = elo.x;
    s.srt_id[f] = i;
}

// One CTA sorts one scene's min-x endpoints by (value, shape id): bitonic
// sort of 64-bit keys in shared memory.
constexpr int kSmallSortThreads = 1024;
__global__ void __launch_bounds__(kSmallSortThreads) k_sort_small(DevState s) {
    extern __shared__ unsigned long long sk[];
    const uint32_t scene = s.small_scenes[blockIdx.x];
    const uint32_t begin = s.sc_fbegin[scene], end = s.sc_fbegin[scene + 1];
    const uint32_t n = end - begin;
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x)
        sk[i] = i < n ? ((unsigned long long)s.srt_key[begin + i] << 32) | s.srt_id[begin + i]
                      : ~0ull;
    __syncthreads();
    for (uint32_t k = 2; k <= m; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = sk[i], b = sk[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) { sk[i] = b; sk[ixj] = a; }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        s.srt_key[begin + i] = uint32_t(sk[i] >> 32);
        s.srt_id[begin + i] = uint32_t(sk[i]);
    }
}

// ---- z bands of large scenes ----
// A one-axis sweep of a wide scene tests every shape against all shapes
// whose x ranges overlap its own, most of them far away in z (a settled
// 200 x 200 m pile: ~360 candidates per shape for 2.7 pairs).  Large scenes
// are therefore swept per band of z: bands are at least as wide as the
// widest shape's z extent, so a shape lies in one or two bands; each band's
// entries keep the x order of the sorted endpoints, and a pair found in a
// band counts only in the band of the larger of the two min z (a band both
// shapes lie in, since the band index is monotone in z), which makes the
// published pair set identical to the one-axis sweep's.
__device__ __forceinline__ float decode_enc(uint32_t e) {
    return __uint_as_float((e & 0x80000000u) ? (e & 0x7fffffffu) : ~e);
}
// Band of an encoded z bound: floor((z - z0) / width), clamped; monotone in
// the encoded value (float subtraction and scaling by a non-negative
// factor are monotone).
__device__ __forceinline__ uint32_t band_of(uint32_t e, float4 par) {
    const float t = (decode_enc(e) - par.x) * par.y;
    if (!(t > 0.0f)) return 0u;
    return t >= float(DevState::kBands - 1) ? DevState::kBands - 1 : uint32_t(t);
}
// Per block of one large scene (blockIdx.y): min z, max z and the widest z
// extent of its shapes.
__global__ void __launch_bounds__(256) k_band_stats(DevState s, const uint4* __restrict__ rec) {
    const uint32_t L = blockIdx.y, begin = s.large_begin[L], n = s.large_n[L];
    uint32_t zmin = ~0u, zmax = 0u;
    float ext = 0.0f;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint4 r = rec[begin + k];
        zmin = min(zmin, r.z);
        zmax = max(zmax, r.w);
        const float e = decode_enc(r.w) - decode_enc(r.z);
        ext = e > ext ? e : ext;
    }
    for (int o = 16; o > 0; o >>= 1) {
        zmin = min(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
        zmax = max(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
        const float e = __shfl_xor_sync(0xffffffffu, ext, o);
        ext = e > ext ? e : ext;
    }
    __shared__ uint4 part[8];
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    if (lane == 0) part[w] = make_uint4(zmin, zmax, __float_as_uint(ext), 0u);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint4 r = part[0];
        for (uint32_t k = 1; k < blockDim.x / 32u; ++k) {
            r.x = min(r.x, part[k].x);
            r.y = max(r.y, part[k].y);
            r.z = __uint_as_float(part[k].z) > __uint_as_float(r.z) ? part[k].z : r.z;
        }
        s.bd_part[L * DevState::kBandStatBlocks + blockIdx.x] = r;
    }
}
// One warp per large scene: band origin and width (the widest shape's z
// extent with a margin, and at least 1/250 of the scene's z range).
__global__ void k_band_params(DevState s) {
    const uint32_t L = blockIdx.x, lane = threadIdx.x;
    uint32_t zmin = ~0u, zmax = 0u;
    float ext = 0.0f;
    for (uint32_t k = lane; k < DevState::kBandStatBlocks; k += 32) {
        const uint4 r = s.bd_part[L * DevState::kBandStatBlocks + k];
        zmin = min(zmin, r.x);
        zmax = max(zmax, r.y);
        ext = __uint_as_float(r.z) > ext ? __uint_as_float(r.z) : ext;
    }
    for (int o = 16; o > 0; o >>= 1) {
        zmin = min(zmin, __shfl_xor_sync(0xffffffffu, zmin, o));
        zmax = max(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
        const float e = __shfl_xor_sync(0xffffffffu, ext, o);
        ext = e > ext ? e : ext;
    }
    if (lane == 0) {
        const float z0 = decode_enc(zmin), z1 = decode_enc(zmax);
        float width = ext * 1.001f;
        const float floor_w = (z1 - z0) / 250.0f;
        if (floor_w > width) width = floor_w;
        const bool ok = isfinite(z0) && isfinite(z1) && isfinite(width) && width > 0.0f;
        s.bd_par[L] = make_float4(ok ? z0 : 0.0f, ok ? 1.0f / width : 0.0f, 0.0f, 0.0f);
    }
}
// Bands each x-sorted finite shape of a large scene lies in (one or two).
__global__ void k_band_count(DevState s, const uint4* __restrict__ rec) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n_finite) return;
    const int32_t L = s.sc_large[s.s_scene[s.srt_id[p]]];
    uint32_t c = 0;
    if (L >= 0) {
        const float4 par = s.bd_par[L];
        const uint4 r = rec[p];
        const uint32_t b0 = band_of(r.z, par), b1 = band_of(r.w, par);
        c = b1 >= b0 ? b1 - b0 + 1u : 1u;
        if (c > 2u) {
            // bands are wider than every extent: only non-finite bounds (an
            // error of their own) get here
            if (isfinite(decode_enc(r.z)) && isfinite(decode_enc(r.w))) atomicOr(s.err, kErrLogic);
            c = 2u;
        }
    }
    s.bd_cnt[p] = c;
}
// Band entries in x order: key (large scene << 8 | band), value the x-sorted
// position.
__global__ void k_band_expand(DevState s, const uint4* __restrict__ rec) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= s.n_finite) return;
    const uint32_t c = s.bd_cnt[p];
    if (c == 0u) return;
    const int32_t L = s.sc_large[s.s_scene[s.srt_id[p]]];
    const uint32_t b0 = band_of(rec[p].z, s.bd_par[L]);
    const uint32_t q = s.bd_off[p];
    for (uint32_t k = 0; k < c; ++k) {
        if (q + k >= s.bx_cap) { atomicOr(s.err, kErrLogic); return; }   // never: 2 entries per shape at most
        s.bx_key[q + k] = (uint32_t(L) << 8) | min(b0 + k, DevState::kBands - 1);
        s.bx_val[q + k] = p;
    }
}
// The band entries (sorted by key, x order within) appended to the sweep
// list after the x-sorted finite shapes, and each band's end.
__global__ void k_band_gather(DevState s, uint4* rec, uint2* meta) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t n = *s.bd_n;
    if (q >= n) return;
    const uint32_t key = s.bx_key[q], p = s.bx_val[q], nf = s.n_finite;
    if (q + 1 == n || s.bx_key[q + 1] != key) s.bd_end[key] = q + 1;
    s.srt_key[nf + q] = s.srt_key[p];
    s.srt_id[nf + q] = s.srt_id[p];
    rec[nf + q] = rec[p];
    meta[nf + q] = meta[p];
}

// Gather the sweep records into sorted order: (min y, max y, min z, max z)
// and (max x, body | dynamic << 31).
__global__ void k_sweep_gather(DevState s, uint4* rec, uint2* meta) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_finite) return;
    const uint32_t id = s.srt_id[i];
    const uint4 lo = s.s_lo[id], hi = s.s_hi[id];
    const uint32_t body = s.s_body[id];
    const uint32_t dyn = s.b_flags[body] & kBodyDynamic;
    rec[i] = make_uint4(lo.y, hi.y, lo.z, hi.z);
    meta[i] = make_uint2(hi.x, body | (dyn << 31));
}

__device__ __forceinline__ void emit_pair(const DevState& s, uint32_t id, uint32_t other) {
    const uint32_t owner = min(id, other), partner = max(id, other);
    const uint32_t pos = s.own_off[owner] + s.s_static_pairs[owner] + atomicAdd(&s.own_cur[owner], 1u);
    if (pos < s.pair_cap) s.cur.key[pos] = (uint64_t(owner) << 32) | partner;
    else atomicOr(s.err, kErrPairCapacity);
}

// Warp-cooperative sweep.  Lane l owns sorted shape i = base + l; the warp
// walks the candidates after base in chunks of 32 loaded once (coalesced)
// into shared memory, and every lane tests its own shape against each
// staged candidate (j > i, same scene, min x <= its max x, different body,
// one dynamic, y/z overlap) until all lanes have passed their max x.
// fill = 0: count each pair for its owner and keep up to kSweepCache
// partners per shape.  fill = 1: write the kept partners into the owner
// buckets; lanes that found more rescan (the warp walks again only if one
// of its lanes needs it).
constexpr int kSweepWarps = 8;
struct SweepCand { uint32_t key, id, body, pad; uint4 yz; };

__global__ void __launch_bounds__(kSweepWarps * 32) k_sweep(DevState s, const uint4* __restrict__ rec,
                                                           const uint2* __restrict__ meta, int fill) {
    constexpr uint32_t C = DevState::kSweepCache;
    __shared__ SweepCand stage[kSweepWarps][32];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    SweepCand* st = stage[wib];
    const uint32_t nwarps = gridDim.x * kSweepWarps;
    const uint32_t nf = s.n_finite;
    const uint32_t n = nf + (s.n_large ? *s.bd_n : 0u);
    constexpr uint32_t kNoBand = ~0u;
    for (uint32_t base = (blockIdx.x * kSweepWarps + wib) * 32u; base < n; base += nwarps * 32u) {
        const uint32_t i = base + lane;
        const bool valid = i < n;
        uint32_t id = 0, scene_end = 0, abody = 0, band = kNoBand;
        float4 par = make_float4(0, 0, 0, 0);
        bool sweeps = valid;
        uint2 am = make_uint2(0, 0);
        uint4 a = make_uint4(0, 0, 0, 0);
        bool adyn = false;
        uint32_t nfound = 0;
        if (valid) {
            id = s.srt_id[i];
            if (i < nf) {
                const uint32_t sc = s.s_scene[id];
                scene_end = s.sc_fbegin[sc + 1];
                // a large scene's x-sorted entries publish plane pairs only;
                // its band entries sweep
                if (s.n_large && s.sc_large[sc] >= 0) sweeps = false;
            } else {
                const uint32_t key = s.bx_key[i - nf];
                scene_end = nf + s.bd_end[key];
                band = key & (DevState::kBands - 1u);
                par = s.bd_par[key >> 8];
            }
            am = meta[i];
            a = rec[i];
            abody = am.y & 0x7fffffffu;
            adyn = (am.y >> 31) != 0u;
        }
        uint32_t* cache = s.sw_cache + size_t(i) * C;
        bool scan = sweeps;
        if (fill && valid) {
            nfound = s.sw_found[i];
            if (nfound <= C) {
                for (uint32_t c = 0; c < nfound; ++c) emit_pair(s, id, cache[c]);
                scan = false;
            }
        }
        uint32_t found = 0;
        bool active = scan;
        for (uint32_t j0 = base + 1; __any_sync(0xffffffffu, active); j0 += 32) {
            const uint32_t jl = j0 + lane;
            if (jl < n) {
                SweepCand c;
                c.key = s.srt_key[jl];
                c.id = s.srt_id[jl];
                c.body = meta[jl].y;
                c.pad = 0u;
                c.yz = rec[jl];
                st[lane] = c;
            }
            __syncwarp();
            if (active) {
                for (uint32_t t = 0; t < 32; ++t) {
                    const uint32_t j = j0 + t;
                    if (j >= scene_end || j >= n) { active = false; break; }
                    if (j <= i) continue;
                    const SweepCand& c = st[t];
                    if (c.key > am.x) { active = false; break; }
                    if ((c.body & 0x7fffffffu) == abody) continue;
                    if (!adyn && (c.body >> 31) == 0u) continue;
                    const uint4 b = c.yz;
                    if (a.x > b.y || b.x > a.y || a.z > b.w || b.z > a.w) continue;
                    if (band != kNoBand && band_of(max(a.z, b.z), par) != band) continue;
                    if (!fill) {
                        atomicAdd(&s.own_cnt[min(id, c.id)], 1u);
                        if (found < C) cache[found] = c.id;
                        ++found;
                    } else {
                        emit_pair(s, id, c.id);
                    }
                }
            }
            __syncwarp();
        }
        if (!fill && valid) s.sw_found[i] = found;
        if (fill && valid && i < nf && adyn) {
            const int32_t p = s.sc_plane[s.s_scene[id]];
            if (p >= 0) {
                const uint32_t pp = uint32_t(p);
                const uint32_t pos = pp < id ? s.own_off[pp] + uint32_t(s.s_dynrank[id]) : s.own_off[id];
                const uint32_t owner = min(pp, id), partner = max(pp, id);
                if (pos < s.pair_cap) s.cur.key[pos] = (uint64_t(owner) << 32) | partner;
                else atomicOr(s.err, kErrPairCapacity);
            }
        }
    }
}

// Sort each owner's bucket by partner id.  Plane owners are filled in
// ascending order already.
__global__ void k_owner_sort(DevState s) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= s.n_shapes || s.s_type[o] == kPlane) return;
    const uint32_t n = s.s_static_pairs[o] + s.own_cur[o];
    if (n < 2) return;
    const uint32_t b = s.own_off[o];
    if (b + n > s.pair_cap) return;
    uint64_t* k = s.cur.key + b;
    for (uint32_t i = 1; i < n; ++i) {
        const uint64_t v = k[i];
        uint32_t j = i;
        while (j > 0 && k[j - 1] > v) { k[j] = k[j - 1]; --j; }
        k[j] = v;
    }
}

__global__ void k_pair_total(DevState s) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const uint32_t total = *s.cur.n;
        if (total > s.pair_cap) {
            atomicOr(s.err, kErrPairCapacity);
            *s.cur.n = s.pair_cap;
        }
    }
}

__device__ __forceinline__ int32_t find_key(const uint64_t* keys, uint32_t lo, uint32_t hi, uint64_t key) {
    const uint32_t end = hi;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return (lo < end && keys[lo] == key) ? int32_t(lo) : -1;
}

// Per shape, before the sweep: its bucket count starts at its plane pairs,
// its fill cursor at zero, and its previous-generation bucket empty.
__global__ void k_owner_init(DevState s) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n_shapes) return;
    s.own_cnt[i] = s.s_static_pairs[i];
    s.own_cur[i] = 0u;
    s.prev_bkt[i] = make_uint2(0u, 0u);
}

// Each generation's keys are sorted by (owner, partner), owners being
// contiguous buckets: the previous generation's bucket of every owner
// (start, end; both zero for an owner without pairs), so that matching
// searches a handful of keys instead of the whole list.
__global__ void k_prev_buckets(DevState s) {
    const uint32_t np = *s.prev.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < np; j += stride) {
        const uint32_t a = uint32_t(s.prev.key[j] >> 32);
        if (a >= s.n_shapes) continue;
        if (j == 0 || uint32_t(s.prev.key[j - 1] >> 32) != a) s.prev_bkt[a].x = j;
        if (j + 1 == np || uint32_t(s.prev.key[j + 1] >> 32) != a) s.prev_bkt[a].y = j + 1;
    }
}

// Found and lost by matching the two generations bucket by bucket: a
// current pair's owner bucket in the previous keys, a previous pair's in
// the current ones (own_off / own_cnt of this step's sweep).
__global__ void k_pair_match(DevState s) {
    const uint32_t n = *s.cur.n, np = *s.prev.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const uint64_t key = s.cur.key[k];
        const uint32_t a = uint32_t(key >> 32);
        const uint2 b = a < s.n_shapes ? s.prev_bkt[a] : make_uint2(0u, 0u);
        const int32_t j = find_key(s.prev.key, b.x, min(b.y, np), key);
        s.prev_idx[k] = j;
        s.found_flag[k] = j < 0 ? 1u : 0u;
    }
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += stride) {
        const uint64_t key = s.prev.key[k];
        const uint32_t a = uint32_t(key >> 32);
        const uint32_t lo = a < s.n_shapes ? min(s.own_off[a], n) : 0u;
        const uint32_t hi = a < s.n_shapes ? min(s.own_off[a] + s.own_cnt[a], n) : 0u;
        s.lost_flag[k] = find_key(s.cur.key, lo, hi, key) < 0 ? 1u : 0u;
    }
}

}  // namespace

void enqueue_broadphase(const DevState& s, cudaStream_t st, const StageHook& hook) {
    uint4* rec = s.sw_rec;
    uint2* meta = s.sw_meta;
    const int T = 256;
    hook(kStBounds, st);
    k_shape_bounds<<<(s.n_shapes + T - 1) / T, T, 0, st>>>(s);
    hook(kStSort, st);
    if (s.n_small) {
        uint32_t m = 1;
        while (m < s.max_small_scene) m <<= 1;
        k_sort_small<<<s.n_small, kSmallSortThreads, m * sizeof(unsigned long long), st>>>(s);
    }
    for (uint32_t i = 0; i < s.n_large; ++i)
        radix_sort_pairs(s.srt_key + s.large_begin[i], s.srt_id + s.large_begin[i],
                         s.srt_key2, s.srt_id2, s.large_n[i], nullptr, 0, 32,
                         s.sort_hist, s.sort_hist_words, s.scan_tmp, s.scan_tmp_words, st, s.err, s.radix_bits, s.sort_os, s.sort_os_words);
    hook(kStPairs, st);
    if (s.n_finite) {
        k_sweep_gather<<<(s.n_finite + T - 1) / T, T, 0, st>>>(s, rec, meta);
    }
    if (s.n_large) {
        int kbits = 0;
        while ((1u << kbits) < s.n_large) ++kbits;
        k_band_stats<<<dim3(DevState::kBandStatBlocks, s.n_large), 256, 0, st>>>(s, rec);
        k_band_params<<<s.n_large, 32, 0, st>>>(s);
        k_band_count<<<(s.n_finite + T - 1) / T, T, 0, st>>>(s, rec);
        scan_exclusive(s.bd_cnt, s.bd_off, s.n_finite, nullptr, s.bd_n, s.scan_tmp, s.scan_tmp_words, st, s.err);
        k_band_expand<<<(s.n_finite + T - 1) / T, T, 0, st>>>(s, rec);
        radix_sort_pairs(s.bx_key, s.bx_val, s.bx_key2, s.bx_val2, s.bx_cap, s.bd_n, 0, 8 + kbits, s.sort_hist,
                         s.sort_hist_words, s.scan_tmp, s.scan_tmp_words, st, s.err, 8, s.sort_os, s.sort_os_words);
        k_band_gather<<<(s.bx_cap + T - 1) / T, T, 0, st>>>(s, rec, meta);
    }
    if (s.n_shapes) k_owner_init<<<(s.n_shapes + T - 1) / T, T, 0, st>>>(s);
    const uint32_t sweep_threads = kSweepWarps * 32;
    const uint32_t n_sweep = s.n_finite + s.bx_cap;
    const uint32_t sweep_blocks = s.n_finite ? (n_sweep + sweep_threads - 1) / sweep_threads : 0;
    if (sweep_blocks) k_sweep<<<sweep_blocks, sweep_threads, 0, st>>>(s, rec, meta, 0);
    scan_exclusive(s.own_cnt, s.own_off, s.n_shapes, nullptr, s.cur.n, s.scan_tmp, s.scan_tmp_words, st, s.err);
    k_pair_total<<<1, 32, 0, st>>>(s);
    if (sweep_blocks) k_sweep<<<sweep_blocks, sweep_threads, 0, st>>>(s, rec, meta, 1);
    k_owner_sort<<<(s.n_shapes + T - 1) / T, T, 0, st>>>(s);
    const uint32_t mb = (s.pair_cap + T - 1) / T;
    k_prev_buckets<<<mb < 1184 ? mb : 1184, T, 0, st>>>(s);
    k_pair_match<<<mb < 1184 ? mb : 1184, T, 0, st>>>(s);
}

}  // namespace fyzz::b200
