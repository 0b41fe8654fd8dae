// Narrowphase: persistent-contact-manifold (PCM) contact generation for every
// broadphase pair, one thread per pair.
//
// Reference routines (paths relative to the reference project):
//   src/native/GuPCMContactBoxBox.cpp:301-436  box/box SAT, reference face,
//                                              incident clipping (<= 64 cands)
//   src/native/GuPCMContactBoxBox.cpp:185-297  batch reduction to 4
//   src/native/GuPCMGjkEpa.cpp:44-570          GJK / EPA zero-face continuation
//   src/native/GuPCMContactSphere.cpp:49-130   sphere/sphere, sphere/plane,
//                                              sphere/box
//   src/native/scene.cpp:3432-3465             manifold refresh
//   src/native/scene.cpp:3319-3431             fifth-point reduction
//   src/native/scene.cpp:3466-3654             box/box manifold lifecycle
//   src/native/scene.cpp:3774-3955             plane/box manifold lifecycle
//   src/native/scene.cpp:4012-4700             per-pair dispatch, Gu order
//                                              (statics second, dynamics by
//                                              descending body id), normal flips
// The manifold cache of each pair is gathered from the previous generation
// through prev_idx and written to the current one, so the step never reads
// and writes the same record.
#include "state.h"
#include <cfloat>

namespace fyzz::b200 {
namespace {

struct Cand { v3 la, lb, nb; float sep; };
// Incident-face clipping emits at most 4 vertices + 4 reference corners +
// 2 points per edge of the 4-edge incident polygon.
constexpr int kMaxBoxCandidates = 16;

// ---------------- box/box face contacts ----------------
struct GBox { v3 half, pos; qt rot; v3 axis[3]; };
__device__ GBox make_box(v3 h, v3 p, qt q) {
    GBox b;
    b.half = h; b.pos = p; b.rot = q;
    b.axis[0] = rot_gu(q, {1, 0, 0});
    b.axis[1] = rot_gu(q, {0, 1, 0});
    b.axis[2] = rot_gu(q, {0, 0, 1});
    return b;
}
struct Frame { v3 x, y, z, p; };
__device__ __forceinline__ v3 fr_project(const Frame& f, v3 w) {
    const v3 d = vsub(w, f.p);
    return {vdot(d, f.x), vdot(d, f.y), vdot(d, f.z)};
}
__device__ __forceinline__ v3 fr_unproject(const Frame& f, v3 v) {
    return vadd(f.p, vadd(vadd(vmul(f.x, v.x), vmul(f.y, v.y)), vmul(f.z, v.z)));
}
__device__ bool poly_contains(const v3* poly, v3 p, v3 low, v3 high) {
    if (p.x < low.x || p.y < low.y || p.x > high.x || p.y > high.y) return false;
    unsigned hits = 0;
    const float eps = FLT_EPSILON;
    for (unsigned i = 0, j = 3; i < 4; j = i++) {
        const v3 a = poly[j], b = poly[i];
        if ((p.x == a.x && p.y == a.y) || (p.x == b.x && p.y == b.y)) return true;
        if ((a.y > p.y) != (b.y > p.y)) {
            const float dx = b.x - a.x, dy = b.y - a.y;
            const float part = (p.y - a.y) * dx + (a.x + eps) * dy;
            const float target = p.x * dy;
            const bool inter = dy > 0.0f ? part >= target : target >= part;
            if (inter && ++hits == 2) return false;
        }
    }
    return hits > 0;
}
__device__ bool seg_aabb(v3 p, v3 delta, v3 high, v3 low, float& enter, float& exit_) {
    enter = 0.0f;
    exit_ = 1.0f;
    for (unsigned axis = 0; axis < 3; ++axis) {
        const float x = vcomp(p, axis), d = vcomp(delta, axis);
        const float mn = vcomp(low, axis), mx = vcomp(high, axis);
        if (fabsf(d) < 1.0e-6f) {
            if (x < mn || x > mx) return false;
            continue;
        }
        const float one = (mn - x) / d, two = (mx - x) / d;
        enter = smax(enter, smin(one, two));
        exit_ = smin(exit_, smax(one, two));
    }
    return enter <= exit_ && enter <= 1.0f;
}
struct Gen {
    const GBox* a; const GBox* b; Cand* out; int count; bool overflow;
    __device__ void emit(const Frame& f, v3 reference, v3 incident, v3 normal, float sep, bool flipped) {
        if (count >= kMaxBoxCandidates) { overflow = true; return; }
        const v3 w0 = fr_unproject(f, flipped ? incident : reference);
        const v3 w1 = fr_unproject(f, flipped ? reference : incident);
        Cand& c = out[count++];
        c.la = rotinv_gu(a->rot, vsub(w0, a->pos));
        c.lb = rotinv_gu(b->rot, vsub(w1, b->pos));
        c.nb = rotinv_gu(b->rot, normal);
        c.sep = sep;
    }
};
__device__ void gen_calculate(Gen& g, const Frame& f, const v3* poly, v3 inc_n, float fx, float fy,
                              v3 normal, float cd, bool flipped) {
    fx *= 1.0001f;
    fy *= 1.0001f;
    bool pen[4] = {false, false, false, false}, ins[4] = {false, false, false, false};
    v3 mn = {FLT_MAX, FLT_MAX, FLT_MAX};
    v3 mx = vneg(mn);
    const v3 high = {fx, fy, FLT_MAX};
    for (unsigned i = 0; i < 4; ++i) {
        const v3 p = poly[i];
        mn.x = smin(mn.x, p.x); mn.y = smin(mn.y, p.y);
        mx.x = smax(mx.x, p.x); mx.y = smax(mx.y, p.y);
        if (-p.z < cd) {
            pen[i] = true;
            ins[i] = fabsf(p.x) <= fx && fabsf(p.y) <= fy;
            if (ins[i]) g.emit(f, {p.x, p.y, 0}, p, normal, -p.z, flipped);
        }
    }
    if (g.count == 4) return;
    if (inc_n.z != 0.0f) {
        const v3 corners[4] = {{fx, fy, 0}, {fx, -fy, 0}, {-fx, fy, 0}, {-fx, -fy, 0}};
        for (int k = 0; k < 4; ++k) {
            const v3 c = corners[k];
            if (!poly_contains(poly, c, mn, mx)) continue;
            const float nom = vdot(inc_n, vsub(poly[0], c));
            const float t = nom / inc_n.z;
            const float sep = -t;
            if (cd > sep) g.emit(f, c, {c.x, c.y, t}, normal, sep, flipped);
        }
    }
    const v3 low = {-fx, -fy, -cd - FLT_EPSILON};
    for (unsigned start = 0, end = 3; start < 4; end = start++) {
        if (!pen[start] && !pen[end]) continue;
        const bool c0 = pen[start] && ins[start];
        const bool c1 = pen[end] && ins[end];
        if (c0 && c1) continue;
        const v3 edge = vsub(poly[end], poly[start]);
        float t0, t1;
        if (!seg_aabb(poly[start], edge, high, low, t0, t1)) continue;
        if (!c0) {
            const v3 p = vadd(poly[start], vmul(edge, t0));
            g.emit(f, {p.x, p.y, 0}, p, normal, -p.z, flipped);
        }
        if (!c1) {
            const v3 p = vadd(poly[start], vmul(edge, t1));
            g.emit(f, {p.x, p.y, 0}, p, normal, -p.z, flipped);
        }
    }
}
// Returns 0 separated, 1 overlapping (count candidates), -1 overflow.
__device__ int box_box_candidates(v3 h0, v3 p0, qt q0, v3 h1, v3 p1, qt q1, float cd,
                                  Cand* out, int& count) {
    const GBox a = make_box(h0, p0, q0), b = make_box(h1, p1, q1);
    Gen g{&a, &b, out, 0, false};
    const v3 delta = vsub(b.pos, a.pos);
    float sign[6], overlap[6];
    const float se = 1.0e-6f;
    count = 0;
    for (unsigned i = 0; i < 6; ++i) {
        const bool first = i < 3;
        const GBox& ref = first ? a : b;
        const GBox& inc = first ? b : a;
        const unsigned axis = i % 3;
        const v3 n = ref.axis[axis];
        sign[i] = vdot(delta, n);
        const float rad = (fabsf(vdot(n, inc.axis[0])) + se) * inc.half.x +
                          (fabsf(vdot(n, inc.axis[1])) + se) * inc.half.y +
                          (fabsf(vdot(n, inc.axis[2])) + se) * inc.half.z;
        overlap[i] = vcomp(ref.half, axis) + rad - fabsf(sign[i]) + cd;
        if (overlap[i] < 0.0f) return 0;
    }
    for (unsigned i = 0; i < 3; ++i)
        for (unsigned j = 0; j < 3; ++j) {
            const v3 ca = vcross(a.axis[i], b.axis[j]);
            float rA = 0.0f, rB = 0.0f;
            for (unsigned k = 0; k < 3; ++k) {
                if (k != i) rA += (fabsf(vdot(ca, a.axis[k])) + se) * vcomp(a.half, k);
                if (k != j) rB += (fabsf(vdot(ca, b.axis[k])) + se) * vcomp(b.half, k);
            }
            if (fabsf(vdot(delta, ca)) > rA + rB + cd) return 0;
        }
    unsigned feature = 0;
    float mo = overlap[0];
    for (unsigned i = 1; i < 6; ++i)
        if (mo > overlap[i]) { mo = overlap[i]; feature = i; }
    const bool flipped = feature >= 3;
    const GBox& inc = flipped ? a : b;
    const bool np = sign[feature] <= 0.0f;
    Frame fr;
    v3 normal;
    float fx, fy;
    switch (feature) {
    case 0:
        normal = np ? a.axis[0] : vneg(a.axis[0]);
        fr = {np ? vneg(a.axis[2]) : a.axis[2], a.axis[1], normal,
              vadd(a.pos, vmul(a.axis[0], np ? -a.half.x : a.half.x))};
        fx = a.half.z; fy = a.half.y; break;
    case 1:
        normal = np ? a.axis[1] : vneg(a.axis[1]);
        fr = {a.axis[0], np ? vneg(a.axis[2]) : a.axis[2], normal,
              vadd(a.pos, vmul(a.axis[1], np ? -a.half.y : a.half.y))};
        fx = a.half.x; fy = a.half.z; break;
    case 2:
        normal = np ? a.axis[2] : vneg(a.axis[2]);
        fr = {a.axis[0], np ? a.axis[1] : vneg(a.axis[1]), normal,
              vadd(a.pos, vmul(a.axis[2], np ? -a.half.z : a.half.z))};
        fx = a.half.x; fy = a.half.y; break;
    case 3:
        normal = np ? b.axis[0] : vneg(b.axis[0]);
        fr = {np ? b.axis[2] : vneg(b.axis[2]), b.axis[1], vneg(normal),
              vadd(b.pos, vmul(b.axis[0], np ? b.half.x : -b.half.x))};
        fx = b.half.z; fy = b.half.y; break;
    case 4:
        normal = np ? b.axis[1] : vneg(b.axis[1]);
        fr = {b.axis[0], np ? b.axis[2] : vneg(b.axis[2]), vneg(normal),
              vadd(b.pos, vmul(b.axis[1], np ? b.half.y : -b.half.y))};
        fx = b.half.x; fy = b.half.z; break;
    default:
        normal = np ? b.axis[2] : vneg(b.axis[2]);
        fr = {b.axis[0], np ? vneg(b.axis[1]) : b.axis[1], vneg(normal),
              vadd(b.pos, vmul(b.axis[2], np ? b.half.z : -b.half.z))};
        fx = b.half.x; fy = b.half.y; break;
    }
    const v3 search = vneg(fr.z);
    const float dx = fabsf(vdot(search, inc.axis[0]));
    const float dy = fabsf(vdot(search, inc.axis[1]));
    const float dz = fabsf(vdot(search, inc.axis[2]));
    const unsigned ia = dx >= dy && dx >= dz ? 0 : (dy >= dz ? 1 : 2);
    const float facing = vdot(search, inc.axis[ia]);
    const float sext = facing > 0.0f ? -vcomp(inc.half, ia) : vcomp(inc.half, ia);
    const v3 fc = vadd(inc.pos, vmul(inc.axis[ia], sext));
    const unsigned ua = ia == 0 ? 1 : 0;
    const unsigned va = ia == 2 ? 1 : 2;
    const v3 u = vmul(inc.axis[ua], vcomp(inc.half, ua));
    const v3 v = vmul(inc.axis[va], vcomp(inc.half, va));
    const v3 pw[4] = {vadd(fc, vadd(u, v)), vadd(fc, vsub(u, v)), vsub(fc, vadd(u, v)), vsub(fc, vsub(u, v))};
    v3 poly[4];
    for (int i = 0; i < 4; ++i) poly[i] = fr_project(fr, pw[i]);
    const v3 fn = fr_project(fr, vadd(fr.p, facing > 0.0f ? vneg(inc.axis[ia]) : inc.axis[ia]));
    gen_calculate(g, fr, poly, fn, fx, fy, normal, cd, flipped);
    if (g.overflow) return -1;
    count = g.count;
    return 1;
}

__device__ void batch_selection(const Cand* c, int n, float tol, int sel[4]) {
    uint8_t avail[64];
    for (int i = 0; i < n; ++i) avail[i] = uint8_t(i);
    int remaining = n;
    float deepest_depth = c[0].sep, shallowest = deepest_depth;
    int deepest = 0;
    for (int i = 1; i < remaining; ++i) {
        const float d = c[i].sep;
        shallowest = smax(shallowest, d);
        if (deepest_depth > d) { deepest_depth = d; deepest = i; }
    }
    sel[0] = deepest;
    avail[deepest] = avail[--remaining];
    int fpos = 0;
    float far2 = vlen2(vsub(c[avail[0]].lb, c[sel[0]].lb));
    for (int i = 1; i < remaining; ++i) {
        const float val = vlen2(vsub(c[avail[i]].lb, c[sel[0]].lb));
        if (val > far2) { far2 = val; fpos = i; }
    }
    sel[1] = avail[fpos];
    avail[fpos] = avail[--remaining];
    const v3 base = vsub(c[sel[1]].lb, c[sel[0]].lb);
    v3 tr = vcross(base, c[sel[0]].nb);
    const float tr2 = vlen2(tr);
    if (tr2 > 0.0f) {
        const float inv = 1.0f / sqrtf(tr2);
        tr = {tr.x * inv, tr.y * inv, tr.z * inv};
    } else {
        tr = c[sel[0]].nb;
    }
    float greatest = -FLT_MAX, least = FLT_MAX;
    int gpos = 0, lpos = 0;
    for (int i = 0; i < remaining; ++i) {
        const float side = vdot(vsub(c[avail[i]].lb, c[sel[0]].lb), tr);
        if (side > greatest) { greatest = side; gpos = i; }
        if (side < least) { least = side; lpos = i; }
    }
    sel[2] = avail[gpos];
    avail[gpos] = avail[--remaining];
    if (lpos == remaining) lpos = gpos;
    if (least * greatest > 0.0f) {
        greatest = -FLT_MAX;
        for (int i = 0; i < remaining; ++i) {
            const float side = vdot(vsub(c[avail[i]].lb, c[sel[0]].lb), tr);
            if (side > greatest) { greatest = side; lpos = i; }
        }
    }
    sel[3] = avail[lpos];
    avail[lpos] = avail[--remaining];
    const float thr = tol * 0.02f;
    if (deepest_depth < thr && shallowest > thr) {
        for (int i = 0; i < 4; ++i) {
            float depth = c[sel[i]].sep;
            if (depth > thr) {
                int rep = remaining;
                for (int j = 0; j < remaining; ++j) {
                    const float cand = c[avail[j]].sep;
                    if (depth > cand && thr > cand) { depth = cand; rep = j; }
                }
                if (rep < remaining) {
                    const uint8_t t = uint8_t(sel[i]);
                    sel[i] = avail[rep];
                    avail[rep] = t;
                }
            }
        }
    }
}

// ---------------- GJK / EPA ----------------
// The search is instantiated twice: G = false for box/box pairs, G = true
// for pairs with a cooked hull, where a hull's support is its first vertex
// of largest projection, a sphere is a point core (its radius applied after
// the search), and facet admission and the witness tolerance scale with the
// shapes (GuPCMGjkEpa.cpp:53-75, 201-218, 296-302, 411-516).
struct Sup { v3 a, b, q; uint32_t ai, bi; };
struct BPair {
    v3 ha, hb, a_in_b; qt rel;
    const float4* va; uint32_t nva;    // hull vertices of A / B (G only)
    const float4* vb; uint32_t nvb;
    float ra, rb;                      // sphere point-core radii (G only)
};
__device__ __forceinline__ v3 box_vertex(v3 e, v3 d, uint32_t& idx) {
    const bool x = d.x > 0.f, y = d.y > 0.f, z = d.z > 0.f;
    idx = (x ? 1u : 0u) | (y ? 2u : 0u) | (z ? 4u : 0u);
    return {x ? e.x : -e.x, y ? e.y : -e.y, z ? e.z : -e.z};
}
// A hull's support: its first vertex of largest projection.  The warp
// splits the scan (lane l takes vertices l, l + 32, ...) and reduces to the
// largest projection, lowest index on ties, which is the vertex the
// sequential first-maximum scan returns; lane 0's result is broadcast so
// every lane holds the same vertex whatever the inputs.  Every lane of the
// warp must call it together.
__device__ __forceinline__ v3 shape_vertex(v3 e, v3 d, const float4* hull, uint32_t n, float radius,
                                           uint32_t& idx) {
    idx = 0;
    if (radius > 0.f) return {0.f, 0.f, 0.f};
    if (n) {
        const uint32_t lane = threadIdx.x & 31u;
        float best = 0.f;
        uint32_t bi = 0xffffffffu;
        for (uint32_t i = lane; i < n; i += 32) {
            const float pr = vdot(ld3(hull[i]), d);
            if (bi == 0xffffffffu || pr > best) { best = pr; bi = i; }
        }
        for (int off = 16; off > 0; off >>= 1) {
            const float ob = __shfl_xor_sync(0xffffffffu, best, off);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, off);
            if (oi != 0xffffffffu && (bi == 0xffffffffu || ob > best || (ob == best && oi < bi))) { best = ob; bi = oi; }
        }
        idx = __shfl_sync(0xffffffffu, bi, 0);
        return ld3(hull[idx]);
    }
    return box_vertex(e, d, idx);
}
template <bool G> __device__ Sup bp_support(const BPair& p, v3 dir) {
    Sup s;
    const v3 da = rotinv_gu(p.rel, dir);
    v3 pa;
    if (G) {
        pa = shape_vertex(p.ha, da, p.va, p.nva, p.ra, s.ai);
        s.b = shape_vertex(p.hb, vneg(dir), p.vb, p.nvb, p.rb, s.bi);
    } else {
        pa = box_vertex(p.ha, da, s.ai);
        s.b = box_vertex(p.hb, vneg(dir), s.bi);
    }
    s.a = vadd(p.a_in_b, rot_gu(p.rel, pa));
    s.q = vsub(s.a, s.b);
    return s;
}
__device__ __forceinline__ v3 bp_local_a(const BPair& p, v3 pb) { return rotinv_gu(p.rel, vsub(pb, p.a_in_b)); }
__device__ __forceinline__ float box_min_margin(v3 h) { return 0.05f * smin(smin(h.x, h.y), h.z); }
__device__ bool solve_small(int n, float a[3][4], float r[3]) {
    float scale = 0.0f;
    for (int i = 0; i < n; ++i) scale = smax(scale, fabsf(a[i][i]));
    if (!(scale > 0.0f) || !isfinite(scale)) return false;
    const float tol = FLT_EPSILON * scale;
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int row = col + 1; row < n; ++row)
            if (fabsf(a[row][col]) > fabsf(a[piv][col])) piv = row;
        if (!(fabsf(a[piv][col]) > tol)) return false;
        for (int j = col; j <= n; ++j) { const float t = a[col][j]; a[col][j] = a[piv][j]; a[piv][j] = t; }
        const float div = a[col][col];
        for (int j = col; j <= n; ++j) a[col][j] /= div;
        for (int row = 0; row < n; ++row)
            if (row != col) {
                const float f = a[row][col];
                for (int j = col; j <= n; ++j) a[row][j] = fmaf(-f, a[col][j], a[row][j]);
            }
    }
    for (int i = 0; i < n; ++i) r[i] = a[i][n];
    return true;
}
struct Closest { v3 point, a, b; float w[4]; unsigned mask; float dist2; };
// Closest point of the simplex to the origin (GuPCMGjkEpa.cpp's sub-simplex
// search): every non-empty vertex subset is solved as an affine system and
// the nearest feasible one wins.  One lane takes one subset (mask = lane + 1,
// at most 15); the warp then keeps the smallest distance, and among equal
// distances the lowest mask, which is the subset the sequential search in
// mask order keeps (it replaces the best only on a strictly smaller
// distance).  Each lane's arithmetic is that of one iteration of the
// sequential search, so the winner is bit for bit the same.  Every lane of
// the warp calls this with the same simplex and gets the same result.
__device__ Closest closest_simplex_warp(const Sup* s, int count) {
    const uint32_t lane = threadIdx.x & 31u;
    const unsigned mask = lane + 1u;
    Closest mine;
    mine.point = mine.a = mine.b = {0, 0, 0};
    mine.w[0] = mine.w[1] = mine.w[2] = mine.w[3] = 0.0f;
    bool ok = mask < (1u << count);
    if (ok) {
        int ids[4] = {0, 0, 0, 0}, n = 0;
        for (int i = 0; i < count; ++i)
            if (mask & (1u << i)) ids[n++] = i;
        float w[4] = {0, 0, 0, 0};
        w[ids[0]] = 1.0f;
        if (n > 1) {
            const v3 base = s[ids[0]].q;
            v3 dirs[3];
            float m[3][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
            for (int i = 1; i < n; ++i) dirs[i - 1] = vsub(s[ids[i]].q, base);
            for (int i = 1; i < n; ++i) {
                for (int j = 1; j < n; ++j) m[i - 1][j - 1] = vdot(dirs[i - 1], dirs[j - 1]);
                m[i - 1][n - 1] = -vdot(dirs[i - 1], base);
            }
            float coef[3] = {0, 0, 0};
            if (!solve_small(n - 1, m, coef)) ok = false;
            for (int i = 1; i < n; ++i) {
                w[ids[i]] = coef[i - 1];
                w[ids[0]] -= coef[i - 1];
            }
        }
        for (int i = 0; i < n; ++i)
            if (w[ids[i]] < -1.0e-5f) ok = false;
        if (ok) {
            v3 q = {0, 0, 0}, pa = {0, 0, 0}, pb = {0, 0, 0};
            for (int i = 0; i < count; ++i) {
                q = vadd(q, vmul(s[i].q, w[i]));
                pa = vadd(pa, vmul(s[i].a, w[i]));
                pb = vadd(pb, vmul(s[i].b, w[i]));
            }
            mine.point = q; mine.a = pa; mine.b = pb;
            for (int i = 0; i < 4; ++i) mine.w[i] = w[i];
            mine.dist2 = vlen2(q);
            ok = mine.dist2 < FLT_MAX;
        }
    }
    float d = ok ? mine.dist2 : FLT_MAX;
    unsigned m = ok ? mask : 0xffffffffu;
    for (int off = 16; off > 0; off >>= 1) {
        const float od = __shfl_xor_sync(0xffffffffu, d, off);
        const unsigned om = __shfl_xor_sync(0xffffffffu, m, off);
        if (od < d || (od == d && om < m)) { d = od; m = om; }
    }
    Closest best;
    if (m == 0xffffffffu) {
        best.point = best.a = best.b = {0, 0, 0};
        best.w[0] = best.w[1] = best.w[2] = best.w[3] = 0.0f;
        best.mask = 0;
        best.dist2 = FLT_MAX;
        return best;
    }
    const int src = int(m - 1u);
    const auto bc = [src](float x) { return __shfl_sync(0xffffffffu, x, src); };
    best.point = {bc(mine.point.x), bc(mine.point.y), bc(mine.point.z)};
    best.a = {bc(mine.a.x), bc(mine.a.y), bc(mine.a.z)};
    best.b = {bc(mine.b.x), bc(mine.b.y), bc(mine.b.z)};
    for (int i = 0; i < 4; ++i) best.w[i] = bc(mine.w[i]);
    best.mask = m;
    best.dist2 = d;
    return best;
}
__device__ void compact_simplex(Sup* s, int& count, const Closest& c) {
    int write = 0;
    for (int read = 0; read < count; ++read)
        if ((c.mask & (1u << read)) && c.w[read] > 1.0e-6f) s[write++] = s[read];
    if (write == 0 && count > 0) write = 1;
    count = write;
}
__device__ bool contact_from_gjk(const BPair& p, const Closest& n, Cand& out) {
    const float dist = sqrtf(n.dist2);
    if (!(dist > 0.0f) || !isfinite(dist)) return false;
    const v3 normal = vmul(n.point, 1.0f / dist);
    out = {bp_local_a(p, n.a), n.b, normal, dist};
    return true;
}
struct Facet { int i, j, k; v3 normal; float distance; bool valid, in_heap; };
template <bool G> __device__ Facet make_facet(const Sup* vtx, int i, int j, int k) {
    Facet f;
    f.i = f.j = f.k = 0; f.normal = {0, 0, 0}; f.distance = 0.0f; f.valid = false; f.in_heap = true;
    const v3 a = vtx[i].q, b = vtx[j].q, c = vtx[k].q;
    const v3 e0 = vsub(b, a), e1 = vsub(c, a);
    v3 n = vcross(e0, e1);
    const float norm2 = vlen2(n);
    float min_area = FLT_EPSILON;
    if (G) min_area *= vlen2(e0) * vlen2(e1);
    if (!(norm2 > min_area)) return f;
    n = vmul(n, 1.0f / sqrtf(norm2));
    f.i = i; f.j = j; f.k = k; f.normal = n; f.distance = vdot(n, a); f.valid = true;
    return f;
}
template <bool G> __device__ bool init_epa(const BPair& p, Sup* vtx, int& count, Facet* facets, int& fc) {
    if (count <= 0 || count > 4) return false;
    if (count == 1) {
        const Sup nx = bp_support<G>(p, {1, 0, 0});
        if (vlen2(vsub(nx.q, vtx[0].q)) == 0.0f) return false;
        vtx[count++] = nx;
    }
    if (count == 2) {
        const v3 edge = vsub(vtx[1].q, vtx[0].q);
        const v3 ab = {fabsf(edge.x), fabsf(edge.y), fabsf(edge.z)};
        v3 axis = {1, 0, 0};
        if (ab.x > ab.y && ab.z > ab.y) axis = {0, 1, 0};
        else if (ab.x > ab.z) axis = {0, 0, 1};
        v3 perp = vcross(axis, edge);
        const float sq = vlen2(perp);
        if (!(sq > 0.0f)) return false;
        perp = vmul(perp, 1.0f / sqrtf(sq));
        vtx[count++] = bp_support<G>(p, perp);
    }
    if (count == 3) {
        const Facet f0 = make_facet<G>(vtx, 0, 1, 2), f1 = make_facet<G>(vtx, 1, 0, 2);
        if (!f0.valid || !f1.valid) return false;
        facets[fc++] = f0;
        facets[fc++] = f1;
        return true;
    }
    const v3 p0 = vtx[0].q;
    const v3 v1 = vsub(vtx[1].q, p0), v2 = vsub(vtx[2].q, p0);
    if (vdot(vcross(v1, v2), vsub(vtx[3].q, p0)) > 0.0f) {
        const Sup t = vtx[1]; vtx[1] = vtx[2]; vtx[2] = t;
    }
    const int faces[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    for (int i = 0; i < 4; ++i) {
        const Facet f = make_facet<G>(vtx, faces[i][0], faces[i][1], faces[i][2]);
        if (!f.valid) return false;
        facets[fc++] = f;
    }
    return true;
}
template <bool G> __device__ bool contact_from_facet(const BPair& p, const Sup* vtx, const Facet& f, Cand& out) {
    const Sup& P = vtx[f.i];
    const Sup& Qv = vtx[f.j];
    const Sup& R = vtx[f.k];
    const v3 e0 = vsub(Qv.q, P.q), e1 = vsub(R.q, P.q);
    const float a = vdot(e0, e0), b = vdot(e0, e1), c = vdot(e1, e1);
    const float den = a * c - b * b;
    if (!(den > FLT_EPSILON * a * c)) return false;
    const float x = -vdot(P.q, e0), y = -vdot(P.q, e1);
    const float u = (x * c - y * b) / den;
    const float v = (y * a - x * b) / den;
    const float w = 1.0f - u - v;
    const v3 pa = vadd(vadd(vmul(P.a, w), vmul(Qv.a, u)), vmul(R.a, v));
    const v3 pb = vadd(vadd(vmul(P.b, w), vmul(Qv.b, u)), vmul(R.b, v));
    if (!isfinite(pa.x) || !isfinite(pb.x) || !isfinite(f.distance)) return false;
    const float depth = fabsf(f.distance);
    out = {bp_local_a(p, pa), pb, vneg(f.normal), -depth};
    float tol = 1.0e-3f;
    if (G) tol *= smax(smax(smax(p.ha.x, p.ha.y), smax(p.ha.z, p.hb.x)), smax(p.hb.y, p.hb.z));
    return sqrtf(vlen2(vsub(pa, pb))) <= depth + tol;
}
// GJK (GuPCMGjkEpa.cpp) up to the point where EPA starts: returns 0 (no
// witness), 1 (witness in out) or 2 (EPA needed from simplex[0, sc)).  The
// whole warp runs it in step on the same pair (every lane holds the same
// simplex; the sub-simplex search is spread over the lanes), so every lane
// returns the same mode, witness and simplex.
// A sphere point core (G only) converges its separated distance before EPA
// is admitted and falls back to EPA where the polyhedral search gives up.
template <bool G> __device__ int gjk_phase(const BPair& p, float cd, Cand& out, Sup* simplex, int& count) {
    const float eps = 0.1f * smin(box_min_margin(p.ha), box_min_margin(p.hb));
    const float progress = 1.0f - 0.000225f;
    const bool pc = G && (p.ra > 0.f || p.rb > 0.f);
    count = 0;
    v3 closest = vlen2(p.a_in_b) > 0.0f ? p.a_in_b : v3{1, 0, 0};
    float previous = FLT_MAX;
    for (int it = 0; it < 32; ++it) {
        const float dist = sqrtf(vlen2(closest));
        if (count > 0 && dist <= eps && !pc) return 2;
        if (dist <= 0.0f) return pc && count > 0 ? 2 : 0;
        const v3 normal = vmul(closest, 1.0f / dist);
        const Sup s = bp_support<G>(p, vneg(closest));
        const float proj = vdot(normal, s.q);
        if (proj > cd) return 0;
        if (count > 0 && proj > dist * progress) {
            const Closest cur = closest_simplex_warp(simplex, count);
            return cur.mask && contact_from_gjk(p, cur, out) ? 1 : 0;
        }
        for (int i = 0; i < count; ++i)
            if (s.ai == simplex[i].ai && s.bi == simplex[i].bi) {
                if (proj > 0.f) {
                    const Closest cur = closest_simplex_warp(simplex, count);
                    return cur.mask && contact_from_gjk(p, cur, out) && out.sep <= cd ? 1 : 0;
                }
                return pc ? 2 : 0;
            }
        if (count == 4) return 2;
        simplex[count++] = s;
        const Closest nx = closest_simplex_warp(simplex, count);
        if (!nx.mask) return 0;
        closest = nx.point;
        const float nd = sqrtf(nx.dist2);
        compact_simplex(simplex, count, nx);
        if (nd >= previous) {
            if (pc) return proj > 0.f ? (contact_from_gjk(p, nx, out) ? 1 : 0) : 2;
            return 0;
        }
        previous = nd;
    }
    return pc && count > 0 ? 2 : 0;
}

// EPA (GuPCMGjkEpa.cpp) with one warp: the polytope lives in shared memory; the closest
// facet search, the duplicate-vertex test, the visibility marking, the free
// slot count and the new facets are spread over the lanes; the horizon walk
// (whose order decides where new facets land) visits the visible facets in
// index order, as the sequential search does, with the edge list held one
// edge per lane.  Every lane returns the same result; out is valid on every
// lane.
struct EpaShared {
    Sup vtx[64];
    Facet facets[64];
    int bc;
    int status;
};
template <bool G> __device__ bool run_epa_warp(const BPair& p, const Sup* simplex, int sc, Cand& out, EpaShared& E) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t full = 0xffffffffu;
    if (G) {
        // every lane builds the initial polytope (its supports are warp
        // scans); lane 0 publishes it
        Sup v0[4];
        Facet f0[4];
        int vc0 = sc, fc0 = 0;
        for (int i = 0; i < sc; ++i) v0[i] = simplex[i];
        const bool ok = init_epa<G>(p, v0, vc0, f0, fc0);
        if (lane == 0) {
            for (int i = 0; i < vc0; ++i) E.vtx[i] = v0[i];
            for (int i = 0; i < fc0; ++i) E.facets[i] = f0[i];
            E.status = ok ? fc0 : -1;
            E.bc = vc0;
        }
    } else if (lane == 0) {
        int vc0 = sc;
        for (int i = 0; i < sc; ++i) E.vtx[i] = simplex[i];
        int fc0 = 0;
        E.status = init_epa<G>(p, E.vtx, vc0, E.facets, fc0) ? fc0 : -1;
        E.bc = vc0;
    }
    __syncwarp();
    if (E.status < 0) return false;
    int fc = E.status, vc = E.bc;
    __syncwarp();
    const float eps = 0.1f * smin(box_min_margin(p.ha), box_min_margin(p.hb));
    float upper = FLT_MAX;
    for (int it = 0; it < 60; ++it) {
        // closest facet: smallest distance, lowest index on ties
        float dist = FLT_MAX;
        int closest = -1;
        for (int i = int(lane); i < fc; i += 32) {
            const Facet& f = E.facets[i];
            if (f.valid && f.in_heap && f.distance < dist) { dist = f.distance; closest = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const float od = __shfl_xor_sync(full, dist, o);
            const int oc = __shfl_xor_sync(full, closest, o);
            if (oc >= 0 && (closest < 0 || od < dist || (od == dist && oc < closest))) { dist = od; closest = oc; }
        }
        if (closest < 0) return false;
        const Facet sel = E.facets[closest];
        const Sup np = bp_support<G>(p, sel.normal);
        const float proj = vdot(np.q, sel.normal);
        if (fabsf(proj - dist) <= eps) return contact_from_facet<G>(p, E.vtx, sel, out);
        if (vc == 64) return false;
        upper = smin(upper, proj);
        bool dup = false;
        for (int i = int(lane); i < vc; i += 32) dup |= E.vtx[i].ai == np.ai && E.vtx[i].bi == np.bi;
        if (__any_sync(full, dup)) return contact_from_facet<G>(p, E.vtx, sel, out);
        const int ni = vc++;
        // visibility (independent per facet)
        bool vis0 = false, vis1 = false;
        for (int r = 0; r < 2; ++r) {
            const int i = int(lane) + 32 * r;
            bool vis = false;
            if (i < fc) {
                const Facet& f = E.facets[i];
                vis = f.valid && !(vdot(f.normal, vsub(np.q, E.vtx[f.i].q)) < 0.0f);
            }
            (r ? vis1 : vis0) = vis;
        }
        const uint32_t vmask0 = __ballot_sync(full, vis0), vmask1 = __ballot_sync(full, vis1);
        if (lane == 0) E.vtx[ni] = np;
        // Horizon edges in the order the sequential search finds them: the
        // visible facets in index order, each edge appended or, when its
        // reverse is listed, removed by moving the last edge into its slot.
        // The list lives in registers, lane t holding edge t, so each test
        // is one ballot.
        int ef0 = -1, et0 = -1;     // this lane's boundary edge
        int bc = 0;
        bool fail = false;
        for (int r = 0; r < 2 && !fail; ++r) {
            uint32_t m = r ? vmask1 : vmask0;
            while (m && !fail) {
                const int i = __ffs(m) - 1 + 32 * r;
                m &= m - 1;
                const Facet& f = E.facets[i];
                const int ef[3] = {f.i, f.j, f.k}, et[3] = {f.j, f.k, f.i};
                for (int e = 0; e < 3; ++e) {
                    const uint32_t hit = __ballot_sync(full, int(lane) < bc && ef0 == et[e] && et0 == ef[e]);
                    if (hit) {
                        const int rev = __ffs(hit) - 1;
                        --bc;
                        const int lf = __shfl_sync(full, ef0, bc), lt = __shfl_sync(full, et0, bc);
                        if (int(lane) == rev) { ef0 = lf; et0 = lt; }
                    } else {
                        if (bc == 32) { fail = true; break; }
                        if (int(lane) == bc) { ef0 = ef[e]; et0 = et[e]; }
                        ++bc;
                    }
                }
            }
        }
        if (fail || bc <= 0) return false;
        __syncwarp();
        // the visible facets leave the polytope
        if (vis0) E.facets[lane].valid = false;
        if (vis1) E.facets[lane + 32].valid = false;
        __syncwarp();
        // free slots among [0, fc): invalid facets, in index order
        bool inv0 = int(lane) < fc && !E.facets[lane].valid;
        bool inv1 = int(lane) + 32 < fc && !E.facets[lane + 32].valid;
        const uint32_t fmask0 = __ballot_sync(full, inv0), fmask1 = __ballot_sync(full, inv1);
        const int nfree = __popc(fmask0) + __popc(fmask1);
        if (bc > 64 - fc + nfree) return false;
        // new facet for horizon edge `lane`, placed in the lane-th free slot
        Facet nf;
        bool ok = true;
        int slot = -1;
        if (int(lane) < bc) {
            nf = make_facet<G>(E.vtx, ef0, et0, ni);
            ok = nf.valid;
            nf.in_heap = nf.distance <= upper;
            const int k = int(lane);
            if (k < __popc(fmask0)) {
                uint32_t m = fmask0;
                for (int t = 0; t < k; ++t) m &= m - 1;
                slot = __ffs(m) - 1;
            } else if (k < nfree) {
                uint32_t m = fmask1;
                for (int t = __popc(fmask0); t < k; ++t) m &= m - 1;
                slot = 32 + __ffs(m) - 1;
            } else {
                slot = fc + (k - nfree);
            }
        }
        if (!__all_sync(full, ok)) return false;
        __syncwarp();
        if (int(lane) < bc) E.facets[slot] = nf;
        fc = bc > nfree ? fc + (bc - nfree) : fc;
        __syncwarp();
    }
    return false;
}


// ---------------- persistent manifolds ----------------
__device__ __forceinline__ v3 lv(const float* f) { return {f[0], f[1], f[2]}; }
__device__ __forceinline__ void sv(float* f, v3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }
__device__ __forceinline__ PcmPoint to_pt(const Cand& c) {
    PcmPoint p;
    sv(p.la, c.la); sv(p.lb, c.lb); sv(p.nb, c.nb); p.sep = c.sep;
    return p;
}
__device__ __forceinline__ uint32_t cache_count(const PcmCache& c) { return c.meta & 255u; }
__device__ __forceinline__ bool cache_init(const PcmCache& c) { return (c.meta >> 8) & 1u; }
__device__ __forceinline__ void set_meta(PcmCache& c, uint32_t count, bool init) {
    c.meta = count | (init ? 256u : 0u);
}

__device__ void refresh_points(PcmCache& c, v3 pa_in_b, qt ra_in_b, float brk) {
    const float brk2 = brk * brk;
    uint32_t count = cache_count(c);
    for (uint32_t i = count; i > 0; --i) {
        PcmPoint& pt = c.pts[i - 1];
        const v3 rr = rot_sc(ra_in_b, lv(pt.la));
        const v3 lab = {pa_in_b.x + rr.x, pa_in_b.y + rr.y, pa_in_b.z + rr.z};
        const v3 nb = lv(pt.nb), lb = lv(pt.lb);
        const v3 v = {lab.x - lb.x, lab.y - lb.y, lab.z - lb.z};
        const float dist = v.x * nb.x + v.y * nb.y + v.z * nb.z;
        const v3 pd = {v.x - nb.x * dist, v.y - nb.y * dist, v.z - nb.z * dist};
        const float t2 = pd.x * pd.x + pd.y * pd.y + pd.z * pd.z;
        if (t2 > brk2) c.pts[i - 1] = c.pts[--count];
        else pt.sep = dist;
    }
    c.meta = (c.meta & ~255u) | count;
}
__device__ float seg_sq(v3 p, v3 a, v3 b) {
    const v3 ab = vsub(b, a), ap = vsub(p, a);
    const float den = vlen2(ab);
    const float t = den == 0.0f ? 0.0f : sclamp(vdot(ap, ab) / den, 0.0f, 1.0f);
    const v3 d = {ap.x - t * ab.x, ap.y - t * ab.y, ap.z - t * ab.z};
    return vlen2(d);
}
__device__ float tri_sq(v3 p, v3 a, v3 b, v3 c) {
    const v3 ab = vsub(b, a), ac = vsub(c, a);
    const v3 ap = vsub(p, a), bp = vsub(p, b), cp = vsub(p, c);
    const float d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    const float d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    const float d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d1 < 0.0f && d2 < 0.0f) return vlen2(ap);
    if (d3 >= 0.0f && d3 >= d4) return vlen2(bp);
    if (d6 >= 0.0f && d6 >= d5) return vlen2(cp);
    const float vc = d1 * d4 - d3 * d2;
    if (vc < 0.0f && d1 >= 0.0f && d3 < 0.0f) return seg_sq(p, a, b);
    const float va = d3 * d6 - d5 * d4;
    if (va < 0.0f && d4 >= d3 && d5 >= d6) return seg_sq(p, b, c);
    const float vb = d5 * d2 - d1 * d6;
    if (vb < 0.0f && d2 >= 0.0f && d6 < 0.0f) return seg_sq(p, a, c);
    const v3 n = {ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x};
    const float den = vlen2(n);
    if (den == 0.0f) return 0.0f;
    const float pr = vdot(n, ap);
    return pr * pr / den;
}
__device__ void reduce_five(PcmCache& c, const PcmPoint& nw) {
    PcmPoint cand[5];
    bool chosen[5] = {false, false, false, false, false};
    int sel[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) cand[i] = c.pts[i];
    cand[4] = nw;
    int deepest = 4;
    for (int i = 0; i < 4; ++i)
        if (cand[i].sep < cand[deepest].sep) deepest = i;
    sel[0] = deepest;
    chosen[deepest] = true;
    int farthest = 0;
    float largest = vlen2(vsub(lv(cand[0].lb), lv(cand[deepest].lb)));
    for (int i = 1; i < 5; ++i)
        if (!chosen[i]) {
            const float v = vlen2(vsub(lv(cand[i].lb), lv(cand[deepest].lb)));
            if (v > largest) { largest = v; farthest = i; }
        }
    sel[1] = farthest;
    chosen[farthest] = true;
    largest = -FLT_MAX;
    int third = 0;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) {
            const float v = seg_sq(lv(cand[i].lb), lv(cand[deepest].lb), lv(cand[farthest].lb));
            if (v > largest) { largest = v; third = i; }
        }
    sel[2] = third;
    chosen[third] = true;
    largest = -FLT_MAX;
    int fourth = third;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) {
            const float v = tri_sq(lv(cand[i].lb), lv(cand[sel[0]].lb), lv(cand[sel[1]].lb), lv(cand[sel[2]].lb));
            if (v > largest) { largest = v; fourth = i; }
        }
    if (chosen[fourth]) {
        for (int i = 0; i < 3; ++i) c.pts[i] = cand[sel[i]];
        c.meta = (c.meta & ~255u) | 3u;
        return;
    }
    sel[3] = fourth;
    chosen[fourth] = true;
    for (int i = 0; i < 4; ++i) c.pts[i] = cand[sel[i]];
    c.meta = (c.meta & ~255u) | 4u;
    int un = -1;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) { un = i; break; }
    if (un < 0) return;
    float closest = FLT_MAX;
    int rep = 0;
    for (int i = 0; i < 4; ++i) {
        const float d = vlen2(vsub(lv(c.pts[i].la), lv(cand[un].la)));
        if (d < closest) { closest = d; rep = i; }
    }
    if (cand[un].sep < c.pts[rep].sep) c.pts[rep] = cand[un];
}
__device__ __forceinline__ float pcm_box_margin(v3 h) { return smin(0.15f * smin(smin(h.x, h.y), h.z), 0.15f); }

__device__ int emit_box_box(qt q1, v3 p1, float cd, const PcmCache& cache, bool direct, bool gjk, v3 gjk_n,
                            ContactPt* out);

// Returns the emitted count, or -1 on an invalid manifold normal / overflow.
// Sets gjk_pending (and emits nothing) when the zero-face GJK/EPA
// continuation must complete the manifold.
__device__ int generate_box_box(v3 h0, v3 p0, qt q0, v3 h1, v3 p1, qt q1, float cd, PcmCache& cache,
                                ContactPt* out, bool& gjk_pending) {
    const v3 delta = {p0.x - p1.x, p0.y - p1.y, p0.z - p1.z};
    const v3 relative = rotinv_sc(q1, delta);
    const qt rotation = qmul(qconj(q1), q0);
    const float mm = smin(pcm_box_margin(h0), pcm_box_margin(h1));
    const uint32_t initial = cache_count(cache);
    refresh_points(cache, relative, rotation, mm * 0.8f);
    const bool lost = cache_count(cache) != initial;
    const float thr[5] = {0.5f, 0.125f, 0.25f, 0.375f, 0.375f};
    const float qthr[5] = {0.9998f, 0.9999f, 0.9999f, 0.9999f, 0.9999f};
    const bool init = cache_init(cache);
    float tdelta = INFINITY;
    if (init)
        tdelta = smax(smax(fabsf(relative.x - cache.rel_p[0]), fabsf(relative.y - cache.rel_p[1])),
                      fabsf(relative.z - cache.rel_p[2]));
    const float qa = qdot(q0, {cache.qa[0], cache.qa[1], cache.qa[2], cache.qa[3]});
    const float qb = qdot(q1, {cache.qb[0], cache.qb[1], cache.qb[2], cache.qb[3]});
    const uint32_t cc = cache_count(cache);
    const float tp = mm * thr[cc];
    bool regen = !init || lost || tdelta > tp || qa < qthr[cc] || qb < qthr[cc];
    if (!regen) {
        const float a0 = qa < 1.0f ? acosf(smax(-1.0f, qa)) : 0.0f;
        const float a1 = qb < 1.0f ? acosf(smax(-1.0f, qb)) : 0.0f;
        regen = a0 * sqrtf(h0.x * h0.x + h0.y * h0.y + h0.z * h0.z) > tp ||
                a1 * sqrtf(h1.x * h1.x + h1.y * h1.y + h1.z * h1.z) > tp;
    }
    bool direct = false;
    const bool gjk = false;
    const v3 gjk_n = {0, 0, 0};
    if (regen) {
        sv(cache.rel_p, relative);
        cache.rel_q[0] = rotation.x; cache.rel_q[1] = rotation.y; cache.rel_q[2] = rotation.z; cache.rel_q[3] = rotation.w;
        cache.qa[0] = q0.x; cache.qa[1] = q0.y; cache.qa[2] = q0.z; cache.qa[3] = q0.w;
        cache.qb[0] = q1.x; cache.qb[1] = q1.y; cache.qb[2] = q1.z; cache.qb[3] = q1.w;
        set_meta(cache, cache_count(cache), true);
        Cand cands[kMaxBoxCandidates];
        int count = 0;
        const int ov = box_box_candidates(h0, p0, q0, h1, p1, q1, cd, cands, count);
        if (ov < 0) return -1;
        if (ov == 0) {
            set_meta(cache, 0, true);
            return 0;
        }
        if (count == 0) {
            // Zero face contacts: the GJK/EPA continuation runs in its own
            // kernel (k_narrowphase_gjk) over the pairs that need it, so its
            // polytope working set stays out of this kernel.
            gjk_pending = true;
            return 0;
        } else if (count <= 4) {
            for (int i = 0; i < count; ++i) cache.pts[i] = to_pt(cands[i]);
            set_meta(cache, uint32_t(count), true);
        } else {
            int sel[4];
            batch_selection(cands, count, 1.0f, sel);
            for (int i = 0; i < 4; ++i) cache.pts[i] = to_pt(cands[sel[i]]);
            set_meta(cache, 4, true);
        }
        direct = count > 0;
    }
    return emit_box_box(q1, p1, cd, cache, direct, gjk, gjk_n, out);
}

// Second half of the zero-face case (scene.cpp:3545-3590): GJK/EPA witness,
// replacement or append into the refreshed cache, then emission.
__device__ int finish_box_box_gjk(v3 h0, v3 h1, v3 p1, qt q1, float cd, PcmCache& cache, bool have,
                                  const Cand& w, ContactPt* out) {
    const float mm = smin(pcm_box_margin(h0), pcm_box_margin(h1));
    if (!have) {
        set_meta(cache, 0, true);
        return 0;
    }
    const float rb = mm * 0.05f;
    const float rsq = rb * rb;
    bool replaced = false;
    const uint32_t n0 = cache_count(cache);
    for (uint32_t i = 0; i < n0; ++i) {
        const PcmPoint& o = cache.pts[i];
        if (smin(vlen2(vsub(lv(o.la), w.la)), vlen2(vsub(lv(o.lb), w.lb))) < rsq) {
            cache.pts[i] = to_pt(w);
            replaced = true;
            break;
        }
    }
    if (!replaced) {
        if (n0 < 4) {
            cache.pts[n0] = to_pt(w);
            set_meta(cache, n0 + 1, true);
        } else {
            reduce_five(cache, to_pt(w));
        }
    }
    return emit_box_box(q1, p1, cd, cache, false, true, w.nb, out);
}

__device__ int emit_box_box(qt q1, v3 p1, float cd, const PcmCache& cache, bool direct, bool gjk, v3 gjk_n,
                            ContactPt* out) {
    const uint32_t n = cache_count(cache);
    if (n == 0) return 0;
    v3 nb = {0, 0, 0};
    if (gjk) nb = gjk_n;
    else if (direct) nb = lv(cache.pts[0].nb);
    else
        for (uint32_t i = 0; i < n; ++i) {
            nb.x += cache.pts[i].nb[0];
            nb.y += cache.pts[i].nb[1];
            nb.z += cache.pts[i].nb[2];
        }
    const float nsq = nb.x * nb.x + nb.y * nb.y + nb.z * nb.z;
    if (!(nsq > 0.0f) || !isfinite(nsq)) return -1;
    const float il = 1.0f / sqrtf(nsq);
    const v3 normal = rot_sc(q1, {nb.x * il, nb.y * il, nb.z * il});
    int emitted = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const PcmPoint& p = cache.pts[i];
        if (!direct && p.sep > cd) continue;
        const v3 r = rot_sc(q1, lv(p.lb));
        ContactPt& o = out[emitted++];
        o.p[0] = r.x + p1.x; o.p[1] = r.y + p1.y; o.p[2] = r.z + p1.z;
        o.n[0] = normal.x; o.n[1] = normal.y; o.n[2] = normal.z;
        o.sep = p.sep;
    }
    return emitted;
}

__device__ int generate_plane_box(v3 pp, v3 h, v3 bp, qt q, float cd, PcmCache& cache, ContactPt* out) {
    const v3 rel = {bp.x - pp.x, bp.y - pp.y, bp.z - pp.z};
    const float margin = pcm_box_margin(h);
    const float brk = margin * 0.2f;
    const uint32_t prev = cache_count(cache);
    refresh_points(cache, rel, q, brk);
    const bool init = cache_init(cache);
    float md = INFINITY;
    if (init)
        md = smax(smax(fabsf(rel.x - cache.rel_p[0]), fabsf(rel.y - cache.rel_p[1])), fabsf(rel.z - cache.rel_p[2]));
    const float rd = q.x * cache.rel_q[0] + q.y * cache.rel_q[1] + q.z * cache.rel_q[2] + q.w * cache.rel_q[3];
    const bool regen = !init || cache_count(cache) != prev || md > brk || rd < 0.99996f;
    if (regen) {
        sv(cache.rel_p, rel);
        cache.rel_q[0] = q.x; cache.rel_q[1] = q.y; cache.rel_q[2] = q.z; cache.rel_q[3] = q.w;
        Cand cands[8];
        int n = 0;
        for (unsigned corner = 0; corner < 8u; ++corner) {
            const v3 local = {(corner & 4u) ? -h.x : h.x, (corner & 2u) ? -h.y : h.y, (corner & 1u) ? -h.z : h.z};
            const v3 r = rot_sc(q, local);
            const v3 ip = {rel.x + r.x, rel.y + r.y, rel.z + r.z};
            if (ip.y >= cd) continue;
            cands[n++] = {local, {ip.x, 0.0f, ip.z}, {0.0f, 1.0f, 0.0f}, ip.y};
        }
        if (n <= 4) {
            for (int i = 0; i < n; ++i) cache.pts[i] = to_pt(cands[i]);
            set_meta(cache, uint32_t(n), true);
        } else {
            bool chosen[8] = {false, false, false, false, false, false, false, false};
            int idx[4];
            int first = 0;
            for (int i = 1; i < n; ++i)
                if (cands[i].sep < cands[first].sep) first = i;
            idx[0] = first;
            chosen[first] = true;
            int far = 0;
            float maxd = vlen2(vsub(cands[0].lb, cands[first].lb));
            for (int i = 1; i < n; ++i) {
                const float d = vlen2(vsub(cands[i].lb, cands[first].lb));
                if (d > maxd) { maxd = d; far = i; }
            }
            idx[1] = far;
            chosen[far] = true;
            const v3 seg = vsub(cands[far].lb, cands[first].lb);
            v3 side = {-seg.z, 0.0f, seg.x};
            const float ns = vlen2(side);
            if (ns > 0.0f) {
                const float inv = 1.0f / sqrtf(ns);
                side = {side.x * inv, 0.0f, side.z * inv};
            } else {
                side = {0.0f, 1.0f, 0.0f};
            }
            float largest = -FLT_MAX, smallest = FLT_MAX;
            int third = 0, fourth = 0;
            for (int i = 0; i < n; ++i) {
                if (chosen[i]) continue;
                const float d = vdot(vsub(cands[i].lb, cands[first].lb), side);
                if (d > largest) { largest = d; third = i; }
                if (d < smallest) { smallest = d; fourth = i; }
            }
            idx[2] = third;
            chosen[third] = true;
            if (smallest * largest > 0.0f) {
                largest = -FLT_MAX;
                for (int i = 0; i < n; ++i) {
                    if (chosen[i]) continue;
                    const float d = vdot(vsub(cands[i].lb, cands[first].lb), side);
                    if (d > largest) { largest = d; fourth = i; }
                }
            }
            idx[3] = fourth;
            chosen[fourth] = true;
            Cand centers[4];
            for (int k = 0; k < 4; ++k) centers[k] = cands[idx[k]];
            for (int i = 0; i < n; ++i) {
                if (chosen[i]) continue;
                float nearest = FLT_MAX;
                int slot = 0;
                for (int j = 0; j < 4; ++j) {
                    const float d = vlen2(vsub(cands[i].lb, centers[j].lb));
                    if (d < nearest) { nearest = d; slot = j; }
                }
                if (cands[i].sep < cands[idx[slot]].sep) idx[slot] = i;
            }
            for (int k = 0; k < 4; ++k) cache.pts[k] = to_pt(cands[idx[k]]);
            set_meta(cache, 4, true);
        }
    }
    int emitted = 0;
    const uint32_t n = cache_count(cache);
    for (uint32_t k = 0; k < n; ++k) {
        const PcmPoint& pt = cache.pts[k];
        if (pt.sep > cd) continue;
        ContactPt& o = out[emitted++];
        o.p[0] = pp.x + pt.lb[0]; o.p[1] = pp.y; o.p[2] = pp.z + pt.lb[2];
        // Plane manifolds are published with the flipped (+y) normal
        // (scene.cpp:4670-4677).
        o.n[0] = 0.0f; o.n[1] = 1.0f; o.n[2] = 0.0f;
        o.sep = pt.sep;
    }
    return emitted;
}

__device__ int sphere_sphere(v3 a, float r0, v3 b, float r1, float cd, ContactPt& o) {
    const v3 delta = vsub(a, b);
    const float d2 = vdot(delta, delta);
    const float rs = r0 + r1;
    const float infl = rs + cd;
    if (!(infl * infl > d2)) return 0;
    const float dist = sqrtf(d2);
    const v3 n = dist <= 0.00001f ? v3{1, 0, 0} : vmul(delta, 1.0f / dist);
    const v3 p = vadd(b, vmul(n, r1));
    o.p[0] = p.x; o.p[1] = p.y; o.p[2] = p.z;
    o.n[0] = n.x; o.n[1] = n.y; o.n[2] = n.z;
    o.sep = dist - rs;
    return 1;
}
__device__ int sphere_plane(v3 c, float r, float ph, float cd, ContactPt& o) {
    const float sep = c.y - ph - r;
    if (!(cd >= sep)) return 0;
    o.p[0] = c.x; o.p[1] = c.y - r; o.p[2] = c.z;
    o.n[0] = 0.f; o.n[1] = 1.f; o.n[2] = 0.f;   // two flips cancel (scene.cpp:4474-4482, 4670)
    o.sep = sep;
    return 1;
}
__device__ int sphere_box(v3 center, float r, v3 h, v3 bc, qt bq, float cd, ContactPt& o) {
    const v3 local = rotinv_gu(bq, vsub(center, bc));
    const v3 cl = {sclamp(local.x, -h.x, h.x), sclamp(local.y, -h.y, h.y), sclamp(local.z, -h.z, h.z)};
    const v3 gap = vsub(local, cl);
    const float l2 = vdot(gap, gap);
    const float infl = r + cd;
    if (!(infl * infl > l2)) return 0;
    const bool inside = fabsf(local.x) <= h.x && fabsf(local.y) <= h.y && fabsf(local.z) <= h.z;
    v3 p, n;
    float sep;
    if (inside) {
        const v3 d = {h.x - fabsf(cl.x), h.y - fabsf(cl.y), h.z - fabsf(cl.z)};
        v3 nl;
        float depth;
        if (d.z <= d.x && d.z <= d.y) { nl = {0, 0, cl.z >= 0.f ? 1.f : -1.f}; depth = d.z; }
        else if (d.x <= d.y && d.x <= d.z) { nl = {cl.x >= 0.f ? 1.f : -1.f, 0, 0}; depth = d.x; }
        else { nl = {0, cl.y >= 0.f ? 1.f : -1.f, 0}; depth = d.y; }
        n = rot_gu(bq, nl);
        p = vadd(center, vmul(n, depth));
        sep = -depth - r;
    } else {
        const float len = sqrtf(l2);
        n = rot_gu(bq, vmul(gap, 1.f / len));
        p = vadd(bc, rot_gu(bq, cl));
        sep = len - r;
    }
    o.p[0] = p.x; o.p[1] = p.y; o.p[2] = p.z;
    o.n[0] = n.x; o.n[1] = n.y; o.n[2] = n.z;
    o.sep = sep;
    return 1;
}

// Gu order of a pair (scene.cpp:4298-4310): planes first, otherwise the
// ScNPhaseCore::shouldSwapBodies orientation (scene.cpp:3275-3283).
struct PairShapes {
    uint32_t sa, sb, ta, tb, first, second;
    bool plane, sphere, convex;
    float cd;
};
__device__ __forceinline__ PairShapes pair_shapes(const DevState& s, uint64_t key) {
    PairShapes p;
    p.sa = uint32_t(key >> 32);
    p.sb = uint32_t(key);
    p.ta = s.s_type[p.sa];
    p.tb = s.s_type[p.sb];
    const uint32_t ba = s.s_body[p.sa], bb = s.s_body[p.sb];
    const bool da = s.b_flags[ba] & kBodyDynamic, db = s.b_flags[bb] & kBodyDynamic;
    const bool reversed = !da || (da && db && ba < bb);
    p.plane = p.ta == kPlane || p.tb == kPlane;
    // a pair with a cooked hull takes the convex generators whatever the
    // other shape is (scene.cpp:4307-4317)
    p.convex = p.ta == kConvex || p.tb == kConvex;
    p.sphere = !p.convex && (p.ta == kSphere || p.tb == kSphere);
    p.first = p.plane ? (p.ta == kPlane ? p.sa : p.sb) : (reversed ? p.sb : p.sa);
    p.second = p.plane ? (p.ta == kPlane ? p.sb : p.sa) : (reversed ? p.sa : p.sb);
    p.cd = s.s_lp[p.sa].w + s.s_lp[p.sb].w;
    return p;
}

__global__ void __launch_bounds__(128) k_narrowphase(DevState s) {
    const uint32_t n = *s.cur.n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        const int32_t pj = s.prev_idx[k];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        // only box and hull manifolds are persistent (PCM): sphere pairs
        // neither read nor carry a cache (their slot is never consumed)
        const bool pcm = !ps.sphere;
        PcmCache cache;
        if (pcm && pj >= 0) cache = s.prev.cache[pj];
        else cache.meta = 0u;
        if (ps.convex) {
            // carried forward here, generated by k_narrowphase_convex
            s.cur.cache[k] = cache;
            s.cvx_list[atomicAdd(&s.counters[kCntConvex], 1u)] = k;
            continue;
        }
        const uint32_t sa = ps.sa, sb = ps.sb, ta = ps.ta, tb = ps.tb, first = ps.first, second = ps.second;
        const bool plane = ps.plane, sphere = ps.sphere;
        const float cd = ps.cd;
        ContactPt out[4];
        int count = 0;
        const v3 p0 = ld3(s.s_wp[first]), p1 = ld3(s.s_wp[second]);
        const qt q0 = ldq(s.s_wq[first]), q1 = ldq(s.s_wq[second]);
        const float4 g0 = s.s_geom[first], g1 = s.s_geom[second];
        if (plane && !sphere) {
            count = generate_plane_box(p0, {g1.x, g1.y, g1.z}, p1, q1, cd, cache, out);
        } else if (!plane && !sphere) {
            bool gjk_pending = false;
            count = generate_box_box({g0.x, g0.y, g0.z}, p0, q0, {g1.x, g1.y, g1.z}, p1, q1, cd, cache, out,
                                     gjk_pending);
            if (gjk_pending) s.gjk_list[atomicAdd(&s.counters[kCntGjk], 1u)] = k;
        } else {
            const uint32_t sp = ta == kSphere ? sa : sb;
            const v3 c = ld3(s.s_wp[sp]);
            const float r = s.s_geom[sp].w;
            if (plane) {
                count = sphere_plane(c, r, p0.y, cd, out[0]);
            } else if (ta == kSphere && tb == kSphere) {
                count = sphere_sphere(p0, g0.w, p1, g1.w, cd, out[0]);
            } else {
                const uint32_t bx = ta == kBox ? sa : sb;
                const float4 gb = s.s_geom[bx];
                count = sphere_box(c, r, {gb.x, gb.y, gb.z}, ld3(s.s_wp[bx]), ldq(s.s_wq[bx]), cd, out[0]);
                if (count && s.s_type[first] == kBox) {
                    out[0].n[0] = -out[0].n[0]; out[0].n[1] = -out[0].n[1]; out[0].n[2] = -out[0].n[2];
                }
            }
        }
        if (count < 0) {
            atomicOr(s.err, kErrContactOverflow);
            count = 0;
        }
        if (pcm) s.cur.cache[k] = cache;
        s.cur.count[k] = uint32_t(count);
        for (int i = 0; i < count; ++i) s.pts[4 * size_t(k) + i] = out[i];
        // friction histories are not carried here: row preparation reads a
        // touching manager's history from the previous generation
    }
}

// Box/box pairs whose regenerated manifold had no face contact: GJK/EPA
// witness and emission from the cache the first kernel left behind.  These
// are few (hundreds to a few thousand per step) and each is a long search,
// so one warp takes a pair: the warp runs GJK in step (the sub-simplex
// search one subset per lane) and EPA together (run_epa_warp) with the
// polytope in shared memory.
constexpr int kGjkWarps = 4;
__global__ void __launch_bounds__(kGjkWarps * 32, 3) k_narrowphase_gjk(DevState s) {
    __shared__ EpaShared epa[kGjkWarps];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t n = s.counters[kCntGjk];
    const uint32_t nwarps = gridDim.x * kGjkWarps;
    for (uint32_t i = blockIdx.x * kGjkWarps + wib; i < n; i += nwarps) {
        const uint32_t k = s.gjk_list[i];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        const float4 g0 = s.s_geom[ps.first], g1 = s.s_geom[ps.second];
        const v3 h0 = {g0.x, g0.y, g0.z}, h1 = {g1.x, g1.y, g1.z};
        const v3 p0 = ld3(s.s_wp[ps.first]), p1 = ld3(s.s_wp[ps.second]);
        const qt q0 = ldq(s.s_wq[ps.first]), q1 = ldq(s.s_wq[ps.second]);
        BPair bp = {};
        bp.ha = h0;
        bp.hb = h1;
        bp.a_in_b = rotinv_gu(q1, vsub(p0, p1));
        bp.rel = qmul(qconj(q1), q0);
        Cand w = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f};
        Sup simplex[4];
        int sc = 0;
        const int mode = gjk_phase<false>(bp, ps.cd, w, simplex, sc);
        bool have = mode == 1;
        if (mode == 2) have = run_epa_warp<false>(bp, simplex, sc, w, epa[wib]);
        if (lane == 0) {
            have = have && w.sep <= ps.cd;
            PcmCache cache = s.cur.cache[k];
            ContactPt out[4];
            int count = finish_box_box_gjk(h0, h1, p1, q1, ps.cd, cache, have, w, out);
            if (count < 0) {
                atomicOr(s.err, kErrContactOverflow);
                count = 0;
            }
            s.cur.cache[k] = cache;
            s.cur.count[k] = uint32_t(count);
            for (int j = 0; j < count; ++j) s.pts[4 * size_t(k) + j] = out[j];
        }
        __syncwarp();
    }
}

// ---------------- cooked convex hulls ----------------
// A finite shape as the convex generators see it (the PcmFiniteShape of
// scene.cpp:3712-3731 plus the attached shape's half extents, which the
// rotation travel test uses).
struct Fin {
    v3 half;            // box: half extents; sphere: radius; hull: half bound size
    v3 shalf;           // attached half extents (zero for spheres)
    v3 p;
    qt q;
    float radius;       // sphere radius, else 0
    float extent;       // margin extent (scene.cpp:3666-3677)
    uint32_t vo, nv, fo, nf;
};
__device__ Fin load_fin(const DevState& s, uint32_t sh) {
    Fin f;
    const uint32_t t = s.s_type[sh];
    const float4 g = s.s_geom[sh];
    f.p = ld3(s.s_wp[sh]);
    f.q = ldq(s.s_wq[sh]);
    f.radius = 0.f;
    f.vo = f.nv = f.fo = f.nf = 0;
    f.shalf = {g.x, g.y, g.z};
    if (t == kConvex) {
        const uint32_t m = s.s_mesh[sh];
        const uint4 mt = s.m_tab[m];
        const float4 mh = s.m_half[m];
        f.half = {mh.x, mh.y, mh.z};
        f.extent = mh.w;
        f.vo = mt.x; f.nv = mt.y; f.fo = mt.z; f.nf = mt.w;
    } else if (t == kSphere) {
        f.radius = g.w;
        f.half = {g.w, g.w, g.w};
        f.extent = g.w;
        f.shalf = {0.f, 0.f, 0.f};
    } else {
        f.half = {g.x, g.y, g.z};
        f.extent = smin(smin(g.x, g.y), g.z);
    }
    return f;
}

// Face geometry for the clipping of GuPCMGjkEpa.cpp:571-804: a hull's planar
// polygons or the six faces of a box, in the shape's frame.
__device__ __forceinline__ unsigned fc_count(const Fin& f) { return f.nv ? f.nf : 6u; }
__device__ __forceinline__ v3 fc_axis(unsigned i) { return i == 0 ? v3{1, 0, 0} : i == 1 ? v3{0, 1, 0} : v3{0, 0, 1}; }
__device__ __forceinline__ v3 fc_normal(const DevState& s, const Fin& f, unsigned k) {
    if (f.nv) return ld3(s.hf[f.fo + k]);
    return vmul(fc_axis(k / 2u), (k & 1u) ? 1.f : -1.f);
}
__device__ __forceinline__ unsigned fc_nvert(const DevState& s, const Fin& f, unsigned k) {
    return f.nv ? s.hfr[f.fo + k].y : 4u;
}
__device__ v3 fc_vertex_local(const DevState& s, const Fin& f, unsigned k, unsigned o) {
    if (f.nv) return ld3(s.hv[f.vo + s.hidx[s.hfr[f.fo + k].x + o]]);
    const float cu = (o == 0 || o == 3) ? 1.f : -1.f;
    const float cv = (o < 2) ? 1.f : -1.f;
    const v3 n = fc_normal(s, f, k);
    const unsigned c = k / 2u;
    const v3 u = fc_axis((c + 1u) % 3u);
    const v3 v = vcross(n, u);
    const float hu = vcomp(f.half, (c + 1u) % 3u), hv = vcomp(f.half, (c + 2u) % 3u);
    return vadd(vmul(n, vcomp(f.half, c)), vadd(vmul(u, cu * hu), vmul(v, cv * hv)));
}
struct Clip {
    const DevState* s;
    const Fin *a, *b, *ref, *inc;
    bool ref_is_a, inc_is_a, reference_b;
    unsigned rf, inf, nr, ni;
    v3 rn, anchor;
    float cd, tol_sq;
    Cand* out;
    unsigned count;
};
__device__ __forceinline__ v3 clip_to_b(const Clip& k, v3 p) {
    return rotinv_gu(k.b->q, vsub(vadd(k.a->p, rot_gu(k.a->q, p)), k.b->p));
}
__device__ __forceinline__ v3 clip_vertex(const Clip& k, const Fin& f, bool is_a, unsigned face, unsigned o) {
    const v3 l = fc_vertex_local(*k.s, f, face, o);
    return is_a ? clip_to_b(k, l) : l;
}
__device__ __forceinline__ v3 clip_normal(const Clip& k, const Fin& f, bool is_a, unsigned face) {
    const v3 n = fc_normal(*k.s, f, face);
    return is_a ? rotinv_gu(k.b->q, rot_gu(k.a->q, n)) : n;
}
__device__ __forceinline__ v3 clip_r(const Clip& k, unsigned i) { return clip_vertex(k, *k.ref, k.ref_is_a, k.rf, i % k.nr); }
__device__ __forceinline__ v3 clip_q(const Clip& k, unsigned i) { return clip_vertex(k, *k.inc, k.inc_is_a, k.inf, i % k.ni); }
__device__ __forceinline__ float clip_cross(const Clip& k, v3 a, v3 b) { return vdot(k.rn, vcross(a, b)); }
// One clipped point: projected onto the reference plane, merged with a
// nearby one (keeping the deeper), or reduced greedily to four.
__device__ void clip_emit(Clip& k, v3 ip) {
    const float sep = vdot(k.rn, vsub(ip, k.anchor));
    if (!isfinite(sep) || sep > k.cd) return;
    const v3 proj = vsub(ip, vmul(k.rn, sep));
    const v3 a = k.reference_b ? ip : proj;
    const v3 b = k.reference_b ? proj : ip;
    const v3 al = rotinv_gu(k.a->q, vsub(vadd(k.b->p, rot_gu(k.b->q, a)), k.a->p));
    const Cand c = {al, b, k.reference_b ? k.rn : vneg(k.rn), sep};
    if (!isfinite(al.x) || !isfinite(b.x)) return;
    for (unsigned i = 0; i < k.count; ++i)
        if (vlen2(vsub(k.out[i].lb, c.lb)) <= k.tol_sq) {
            if (c.sep < k.out[i].sep) k.out[i] = c;
            return;
        }
    if (k.count < 4u) {
        k.out[k.count++] = c;
        return;
    }
    Cand ch[5] = {k.out[0], k.out[1], k.out[2], k.out[3], c};
    unsigned deepest = 0;
    for (unsigned i = 1; i < 5; ++i)
        if (ch[i].sep < ch[deepest].sep) deepest = i;
    float best = -1.f;
    unsigned omit = 4;
    for (unsigned ex = 0; ex < 5; ++ex) {
        if (ex == deepest) continue;
        float score = 0.f;
        for (unsigned i = 0; i < 5; ++i) {
            if (i == ex) continue;
            for (unsigned j = i + 1; j < 5; ++j)
                if (j != ex) score += vlen2(vsub(ch[i].lb, ch[j].lb));
        }
        if (score > best) { best = score; omit = ex; }
    }
    if (omit != 4u) k.out[omit] = c;
}
// GuPCMGjkEpa.cpp:571-804: reference and incident faces most aligned with
// the witness normal, incident vertices inside the reference polygon,
// reference vertices inside the incident one, and edge crossings.
__device__ int face_contacts(const DevState& s, const Fin& a, const Fin& b, float cd, const Cand& w, Cand out[4]) {
    if (a.radius > 0.f || b.radius > 0.f || (a.nv && !a.nf) || (b.nv && !b.nf)) return 0;
    Clip k;
    k.s = &s; k.a = &a; k.b = &b;
    const v3 normal = w.nb;
    if (!(vlen2(normal) > 0.f)) return 0;
    unsigned fa = 0, fb = 0;
    float ala = -2.f, alb = -2.f;
    for (unsigned i = 0; i < fc_count(a); ++i) {
        const float d = vdot(vneg(normal), clip_normal(k, a, true, i));
        if (d > ala) { ala = d; fa = i; }
    }
    for (unsigned i = 0; i < fc_count(b); ++i) {
        const float d = vdot(normal, clip_normal(k, b, false, i));
        if (d > alb) { alb = d; fb = i; }
    }
    k.reference_b = alb >= ala;
    if (smax(ala, alb) < 0.95f) return 0;
    k.ref = k.reference_b ? &b : &a;
    k.inc = k.reference_b ? &a : &b;
    k.ref_is_a = !k.reference_b;
    k.inc_is_a = k.reference_b;
    k.rf = k.reference_b ? fb : fa;
    k.rn = clip_normal(k, *k.ref, k.ref_is_a, k.rf);
    float ial = -2.f;
    k.inf = 0;
    for (unsigned i = 0; i < fc_count(*k.inc); ++i) {
        const float d = vdot(vneg(k.rn), clip_normal(k, *k.inc, k.inc_is_a, i));
        if (d > ial) { ial = d; k.inf = i; }
    }
    const v3 in_n = clip_normal(k, *k.inc, k.inc_is_a, k.inf);
    const float den = vdot(in_n, k.rn);
    if (!(den < -0.25f)) return 0;
    k.nr = fc_nvert(s, *k.ref, k.rf);
    k.ni = fc_nvert(s, *k.inc, k.inf);
    if (k.nr < 3u || k.ni < 3u) return 0;
    k.anchor = clip_r(k, 0);
    const v3 in_anchor = clip_q(k, 0);
    float el = 0.f;
    for (unsigned i = 0; i < k.nr; ++i) el = smax(el, vlen2(vsub(clip_r(k, i + 1), clip_r(k, i))));
    for (unsigned i = 0; i < k.ni; ++i) el = smax(el, vlen2(vsub(clip_q(k, i + 1), clip_q(k, i))));
    const float scale = sqrtf(el);
    if (!(scale > 0.f) || !isfinite(scale)) return 0;
    const float tol = smax(scale * 1.e-5f, 1.e-6f);
    const float ftol = tol / scale;
    k.tol_sq = tol * tol;
    k.cd = cd;
    k.out = out;
    k.count = 0;
    for (unsigned i = 0; i < k.ni; ++i) {
        const v3 v = clip_q(k, i);
        bool inside = true;
        for (unsigned j = 0; j < k.nr && inside; ++j)
            if (clip_cross(k, vsub(clip_r(k, j + 1), clip_r(k, j)), vsub(v, clip_r(k, j))) < -tol * scale) inside = false;
        if (inside) clip_emit(k, v);
    }
    for (unsigned i = 0; i < k.nr; ++i) {
        const v3 v = clip_r(k, i);
        bool inside = true;
        for (unsigned j = 0; j < k.ni && inside; ++j)
            if (clip_cross(k, vsub(clip_q(k, j + 1), clip_q(k, j)), vsub(v, clip_q(k, j))) > tol * scale) inside = false;
        if (!inside) continue;
        const float height = vdot(in_n, vsub(in_anchor, v)) / den;
        if (isfinite(height)) clip_emit(k, vadd(v, vmul(k.rn, height)));
    }
    for (unsigned i = 0; i < k.ni; ++i) {
        const v3 qa = clip_q(k, i), e = vsub(clip_q(k, i + 1), qa);
        for (unsigned j = 0; j < k.nr; ++j) {
            const v3 rb = clip_r(k, j), f = vsub(clip_r(k, j + 1), rb);
            const float det = clip_cross(k, e, f);
            if (fabsf(det) <= k.tol_sq) continue;
            const v3 d = vsub(rb, qa);
            const float t = clip_cross(k, d, f) / det;
            const float u = clip_cross(k, d, e) / det;
            if (t >= -ftol && t <= 1.f + ftol && u >= -ftol && u <= 1.f + ftol)
                clip_emit(k, vadd(qa, vmul(e, sclamp(t, 0.f, 1.f))));
        }
    }
    return int(k.count);
}

// The same clipping with the whole warp: the face searches are warp
// argmax reductions (largest alignment, lowest face on ties: the face the
// sequential first-maximum scan keeps), both polygons are staged once in
// shared memory in B's frame, and each clipping loop tests 32 points at a
// time with lane 0 emitting the accepted ones in the sequential order.
// Every lane calls it; the result is on lane 0.  Polygons of more than
// kClipPoly vertices take the lane-0 version above.
constexpr unsigned kClipPoly = 64;
struct ClipShared {
    float4 rv[kClipPoly], qv[kClipPoly];
};
__device__ __forceinline__ void warp_argmax_first(float& best, unsigned& idx) {
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const unsigned oi = __shfl_xor_sync(0xffffffffu, idx, off);
        if (oi != 0xffffffffu && (idx == 0xffffffffu || ob > best || (ob == best && oi < idx))) { best = ob; idx = oi; }
    }
    best = __shfl_sync(0xffffffffu, best, 0);
    idx = __shfl_sync(0xffffffffu, idx, 0);
}
__device__ int face_contacts_warp(const DevState& s, const Fin& a, const Fin& b, float cd, const Cand& w, Cand out[4],
                                  ClipShared& C) {
    const unsigned lane = threadIdx.x & 31u;
    const uint32_t full = 0xffffffffu;
    if (a.radius > 0.f || b.radius > 0.f || (a.nv && !a.nf) || (b.nv && !b.nf)) return 0;
    Clip k;
    k.s = &s; k.a = &a; k.b = &b;
    const v3 normal = w.nb;
    if (!(vlen2(normal) > 0.f)) return 0;
    // a lane's first maximum over its faces, then the warp's; the scan's
    // initial value -2 is below every alignment, so "no face" never wins
    float ala = -2.f, alb = -2.f;
    unsigned fa = 0xffffffffu, fb = 0xffffffffu;
    for (unsigned i = lane; i < fc_count(a); i += 32) {
        const float d = vdot(vneg(normal), clip_normal(k, a, true, i));
        if (fa == 0xffffffffu ? d > -2.f : d > ala) { ala = d; fa = i; }
    }
    for (unsigned i = lane; i < fc_count(b); i += 32) {
        const float d = vdot(normal, clip_normal(k, b, false, i));
        if (fb == 0xffffffffu ? d > -2.f : d > alb) { alb = d; fb = i; }
    }
    warp_argmax_first(ala, fa);
    warp_argmax_first(alb, fb);
    if (fa == 0xffffffffu) { ala = -2.f; fa = 0; }
    if (fb == 0xffffffffu) { alb = -2.f; fb = 0; }
    k.reference_b = alb >= ala;
    if (smax(ala, alb) < 0.95f) return 0;
    k.ref = k.reference_b ? &b : &a;
    k.inc = k.reference_b ? &a : &b;
    k.ref_is_a = !k.reference_b;
    k.inc_is_a = k.reference_b;
    k.rf = k.reference_b ? fb : fa;
    k.rn = clip_normal(k, *k.ref, k.ref_is_a, k.rf);
    float ial = -2.f;
    unsigned inf = 0xffffffffu;
    for (unsigned i = lane; i < fc_count(*k.inc); i += 32) {
        const float d = vdot(vneg(k.rn), clip_normal(k, *k.inc, k.inc_is_a, i));
        if (inf == 0xffffffffu ? d > -2.f : d > ial) { ial = d; inf = i; }
    }
    warp_argmax_first(ial, inf);
    k.inf = inf == 0xffffffffu ? 0u : inf;
    const v3 in_n = clip_normal(k, *k.inc, k.inc_is_a, k.inf);
    const float den = vdot(in_n, k.rn);
    if (!(den < -0.25f)) return 0;
    k.nr = fc_nvert(s, *k.ref, k.rf);
    k.ni = fc_nvert(s, *k.inc, k.inf);
    if (k.nr < 3u || k.ni < 3u) return 0;
    if (k.nr > kClipPoly || k.ni > kClipPoly) {
        int n = 0;
        if (lane == 0) n = face_contacts(s, a, b, cd, w, out);
        return n;
    }
    for (unsigned i = lane; i < k.nr; i += 32) C.rv[i] = st4(clip_vertex(k, *k.ref, k.ref_is_a, k.rf, i), 0.f);
    for (unsigned i = lane; i < k.ni; i += 32) C.qv[i] = st4(clip_vertex(k, *k.inc, k.inc_is_a, k.inf, i), 0.f);
    __syncwarp();
    const auto R = [&](unsigned i) { return ld3(C.rv[i % k.nr]); };
    const auto Q = [&](unsigned i) { return ld3(C.qv[i % k.ni]); };
    k.anchor = R(0);
    const v3 in_anchor = Q(0);
    float el = 0.f;
    for (unsigned i = lane; i < k.nr; i += 32) el = smax(el, vlen2(vsub(R(i + 1), R(i))));
    for (unsigned i = lane; i < k.ni; i += 32) el = smax(el, vlen2(vsub(Q(i + 1), Q(i))));
    for (int off = 16; off > 0; off >>= 1) el = smax(el, __shfl_xor_sync(full, el, off));
    el = __shfl_sync(full, el, 0);
    const float scale = sqrtf(el);
    if (!(scale > 0.f) || !isfinite(scale)) return 0;
    const float tol = smax(scale * 1.e-5f, 1.e-6f);
    const float ftol = tol / scale;
    k.tol_sq = tol * tol;
    k.cd = cd;
    k.out = out;
    k.count = 0;
    // lane 0 emits the chunk's accepted points in order
    const auto emit_chunk = [&](bool ok, v3 p) {
        uint32_t m = __ballot_sync(full, ok);
        while (m) {
            const int src = __ffs(m) - 1;
            m &= m - 1;
            const v3 q = {__shfl_sync(full, p.x, src), __shfl_sync(full, p.y, src), __shfl_sync(full, p.z, src)};
            if (lane == 0) clip_emit(k, q);
        }
    };
    for (unsigned c = 0; c < k.ni; c += 32) {
        const unsigned i = c + lane;
        bool inside = i < k.ni;
        const v3 v = inside ? Q(i) : v3{0, 0, 0};
        for (unsigned j = 0; j < k.nr && inside; ++j)
            if (clip_cross(k, vsub(R(j + 1), R(j)), vsub(v, R(j))) < -tol * scale) inside = false;
        emit_chunk(inside, v);
    }
    for (unsigned c = 0; c < k.nr; c += 32) {
        const unsigned i = c + lane;
        bool ok = i < k.nr;
        v3 p = {0, 0, 0};
        if (ok) {
            const v3 v = R(i);
            for (unsigned j = 0; j < k.ni && ok; ++j)
                if (clip_cross(k, vsub(Q(j + 1), Q(j)), vsub(v, Q(j))) > tol * scale) ok = false;
            if (ok) {
                const float height = vdot(in_n, vsub(in_anchor, v)) / den;
                ok = isfinite(height);
                p = vadd(v, vmul(k.rn, height));
            }
        }
        emit_chunk(ok, p);
    }
    const unsigned np = k.ni * k.nr;
    for (unsigned c = 0; c < np; c += 32) {
        const unsigned t = c + lane;
        bool ok = false;
        v3 p = {0, 0, 0};
        if (t < np) {
            const unsigned i = t / k.nr, j = t % k.nr;
            const v3 qa = Q(i), e = vsub(Q(i + 1), qa);
            const v3 rb = R(j), f = vsub(R(j + 1), rb);
            const float det = clip_cross(k, e, f);
            if (!(fabsf(det) <= k.tol_sq)) {
                const v3 d = vsub(rb, qa);
                const float tt = clip_cross(k, d, f) / det;
                const float u = clip_cross(k, d, e) / det;
                ok = tt >= -ftol && tt <= 1.f + ftol && u >= -ftol && u <= 1.f + ftol;
                p = vadd(qa, vmul(e, sclamp(tt, 0.f, 1.f)));
            }
        }
        emit_chunk(ok, p);
    }
    __syncwarp();
    return int(k.count);
}

// Hull vertices against the floor plane (scene.cpp:3774-3972): candidates
// are the vertices below the contact distance in vertex order; more than
// four are reduced to the deepest, the farthest from it, the two sideways
// extremes and the deepest of each cluster around those.  Candidates are
// recomputed from their vertex on every pass instead of being stored.
__device__ __forceinline__ bool plane_cand(const DevState& s, uint32_t vo, uint32_t v, v3 rel, qt q, float cd,
                                           Cand& c) {
    const v3 local = ld3(s.hv[vo + v]);
    const v3 r = rot_sc(q, local);
    const v3 ip = {rel.x + r.x, rel.y + r.y, rel.z + r.z};
    if (ip.y >= cd) return false;
    c = {local, {ip.x, 0.0f, ip.z}, {0.0f, 1.0f, 0.0f}, ip.y};
    return true;
}
__device__ int plane_hull(const DevState& s, const PairShapes& ps, PcmCache& cache, ContactPt* out) {
    const v3 pp = ld3(s.s_wp[ps.first]);
    const uint32_t sh = ps.second;
    const float4 g = s.s_geom[sh];
    const v3 bp = ld3(s.s_wp[sh]);
    const qt q = ldq(s.s_wq[sh]);
    const uint4 mt = s.m_tab[s.s_mesh[sh]];
    const float cd = ps.cd;
    const v3 rel = {bp.x - pp.x, bp.y - pp.y, bp.z - pp.z};
    const float brk = pcm_box_margin({g.x, g.y, g.z}) * 0.2f;
    const uint32_t prev = cache_count(cache);
    refresh_points(cache, rel, q, brk);
    const bool init = cache_init(cache);
    float md = INFINITY;
    if (init)
        md = smax(smax(fabsf(rel.x - cache.rel_p[0]), fabsf(rel.y - cache.rel_p[1])), fabsf(rel.z - cache.rel_p[2]));
    const float rd = q.x * cache.rel_q[0] + q.y * cache.rel_q[1] + q.z * cache.rel_q[2] + q.w * cache.rel_q[3];
    if (!init || cache_count(cache) != prev || md > brk || rd < 0.99996f) {
        sv(cache.rel_p, rel);
        cache.rel_q[0] = q.x; cache.rel_q[1] = q.y; cache.rel_q[2] = q.z; cache.rel_q[3] = q.w;
        Cand c;
        uint32_t n = 0, i0 = 0, first = 0;
        float fsep = 0.f;
        for (uint32_t v = 0; v < mt.y; ++v) {
            if (!plane_cand(s, mt.x, v, rel, q, cd, c)) continue;
            if (n == 0 || c.sep < fsep) { first = v; fsep = c.sep; }
            if (n == 0) i0 = v;
            if (n < 4) cache.pts[n] = to_pt(c);
            ++n;
        }
        if (n <= 4) {
            set_meta(cache, n, true);
        } else {
            uint32_t idx[4];
            int nch = 0;
            const auto chosen = [&](uint32_t v) {
                for (int j = 0; j < nch; ++j)
                    if (idx[j] == v) return true;
                return false;
            };
            Cand cf, cv;
            plane_cand(s, mt.x, first, rel, q, cd, cf);
            idx[nch++] = first;
            uint32_t far = i0;
            plane_cand(s, mt.x, i0, rel, q, cd, cv);
            float maxd = vlen2(vsub(cv.lb, cf.lb));
            for (uint32_t v = i0 + 1; v < mt.y; ++v) {
                if (!plane_cand(s, mt.x, v, rel, q, cd, cv)) continue;
                const float d = vlen2(vsub(cv.lb, cf.lb));
                if (d > maxd) { maxd = d; far = v; }
            }
            idx[nch++] = far;
            Cand cfar;
            plane_cand(s, mt.x, far, rel, q, cd, cfar);
            const v3 seg = vsub(cfar.lb, cf.lb);
            v3 side = {-seg.z, 0.0f, seg.x};
            const float ns = vlen2(side);
            if (ns > 0.0f) {
                const float inv = 1.0f / sqrtf(ns);
                side = {side.x * inv, 0.0f, side.z * inv};
            } else {
                side = {0.0f, 1.0f, 0.0f};
            }
            float largest = -FLT_MAX, smallest = FLT_MAX;
            uint32_t third = i0, fourth = i0;
            for (uint32_t v = 0; v < mt.y; ++v) {
                if (!plane_cand(s, mt.x, v, rel, q, cd, cv) || chosen(v)) continue;
                const float d = vdot(vsub(cv.lb, cf.lb), side);
                if (d > largest) { largest = d; third = v; }
                if (d < smallest) { smallest = d; fourth = v; }
            }
            idx[nch++] = third;
            if (smallest * largest > 0.0f) {
                largest = -FLT_MAX;
                for (uint32_t v = 0; v < mt.y; ++v) {
                    if (!plane_cand(s, mt.x, v, rel, q, cd, cv) || chosen(v)) continue;
                    const float d = vdot(vsub(cv.lb, cf.lb), side);
                    if (d > largest) { largest = d; fourth = v; }
                }
            }
            idx[nch++] = fourth;
            v3 centre[4];
            float cur_sep[4];
            for (int j = 0; j < 4; ++j) {
                plane_cand(s, mt.x, idx[j], rel, q, cd, cv);
                centre[j] = cv.lb;
                cur_sep[j] = cv.sep;
            }
            uint32_t best[4] = {idx[0], idx[1], idx[2], idx[3]};
            for (uint32_t v = 0; v < mt.y; ++v) {
                if (!plane_cand(s, mt.x, v, rel, q, cd, cv) || chosen(v)) continue;
                float nearest = FLT_MAX;
                int slot = 0;
                for (int j = 0; j < 4; ++j) {
                    const float d = vlen2(vsub(cv.lb, centre[j]));
                    if (d < nearest) { nearest = d; slot = j; }
                }
                if (cv.sep < cur_sep[slot]) { best[slot] = v; cur_sep[slot] = cv.sep; }
            }
            for (int j = 0; j < 4; ++j) {
                plane_cand(s, mt.x, best[j], rel, q, cd, cv);
                cache.pts[j] = to_pt(cv);
            }
            set_meta(cache, 4, true);
        }
    }
    int emitted = 0;
    const uint32_t n = cache_count(cache);
    for (uint32_t k = 0; k < n; ++k) {
        const PcmPoint& pt = cache.pts[k];
        if (pt.sep > cd) continue;
        ContactPt& o = out[emitted++];
        o.p[0] = pp.x + pt.lb[0]; o.p[1] = pp.y; o.p[2] = pp.z + pt.lb[2];
        o.n[0] = 0.0f; o.n[1] = 1.0f; o.n[2] = 0.0f;
        o.sep = pt.sep;
    }
    return emitted;
}

// Refresh and regeneration test of a finite pair with a cooked hull
// (scene.cpp:3655-3700): the refreshed cache, B-local pose of A, and whether
// the manifold must be regenerated.
__device__ bool convex_refresh(const Fin& f0, const Fin& f1, PcmCache& cache, v3& relative, qt& rotation) {
    const v3 delta = {f0.p.x - f1.p.x, f0.p.y - f1.p.y, f0.p.z - f1.p.z};
    relative = rotinv_sc(f1.q, delta);
    rotation = qmul(qconj(f1.q), f0.q);
    const float mm = smin(smin(0.15f * f0.extent, 0.15f), smin(0.15f * f1.extent, 0.15f));
    const uint32_t prev = cache_count(cache);
    refresh_points(cache, relative, rotation, mm * 0.8f);
    const bool init = cache_init(cache);
    const float tr = init ? smax(smax(fabsf(relative.x - cache.rel_p[0]), fabsf(relative.y - cache.rel_p[1])),
                                 fabsf(relative.z - cache.rel_p[2]))
                          : INFINITY;
    const float qa = qdot(f0.q, {cache.qa[0], cache.qa[1], cache.qa[2], cache.qa[3]});
    const float qb = qdot(f1.q, {cache.qb[0], cache.qb[1], cache.qb[2], cache.qb[3]});
    const float thr = mm * (cache_count(cache) == 0 ? 0.5f : 0.125f);
    if (!init || cache_count(cache) != prev || tr > thr || qa < 0.9999f || qb < 0.9999f) return true;
    const v3 ha = f0.shalf, hb = f1.shalf;
    const float ta = (qa < 1.f ? acosf(smax(-1.f, qa)) : 0.f) * sqrtf(ha.x * ha.x + ha.y * ha.y + ha.z * ha.z);
    const float tb = (qb < 1.f ? acosf(smax(-1.f, qb)) : 0.f) * sqrtf(hb.x * hb.x + hb.y * hb.y + hb.z * hb.z);
    return ta > thr || tb > thr;
}
// Cached witnesses within the contact distance, each with its own normal,
// in world space (scene.cpp:3752-3771).  -1 on a non-finite contact.
__device__ int convex_emit(const Fin& f1, float cd, const PcmCache& cache, ContactPt* out) {
    int count = 0;
    const uint32_t nc = cache_count(cache);
    for (uint32_t j = 0; j < nc; ++j) {
        const PcmPoint& pt = cache.pts[j];
        if (pt.sep > cd) continue;
        const v3 nrm = rot_sc(f1.q, lv(pt.nb));
        const v3 l = rot_sc(f1.q, lv(pt.lb));
        ContactPt& o = out[count++];
        o.p[0] = f1.p.x + l.x; o.p[1] = f1.p.y + l.y; o.p[2] = f1.p.z + l.z;
        o.n[0] = nrm.x; o.n[1] = nrm.y; o.n[2] = nrm.z;
        o.sep = pt.sep;
        if (!isfinite(o.p[0]) || !isfinite(o.p[1]) || !isfinite(o.p[2]) || !isfinite(nrm.x) || !isfinite(nrm.y) ||
            !isfinite(nrm.z) || !isfinite(o.sep))
            return -1;
    }
    return count;
}
__device__ __forceinline__ void store_manifold(const DevState& s, uint32_t k, const PcmCache& cache, int count,
                                               const ContactPt* out) {
    if (count < 0) {
        atomicOr(s.err, kErrContactOverflow);
        count = 0;
    }
    s.cur.cache[k] = cache;
    s.cur.count[k] = uint32_t(count);
    for (int j = 0; j < count; ++j) s.pts[4 * size_t(k) + j] = out[j];
}

// Pairs with a cooked hull, one thread each: hull vertices against the
// floor, and finite pairs whose cached manifold stays valid.  Finite pairs
// that regenerate go on to the warp kernel below.
__global__ void __launch_bounds__(128) k_narrowphase_convex(DevState s) {
    const uint32_t n = s.counters[kCntConvex];
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t k = s.cvx_list[i];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        PcmCache cache = s.cur.cache[k];
        ContactPt out[4];
        if (ps.plane) {
            const int count = plane_hull(s, ps, cache, out);
            store_manifold(s, k, cache, count, out);
            continue;
        }
        const Fin f0 = load_fin(s, ps.first), f1 = load_fin(s, ps.second);
        v3 relative;
        qt rotation;
        if (convex_refresh(f0, f1, cache, relative, rotation)) {
            s.cvx_gjk_list[atomicAdd(&s.counters[kCntConvexGjk], 1u)] = k;
            continue;
        }
        store_manifold(s, k, cache, convex_emit(f1, ps.cd, cache, out), out);
    }
}

// Finite hull pairs whose manifold regenerates (scene.cpp:3701-3751).  One
// warp takes a pair: GJK/EPA run together on every lane (hull supports are
// each lane's own scan of the vertices), faces are clipped on lane 0.
constexpr int kCvxWarps = 4;
// The regenerated pair's cache, B-local pose of A and GJK pair setup
// (shared by the GJK and EPA kernels).
__device__ __forceinline__ BPair convex_pair(const DevState& s, const Fin& f0, const Fin& f1) {
    BPair bp;
    bp.ha = f0.half;
    bp.hb = f1.half;
    bp.a_in_b = rotinv_gu(f1.q, vsub(f0.p, f1.p));
    bp.rel = qmul(qconj(f1.q), f0.q);
    bp.va = s.hv + f0.vo; bp.nva = f0.nv;
    bp.vb = s.hv + f1.vo; bp.nvb = f1.nv;
    bp.ra = f0.radius; bp.rb = f1.radius;
    return bp;
}
// After GJK or EPA: a witness within the contact distance goes to face
// clipping (the cache is stored for it); otherwise the manifold is stored
// now.  Every lane calls it with the same values.
__device__ void convex_finish(const DevState& s, uint32_t k, bool have, Cand w, const Fin& f0, const Fin& f1,
                              qt rel, float cd, PcmCache& cache) {
    const uint32_t lane = threadIdx.x & 31u;
    if (have) {
        // sphere radii applied along the final normal
        if (f0.radius > 0.f) {
            w.la = vadd(w.la, rotinv_gu(rel, vmul(w.nb, -f0.radius)));
            w.sep -= f0.radius;
        }
        if (f1.radius > 0.f) {
            w.lb = vadd(w.lb, vmul(w.nb, f1.radius));
            w.sep -= f1.radius;
        }
        if (w.sep <= cd) {
            if (lane == 0) {
                s.cur.cache[k] = cache;
                const uint32_t j = atomicAdd(&s.counters[kCntConvexClip], 1u);
                s.cvx_clip_list[j] = k;
                s.cvx_wit[3 * size_t(j)] = make_float4(w.la.x, w.la.y, w.la.z, w.lb.x);
                s.cvx_wit[3 * size_t(j) + 1] = make_float4(w.lb.y, w.lb.z, w.nb.x, w.nb.y);
                s.cvx_wit[3 * size_t(j) + 2] = make_float4(w.nb.z, w.sep, 0.f, 0.f);
            }
            return;
        }
    }
    if (lane == 0) {
        ContactPt out[4];
        store_manifold(s, k, cache, convex_emit(f1, cd, cache, out), out);
    }
}
__global__ void __launch_bounds__(kCvxWarps * 32, 3) k_narrowphase_convex_gjk(DevState s) {
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t n = s.counters[kCntConvexGjk];
    const uint32_t nwarps = gridDim.x * kCvxWarps;
    for (uint32_t i = blockIdx.x * kCvxWarps + wib; i < n; i += nwarps) {
        const uint32_t k = s.cvx_gjk_list[i];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        PcmCache cache = s.cur.cache[k];
        const Fin f0 = load_fin(s, ps.first), f1 = load_fin(s, ps.second);
        const float cd = ps.cd;
        v3 relative;
        qt rotation;
        convex_refresh(f0, f1, cache, relative, rotation);     // regenerates: listed by the kernel above
        sv(cache.rel_p, relative);
        cache.rel_q[0] = rotation.x; cache.rel_q[1] = rotation.y; cache.rel_q[2] = rotation.z; cache.rel_q[3] = rotation.w;
        cache.qa[0] = f0.q.x; cache.qa[1] = f0.q.y; cache.qa[2] = f0.q.z; cache.qa[3] = f0.q.w;
        cache.qb[0] = f1.q.x; cache.qb[1] = f1.q.y; cache.qb[2] = f1.q.z; cache.qb[3] = f1.q.w;
        set_meta(cache, 0, true);
        const BPair bp = convex_pair(s, f0, f1);
        Cand w = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f};
        Sup simplex[4];
        int sc = 0;
        const int mode = gjk_phase<true>(bp, cd + f0.radius + f1.radius, w, simplex, sc);
        if (mode == 2) {
            // EPA continues in its own kernel from this simplex
            if (lane == 0) {
                s.cur.cache[k] = cache;
                const uint32_t j = atomicAdd(&s.counters[kCntConvexEpa], 1u);
                s.cvx_epa_list[j] = k;
                float4* o = s.cvx_simplex + 12 * size_t(j);
                for (int q = 0; q < 4; ++q) {
                    const Sup& u = simplex[q];
                    o[3 * q] = make_float4(u.a.x, u.a.y, u.a.z, u.b.x);
                    o[3 * q + 1] = make_float4(u.b.y, u.b.z, u.q.x, u.q.y);
                    o[3 * q + 2] = make_float4(u.q.z, __uint_as_float(u.ai), __uint_as_float(u.bi),
                                               q == 3 ? __int_as_float(sc) : 0.f);
                }
            }
            __syncwarp();
            continue;
        }
        convex_finish(s, k, mode == 1, w, f0, f1, bp.rel, cd, cache);
        __syncwarp();
    }
}
// EPA of the regenerated hull pairs whose GJK reached it, one warp per pair.
__global__ void __launch_bounds__(kCvxWarps * 32, 3) k_narrowphase_convex_epa(DevState s) {
    __shared__ EpaShared epa[kCvxWarps];
    const uint32_t wib = threadIdx.x >> 5;
    const uint32_t n = s.counters[kCntConvexEpa];
    const uint32_t nwarps = gridDim.x * kCvxWarps;
    for (uint32_t i = blockIdx.x * kCvxWarps + wib; i < n; i += nwarps) {
        const uint32_t k = s.cvx_epa_list[i];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        PcmCache cache = s.cur.cache[k];
        const Fin f0 = load_fin(s, ps.first), f1 = load_fin(s, ps.second);
        const BPair bp = convex_pair(s, f0, f1);
        const float4* o = s.cvx_simplex + 12 * size_t(i);
        Sup simplex[4];
        for (int q = 0; q < 4; ++q) {
            const float4 x = o[3 * q], y = o[3 * q + 1], z = o[3 * q + 2];
            simplex[q].a = {x.x, x.y, x.z};
            simplex[q].b = {x.w, y.x, y.y};
            simplex[q].q = {y.z, y.w, z.x};
            simplex[q].ai = __float_as_uint(z.y);
            simplex[q].bi = __float_as_uint(z.z);
        }
        const int sc = __float_as_int(o[11].w);
        Cand w = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, 0.0f};
        const bool have = run_epa_warp<true>(bp, simplex, sc, w, epa[wib]);
        convex_finish(s, k, have, w, f0, f1, bp.rel, ps.cd, cache);
        __syncwarp();
    }
}

// Face clipping around the witnesses of the kernel above (its own kernel so
// that neither carries the other's code), one warp per pair, then the
// manifold's emission.
__global__ void __launch_bounds__(kCvxWarps * 32) k_narrowphase_convex_clip(DevState s) {
    __shared__ ClipShared clip[kCvxWarps];
    const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
    const uint32_t n = s.counters[kCntConvexClip];
    const uint32_t nwarps = gridDim.x * kCvxWarps;
    for (uint32_t i = blockIdx.x * kCvxWarps + wib; i < n; i += nwarps) {
        const uint32_t k = s.cvx_clip_list[i];
        const PairShapes ps = pair_shapes(s, s.cur.key[k]);
        PcmCache cache = s.cur.cache[k];
        const Fin f0 = load_fin(s, ps.first), f1 = load_fin(s, ps.second);
        const float4 w0 = s.cvx_wit[3 * size_t(i)], w1 = s.cvx_wit[3 * size_t(i) + 1], w2 = s.cvx_wit[3 * size_t(i) + 2];
        const Cand w = {{w0.x, w0.y, w0.z}, {w0.w, w1.x, w1.y}, {w1.z, w1.w, w2.x}, w2.y};
        Cand clipped[4];
        const int nc = face_contacts_warp(s, f0, f1, ps.cd, w, clipped, clip[wib]);
        if (lane == 0) {
            if (nc) {
                for (int j = 0; j < nc; ++j) cache.pts[j] = to_pt(clipped[j]);
                set_meta(cache, uint32_t(nc), true);
            } else {
                cache.pts[0] = to_pt(w);
                set_meta(cache, 1, true);
            }
            ContactPt out[4];
            store_manifold(s, k, cache, convex_emit(f1, ps.cd, cache, out), out);
        }
        __syncwarp();
    }
}

}  // namespace

void enqueue_narrowphase(const DevState& s, cudaStream_t st, const StageHook& hook) {
    const int T = 128;
    hook(kStNarrow, st);
    cudaMemsetAsync(s.counters + kCntGjk, 0, 4, st);
    cudaMemsetAsync(s.counters + kCntConvex, 0, 8, st);
    const uint32_t blocks = (s.pair_cap + T - 1) / T;
    k_narrowphase<<<blocks < 148u * 16u ? blocks : 148u * 16u, T, 0, st>>>(s);
    const uint32_t gb = (s.pair_cap + kGjkWarps - 1) / kGjkWarps;
    k_narrowphase_gjk<<<gb < 148u * 8u ? gb : 148u * 8u, kGjkWarps * 32, 0, st>>>(s);
    if (s.n_meshes) {
        cudaMemsetAsync(s.counters + kCntConvexClip, 0, 8, st);   // clip and EPA lists
        k_narrowphase_convex<<<blocks < 148u * 16u ? blocks : 148u * 16u, T, 0, st>>>(s);
        const uint32_t cb = (s.pair_cap + kCvxWarps - 1) / kCvxWarps;
        k_narrowphase_convex_gjk<<<cb < 148u * 8u ? cb : 148u * 8u, kCvxWarps * 32, 0, st>>>(s);
        k_narrowphase_convex_epa<<<cb < 148u * 8u ? cb : 148u * 8u, kCvxWarps * 32, 0, st>>>(s);
        k_narrowphase_convex_clip<<<cb < 148u * 8u ? cb : 148u * 8u, kCvxWarps * 32, 0, st>>>(s);
    }
}

}  // namespace fyzz::b200
