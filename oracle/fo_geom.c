/* Test infrastructure: C restatement of the reference's narrowphase
 * (Gu PCM) for the rigid-body step oracle.  Each function cites the
 * reference routine it restates; all paths are relative to the reference
 * project root.  Compiled with -ffp-contract=off. */
#include "fyzz_oracle.h"
#include "fo_math.h"
#include <string.h>
#include <stdlib.h>

/* ---------------- bounds (scene.cpp:26-35, 1233-1316) ---------------- */
static uint32_t encode_float(float v) {
    uint32_t bits;
    memcpy(&bits, &v, 4);
    return (bits & 0x80000000u) ? ~bits : (bits | 0x80000000u);
}
uint32_t fo_encode_min(float v) { return ((encode_float(v) >> 4) - 1u) << 4; }
uint32_t fo_encode_max(float v) { return (((encode_float(v) >> 4) + 1u) << 4) | 4u; }

/* Scene::update_shape_bounds for box and sphere shapes.  pose: world
 * position(3) + orientation(4); geom: half extents or radius. */
int fo_shape_bounds(uint32_t type, const float* pose, const float* geom,
                    float contact_offset, uint32_t* out6) {
    const v3 p = V3(pose[0], pose[1], pose[2]);
    const qt q = Q4(pose[3], pose[4], pose[5], pose[6]);
    v3 h = V3(geom[0], geom[1], geom[2]);
    v3 extent = type == FO_SPHERE ? V3(geom[0], geom[0], geom[0]) : h;
    if (type == FO_BOX && (q.x != 0.0f || q.y != 0.0f || q.z != 0.0f || q.w != 1.0f)) {
        const v3 x = rot_sc(q, V3(1, 0, 0)), y = rot_sc(q, V3(0, 1, 0)), z = rot_sc(q, V3(0, 0, 1));
        extent = V3(fabsf(x.x) * h.x + fabsf(y.x) * h.y + fabsf(z.x) * h.z,
                    fabsf(x.y) * h.x + fabsf(y.y) * h.y + fabsf(z.y) * h.z,
                    fabsf(x.z) * h.x + fabsf(y.z) * h.y + fabsf(z.z) * h.z);
    }
    extent.x += contact_offset;
    extent.y += contact_offset;
    extent.z += contact_offset;
    const float e[6] = {p.x - extent.x, p.y - extent.y, p.z - extent.z,
                        p.x + extent.x, p.y + extent.y, p.z + extent.z};
    for (int i = 0; i < 6; ++i)
        if (!isfinite(e[i])) return FO_OVERFLOW;
    for (int a = 0; a < 3; ++a) {
        out6[a] = fo_encode_min(e[a]);
        out6[a + 3] = fo_encode_max(e[a + 3]);
    }
    return 0;
}

/* ---------------- PCM box/box face contacts ----------------
 * GuPCMContactBoxBox.cpp:301-436 source_pcm_box_box_candidates and its
 * helpers contains (65-83), intersect_segment (87-103), calculate (119-179). */
typedef struct { v3 half, position; qt rotation; v3 axis[3]; } gbox;
static gbox make_box(v3 h, v3 p, qt q) {
    gbox b;
    b.half = h; b.position = p; b.rotation = q;
    b.axis[0] = rot_gu(q, V3(1, 0, 0));
    b.axis[1] = rot_gu(q, V3(0, 1, 0));
    b.axis[2] = rot_gu(q, V3(0, 0, 1));
    return b;
}
static v3 box_local(const gbox* b, v3 w) { return rotinv_gu(b->rotation, vsub(w, b->position)); }
typedef struct { v3 x, y, z, position; } frame_t;
static v3 fr_project(const frame_t* f, v3 w) {
    const v3 d = vsub(w, f->position);
    return V3(vdot(d, f->x), vdot(d, f->y), vdot(d, f->z));
}
static v3 fr_unproject(const frame_t* f, v3 v) {
    return vadd(f->position, vadd(vadd(vmul(f->x, v.x), vmul(f->y, v.y)), vmul(f->z, v.z)));
}
static int poly_contains(const v3 poly[4], v3 p, v3 low, v3 high) {
    if (p.x < low.x || p.y < low.y || p.x > high.x || p.y > high.y) return 0;
    unsigned hits = 0;
    const float eps = FLT_EPSILON;
    for (unsigned i = 0, j = 3; i < 4; j = i++) {
        const v3 a = poly[j], b = poly[i];
        if ((p.x == a.x && p.y == a.y) || (p.x == b.x && p.y == b.y)) return 1;
        if ((a.y > p.y) != (b.y > p.y)) {
            const float dx = b.x - a.x, dy = b.y - a.y;
            const float part = (p.y - a.y) * dx + (a.x + eps) * dy;
            const float target = p.x * dy;
            const int inter = dy > 0.0f ? part >= target : target >= part;
            if (inter && ++hits == 2) return 0;
        }
    }
    return hits > 0;
}
static int seg_aabb(v3 p, v3 delta, v3 high, v3 low, float* enter, float* exit_) {
    *enter = 0.0f;
    *exit_ = 1.0f;
    for (unsigned axis = 0; axis < 3; ++axis) {
        const float x = vcomp(p, axis), d = vcomp(delta, axis);
        const float mn = vcomp(low, axis), mx = vcomp(high, axis);
        if (fabsf(d) < 1.0e-6f) {
            if (x < mn || x > mx) return 0;
            continue;
        }
        const float one = (mn - x) / d, two = (mx - x) / d;
        *enter = fmaxf_(*enter, fminf_(one, two));
        *exit_ = fminf_(*exit_, fmaxf_(one, two));
    }
    return *enter <= *exit_ && *enter <= 1.0f;
}
typedef struct { const gbox* a; const gbox* b; fo_candidate* out; int cap; int count; int overflow; } gen_t;
static void gen_emit(gen_t* g, const frame_t* f, v3 reference, v3 incident, v3 normal,
                     float separation, int flipped) {
    if (g->count >= g->cap) { g->overflow = 1; return; }
    const v3 w0 = fr_unproject(f, flipped ? incident : reference);
    const v3 w1 = fr_unproject(f, flipped ? reference : incident);
    fo_candidate* c = &g->out[g->count++];
    const v3 la = box_local(g->a, w0), lb = box_local(g->b, w1);
    const v3 nb = rotinv_gu(g->b->rotation, normal);
    c->la[0] = la.x; c->la[1] = la.y; c->la[2] = la.z;
    c->lb[0] = lb.x; c->lb[1] = lb.y; c->lb[2] = lb.z;
    c->nb[0] = nb.x; c->nb[1] = nb.y; c->nb[2] = nb.z;
    c->sep = separation;
}
static void gen_calculate(gen_t* g, const frame_t* f, const v3 poly[4], v3 inc_n,
                          float face_x, float face_y, v3 normal, float cd, int flipped) {
    face_x *= 1.0001f;
    face_y *= 1.0001f;
    int pen[4] = {0, 0, 0, 0}, ins[4] = {0, 0, 0, 0};
    v3 mn = V3(FLT_MAX, FLT_MAX, FLT_MAX);
    v3 mx = vneg(mn);
    const v3 high = V3(face_x, face_y, FLT_MAX);
    for (unsigned i = 0; i < 4; ++i) {
        const v3 p = poly[i];
        mn.x = fminf_(mn.x, p.x); mn.y = fminf_(mn.y, p.y);
        mx.x = fmaxf_(mx.x, p.x); mx.y = fmaxf_(mx.y, p.y);
        if (-p.z < cd) {
            pen[i] = 1;
            ins[i] = fabsf(p.x) <= face_x && fabsf(p.y) <= face_y;
            if (ins[i]) gen_emit(g, f, V3(p.x, p.y, 0), p, normal, -p.z, flipped);
        }
    }
    if (g->count == 4) return;
    if (inc_n.z != 0.0f) {
        const v3 corners[4] = {{face_x, face_y, 0}, {face_x, -face_y, 0},
                               {-face_x, face_y, 0}, {-face_x, -face_y, 0}};
        for (int k = 0; k < 4; ++k) {
            const v3 corner = corners[k];
            if (!poly_contains(poly, corner, mn, mx)) continue;
            const float nom = vdot(inc_n, vsub(poly[0], corner));
            const float t = nom / inc_n.z;
            const float separation = -t;
            if (cd > separation)
                gen_emit(g, f, corner, V3(corner.x, corner.y, t), normal, separation, flipped);
        }
    }
    const v3 low = V3(-face_x, -face_y, -cd - FLT_EPSILON);
    for (unsigned start = 0, end = 3; start < 4; end = start++) {
        if (!pen[start] && !pen[end]) continue;
        const int c0 = pen[start] && ins[start];
        const int c1 = pen[end] && ins[end];
        if (c0 && c1) continue;
        const v3 edge = vsub(poly[end], poly[start]);
        float t0, t1;
        if (!seg_aabb(poly[start], edge, high, low, &t0, &t1)) continue;
        if (!c0) {
            const v3 p = vadd(poly[start], vmul(edge, t0));
            gen_emit(g, f, V3(p.x, p.y, 0), p, normal, -p.z, flipped);
        }
        if (!c1) {
            const v3 p = vadd(poly[start], vmul(edge, t1));
            gen_emit(g, f, V3(p.x, p.y, 0), p, normal, -p.z, flipped);
        }
    }
}

int fo_pcm_box_box_candidates(const float* ra, const float* rb, float cd,
                              fo_candidate* out, int cap, int* count) {
    const gbox a = make_box(V3(ra[0], ra[1], ra[2]), V3(ra[3], ra[4], ra[5]),
                            Q4(ra[6], ra[7], ra[8], ra[9]));
    const gbox b = make_box(V3(rb[0], rb[1], rb[2]), V3(rb[3], rb[4], rb[5]),
                            Q4(rb[6], rb[7], rb[8], rb[9]));
    gen_t g = {&a, &b, out, cap, 0, 0};
    const v3 delta = vsub(b.position, a.position);
    float sign[6], overlap[6];
    const float sat_eps = 1.0e-6f;
    *count = 0;
    for (unsigned i = 0; i < 6; ++i) {
        const int first = i < 3;
        const gbox* ref = first ? &a : &b;
        const gbox* inc = first ? &b : &a;
        const unsigned axis = i % 3;
        const v3 n = ref->axis[axis];
        sign[i] = vdot(delta, n);
        const float rad = (fabsf(vdot(n, inc->axis[0])) + sat_eps) * inc->half.x +
                          (fabsf(vdot(n, inc->axis[1])) + sat_eps) * inc->half.y +
                          (fabsf(vdot(n, inc->axis[2])) + sat_eps) * inc->half.z;
        overlap[i] = vcomp(ref->half, axis) + rad - fabsf(sign[i]) + cd;
        if (overlap[i] < 0.0f) return 0;
    }
    for (unsigned i = 0; i < 3; ++i)
        for (unsigned j = 0; j < 3; ++j) {
            const v3 ca = vcross(a.axis[i], b.axis[j]);
            float rA = 0.0f, rB = 0.0f;
            for (unsigned k = 0; k < 3; ++k) {
                if (k != i) rA += (fabsf(vdot(ca, a.axis[k])) + sat_eps) * vcomp(a.half, k);
                if (k != j) rB += (fabsf(vdot(ca, b.axis[k])) + sat_eps) * vcomp(b.half, k);
            }
            if (fabsf(vdot(delta, ca)) > rA + rB + cd) return 0;
        }
    unsigned feature = 0;
    float min_overlap = overlap[0];
    for (unsigned i = 1; i < 6; ++i)
        if (min_overlap > overlap[i]) { min_overlap = overlap[i]; feature = i; }
    const int flipped = feature >= 3;
    const gbox* inc = flipped ? &a : &b;
    const int nonpos = sign[feature] <= 0.0f;
    frame_t fr;
    v3 normal;
    float fx = 0, fy = 0;
    switch (feature) {
    case 0:
        normal = nonpos ? a.axis[0] : vneg(a.axis[0]);
        fr.x = nonpos ? vneg(a.axis[2]) : a.axis[2]; fr.y = a.axis[1]; fr.z = normal;
        fr.position = vadd(a.position, vmul(a.axis[0], nonpos ? -a.half.x : a.half.x));
        fx = a.half.z; fy = a.half.y; break;
    case 1:
        normal = nonpos ? a.axis[1] : vneg(a.axis[1]);
        fr.x = a.axis[0]; fr.y = nonpos ? vneg(a.axis[2]) : a.axis[2]; fr.z = normal;
        fr.position = vadd(a.position, vmul(a.axis[1], nonpos ? -a.half.y : a.half.y));
        fx = a.half.x; fy = a.half.z; break;
    case 2:
        normal = nonpos ? a.axis[2] : vneg(a.axis[2]);
        fr.x = a.axis[0]; fr.y = nonpos ? a.axis[1] : vneg(a.axis[1]); fr.z = normal;
        fr.position = vadd(a.position, vmul(a.axis[2], nonpos ? -a.half.z : a.half.z));
        fx = a.half.x; fy = a.half.y; break;
    case 3:
        normal = nonpos ? b.axis[0] : vneg(b.axis[0]);
        fr.x = nonpos ? b.axis[2] : vneg(b.axis[2]); fr.y = b.axis[1]; fr.z = vneg(normal);
        fr.position = vadd(b.position, vmul(b.axis[0], nonpos ? b.half.x : -b.half.x));
        fx = b.half.z; fy = b.half.y; break;
    case 4:
        normal = nonpos ? b.axis[1] : vneg(b.axis[1]);
        fr.x = b.axis[0]; fr.y = nonpos ? b.axis[2] : vneg(b.axis[2]); fr.z = vneg(normal);
        fr.position = vadd(b.position, vmul(b.axis[1], nonpos ? b.half.y : -b.half.y));
        fx = b.half.x; fy = b.half.z; break;
    default:
        normal = nonpos ? b.axis[2] : vneg(b.axis[2]);
        fr.x = b.axis[0]; fr.y = nonpos ? vneg(b.axis[1]) : b.axis[1]; fr.z = vneg(normal);
        fr.position = vadd(b.position, vmul(b.axis[2], nonpos ? b.half.z : -b.half.z));
        fx = b.half.x; fy = b.half.y; break;
    }
    const v3 search = vneg(fr.z);
    const float dx = fabsf(vdot(search, inc->axis[0]));
    const float dy = fabsf(vdot(search, inc->axis[1]));
    const float dz = fabsf(vdot(search, inc->axis[2]));
    const unsigned ia = dx >= dy && dx >= dz ? 0 : (dy >= dz ? 1 : 2);
    const float facing = vdot(search, inc->axis[ia]);
    const float sext = facing > 0.0f ? -vcomp(inc->half, ia) : vcomp(inc->half, ia);
    const v3 fc = vadd(inc->position, vmul(inc->axis[ia], sext));
    const unsigned ua = ia == 0 ? 1 : 0;
    const unsigned va = ia == 2 ? 1 : 2;
    const v3 u = vmul(inc->axis[ua], vcomp(inc->half, ua));
    const v3 v = vmul(inc->axis[va], vcomp(inc->half, va));
    const v3 pw[4] = {vadd(fc, vadd(u, v)), vadd(fc, vsub(u, v)),
                      vsub(fc, vadd(u, v)), vsub(fc, vsub(u, v))};
    v3 poly[4];
    for (int i = 0; i < 4; ++i) poly[i] = fr_project(&fr, pw[i]);
    const v3 face_n = fr_project(&fr, vadd(fr.position, facing > 0.0f ? vneg(inc->axis[ia])
                                                                       : inc->axis[ia]));
    gen_calculate(&g, &fr, poly, face_n, fx, fy, normal, cd, flipped);
    if (g.overflow) return FO_OVERFLOW_NEG;
    *count = g.count;
    return 1;
}

/* GuPCMContactBoxBox.cpp:185-297 source_pcm_box_batch_selection. */
int fo_pcm_batch_selection(const fo_candidate* c, int n, float tol, uint8_t sel[4]) {
    if (n <= 4 || n > 64) return FO_LOGIC_NEG;
    uint8_t avail[64];
    for (int i = 0; i < n; ++i) avail[i] = (uint8_t)i;
    int remaining = n;
#define LB(i) V3(c[i].lb[0], c[i].lb[1], c[i].lb[2])
    float deepest_depth = c[0].sep, shallowest = deepest_depth;
    int deepest = 0;
    for (int i = 1; i < remaining; ++i) {
        const float d = c[i].sep;
        shallowest = fmaxf_(shallowest, d);
        if (deepest_depth > d) { deepest_depth = d; deepest = i; }
    }
    sel[0] = (uint8_t)deepest;
    avail[deepest] = avail[--remaining];
    int fpos = 0;
    float far2 = vlen2(vsub(LB(avail[0]), LB(sel[0])));
    for (int i = 1; i < remaining; ++i) {
        const float val = vlen2(vsub(LB(avail[i]), LB(sel[0])));
        if (val > far2) { far2 = val; fpos = i; }
    }
    sel[1] = avail[fpos];
    avail[fpos] = avail[--remaining];
    const v3 base = vsub(LB(sel[1]), LB(sel[0]));
    v3 tr = vcross(base, V3(c[sel[0]].nb[0], c[sel[0]].nb[1], c[sel[0]].nb[2]));
    const float tr2 = vlen2(tr);
    if (tr2 > 0.0f) {
        const float inv = 1.0f / sqrtf(tr2);
        tr = V3(tr.x * inv, tr.y * inv, tr.z * inv);
    } else {
        tr = V3(c[sel[0]].nb[0], c[sel[0]].nb[1], c[sel[0]].nb[2]);
    }
    float greatest = -FLT_MAX, least = FLT_MAX;
    int gpos = 0, lpos = 0;
    for (int i = 0; i < remaining; ++i) {
        const float side = vdot(vsub(LB(avail[i]), LB(sel[0])), tr);
        if (side > greatest) { greatest = side; gpos = i; }
        if (side < least) { least = side; lpos = i; }
    }
    sel[2] = avail[gpos];
    avail[gpos] = avail[--remaining];
    if (lpos == remaining) lpos = gpos;
    if (least * greatest > 0.0f) {
        greatest = -FLT_MAX;
        for (int i = 0; i < remaining; ++i) {
            const float side = vdot(vsub(LB(avail[i]), LB(sel[0])), tr);
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
                    const uint8_t t = sel[i];
                    sel[i] = avail[rep];
                    avail[rep] = t;
                }
            }
        }
    }
#undef LB
    return 0;
}

/* ---------------- GJK / EPA (GuPCMGjkEpa.cpp:44-570) ----------------------
 * One pair of finite shapes in B's frame: boxes (extents), sphere point
 * cores (radius > 0; the radius is applied after the search) and cooked
 * hulls (extreme-vertex supports, scale-relative facet admission). */
typedef struct { v3 a, b, q; uint32_t ai, bi; } sup_t;
typedef struct {
    v3 ha, hb, a_in_b; qt rel;
    const float* va; uint32_t nva;
    const float* vb; uint32_t nvb;
    float ra, rb;
} bpair_t;
static int bp_hull(const bpair_t* p) { return p->nva > 0 || p->nvb > 0; }
static v3 box_vertex(v3 e, v3 d, uint32_t* idx) {
    const int x = d.x > 0.f, y = d.y > 0.f, z = d.z > 0.f;
    *idx = (x ? 1u : 0u) | (y ? 2u : 0u) | (z ? 4u : 0u);
    return V3(x ? e.x : -e.x, y ? e.y : -e.y, z ? e.z : -e.z);
}
/* GuPCMGjkEpa.cpp:53-75 BoxPair::vertex: a point core is its centre; a hull
 * returns its first vertex of largest projection. */
static v3 shape_vertex(v3 e, v3 d, const float* hull, uint32_t n, float radius, uint32_t* idx) {
    *idx = 0;
    if (radius > 0.f) return V3(0, 0, 0);
    if (n) {
        float best = vdot(V3(hull[0], hull[1], hull[2]), d);
        for (uint32_t i = 1; i < n; ++i) {
            const float pr = vdot(V3(hull[3 * i], hull[3 * i + 1], hull[3 * i + 2]), d);
            if (pr > best) { best = pr; *idx = i; }
        }
        return V3(hull[3 * *idx], hull[3 * *idx + 1], hull[3 * *idx + 2]);
    }
    return box_vertex(e, d, idx);
}
static sup_t bp_support(const bpair_t* p, v3 dir) {
    sup_t s;
    const v3 da = rotinv_gu(p->rel, dir);
    const v3 pa = shape_vertex(p->ha, da, p->va, p->nva, p->ra, &s.ai);
    s.b = shape_vertex(p->hb, vneg(dir), p->vb, p->nvb, p->rb, &s.bi);
    s.a = vadd(p->a_in_b, rot_gu(p->rel, pa));
    s.q = vsub(s.a, s.b);
    return s;
}
static v3 bp_local_a(const bpair_t* p, v3 pb) { return rotinv_gu(p->rel, vsub(pb, p->a_in_b)); }
static float box_min_margin(v3 h) { return 0.05f * fminf_(fminf_(h.x, h.y), h.z); }
static int solve_small(int n, float a[3][4], float r[3]) {
    float scale = 0.0f;
    for (int i = 0; i < n; ++i) scale = fmaxf_(scale, fabsf(a[i][i]));
    if (!(scale > 0.0f) || !isfinite(scale)) return 0;
    const float tol = FLT_EPSILON * scale;
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int row = col + 1; row < n; ++row)
            if (fabsf(a[row][col]) > fabsf(a[piv][col])) piv = row;
        if (!(fabsf(a[piv][col]) > tol)) return 0;
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
    return 1;
}
typedef struct { v3 point, a, b; float w[4]; unsigned mask; float dist2; } closest_t;
static closest_t closest_simplex(const sup_t* s, int count) {
    closest_t best;
    memset(&best, 0, sizeof best);
    best.dist2 = FLT_MAX;
    for (unsigned mask = 1; mask < (1u << count); ++mask) {
        int ids[4] = {0, 0, 0, 0}, n = 0;
        for (int i = 0; i < count; ++i)
            if (mask & (1u << i)) ids[n++] = i;
        float w[4] = {0, 0, 0, 0};
        w[ids[0]] = 1.0f;
        if (n > 1) {
            const v3 base = s[ids[0]].q;
            v3 dirs[3];
            float m[3][4];
            memset(m, 0, sizeof m);
            for (int i = 1; i < n; ++i) dirs[i - 1] = vsub(s[ids[i]].q, base);
            for (int i = 1; i < n; ++i) {
                for (int j = 1; j < n; ++j) m[i - 1][j - 1] = vdot(dirs[i - 1], dirs[j - 1]);
                m[i - 1][n - 1] = -vdot(dirs[i - 1], base);
            }
            float coef[3] = {0, 0, 0};
            if (!solve_small(n - 1, m, coef)) continue;
            for (int i = 1; i < n; ++i) {
                w[ids[i]] = coef[i - 1];
                w[ids[0]] -= coef[i - 1];
            }
        }
        int feasible = 1;
        for (int i = 0; i < n; ++i)
            if (w[ids[i]] < -1.0e-5f) feasible = 0;
        if (!feasible) continue;
        v3 q = V3(0, 0, 0), pa = V3(0, 0, 0), pb = V3(0, 0, 0);
        for (int i = 0; i < count; ++i) {
            q = vadd(q, vmul(s[i].q, w[i]));
            pa = vadd(pa, vmul(s[i].a, w[i]));
            pb = vadd(pb, vmul(s[i].b, w[i]));
        }
        const float d = vlen2(q);
        if (d < best.dist2) {
            best.point = q; best.a = pa; best.b = pb;
            memcpy(best.w, w, sizeof w);
            best.mask = mask; best.dist2 = d;
        }
    }
    return best;
}
static void compact_simplex(sup_t* s, int* count, const closest_t* c) {
    int write = 0;
    for (int read = 0; read < *count; ++read)
        if ((c->mask & (1u << read)) && c->w[read] > 1.0e-6f) s[write++] = s[read];
    if (write == 0 && *count > 0) write = 1;
    *count = write;
}
static int contact_from_gjk(const bpair_t* p, const closest_t* n, fo_candidate* out) {
    const float dist = sqrtf(n->dist2);
    if (!(dist > 0.0f) || !isfinite(dist)) return 0;
    const v3 normal = vmul(n->point, 1.0f / dist);
    const v3 la = bp_local_a(p, n->a);
    out->la[0] = la.x; out->la[1] = la.y; out->la[2] = la.z;
    out->lb[0] = n->b.x; out->lb[1] = n->b.y; out->lb[2] = n->b.z;
    out->nb[0] = normal.x; out->nb[1] = normal.y; out->nb[2] = normal.z;
    out->sep = dist;
    return 1;
}
typedef struct { int i, j, k; v3 normal; float distance; int valid, in_heap; } facet_t;
static facet_t make_facet(const bpair_t* p, const sup_t* vtx, int i, int j, int k) {
    facet_t f;
    memset(&f, 0, sizeof f);
    const v3 a = vtx[i].q, b = vtx[j].q, c = vtx[k].q;
    const v3 e0 = vsub(b, a), e1 = vsub(c, a);
    v3 n = vcross(e0, e1);
    const float norm2 = vlen2(n);
    float min_area = FLT_EPSILON;
    if (bp_hull(p)) min_area *= vlen2(e0) * vlen2(e1);   /* GuPCMGjkEpa.cpp:210-213 */
    if (!(norm2 > min_area)) return f;
    n = vmul(n, 1.0f / sqrtf(norm2));
    f.i = i; f.j = j; f.k = k; f.normal = n; f.distance = vdot(n, a);
    f.valid = 1; f.in_heap = 1;
    return f;
}
static int init_epa(const bpair_t* p, sup_t* vtx, int* count, facet_t* facets, int* fc) {
    if (*count <= 0 || *count > 4) return 0;
    if (*count == 1) {
        const sup_t nx = bp_support(p, V3(1, 0, 0));
        if (vlen2(vsub(nx.q, vtx[0].q)) == 0.0f) return 0;
        vtx[(*count)++] = nx;
    }
    if (*count == 2) {
        const v3 edge = vsub(vtx[1].q, vtx[0].q);
        const v3 ab = V3(fabsf(edge.x), fabsf(edge.y), fabsf(edge.z));
        v3 axis = V3(1, 0, 0);
        if (ab.x > ab.y && ab.z > ab.y) axis = V3(0, 1, 0);
        else if (ab.x > ab.z) axis = V3(0, 0, 1);
        v3 perp = vcross(axis, edge);
        const float sq = vlen2(perp);
        if (!(sq > 0.0f)) return 0;
        perp = vmul(perp, 1.0f / sqrtf(sq));
        vtx[(*count)++] = bp_support(p, perp);
    }
    if (*count == 3) {
        const facet_t f0 = make_facet(p, vtx, 0, 1, 2), f1 = make_facet(p, vtx, 1, 0, 2);
        if (!f0.valid || !f1.valid) return 0;
        facets[(*fc)++] = f0;
        facets[(*fc)++] = f1;
        return 1;
    }
    const v3 p0 = vtx[0].q;
    const v3 v1 = vsub(vtx[1].q, p0), v2 = vsub(vtx[2].q, p0);
    if (vdot(vcross(v1, v2), vsub(vtx[3].q, p0)) > 0.0f) {
        const sup_t t = vtx[1]; vtx[1] = vtx[2]; vtx[2] = t;
    }
    static const int faces[4][3] = {{0, 1, 2}, {0, 3, 1}, {0, 2, 3}, {1, 3, 2}};
    for (int i = 0; i < 4; ++i) {
        const facet_t f = make_facet(p, vtx, faces[i][0], faces[i][1], faces[i][2]);
        if (!f.valid) return 0;
        facets[(*fc)++] = f;
    }
    return 1;
}
static int contact_from_facet(const bpair_t* p, const sup_t* vtx, const facet_t* f,
                              fo_candidate* out) {
    const sup_t* P = &vtx[f->i];
    const sup_t* Qv = &vtx[f->j];
    const sup_t* R = &vtx[f->k];
    const v3 e0 = vsub(Qv->q, P->q), e1 = vsub(R->q, P->q);
    const float a = vdot(e0, e0), b = vdot(e0, e1), c = vdot(e1, e1);
    const float den = a * c - b * b;
    if (!(den > FLT_EPSILON * a * c)) return 0;
    const float x = -vdot(P->q, e0), y = -vdot(P->q, e1);
    const float u = (x * c - y * b) / den;
    const float v = (y * a - x * b) / den;
    const float w = 1.0f - u - v;
    const v3 pa = vadd(vadd(vmul(P->a, w), vmul(Qv->a, u)), vmul(R->a, v));
    const v3 pb = vadd(vadd(vmul(P->b, w), vmul(Qv->b, u)), vmul(R->b, v));
    if (!isfinite(pa.x) || !isfinite(pb.x) || !isfinite(f->distance)) return 0;
    const v3 normal = vneg(f->normal);
    const float depth = fabsf(f->distance);
    const v3 la = bp_local_a(p, pa);
    out->la[0] = la.x; out->la[1] = la.y; out->la[2] = la.z;
    out->lb[0] = pb.x; out->lb[1] = pb.y; out->lb[2] = pb.z;
    out->nb[0] = normal.x; out->nb[1] = normal.y; out->nb[2] = normal.z;
    out->sep = -depth;
    const v3 diff = vsub(pa, pb);
    const float scale = fmaxf_(fmaxf_(fmaxf_(p->ha.x, p->ha.y), fmaxf_(p->ha.z, p->hb.x)), fmaxf_(p->hb.y, p->hb.z));
    const float tol = bp_hull(p) ? 1.0e-3f * scale : 1.0e-3f;     /* GuPCMGjkEpa.cpp:297-301 */
    return sqrtf(vlen2(diff)) <= depth + tol;
}
static int run_epa(const bpair_t* p, const sup_t* simplex, int sc, fo_candidate* out) {
    sup_t vtx[64];
    int vc = sc;
    for (int i = 0; i < sc; ++i) vtx[i] = simplex[i];
    facet_t facets[64];
    int fc = 0;
    if (!init_epa(p, vtx, &vc, facets, &fc)) return 0;
    const float eps = 0.1f * fminf_(box_min_margin(p->ha), box_min_margin(p->hb));
    int bfrom[32], bto[32];
    float upper = FLT_MAX;
    for (int it = 0; it < 60; ++it) {
        int closest = -1;
        float dist = FLT_MAX;
        for (int i = 0; i < fc; ++i)
            if (facets[i].valid && facets[i].in_heap && facets[i].distance < dist) {
                closest = i;
                dist = facets[i].distance;
            }
        if (closest < 0) return 0;
        const facet_t sel = facets[closest];
        const sup_t np = bp_support(p, sel.normal);
        const float proj = vdot(np.q, sel.normal);
        if (fabsf(proj - dist) <= eps) return contact_from_facet(p, vtx, &sel, out);
        if (vc == 64) return 0;
        upper = fminf_(upper, proj);
        for (int i = 0; i < vc; ++i)
            if (vtx[i].ai == np.ai && vtx[i].bi == np.bi) return contact_from_facet(p, vtx, &sel, out);
        const int ni = vc++;
        vtx[ni] = np;
        int bc = 0;
        for (int i = 0; i < fc; ++i) {
            facet_t* f = &facets[i];
            if (!f->valid) continue;
            if (vdot(f->normal, vsub(np.q, vtx[f->i].q)) < 0.0f) continue;
            f->valid = 0;
            const int ef[3] = {f->i, f->j, f->k}, et[3] = {f->j, f->k, f->i};
            for (int e = 0; e < 3; ++e) {
                int rev = -1;
                for (int j = 0; j < bc; ++j)
                    if (bfrom[j] == et[e] && bto[j] == ef[e]) { rev = j; break; }
                if (rev >= 0) {
                    --bc;
                    bfrom[rev] = bfrom[bc];
                    bto[rev] = bto[bc];
                } else {
                    if (bc == 32) return 0;
                    bfrom[bc] = ef[e];
                    bto[bc] = et[e];
                    ++bc;
                }
            }
        }
        if (bc == 0) return 0;
        int avail = 64 - fc;
        for (int i = 0; i < fc; ++i) avail += !facets[i].valid;
        if (bc > avail) return 0;
        for (int i = 0; i < bc; ++i) {
            facet_t f = make_facet(p, vtx, bfrom[i], bto[i], ni);
            if (!f.valid) return 0;
            f.in_heap = f.distance <= upper;
            int slot = -1;
            for (int j = 0; j < fc; ++j)
                if (!facets[j].valid) { slot = j; break; }
            if (slot < 0) slot = fc++;
            facets[slot] = f;
        }
    }
    return 0;
}
/* GuPCMGjkEpa.cpp:411-516 gjk_epa.  A sphere point core converges its
 * separated distance before EPA is admitted. */
static int gjk_epa(const bpair_t* p, float cd, fo_candidate* out) {
    const float eps = 0.1f * fminf_(box_min_margin(p->ha), box_min_margin(p->hb));
    const float progress = 1.0f - 0.000225f;
    const int point_core = p->ra > 0.f || p->rb > 0.f;
    sup_t simplex[4];
    int count = 0;
    v3 closest = vlen2(p->a_in_b) > 0.0f ? p->a_in_b : V3(1, 0, 0);
    float previous = FLT_MAX;
    for (int it = 0; it < 32; ++it) {
        const float dist = sqrtf(vlen2(closest));
        if (count > 0 && dist <= eps && !point_core) return run_epa(p, simplex, count, out);
        if (dist <= 0.0f) {
            if (!point_core || count == 0) return 0;
            return run_epa(p, simplex, count, out);
        }
        const v3 normal = vmul(closest, 1.0f / dist);
        const sup_t s = bp_support(p, vneg(closest));
        const float proj = vdot(normal, s.q);
        if (proj > cd) return 0;
        if (count > 0 && proj > dist * progress) {
            const closest_t cur = closest_simplex(simplex, count);
            return cur.mask && contact_from_gjk(p, &cur, out);
        }
        for (int i = 0; i < count; ++i)
            if (s.ai == simplex[i].ai && s.bi == simplex[i].bi) {
                if (proj > 0.f) {
                    const closest_t cur = closest_simplex(simplex, count);
                    return cur.mask && contact_from_gjk(p, &cur, out) && out->sep <= cd;
                }
                return point_core && run_epa(p, simplex, count, out);
            }
        if (count == 4) return run_epa(p, simplex, count, out);
        simplex[count++] = s;
        const closest_t nx = closest_simplex(simplex, count);
        if (!nx.mask) return 0;
        closest = nx.point;
        const float nd = sqrtf(nx.dist2);
        compact_simplex(simplex, &count, &nx);
        if (nd >= previous) {
            if (point_core) {
                if (proj > 0.f) return contact_from_gjk(p, &nx, out);
                return run_epa(p, simplex, count, out);
            }
            return 0;
        }
        previous = nd;
    }
    if (point_core && count > 0) return run_epa(p, simplex, count, out);
    return 0;
}
/* GuPCMGjkEpa.cpp:517-568 source_pcm_box_box_gjk_epa (box/box, no radii). */
int fo_pcm_box_box_gjk_epa(const float* ra, const float* rb, float cd, fo_candidate* out) {
    const qt q0 = Q4(ra[6], ra[7], ra[8], ra[9]);
    const qt q1 = Q4(rb[6], rb[7], rb[8], rb[9]);
    bpair_t p;
    memset(&p, 0, sizeof p);
    p.ha = V3(ra[0], ra[1], ra[2]);
    p.hb = V3(rb[0], rb[1], rb[2]);
    p.a_in_b = rotinv_gu(q1, vsub(V3(ra[3], ra[4], ra[5]), V3(rb[3], rb[4], rb[5])));
    p.rel = qmul(qconj(q1), q0);
    memset(out, 0, sizeof *out);
    if (!gjk_epa(&p, cd, out)) return 0;
    return out->sep <= cd;
}

/* ---------------- sphere contacts (GuPCMContactSphere.cpp:49-130) -------- */
int fo_pcm_sphere_sphere(const float* c0, float r0, const float* c1, float r1,
                         float cd, fo_point* out) {
    const v3 a = V3(c0[0], c0[1], c0[2]), b = V3(c1[0], c1[1], c1[2]);
    const v3 delta = vsub(a, b);
    const float d2 = vdot(delta, delta);
    const float rs = r0 + r1;
    const float infl = rs + cd;
    if (!(infl * infl > d2)) return 0;
    const float dist = sqrtf(d2);
    const v3 n = dist <= 0.00001f ? V3(1, 0, 0) : vmul(delta, 1.0f / dist);
    const v3 p = vadd(b, vmul(n, r1));
    out->p[0] = p.x; out->p[1] = p.y; out->p[2] = p.z;
    out->n[0] = n.x; out->n[1] = n.y; out->n[2] = n.z;
    out->sep = dist - rs;
    return 1;
}
int fo_pcm_sphere_plane(const float* c, float r, float plane_h, float cd, fo_point* out) {
    const float sep = c[1] - plane_h - r;
    if (!(cd >= sep)) return 0;
    out->p[0] = c[0]; out->p[1] = c[1] - r; out->p[2] = c[2];
    out->n[0] = 0.f; out->n[1] = 1.f; out->n[2] = 0.f;
    out->sep = sep;
    return 1;
}
int fo_pcm_sphere_box(const float* cs, float r, const float* box, float cd, fo_point* out) {
    const v3 center = V3(cs[0], cs[1], cs[2]);
    const v3 h = V3(box[0], box[1], box[2]);
    const v3 bc = V3(box[3], box[4], box[5]);
    const qt bq = Q4(box[6], box[7], box[8], box[9]);
    const v3 local = rotinv_gu(bq, vsub(center, bc));
    const v3 cl = V3(fclamp(local.x, -h.x, h.x), fclamp(local.y, -h.y, h.y), fclamp(local.z, -h.z, h.z));
    const v3 gap = vsub(local, cl);
    const float l2 = vdot(gap, gap);
    const float infl = r + cd;
    if (!(infl * infl > l2)) return 0;
    const int inside = fabsf(local.x) <= h.x && fabsf(local.y) <= h.y && fabsf(local.z) <= h.z;
    v3 p, n;
    float sep;
    if (inside) {
        const v3 d = V3(h.x - fabsf(cl.x), h.y - fabsf(cl.y), h.z - fabsf(cl.z));
        v3 nl;
        float depth;
        if (d.z <= d.x && d.z <= d.y) {
            nl = V3(0, 0, cl.z >= 0.f ? 1.f : -1.f); depth = d.z;
        } else if (d.x <= d.y && d.x <= d.z) {
            nl = V3(cl.x >= 0.f ? 1.f : -1.f, 0, 0); depth = d.x;
        } else {
            nl = V3(0, cl.y >= 0.f ? 1.f : -1.f, 0); depth = d.y;
        }
        n = rot_gu(bq, nl);
        p = vadd(center, vmul(n, depth));
        sep = -depth - r;
    } else {
        const float len = sqrtf(l2);
        n = rot_gu(bq, vmul(gap, 1.f / len));
        p = vadd(bc, rot_gu(bq, cl));
        sep = len - r;
    }
    out->p[0] = p.x; out->p[1] = p.y; out->p[2] = p.z;
    out->n[0] = n.x; out->n[1] = n.y; out->n[2] = n.z;
    out->sep = sep;
    return 1;
}

/* ---------------- persistent PCM manifolds ---------------- */
static v3 ptv(const float* f) { return V3(f[0], f[1], f[2]); }
static void setv(float* f, v3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }

/* scene.cpp:3432-3465 refresh_pcm_contact_points */
static void refresh_points(fo_pcm_cache* c, v3 pa_in_b, qt ra_in_b, float brk) {
    const float brk2 = brk * brk;
    for (int i = c->count; i > 0; --i) {
        fo_candidate* pt = &c->pts[i - 1];
        const v3 rr = rot_sc(ra_in_b, ptv(pt->la));
        const v3 lab = V3(pa_in_b.x + rr.x, pa_in_b.y + rr.y, pa_in_b.z + rr.z);
        const v3 nb = ptv(pt->nb), lb = ptv(pt->lb);
        const v3 v = V3(lab.x - lb.x, lab.y - lb.y, lab.z - lb.z);
        const float dist = v.x * nb.x + v.y * nb.y + v.z * nb.z;
        const v3 pd = V3(v.x - nb.x * dist, v.y - nb.y * dist, v.z - nb.z * dist);
        const float t2 = pd.x * pd.x + pd.y * pd.y + pd.z * pd.z;
        if (t2 > brk2) c->pts[i - 1] = c->pts[--c->count];
        else pt->sep = dist;
    }
}

/* scene.cpp:3319-3431 reduce_pcm_box_five */
static float seg_sq(v3 p, v3 a, v3 b) {
    const v3 ab = vsub(b, a), ap = vsub(p, a);
    const float den = vlen2(ab);
    const float t = den == 0.0f ? 0.0f : fclamp(vdot(ap, ab) / den, 0.0f, 1.0f);
    const v3 d = V3(ap.x - t * ab.x, ap.y - t * ab.y, ap.z - t * ab.z);
    return vlen2(d);
}
static float tri_sq(v3 p, v3 a, v3 b, v3 c) {
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
    const v3 n = V3(ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x);
    const float den = vlen2(n);
    if (den == 0.0f) return 0.0f;
    const float pr = vdot(n, ap);
    return pr * pr / den;
}
static void reduce_five(fo_pcm_cache* c, const fo_candidate* nw) {
    fo_candidate cand[5];
    int chosen[5] = {0, 0, 0, 0, 0}, sel[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) cand[i] = c->pts[i];
    cand[4] = *nw;
#define LBC(i) ptv(cand[i].lb)
    int deepest = 4;
    for (int i = 0; i < 4; ++i)
        if (cand[i].sep < cand[deepest].sep) deepest = i;
    sel[0] = deepest;
    chosen[deepest] = 1;
    int farthest = 0;
    float largest = vlen2(vsub(LBC(0), LBC(deepest)));
    for (int i = 1; i < 5; ++i)
        if (!chosen[i]) {
            const float v = vlen2(vsub(LBC(i), LBC(deepest)));
            if (v > largest) { largest = v; farthest = i; }
        }
    sel[1] = farthest;
    chosen[farthest] = 1;
    largest = -FLT_MAX;
    int third = 0;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) {
            const float v = seg_sq(LBC(i), LBC(deepest), LBC(farthest));
            if (v > largest) { largest = v; third = i; }
        }
    sel[2] = third;
    chosen[third] = 1;
    largest = -FLT_MAX;
    int fourth = third;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) {
            const float v = tri_sq(LBC(i), LBC(sel[0]), LBC(sel[1]), LBC(sel[2]));
            if (v > largest) { largest = v; fourth = i; }
        }
    if (chosen[fourth]) {
        c->count = 3;
        for (int i = 0; i < 3; ++i) c->pts[i] = cand[sel[i]];
        return;
    }
    sel[3] = fourth;
    chosen[fourth] = 1;
    for (int i = 0; i < 4; ++i) c->pts[i] = cand[sel[i]];
    c->count = 4;
    int un = -1;
    for (int i = 0; i < 5; ++i)
        if (!chosen[i]) { un = i; break; }
    if (un < 0) return;
    float closest = FLT_MAX;
    int rep = 0;
    for (int i = 0; i < 4; ++i) {
        const float d = vlen2(vsub(ptv(c->pts[i].la), ptv(cand[un].la)));
        if (d < closest) { closest = d; rep = i; }
    }
    if (cand[un].sep < c->pts[rep].sep) c->pts[rep] = cand[un];
#undef LBC
}

static float pcm_box_margin(v3 h) {
    return fminf_(0.15f * fminf_(fminf_(h.x, h.y), h.z), 0.15f);
}

/* scene.cpp:3466-3654 generate_pcm_box_box.  first/second are the
 * Gu-ordered shapes: half(3) position(3) orientation(4). */
int fo_generate_pcm_box_box(const float* first, const float* second, float cd,
                            fo_pcm_cache* cache, fo_point out[4]) {
    const v3 h0 = ptv(first), h1 = ptv(second);
    const v3 p0 = ptv(first + 3), p1 = ptv(second + 3);
    const qt q0 = Q4(first[6], first[7], first[8], first[9]);
    const qt q1 = Q4(second[6], second[7], second[8], second[9]);
    const v3 delta = V3(p0.x - p1.x, p0.y - p1.y, p0.z - p1.z);
    const v3 relative = rotinv_sc(q1, delta);
    const qt rotation = qmul(qconj(q1), q0);
    const float mm = fminf_(pcm_box_margin(h0), pcm_box_margin(h1));
    const int initial = cache->count;
    refresh_points(cache, relative, rotation, mm * 0.8f);
    const int lost = cache->count != initial;
    static const float thr[5] = {0.5f, 0.125f, 0.25f, 0.375f, 0.375f};
    static const float qthr[5] = {0.9998f, 0.9999f, 0.9999f, 0.9999f, 0.9999f};
    float tdelta = INFINITY;
    if (cache->initialized)
        tdelta = fmaxf_(fmaxf_(fabsf(relative.x - cache->rel_p[0]), fabsf(relative.y - cache->rel_p[1])),
                        fabsf(relative.z - cache->rel_p[2]));
    const float qa = qdot(q0, Q4(cache->qa[0], cache->qa[1], cache->qa[2], cache->qa[3]));
    const float qb = qdot(q1, Q4(cache->qb[0], cache->qb[1], cache->qb[2], cache->qb[3]));
    const float tp = mm * thr[cache->count];
    int regen = !cache->initialized || lost || tdelta > tp || qa < qthr[cache->count] ||
                qb < qthr[cache->count];
    if (!regen) {
        const float ang0 = qa < 1.0f ? acosf(fmaxf_(-1.0f, qa)) : 0.0f;
        const float ang1 = qb < 1.0f ? acosf(fmaxf_(-1.0f, qb)) : 0.0f;
        regen = ang0 * sqrtf(h0.x * h0.x + h0.y * h0.y + h0.z * h0.z) > tp ||
                ang1 * sqrtf(h1.x * h1.x + h1.y * h1.y + h1.z * h1.z) > tp;
    }
    int direct = 0, gjk = 0;
    v3 gjk_n = V3(0, 0, 0);
    if (regen) {
        setv(cache->rel_p, relative);
        cache->rel_q[0] = rotation.x; cache->rel_q[1] = rotation.y;
        cache->rel_q[2] = rotation.z; cache->rel_q[3] = rotation.w;
        cache->qa[0] = q0.x; cache->qa[1] = q0.y; cache->qa[2] = q0.z; cache->qa[3] = q0.w;
        cache->qb[0] = q1.x; cache->qb[1] = q1.y; cache->qb[2] = q1.z; cache->qb[3] = q1.w;
        cache->initialized = 1;
        fo_candidate cands[64];
        int count = 0;
        const int ov = fo_pcm_box_box_candidates(first, second, cd, cands, 64, &count);
        if (ov < 0) return FO_OVERFLOW_NEG;
        if (!ov) {
            cache->count = 0;
            return 0;
        }
        if (count == 0) {
            fo_candidate w;
            if (!fo_pcm_box_box_gjk_epa(first, second, cd, &w)) {
                cache->count = 0;
                return 0;
            }
            gjk = 1;
            gjk_n = ptv(w.nb);
            const float rb = mm * 0.05f;
            const float rsq = rb * rb;
            int replaced = 0;
            for (int i = 0; i < cache->count; ++i) {
                const fo_candidate* o = &cache->pts[i];
                if (fminf_(vlen2(vsub(ptv(o->la), ptv(w.la))), vlen2(vsub(ptv(o->lb), ptv(w.lb)))) < rsq) {
                    cache->pts[i] = w;
                    replaced = 1;
                    break;
                }
            }
            if (!replaced) {
                if (cache->count < 4) cache->pts[cache->count++] = w;
                else reduce_five(cache, &w);
            }
        } else if (count <= 4) {
            for (int i = 0; i < count; ++i) cache->pts[i] = cands[i];
            cache->count = (uint8_t)count;
        } else {
            uint8_t sel[4];
            fo_pcm_batch_selection(cands, count, 1.0f, sel);
            for (int i = 0; i < 4; ++i) cache->pts[i] = cands[sel[i]];
            cache->count = 4;
        }
        direct = count > 0;
    }
    if (cache->count == 0) return 0;
    v3 nb = V3(0, 0, 0);
    if (gjk) nb = gjk_n;
    else if (direct) nb = ptv(cache->pts[0].nb);
    else
        for (int i = 0; i < cache->count; ++i) {
            nb.x += cache->pts[i].nb[0];
            nb.y += cache->pts[i].nb[1];
            nb.z += cache->pts[i].nb[2];
        }
    const float nsq = nb.x * nb.x + nb.y * nb.y + nb.z * nb.z;
    if (!(nsq > 0.0f) || !isfinite(nsq)) return FO_OVERFLOW_NEG;
    const float il = 1.0f / sqrtf(nsq);
    const v3 nn = V3(nb.x * il, nb.y * il, nb.z * il);
    const v3 normal = rot_sc(q1, nn);
    int emitted = 0;
    for (int i = 0; i < cache->count; ++i) {
        const fo_candidate* p = &cache->pts[i];
        if (!direct && p->sep > cd) continue;
        const v3 r = rot_sc(q1, ptv(p->lb));
        fo_point* o = &out[emitted++];
        o->p[0] = r.x + p1.x; o->p[1] = r.y + p1.y; o->p[2] = r.z + p1.z;
        o->n[0] = normal.x; o->n[1] = normal.y; o->n[2] = normal.z;
        o->sep = p->sep;
    }
    return emitted;
}

/* scene.cpp:3774-3955 generate_pcm_plane_box.  plane: position(3);
 * box: half(3) position(3) orientation(4).  Emits the raw plane-first
 * normal (0,-1,0); the scene flips plane manifolds afterwards. */
/* Candidates are the box corners, or a cooked hull's vertices in vertex
 * order (scene.cpp:3826-3846). */
static int plane_generate(const float* plane_p, v3 h, v3 bp, qt q, const fo_mesh* hull, float cd,
                          fo_pcm_cache* cache, fo_point out[4]) {
    const v3 rel = V3(bp.x - plane_p[0], bp.y - plane_p[1], bp.z - plane_p[2]);
    const float margin = pcm_box_margin(h);
    const float brk = margin * 0.2f;
    const int prev = cache->count;
    refresh_points(cache, rel, q, brk);
    float md = INFINITY;
    if (cache->initialized)
        md = fmaxf_(fmaxf_(fabsf(rel.x - cache->rel_p[0]), fabsf(rel.y - cache->rel_p[1])),
                    fabsf(rel.z - cache->rel_p[2]));
    const float rd = q.x * cache->rel_q[0] + q.y * cache->rel_q[1] + q.z * cache->rel_q[2] +
                     q.w * cache->rel_q[3];
    const int regen = !cache->initialized || cache->count != prev || md > brk || rd < 0.99996f;
    if (regen) {
        setv(cache->rel_p, rel);
        cache->rel_q[0] = q.x; cache->rel_q[1] = q.y; cache->rel_q[2] = q.z; cache->rel_q[3] = q.w;
        cache->initialized = 1;
        cache->count = 0;
        const unsigned nc = hull ? hull->nv : 8u;
        fo_candidate* cands = (fo_candidate*)malloc(sizeof(fo_candidate) * nc);
        int* chosen = (int*)calloc(nc, sizeof(int));
        int n = 0;
        for (unsigned corner = 0; corner < nc; ++corner) {
            const v3 local = hull ? V3(hull->verts[3 * corner], hull->verts[3 * corner + 1], hull->verts[3 * corner + 2])
                                  : V3((corner & 4u) ? -h.x : h.x, (corner & 2u) ? -h.y : h.y,
                                       (corner & 1u) ? -h.z : h.z);
            const v3 r = rot_sc(q, local);
            const v3 ip = V3(rel.x + r.x, rel.y + r.y, rel.z + r.z);
            if (ip.y >= cd) continue;
            fo_candidate* c = &cands[n++];
            setv(c->la, local);
            c->lb[0] = ip.x; c->lb[1] = 0.0f; c->lb[2] = ip.z;
            c->nb[0] = 0.0f; c->nb[1] = 1.0f; c->nb[2] = 0.0f;
            c->sep = ip.y;
        }
        if (n <= 4) {
            for (int i = 0; i < n; ++i) cache->pts[i] = cands[i];
            cache->count = (uint8_t)n;
        } else {
            int idx[4];
            int first = 0;
            for (int i = 1; i < n; ++i)
                if (cands[i].sep < cands[first].sep) first = i;
            idx[0] = first;
            chosen[first] = 1;
            int far = 0;
            float maxd = vlen2(vsub(ptv(cands[0].lb), ptv(cands[first].lb)));
            for (int i = 1; i < n; ++i) {
                const float d = vlen2(vsub(ptv(cands[i].lb), ptv(cands[first].lb)));
                if (d > maxd) { maxd = d; far = i; }
            }
            idx[1] = far;
            chosen[far] = 1;
            const v3 seg = vsub(ptv(cands[far].lb), ptv(cands[first].lb));
            v3 side = V3(-seg.z, 0.0f, seg.x);
            const float ns = vlen2(side);
            if (ns > 0.0f) {
                const float inv = 1.0f / sqrtf(ns);
                side = V3(side.x * inv, 0.0f, side.z * inv);
            } else {
                side = V3(0.0f, 1.0f, 0.0f);
            }
            float largest = -FLT_MAX, smallest = FLT_MAX;
            int third = 0, fourth = 0;
            for (int i = 0; i < n; ++i) {
                if (chosen[i]) continue;
                const float d = vdot(vsub(ptv(cands[i].lb), ptv(cands[first].lb)), side);
                if (d > largest) { largest = d; third = i; }
                if (d < smallest) { smallest = d; fourth = i; }
            }
            idx[2] = third;
            chosen[third] = 1;
            if (smallest * largest > 0.0f) {
                largest = -FLT_MAX;
                for (int i = 0; i < n; ++i) {
                    if (chosen[i]) continue;
                    const float d = vdot(vsub(ptv(cands[i].lb), ptv(cands[first].lb)), side);
                    if (d > largest) { largest = d; fourth = i; }
                }
            }
            idx[3] = fourth;
            chosen[fourth] = 1;
            fo_candidate centers[4];
            for (int k = 0; k < 4; ++k) centers[k] = cands[idx[k]];
            for (int i = 0; i < n; ++i) {
                if (chosen[i]) continue;
                float nearest = FLT_MAX;
                int slot = 0;
                for (int j = 0; j < 4; ++j) {
                    const float d = vlen2(vsub(ptv(cands[i].lb), ptv(centers[j].lb)));
                    if (d < nearest) { nearest = d; slot = j; }
                }
                if (cands[i].sep < cands[idx[slot]].sep) idx[slot] = i;
            }
            for (int k = 0; k < 4; ++k) cache->pts[k] = cands[idx[k]];
            cache->count = 4;
        }
        free(cands);
        free(chosen);
    }
    int emitted = 0;
    for (int k = 0; k < cache->count; ++k) {
        const fo_candidate* pt = &cache->pts[k];
        if (pt->sep > cd) continue;
        fo_point* o = &out[emitted++];
        o->p[0] = plane_p[0] + pt->lb[0]; o->p[1] = plane_p[1]; o->p[2] = plane_p[2] + pt->lb[2];
        o->n[0] = 0.0f; o->n[1] = -1.0f; o->n[2] = 0.0f;
        o->sep = pt->sep;
    }
    return emitted;
}

int fo_generate_pcm_plane_box(const float* plane_p, const float* box, float cd,
                              fo_pcm_cache* cache, fo_point out[4]) {
    return plane_generate(plane_p, ptv(box), ptv(box + 3), Q4(box[6], box[7], box[8], box[9]), NULL, cd, cache, out);
}
int fo_generate_pcm_plane_convex(const float* plane_p, const float* shape_half, const float* pose7,
                                 const fo_mesh* hull, float cd, fo_pcm_cache* cache, fo_point out[4]) {
    return plane_generate(plane_p, ptv(shape_half), ptv(pose7), Q4(pose7[3], pose7[4], pose7[5], pose7[6]), hull, cd,
                          cache, out);
}

/* ---------------- cooked convex hulls ---------------- */
/* scene.cpp:1258-1298: the world AABB of the rotated hull vertices, centred
 * where the hull is, plus the contact offset. */
int fo_convex_bounds(const float* pose7, const fo_mesh* hull, float contact_offset, uint32_t* out6) {
    const v3 p = V3(pose7[0], pose7[1], pose7[2]);
    const qt q = Q4(pose7[3], pose7[4], pose7[5], pose7[6]);
    v3 lo = V3(INFINITY, INFINITY, INFINITY), hi = V3(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t i = 0; i < hull->nv; ++i) {
        const v3 r = rot_sc(q, V3(hull->verts[3 * i], hull->verts[3 * i + 1], hull->verts[3 * i + 2]));
        lo = V3(fminf_(lo.x, r.x), fminf_(lo.y, r.y), fminf_(lo.z, r.z));
        hi = V3(fmaxf_(hi.x, r.x), fmaxf_(hi.y, r.y), fmaxf_(hi.z, r.z));
    }
    const v3 c = V3((hi.x + lo.x) * 0.5f, (hi.y + lo.y) * 0.5f, (hi.z + lo.z) * 0.5f);
    const v3 e = V3((hi.x - lo.x) * 0.5f, (hi.y - lo.y) * 0.5f, (hi.z - lo.z) * 0.5f);
    const v3 add = V3(e.x + contact_offset, e.y + contact_offset, e.z + contact_offset);
    const float b[6] = {p.x + c.x - add.x, p.y + c.y - add.y, p.z + c.z - add.z,
                        p.x + c.x + add.x, p.y + c.y + add.y, p.z + c.z + add.z};
    for (int i = 0; i < 6; ++i)
        if (!isfinite(b[i])) return FO_OVERFLOW;
    for (int a = 0; a < 3; ++a) {
        out6[a] = fo_encode_min(b[a]);
        out6[a + 3] = fo_encode_max(b[a + 3]);
    }
    return 0;
}

static void setcand(fo_candidate* c, v3 la, v3 lb, v3 nb, float sep) {
    setv(c->la, la); setv(c->lb, lb); setv(c->nb, nb); c->sep = sep;
}

/* GuPCMGjkEpa.cpp:528-569 source_pcm_convex_gjk_epa */
int fo_pcm_convex_gjk_epa(const fo_finite* a, const fo_finite* b, float cd, fo_candidate* out) {
    const qt qb = Q4(b->q[0], b->q[1], b->q[2], b->q[3]);
    const qt q0 = Q4(a->q[0], a->q[1], a->q[2], a->q[3]);
    bpair_t p;
    memset(&p, 0, sizeof p);
    p.ha = ptv(a->half);
    p.hb = ptv(b->half);
    p.a_in_b = rotinv_gu(qb, vsub(ptv(a->p), ptv(b->p)));
    p.rel = qmul(qconj(qb), q0);
    if (a->hull) { p.va = a->hull->verts; p.nva = a->hull->nv; }
    if (b->hull) { p.vb = b->hull->verts; p.nvb = b->hull->nv; }
    p.ra = a->radius;
    p.rb = b->radius;
    memset(out, 0, sizeof *out);
    if (!gjk_epa(&p, cd + a->radius + b->radius, out)) return 0;
    if (a->radius > 0.f) {
        const v3 off = rotinv_gu(p.rel, vmul(ptv(out->nb), -a->radius));
        setv(out->la, vadd(ptv(out->la), off));
        out->sep -= a->radius;
    }
    if (b->radius > 0.f) {
        setv(out->lb, vadd(ptv(out->lb), vmul(ptv(out->nb), b->radius)));
        out->sep -= b->radius;
    }
    return out->sep <= cd;
}

/* Face geometry of a finite shape: a hull's planar polygons or the six box
 * faces (GuPCMGjkEpa.cpp:580-621). */
static const v3 kAxis[3] = {{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}};
static unsigned face_count(const fo_finite* s) { return s->hull ? s->hull->nf : 6u; }
static v3 face_normal(const fo_finite* s, unsigned f) {
    if (s->hull) return ptv(s->hull->faces[f].n);
    return vmul(kAxis[f / 2u], (f & 1u) ? 1.f : -1.f);
}
static unsigned vertex_count(const fo_finite* s, unsigned f) { return s->hull ? s->hull->faces[f].count : 4u; }
static v3 vertex_local(const fo_finite* s, unsigned f, unsigned k) {
    if (s->hull) {
        const uint32_t v = s->hull->idx[s->hull->faces[f].first + k];
        return V3(s->hull->verts[3 * v], s->hull->verts[3 * v + 1], s->hull->verts[3 * v + 2]);
    }
    static const float corners[4][2] = {{1.f, 1.f}, {-1.f, 1.f}, {-1.f, -1.f}, {1.f, -1.f}};
    const v3 n = face_normal(s, f);
    const unsigned c = f / 2u;
    const v3 u = kAxis[(c + 1u) % 3u];
    const v3 v = vcross(n, u);
    const v3 h = ptv(s->half);
    const float hu = vcomp(h, (c + 1u) % 3u), hv = vcomp(h, (c + 2u) % 3u);
    return vadd(vmul(n, vcomp(h, c)), vadd(vmul(u, corners[k][0] * hu), vmul(v, corners[k][1] * hv)));
}
typedef struct {
    const fo_finite *a, *b;
    qt qa, qb;
    v3 pa, pb;
} fc_ctx;
static v3 fc_to_b(const fc_ctx* c, v3 p) { return rotinv_gu(c->qb, vsub(vadd(c->pa, rot_gu(c->qa, p)), c->pb)); }
static v3 fc_vertex(const fc_ctx* c, const fo_finite* s, int is_a, unsigned f, unsigned k) {
    const v3 l = vertex_local(s, f, k);
    return is_a ? fc_to_b(c, l) : l;
}
static v3 fc_normal_b(const fc_ctx* c, const fo_finite* s, int is_a, unsigned f) {
    const v3 n = face_normal(s, f);
    return is_a ? rotinv_gu(c->qb, rot_gu(c->qa, n)) : n;
}
typedef struct {
    const fc_ctx* c;
    const fo_finite *ref, *inc;
    int ref_is_a, inc_is_a, reference_b;
    unsigned rf, inf, nr, ni;
    v3 rn, anchor;
    float cd, tol_sq;
    fo_candidate* out;
    unsigned count;
} fc_clip;
static v3 fc_r(const fc_clip* k, unsigned i) { return fc_vertex(k->c, k->ref, k->ref_is_a, k->rf, i % k->nr); }
static v3 fc_q(const fc_clip* k, unsigned i) { return fc_vertex(k->c, k->inc, k->inc_is_a, k->inf, i % k->ni); }
static float fc_cross2(const fc_clip* k, v3 a, v3 b) { return vdot(k->rn, vcross(a, b)); }
/* GuPCMGjkEpa.cpp:710-765 emit: projected reference point, duplicate merge
 * and the greedy five-point reduction. */
static void fc_emit(fc_clip* k, v3 ip) {
    const float sep = vdot(k->rn, vsub(ip, k->anchor));
    if (!isfinite(sep) || sep > k->cd) return;
    const v3 proj = vsub(ip, vmul(k->rn, sep));
    const v3 a = k->reference_b ? ip : proj;
    const v3 b = k->reference_b ? proj : ip;
    const fc_ctx* c = k->c;
    const v3 al = rotinv_gu(c->qa, vsub(vadd(c->pb, rot_gu(c->qb, a)), c->pa));
    fo_candidate cand;
    setcand(&cand, al, b, k->reference_b ? k->rn : vneg(k->rn), sep);
    if (!isfinite(al.x) || !isfinite(b.x)) return;
    for (unsigned i = 0; i < k->count; ++i)
        if (vlen2(vsub(ptv(k->out[i].lb), ptv(cand.lb))) <= k->tol_sq) {
            if (cand.sep < k->out[i].sep) k->out[i] = cand;
            return;
        }
    if (k->count < 4u) {
        k->out[k->count++] = cand;
        return;
    }
    fo_candidate ch[5] = {k->out[0], k->out[1], k->out[2], k->out[3], cand};
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
                if (j != ex) score += vlen2(vsub(ptv(ch[i].lb), ptv(ch[j].lb)));
        }
        if (score > best) { best = score; omit = ex; }
    }
    if (omit != 4u) k->out[omit] = cand;
}
/* GuPCMGjkEpa.cpp:571-804 source_pcm_convex_face_contacts */
int fo_pcm_convex_face_contacts(const fo_finite* a, const fo_finite* b, float cd,
                                const fo_candidate* witness, fo_candidate out[4]) {
    if (a->radius > 0.f || b->radius > 0.f || (a->hull && !a->hull->nf) || (b->hull && !b->hull->nf)) return 0;
    fc_ctx c = {a, b, Q4(a->q[0], a->q[1], a->q[2], a->q[3]), Q4(b->q[0], b->q[1], b->q[2], b->q[3]), ptv(a->p),
                ptv(b->p)};
    const v3 normal = ptv(witness->nb);
    if (!(vlen2(normal) > 0.f)) return 0;
    unsigned fa = 0, fb = 0;
    float ala = -2.f, alb = -2.f;
    for (unsigned i = 0; i < face_count(a); ++i) {
        const float d = vdot(vneg(normal), fc_normal_b(&c, a, 1, i));
        if (d > ala) { ala = d; fa = i; }
    }
    for (unsigned i = 0; i < face_count(b); ++i) {
        const float d = vdot(normal, fc_normal_b(&c, b, 0, i));
        if (d > alb) { alb = d; fb = i; }
    }
    fc_clip k;
    memset(&k, 0, sizeof k);
    k.c = &c;
    k.reference_b = alb >= ala;
    if (fmaxf_(ala, alb) < 0.95f) return 0;
    k.ref = k.reference_b ? b : a;
    k.inc = k.reference_b ? a : b;
    k.ref_is_a = !k.reference_b;
    k.inc_is_a = k.reference_b;
    k.rf = k.reference_b ? fb : fa;
    k.rn = fc_normal_b(&c, k.ref, k.ref_is_a, k.rf);
    float ial = -2.f;
    for (unsigned i = 0; i < face_count(k.inc); ++i) {
        const float d = vdot(vneg(k.rn), fc_normal_b(&c, k.inc, k.inc_is_a, i));
        if (d > ial) { ial = d; k.inf = i; }
    }
    const v3 in_n = fc_normal_b(&c, k.inc, k.inc_is_a, k.inf);
    const float den = vdot(in_n, k.rn);
    if (!(den < -0.25f)) return 0;
    k.nr = vertex_count(k.ref, k.rf);
    k.ni = vertex_count(k.inc, k.inf);
    if (k.nr < 3u || k.ni < 3u) return 0;
    k.anchor = fc_r(&k, 0);
    const v3 in_anchor = fc_q(&k, 0);
    float el = 0.f;
    for (unsigned i = 0; i < k.nr; ++i) el = fmaxf_(el, vlen2(vsub(fc_r(&k, i + 1), fc_r(&k, i))));
    for (unsigned i = 0; i < k.ni; ++i) el = fmaxf_(el, vlen2(vsub(fc_q(&k, i + 1), fc_q(&k, i))));
    const float scale = sqrtf(el);
    if (!(scale > 0.f) || !isfinite(scale)) return 0;
    const float tol = fmaxf_(scale * 1.e-5f, 1.e-6f);
    const float ftol = tol / scale;
    k.tol_sq = tol * tol;
    k.cd = cd;
    k.out = out;
    for (unsigned i = 0; i < k.ni; ++i) {
        const v3 v = fc_q(&k, i);
        int inside = 1;
        for (unsigned j = 0; j < k.nr && inside; ++j)
            if (fc_cross2(&k, vsub(fc_r(&k, j + 1), fc_r(&k, j)), vsub(v, fc_r(&k, j))) < -tol * scale) inside = 0;
        if (inside) fc_emit(&k, v);
    }
    for (unsigned i = 0; i < k.nr; ++i) {
        const v3 v = fc_r(&k, i);
        int inside = 1;
        for (unsigned j = 0; j < k.ni && inside; ++j)
            if (fc_cross2(&k, vsub(fc_q(&k, j + 1), fc_q(&k, j)), vsub(v, fc_q(&k, j))) > tol * scale) inside = 0;
        if (!inside) continue;
        const float height = vdot(in_n, vsub(in_anchor, v)) / den;
        if (isfinite(height)) fc_emit(&k, vadd(v, vmul(k.rn, height)));
    }
    for (unsigned i = 0; i < k.ni; ++i) {
        const v3 qa = fc_q(&k, i), e = vsub(fc_q(&k, i + 1), qa);
        for (unsigned j = 0; j < k.nr; ++j) {
            const v3 rb = fc_r(&k, j), f = vsub(fc_r(&k, j + 1), rb);
            const float det = fc_cross2(&k, e, f);
            if (fabsf(det) <= k.tol_sq) continue;
            const v3 d = vsub(rb, qa);
            const float t = fc_cross2(&k, d, f) / det;
            const float u = fc_cross2(&k, d, e) / det;
            if (t >= -ftol && t <= 1.f + ftol && u >= -ftol && u <= 1.f + ftol)
                fc_emit(&k, vadd(qa, vmul(e, fclamp(t, 0.f, 1.f))));
        }
    }
    return (int)k.count;
}

/* scene.cpp:3655-3772 Scene::generate_pcm_convex_pair */
static float finite_margin(const fo_finite* s) {
    float extent;
    if (s->radius > 0.f) extent = s->radius;
    else if (s->hull) extent = 0.5f * fminf_(fminf_(s->hull->hi[0] - s->hull->lo[0], s->hull->hi[1] - s->hull->lo[1]),
                                             s->hull->hi[2] - s->hull->lo[2]);
    else extent = fminf_(fminf_(s->half[0], s->half[1]), s->half[2]);
    return fminf_(0.15f * extent, 0.15f);
}
int fo_generate_pcm_convex_pair(const fo_finite* first, const float* first_shape_half,
                                const fo_finite* second, const float* second_shape_half, float cd,
                                fo_pcm_cache* cache, fo_point out[4]) {
    const qt q0 = Q4(first->q[0], first->q[1], first->q[2], first->q[3]);
    const qt q1 = Q4(second->q[0], second->q[1], second->q[2], second->q[3]);
    const v3 p0 = ptv(first->p), p1 = ptv(second->p);
    const v3 delta = V3(p0.x - p1.x, p0.y - p1.y, p0.z - p1.z);
    const v3 relative = rotinv_sc(q1, delta);
    const qt rotation = qmul(qconj(q1), q0);
    const float mm = fminf_(finite_margin(first), finite_margin(second));
    const int prev = cache->count;
    refresh_points(cache, relative, rotation, mm * 0.8f);
    const float tr = cache->initialized
        ? fmaxf_(fmaxf_(fabsf(relative.x - cache->rel_p[0]), fabsf(relative.y - cache->rel_p[1])),
                 fabsf(relative.z - cache->rel_p[2]))
        : INFINITY;
    const float qa = qdot(q0, Q4(cache->qa[0], cache->qa[1], cache->qa[2], cache->qa[3]));
    const float qb = qdot(q1, Q4(cache->qb[0], cache->qb[1], cache->qb[2], cache->qb[3]));
    const float thr = mm * (cache->count == 0 ? 0.5f : 0.125f);
    int regen = !cache->initialized || cache->count != prev || tr > thr || qa < 0.9999f || qb < 0.9999f;
    if (!regen) {
        const v3 ha = ptv(first_shape_half), hb = ptv(second_shape_half);
        const float ta = (qa < 1.f ? acosf(fmaxf_(-1.f, qa)) : 0.f) * sqrtf(ha.x * ha.x + ha.y * ha.y + ha.z * ha.z);
        const float tb = (qb < 1.f ? acosf(fmaxf_(-1.f, qb)) : 0.f) * sqrtf(hb.x * hb.x + hb.y * hb.y + hb.z * hb.z);
        regen = ta > thr || tb > thr;
    }
    if (regen) {
        setv(cache->rel_p, relative);
        cache->rel_q[0] = rotation.x; cache->rel_q[1] = rotation.y; cache->rel_q[2] = rotation.z; cache->rel_q[3] = rotation.w;
        memcpy(cache->qa, first->q, 16);
        memcpy(cache->qb, second->q, 16);
        cache->initialized = 1;
        cache->count = 0;
        fo_candidate w;
        if (fo_pcm_convex_gjk_epa(first, second, cd, &w)) {
            fo_candidate clipped[4];
            const int n = fo_pcm_convex_face_contacts(first, second, cd, &w, clipped);
            if (n) {
                for (int i = 0; i < n; ++i) cache->pts[i] = clipped[i];
                cache->count = (uint8_t)n;
            } else {
                cache->pts[0] = w;
                cache->count = 1;
            }
        }
    }
    int emitted = 0;
    for (int i = 0; i < cache->count; ++i) {
        const fo_candidate* pt = &cache->pts[i];
        if (pt->sep > cd) continue;
        const v3 n = rot_sc(q1, ptv(pt->nb));
        const v3 l = rot_sc(q1, ptv(pt->lb));
        fo_point* o = &out[emitted++];
        o->p[0] = p1.x + l.x; o->p[1] = p1.y + l.y; o->p[2] = p1.z + l.z;
        setv(o->n, n);
        o->sep = pt->sep;
        if (!vfinite(ptv(o->p)) || !vfinite(n) || !isfinite(o->sep)) return -1;
    }
    return emitted;
}
