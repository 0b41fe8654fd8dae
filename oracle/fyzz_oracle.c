/* Test infrastructure: C restatement of the reference NativeCpu rigid-body
 * step (src/native/scene.cpp, compound.cpp) for the configurations the B200
 * path supports: dynamic box / sphere / box+sphere compound bodies, one
 * static floor per scene, centre-anchored distance constraints, default
 * RigidBodyDynamics, PCM contacts.
 *
 * Deliberate scope limits (recorded in the design notes):
 *  - no island sleep / wake (scene.cpp:5119-6884): every dynamic body stays
 *    awake, which the reference also does until a whole island has been
 *    quiet for 0.4 s;
 *  - the Dy descriptor input order is either replayed from the reference
 *    or the canonical order (joints by constraint slot descending, then
 *    touching managers in shape-pair order).  Per-island greedy partitioning
 *    of that sequence is identical to the reference's per-task partitioning
 *    because islands share no dynamic body.
 */
#include "fyzz_oracle.h"
#include "fo_math.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

static __thread char g_err[256];
const char* fo_error(void) { return g_err; }
#define FAIL(code, ...) do { snprintf(g_err, sizeof g_err, __VA_ARGS__); return (code); } while (0)

typedef struct {
    int dynamic;
    v3 p, v, w;
    qt q;
    float inv_mass;
    v3 inv_inertia;
    v3 ml_p; qt ml_q;      /* mass_local_pose */
    float max_contact_impulse, max_depenetration, slop;
    float lin_damp, ang_damp, max_lin, max_ang;
    int pos_iters, vel_iters;
    /* sleep state (scene.h:1147-1156) */
    float wake;
    v3 lin_acc, ang_acc;
    int sleeping, ready;
    uint32_t counted, joints;
    /* kinematic body (scene.h Actor kinematic_target_*): target, a target
     * waiting for the step, set since the last step, settling after it */
    int kinematic, kin_pending, kin_new, kin_settling;
    v3 kp; qt kq;
} actor_t;
typedef struct {
    uint32_t body, type;
    v3 half; float radius;
    v3 lp; qt lq;
    v3 wp; qt wq;
    float sf, df, rest, damping;
    float contact_offset, rest_offset;
    uint32_t bounds[6];
    const fo_mesh* hull;       /* cooked hull of an FO_CONVEX shape */
} shape_t;
typedef struct {
    v3 body0_normal, body1_normal, normal;
    float sf, df, rest, damping;
    v3 a0[2], a1[2];
    v3 bmin, bmax;
    uint16_t contact_count;
    uint8_t anchor_count, broken;
    uint32_t row_offset;
} patch_t;
typedef struct {
    uint64_t key;              /* (a << 32) | b, canonical shape pair */
    int reversed;              /* gu_order_reversed (scene.cpp:3275-3283) */
    fo_pcm_cache cache;
    int touching;              /* published manifold count > 0 */
    uint8_t found_now;         /* overlap found this step */
    uint8_t new_touch;         /* touching now, not the step before */
    uint8_t count;
    fo_point pts[4];
    /* friction history (prepared in the previous step) */
    uint64_t fr_epoch;
    int fr_count;
    patch_t fr[2];
} mgr_t;
typedef struct {
    v3 n, ra, rb;
    float vel_mult, imp_mult, biased, unbiased, applied, max_impulse;
} crow_t;
typedef struct { v3 t, ra, rb; float vel_mult, bias, target, applied; } frow_t;
typedef struct {
    v3 axis, ang_a, ang_b;
    float ima, imb, constant, unbiased, vel_mult, applied;
} jrow_t;
typedef struct {
    v3 dv, dw;                  /* SolverBody linear delta / angular state */
    v3 mdv, mdw;                /* saved motion */
    v3 v, w, p; qt q;           /* SolverBodyData */
    float inv_mass;
    v3 sqrt_i[3];               /* columns */
    uint32_t mask; size_t max_dyn; size_t static_count;
    int admitted;
} srow_t;
struct fo_scene {
    uint32_t na, ns, nj;
    actor_t* actors;
    shape_t* shapes;
    uint32_t* joint_a; uint32_t* joint_b; float* joint_len;
    /* joint kind, authored endpoints and local frames (ConstraintRecord,
     * scene.h:1529-1545) */
    uint8_t* joint_kind; uint32_t* joint_auth; v3* joint_lp; qt* joint_lq;
    /* constraint slots (scene.cpp:3110-3140, 3195-3228): live flag,
     * generation, LIFO free list of retired slots; nj counts slots */
    uint8_t* joint_live; uint32_t* joint_gen; uint32_t* joint_free; uint32_t nfree, jcap;
    int has_floor;
    uint32_t plane_shape;
    /* pair state */
    mgr_t* mgr; uint64_t nmgr;
    uint64_t* found; uint64_t nfound;
    uint64_t* lost; uint64_t nlost;
    /* touching manifolds: indices into mgr */
    uint64_t* man; uint64_t nman;
    uint64_t frame, fr_epoch;
    /* last partition result */
    uint32_t* desc; uint64_t ndesc;
    uint64_t* pend; uint64_t npend;
    double* impulses; uint64_t nimp;
    uint32_t* sorted_minx_val; uint32_t* sorted_minx_id; uint64_t nsorted;
    int sleep;                 /* sleeping enabled */
    fo_mesh* meshes; uint32_t nmeshes;
};

/* ------------------------- setup ------------------------- */
static qt normalize_once(qt q) {
    const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    return Q4(q.x / len, q.y / len, q.z / len, q.w / len);
}
/* World::validated_transform (src/world.cpp:38-55) followed by the scene's
 * own Scene::validated_pose (src/native/compound.cpp:9-18): the public
 * path divides by the length twice. */
static qt normalize_q(const float* q) {
    return normalize_once(normalize_once(Q4(q[0], q[1], q[2], q[3])));
}
/* PxMat33(PxQuat): rotation matrix columns */
typedef struct { v3 c[3]; } m33;
static m33 m_from_q(qt q) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x2 * x, yy = y2 * y, zz = z2 * z;
    const float xy = x2 * y, xz = x2 * z, xw = x2 * w;
    const float yz = y2 * z, yw = y2 * w, zw = z2 * w;
    m33 m;
    m.c[0] = V3(1.0f - yy - zz, xy + zw, xz - yw);
    m.c[1] = V3(xy - zw, 1.0f - xx - zz, yz + xw);
    m.c[2] = V3(xz + yw, yz - xw, 1.0f - xx - yy);
    return m;
}
static float mel(const m33* m, int row, int col) { return vcomp(m->c[col], row); }
static m33 m_mul(m33 a, m33 b) {
    m33 r;
    for (int c = 0; c < 3; ++c) {
        const v3 bc = b.c[c];
        r.c[c] = vadd(vadd(vmul(a.c[0], bc.x), vmul(a.c[1], bc.y)), vmul(a.c[2], bc.z));
    }
    return r;
}
static m33 m_t(m33 a) {
    m33 r;
    r.c[0] = V3(a.c[0].x, a.c[1].x, a.c[2].x);
    r.c[1] = V3(a.c[0].y, a.c[1].y, a.c[2].y);
    r.c[2] = V3(a.c[0].z, a.c[1].z, a.c[2].z);
    return r;
}
static qt q_normalized(qt q) {
    const float m = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    const float s = 1.0f / m;
    return Q4(q.x * s, q.y * s, q.z * s, q.w * s);
}
/* Jacobi diagonalisation with quaternion rotations (S. Melax), as used by
 * compound.cpp:170 through the foundation's diagonalisation helper:
 * at most 24 sweeps, each rotating away the largest off-diagonal term. */
static v3 diagonalize(m33 m, qt* frame) {
    qt q = Q4(0, 0, 0, 1);
    m33 d = m;
    for (int it = 0; it < 24; ++it) {
        const m33 axes = m_from_q(q);
        d = m_mul(m_mul(m_t(axes), m), axes);
        const float d0 = fabsf(mel(&d, 2, 1)), d1 = fabsf(mel(&d, 2, 0)), d2 = fabsf(mel(&d, 1, 0));
        const int a = (d0 > d1 && d0 > d2) ? 0 : (d1 > d2 ? 1 : 2);
        const int a1 = (a + 1) % 3, a2 = (a1 + 1) % 3;
        const float off = mel(&d, a2, a1);
        if (off == 0.0f || fabsf(mel(&d, a1, a1) - mel(&d, a2, a2)) > 2e6f * fabsf(2.0f * off)) break;
        const float w = (mel(&d, a1, a1) - mel(&d, a2, a2)) / (2.0f * off);
        const float absw = fabsf(w);
        float v[3] = {0, 0, 0};
        float c;
        if (absw > 1000) {
            v[a] = 1.0f / (4.0f * w);
            c = 1.0f;
        } else {
            const float t = 1.0f / (absw + sqrtf(w * w + 1.0f));
            const float h = 1.0f / sqrtf(t * t + 1.0f);
            v[a] = sqrtf((1.0f - h) / 2.0f) * (w < 0 ? -1.0f : 1.0f);
            c = sqrtf((1.0f + h) / 2.0f);
        }
        q = q_normalized(qmul(q, Q4(v[0], v[1], v[2], c)));
    }
    *frame = q;
    return V3(d.c[0].x, d.c[1].y, d.c[2].z);
}
/* compound.cpp:113-203 Scene::update_mass_properties (box / sphere).
 * Shapes are visited in the body's shape-list order, which is the reverse
 * of attachment order (scene.cpp:240-243). */
static int update_mass(fo_scene* s, uint32_t body, const uint32_t* shape_ids, int n, float density) {
    actor_t* A = &s->actors[body];
    float mass = 0.0f;
    v3 center = V3(0, 0, 0);
    const float pi = 3.14159265358979323846f;
    float um[8];
    v3 lc[8];
    for (int k = n - 1, i = 0; k >= 0; --k, ++i) {
        const shape_t* sh = &s->shapes[shape_ids[k]];
        um[i] = sh->type == FO_BOX ? sh->half.x * sh->half.y * sh->half.z * 8.0f
              : sh->type == FO_CONVEX ? (float)sh->hull->volume
                                      : (4.0f / 3.0f) * pi * sh->radius * sh->radius * sh->radius;
        const float m = um[i] * density;
        mass += m;
        /* a hull's centre of mass sits away from its authoring origin */
        lc[i] = sh->type == FO_CONVEX ? vadd(sh->lp, rot_px(sh->lq, V3(sh->hull->center[0], sh->hull->center[1],
                                                                       sh->hull->center[2])))
                                      : sh->lp;
        center = vadd(center, vmul(lc[i], m));
    }
    if (!(mass > 0.0f) || !isfinite(mass)) FAIL(FO_INVALID, "Compound mass outside supported range");
    center = vmul(center, 1.0f / mass);
    m33 tensor;
    memset(&tensor, 0, sizeof tensor);
    for (int k = n - 1, i = 0; k >= 0; --k, ++i) {
        const shape_t* sh = &s->shapes[shape_ids[k]];
        const float m = um[i] * density;
        m33 local;
        memset(&local, 0, sizeof local);
        if (sh->type == FO_CONVEX) {
            const float* I = sh->hull->inertia;
            for (int c = 0; c < 3; ++c) local.c[c] = vmul(V3(I[3 * c], I[3 * c + 1], I[3 * c + 2]), density);
        } else {
            v3 diag;
            if (sh->type == FO_BOX) {
                const v3 h = sh->half;
                diag = vmul(V3(h.y * h.y + h.z * h.z, h.x * h.x + h.z * h.z, h.x * h.x + h.y * h.y), m / 3.0f);
            } else {
                const float v = (2.0f / 5.0f) * m * sh->radius * sh->radius;
                diag = V3(v, v, v);
            }
            local.c[0].x = diag.x; local.c[1].y = diag.y; local.c[2].z = diag.z;
        }
        const m33 rot = m_from_q(sh->lq);
        const m33 rt = m_mul(m_mul(rot, local), m_t(rot));
        const v3 d = vsub(lc[i], center);
        const float dd = vdot(d, d);
        for (int c = 0; c < 3; ++c) {
            tensor.c[c] = vadd(tensor.c[c], rt.c[c]);
            const float dc = vcomp(d, c);
            v3 pc = V3(-d.x * dc, -d.y * dc, -d.z * dc);
            if (c == 0) pc.x += dd; else if (c == 1) pc.y += dd; else pc.z += dd;
            tensor.c[c] = vadd(tensor.c[c], vmul(pc, m));
        }
    }
    qt axes;
    const v3 inertia = diagonalize(tensor, &axes);
    const v3 inv = V3(1.0f / inertia.x, 1.0f / inertia.y, 1.0f / inertia.z);
    A->inv_mass = 1.0f / mass;
    A->inv_inertia = inv;
    A->ml_p = center;
    A->ml_q = axes;
    return 0;
}

fo_scene* fo_scene_create(uint32_t nb, const float* bodies, uint32_t ns,
                          const uint32_t* shape_body, const uint32_t* shape_type,
                          const float* shape_geom, const float* shape_local,
                          const float* shape_mat, uint32_t nj,
                          const uint32_t* joint_bodies, const float* joint_dist,
                          int has_floor, float floor_height, const float* floor_mat) {
    return fo_scene_create_ex(nb, bodies, ns, shape_body, shape_type, shape_geom, shape_local, shape_mat, nj,
                              joint_bodies, joint_dist, has_floor, floor_height, floor_mat, 0, NULL, NULL, NULL, NULL);
}
fo_scene* fo_scene_create_ex(uint32_t nb, const float* bodies, uint32_t ns,
                             const uint32_t* shape_body, const uint32_t* shape_type,
                             const float* shape_geom, const float* shape_local,
                             const float* shape_mat, uint32_t nj,
                             const uint32_t* joint_bodies, const float* joint_dist,
                             int has_floor, float floor_height, const float* floor_mat,
                             uint32_t n_meshes, const uint32_t* mesh_nv, const float* mesh_verts,
                             const uint32_t* mesh_nt, const uint32_t* mesh_tris) {
    fo_scene* s = (fo_scene*)calloc(1, sizeof *s);
    s->meshes = (fo_mesh*)calloc(n_meshes + 1, sizeof(fo_mesh));
    s->nmeshes = n_meshes;
    for (uint32_t m = 0, vo = 0, to = 0; m < n_meshes; vo += mesh_nv[m], to += mesh_nt[m], ++m)
        if (fo_cook_convex(mesh_verts + 3ull * vo, mesh_nv[m], mesh_tris + 3ull * to, mesh_nt[m], &s->meshes[m])) {
            fo_scene_destroy(s);
            return NULL;
        }
    const uint32_t off = has_floor ? 1u : 0u;
    s->na = nb + off;
    s->ns = ns + off;
    s->nj = nj;
    s->has_floor = has_floor;
    s->actors = (actor_t*)calloc(s->na, sizeof(actor_t));
    s->shapes = (shape_t*)calloc(s->ns, sizeof(shape_t));
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        a->q = Q4(0, 0, 0, 1);
        a->ml_q = Q4(0, 0, 0, 1);
        a->max_contact_impulse = FLT_MAX;
        a->max_depenetration = 1.0e32f;
        a->lin_damp = 0.0f; a->ang_damp = 0.05f; a->max_lin = 1.0e16f; a->max_ang = 100.0f;
        a->pos_iters = 4; a->vel_iters = 1;
        a->wake = 0.4f;
    }
    s->sleep = 1;
    if (has_floor) {
        s->actors[0].p = V3(0, floor_height, 0);
        shape_t* f = &s->shapes[0];
        f->body = 0; f->type = FO_PLANE; f->lq = Q4(0, 0, 0, 1);
        f->wp = s->actors[0].p; f->wq = Q4(0, 0, 0, 1);
        f->sf = floor_mat ? floor_mat[0] : 0.5f;
        f->df = floor_mat ? floor_mat[1] : 0.5f;
        f->rest = floor_mat ? floor_mat[2] : 0.2f;
        f->contact_offset = 0.02f;
        s->plane_shape = 0;
    }
    uint32_t si = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const float* r = bodies + 14ull * b;
        actor_t* a = &s->actors[b + off];
        a->dynamic = 1;
        a->p = V3(r[0], r[1], r[2]);
        a->q = normalize_q(r + 3);
        a->inv_mass = 1.0f;
        a->inv_inertia = V3(1, 1, 1);
        uint32_t ids[8];
        int n = 0;
        while (si < ns && shape_body[si] == b) {
            shape_t* sh = &s->shapes[si + off];
            sh->body = b + off;
            sh->type = shape_type[si];
            const float* g = shape_geom + 4ull * si;
            sh->half = V3(g[0], g[1], g[2]);
            sh->radius = g[0];
            if (sh->type == FO_CONVEX) {
                /* Scene::attach_convex (scene.cpp:301-305): half extents
                 * are the larger absolute bound per axis */
                const uint32_t mi = (uint32_t)g[0];
                if (mi >= n_meshes) { fo_scene_destroy(s); return NULL; }
                sh->hull = &s->meshes[mi];
                const float* lo = sh->hull->lo;
                const float* hi = sh->hull->hi;
                sh->half = V3(fmaxf_(fabsf(lo[0]), fabsf(hi[0])), fmaxf_(fabsf(lo[1]), fabsf(hi[1])),
                              fmaxf_(fabsf(lo[2]), fabsf(hi[2])));
                sh->radius = 0.0f;
            }
            const float* l = shape_local + 7ull * si;
            sh->lp = V3(l[0], l[1], l[2]);
            sh->lq = normalize_q(l + 3);
            sh->sf = shape_mat[3 * si]; sh->df = shape_mat[3 * si + 1]; sh->rest = shape_mat[3 * si + 2];
            sh->contact_offset = 0.02f;
            if (n < 8) ids[n++] = si + off;
            ++si;
        }
        if (update_mass(s, b + off, ids, n, r[13])) { fo_scene_destroy(s); return NULL; }
        a->v = V3(r[7], r[8], r[9]);
        a->w = V3(r[10], r[11], r[12]);
    }
    s->joint_a = (uint32_t*)calloc(nj + 1, 4);
    s->joint_b = (uint32_t*)calloc(nj + 1, 4);
    s->joint_len = (float*)calloc(nj + 1, 4);
    s->joint_kind = (uint8_t*)calloc(nj + 1, 1);
    s->joint_auth = (uint32_t*)calloc(2 * nj + 2, 4);
    s->joint_lp = (v3*)calloc(2 * nj + 2, sizeof(v3));
    s->joint_lq = (qt*)calloc(2 * nj + 2, sizeof(qt));
    s->joint_live = (uint8_t*)calloc(nj + 1, 1);
    s->joint_gen = (uint32_t*)calloc(nj + 1, 4);
    s->joint_free = (uint32_t*)calloc(nj + 1, 4);
    s->jcap = nj + 1;
    for (uint32_t j = 0; j < nj; ++j) {
        s->joint_live[j] = 1;
        s->joint_gen[j] = 1;
        /* 0xffffffff names the floor (actor 0) */
        const uint32_t a = joint_bodies[2 * j] == 0xffffffffu ? 0u : joint_bodies[2 * j] + off;
        const uint32_t b = joint_bodies[2 * j + 1] == 0xffffffffu ? 0u : joint_bodies[2 * j + 1] + off;
        s->joint_a[j] = a < b ? a : b;   /* edge pair is ordered (scene.cpp:3154) */
        s->joint_b[j] = a < b ? b : a;
        s->joint_len[j] = joint_dist[j];
        s->joint_auth[2 * j] = a;
        s->joint_auth[2 * j + 1] = b;
        s->joint_lq[2 * j] = s->joint_lq[2 * j + 1] = Q4(0, 0, 0, 1);
        if (s->actors[a].dynamic) ++s->actors[a].joints;
        if (s->actors[b].dynamic) ++s->actors[b].joints;
    }
    return s;
}

/* World::add_*_constraint (src/world.cpp:231-276) and Scene::create_*
 * (scene.cpp:3046-3120): local frames validated and normalised twice; the
 * distance kinds keep the ordered body pair with the authored anchors
 * (scene.cpp:3097-3108); the other kinds keep the authored endpoint order
 * (record.swapped, scene.cpp:3050-3060). */
static int validated_q(const float* q4, qt* out) {
    qt q = Q4(q4[0], q4[1], q4[2], q4[3]);
    for (int pass = 0; pass < 2; ++pass) {
        const float len = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
        if (!isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z) || !isfinite(q.w) || !isfinite(len) ||
            fabsf(len - 1.0f) >= 1.0e-2f)
            return 0;
        q = Q4(q.x / len, q.y / len, q.z / len, q.w / len);
    }
    *out = q;
    return 1;
}
int fo_scene_set_joint(fo_scene* s, uint32_t j, uint32_t kind, const float* la, const float* lb) {
    if (j >= s->nj || kind > FO_JOINT_PRISMATIC) FAIL(FO_INVALID, "joint index or kind out of range");
    const float* l[2] = {la, lb};
    for (int k = 0; k < 2; ++k) {
        if (!isfinite(l[k][0]) || !isfinite(l[k][1]) || !isfinite(l[k][2])) FAIL(FO_INVALID, "Position must be finite");
        s->joint_lp[2 * j + k] = V3(l[k][0], l[k][1], l[k][2]);
        s->joint_lq[2 * j + k] = Q4(0, 0, 0, 1);
        if (kind >= FO_JOINT_FIXED && !validated_q(l[k] + 3, &s->joint_lq[2 * j + k]))
            FAIL(FO_INVALID, "Rigid pose orientation is not sane");
    }
    if (kind == FO_JOINT_CENTER) s->joint_lp[2 * j] = s->joint_lp[2 * j + 1] = V3(0, 0, 0);
    s->joint_kind[j] = (uint8_t)kind;
    const uint32_t a = s->joint_auth[2 * j], b = s->joint_auth[2 * j + 1];
    if (kind >= FO_JOINT_FIXED) {
        s->joint_a[j] = a;
        s->joint_b[j] = b;
    }
    return 0;
}
/* Scene::add_joint / create_*_constraint after creation (scene.cpp:3110-
 * 3140): the most recently retired slot is reused with its generation
 * bumped, else a new slot is appended; counted interactions follow. */
int fo_scene_add_joint(fo_scene* s, uint32_t kind, uint32_t a_in, uint32_t b_in, const float* la, const float* lb,
                       float dist, uint64_t* id_out) {
    const uint32_t off = s->has_floor ? 1u : 0u;
    const uint32_t a = a_in == 0xffffffffu ? 0u : a_in + off;
    const uint32_t b = b_in == 0xffffffffu ? 0u : b_in + off;
    if (kind > FO_JOINT_PRISMATIC || a >= s->na || b >= s->na || a == b) FAIL(FO_INVALID, "joint endpoints or kind");
    if (!s->actors[a].dynamic && !s->actors[b].dynamic)
        FAIL(FO_LOGIC, "Rigid constraint requires a dynamic solver node");
    uint32_t j;
    if (s->nfree) {
        j = s->joint_free[--s->nfree];
    } else {
        j = s->nj;
        if (j + 1 >= s->jcap) {
            const uint32_t cap = 2 * s->jcap + 4;
            s->joint_a = (uint32_t*)realloc(s->joint_a, 4ull * cap);
            s->joint_b = (uint32_t*)realloc(s->joint_b, 4ull * cap);
            s->joint_len = (float*)realloc(s->joint_len, 4ull * cap);
            s->joint_kind = (uint8_t*)realloc(s->joint_kind, cap);
            s->joint_auth = (uint32_t*)realloc(s->joint_auth, 8ull * cap);
            s->joint_lp = (v3*)realloc(s->joint_lp, 2 * sizeof(v3) * cap);
            s->joint_lq = (qt*)realloc(s->joint_lq, 2 * sizeof(qt) * cap);
            s->joint_live = (uint8_t*)realloc(s->joint_live, cap);
            s->joint_gen = (uint32_t*)realloc(s->joint_gen, 4ull * cap);
            s->joint_free = (uint32_t*)realloc(s->joint_free, 4ull * cap);
            s->jcap = cap;
        }
        s->joint_gen[j] = 0;
        ++s->nj;
    }
    s->joint_a[j] = a < b ? a : b;
    s->joint_b[j] = a < b ? b : a;
    s->joint_len[j] = dist;
    s->joint_kind[j] = FO_JOINT_CENTER;
    s->joint_auth[2 * j] = a;
    s->joint_auth[2 * j + 1] = b;
    s->joint_lp[2 * j] = s->joint_lp[2 * j + 1] = V3(0, 0, 0);
    s->joint_lq[2 * j] = s->joint_lq[2 * j + 1] = Q4(0, 0, 0, 1);
    s->joint_live[j] = 1;
    s->joint_gen[j] += 1;
    if (kind != FO_JOINT_CENTER) {
        const int rc = fo_scene_set_joint(s, j, kind, la, lb);
        if (rc) return rc;
    }
    if (s->actors[a].dynamic) ++s->actors[a].joints;
    if (s->actors[b].dynamic) ++s->actors[b].joints;
    if (id_out) *id_out = ((uint64_t)s->joint_gen[j] << 32) | j;
    return 0;
}
/* Scene::retire_constraint (scene.cpp:3088-3096, 3195-3228) */
int fo_scene_remove_joint(fo_scene* s, uint64_t id) {
    const uint32_t j = (uint32_t)id, gen = (uint32_t)(id >> 32);
    if (j >= s->nj || !gen || !s->joint_live[j] || s->joint_gen[j] != gen)
        FAIL(FO_INVALID, "Unknown or expired rigid constraint");
    s->joint_live[j] = 0;
    s->joint_free[s->nfree++] = j;
    const uint32_t a = s->joint_a[j], b = s->joint_b[j];
    if (s->actors[a].dynamic) --s->actors[a].joints;
    if (s->actors[b].dynamic) --s->actors[b].joints;
    return 0;
}
static uint32_t joint_rows(uint8_t kind) {
    return kind <= FO_JOINT_ANCHORED ? 1u : kind == FO_JOINT_SPHERICAL ? 3u : kind == FO_JOINT_FIXED ? 6u : 5u;
}

void fo_scene_destroy(fo_scene* s) {
    if (!s) return;
    free(s->actors); free(s->shapes); free(s->joint_a); free(s->joint_b); free(s->joint_len);
    free(s->joint_kind); free(s->joint_auth); free(s->joint_lp); free(s->joint_lq);
    free(s->joint_live); free(s->joint_gen); free(s->joint_free);
    free(s->mgr); free(s->found); free(s->lost); free(s->man); free(s->desc); free(s->pend);
    free(s->impulses); free(s->sorted_minx_val); free(s->sorted_minx_id);
    for (uint32_t m = 0; m < s->nmeshes; ++m) fo_mesh_free(&s->meshes[m]);
    free(s->meshes);
    free(s);
}

/* ------------------------- collision ------------------------- */
static v3 mass_position(const actor_t* a) { return vadd(a->p, rot_sc(a->q, a->ml_p)); }
static qt mass_orientation(const actor_t* a) { return qmul(a->q, a->ml_q); }

static int cmp_u64(const void* x, const void* y) {
    const uint64_t a = *(const uint64_t*)x, b = *(const uint64_t*)y;
    return a < b ? -1 : a > b;
}
typedef struct { uint32_t v, id; } ep_t;
static int cmp_ep(const void* x, const void* y) {
    const ep_t* a = (const ep_t*)x; const ep_t* b = (const ep_t*)y;
    if (a->v != b->v) return a->v < b->v ? -1 : 1;
    return a->id < b->id ? -1 : a->id > b->id;
}

/* Scene::update_bounds + update_pairs full sweep (scene.cpp:1336-1420,
 * 2564-2704): the overlap set of the encoded AABBs; planes pair with every
 * dynamic finite shape. */
static int build_pairs(fo_scene* s, uint64_t** out, uint64_t* nout) {
    for (uint32_t i = 0; i < s->ns; ++i) {
        shape_t* sh = &s->shapes[i];
        const actor_t* a = &s->actors[sh->body];
        sh->wp = vadd(a->p, rot_sc(a->q, sh->lp));      /* scene.cpp:366-371 */
        sh->wq = qmul(a->q, sh->lq);
        if (sh->type == FO_PLANE) continue;
        const float pose[7] = {sh->wp.x, sh->wp.y, sh->wp.z, sh->wq.x, sh->wq.y, sh->wq.z, sh->wq.w};
        const float geom[4] = {sh->half.x, sh->half.y, sh->half.z, 0};
        const float sg[4] = {sh->radius, 0, 0, 0};
        if (sh->type == FO_CONVEX) {
            if (fo_convex_bounds(pose, sh->hull, sh->contact_offset, sh->bounds))
                FAIL(FO_OVERFLOW, "Convex scene AABB is not finite");
        } else if (fo_shape_bounds(sh->type, pose, sh->type == FO_SPHERE ? sg : geom, sh->contact_offset, sh->bounds))
            FAIL(FO_OVERFLOW, "Native scene AABB is not finite");
    }
    ep_t* ep = (ep_t*)malloc(sizeof(ep_t) * (s->ns + 1));
    uint64_t n = 0;
    for (uint32_t i = 0; i < s->ns; ++i)
        if (s->shapes[i].type != FO_PLANE) { ep[n].v = s->shapes[i].bounds[0]; ep[n].id = i; ++n; }
    qsort(ep, n, sizeof(ep_t), cmp_ep);
    free(s->sorted_minx_val); free(s->sorted_minx_id);
    s->sorted_minx_val = (uint32_t*)malloc(4 * (n + 1));
    s->sorted_minx_id = (uint32_t*)malloc(4 * (n + 1));
    s->nsorted = n;
    for (uint64_t i = 0; i < n; ++i) { s->sorted_minx_val[i] = ep[i].v; s->sorted_minx_id[i] = ep[i].id; }
    uint64_t cap = 1024, np = 0;
    uint64_t* pairs = (uint64_t*)malloc(8 * cap);
#define PUSH(k) do { if (np == cap) { cap *= 2; pairs = (uint64_t*)realloc(pairs, 8 * cap); } pairs[np++] = (k); } while (0)
    for (uint64_t i = 0; i < n; ++i) {
        const uint32_t ai = ep[i].id;
        const shape_t* A = &s->shapes[ai];
        const uint32_t* a = A->bounds;
        for (uint64_t j = i + 1; j < n && ep[j].v <= a[3]; ++j) {
            const uint32_t bi = ep[j].id;
            const shape_t* B = &s->shapes[bi];
            const uint32_t* b = B->bounds;
            if (A->body == B->body) continue;
            if (!s->actors[A->body].dynamic && !s->actors[B->body].dynamic) continue;
            if (a[1] > b[4] || b[1] > a[4] || a[2] > b[5] || b[2] > a[5]) continue;
            const uint32_t lo = ai < bi ? ai : bi, hi = ai < bi ? bi : ai;
            PUSH(((uint64_t)lo << 32) | hi);
        }
    }
    for (uint32_t p = 0; p < s->ns; ++p) {
        if (s->shapes[p].type != FO_PLANE) continue;
        for (uint64_t i = 0; i < n; ++i) {
            const uint32_t v = ep[i].id;
            if (!s->actors[s->shapes[v].body].dynamic) continue;
            const uint32_t lo = p < v ? p : v, hi = p < v ? v : p;
            PUSH(((uint64_t)lo << 32) | hi);
        }
    }
#undef PUSH
    free(ep);
    qsort(pairs, np, 8, cmp_u64);
    uint64_t u = 0;
    for (uint64_t i = 0; i < np; ++i)
        if (u == 0 || pairs[u - 1] != pairs[i]) pairs[u++] = pairs[i];
    *out = pairs;
    *nout = u;
    return 0;
}

static void shape_record(const shape_t* sh, float out[10]) {
    out[0] = sh->half.x; out[1] = sh->half.y; out[2] = sh->half.z;
    out[3] = sh->wp.x; out[4] = sh->wp.y; out[5] = sh->wp.z;
    out[6] = sh->wq.x; out[7] = sh->wq.y; out[8] = sh->wq.z; out[9] = sh->wq.w;
}
/* The PcmFiniteShape descriptor of scene.cpp:3712-3731: spheres carry their
 * radius, hulls the half size of their vertex bounds. */
static void finite_of(const shape_t* sh, fo_finite* f) {
    memset(f, 0, sizeof *f);
    f->half[0] = sh->half.x; f->half[1] = sh->half.y; f->half[2] = sh->half.z;
    if (sh->type == FO_SPHERE) {
        f->radius = sh->radius;
        f->half[0] = f->half[1] = f->half[2] = sh->radius;
    }
    if (sh->type == FO_CONVEX) {
        f->hull = sh->hull;
        for (int k = 0; k < 3; ++k) f->half[k] = 0.5f * (sh->hull->hi[k] - sh->hull->lo[k]);
    }
    f->p[0] = sh->wp.x; f->p[1] = sh->wp.y; f->p[2] = sh->wp.z;
    f->q[0] = sh->wq.x; f->q[1] = sh->wq.y; f->q[2] = sh->wq.z; f->q[3] = sh->wq.w;
}

/* Scene::publish_pairs + update_contacts, CPU Gu path (scene.cpp:3230-3304,
 * 4012-4758): carry each surviving manager's persistent PCM cache, generate
 * manifolds in pair order and publish touch transitions. */
static int collide(fo_scene* s) {
    uint64_t* pairs = NULL;
    uint64_t np = 0;
    int rc = build_pairs(s, &pairs, &np);
    if (rc) return rc;
    mgr_t* nm = (mgr_t*)calloc(np + 1, sizeof(mgr_t));
    free(s->found); free(s->lost);
    s->found = (uint64_t*)malloc(8 * (np + 1));
    s->lost = (uint64_t*)malloc(8 * (s->nmgr + 1));
    s->nfound = s->nlost = 0;
    uint64_t o = 0, k = 0;
    while (o < s->nmgr || k < np) {
        if (k == np || (o < s->nmgr && s->mgr[o].key < pairs[k])) {
            s->lost[s->nlost++] = s->mgr[o].key;
            ++o;
        } else if (o == s->nmgr || pairs[k] < s->mgr[o].key) {
            mgr_t* m = &nm[k];
            m->key = pairs[k];
            const shape_t* A = &s->shapes[(uint32_t)(pairs[k] >> 32)];
            const shape_t* B = &s->shapes[(uint32_t)pairs[k]];
            const int a_static = !s->actors[A->body].dynamic;
            const int both = s->actors[A->body].dynamic && s->actors[B->body].dynamic;
            m->reversed = a_static || (both && A->body < B->body);
            m->found_now = 1;
            s->found[s->nfound++] = pairs[k];
            ++k;
        } else {
            nm[k] = s->mgr[o];
            nm[k].found_now = 0;
            ++o; ++k;
        }
    }
    free(pairs);
    free(s->mgr);
    s->mgr = nm;
    s->nmgr = np;
    free(s->man);
    s->man = (uint64_t*)malloc(8 * (np + 1));
    s->nman = 0;
    for (uint64_t i = 0; i < np; ++i) {
        mgr_t* m = &s->mgr[i];
        const shape_t* A = &s->shapes[(uint32_t)(m->key >> 32)];
        const shape_t* B = &s->shapes[(uint32_t)m->key];
        const float cd = A->contact_offset + B->contact_offset;
        const int plane = A->type == FO_PLANE || B->type == FO_PLANE;
        /* cooked hulls take the PCM plane or convex generator, whatever the
         * other shape is (scene.cpp:4307-4317) */
        const int convex = A->type == FO_CONVEX || B->type == FO_CONVEX;
        const int sphere = !convex && (A->type == FO_SPHERE || B->type == FO_SPHERE);
        const shape_t* first = plane ? (A->type == FO_PLANE ? A : B) : (m->reversed ? B : A);
        const shape_t* second = plane ? (A->type == FO_PLANE ? B : A) : (m->reversed ? A : B);
        int count = 0;
        fo_point pts[4];
        if (plane && !sphere) {
            float box[10];
            shape_record(second, box);
            const float pp[3] = {first->wp.x, first->wp.y, first->wp.z};
            if (second->type == FO_CONVEX)
                count = fo_generate_pcm_plane_convex(pp, box, box + 3, second->hull, cd, &m->cache, pts);
            else
                count = fo_generate_pcm_plane_box(pp, box, cd, &m->cache, pts);
        } else if (!plane && convex) {
            fo_finite f0, f1;
            finite_of(first, &f0);
            finite_of(second, &f1);
            const float h0[3] = {first->type == FO_SPHERE ? 0.f : first->half.x, first->type == FO_SPHERE ? 0.f : first->half.y,
                                 first->type == FO_SPHERE ? 0.f : first->half.z};
            const float h1[3] = {second->type == FO_SPHERE ? 0.f : second->half.x,
                                 second->type == FO_SPHERE ? 0.f : second->half.y,
                                 second->type == FO_SPHERE ? 0.f : second->half.z};
            count = fo_generate_pcm_convex_pair(&f0, h0, &f1, h1, cd, &m->cache, pts);
        } else if (!plane && !sphere) {
            float r0[10], r1[10];
            shape_record(first, r0);
            shape_record(second, r1);
            count = fo_generate_pcm_box_box(r0, r1, cd, &m->cache, pts);
        } else {
            const shape_t* sp = A->type == FO_SPHERE ? A : B;
            const float c[3] = {sp->wp.x, sp->wp.y, sp->wp.z};
            if (plane) {
                count = fo_pcm_sphere_plane(c, sp->radius, first->wp.y, cd, pts);
                if (count) { pts[0].n[0] = -pts[0].n[0]; pts[0].n[1] = -pts[0].n[1]; pts[0].n[2] = -pts[0].n[2]; }
            } else if (A->type == FO_SPHERE && B->type == FO_SPHERE) {
                const float c0[3] = {first->wp.x, first->wp.y, first->wp.z};
                const float c1[3] = {second->wp.x, second->wp.y, second->wp.z};
                count = fo_pcm_sphere_sphere(c0, first->radius, c1, second->radius, cd, pts);
            } else {
                const shape_t* bx = A->type == FO_BOX ? A : B;
                float box[10];
                shape_record(bx, box);
                count = fo_pcm_sphere_box(c, sp->radius, box, cd, pts);
                if (count && first->type == FO_BOX) {
                    pts[0].n[0] = -pts[0].n[0]; pts[0].n[1] = -pts[0].n[1]; pts[0].n[2] = -pts[0].n[2];
                }
            }
        }
        if (count < 0) FAIL(FO_OVERFLOW, "PCM generation overflow");
        if (plane)
            for (int j = 0; j < count; ++j) {
                pts[j].n[0] = -pts[j].n[0]; pts[j].n[1] = -pts[j].n[1]; pts[j].n[2] = -pts[j].n[2];
            }
        m->count = (uint8_t)count;
        memcpy(m->pts, pts, sizeof(fo_point) * (size_t)count);
        m->new_touch = count > 0 && !m->touching;
        m->touching = count > 0;
        if (count > 0) s->man[s->nman++] = i;
    }
    ++s->frame;
    return 0;
}

int fo_scene_advance_collision(fo_scene* s) { return collide(s); }

/* ------------------------- dynamics ------------------------- */
/* scene.cpp:10383-10507 prepare_unconstrained_velocities */
/* scene.cpp:2005-2043 calculate_kinematic_velocities */
static void kinematic_velocities(fo_scene* s, float inv_dt) {
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->kinematic) continue;
        if (!a->kin_pending) { a->v = V3(0, 0, 0); a->w = V3(0, 0, 0); continue; }
        const v3 off = rot_sc(a->kq, a->ml_p);
        const v3 target = V3(a->kp.x + off.x, a->kp.y + off.y, a->kp.z + off.z);
        const v3 center = mass_position(a);
        a->v = V3((target.x - center.x) * inv_dt, (target.y - center.y) * inv_dt, (target.z - center.z) * inv_dt);
        qt rel = qmul(a->kq, qconj(a->q));
        if (rel.w < 0.0f) rel = Q4(-rel.x, -rel.y, -rel.z, -rel.w);
        const float len = sqrtf(rel.x * rel.x + rel.y * rel.y + rel.z * rel.z);
        if (len > 0.0f) {
            const float angle = 2.0f * atan2f(len, rel.w);
            const float scale = angle * inv_dt / len;
            a->w = V3(rel.x * scale, rel.y * scale, rel.z * scale);
        } else {
            a->w = V3(0, 0, 0);
        }
    }
}
static void pre_integrate(fo_scene* s, float dt) {
    const float gravity = -9.81f;
    kinematic_velocities(s, 1.0f / dt);
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->dynamic || a->sleeping) continue;
        float vx = a->v.x, vy = a->v.y + gravity * dt, vz = a->v.z;
        const float lm = fmaxf_(1.0f - a->lin_damp * dt, 0.0f);
        vx *= lm; vy *= lm; vz *= lm;
        v3 w = a->w;
        const float am = fmaxf_(1.0f - a->ang_damp * dt, 0.0f);
        w.x *= am; w.y *= am; w.z *= am;
        const float s2 = vx * vx + vy * vy + vz * vz;
        const float ml2 = a->max_lin * a->max_lin, ma2 = a->max_ang * a->max_ang;
        if (s2 > ml2) {
            const float f = sqrtf(ml2 / s2);
            vx *= f; vy *= f; vz *= f;
        }
        const float w2 = w.x * w.x + w.y * w.y + w.z * w.z;
        if (w2 > ma2) {
            const float f = sqrtf(ma2 / w2);
            w.x *= f; w.y *= f; w.z *= f;
        }
        a->v = V3(vx, vy, vz);
        a->w = w;
    }
}
/* scene.cpp:114-143 integrate_quaternion */
static qt integrate_q(qt pose, v3 w, float dt) {
    float m = w.x * w.x + w.y * w.y + w.z * w.z;
    if (m != 0.0f) {
        m = sqrtf(m);
        if (m > 1.0e7f) {
            const float sc = 1.0e7f / m;
            w = V3(w.x * sc, w.y * sc, w.z * sc);
            m = 1.0e7f;
        }
        const float v = dt * m * 0.5f;
        const float sn = sinf(v) / m;
        const float cs = cosf(v);
        const qt dq = qmul(Q4(w.x * sn, w.y * sn, w.z * sn, 0.0f), pose);
        const qt nx = Q4(dq.x + pose.x * cs, dq.y + pose.y * cs, dq.z + pose.z * cs, dq.w + pose.w * cs);
        const float len = sqrtf(nx.x * nx.x + nx.y * nx.y + nx.z * nx.z + nx.w * nx.w);
        pose = Q4(nx.x / len, nx.y / len, nx.z / len, nx.w / len);
    }
    return pose;
}
static v3 xform(const srow_t* d, v3 v) {
    const v3* c = d->sqrt_i;
    return V3(c[0].x * v.x + c[1].x * v.y + c[2].x * v.z,
              c[0].y * v.x + c[1].y * v.y + c[2].y * v.z,
              c[0].z * v.x + c[1].z * v.y + c[2].z * v.z);
}
/* scene.cpp:7040-7110: R * sqrt(I^-1) * R^T from six unique terms */
static void sqrt_inertia(const actor_t* a, srow_t* r) {
    const v3 l = V3(sqrtf(a->inv_inertia.x), sqrtf(a->inv_inertia.y), sqrtf(a->inv_inertia.z));
    const qt q = mass_orientation(a);
    if (q.x == 0.0f && q.y == 0.0f && q.z == 0.0f && q.w == 1.0f) {
        r->sqrt_i[0] = V3(l.x, 0, 0); r->sqrt_i[1] = V3(0, l.y, 0); r->sqrt_i[2] = V3(0, 0, l.z);
        return;
    }
    const v3 rx = rot_sc(q, V3(1, 0, 0)), ry = rot_sc(q, V3(0, 1, 0)), rz = rot_sc(q, V3(0, 0, 1));
    const float xx = l.x * rx.x * rx.x + l.y * ry.x * ry.x + l.z * rz.x * rz.x;
    const float yy = l.x * rx.y * rx.y + l.y * ry.y * ry.y + l.z * rz.y * rz.y;
    const float zz = l.x * rx.z * rx.z + l.y * ry.z * ry.z + l.z * rz.z * rz.z;
    const float xy = l.x * rx.x * rx.y + l.y * ry.x * ry.y + l.z * rz.x * rz.y;
    const float xz = l.x * rx.x * rx.z + l.y * ry.x * ry.z + l.z * rz.x * rz.z;
    const float yz = l.x * rx.y * rx.z + l.y * ry.y * ry.z + l.z * rz.y * rz.z;
    r->sqrt_i[0] = V3(xx, xy, xz); r->sqrt_i[1] = V3(xy, yy, yz); r->sqrt_i[2] = V3(xz, yz, zz);
}

typedef struct { uint32_t index, b0, b1, rows; int joint; } desc_t;
typedef struct {
    uint32_t crow0, ncrow;          /* contact rows in solve order */
    uint32_t frow0, nfrow;          /* friction rows (2 per anchor) */
    uint32_t npatch;
    float sf, df;
    uint8_t anchors;
    uint32_t b0, b1;                /* actor ids of shape0 / shape1 */
} mprep_t;

/* ------------------------- sleep ------------------------- */
/* Union-find with path halving; the smaller index becomes the root. */
static uint32_t uf_root(uint32_t* p, uint32_t x) {
    while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
    return x;
}
static void uf_join(uint32_t* p, uint32_t a, uint32_t b) {
    a = uf_root(p, a); b = uf_root(p, b);
    if (a < b) p[b] = a; else if (b < a) p[a] = b;
}
static void clear_sleep_filter(actor_t* a) { a->lin_acc = V3(0, 0, 0); a->ang_acc = V3(0, 0, 0); }
/* Counted interactions (scene.cpp:2728-2749: overlap pairs and constraints
 * on their dynamic bodies), activation (scene.cpp:6148-6250: a newly found
 * overlap of two dynamic bodies, one awake, or a newly found touch marks its
 * bodies activating -- the touch also clears readiness -- and every sleeping
 * body in the overlap-graph island of an activating body wakes, the islands
 * being those of the previous step's pairs) and
 * deactivation (scene.cpp:6465-6530: an island of the touch and constraint
 * graph whose bodies are all ready and not all asleep falls asleep). */
static void sleep_islands(fo_scene* s) {
    const uint32_t na = s->na;
    for (uint32_t i = 0; i < na; ++i) s->actors[i].counted = s->actors[i].joints;
    int any_asleep = 0;
    for (uint32_t i = 0; i < na; ++i) any_asleep |= s->actors[i].dynamic && s->actors[i].sleeping;
    uint8_t* act = (uint8_t*)calloc(na + 1, 1);
    for (uint64_t i = 0; i < s->nmgr; ++i) {
        const mgr_t* m = &s->mgr[i];
        const uint32_t a = s->shapes[(uint32_t)(m->key >> 32)].body, b = s->shapes[(uint32_t)m->key].body;
        actor_t* A = &s->actors[a];
        actor_t* B = &s->actors[b];
        if (A->dynamic) ++A->counted;
        if (B->dynamic) ++B->counted;
        if (m->found_now && A->dynamic && B->dynamic && (!A->sleeping || !B->sleeping)) act[a] = act[b] = 1;
        if (m->new_touch) {
            if (A->dynamic) { act[a] = 1; A->ready = 0; }
            if (B->dynamic) { act[b] = 1; B->ready = 0; }
        }
    }
    /* kinematic links (touching managers and joints): a pending target
     * keeps the dynamic partner's island awake (scene.cpp:6430-6463); a new
     * target wakes a sleeping or sleep-ready partner (scene.cpp:893-911) */
    uint8_t* kin = (uint8_t*)calloc(na + 1, 1);
    for (uint64_t i = 0; i < s->nmgr + s->nj; ++i) {
        uint32_t a, b;
        if (i < s->nmgr) {
            const mgr_t* m = &s->mgr[i];
            if (!m->touching) continue;
            a = s->shapes[(uint32_t)(m->key >> 32)].body;
            b = s->shapes[(uint32_t)m->key].body;
        } else {
            if (!s->joint_live[i - s->nmgr]) continue;
            a = s->joint_a[i - s->nmgr];
            b = s->joint_b[i - s->nmgr];
        }
        const actor_t* A = &s->actors[a];
        const actor_t* B = &s->actors[b];
        if (A->kinematic == B->kinematic) continue;
        const actor_t* K = A->kinematic ? A : B;
        const uint32_t d = A->kinematic ? b : a;
        if (!s->actors[d].dynamic) continue;
        if (K->kin_pending) kin[d] |= 1;
        if (K->kin_new) { kin[d] |= 2; act[d] = 1; }
    }
    for (uint32_t i = 0; i < na; ++i) {
        actor_t* a = &s->actors[i];
        if (!(kin[i] & 2) || !a->dynamic || (!a->sleeping && !a->ready)) continue;
        if (a->sleeping) any_asleep = 1;
        a->sleeping = 0;
        a->ready = 0;
        a->wake = fmaxf_(a->wake, 0.4f);
        clear_sleep_filter(a);
    }
    uint32_t* par = (uint32_t*)malloc(4 * (na + 1));
    uint8_t* flag = (uint8_t*)calloc(na + 1, 1);
    if (any_asleep) {
        /* The overlap graph's islands as the previous step left them: its
         * pairs (the kept and the lost ones of this step) and constraints.
         * This step's lost pairs split them only after activation; its new
         * pairs activate both of their bodies instead. */
        for (uint32_t i = 0; i < na; ++i) par[i] = i;
        for (uint64_t i = 0; i < s->nmgr + s->nlost; ++i) {
            uint64_t key;
            if (i < s->nmgr) {
                if (s->mgr[i].found_now) continue;
                key = s->mgr[i].key;
            } else {
                key = s->lost[i - s->nmgr];
            }
            const uint32_t a = s->shapes[(uint32_t)(key >> 32)].body, b = s->shapes[(uint32_t)key].body;
            if (s->actors[a].dynamic && s->actors[b].dynamic) uf_join(par, a, b);
        }
        for (uint32_t j = 0; j < s->nj; ++j)
            if (s->joint_live[j] && s->actors[s->joint_a[j]].dynamic && s->actors[s->joint_b[j]].dynamic)
                uf_join(par, s->joint_a[j], s->joint_b[j]);
        for (uint32_t i = 0; i < na; ++i)
            if (act[i]) flag[uf_root(par, i)] = 1;
        for (uint32_t i = 0; i < na; ++i) {
            actor_t* a = &s->actors[i];
            if (!a->dynamic || !a->sleeping || !flag[uf_root(par, i)]) continue;
            a->sleeping = 0;
            a->ready = 0;
            a->wake = fmaxf_(a->wake, 0.4f);
            clear_sleep_filter(a);
        }
    }
    for (uint32_t i = 0; i < na; ++i) { par[i] = i; flag[i] = 0; }
    for (uint64_t i = 0; i < s->nmgr; ++i) {
        const mgr_t* m = &s->mgr[i];
        if (!m->touching) continue;
        const uint32_t a = s->shapes[(uint32_t)(m->key >> 32)].body, b = s->shapes[(uint32_t)m->key].body;
        if (s->actors[a].dynamic && s->actors[b].dynamic) uf_join(par, a, b);
    }
    for (uint32_t j = 0; j < s->nj; ++j)
        if (s->joint_live[j] && s->actors[s->joint_a[j]].dynamic && s->actors[s->joint_b[j]].dynamic)
            uf_join(par, s->joint_a[j], s->joint_b[j]);
    for (uint32_t i = 0; i < na; ++i) {
        const actor_t* a = &s->actors[i];
        if (!a->dynamic) continue;
        const uint32_t r = uf_root(par, i);
        if (!a->ready || (kin[i] & 1)) flag[r] |= 1;
        if (!a->sleeping) flag[r] |= 2;
    }
    for (uint32_t i = 0; i < na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->dynamic || a->sleeping || flag[uf_root(par, i)] != 2) continue;
        a->sleeping = 1;
        a->wake = 0.0f;
        a->v = V3(0, 0, 0);
        a->w = V3(0, 0, 0);
        clear_sleep_filter(a);
    }
    free(act); free(par); free(flag); free(kin);
}
/* Dy sleepCheck without stabilization (scene.cpp:10640-10705). */
static void sleep_check(actor_t* a, qt q, v3 ml, v3 mw, float dt) {
    const float wake_reset = 20.0f * 0.02f;
    const float energy_threshold = 5.0e-5f * 10.0f * 10.0f;
    float wc = a->wake;
    if (wc < wake_reset * 0.5f || wc < dt) {
        const v3 la = rotinv_sc(q, mw);
        const v3 lacc = V3(a->lin_acc.x + ml.x, a->lin_acc.y + ml.y, a->lin_acc.z + ml.z);
        const v3 aacc = V3(a->ang_acc.x + la.x, a->ang_acc.y + la.y, a->ang_acc.z + la.z);
        const v3 ii = a->inv_inertia;
        const v3 inertia = V3(ii.x > 0.0f ? 1.0f / ii.x : 1.0f, ii.y > 0.0f ? 1.0f / ii.y : 1.0f,
                              ii.z > 0.0f ? 1.0f / ii.z : 1.0f);
        const float angular = (aacc.x * aacc.x * inertia.x + aacc.y * aacc.y * inertia.y +
                               aacc.z * aacc.z * inertia.z) * a->inv_mass;
        const float linear = lacc.x * lacc.x + lacc.y * lacc.y + lacc.z * lacc.z;
        const float energy = 0.5f * (angular + linear);
        const float cluster = 1.0f + (float)a->counted;
        const float threshold = cluster * energy_threshold;
        if (energy >= threshold) {
            clear_sleep_filter(a);
            const float factor = threshold == 0.0f ? 2.0f : fminf_(energy / threshold, 2.0f);
            wc = factor * 0.5f * wake_reset + dt * (cluster - 1.0f);
        } else {
            a->lin_acc = lacc;
            a->ang_acc = aacc;
            wc = fmaxf_(wc - dt, 0.0f);
        }
    } else {
        wc = fmaxf_(wc - dt, 0.0f);
    }
    a->wake = wc;
    a->ready = wc == 0.0f;
    if (a->ready) clear_sleep_filter(a);
}

int fo_scene_step(fo_scene* s, float dt, const uint64_t* manager_order, uint64_t n_mgr,
                  const uint64_t* joint_order, uint64_t n_joint) {
    if (!isfinite(dt) || dt <= 0.0f) FAIL(FO_INVALID, "Native CPU timestep must be finite and positive");
    int rc = collide(s);
    if (rc) return rc;
    if (s->sleep) sleep_islands(s);
    pre_integrate(s, dt);
    const float inv_dt = 1.0f / dt;
    /* ---- descriptor order (scene.cpp:7174-7216) ---- */
    /* managers and joints of sleeping islands are not solved */
#define ASLEEP(b) (s->actors[b].dynamic && s->actors[b].sleeping)
    const uint64_t nmo_in = manager_order ? n_mgr : s->nman;
    uint64_t nmo = 0;
    uint64_t* mo = (uint64_t*)malloc(8 * (nmo_in + 1));
    for (uint64_t i = 0; i < nmo_in; ++i) {
        const uint64_t mi = manager_order ? manager_order[i] : i;
        if (mi >= s->nman) { free(mo); FAIL(FO_LOGIC, "manager order out of range"); }
        const uint64_t key = s->mgr[s->man[mi]].key;
        if (ASLEEP(s->shapes[(uint32_t)(key >> 32)].body) || ASLEEP(s->shapes[(uint32_t)key].body)) continue;
        mo[nmo++] = mi;
    }
    const uint64_t njo_in = joint_order ? n_joint : s->nj;
    uint64_t njo = 0;
    uint64_t* jo = (uint64_t*)malloc(8 * (njo_in + 1));
    for (uint64_t i = 0; i < njo_in; ++i) {
        const uint64_t ji = joint_order ? joint_order[i] : (s->nj - 1 - i);
        if (ji >= s->nj || !s->joint_live[ji]) continue;
        if (ASLEEP(s->joint_a[ji]) || ASLEEP(s->joint_b[ji])) continue;
        jo[njo++] = ji;
    }
#undef ASLEEP
    /* ---- solver body admission (scene.cpp:6940-7040) ---- */
    srow_t* rows = (srow_t*)calloc(s->na + 1, sizeof(srow_t));
    srow_t world;
    memset(&world, 0, sizeof world);
    world.q = Q4(0, 0, 0, 1);
    for (uint64_t i = 0; i < nmo; ++i) {
        const mgr_t* m = &s->mgr[s->man[mo[i]]];
        const uint32_t ba = s->shapes[(uint32_t)(m->key >> 32)].body;
        const uint32_t bb = s->shapes[(uint32_t)m->key].body;
        const int responds = fminf_(s->actors[ba].max_contact_impulse, s->actors[bb].max_contact_impulse) != 0.0f;
        if (s->actors[ba].dynamic && responds) rows[ba].admitted = 1;
        if (s->actors[bb].dynamic && responds) rows[bb].admitted = 1;
    }
    for (uint64_t i = 0; i < njo; ++i) {
        rows[s->joint_a[jo[i]]].admitted |= s->actors[s->joint_a[jo[i]]].dynamic;
        rows[s->joint_b[jo[i]]].admitted |= s->actors[s->joint_b[jo[i]]].dynamic;
    }
    for (uint32_t i = 0; i < s->na; ++i) {
        if (!rows[i].admitted) continue;
        const actor_t* a = &s->actors[i];
        srow_t* r = &rows[i];
        r->p = mass_position(a);
        r->q = mass_orientation(a);
        r->v = a->v;
        r->w = a->w;
        r->inv_mass = a->inv_mass;
        sqrt_inertia(a, r);
    }
    /* a kinematic body's solver record: its target velocity, no inverse
     * mass or inertia (scene.cpp:6956-6973) */
    for (uint32_t i = 0; i < s->na; ++i) {
        const actor_t* a = &s->actors[i];
        if (!a->kinematic) continue;
        srow_t* r = &rows[i];
        r->p = mass_position(a);
        r->q = mass_orientation(a);
        r->v = a->v;
        r->w = a->w;
        r->inv_mass = 0.0f;
    }
#define ROW(b) ((s->actors[b].dynamic || s->actors[b].kinematic) ? &rows[b] : &world)
    /* ---- partition (scene.cpp:7113-7488, one task) ---- */
    const uint64_t nd = njo + nmo;
    uint32_t jrow_n = 0;
    desc_t* d = (desc_t*)calloc(nd + 1, sizeof(desc_t));
    for (uint64_t i = 0; i < njo; ++i) {
        d[i].index = jrow_n;   /* first row of the joint, rows in joint order */
        jrow_n += joint_rows(s->joint_kind[jo[i]]);
        d[i].b0 = s->joint_a[jo[i]]; d[i].b1 = s->joint_b[jo[i]]; d[i].joint = 1;
        d[i].rows = joint_rows(s->joint_kind[jo[i]]);
    }
    for (uint64_t i = 0; i < nmo; ++i) {
        const mgr_t* m = &s->mgr[s->man[mo[i]]];
        const uint32_t sa = (uint32_t)(m->key >> 32), sb = (uint32_t)m->key;
        d[njo + i].index = (uint32_t)mo[i];
        d[njo + i].b0 = s->shapes[m->reversed ? sb : sa].body;
        d[njo + i].b1 = s->shapes[m->reversed ? sa : sb].body;
    }
    uint64_t* part = (uint64_t*)malloc(8 * (nd + 1));
    uint64_t* pending = (uint64_t*)malloc(8 * (nd + 1));
    uint64_t npending = 0;
    const uint64_t INV = UINT64_MAX;
    for (uint64_t i = 0; i < nd; ++i) {
        part[i] = INV;
        if (s->actors[d[i].b0].dynamic && s->actors[d[i].b1].dynamic) pending[npending++] = i;
    }
    uint64_t nparts = 0;
    for (uint64_t wave = 0; npending; wave += 32) {
        if (wave)
            for (uint64_t k = 0; k < npending; ++k) {
                rows[d[pending[k]].b0].mask = 0;
                rows[d[pending[k]].b1].mask = 0;
            }
        uint64_t over = 0;
        for (uint64_t k = 0; k < npending; ++k) {
            const uint64_t i = pending[k];
            srow_t* a = &rows[d[i].b0];
            srow_t* b = &rows[d[i].b1];
            const uint32_t avail = ~(a->mask | b->mask);
            if (!avail) { pending[over++] = i; continue; }
            const unsigned bit = (unsigned)__builtin_ctz(avail);
            a->mask |= 1u << bit;
            b->mask |= 1u << bit;
            const uint64_t lp = wave + bit;
            if (a->max_dyn < lp + 1) a->max_dyn = lp + 1;
            if (b->max_dyn < lp + 1) b->max_dyn = lp + 1;
            part[i] = lp;
            if (nparts < lp + 1) nparts = lp + 1;
        }
        if (over == npending) { FAIL(FO_LOGIC, "partition made no progress"); }
        npending = over;
    }
    for (uint64_t i = 0; i < nd; ++i) {
        if (part[i] != INV) continue;
        const int da = s->actors[d[i].b0].dynamic, db = s->actors[d[i].b1].dynamic;
        if (!da && !db) continue;
        srow_t* act = &rows[da ? d[i].b0 : d[i].b1];
        const uint64_t lp = act->max_dyn + act->static_count++;
        part[i] = lp;
        if (nparts < lp + 1) nparts = lp + 1;
    }
    free(s->pend);
    s->pend = (uint64_t*)calloc(nparts + 1, 8);
    s->npend = nparts;
    uint64_t nordered = 0;
    for (uint64_t i = 0; i < nd; ++i)
        if (part[i] != INV) { ++s->pend[part[i]]; ++nordered; }
    uint64_t cum = 0;
    uint64_t* cursor = (uint64_t*)calloc(nparts + 1, 8);
    for (uint64_t p = 0; p < nparts; ++p) { cursor[p] = cum; cum += s->pend[p]; s->pend[p] = cum; }
    uint64_t* ordered = (uint64_t*)malloc(8 * (nordered + 1));
    for (uint64_t i = 0; i < nd; ++i)
        if (part[i] != INV) ordered[cursor[part[i]]++] = i;
    free(cursor);
    free(s->desc);
    s->desc = (uint32_t*)malloc(16 * (nordered + 1));
    s->ndesc = nordered;
    for (uint64_t i = 0; i < nordered; ++i) {
        const desc_t* e = &d[ordered[i]];
        s->desc[4 * i] = e->index;
        s->desc[4 * i + 1] = e->b0;
        s->desc[4 * i + 2] = e->b1;
        s->desc[4 * i + 3] = e->rows;
    }
    /* ---- joint rows (scene.cpp:7615-7767) ---- */
    jrow_t* jr = (jrow_t*)calloc(jrow_n + 1, sizeof(jrow_t));
    for (uint64_t i = 0; i < njo; ++i) {
        const uint32_t j = (uint32_t)jo[i];
        const uint32_t id0 = s->joint_a[j], id1 = s->joint_b[j];
        const actor_t* b0 = &s->actors[id0];
        const actor_t* b1 = &s->actors[id1];
        const uint8_t kind = s->joint_kind[j];
        const v3 an0 = rot_sc(b0->q, s->joint_lp[2 * j]), an1 = rot_sc(b1->q, s->joint_lp[2 * j + 1]);
        const v3 world0 = vadd(b0->p, an0), world1 = vadd(b1->p, an1);
        const v3 c0 = mass_position(b0), c1 = mass_position(b1);
        const v3 ra = vsub(world0, c0), rb = vsub(world1, c1);
        const float m0 = b0->dynamic ? b0->inv_mass : 0.0f;
        const float m1 = b1->dynamic ? b1->inv_mass : 0.0f;
        const v3 rel = vsub(b0->v, b1->v);
        jrow_t* out = &jr[d[i].index];
        uint32_t emitted = 0;
#define RESP0(v) (b0->dynamic ? xform(&rows[id0], (v)) : V3(0, 0, 0))
#define RESP1(v) (b1->dynamic ? xform(&rows[id1], (v)) : V3(0, 0, 0))
#define EMIT(AX, A0, A1, JA, JB, ERR, RESP)                                                          \
        do {                                                                                         \
            const float resp_ = (RESP);                                                              \
            if (!(resp_ > 0.0f) || !isfinite(resp_)) FAIL(FO_LOGIC, "joint response");               \
            const float rcp_ = 1.0f / resp_;                                                         \
            jrow_t* r_ = &out[emitted++];                                                            \
            r_->axis = (AX); r_->ang_a = (JA); r_->ang_b = (JB); r_->ima = m0; r_->imb = m1;          \
            r_->vel_mult = -rcp_;                                                                    \
            const float speed_ = vdot((AX), rel) + vdot((A0), b0->w) - vdot((A1), b1->w);            \
            r_->constant = -rcp_ * ((ERR) * inv_dt + speed_);                                        \
            r_->unbiased = -rcp_ * speed_;                                                           \
        } while (0)
        if (kind <= FO_JOINT_ANCHORED) {
            const v3 off = V3(c0.x + ra.x - c1.x - rb.x, c0.y + ra.y - c1.y - rb.y, c0.z + ra.z - c1.z - rb.z);
            const float dist = sqrtf(vdot(off, off));
            const v3 axis = dist < 1.192092896e-07f ? V3(1, 0, 0) : V3(off.x / dist, off.y / dist, off.z / dist);
            const v3 a0 = vcross(ra, axis), a1 = vcross(rb, axis);
            const v3 ja = RESP0(a0), jb = RESP1(a1);
            EMIT(axis, a0, a1, ja, jb, dist - s->joint_len[j], m0 + m1 + vdot(ja, ja) + vdot(jb, jb));
            continue;
        }
        /* locked axes in frame A; rotation errors from the relative
         * quaternion, rows orthogonalised in the inverse-mass metric */
        const qt qa = qmul(b0->q, s->joint_lq[2 * j]);
        const v3 error_p = rotinv_sc(qa, vsub(world0, world1));
        v3 error_angle = V3(0, 0, 0), va = V3(0, 0, 0), vb = V3(0, 0, 0), c = V3(0, 0, 0);
        float dd = 0.0f, overlap = 0.0f;
        if (kind != FO_JOINT_SPHERICAL) {
            qt qb = qmul(b1->q, s->joint_lq[2 * j + 1]);
            if (qa.x * qb.x + qa.y * qb.y + qa.z * qb.z + qa.w * qb.w < 0.0f) qb = Q4(-qb.x, -qb.y, -qb.z, -qb.w);
            const qt eq = qmul(qconj(qa), qb);
            error_angle = V3(eq.x, eq.y, eq.z);
            va = V3(qa.x, qa.y, qa.z);
            vb = V3(qb.x, qb.y, qb.z);
            dd = qa.w * qb.w - vdot(va, vb);
            overlap = qa.w * qb.w + vdot(va, vb);
            c = V3(qa.w * vb.x + qb.w * va.x, qa.w * vb.y + qb.w * va.y, qa.w * vb.z + qb.w * va.z);
        }
        const float errors[6] = {error_p.x, error_p.y, error_p.z, -error_angle.x, -error_angle.y, -error_angle.z};
        const v3 basis[3] = {V3(1, 0, 0), V3(0, 1, 0), V3(0, 0, 1)};
        const float avc[3] = {va.x, va.y, va.z}, bvc[3] = {vb.x, vb.y, vb.z};
        const v3 diag[3] = {V3(dd, c.z, -c.y), V3(-c.z, dd, c.x), V3(c.y, -c.x, dd)};
        struct { v3 lin, a0, a1, ja, jb; float err, inv; } er[6];
        memset(er, 0, sizeof er);
        const uint32_t count = joint_rows(kind);
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t comp = k + (kind == FO_JOINT_PRISMATIC ? 1u : 0u) +
                                  (kind == FO_JOINT_REVOLUTE && k >= 3u ? 1u : 0u);
            er[k].err = errors[comp];
            if (comp < 3u) {
                er[k].lin = rot_sc(qa, basis[comp]);
                const v3 arm = kind == FO_JOINT_PRISMATIC ? vsub(world1, c0) : ra;
                er[k].a0 = vcross(arm, er[k].lin);
                er[k].a1 = vcross(rb, er[k].lin);
            } else {
                const uint32_t q = comp - 3u;
                const v3 v = diag[q];
                er[k].a0 = V3(0.5f * (va.x * bvc[q] + vb.x * avc[q] + v.x), 0.5f * (va.y * bvc[q] + vb.y * avc[q] + v.y),
                              0.5f * (va.z * bvc[q] + vb.z * avc[q] + v.z));
                if (overlap == 0.0f) {
                    const float t = -FLT_EPSILON;
                    er[k].a0 = V3(er[k].a0.x - basis[q].x * t, er[k].a0.y - basis[q].y * t, er[k].a0.z - basis[q].z * t);
                }
                er[k].a1 = er[k].a0;
            }
            er[k].ja = RESP0(er[k].a0);
            er[k].jb = RESP1(er[k].a1);
            for (uint32_t p = 0; p < k; ++p) {
                const float w = (m0 + m1) * vdot(er[k].lin, er[p].lin) + vdot(er[k].ja, er[p].ja) + vdot(er[k].jb, er[p].jb);
                const float t = w * er[p].inv;
#define PROJ(F) er[k].F = V3(er[k].F.x - er[p].F.x * t, er[k].F.y - er[p].F.y * t, er[k].F.z - er[p].F.z * t)
                PROJ(lin); PROJ(a0); PROJ(a1); PROJ(ja); PROJ(jb);
#undef PROJ
                er[k].err -= er[p].err * t;
            }
            const float resp = (m0 + m1) * vdot(er[k].lin, er[k].lin) + vdot(er[k].ja, er[k].ja) + vdot(er[k].jb, er[k].jb);
            er[k].inv = resp > 0.0f ? 1.0f / resp : 0.0f;
            EMIT(er[k].lin, er[k].a0, er[k].a1, er[k].ja, er[k].jb, er[k].err, resp);
        }
#undef EMIT
#undef RESP0
#undef RESP1
    }
    /* ---- contact and friction rows (scene.cpp:7631-8510, CPU path) ---- */
    const float bias_coeff = 0.8f, bounce = -2.0f, same_normal = 0.999f, fr_thr = 0.04f;
    crow_t* cr = (crow_t*)calloc(4 * nmo + 1, sizeof(crow_t));
    frow_t* fr = (frow_t*)calloc(8 * nmo + 1, sizeof(frow_t));
    mprep_t* mp = (mprep_t*)calloc(s->nman + 1, sizeof(mprep_t));
    uint32_t ncr = 0, nfr = 0;
    const uint64_t epoch = s->fr_epoch + 1;
    for (uint64_t oi = 0; oi < nmo; ++oi) {
        const uint64_t mi = mo[oi];
        mgr_t* m = &s->mgr[s->man[mi]];
        mprep_t* P = &mp[mi];
        const uint32_t sa = (uint32_t)(m->key >> 32), sb = (uint32_t)m->key;
        const shape_t* sh0 = &s->shapes[m->reversed ? sb : sa];
        const shape_t* sh1 = &s->shapes[m->reversed ? sa : sb];
        const actor_t* act0 = &s->actors[sh0->body];
        const actor_t* act1 = &s->actors[sh1->body];
        P->b0 = sh0->body; P->b1 = sh1->body;
        const srow_t* A = ROW(sh0->body);
        const srow_t* B = ROW(sh1->body);
        const float rest_d = sh0->rest_offset + sh1->rest_offset;
        const float maximp = fminf_(act0->max_contact_impulse, act1->max_contact_impulse);
        const float maxpen = -fminf_(act0->max_depenetration, act1->max_depenetration);
        const float restitution = 0.5f * (sh0->rest + sh1->rest);
        const float damping = 0.5f * (sh0->damping + sh1->damping);
        const float dfr = fmaxf_(0.0f, 0.5f * (sh0->df + sh1->df));
        const float sfr = fmaxf_(dfr, 0.5f * (sh0->sf + sh1->sf));
        /* createContactPatches: one run per compatible normal */
        int cps[4], cpn[4], ncp = 0;
        v3 cpnorm[4], cpmin[4], cpmax[4];
        for (int j = 0; j < m->count; ++j) {
            const v3 n = V3(m->pts[j].n[0], m->pts[j].n[1], m->pts[j].n[2]);
            const v3 p = V3(m->pts[j].p[0], m->pts[j].p[1], m->pts[j].p[2]);
            if (ncp == 0 || vdot(cpnorm[ncp - 1], n) < same_normal) {
                cps[ncp] = j; cpn[ncp] = 1; cpnorm[ncp] = n; cpmin[ncp] = p; cpmax[ncp] = p; ++ncp;
            } else {
                ++cpn[ncp - 1];
                cpmin[ncp - 1] = V3(fminf_(cpmin[ncp - 1].x, p.x), fminf_(cpmin[ncp - 1].y, p.y), fminf_(cpmin[ncp - 1].z, p.z));
                cpmax[ncp - 1] = V3(fmaxf_(cpmax[ncp - 1].x, p.x), fmaxf_(cpmax[ncp - 1].y, p.y), fmaxf_(cpmax[ncp - 1].z, p.z));
            }
        }
        /* correlatePatches with valid previous anchors first */
        patch_t pl[8];
        int npl = 0;
        if (m->fr_epoch == s->fr_epoch && m->fr_count) {
            for (int h = 0; h < m->fr_count; ++h) {
                const patch_t* old = &m->fr[h];
                /* cached_friction_patch_valid (scene.cpp:3981-4011) */
                int valid = !(old->broken || old->anchor_count == 0);
                if (valid) {
                    const qt q0 = mass_orientation(act0), q1 = mass_orientation(act1);
                    const v3 on = rotinv_sc(q0, rot_sc(q1, old->body1_normal));
                    if (vdot(old->body0_normal, on) <= same_normal) valid = 0;
                    const v3 p0 = mass_position(act0), p1 = mass_position(act1);
                    for (int k = 0; valid && k < old->anchor_count; ++k) {
                        const v3 lc = rot_sc(q1, old->a1[k]);
                        const v3 wld = V3(lc.x + p1.x, lc.y + p1.y, lc.z + p1.z);
                        const v3 in0 = rotinv_sc(q0, V3(wld.x - p0.x, wld.y - p0.y, wld.z - p0.z));
                        const v3 dl = V3(old->a0[k].x - in0.x, old->a0[k].y - in0.y, old->a0[k].z - in0.z);
                        if (fabsf(vdot(dl, old->body0_normal)) >= 0.025f) valid = 0;
                    }
                }
                if (!valid) continue;
                patch_t c = *old;
                c.normal = rot_sc(mass_orientation(act0), old->body0_normal);
                c.contact_count = 0;
                c.bmin = V3(FLT_MAX, FLT_MAX, FLT_MAX);
                c.bmax = V3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
                pl[npl++] = c;
            }
        }
        int heads[8], nxt[4], cpid[4];
        for (int h = 0; h < 8; ++h) heads[h] = -1;
        for (int c = 0; c < ncp; ++c) {
            int lp = 0;
            for (; lp < npl; ++lp) {
                const patch_t* q = &pl[lp];
                if (vdot(q->normal, cpnorm[c]) >= same_normal && q->rest == restitution &&
                    q->damping == damping && q->sf == sfr && q->df == dfr)
                    break;
            }
            if (lp == npl) {
                patch_t np_;
                memset(&np_, 0, sizeof np_);
                np_.normal = cpnorm[c];
                np_.sf = sfr; np_.df = dfr; np_.rest = restitution; np_.damping = damping;
                np_.body0_normal = rotinv_sc(mass_orientation(act0), cpnorm[c]);
                np_.body1_normal = rotinv_sc(mass_orientation(act1), cpnorm[c]);
                pl[npl++] = np_;
            }
            patch_t* q = &pl[lp];
            if (q->contact_count == 0) { q->bmin = cpmin[c]; q->bmax = cpmax[c]; }
            else {
                q->bmin = V3(fminf_(q->bmin.x, cpmin[c].x), fminf_(q->bmin.y, cpmin[c].y), fminf_(q->bmin.z, cpmin[c].z));
                q->bmax = V3(fmaxf_(q->bmax.x, cpmax[c].x), fmaxf_(q->bmax.y, cpmax[c].y), fmaxf_(q->bmax.z, cpmax[c].z));
            }
            q->contact_count = (uint16_t)(q->contact_count + cpn[c]);
            nxt[c] = heads[lp];
            heads[lp] = c;
            cpid[c] = lp;
        }
        int remap[8], used[8], kept = 0;
        for (int j = 0; j < npl; ++j) {
            if (pl[j].contact_count == 0) continue;
            remap[j] = kept;
            used[kept] = heads[j];
            if (kept != j) pl[kept] = pl[j];
            ++kept;
        }
        int ptpatch[4];
        for (int c = 0; c < ncp; ++c)
            for (int j = cps[c]; j < cps[c] + cpn[c]; ++j) ptpatch[j] = remap[cpid[c]];
        v3 hn[8];
        for (int j = 0; j < kept; ++j) {
            const int h = used[j];
            hn[j] = V3(m->pts[cps[h]].n[0], m->pts[cps[h]].n[1], m->pts[cps[h]].n[2]);
        }
        /* Supported shapes publish one common normal per manifold, so the
         * correlation yields one patch holding one contact run and the
         * solver's patch order equals Gu point order (scene.cpp:8206-8224). */
        if (kept > 1 || ncp > 1) FAIL(FO_LOGIC, "multi-patch managers are outside the supported shapes");
        P->crow0 = ncr;
        P->npatch = (uint32_t)kept;
        crow_t tmp[4];
        for (int j = 0; j < m->count; ++j) {
            const fo_point* ct = &m->pts[j];
            const v3 pos = V3(ct->p[0], ct->p[1], ct->p[2]);
            const v3 n = hn[ptpatch[j]];
            const v3 raxn = vcross(vsub(pos, A->p), n);
            const v3 rbxn = vcross(vsub(pos, B->p), n);
            const float lin_vrel = vdot(n, vsub(A->v, B->v));
            const v3 ra = xform(A, raxn), rb = xform(B, rbxn);
            const float ang_vrel = vdot(raxn, A->w) - vdot(rbxn, B->w);
            const float vrel = lin_vrel + ang_vrel;
            const float response = (A->inv_mass + vdot(ra, ra)) + (B->inv_mass + vdot(rb, rb));
            const float vm = response > 0.0f ? 1.0f / response : 0.0f;
            const float pen = ct->sep - rest_d;
            const float pen_dt = pen * inv_dt;
            const int separated = pen >= 0.0f;
            const int closing = -vrel > pen_dt;
            const int bouncing = restitution > 0.0f && bounce > vrel && closing;
            const float tv = bouncing ? -vrel * restitution : 0.0f;
            crow_t* r = &tmp[j];
            memset(r, 0, sizeof *r);
            r->n = n; r->ra = ra; r->rb = rb; r->max_impulse = maximp; r->imp_mult = 1.0f;
            const float target = tv - vrel;
            const float pds = separated ? pen_dt : pen * (inv_dt * bias_coeff);
            const float sb_ = bouncing ? 0.0f : vm * fmaxf_(maxpen, pds);
            r->vel_mult = vm;
            r->biased = target * vm - sb_;
            r->unbiased = target * vm - (bouncing ? 0.0f : fmaxf_(sb_, 0.0f));
            if (!isfinite(response) || !isfinite(r->biased) || !isfinite(r->unbiased))
                FAIL(FO_OVERFLOW, "Native Dy contact preparation overflow");
        }
        for (int j = 0; j < m->count; ++j) cr[ncr + j] = tmp[j];
        P->ncrow = m->count;
        ncr += m->count;
        /* growPatches + tangent rows (scene.cpp:8296-8450) */
        P->frow0 = nfr;
        P->nfrow = 0;
        for (int pi = 0; pi < kept; ++pi) {
            patch_t* q = &pl[pi];
            const v3 ext = vsub(q->bmax, q->bmin);
            const float dsq = vlen2(ext);
            int keep_pair = 0;
            if (q->anchor_count == 2) {
                const v3 df_ = vsub(q->a0[0], q->a0[1]);
                keep_pair = vlen2(df_) * 4.0f >= dsq;
                if (!keep_pair) q->anchor_count = 0;
            }
            v3 anch[2] = {V3(0, 0, 0), V3(0, 0, 0)};
            int changed[2] = {0, 0};
            int cnt = q->anchor_count;
            if (!keep_pair) {
                if (cnt == 1) anch[0] = vadd(rot_sc(mass_orientation(act0), q->a0[0]), mass_position(act0));
                float pd2 = 0.0f;
                for (int c = used[pi]; c >= 0; c = nxt[c])
                    for (int j = cps[c]; j < cps[c] + cpn[c]; ++j) {
                        const fo_point* pt = &m->pts[j];
                        if (pt->sep >= fr_thr + rest_d) continue;
                        const v3 w = V3(pt->p[0], pt->p[1], pt->p[2]);
                        if (cnt == 0) { anch[0] = w; changed[0] = 1; ++cnt; }
                        else if (cnt == 1) {
                            const float dd = vlen2(vsub(w, anch[0]));
                            if (dd > 1.0e-8f) { anch[1] = w; changed[1] = 1; pd2 = dd; ++cnt; }
                        } else {
                            const float d0 = vlen2(vsub(w, anch[0]));
                            const float d1 = vlen2(vsub(w, anch[1]));
                            if (d0 > d1 && d0 > pd2) { anch[1] = w; changed[1] = 1; pd2 = d0; }
                            else if (d1 >= d0 && d1 > pd2) { anch[0] = w; changed[0] = 1; pd2 = d1; }
                        }
                    }
                for (int k = 0; k < cnt; ++k) {
                    if (!changed[k]) continue;
                    const qt q0 = mass_orientation(act0), q1 = mass_orientation(act1);
                    const v3 p0 = mass_position(act0), p1 = mass_position(act1);
                    q->a0[k] = rotinv_sc(q0, V3(anch[k].x - p0.x, anch[k].y - p0.y, anch[k].z - p0.z));
                    q->a1[k] = rotinv_sc(q1, V3(anch[k].x - p1.x, anch[k].y - p1.y, anch[k].z - p1.z));
                }
                if (cnt == 0) { q->a0[0] = V3(0, 0, 0); q->a1[0] = V3(0, 0, 0); }
            }
            q->anchor_count = (uint8_t)cnt;
            q->row_offset = nfr;
            if (cnt == 0) continue;
            const v3 n = hn[pi];
            const v3 rel = vsub(A->v, B->v);
            v3 t0 = vsub(rel, V3(n.x * vdot(rel, n), n.y * vdot(rel, n), n.z * vdot(rel, n)));
            if (vlen2(t0) <= 0.0001f)
                t0 = fabsf(n.x) < 0.70710678f ? V3(0.0f, -n.z, n.y) : V3(-n.y, n.x, 0.0f);
            const float il = 1.0f / sqrtf(vlen2(t0));
            t0 = V3(t0.x * il, t0.y * il, t0.z * il);
            const v3 t1 = vcross(n, t0);
            for (int k = 0; k < cnt; ++k) {
                const v3 ra = rot_sc(mass_orientation(act0), q->a0[k]);
                const v3 rb = rot_sc(mass_orientation(act1), q->a1[k]);
                const v3 c0 = mass_position(act0), c1 = mass_position(act1);
                const v3 err = vsub(V3(ra.x + c0.x, ra.y + c0.y, ra.z + c0.z), V3(rb.x + c1.x, rb.y + c1.y, rb.z + c1.z));
                for (int t = 0; t < 2; ++t) {
                    const v3 tg = t == 0 ? t0 : t1;
                    const v3 ax0 = vcross(ra, tg), ax1 = vcross(rb, tg);
                    const v3 j0 = xform(A, ax0), j1 = xform(B, ax1);
                    const float resp = (A->inv_mass + vdot(j0, j0)) + (B->inv_mass + vdot(j1, j1));
                    frow_t* f = &fr[nfr++];
                    memset(f, 0, sizeof *f);
                    f->t = tg; f->ra = j0; f->rb = j1;
                    f->vel_mult = resp > 0.0f ? bias_coeff / resp : 0.0f;
                    f->bias = vdot(tg, err) * inv_dt;
                    f->target = -(vdot(tg, rel) + vdot(ax0, A->w) - vdot(ax1, B->w));
                }
            }
            P->nfrow += (uint32_t)(2 * cnt);
        }
        /* keep the new history on the manager (friction_by_edge_) */
        m->fr_count = kept > 2 ? 2 : kept;
        for (int j = 0; j < m->fr_count; ++j) m->fr[j] = pl[j];
        m->fr_epoch = epoch;
        P->sf = kept ? pl[0].sf : 0;
        P->df = kept ? pl[0].df : 0;
        P->anchors = kept ? pl[0].anchor_count : 0;
    }
    s->fr_epoch = epoch;
    /* ---- PGS (scene.cpp:8853-9148) ---- */
    const float maxf = FLT_MAX;
    int pos = 0, vel = 0;
    for (uint32_t i = 0; i < s->na; ++i)
        if (s->actors[i].dynamic) {
            if (s->actors[i].pos_iters > pos) pos = s->actors[i].pos_iters;
            if (s->actors[i].vel_iters > vel) vel = s->actors[i].vel_iters;
        }
    if (vel < 1) vel = 1;
    for (int it = 0; it < pos + vel; ++it) {
        for (uint64_t k = 0; k < nordered; ++k) {
            const desc_t* e = &d[ordered[k]];
            srow_t wl = world;
            srow_t* a = s->actors[e->b0].dynamic ? &rows[e->b0] : &wl;
            srow_t* b = s->actors[e->b1].dynamic ? &rows[e->b1] : &wl;
            if (e->joint) {
                for (uint32_t q = 0; q < e->rows; ++q) {
                    jrow_t* r = &jr[e->index + q];
                    const float nd_ = r->axis.x * (a->dv.x - b->dv.x) + r->axis.y * (a->dv.y - b->dv.y) +
                                      r->axis.z * (a->dv.z - b->dv.z) + vdot(r->ang_a, a->dw) - vdot(r->ang_b, b->dw);
                    const float cst = it < pos ? r->constant : r->unbiased;
                    const float nx = fclamp(r->applied + nd_ * r->vel_mult + cst, -maxf, maxf);
                    const float imp = nx - r->applied;
                    const float ia = imp * r->ima, ib = imp * r->imb;
                    a->dv = V3(a->dv.x + ia * r->axis.x, a->dv.y + ia * r->axis.y, a->dv.z + ia * r->axis.z);
                    b->dv = V3(b->dv.x - ib * r->axis.x, b->dv.y - ib * r->axis.y, b->dv.z - ib * r->axis.z);
                    a->dw = V3(a->dw.x + imp * r->ang_a.x, a->dw.y + imp * r->ang_a.y, a->dw.z + imp * r->ang_a.z);
                    b->dw = V3(b->dw.x - imp * r->ang_b.x, b->dw.y - imp * r->ang_b.y, b->dw.z - imp * r->ang_b.z);
                    r->applied = nx;
                }
                continue;
            }
            const mprep_t* P = &mp[e->index];
            if (P->npatch == 0) continue;
            float nsum = 0.0f;
            for (uint32_t j = 0; j < P->ncrow; ++j) {
                crow_t* r = &cr[P->crow0 + j];
                const v3 n = r->n;
                const float nvel = vdot(n, a->dv) - vdot(n, b->dv) + vdot(a->dw, r->ra) - vdot(b->dw, r->rb);
                const float err = it < pos ? r->biased : r->unbiased;
                const float dc = fmaxf_(-nvel * r->vel_mult + err, -r->applied);
                const float ni = fminf_(r->max_impulse, r->imp_mult * r->applied + dc);
                const float dl = ni - r->applied;
                const float da = dl * a->inv_mass, db = dl * b->inv_mass;
                a->dv = V3(a->dv.x + n.x * da, a->dv.y + n.y * da, a->dv.z + n.z * da);
                b->dv = V3(b->dv.x - n.x * db, b->dv.y - n.y * db, b->dv.z - n.z * db);
                a->dw = V3(a->dw.x + r->ra.x * dl, a->dw.y + r->ra.y * dl, a->dw.z + r->ra.z * dl);
                b->dw = V3(b->dw.x - r->rb.x * dl, b->dw.y - r->rb.y * dl, b->dw.z - r->rb.z * dl);
                r->applied = ni;
                nsum += ni;
            }
            if ((it >= pos || pos - it <= 3) && P->anchors) {
                const float coeff = P->anchors == 2 ? 0.5f : 1.0f;
                const float ms = P->sf * coeff * nsum;
                const float md = P->df * coeff * nsum;
                int broken = 0;
                for (uint32_t k2 = 0; k2 < P->nfrow; ++k2) {
                    frow_t* f = &fr[P->frow0 + k2];
                    const v3 n = f->t;
                    const float td = vdot(n, a->dv) - vdot(n, b->dv) + vdot(a->dw, f->ra) - vdot(b->dw, f->rb);
                    const float bias = it < pos ? f->bias : 0.0f;
                    const float cand = f->applied + (f->target - bias - td) * f->vel_mult;
                    const int clamped = fabsf(cand) > ms;
                    const float nx = clamped ? fminf_(md, fmaxf_(-md, cand)) : cand;
                    const float dl = nx - f->applied;
                    const float da = dl * a->inv_mass, db = dl * b->inv_mass;
                    a->dv = V3(a->dv.x + n.x * da, a->dv.y + n.y * da, a->dv.z + n.z * da);
                    b->dv = V3(b->dv.x - n.x * db, b->dv.y - n.y * db, b->dv.z - n.z * db);
                    a->dw = V3(a->dw.x + f->ra.x * dl, a->dw.y + f->ra.y * dl, a->dw.z + f->ra.z * dl);
                    b->dw = V3(b->dw.x - f->rb.x * dl, b->dw.y - f->rb.y * dl, b->dw.z - f->rb.z * dl);
                    f->applied = nx;
                    broken |= clamped;
                }
                if (it + 1 == pos + vel) {
                    mgr_t* m = &s->mgr[s->man[e->index]];
                    if (m->fr_count) m->fr[0].broken = (uint8_t)broken;
                }
            }
        }
        if (it + 1 == pos)
            for (uint32_t i = 0; i < s->na; ++i)
                if (rows[i].admitted) { rows[i].mdv = rows[i].dv; rows[i].mdw = rows[i].dw; }
    }
    /* ---- writeback, final velocity and integration (scene.cpp:9294-9548,
     *      10508-10707) ---- */
    free(s->impulses);
    uint64_t npts = 0;
    for (uint64_t i = 0; i < s->nman; ++i) npts += s->mgr[s->man[i]].count;
    s->impulses = (double*)calloc(npts + 1, sizeof(double));
    s->nimp = npts;
    {
        uint64_t off = 0;
        for (uint64_t i = 0; i < s->nman; ++i) {
            const mprep_t* P = &mp[i];
            const mgr_t* m = &s->mgr[s->man[i]];
            if (P->npatch)
                for (int j = 0; j < m->count; ++j) s->impulses[off + j] = cr[P->crow0 + j].applied;
            off += m->count;
        }
    }
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->dynamic || a->sleeping) continue;
        v3 ml = a->v, mw = a->w;
        if (rows[i].admitted) {
            const srow_t* r = &rows[i];
            ml = V3(r->v.x + r->mdv.x, r->v.y + r->mdv.y, r->v.z + r->mdv.z);
            const v3* c = r->sqrt_i;
            const v3 ad = r->mdw;
            mw = V3(r->w.x + c[0].x * ad.x + c[1].x * ad.y + c[2].x * ad.z,
                    r->w.y + c[0].y * ad.x + c[1].y * ad.y + c[2].y * ad.z,
                    r->w.z + c[0].z * ad.x + c[1].z * ad.y + c[2].z * ad.z);
            const v3 fd = r->dw;
            a->v = V3(r->v.x + r->dv.x, r->v.y + r->dv.y, r->v.z + r->dv.z);
            a->w = V3(r->w.x + c[0].x * fd.x + c[1].x * fd.y + c[2].x * fd.z,
                      r->w.y + c[0].y * fd.x + c[1].y * fd.y + c[2].y * fd.z,
                      r->w.z + c[0].z * fd.x + c[1].z * fd.y + c[2].z * fd.z);
        }
        const v3 center = mass_position(a);
        v3 p = V3(center.x + ml.x * dt, center.y + ml.y * dt, center.z + ml.z * dt);
        qt q = integrate_q(mass_orientation(a), mw, dt);
        q = qmul(q, qconj(a->ml_q));
        const v3 offv = rot_sc(q, a->ml_p);
        p = V3(p.x - offv.x, p.y - offv.y, p.z - offv.z);
        a->p = p;
        a->q = q;
        if (s->sleep) sleep_check(a, q, ml, mw, dt);
    }
    /* kinematic bodies take their targets after the solve and settle for
     * one step (scene.cpp:2045-2065, 10992-11005) */
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->kinematic) continue;
        if (a->kin_pending) {
            a->p = a->kp;
            a->q = a->kq;
            a->kin_pending = 0;
            a->ready = 1;
            a->kin_settling = 1;
        } else {
            a->kin_settling = 0;
        }
        a->kin_new = 0;
    }
#undef ROW
    free(mo); free(jo); free(rows); free(d); free(part); free(pending); free(ordered);
    free(jr); free(cr); free(fr); free(mp);
    return 0;
}

/* ------------------------- readers ------------------------- */
void fo_scene_counts(const fo_scene* s, uint64_t* o) {
    o[0] = s->na; o[1] = s->ns; o[2] = s->nmgr; o[3] = s->nfound; o[4] = s->nlost;
    o[5] = s->nman;
    uint64_t pts = 0;
    for (uint64_t i = 0; i < s->nman; ++i) pts += s->mgr[s->man[i]].count;
    o[6] = pts; o[7] = s->npend; o[8] = s->ndesc; o[9] = 1;
}
void fo_scene_body_states(const fo_scene* s, float* out) {
    for (uint32_t i = 0; i < s->na; ++i) {
        const actor_t* a = &s->actors[i];
        float* o = out + 14 * i;
        o[0] = a->p.x; o[1] = a->p.y; o[2] = a->p.z;
        o[3] = a->v.x; o[4] = a->v.y; o[5] = a->v.z;
        o[6] = a->q.x; o[7] = a->q.y; o[8] = a->q.z; o[9] = a->q.w;
        o[10] = a->w.x; o[11] = a->w.y; o[12] = a->w.z;
        o[13] = (a->dynamic || a->kinematic) && a->sleeping ? 1.0f : 0.0f;
    }
}
/* Scene::set_kinematic (scene.cpp:916-1003) before the first step. */
int fo_scene_set_kinematic(fo_scene* s, uint32_t actor, int on) {
    if (actor >= s->na) FAIL(FO_INVALID, "actor out of range");
    actor_t* a = &s->actors[actor];
    if (!a->dynamic && !a->kinematic) FAIL(FO_LOGIC, "Kinematic flag requires a rigid box");
    if (a->kinematic == (on != 0)) return 0;
    a->kinematic = on != 0;
    a->dynamic = on == 0;
    a->v = V3(0, 0, 0);
    a->w = V3(0, 0, 0);
    clear_sleep_filter(a);
    a->kin_pending = a->kin_new = a->kin_settling = 0;
    if (on) { a->sleeping = 1; a->ready = 1; }
    else { a->sleeping = 0; a->ready = 0; a->wake = 0.4f; }
    return 0;
}
/* Scene::set_kinematic_target (scene.cpp:858-912): normalised once. */
int fo_scene_set_kinematic_target(fo_scene* s, uint32_t actor, const float* pose) {
    if (actor >= s->na || !s->actors[actor].kinematic) FAIL(FO_LOGIC, "target requires a kinematic body");
    actor_t* a = &s->actors[actor];
    const float m = sqrtf(pose[3] * pose[3] + pose[4] * pose[4] + pose[5] * pose[5] + pose[6] * pose[6]);
    if (!isfinite(m) || fabsf(m - 1.0f) >= 1.0e-2f) FAIL(FO_INVALID, "Native kinematic target is not sane");
    a->kp = V3(pose[0], pose[1], pose[2]);
    a->kq = Q4(pose[3] / m, pose[4] / m, pose[5] / m, pose[6] / m);
    a->kin_pending = a->kin_new = 1;
    a->sleeping = 0;
    a->ready = 0;
    a->wake = 0.4f;
    return 0;
}
void fo_scene_set_sleeping(fo_scene* s, int on) {
    if (!on)
        for (uint32_t i = 0; i < s->na; ++i) {
            actor_t* a = &s->actors[i];
            if (!a->dynamic) continue;
            if (a->sleeping) clear_sleep_filter(a);
            a->wake = fmaxf_(a->wake, 0.4f);
            a->sleeping = a->ready = 0;
        }
    s->sleep = on;
}
/* Per actor: wake counter, sleeping, ready, counted interactions, linear and
 * local angular filter motion = 10 floats. */
void fo_scene_sleep_state(const fo_scene* s, float* out) {
    for (uint32_t i = 0; i < s->na; ++i) {
        const actor_t* a = &s->actors[i];
        float* o = out + 10 * i;
        o[0] = a->wake; o[1] = (float)a->sleeping; o[2] = (float)a->ready; o[3] = (float)a->counted;
        o[4] = a->lin_acc.x; o[5] = a->lin_acc.y; o[6] = a->lin_acc.z;
        o[7] = a->ang_acc.x; o[8] = a->ang_acc.y; o[9] = a->ang_acc.z;
    }
}
void fo_scene_set_body_states(fo_scene* s, const float* in) {
    for (uint32_t i = 0; i < s->na; ++i) {
        actor_t* a = &s->actors[i];
        if (!a->dynamic) continue;
        const float* o = in + 14 * i;
        a->p = V3(o[0], o[1], o[2]);
        a->v = V3(o[3], o[4], o[5]);
        a->q = Q4(o[6], o[7], o[8], o[9]);
        a->w = V3(o[10], o[11], o[12]);
    }
}
void fo_scene_mass_props(const fo_scene* s, float* out) {
    for (uint32_t i = 0; i < s->na; ++i) {
        const actor_t* a = &s->actors[i];
        float* o = out + 11 * i;
        memset(o, 0, 11 * sizeof(float));
        o[10] = 1.0f;
        if (!a->dynamic) continue;
        o[0] = a->inv_mass;
        o[1] = a->inv_inertia.x; o[2] = a->inv_inertia.y; o[3] = a->inv_inertia.z;
        o[4] = a->ml_p.x; o[5] = a->ml_p.y; o[6] = a->ml_p.z;
        o[7] = a->ml_q.x; o[8] = a->ml_q.y; o[9] = a->ml_q.z; o[10] = a->ml_q.w;
    }
}
void fo_scene_encoded_bounds(const fo_scene* s, uint32_t* out) {
    for (uint32_t i = 0; i < s->ns; ++i)
        for (int k = 0; k < 6; ++k) out[6 * i + k] = s->shapes[i].bounds[k];
}
uint64_t fo_scene_pairs(const fo_scene* s, int which, uint32_t* out) {
    const uint64_t n = which == 0 ? s->nmgr : which == 1 ? s->nfound : s->nlost;
    if (out)
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t k = which == 0 ? s->mgr[i].key : which == 1 ? s->found[i] : s->lost[i];
            out[2 * i] = (uint32_t)(k >> 32);
            out[2 * i + 1] = (uint32_t)k;
        }
    return n;
}
uint64_t fo_scene_manifolds(const fo_scene* s, uint32_t* pairs, uint32_t* counts,
                            uint32_t* reversed, float* pts) {
    if (pairs)
        for (uint64_t i = 0; i < s->nman; ++i) {
            const mgr_t* m = &s->mgr[s->man[i]];
            pairs[2 * i] = (uint32_t)(m->key >> 32);
            pairs[2 * i + 1] = (uint32_t)m->key;
            counts[i] = m->count;
            reversed[i] = (uint32_t)m->reversed;
            for (int k = 0; k < 4; ++k) {
                float* o = pts + 28 * i + 7 * k;
                if (k < m->count) {
                    memcpy(o, m->pts[k].p, 3 * 4); memcpy(o + 3, m->pts[k].n, 3 * 4); o[6] = m->pts[k].sep;
                } else memset(o, 0, 7 * 4);
            }
        }
    return s->nman;
}
uint64_t fo_scene_partitions(const fo_scene* s, uint32_t* desc, uint64_t* ends) {
    if (desc) memcpy(desc, s->desc, 16 * s->ndesc);
    if (ends) memcpy(ends, s->pend, 8 * s->npend);
    return s->ndesc;
}
uint64_t fo_scene_normal_impulses(const fo_scene* s, double* out) {
    if (out) memcpy(out, s->impulses, 8 * s->nimp);
    return s->nimp;
}
uint64_t fo_scene_sorted_min_x(const fo_scene* s, uint32_t* values, uint32_t* ids) {
    if (values) {
        memcpy(values, s->sorted_minx_val, 4 * s->nsorted);
        memcpy(ids, s->sorted_minx_id, 4 * s->nsorted);
    }
    return s->nsorted;
}
