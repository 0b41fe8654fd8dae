// Device helpers shared by the step kernels (solver.cu) and their adjoint
// (adjoint.cu): mass frames, Gu-ordered manager bodies, solver-body
// records with the world sqrt-inverse-inertia tensor, and the quaternion
// integrator.
#pragma once
#include "state.h"

namespace fyzz::b200 {
namespace {

__device__ __forceinline__ bool is_dyn(const DevState& s, uint32_t b) { return s.b_flags[b] & kBodyDynamic; }

__device__ __forceinline__ v3 mass_position(const DevState& s, uint32_t b) {
    return vadd(ld3(s.b_p[b]), rot_sc(ldq(s.b_q[b]), ld3(s.b_ml_p[b])));
}
__device__ __forceinline__ qt mass_orientation(const DevState& s, uint32_t b) {
    return qmul(ldq(s.b_q[b]), ldq(s.b_ml_q[b]));
}

// Gu-ordered bodies of a touching manager: shape0 (dynamic first) / shape1.
__device__ __forceinline__ void manager_bodies(const DevState& s, uint32_t pair, uint32_t& sh0, uint32_t& sh1) {
    const uint64_t key = s.cur.key[pair];
    const uint32_t sa = uint32_t(key >> 32), sb = uint32_t(key);
    const uint32_t ba = s.s_body[sa], bb = s.s_body[sb];
    const bool da = is_dyn(s, ba), db = is_dyn(s, bb);
    const bool reversed = !da || (da && db && ba < bb);
    sh0 = reversed ? sb : sa;
    sh1 = reversed ? sa : sb;
}

struct SBody { v3 v, w, p; float inv_mass; v3 c0, c1, c2; };
__device__ __forceinline__ SBody load_sbody(const DevState& s, int32_t b) {
    SBody r;
    if (b < 0) {
        r.v = r.w = r.p = {0, 0, 0};
        r.inv_mass = 0.0f;
        r.c0 = r.c1 = r.c2 = {0, 0, 0};
        return r;
    }
    r.v = ld3(s.sb_v[b]);
    r.w = ld3(s.sb_w[b]);
    r.p = mass_position(s, uint32_t(b));
    r.inv_mass = s.b_inv[b].w;
    const float4* si = s.sb_sqrt_i + 3 * size_t(b);
    r.c0 = ld3(si[0]); r.c1 = ld3(si[1]); r.c2 = ld3(si[2]);
    return r;
}
// Solver-body data of any actor: a dynamic body's (index b >= 0), or for an
// actor `a` that is not dynamic, the infinite-mass record of the world or
// of a kinematic body moving with its target velocity (scene.cpp:6956-6973).
__device__ __forceinline__ SBody load_sbody_any(const DevState& s, uint32_t a, int32_t b) {
    if (b >= 0 || !(s.b_flags[a] & kBodyKinematic)) return load_sbody(s, b);
    SBody r;
    r.v = ld3(s.b_v[a]);
    r.w = ld3(s.b_w[a]);
    r.p = mass_position(s, a);
    r.inv_mass = 0.0f;
    r.c0 = r.c1 = r.c2 = {0, 0, 0};
    return r;
}
__device__ __forceinline__ v3 xform(const SBody& d, v3 v) {
    return {d.c0.x * v.x + d.c1.x * v.y + d.c2.x * v.z,
            d.c0.y * v.x + d.c1.y * v.y + d.c2.y * v.z,
            d.c0.z * v.x + d.c1.z * v.y + d.c2.z * v.z};
}

__device__ __forceinline__ v3 lv(const float* f) { return {f[0], f[1], f[2]}; }
__device__ __forceinline__ void sv(float* f, v3 v) { f[0] = v.x; f[1] = v.y; f[2] = v.z; }

// scene.cpp:114-143
__device__ qt integrate_q(qt pose, v3 w, float dt) {
    float m = w.x * w.x + w.y * w.y + w.z * w.z;
    if (m != 0.0f) {
        m = sqrtf(m);
        if (m > 1.0e7f) {
            const float sc = 1.0e7f / m;
            w = {w.x * sc, w.y * sc, w.z * sc};
            m = 1.0e7f;
        }
        const float v = dt * m * 0.5f;
        const float sn = sinf(v) / m;
        const float cs = cosf(v);
        const qt dq = qmul({w.x * sn, w.y * sn, w.z * sn, 0.0f}, pose);
        const qt nx = {dq.x + pose.x * cs, dq.y + pose.y * cs, dq.z + pose.z * cs, dq.w + pose.w * cs};
        const float len = sqrtf(nx.x * nx.x + nx.y * nx.y + nx.z * nx.z + nx.w * nx.w);
        pose = {nx.x / len, nx.y / len, nx.z / len, nx.w / len};
    }
    return pose;
}

}  // namespace
}  // namespace fyzz::b200
