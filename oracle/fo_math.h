/* Test infrastructure: scalar float helpers for the C restatement oracle.
 *
 * The reference evaluates every expression in float32 without FMA
 * contraction (x86-64 SSE, reference CMakeLists.txt:115-121).  Its two
 * quaternion rotation helpers associate differently and both are kept:
 *   rot_sc   src/native/scene.cpp:63-71      (v + w*t) + d
 *   rot_gu   src/native/GuPCMContactBoxBox.cpp:29-37,
 *            GuPCMContactSphere.cpp:28-35, GuPCMGjkEpa.cpp:33-41
 *                                            v + (t*w + d)
 */
#ifndef FO_MATH_H
#define FO_MATH_H
#include <math.h>
#include <float.h>
#include <stdint.h>

typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } qt;

static inline v3 V3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline qt Q4(float x, float y, float z, float w) { qt r = {x, y, z, w}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float vlen2(v3 a) { return vdot(a, a); }
static inline v3 vcross(v3 a, v3 b) {
    return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vcomp(v3 v, unsigned i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
static inline float fminf_(float a, float b) { return b < a ? b : a; }   /* std::min(a,b) */
static inline float fmaxf_(float a, float b) { return a < b ? b : a; }   /* std::max(a,b) */
static inline float fclamp(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }
static inline int vfinite(v3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

static inline v3 rot_sc(qt q, v3 v) {
    const v3 u = V3(q.x, q.y, q.z);
    const v3 c = vcross(u, v);
    const v3 t = V3(c.x * 2.0f, c.y * 2.0f, c.z * 2.0f);
    const v3 d = vcross(u, t);
    return V3(v.x + q.w * t.x + d.x, v.y + q.w * t.y + d.y, v.z + q.w * t.z + d.z);
}
static inline v3 rotinv_sc(qt q, v3 v) { return rot_sc(Q4(-q.x, -q.y, -q.z, q.w), v); }
static inline v3 rot_gu(qt q, v3 v) {
    const v3 u = V3(q.x, q.y, q.z);
    const v3 t = vmul(vcross(u, v), 2.0f);
    return vadd(v, vadd(vmul(t, q.w), vcross(u, t)));
}
static inline v3 rotinv_gu(qt q, v3 v) { return rot_gu(Q4(-q.x, -q.y, -q.z, q.w), v); }
/* src/physx_port/foundation/PxQuat.h:262-271 PxQuat::rotate (compound.cpp) */
static inline v3 rot_px(qt q, v3 v) {
    const float vx = 2.0f * v.x, vy = 2.0f * v.y, vz = 2.0f * v.z;
    const float w2 = q.w * q.w - 0.5f;
    const float dot2 = q.x * vx + q.y * vy + q.z * vz;
    return V3(vx * w2 + (q.y * vz - q.z * vy) * q.w + q.x * dot2,
              vy * w2 + (q.z * vx - q.x * vz) * q.w + q.y * dot2,
              vz * w2 + (q.x * vy - q.y * vx) * q.w + q.z * dot2);
}
/* scene.cpp:105-112 PxQuat::operator* */
static inline qt qmul(qt a, qt b) {
    return Q4(a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y,
              a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
              a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x,
              a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
static inline qt qconj(qt q) { return Q4(-q.x, -q.y, -q.z, q.w); }
static inline float qdot(qt a, qt b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
#endif
