// Shared device-side definitions for the B200 rigid-body step.
//
// Arithmetic follows the reference NativeCpu scene operation by operation
// (float32, no FMA contraction: every .cu file is compiled with
// -fmad=false).  The reference uses two quaternion-rotation associativities;
// both are kept:
//   rot_sc  src/native/scene.cpp:63-71                 (v + w*t) + d
//   rot_gu  src/native/GuPCMContactBoxBox.cpp:29-37    v + (t*w + d)
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace fyzz::b200 {
using std::isfinite;

enum : uint32_t { kBox = 0, kSphere = 1, kPlane = 2, kConvex = 3 };
enum : uint32_t { kBodyDynamic = 1u, kBodyKinematic = 2u };
// b_sleep bits.  A kinematic body also uses the last three: a target
// waiting for the step (kKinPending, set on the host; cleared when the step
// moves the body there), a target set since the last step (kKinNew: its
// touching partners are woken) and the step after it reached its target
// (kKinSettling: at rest, still reported active).
enum : uint32_t { kSleeping = 1u, kReady = 2u, kKinPending = 4u, kKinNew = 8u, kKinSettling = 16u };
// joint kinds: the two distance authorings, then JointKind (scene.h:1528)
enum : uint32_t { kJointCenter = 0u, kJointAnchored = 1u, kJointFixed = 2u, kJointSpherical = 3u,
                  kJointRevolute = 4u, kJointPrismatic = 5u };

// Device error bits (published to the host after each step; the C ABI maps
// them to status codes like the reference's task error words,
// source_dy_distance_native.h:1336-1345).
enum : uint32_t {
    kErrPairCapacity = 1u << 0,
    kErrContactOverflow = 1u << 1,
    kErrNonFinite = 1u << 2,
    kErrPartition = 1u << 3,
    kErrLevelRange = 1u << 4,
    kErrUnionFind = 1u << 5,
    kErrIslandSize = 1u << 6,
    kErrLogic = 1u << 7,
};

struct v3 { float x, y, z; };
struct qt { float x, y, z, w; };

__host__ __device__ __forceinline__ v3 V3(float x, float y, float z) { return {x, y, z}; }
__host__ __device__ __forceinline__ qt Q4(float x, float y, float z, float w) { return {x, y, z, w}; }
__host__ __device__ __forceinline__ v3 vadd(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__host__ __device__ __forceinline__ v3 vsub(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__host__ __device__ __forceinline__ v3 vmul(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__host__ __device__ __forceinline__ v3 vneg(v3 a) { return {-a.x, -a.y, -a.z}; }
__host__ __device__ __forceinline__ float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float vlen2(v3 a) { return vdot(a, a); }
__host__ __device__ __forceinline__ v3 vcross(v3 a, v3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__host__ __device__ __forceinline__ float vcomp(v3 v, unsigned i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
// std::min / std::max / std::clamp semantics (first argument wins ties).
__host__ __device__ __forceinline__ float smin(float a, float b) { return b < a ? b : a; }
__host__ __device__ __forceinline__ float smax(float a, float b) { return a < b ? b : a; }
__host__ __device__ __forceinline__ float sclamp(float v, float lo, float hi) {
    return v < lo ? lo : (hi < v ? hi : v);
}
__device__ __forceinline__ bool vfinite(v3 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

__host__ __device__ __forceinline__ v3 rot_sc(qt q, v3 v) {
    const v3 u = {q.x, q.y, q.z};
    const v3 c = vcross(u, v);
    const v3 t = {c.x * 2.0f, c.y * 2.0f, c.z * 2.0f};
    const v3 d = vcross(u, t);
    return {v.x + q.w * t.x + d.x, v.y + q.w * t.y + d.y, v.z + q.w * t.z + d.z};
}
__host__ __device__ __forceinline__ v3 rotinv_sc(qt q, v3 v) { return rot_sc({-q.x, -q.y, -q.z, q.w}, v); }
__host__ __device__ __forceinline__ v3 rot_gu(qt q, v3 v) {
    const v3 u = {q.x, q.y, q.z};
    const v3 t = vmul(vcross(u, v), 2.0f);
    return vadd(v, vadd(vmul(t, q.w), vcross(u, t)));
}
__host__ __device__ __forceinline__ v3 rotinv_gu(qt q, v3 v) { return rot_gu({-q.x, -q.y, -q.z, q.w}, v); }
// PxQuat::operator* (scene.cpp:105-112)
__host__ __device__ __forceinline__ qt qmul(qt a, qt b) {
    return {a.w * b.x + b.w * a.x + a.y * b.z - a.z * b.y,
            a.w * b.y + b.w * a.y + a.z * b.x - a.x * b.z,
            a.w * b.z + b.w * a.z + a.x * b.y - a.y * b.x,
            a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__host__ __device__ __forceinline__ qt qconj(qt q) { return {-q.x, -q.y, -q.z, q.w}; }
__host__ __device__ __forceinline__ float qdot(qt a, qt b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

__device__ __forceinline__ v3 ld3(float4 f) { return {f.x, f.y, f.z}; }
__device__ __forceinline__ qt ldq(float4 f) { return {f.x, f.y, f.z, f.w}; }
__device__ __forceinline__ float4 st4(v3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
__device__ __forceinline__ float4 stq(qt q) { return make_float4(q.x, q.y, q.z, q.w); }

// ---------------------------------------------------------------------------
// Persistent per-contact-manager state.  One record per broadphase pair,
// carried from frame to frame by pair identity.
// PcmPersistentContact / PcmManifoldCache (scene.h:1444-1459).
struct PcmPoint { float la[3], lb[3], nb[3], sep; };
// 256 bytes: a record is whole 32-byte sectors, so pairs that skip their
// cache (sphere pairs) leave no partly written sector beside a neighbour's.
struct alignas(32) PcmCache {
    PcmPoint pts[4];
    float rel_p[3], rel_q[4], qa[4], qb[4];
    uint32_t meta;  // bits 0-7 count, bit 8 initialized
    uint32_t pad[8];
};
static_assert(sizeof(PcmCache) == 256, "PcmCache layout");
// One retained friction patch (FrictionPatch, scene.h:1588-1614) plus the
// epoch of the step that prepared it (friction_by_edge_, scene.cpp:8082).
struct alignas(16) FrictionHist {
    float n0[3], n1[3];
    float a0[2][3], a1[2][3];
    float sf, df, rest, damping;
    uint32_t meta;   // bits 0-7 anchor count, bit 8 broken, bit 9 valid patch,
                     // bits 10-11 anchor k taken from this step's contact point
                     // (bits 12-13 / 14-15: that point's index)
    uint32_t epoch;
};
static_assert(sizeof(FrictionHist) == 96, "FrictionHist layout");
// ContactPoint (scene.h:510-514), four slots per manager.
struct alignas(16) ContactPt { float p[3], n[3], sep; };

// Records are 16-byte aligned so that whole-record copies move as 128-bit
// loads and stores.
// Solver rows.  SolverContactPoint (scene.h:1561-1576) without the
// per-point patch index (one patch per manager for the supported shapes).
struct alignas(16) NormalRow {
    float n[3], ra[3], rb[3];
    float vel_mult, imp_mult, biased, unbiased, applied, max_impulse, pad;
};
static_assert(sizeof(NormalRow) == 64, "NormalRow layout");
// SolverContactFriction (scene.h:1622-1630)
struct alignas(16) FrictionRow {
    float t[3], ra[3], rb[3];
    float vel_mult, bias, target, applied, pad[3];
};
static_assert(sizeof(FrictionRow) == 64, "FrictionRow layout");
// JointRow (scene.h:1983-1990)
struct alignas(16) JointRow {
    float axis[3], ang_a[3], ang_b[3];
    float ima, imb, constant, unbiased, vel_mult, applied, pad;
};
static_assert(sizeof(JointRow) == 64, "JointRow layout");
// Per-manager solver header: bodies (-1 = static world), counts and the
// combined friction coefficients.
struct alignas(16) ManagerHeader {
    int32_t b0, b1;
    uint32_t count, anchors;
    float sf, df, ima, imb;    // friction coefficients, inverse masses
};

}  // namespace fyzz::b200
