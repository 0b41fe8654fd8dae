// Host side of the B200 rigid-body world: authoring tables that mirror the
// reference's fyzz::World / WorldBackend semantics, mass properties, the
// device upload, CUDA-graph stepping and the C ABI (include/fyzz_b200.h).
//
// Authoring follows the reference NativeCpu scene:
//   transforms are validated and normalised twice, once by World
//   (src/world.cpp:38-55) and once by Scene::validated_pose
//   (src/native/compound.cpp:9-18);
//   create_body gives unit inverse mass / inertia until
//   update_mass_properties (scene.cpp:254-265, compound.cpp:113-203);
//   shapes default to contact offset 0.02, rest offset 0 and the default
//   Material (world.h:78-90, scene.h:1189).
// Stepping is failure-atomic like Scene::step (scene.cpp:10725-11016): body
// state is checkpointed before a launch and restored when the device
// reports an error; a pair-capacity overflow grows the pair arrays, drops the
// contact-manager history (the reference's invalidate_after_rollback,
// source_sc_owned_gpu_broadphase_native.h:479-484) and replays the steps.
#include "state.h"
#include "convex.h"
#include "../../include/fyzz_b200.h"

#include <dlfcn.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace fyzz::b200 {
namespace {

struct HostBody {
    uint32_t scene = 0;
    bool dynamic = false;
    std::array<float, 3> p{}, v{}, w{};
    std::array<float, 4> q{0, 0, 0, 1};
    float inv_mass = 0.0f;
    std::array<float, 3> inv_inertia{0, 0, 0};
    std::array<float, 3> ml_p{0, 0, 0};
    std::array<float, 4> ml_q{0, 0, 0, 1};
    std::vector<uint32_t> shapes;   // attachment order
    // kinematic: moved to its target each step, infinite mass in contacts
    bool kinematic = false;
    std::array<float, 3> kp{0, 0, 0};
    std::array<float, 4> kq{0, 0, 0, 1};
    // sleep state (scene.h:1147-1153 Actor defaults)
    float wake = 0.4f;
    uint32_t sleep = 0;              // kSleeping | kReady
    std::array<float, 6> sacc{};     // accumulated linear, local angular motion
    // ScBodyCore::contactReportThreshold (scene.h:1122): FLT_MAX disables
    float report_threshold = FLT_MAX;
    // NpRigidDynamic wake on an authored velocity (scene.cpp:728-783): a
    // sleeping body starts with cleared sleep filters.
    void wake_up() {
        if (sleep & kSleeping) sacc = {};
        wake = std::max(wake, 0.4f);
        sleep = 0;
    }
};
struct HostShape {
    uint32_t body = 0, scene = 0, type = kBox;
    std::array<float, 3> half{0, 0, 0};
    float radius = 0.0f;
    std::array<float, 3> lp{0, 0, 0};
    std::array<float, 4> lq{0, 0, 0, 1};
    std::array<float, 4> mat{0.5f, 0.5f, 0.2f, 0.0f};   // static, dynamic, restitution, rest offset
    float contact_offset = 0.02f;
    uint32_t mesh = ~0u;            // cooked hull (index into the world's meshes)
};
// A joint: its descriptor bodies (distance kinds: the ordered pair with the
// anchors as authored, scene.cpp:3097-3108; other kinds: the authored order,
// record.swapped, scene.cpp:3050-3060), kind and local frames.
struct HostJoint {
    uint32_t a = 0, b = 0;
    float len = 0.0f;
    uint32_t scene = 0, slot = 0, kind = kJointCenter;
    uint32_t gen = 1;      // constraint slot generation (scene.cpp:3129-3137)
    bool live = true;      // retired slots wait on their scene's free list
    std::array<float, 3> la{0, 0, 0}, lb{0, 0, 0};
    std::array<float, 4> qa{0, 0, 0, 1}, qb{0, 0, 0, 1};
};
uint32_t joint_rows(uint32_t kind) {
    return kind <= kJointAnchored ? 1u : kind == kJointSpherical ? 3u : kind == kJointFixed ? 6u : 5u;
}

void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess)
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

std::array<float, 4> normalize_once(std::array<float, 4> q) {
    const float len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    return {q[0] / len, q[1] / len, q[2] / len, q[3] / len};
}
// World::validated_transform then Scene::validated_pose (passes = 2), or
// only the latter when fyzz::World already validated the transform (a
// WorldBackend caller, passes = 1).
std::array<float, 4> validated_orientation(const float* q4, int passes = 2) {
    std::array<float, 4> q{q4[0], q4[1], q4[2], q4[3]};
    for (int pass = 0; pass < passes; ++pass) {
        const float len = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!std::isfinite(q[0]) || !std::isfinite(q[1]) || !std::isfinite(q[2]) || !std::isfinite(q[3]) ||
            !std::isfinite(len) || std::abs(len - 1.0f) >= 1.0e-2f)
            throw std::invalid_argument("Rigid pose orientation is not sane");
        q = normalize_once(q);
    }
    return q;
}
void validate_position(const float* p) {
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2]))
        throw std::invalid_argument("Position must be finite");
}

// ---- mass properties (compound.cpp:113-203) ----
struct M3 { v3 c[3]; };
M3 m_from_q(qt q) {
    const float x = q.x, y = q.y, z = q.z, w = q.w;
    const float x2 = x + x, y2 = y + y, z2 = z + z;
    const float xx = x2 * x, yy = y2 * y, zz = z2 * z;
    const float xy = x2 * y, xz = x2 * z, xw = x2 * w;
    const float yz = y2 * z, yw = y2 * w, zw = z2 * w;
    M3 m;
    m.c[0] = {1.0f - yy - zz, xy + zw, xz - yw};
    m.c[1] = {xy - zw, 1.0f - xx - zz, yz + xw};
    m.c[2] = {xz + yw, yz - xw, 1.0f - xx - yy};
    return m;
}
float mel(const M3& m, int row, int col) { return vcomp(m.c[col], row); }
M3 m_mul(const M3& a, const M3& b) {
    M3 r;
    for (int c = 0; c < 3; ++c) {
        const v3 bc = b.c[c];
        r.c[c] = vadd(vadd(vmul(a.c[0], bc.x), vmul(a.c[1], bc.y)), vmul(a.c[2], bc.z));
    }
    return r;
}
// PxQuat::rotate (src/physx_port/foundation/PxQuat.h:262-271), which the
// compound mass uses to place a hull's centre of mass.
v3 rot_px(const std::array<float, 4>& q, v3 v) {
    const float vx = 2.0f * v.x, vy = 2.0f * v.y, vz = 2.0f * v.z;
    const float w2 = q[3] * q[3] - 0.5f;
    const float dot2 = q[0] * vx + q[1] * vy + q[2] * vz;
    return {vx * w2 + (q[1] * vz - q[2] * vy) * q[3] + q[0] * dot2,
            vy * w2 + (q[2] * vx - q[0] * vz) * q[3] + q[1] * dot2,
            vz * w2 + (q[0] * vy - q[1] * vx) * q[3] + q[2] * dot2};
}
M3 m_t(const M3& a) {
    M3 r;
    r.c[0] = {a.c[0].x, a.c[1].x, a.c[2].x};
    r.c[1] = {a.c[0].y, a.c[1].y, a.c[2].y};
    r.c[2] = {a.c[0].z, a.c[1].z, a.c[2].z};
    return r;
}
// Jacobi diagonalisation with quaternion rotations (S. Melax), as PhysX's
// PxDiagonalize does it (src/physx_port/foundation_source/FdMathUtils.cpp:
// 66-110 of the reference, which compound.cpp calls for the mass frame): at
// most 24 sweeps, each rotating away the largest off-diagonal element, with
// the same cut-offs, so the principal frames are bit-identical.
v3 diagonalize(const M3& m, qt& frame) {
    qt q = {0, 0, 0, 1};
    M3 d = m;
    for (int it = 0; it < 24; ++it) {
        const M3 axes = m_from_q(q);
        d = m_mul(m_mul(m_t(axes), m), axes);
        const float d0 = std::abs(mel(d, 2, 1)), d1 = std::abs(mel(d, 2, 0)), d2 = std::abs(mel(d, 1, 0));
        const int a = (d0 > d1 && d0 > d2) ? 0 : (d1 > d2 ? 1 : 2);
        const int a1 = (a + 1) % 3, a2 = (a1 + 1) % 3;
        const float off = mel(d, a2, a1);
        if (off == 0.0f || std::abs(mel(d, a1, a1) - mel(d, a2, a2)) > 2e6f * std::abs(2.0f * off)) break;
        const float w = (mel(d, a1, a1) - mel(d, a2, a2)) / (2.0f * off);
        const float absw = std::abs(w);
        float v[3] = {0, 0, 0};
        float c;
        if (absw > 1000) {
            v[a] = 1.0f / (4.0f * w);
            c = 1.0f;
        } else {
            const float t = 1.0f / (absw + std::sqrt(w * w + 1.0f));
            const float h = 1.0f / std::sqrt(t * t + 1.0f);
            v[a] = std::sqrt((1.0f - h) / 2.0f) * (w < 0 ? -1.0f : 1.0f);
            c = std::sqrt((1.0f + h) / 2.0f);
        }
        const qt r = qmul(q, {v[0], v[1], v[2], c});
        const float mag = std::sqrt(r.x * r.x + r.y * r.y + r.z * r.z + r.w * r.w);
        const float sc = 1.0f / mag;
        q = {r.x * sc, r.y * sc, r.z * sc, r.w * sc};
    }
    frame = q;
    return {d.c[0].x, d.c[1].y, d.c[2].z};
}

// The tuning table next to the library (fyzzxyzzy-sdk_b200/tuning.txt for
// fyzzxyzzy-sdk_b200/lib/libfyzz_b200.so), or FYZZ_B200_TUNING; lines
// "<class> island_thread island_warp island_cta radix_bits elem_block
// work_queue",
// '#' comments.  Returns false when the class has no line.
bool load_tuning(const std::string& cls, fyzz_b200_tuning_t& out) {
    std::string path;
    if (const char* e = std::getenv("FYZZ_B200_TUNING")) {
        if (std::string(e) == "none") return false;
        path = e;
    } else {
        Dl_info info{};
        if (!dladdr(reinterpret_cast<void*>(&load_tuning), &info) || !info.dli_fname) return false;
        std::string lib = info.dli_fname;
        for (int up = 0; up < 2; ++up) {
            const size_t slash = lib.find_last_of('/');
            lib = slash == std::string::npos ? std::string(".") : lib.substr(0, slash);
        }
        path = lib + "/tuning.txt";
    }
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream in(line);
        std::string name;
        fyzz_b200_tuning_t t{};
        if (in >> name >> t.island_thread >> t.island_warp >> t.island_cta >> t.radix_bits >> t.elem_block >>
                t.work_queue &&
            name == cls) {
            out = t;
            return true;
        }
    }
    return false;
}
void validate_tuning(const fyzz_b200_tuning_t& t) {
    if (t.island_thread > 8 || t.island_warp < 32 || t.island_warp > 96 || t.island_cta < 128 || t.island_cta > 512 ||
        t.radix_bits < 8 || t.radix_bits > 11 || t.elem_block < 64 || t.elem_block > 1024 || t.elem_block % 32 ||
        t.work_queue > 1)
        throw std::invalid_argument("Tuning parameters outside their ranges");
}

template <class T> void dalloc(T*& p, size_t n, std::vector<void*>& owned) {
    if (n == 0) n = 1;
    check_cuda(cudaMalloc(reinterpret_cast<void**>(&p), n * sizeof(T)), "cudaMalloc");
    owned.push_back(p);
}
template <class T> void upload(T* dst, const std::vector<T>& src, cudaStream_t st) {
    if (!src.empty())
        check_cuda(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st), "upload");
}

}  // namespace

class World {
public:
    explicit World(int device) : device_(device) {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        check_cuda(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "cudaStreamCreate");
        for (int i = 0; i < Branches::kN; ++i) {
            check_cuda(cudaStreamCreateWithFlags(&br_.st[i], cudaStreamNonBlocking), "cudaStreamCreate");
            check_cuda(cudaEventCreateWithFlags(&br_.join[i], cudaEventDisableTiming), "cudaEventCreate");
        }
        check_cuda(cudaEventCreateWithFlags(&br_.fork, cudaEventDisableTiming), "cudaEventCreate");
        init_solver_kernels();
        check_cuda(cudaGetLastError(), "kernel attributes");
        check_cuda(cudaMallocHost(reinterpret_cast<void**>(&host_err_), 64), "cudaMallocHost");
        scene_body_begin_.push_back(0);
        scene_shape_begin_.push_back(0);
        scene_has_floor_.push_back(false);
    }
    ~World() {
        cudaSetDevice(device_);
        release_device();
        if (host_err_) cudaFreeHost(host_err_);
        for (int i = 0; i < Branches::kN; ++i) {
            if (br_.st[i]) cudaStreamDestroy(br_.st[i]);
            if (br_.join[i]) cudaEventDestroy(br_.join[i]);
        }
        if (br_.fork) cudaEventDestroy(br_.fork);
        if (stream_) cudaStreamDestroy(stream_);
    }
    std::string error;

    // ---------------- authoring ----------------
    uint32_t begin_scene() {
        pull_state();
        if (bodies_.size() == scene_body_begin_.back() && shapes_.size() == scene_shape_begin_.back())
            return uint32_t(scene_body_begin_.size() - 1);
        scene_body_begin_.push_back(uint32_t(bodies_.size()));
        scene_shape_begin_.push_back(uint32_t(shapes_.size()));
        scene_has_floor_.push_back(false);
        topology_dirty_ = true;
        return uint32_t(scene_body_begin_.size() - 1);
    }
    uint32_t current_scene() const { return uint32_t(scene_body_begin_.size() - 1); }
    // Authoring transforms arrive validated and normalised by fyzz::World
    // (src/world.cpp:38-55) when this world sits behind a WorldBackend; only
    // the scene's own normalisation (Scene::validated_pose) is applied then.
    void set_caller_validated(bool on) { norm_passes_ = on ? 1 : 2; }
    uint32_t add_static_floor(float height) {
        if (!std::isfinite(height)) throw std::invalid_argument("Native scene floor must be finite");
        if (scene_has_floor_.back()) throw std::logic_error("One static floor per scene is supported");
        pull_state();
        HostBody b;
        b.scene = current_scene();
        b.dynamic = false;
        b.p = {0.0f, height, 0.0f};
        bodies_.push_back(b);
        HostShape s;
        s.body = uint32_t(bodies_.size() - 1);
        s.scene = b.scene;
        s.type = kPlane;
        bodies_.back().shapes.push_back(uint32_t(shapes_.size()));
        shapes_.push_back(s);
        scene_has_floor_.back() = true;
        topology_dirty_ = true;
        return uint32_t(bodies_.size() - 1);
    }
    uint32_t create_dynamic_body(const float* pose) {
        validate_position(pose);
        const auto q = validated_orientation(pose + 3, norm_passes_);
        pull_state();
        HostBody b;
        b.scene = current_scene();
        b.dynamic = true;
        b.p = {pose[0], pose[1], pose[2]};
        b.q = q;
        b.inv_mass = 1.0f;
        b.inv_inertia = {1.0f, 1.0f, 1.0f};
        bodies_.push_back(b);
        topology_dirty_ = true;
        return uint32_t(bodies_.size() - 1);
    }
    HostBody& require_body(uint32_t id) {
        if (id >= bodies_.size()) throw std::out_of_range("Unknown rigid body");
        return bodies_[id];
    }
    const HostBody& require_body(uint32_t id) const {
        if (id >= bodies_.size()) throw std::out_of_range("Unknown rigid body");
        return bodies_[id];
    }
    uint32_t attach(uint32_t body, uint32_t type, const float* half, float radius, const float* local) {
        HostBody& b = require_body(body);
        if (!b.dynamic) throw std::logic_error("Shapes attach to dynamic bodies on this backend");
        if (b.scene != current_scene()) throw std::logic_error("Bodies of a closed scene cannot gain shapes");
        validate_position(local);
        const auto lq = validated_orientation(local + 3, norm_passes_);
        if (type == kBox) {
            if (!std::isfinite(half[0]) || !std::isfinite(half[1]) || !std::isfinite(half[2]) ||
                half[0] <= 0.0f || half[1] <= 0.0f || half[2] <= 0.0f)
                throw std::invalid_argument("Box half-extents must be finite and positive");
        } else if (!std::isfinite(radius) || radius <= 0.0f) {
            throw std::invalid_argument("Sphere radius must be finite and positive");
        }
        if (b.shapes.size() >= 8) throw std::logic_error("At most 8 shapes per body are supported");
        pull_state();
        HostShape s;
        s.body = body;
        s.scene = b.scene;
        s.type = type;
        if (type == kBox) s.half = {half[0], half[1], half[2]};
        s.radius = radius;
        s.lp = {local[0], local[1], local[2]};
        s.lq = lq;
        b.shapes.push_back(uint32_t(shapes_.size()));
        shapes_.push_back(s);
        topology_dirty_ = true;
        return uint32_t(shapes_.size() - 1);
    }
    // World::attach_convex_shape (scene.cpp:283-340): the shape's half
    // extents are the larger absolute vertex bound per axis; instances of one
    // cooked mesh share its device vertex range.
    uint32_t attach_convex(uint32_t body, std::shared_ptr<const CookedMesh> mesh, const float* local) {
        if (!mesh || mesh->verts.empty()) throw std::invalid_argument("Cooked convex geometry is missing");
        HostBody& b = require_body(body);
        if (!b.dynamic) throw std::logic_error("Shapes attach to dynamic bodies on this backend");
        if (b.scene != current_scene()) throw std::logic_error("Bodies of a closed scene cannot gain shapes");
        validate_position(local);
        const auto lq = validated_orientation(local + 3, norm_passes_);
        if (b.shapes.size() >= 8) throw std::logic_error("At most 8 shapes per body are supported");
        uint32_t m = 0;
        while (m < meshes_.size() && meshes_[m] != mesh) ++m;
        if (m == meshes_.size()) {
            uint64_t nv = mesh->verts.size();
            for (const auto& x : meshes_) nv += x->verts.size();
            if (nv > std::numeric_limits<uint32_t>::max())
                throw std::overflow_error("Convex vertex arena exceeds 32-bit device indexing");
        }
        pull_state();
        if (m == meshes_.size()) meshes_.push_back(mesh);
        HostShape s;
        s.body = body;
        s.scene = b.scene;
        s.type = kConvex;
        for (int k = 0; k < 3; ++k) s.half[k] = std::max(std::abs(mesh->lo[k]), std::abs(mesh->hi[k]));
        s.mesh = m;
        s.lp = {local[0], local[1], local[2]};
        s.lq = lq;
        b.shapes.push_back(uint32_t(shapes_.size()));
        shapes_.push_back(s);
        topology_dirty_ = true;
        return uint32_t(shapes_.size() - 1);
    }
    void update_mass_properties(uint32_t body, float density) {
        HostBody& b = require_body(body);
        if (!b.dynamic) throw std::logic_error("Static body has no mass properties");
        if (!std::isfinite(density) || density <= 0.0f)
            throw std::invalid_argument("Mass density must be positive and finite");
        pull_state();
        const float pi = 3.14159265358979323846f;
        // Shapes are visited in list order: most recently attached first.
        std::vector<uint32_t> order(b.shapes.rbegin(), b.shapes.rend());
        std::vector<float> um(order.size());
        std::vector<v3> lc(order.size());   // shape centre of mass in the body frame
        float mass = 0.0f;
        v3 center = {0, 0, 0};
        for (size_t i = 0; i < order.size(); ++i) {
            const HostShape& s = shapes_[order[i]];
            um[i] = s.type == kBox ? s.half[0] * s.half[1] * s.half[2] * 8.0f
                  : s.type == kConvex ? static_cast<float>(meshes_[s.mesh]->volume)
                                      : (4.0f / 3.0f) * pi * s.radius * s.radius * s.radius;
            const float m = um[i] * density;
            mass += m;
            lc[i] = {s.lp[0], s.lp[1], s.lp[2]};
            if (s.type == kConvex) {
                const auto& c = meshes_[s.mesh]->center;
                lc[i] = vadd(lc[i], rot_px(s.lq, {c[0], c[1], c[2]}));
            }
            center = vadd(center, vmul(lc[i], m));
        }
        if (!std::isfinite(mass) || !(mass > 0.0f)) throw std::invalid_argument("Compound mass outside supported range");
        center = vmul(center, 1.0f / mass);
        M3 tensor{};
        for (size_t i = 0; i < order.size(); ++i) {
            const HostShape& s = shapes_[order[i]];
            const float m = um[i] * density;
            M3 local{};
            if (s.type == kConvex) {
                const auto& I = meshes_[s.mesh]->inertia;
                for (int c = 0; c < 3; ++c) local.c[c] = vmul({I[c][0], I[c][1], I[c][2]}, density);
            } else {
                v3 diag;
                if (s.type == kBox) {
                    const v3 h = {s.half[0], s.half[1], s.half[2]};
                    diag = vmul({h.y * h.y + h.z * h.z, h.x * h.x + h.z * h.z, h.x * h.x + h.y * h.y}, m / 3.0f);
                } else {
                    const float v = (2.0f / 5.0f) * m * s.radius * s.radius;
                    diag = {v, v, v};
                }
                local.c[0].x = diag.x; local.c[1].y = diag.y; local.c[2].z = diag.z;
            }
            const M3 rot = m_from_q({s.lq[0], s.lq[1], s.lq[2], s.lq[3]});
            const M3 rt = m_mul(m_mul(rot, local), m_t(rot));
            const v3 d = vsub(lc[i], center);
            const float dd = vdot(d, d);
            for (int c = 0; c < 3; ++c) {
                tensor.c[c] = vadd(tensor.c[c], rt.c[c]);
                const float dc = vcomp(d, c);
                v3 pc = {-d.x * dc, -d.y * dc, -d.z * dc};
                if (c == 0) pc.x += dd; else if (c == 1) pc.y += dd; else pc.z += dd;
                tensor.c[c] = vadd(tensor.c[c], vmul(pc, m));
            }
        }
        qt axes;
        const v3 inertia = diagonalize(tensor, axes);
        const v3 inv = {1.0f / inertia.x, 1.0f / inertia.y, 1.0f / inertia.z};
        const float inv_mass = 1.0f / mass;
        if (!std::isfinite(inv.x) || !std::isfinite(inv.y) || !std::isfinite(inv.z) ||
            std::min({inv.x, inv.y, inv.z}) <= 0.0f || !std::isfinite(inv_mass) || inv_mass <= 0.0f)
            throw std::invalid_argument("Compound inverse mass/inertia outside supported range");
        b.inv_mass = inv_mass;
        b.inv_inertia = {inv.x, inv.y, inv.z};
        b.ml_p = {center.x, center.y, center.z};
        b.ml_q = {axes.x, axes.y, axes.z, axes.w};
        mass_dirty_ = true;
    }
    void set_shape_material(uint32_t shape, const fyzz_b200_material& m) {
        if (shape >= shapes_.size()) throw std::out_of_range("Unknown shape");
        if (!std::isfinite(m.static_friction) || !std::isfinite(m.dynamic_friction) ||
            !std::isfinite(m.restitution) || m.static_friction < 0.0f || m.dynamic_friction < 0.0f ||
            m.restitution > 1.0f)
            throw std::invalid_argument("PhysX contact material coefficients/modes invalid");
        pull_state();
        shapes_[shape].mat[0] = m.static_friction;
        shapes_[shape].mat[1] = m.dynamic_friction;
        shapes_[shape].mat[2] = m.restitution;
        mass_dirty_ = true;
    }
    // World::set_body_kinematic (scene.cpp:916-1003): a dynamic body becomes
    // kinematic (at rest, asleep until it gets a target) or back (awake).
    // The pair set changes (kinematic bodies pair with dynamic ones only), so
    // the device state is rebuilt and the contact-manager history restarts.
    void set_kinematic(uint32_t body, bool on) {
        HostBody& b = require_body(body);
        if (!b.dynamic && !b.kinematic) throw std::logic_error("Kinematic flag requires a rigid box");
        if (b.kinematic == on) return;
        pull_state();
        b.kinematic = on;
        b.dynamic = !on;
        b.v = {0, 0, 0};
        b.w = {0, 0, 0};
        b.sacc = {};
        if (on) {
            b.sleep = kSleeping | kReady;
        } else {
            b.sleep = 0u;
            b.wake = 0.4f;
        }
        topology_dirty_ = true;
    }
    // World::set_body_kinematic_target (scene.cpp:858-912): the pose the
    // body reaches at the end of the next step; touching partners wake.
    void set_kinematic_target(uint32_t body, const float* pose) {
        HostBody& b = require_body(body);
        if (!b.kinematic) throw std::logic_error("Source kinematic target requires eKINEMATIC rigid body");
        validate_position(pose);
        const float* q = pose + 3;
        const float m = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
        if (!std::isfinite(q[0]) || !std::isfinite(q[1]) || !std::isfinite(q[2]) || !std::isfinite(q[3]) ||
            !std::isfinite(m) || std::abs(m - 1.0f) >= 1.0e-2f)
            throw std::invalid_argument("Native kinematic target is not sane");
        pull_state();
        b.kp = {pose[0], pose[1], pose[2]};
        b.kq = {q[0] / m, q[1] / m, q[2] / m, q[3] / m};
        b.sleep = kKinPending | kKinNew;
        b.wake = 0.4f;
        mass_dirty_ = true;
    }
    void set_velocity(uint32_t body, const float* v, bool angular) {
        HostBody& b = require_body(body);
        if (!std::isfinite(v[0]) || !std::isfinite(v[1]) || !std::isfinite(v[2]))
            throw std::invalid_argument("Velocity must be finite");
        if (!b.dynamic) throw std::logic_error("Static actors have no velocity");
        pull_state();
        (angular ? b.w : b.v) = {v[0], v[1], v[2]};
        b.wake_up();
        mass_dirty_ = true;
    }
    // World::set_body_contact_report_threshold (src/world.cpp:355-359) then
    // Scene::set_contact_report_threshold (scene.cpp:1148-1161).  The first
    // finite threshold turns the world's force-threshold stream on (its
    // device arrays are allocated and the step graphs rebuilt); it then
    // stays on, so pairs that stop exceeding still report Lost.
    void set_report_threshold(uint32_t body, float force) {
        if (!std::isfinite(force) || force < 0.0f) throw std::invalid_argument("Invalid source contact report threshold");
        HostBody& b = require_body(body);
        if (!b.dynamic && !b.kinematic) throw std::logic_error("Source contact report threshold requires PxRigidDynamic");
        pull_state();
        b.report_threshold = force;
        mass_dirty_ = true;
        if (force != FLT_MAX && !thresholds_) {
            thresholds_ = true;
            if (uploaded_) {
                check_cuda(cudaSetDevice(device_), "cudaSetDevice");
                alloc_threshold_arrays();
                d_.thresholds = true;
                for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
                release_segment_graphs();
            }
        }
    }
    uint64_t add_distance(uint32_t a, uint32_t b, float len) {
        const float zero7[7] = {0, 0, 0, 0, 0, 0, 1};
        return add_joint(kJointCenter, a, b, zero7, zero7, len);
    }
    // World::add_*_constraint (src/world.cpp:231-276) then Scene::create_*
    // (scene.cpp:3046-3141).  local_a / local_b: position 3 + orientation 4.
    uint64_t add_joint(uint32_t kind, uint32_t a, uint32_t b, const float* local_a, const float* local_b, float len) {
        if (kind > kJointPrismatic) throw std::invalid_argument("Unknown joint kind");
        const HostBody& A = require_body(a);
        const HostBody& B = require_body(b);
        if (a == b) throw std::invalid_argument("Joint requires distinct actors");
        if (kind <= kJointAnchored && (!std::isfinite(len) || len < 0.0f))
            throw std::invalid_argument("Rigid 1D distance must be finite and nonnegative");
        HostJoint j;
        if (kind != kJointCenter) {
            validate_position(local_a);
            validate_position(local_b);
            j.la = {local_a[0], local_a[1], local_a[2]};
            j.lb = {local_b[0], local_b[1], local_b[2]};
        }
        if (kind >= kJointFixed) {
            j.qa = validated_orientation(local_a + 3, norm_passes_);
            j.qb = validated_orientation(local_b + 3, norm_passes_);
        }
        if (!A.dynamic && !B.dynamic) throw std::logic_error("Rigid constraint requires a dynamic solver node");
        if (A.scene != B.scene) throw std::invalid_argument("Constraint endpoints must share a scene");
        pull_state();
        j.kind = kind;
        j.a = kind <= kJointAnchored ? std::min(a, b) : a;
        j.b = kind <= kJointAnchored ? std::max(a, b) : b;
        j.len = kind <= kJointAnchored ? len : 0.0f;
        j.scene = A.scene;
        // Constraint slots (scene.cpp:3110-3140): the scene's most recently
        // retired slot is reused with its generation bumped, else a new one
        // is appended.  Slots index joints_, so they are unique in the
        // world; in a one-scene world they are the reference's slots.
        if (free_joints_.size() <= j.scene) free_joints_.resize(j.scene + 1);
        auto& fl = free_joints_[j.scene];
        uint32_t slot;
        if (!fl.empty()) {
            slot = fl.back();
            fl.pop_back();
            j.gen = joints_[slot].gen + 1;
            j.slot = slot;
            joints_[slot] = j;
        } else {
            slot = uint32_t(joints_.size());
            j.slot = slot;
            joints_.push_back(j);
        }
        joints_dirty_ = true;
        mass_dirty_ = true;     // the pulled host copy goes back with the joint tables
        return (uint64_t(j.gen) << 32) | slot;
    }
    // World::remove_constraint (Scene::retire_constraint, scene.cpp:3088-
    // 3096, 3195-3228): the joint leaves the step; its slot is reused next.
    void remove_joint(uint64_t id) {
        const uint32_t slot = uint32_t(id), gen = uint32_t(id >> 32);
        if (slot >= joints_.size() || !gen || !joints_[slot].live || joints_[slot].gen != gen)
            throw std::out_of_range("Unknown or expired rigid constraint");
        pull_state();
        HostJoint& j = joints_[slot];
        j.live = false;
        if (free_joints_.size() <= j.scene) free_joints_.resize(j.scene + 1);
        free_joints_[j.scene].push_back(slot);
        joints_dirty_ = true;
        mass_dirty_ = true;
    }
    void mass_props(uint32_t body, float* out) const {
        const HostBody& b = require_body(body);
        if (!b.dynamic) throw std::logic_error("Static body has no mass properties");
        out[0] = b.inv_mass;
        for (int i = 0; i < 3; ++i) out[1 + i] = b.inv_inertia[i];
        for (int i = 0; i < 3; ++i) out[4 + i] = b.ml_p[i];
        for (int i = 0; i < 4; ++i) out[7 + i] = b.ml_q[i];
    }

    // ---------------- device state ----------------
    void ensure_device() {
        if (topology_dirty_ || !uploaded_) {
            build_device();
        } else {
            if (joints_dirty_) refresh_joints();
            if (mass_dirty_) upload_bodies();
        }
        mass_dirty_ = false;
        joints_dirty_ = false;
    }
    // Device -> host body state, before any host authoring edit.
    void pull_state() {
        if (!uploaded_ || host_authoritative_) return;
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        const size_t n = bodies_.size() < d_.n_bodies ? bodies_.size() : d_.n_bodies;
        std::vector<float4> p(n), q(n), v(n), w(n), acc(2 * n);
        std::vector<float> wake(n);
        std::vector<uint32_t> sl(n);
        if (n) {
            check_cuda(cudaMemcpyAsync(p.data(), d_.b_p, n * 16, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(q.data(), d_.b_q, n * 16, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(v.data(), d_.b_v, n * 16, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(w.data(), d_.b_w, n * 16, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(wake.data(), d_.b_wake, n * 4, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(sl.data(), d_.b_sleep, n * 4, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaMemcpyAsync(acc.data(), d_.b_sacc, n * 32, cudaMemcpyDeviceToHost, stream_), "pull");
            check_cuda(cudaStreamSynchronize(stream_), "pull sync");
        }
        for (size_t i = 0; i < n; ++i) {
            auto& b = bodies_[i];
            if (b.kinematic) {   // pose moved to its targets, velocity derived, flags
                b.p = {p[i].x, p[i].y, p[i].z};
                b.q = {q[i].x, q[i].y, q[i].z, q[i].w};
                b.v = {v[i].x, v[i].y, v[i].z};
                b.w = {w[i].x, w[i].y, w[i].z};
                b.sleep = sl[i];
                continue;
            }
            if (!b.dynamic) continue;
            b.p = {p[i].x, p[i].y, p[i].z};
            b.q = {q[i].x, q[i].y, q[i].z, q[i].w};
            b.v = {v[i].x, v[i].y, v[i].z};
            b.w = {w[i].x, w[i].y, w[i].z};
            b.wake = wake[i];
            b.sleep = sl[i];
            b.sacc = {acc[2 * i].x, acc[2 * i].y, acc[2 * i].z, acc[2 * i + 1].x, acc[2 * i + 1].y, acc[2 * i + 1].z};
        }
        host_authoritative_ = true;
    }

    void step(float dt, uint32_t steps) {
        if (!std::isfinite(dt) || dt <= 0.0f) throw std::invalid_argument("Native CPU timestep must be finite and positive");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        if (steps == 0) return;
        for (int attempt = 0; attempt < 8; ++attempt) {
            snapshot(steps);
            run_steps(dt, steps);
            const uint32_t err = read_err();
            if (!err) {
                steps_done_ += steps;
                ev_device_valid_ = true;
                th_device_valid_ = true;
                return;
            }
            restore();
            if (err & kErrPairCapacity) {
                grow_pairs(d_.pair_cap * 2u);
                continue;
            }
            ev_device_valid_ = false;
            th_device_valid_ = false;
            raise_step_error(err);
        }
        ev_device_valid_ = false;
        th_device_valid_ = false;
        throw std::overflow_error("Pair capacity could not be satisfied");
    }

    // Re-sizes the pair budget to the live pairs times `headroom`, keeping
    // both contact-manager generations (keys, PCM caches, friction
    // histories, touch counts): the next step continues exactly as it would
    // have.  Per-step buffers are reallocated; the step graphs re-captured.
    void fit_pair_budget(float headroom) {
        if (!(headroom >= 1.0f)) throw std::invalid_argument("Pair budget headroom must be at least 1");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        release_rollout();
        uint32_t live[2] = {0, 0};
        for (int k = 0; k < 2; ++k)
            check_cuda(cudaMemcpy(&live[k], sets_[k].n, 4, cudaMemcpyDeviceToHost), "read");
        const uint64_t want = uint64_t(double(std::max(live[0], live[1])) * headroom) + 4096;
        const uint32_t cap = uint32_t(std::min<uint64_t>(want, 0x7fffffffull));
        if (cap < std::max(live[0], live[1])) throw std::overflow_error("Pair budget below the live pairs");
        resize_pairs_keeping(cap, live);
    }
    // Sets the pair budget to `cap` pairs (at least the live pairs of both
    // generations), keeping the contact-manager history.
    uint32_t set_pair_budget(uint32_t cap) {
        if (cap == 0 || cap > 0x7fffffffu) throw std::invalid_argument("Pair budget must be in [1, 2^31)");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        release_rollout();
        uint32_t live[2] = {0, 0};
        for (int k = 0; k < 2; ++k)
            check_cuda(cudaMemcpy(&live[k], sets_[k].n, 4, cudaMemcpyDeviceToHost), "read");
        resize_pairs_keeping(std::max({cap, live[0], live[1], 1u}), live);
        return d_.pair_cap;
    }
    // Re-allocates the pair arrays for `cap` pairs; both generations' live
    // records (keys, PCM caches, friction histories, touch counts) are
    // carried over, so the next step continues exactly as it would have.
    void resize_pairs_keeping(uint32_t cap, const uint32_t live[2]) {
        std::vector<void*> tmp;
        ManagerSet keep[2];
        for (int k = 0; k < 2; ++k) {
            dalloc(keep[k].key, std::max(live[k], 1u), tmp); dalloc(keep[k].cache, std::max(live[k], 1u), tmp);
            dalloc(keep[k].fric, std::max(live[k], 1u), tmp); dalloc(keep[k].count, std::max(live[k], 1u), tmp);
            dalloc(keep[k].n, 1, tmp);
            enqueue_copy_set(keep[k], sets_[k], live[k], stream_);
        }
        ThresholdSet keep_th[2];
        uint32_t live_th[2] = {0, 0};
        if (d_.thresholds)
            for (int k = 0; k < 2; ++k) {
                check_cuda(cudaMemcpy(&live_th[k], th_sets_[k].n, 4, cudaMemcpyDeviceToHost), "read");
                const size_t c = std::max(live_th[k], 1u);
                dalloc(keep_th[k].key, c, tmp); dalloc(keep_th[k].impulse, c, tmp);
                dalloc(keep_th[k].thr, c, tmp); dalloc(keep_th[k].n, 1, tmp);
                enqueue_copy_threshold_set(keep_th[k], th_sets_[k], live_th[k], stream_);
            }
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        const int parity = parity_, last = last_cur_;
        alloc_pairs(cap);
        for (int k = 0; k < 2; ++k) enqueue_copy_set(sets_[k], keep[k], live[k], stream_);
        if (d_.thresholds)
            for (int k = 0; k < 2; ++k) enqueue_copy_threshold_set(th_sets_[k], keep_th[k], live_th[k], stream_);
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        for (void* p : tmp) cudaFree(p);
        parity_ = parity;
        last_cur_ = last;
    }
    uint32_t pair_budget() const { return d_.pair_cap; }
    // Performance parameters; an explicit setting outlives rebuilds of the
    // device state, otherwise the world's class line of the tuning table
    // applies when the device state is built.
    void set_tuning(const fyzz_b200_tuning_t& t) {
        validate_tuning(t);
        tuning_ = t;
        tuning_explicit_ = true;
        apply_tuning();
    }
    fyzz_b200_tuning_t tuning() {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        return tuning_;
    }
    std::string tuning_class() const { return tuning_class_; }
    // The solver order of the next step, as the reference's Scene chose it
    // (partition_constraints' input: joints in constraint order, then the
    // touching managers in its island-edge order, scene.cpp:7153-7216):
    // pairs (shape a < shape b) in order, joint constraint ids (matched by
    // slot) in order.  Managers and joints the lists do not name follow in
    // canonical order.  Applies to exactly one step.
    void set_descriptor_order(const uint32_t* pairs, uint64_t n_pairs, const uint64_t* joint_ids, uint64_t n_joint_ids) {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        if (n_pairs > d_.pair_cap) throw std::invalid_argument("Descriptor order names more pairs than the pair budget");
        std::vector<std::pair<uint64_t, uint32_t>> keyed(n_pairs);
        for (uint64_t i = 0; i < n_pairs; ++i) {
            const uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
            if (a >= b || b >= shapes_.size()) throw std::invalid_argument("Descriptor order pair must be (a < b) shapes");
            keyed[i] = {(uint64_t(a) << 32) | b, uint32_t(i)};
        }
        std::sort(keyed.begin(), keyed.end());
        for (uint64_t i = 1; i < n_pairs; ++i)
            if (keyed[i].first == keyed[i - 1].first) throw std::invalid_argument("Descriptor order names a pair twice");
        std::vector<uint64_t> keys(n_pairs);
        std::vector<uint32_t> pos(n_pairs);
        for (uint64_t i = 0; i < n_pairs; ++i) { keys[i] = keyed[i].first; pos[i] = keyed[i].second; }
        // joint descriptors are the live joints by scene, slot descending
        std::vector<uint32_t> slots;
        for (const auto& j : joints_) if (j.live) slots.push_back(j.slot);
        std::stable_sort(slots.begin(), slots.end(), [&](uint32_t x, uint32_t y) {
            return joints_[x].scene != joints_[y].scene ? joints_[x].scene < joints_[y].scene : x > y;
        });
        std::vector<uint32_t> jrank(slots.size(), ~0u);
        uint32_t next = 0;
        for (uint64_t i = 0; i < n_joint_ids; ++i) {
            const uint32_t slot = uint32_t(joint_ids[i]);
            for (size_t d = 0; d < slots.size(); ++d)
                if (slots[d] == slot && jrank[d] == ~0u) jrank[d] = next++;
        }
        for (auto& r : jrank) if (r == ~0u) r = next++;
        if (replay_cap_ < std::max<uint64_t>(n_pairs, 1) || replay_jcap_ < std::max<size_t>(jrank.size(), 1)) {
            check_cuda(cudaStreamSynchronize(stream_), "sync");
            for (void* p : {static_cast<void*>(d_.rp_keys), static_cast<void*>(d_.rp_pos), static_cast<void*>(d_.rp_jrank)})
                if (p) {
                    owned_.erase(std::find(owned_.begin(), owned_.end(), p));
                    cudaFree(p);
                }
            replay_cap_ = std::max<uint64_t>(n_pairs, 1);
            replay_jcap_ = std::max<size_t>(jrank.size(), 1);
            dalloc(d_.rp_keys, replay_cap_, owned_); dalloc(d_.rp_pos, replay_cap_, owned_);
            dalloc(d_.rp_jrank, replay_jcap_, owned_);
        }
        upload(d_.rp_keys, keys, stream_);
        upload(d_.rp_pos, pos, stream_);
        upload(d_.rp_jrank, jrank, stream_);
        check_cuda(cudaStreamSynchronize(stream_), "replay upload");
        d_.rp_n = uint32_t(n_pairs);
        replay_pending_ = true;
    }
    // Test hook of the step's exclusive scan (the look-back scan every
    // step runs, on this world's scan scratch): scans n ones into a
    // temporary buffer.  With skip_first_tile the scan's tile ticket starts
    // at 1, so no block ever takes tile 0 and the block that takes tile 1
    // waits for a tile state that is never published: its bounded wait
    // gives up and sets the logic error bit.  The scan's last block still
    // resets the ticket, so later scans (and steps) run clean.  Returns the
    // device error bits; mismatches counts outputs other than their index.
    uint32_t scan_selftest(uint32_t n, bool skip_first_tile, uint64_t* mismatches) {
        if (n == 0 || n > (1u << 26)) throw std::invalid_argument("Scan self-test size must be in [1, 2^26]");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        if (scan_tmp_words_for(n) > d_.scan_tmp_words)
            throw std::invalid_argument("Scan self-test larger than the world's scan scratch");
        std::vector<void*> tmp;
        uint32_t *in = nullptr, *out = nullptr, *err = nullptr, *total = nullptr;
        dalloc(in, n, tmp); dalloc(out, n, tmp); dalloc(err, 1, tmp); dalloc(total, 1, tmp);
        upload(in, std::vector<uint32_t>(n, 1u), stream_);
        check_cuda(cudaMemsetAsync(out, 0xff, size_t(n) * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(err, 0, 4, stream_), "memset");
        if (skip_first_tile) {
            const uint32_t one = 1u;
            check_cuda(cudaMemcpyAsync(d_.scan_tmp + 1, &one, 4, cudaMemcpyHostToDevice, stream_), "ticket");
        }
        scan_exclusive(in, out, n, nullptr, total, d_.scan_tmp, d_.scan_tmp_words, stream_, err);
        check_cuda(cudaGetLastError(), "scan launch");
        std::vector<uint32_t> h(n);
        uint32_t bits = 0;
        check_cuda(cudaMemcpyAsync(h.data(), out, size_t(n) * 4, cudaMemcpyDeviceToHost, stream_), "read");
        check_cuda(cudaMemcpyAsync(&bits, err, 4, cudaMemcpyDeviceToHost, stream_), "read");
        check_cuda(cudaStreamSynchronize(stream_), "scan sync");
        for (void* p : tmp) cudaFree(p);
        uint64_t bad = 0;
        for (uint32_t i = 0; i < n; ++i) bad += h[i] != i ? 1u : 0u;
        if (mismatches) *mismatches = bad;
        return bits;
    }
    // ---------------- differentiable rollouts ----------------
    // A rollout of `steps` steps keeps a full-state checkpoint every `every`
    // steps.  The backward pass walks the segments in reverse: it restores
    // the segment's checkpoint and re-runs the segment forward with each
    // step writing its per-step solver data (solver bodies, manager rows and
    // headers, contact points, island and partition structure, impulse tape)
    // straight into its own frame, plus a copy of the step's pair keys,
    // touch counts and friction histories; then it applies the step adjoints
    // over the frames in reverse (enqueue_adjoint_step).  The persistent state
    // of a step (checkpoints) is the bodies, both contact-manager generations
    // (keys, PCM caches, friction histories, touch counts), the device
    // counters and the ping-pong parity.
    struct Slot {
        float4 *p = nullptr, *q = nullptr, *v = nullptr, *w = nullptr;
        ManagerSet sets[2];
        uint32_t* counters = nullptr;
        int parity = 0, last = 1;
        uint64_t steps = 0;
    };
    void alloc_slot(Slot& sl) {
        const size_t nb = d_.n_bodies, cap = d_.pair_cap;
        dalloc(sl.p, nb, roll_owned_); dalloc(sl.q, nb, roll_owned_);
        dalloc(sl.v, nb, roll_owned_); dalloc(sl.w, nb, roll_owned_);
        for (auto& m : sl.sets) {
            dalloc(m.key, cap, roll_owned_); dalloc(m.cache, cap, roll_owned_);
            dalloc(m.fric, cap, roll_owned_); dalloc(m.count, cap, roll_owned_);
            dalloc(m.n, 1, roll_owned_);
        }
        dalloc(sl.counters, kCntSlots, roll_owned_);
    }
    template <class T> void d2d(T* dst, const T* src, size_t n) {
        if (n) check_cuda(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, stream_), "state copy");
    }
    // Bodies, the live pairs of both generations, counters and parity.
    void save_slot(Slot& sl) {
        const size_t nb = d_.n_bodies;
        d2d(sl.p, d_.b_p, nb); d2d(sl.q, d_.b_q, nb); d2d(sl.v, d_.b_v, nb); d2d(sl.w, d_.b_w, nb);
        for (int k = 0; k < 2; ++k) enqueue_copy_set(sl.sets[k], sets_[k], d_.pair_cap, stream_);
        d2d(sl.counters, d_.counters, size_t(kCntSlots));
        sl.parity = parity_; sl.last = last_cur_; sl.steps = steps_done_;
    }
    void load_slot(const Slot& sl) {
        const size_t nb = d_.n_bodies;
        d2d(d_.b_p, sl.p, nb); d2d(d_.b_q, sl.q, nb); d2d(d_.b_v, sl.v, nb); d2d(d_.b_w, sl.w, nb);
        for (int k = 0; k < 2; ++k) enqueue_copy_set(sets_[k], sl.sets[k], d_.pair_cap, stream_);
        d2d(d_.counters, sl.counters, size_t(kCntSlots));
        parity_ = sl.parity; last_cur_ = sl.last; steps_done_ = sl.steps;
        host_authoritative_ = false;
    }
    struct Frame {
        float4 *sb_v = nullptr, *sb_w = nullptr, *sb_dv = nullptr, *sb_dw = nullptr, *sb_mdv = nullptr,
               *sb_mdw = nullptr, *sb_sqrt_i = nullptr, *x_c = nullptr, *x_q = nullptr;
        uint32_t* man_list = nullptr;
        ManagerHeader* mh = nullptr;
        NormalRow* nrow = nullptr;
        FrictionRow* frow = nullptr;
        JointRow* jrow = nullptr;
        ContactPt* pts = nullptr;
        ManagerSet cur;                 // keys, friction histories and touch counts of the step
        float *tn = nullptr, *tf = nullptr, *tj = nullptr;
        uint32_t *d_val2 = nullptr, *d_lbod = nullptr, *lvl_bound = nullptr, *isl_begin = nullptr,
                 *isl_end = nullptr, *isl_nbod = nullptr, *n_isl = nullptr, *counters = nullptr;
        uint32_t* lists[DevState::kIslLists] = {};
        int32_t* isl_bod = nullptr;
        int parity = 0;
    };
    void alloc_frame(Frame& f) {
        const size_t nb = d_.n_bodies, cap = d_.pair_cap, dc = d_.desc_cap;
        const size_t passes = size_t(d_.pos_iters + std::max(d_.vel_iters, 1));
        auto& o = roll_owned_;
        for (float4** b : {&f.sb_v, &f.sb_w, &f.sb_dv, &f.sb_dw, &f.sb_mdv, &f.sb_mdw, &f.x_c, &f.x_q})
            dalloc(*b, nb, o);
        dalloc(f.sb_sqrt_i, 3 * nb, o);
        dalloc(f.man_list, cap, o); dalloc(f.mh, cap, o);
        dalloc(f.nrow, 4 * cap, o); dalloc(f.frow, 4 * cap, o);
        dalloc(f.jrow, std::max<size_t>(d_.n_jrows, 1), o);
        dalloc(f.pts, 4 * cap, o);
        dalloc(f.cur.key, cap, o); dalloc(f.cur.fric, cap, o); dalloc(f.cur.count, cap, o); dalloc(f.cur.n, 1, o);
        dalloc(f.tn, passes * cap * 4, o); dalloc(f.tf, passes * cap * 4, o);
        dalloc(f.tj, passes * std::max<size_t>(d_.n_jrows, 1), o);
        dalloc(f.d_val2, dc, o); dalloc(f.d_lbod, dc, o);
        dalloc(f.lvl_bound, 2 * dc + 2, o); dalloc(f.isl_bod, 2 * dc + 2, o);
        dalloc(f.isl_begin, dc + 1, o); dalloc(f.isl_end, dc + 1, o); dalloc(f.isl_nbod, dc + 1, o);
        dalloc(f.n_isl, 1, o); dalloc(f.counters, kCntSlots, o);
        for (int k = 0; k < DevState::kIslLists; ++k) dalloc(f.lists[k], dc / (kListMinDesc[k] + 1) + 2, o);
    }
    // The step's DevState with its per-step arrays in frame f.
    DevState framed(const Frame& f, int parity) const {
        DevState s = view(parity);
        s.dt = roll_dt_;
        s.sleep = false;
        s.sb_v = f.sb_v; s.sb_w = f.sb_w; s.sb_dv = f.sb_dv; s.sb_dw = f.sb_dw;
        s.sb_mdv = f.sb_mdv; s.sb_mdw = f.sb_mdw; s.sb_sqrt_i = f.sb_sqrt_i;
        s.man_list = f.man_list; s.mh = f.mh; s.nrow = f.nrow; s.frow = f.frow; s.jrow = f.jrow;
        s.pts = f.pts;
        s.tape_n = f.tn; s.tape_f = f.tf; s.tape_j = d_.n_joints ? f.tj : nullptr;
        s.d_val2 = f.d_val2; s.d_lbod = f.d_lbod; s.lvl_bound = f.lvl_bound; s.isl_bod = f.isl_bod;
        s.isl_begin = f.isl_begin; s.isl_end = f.isl_end; s.isl_nbod = f.isl_nbod; s.n_isl = f.n_isl;
        for (int k = 0; k < DevState::kIslLists; ++k) s.isl_list[k] = f.lists[k];
        return s;
    }
    void release_segment_graphs() {
        for (auto& g : seg_graphs_) if (g.exec) cudaGraphExecDestroy(g.exec);
        seg_graphs_.clear();
    }
    void release_rollout() {
        release_segment_graphs();
        for (void* p : roll_owned_) cudaFree(p);
        roll_owned_.clear();
        ckpt_.clear();
        frames_.clear();
        roll_steps_ = 0;
        roll_done_ = false;
    }
    void rollout_begin(uint32_t steps, uint32_t every) {
        if (steps == 0 || every == 0) throw std::invalid_argument("Rollout needs steps and a checkpoint interval");
        for (const auto& j : joints_)
            if (j.live && j.kind != kJointCenter)
                throw std::logic_error("Differentiable rollouts support center distance joints only");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        pull_state();
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        // a differentiable rollout simulates every body: wake them all
        enqueue_wake_bodies(d_, stream_);
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        if (roll_steps_ == steps && roll_every_ == every && roll_cap_ == d_.pair_cap && !ckpt_.empty()) {
            // same shape as the previous rollout: checkpoints, frames and the
            // captured segment graphs are reused
            roll_done_ = false;
            check_cuda(cudaMemsetAsync(adj_.mark, 0, size_t(d_.n_bodies) * 4, stream_), "memset");
            check_cuda(cudaMemsetAsync(adj_.epoch, 0, 4, stream_), "memset");
            check_cuda(cudaStreamSynchronize(stream_), "sync");
            return;
        }
        release_rollout();
        roll_steps_ = steps;
        roll_every_ = every;
        roll_cap_ = d_.pair_cap;
        ckpt_.resize((steps + every - 1) / every + 1);   // last one: the final state
        frames_.resize(std::min(every, steps));
        for (auto& sl : ckpt_) alloc_slot(sl);
        for (auto& f : frames_) alloc_frame(f);
        const size_t cap = d_.pair_cap, nb = d_.n_bodies;
        AdjState& A = adj_;
        A = AdjState{};
        for (float4** f : {&A.c, &A.q, &A.v, &A.w, &A.x_c, &A.x_q, &A.dvm, &A.dwm, &A.dv, &A.dw, &A.rdv,
                           &A.rdw, &A.v1, &A.w1, &A.iI, &A.g_iI})
            dalloc(*f, nb, roll_owned_);
        dalloc(A.C, 3 * nb, roll_owned_);
        dalloc(A.im, nb, roll_owned_); dalloc(A.g_im, nb, roll_owned_);
        dalloc(A.g_fs, d_.n_shapes, roll_owned_); dalloc(A.g_fd, d_.n_shapes, roll_owned_);
        dalloc(A.nrow, 4 * cap, roll_owned_); dalloc(A.frow, 4 * cap, roll_owned_);
        dalloc(A.jrow, std::max<size_t>(d_.n_jrows, 1), roll_owned_);
        dalloc(A.hd, cap, roll_owned_);
        dalloc(A.yn, 4 * cap, roll_owned_); dalloc(A.yf, 4 * cap, roll_owned_);
        dalloc(A.yj, std::max<size_t>(d_.n_jrows, 1), roll_owned_);
        dalloc(A.mark, nb, roll_owned_);
        dalloc(A.epoch, 1, roll_owned_);
        check_cuda(cudaMemsetAsync(A.mark, 0, nb * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(A.epoch, 0, 4, stream_), "memset");
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }
    // Back to the state the last rollout_forward started from (its first
    // checkpoint), e.g. to run the rollout again with new parameters.
    void rollout_rewind() {
        if (!roll_done_) throw std::logic_error("rollout_forward must come first");
        load_slot(ckpt_.front());
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        host_authoritative_ = false;
    }
    void require_rollout_capacity() {
        if (d_.pair_cap != roll_cap_)
            throw std::logic_error("Pair capacity grew during a differentiable rollout; step the scene once "
                                   "before rollout_begin so the pair budget is settled");
    }
    void rollout_forward(float dt) {
        if (!roll_steps_) throw std::logic_error("rollout_begin must come first");
        roll_dt_ = dt;
        // the forward runs without sleeping, like its recompute (framed())
        struct SleepOff {
            World& w;
            explicit SleepOff(World& x) : w(x) { flip(false); }
            ~SleepOff() { flip(w.sleep_enabled_); }
            void flip(bool on) { w.d_.sleep = on; }   // the step graphs are cached per sleep mode
        } off(*this);
        for (uint32_t t0 = 0; t0 < roll_steps_; t0 += roll_every_) {
            save_slot(ckpt_[t0 / roll_every_]);
            step(dt, std::min(roll_every_, roll_steps_ - t0));
            require_rollout_capacity();
        }
        save_slot(ckpt_.back());
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        roll_done_ = true;
    }
    // One step of the segment recompute, its per-step data written to frame f.
    void framed_step(Frame& f) {
        f.parity = parity_;
        const DevState s = framed(f, parity_);
        AdjState a = adj_;
        a.x_c = f.x_c; a.x_q = f.x_q;
        enqueue_adjoint_save_start(s, a, stream_);
        enqueue_broadphase(s, stream_);
        enqueue_narrowphase(s, stream_);
        enqueue_solver(s, stream_, {}, &br_);
        enqueue_copy_set(f.cur, sets_[parity_], d_.pair_cap, stream_);
        d2d(f.counters, d_.counters, size_t(kCntSlots));
        last_cur_ = parity_;
        parity_ ^= 1;
    }
    // One segment of the backward pass: its recompute into frames [0, len)
    // and the step adjoints in reverse, as one CUDA graph per (start parity,
    // length), captured on first use and replayed for the other segments
    // (the frames and the live buffers they read are the same each time;
    // the checkpoint is loaded before the launch).
    void segment_backward(uint32_t len) {
        if (seg_dt_ != roll_dt_) { release_segment_graphs(); seg_dt_ = roll_dt_; }
        const int p0 = parity_;
        SegGraph* g = nullptr;
        for (auto& x : seg_graphs_) if (x.parity == p0 && x.len == len) g = &x;
        if (!g) {
            cudaGraph_t graph;
            check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
            for (uint32_t t = 0; t < len; ++t) framed_step(frames_[t]);
            for (int t = int(len) - 1; t >= 0; --t) frame_adjoint(frames_[t]);
            check_cuda(cudaStreamEndCapture(stream_, &graph), "end capture");
            SegGraph ng;
            ng.parity = p0;
            ng.len = len;
            check_cuda(cudaGraphInstantiateWithFlags(&ng.exec, graph, cudaGraphInstantiateFlagUseNodePriority),
                       "instantiate");
            cudaGraphDestroy(graph);
            seg_graphs_.push_back(ng);
            g = &seg_graphs_.back();
            parity_ = p0;   // the capture advanced the host-side parities; replay below does it again
        }
        for (uint32_t t = 0; t < len; ++t) {
            frames_[t].parity = parity_;
            last_cur_ = parity_;
            parity_ ^= 1;
        }
        check_cuda(cudaGraphLaunch(g->exec, stream_), "segment launch");
    }
    // The step's adjoint over frame f.
    void frame_adjoint(const Frame& f) {
        DevState s = framed(f, f.parity);
        s.cur = f.cur;
        s.counters = f.counters;
        AdjState a = adj_;
        a.x_c = f.x_c; a.x_q = f.x_q;
        enqueue_adjoint_step(s, a, stream_);
    }
    void rollout_backward(const float* gc, const float* gq, const float* gv, const float* gw,
                          float* gv0, float* gw0, float* gmass, float* gfs, float* gfd) {
        if (!roll_done_) throw std::logic_error("rollout_forward must come first");
        const uint32_t nb = d_.n_bodies, ns = d_.n_shapes;
        auto up3 = [&](float4* dst, const float* src) {
            std::vector<float4> h(nb, make_float4(0, 0, 0, 0));
            if (src) for (uint32_t i = 0; i < nb; ++i) h[i] = make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0);
            upload(dst, h, stream_);
            check_cuda(cudaStreamSynchronize(stream_), "sync");
        };
        up3(adj_.c, gc); up3(adj_.v, gv); up3(adj_.w, gw);
        {
            std::vector<float4> h(nb, make_float4(0, 0, 0, 0));
            if (gq) for (uint32_t i = 0; i < nb; ++i) h[i] = make_float4(gq[4 * i], gq[4 * i + 1], gq[4 * i + 2], gq[4 * i + 3]);
            upload(adj_.q, h, stream_);
        }
        check_cuda(cudaMemsetAsync(adj_.g_im, 0, nb * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(adj_.g_iI, 0, nb * 16, stream_), "memset");
        check_cuda(cudaMemsetAsync(adj_.g_fs, 0, ns * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(adj_.g_fd, 0, ns * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "memset");
        const uint32_t nseg = uint32_t(ckpt_.size() - 1);
        for (int seg = int(nseg) - 1; seg >= 0; --seg) {
            const uint32_t t0 = uint32_t(seg) * roll_every_, t1 = std::min(roll_steps_, t0 + roll_every_);
            load_slot(ckpt_[seg]);
            segment_backward(t1 - t0);
        }
        check_cuda(cudaStreamSynchronize(stream_), "backward sync");
        if (read_err()) throw std::overflow_error("Device error during the backward pass");
        // outputs
        std::vector<float4> v(nb), w(nb), iI(nb), inv(nb);
        std::vector<float> im(nb);
        check_cuda(cudaMemcpy(v.data(), adj_.v, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(w.data(), adj_.w, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(iI.data(), adj_.g_iI, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(im.data(), adj_.g_im, nb * 4, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(inv.data(), d_.b_inv, nb * 16, cudaMemcpyDeviceToHost), "read");
        for (uint32_t i = 0; i < nb; ++i) {
            if (gv0) { gv0[3 * i] = v[i].x; gv0[3 * i + 1] = v[i].y; gv0[3 * i + 2] = v[i].z; }
            if (gw0) { gw0[3 * i] = w[i].x; gw0[3 * i + 1] = w[i].y; gw0[3 * i + 2] = w[i].z; }
            // inverse mass and inertia scale as 1/m: dm = -im (im g_im + iI . g_iI)
            if (gmass) gmass[i] = -inv[i].w * (inv[i].w * im[i] + inv[i].x * iI[i].x + inv[i].y * iI[i].y + inv[i].z * iI[i].z);
        }
        if (gfs) check_cuda(cudaMemcpy(gfs, adj_.g_fs, ns * 4, cudaMemcpyDeviceToHost), "read");
        if (gfd) check_cuda(cudaMemcpy(gfd, adj_.g_fd, ns * 4, cudaMemcpyDeviceToHost), "read");
        // leave the world at the end of the rollout
        load_slot(ckpt_.back());
        check_cuda(cudaStreamSynchronize(stream_), "sync");
    }
    // Friction patches of the touching managers (pair order) after the last
    // step: anchor count and the anchors in both bodies' mass frames.
    uint64_t read_friction_anchors(uint32_t* anchors, float* a0, float* a1, uint64_t cap) {
        if (!uploaded_) return 0;
        const auto c = read_counters();
        if (!anchors || !c.man) return c.man;
        const uint64_t n = std::min<uint64_t>(c.man, cap);
        std::vector<uint32_t> ml(n);
        check_cuda(cudaMemcpy(ml.data(), d_.man_list, n * 4, cudaMemcpyDeviceToHost), "read");
        std::vector<FrictionHist> h(d_.pair_cap);
        check_cuda(cudaMemcpy(h.data(), sets_[last_cur_].fric, size_t(d_.pair_cap) * sizeof(FrictionHist),
                              cudaMemcpyDeviceToHost), "read");
        for (uint64_t m = 0; m < n; ++m) {
            const FrictionHist& f = h[ml[m]];
            anchors[m] = (f.meta & 255u) | (f.meta & 0xfc00u);
            for (int k = 0; k < 2; ++k)
                for (int i = 0; i < 3; ++i) {
                    a0[6 * m + 3 * k + i] = f.a0[k][i];
                    a1[6 * m + 3 * k + i] = f.a1[k][i];
                }
        }
        return c.man;
    }
    // Mass-frame centres and orientations of all bodies (loss inputs).
    void read_mass_frames(float* c3, float* q4) {
        ensure_device();
        const uint32_t nb = d_.n_bodies;
        std::vector<float4> p(nb), q(nb), mlp(nb), mlq(nb);
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        check_cuda(cudaMemcpy(p.data(), d_.b_p, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(q.data(), d_.b_q, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(mlp.data(), d_.b_ml_p, nb * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(mlq.data(), d_.b_ml_q, nb * 16, cudaMemcpyDeviceToHost), "read");
        for (uint32_t i = 0; i < nb; ++i) {
            const qt bq = {q[i].x, q[i].y, q[i].z, q[i].w};
            const v3 off = rot_sc(bq, {mlp[i].x, mlp[i].y, mlp[i].z});
            const qt mq = qmul(bq, {mlq[i].x, mlq[i].y, mlq[i].z, mlq[i].w});
            if (c3) { c3[3 * i] = p[i].x + off.x; c3[3 * i + 1] = p[i].y + off.y; c3[3 * i + 2] = p[i].z + off.z; }
            if (q4) { q4[4 * i] = mq.x; q4[4 * i + 1] = mq.y; q4[4 * i + 2] = mq.z; q4[4 * i + 3] = mq.w; }
        }
    }

    // ---------------- contact events ----------------
    // WorldOptions::contact_notifications (world.h:61).  Event buffers are
    // allocated only while notifications are on; the step graph is rebuilt.
    // Sleeping (on by default, as in the reference scene).  Turning it off
    // wakes every body.
    void set_sleeping(bool on) {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        if (on == sleep_enabled_) return;
        if (uploaded_ && !host_authoritative_) {
            if (!on) {
                enqueue_wake_bodies(d_, stream_);
                check_cuda(cudaStreamSynchronize(stream_), "sync");
            }
        } else {
            for (auto& b : bodies_) if (!on && b.dynamic) b.wake_up();
            mass_dirty_ = true;
        }
        sleep_enabled_ = on;
        d_.sleep = on;
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
    }
    bool sleeping_enabled() const { return sleep_enabled_; }
    void read_sleep_state(float* wake, uint32_t* flags, float* motion6, uint32_t* counted, uint32_t n) {
        if (n != bodies_.size()) throw std::invalid_argument("Body count mismatch");
        if (!uploaded_ || host_authoritative_) {
            for (uint32_t i = 0; i < n; ++i) {
                const HostBody& b = bodies_[i];
                if (wake) wake[i] = b.dynamic ? b.wake : 0.0f;
                if (flags) flags[i] = b.dynamic ? b.sleep : 0u;
                if (motion6) for (int k = 0; k < 6; ++k) motion6[6 * size_t(i) + k] = b.dynamic ? b.sacc[k] : 0.0f;
                if (counted) counted[i] = 0u;
            }
            return;
        }
        std::vector<float4> acc(motion6 ? 2 * size_t(n) : 0);
        if (wake) check_cuda(cudaMemcpyAsync(wake, d_.b_wake, size_t(n) * 4, cudaMemcpyDeviceToHost, stream_), "read");
        if (flags) check_cuda(cudaMemcpyAsync(flags, d_.b_sleep, size_t(n) * 4, cudaMemcpyDeviceToHost, stream_), "read");
        if (counted) check_cuda(cudaMemcpyAsync(counted, d_.b_counted, size_t(n) * 4, cudaMemcpyDeviceToHost, stream_), "read");
        if (motion6) check_cuda(cudaMemcpyAsync(acc.data(), d_.b_sacc, size_t(n) * 32, cudaMemcpyDeviceToHost, stream_), "read");
        check_cuda(cudaStreamSynchronize(stream_), "read sync");
        if (motion6)
            for (uint32_t i = 0; i < n; ++i) {
                const float4 l = acc[2 * size_t(i)], a = acc[2 * size_t(i) + 1];
                const float r[6] = {l.x, l.y, l.z, a.x, a.y, a.z};
                std::memcpy(motion6 + 6 * size_t(i), r, sizeof r);
            }
    }
    void set_contact_notifications(bool on) {
        if (on == notify_) return;
        notify_ = on;
        d_.events = on;
        if (uploaded_ && on) alloc_events();
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
    }
    // World::contact_events / contact_event_points (world.h:466-468): the
    // last completed step's events, copied from the device on the first
    // request after the step and valid until the next step.
    void contact_events(const EventRecord** ev, uint64_t* nev, const EventPoint** pts, uint64_t* npts) {
        if (notify_ && uploaded_ && steps_done_ && ev_device_valid_ && ev_fetched_ != steps_done_) {
            check_cuda(cudaStreamSynchronize(stream_), "sync");
            uint32_t h[kCntSlots] = {};
            check_cuda(cudaMemcpy(h, d_.counters, sizeof h, cudaMemcpyDeviceToHost), "read");
            const uint64_t n_ev = uint64_t(h[kCntReported]) + h[kCntLost], n_pts = h[kCntEvPts];
            h_ev_.resize(n_ev);
            h_ev_pts_.resize(n_pts);
            if (n_ev)
                check_cuda(cudaMemcpy(h_ev_.data(), d_.ev, n_ev * sizeof(EventRecord), cudaMemcpyDeviceToHost), "read");
            if (n_pts)
                check_cuda(cudaMemcpy(h_ev_pts_.data(), d_.ev_pts, n_pts * sizeof(EventPoint), cudaMemcpyDeviceToHost), "read");
            ev_fetched_ = steps_done_;
        }
        const bool have = notify_ && ev_fetched_ == steps_done_ && steps_done_;
        *ev = have ? h_ev_.data() : nullptr;
        *nev = have ? h_ev_.size() : 0;
        *pts = have ? h_ev_pts_.data() : nullptr;
        *npts = have ? h_ev_pts_.size() : 0;
    }
    // World::force_threshold_changes (world.h:472): the last completed
    // step's changes, copied from the device on the first request after it,
    // valid until the next step.  Empty after a collision pass.
    void threshold_changes(const ForceThresholdRecord** out, uint64_t* n) {
        if (thresholds_ && uploaded_ && steps_done_ && th_device_valid_ && th_fetched_ != steps_done_) {
            check_cuda(cudaStreamSynchronize(stream_), "sync");
            uint32_t cnt = 0;
            check_cuda(cudaMemcpy(&cnt, d_.counters + kCntThChanges, 4, cudaMemcpyDeviceToHost), "read");
            h_th_.resize(cnt);
            if (cnt)
                check_cuda(cudaMemcpy(h_th_.data(), d_.th_changes, size_t(cnt) * sizeof(ForceThresholdRecord),
                                      cudaMemcpyDeviceToHost), "read");
            th_fetched_ = steps_done_;
        }
        const bool have = thresholds_ && th_device_valid_ && th_fetched_ == steps_done_ && steps_done_;
        *out = have ? h_th_.data() : nullptr;
        *n = have ? h_th_.size() : 0;
    }
    void collide() {
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        for (int attempt = 0; attempt < 8; ++attempt) {
            snapshot(1);
            check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "memset");
            const DevState s = view(parity_);
            enqueue_broadphase(s, stream_);
            enqueue_narrowphase(s, stream_);
            check_cuda(cudaGetLastError(), "collide launch");
            const uint32_t err = read_err();
            if (!err) {
                // a collision pass solves nothing: the last step's exceeded
                // force pairs stay the previous generation of the next step
                if (d_.thresholds) enqueue_copy_threshold_set(th_sets_[parity_], th_sets_[last_cur_], d_.pair_cap, stream_);
                check_cuda(cudaStreamSynchronize(stream_), "collide sync");
                last_cur_ = parity_;
                parity_ ^= 1;
                th_device_valid_ = false;
                return;
            }
            restore();
            if (err & kErrPairCapacity) { grow_pairs(d_.pair_cap * 2u); continue; }
            raise_step_error(err);
        }
    }
    void synchronize() { check_cuda(cudaStreamSynchronize(stream_), "synchronize"); }

    // One step launched eagerly (not from the graph) with a CUDA event on the
    // world's stream at every stage boundary; returns per-stage milliseconds
    // in Stage order.
    void profile_step(float dt, float* ms, uint32_t n) {
        if (!std::isfinite(dt) || dt <= 0.0f) throw std::invalid_argument("timestep must be finite and positive");
        check_cuda(cudaSetDevice(device_), "cudaSetDevice");
        ensure_device();
        struct Ctx { cudaEvent_t ev[kStEnd + 1]; bool seen[kStEnd + 1]; } ctx{};
        for (int i = 0; i <= kStEnd; ++i) check_cuda(cudaEventCreate(&ctx.ev[i]), "event");
        StageHook hook;
        hook.ctx = &ctx;
        hook.fn = [](void* c, int stage, cudaStream_t st) {
            auto* x = static_cast<Ctx*>(c);
            cudaEventRecord(x->ev[stage], st);
            x->seen[stage] = true;
        };
        snapshot(1);
        d_.dt = dt;
        check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "memset");
        const DevState s = view(parity_);
        enqueue_broadphase(s, stream_, hook);
        enqueue_narrowphase(s, stream_, hook);
        enqueue_solver(s, stream_, hook, &br_);
        check_cuda(cudaGetLastError(), "profile launch");
        const uint32_t err = read_err();
        last_cur_ = parity_;
        parity_ ^= 1;
        for (uint32_t i = 0; i < n && i < uint32_t(kStEnd); ++i) {
            float t = 0.0f;
            if (ctx.seen[i] && ctx.seen[i + 1]) cudaEventElapsedTime(&t, ctx.ev[i], ctx.ev[i + 1]);
            ms[i] = t;
        }
        for (int i = 0; i <= kStEnd; ++i) cudaEventDestroy(ctx.ev[i]);
        if (err) {
            restore();
            th_device_valid_ = false;
            raise_step_error(err);
        }
        ++steps_done_;
        th_device_valid_ = true;
    }
    uint32_t kernels_per_step() const { return kernels_per_step_; }

    void read_bodies(float* out, uint32_t n) {
        if (n != bodies_.size()) throw std::invalid_argument("Body count mismatch");
        if (!uploaded_ || host_authoritative_) {
            for (uint32_t i = 0; i < n; ++i) pack_host(i, out + 14 * size_t(i));
            return;
        }
        // packed on the device, one copy into the caller's buffer
        if (!d_pack_) dalloc(d_pack_, 14 * size_t(d_.n_bodies), owned_);
        enqueue_pack_bodies(d_, d_pack_, stream_);
        check_cuda(cudaGetLastError(), "pack");
        check_cuda(cudaMemcpyAsync(out, d_pack_, size_t(n) * 56, cudaMemcpyDeviceToHost, stream_), "read");
        check_cuda(cudaStreamSynchronize(stream_), "read sync");
    }
    void body_state(uint32_t id, fyzz_b200_body_state_t* out) {
        require_body(id);
        float rec[14];
        if (!uploaded_ || host_authoritative_) {
            pack_host(id, rec);
        } else {
            float4 t[4];
            uint32_t sl = 0;
            check_cuda(cudaMemcpyAsync(&t[0], d_.b_p + id, 16, cudaMemcpyDeviceToHost, stream_), "read");
            check_cuda(cudaMemcpyAsync(&t[1], d_.b_v + id, 16, cudaMemcpyDeviceToHost, stream_), "read");
            check_cuda(cudaMemcpyAsync(&t[2], d_.b_q + id, 16, cudaMemcpyDeviceToHost, stream_), "read");
            check_cuda(cudaMemcpyAsync(&t[3], d_.b_w + id, 16, cudaMemcpyDeviceToHost, stream_), "read");
            check_cuda(cudaMemcpyAsync(&sl, d_.b_sleep + id, 4, cudaMemcpyDeviceToHost, stream_), "read");
            check_cuda(cudaStreamSynchronize(stream_), "read sync");
            const float r[14] = {t[0].x, t[0].y, t[0].z, t[1].x, t[1].y, t[1].z, t[2].x, t[2].y, t[2].z, t[2].w,
                                 t[3].x, t[3].y, t[3].z, (sl & kSleeping) ? 1.0f : 0.0f};
            std::memcpy(rec, r, sizeof rec);
        }
        std::memcpy(out->position, rec, 12);
        std::memcpy(out->velocity, rec + 3, 12);
        std::memcpy(out->orientation, rec + 6, 16);
        std::memcpy(out->angular_velocity, rec + 10, 12);
        out->sleeping = rec[13] != 0.0f ? 1 : 0;
    }
    void write_velocities(const float* rec, uint32_t n, uint32_t stride = 6, uint32_t lin = 0, uint32_t ang = 3) {
        if (n != bodies_.size()) throw std::invalid_argument("Body count mismatch");
        if (stride < 3 || lin + 3 > stride || ang + 3 > stride)
            throw std::invalid_argument("Velocity offsets must lie inside the record");
        ensure_device();
        // one copy of the caller's records, unpacked (and every body woken)
        // on the device; the caller's buffer is free again on return
        if (stride > vel_stride_cap_) {
            dalloc(d_vel6_, size_t(stride) * d_.n_bodies, owned_);
            vel_stride_cap_ = stride;
        }
        check_cuda(cudaMemcpyAsync(d_vel6_, rec, size_t(n) * stride * 4, cudaMemcpyHostToDevice, stream_), "write");
        enqueue_unpack_velocities(d_, d_vel6_, stride, lin, ang, stream_);
        check_cuda(cudaGetLastError(), "unpack");
        check_cuda(cudaStreamSynchronize(stream_), "write sync");
    }
    void counts(uint64_t* out) {
        out[0] = bodies_.size(); out[1] = shapes_.size(); out[2] = scene_body_begin_.size();
        out[3] = out[4] = out[5] = out[6] = out[7] = out[10] = out[11] = 0;
        out[8] = live_joints(); out[9] = steps_done_;
        if (!uploaded_) return;
        const auto c = read_counters();
        out[3] = c.pairs; out[4] = c.man; out[6] = c.desc; out[7] = c.isl;
        std::vector<uint32_t> cnt(c.pairs), found(c.pairs), lost(c.prev_pairs);
        std::vector<ManagerHeader> mh(c.man);
        if (c.pairs) {
            check_cuda(cudaMemcpy(cnt.data(), sets_[last_cur_].count, size_t(c.pairs) * 4, cudaMemcpyDeviceToHost), "read");
            check_cuda(cudaMemcpy(found.data(), d_.found_flag, size_t(c.pairs) * 4, cudaMemcpyDeviceToHost), "read");
        }
        if (c.prev_pairs)
            check_cuda(cudaMemcpy(lost.data(), d_.lost_flag, size_t(c.prev_pairs) * 4, cudaMemcpyDeviceToHost), "read");
        if (c.man && steps_done_)
            check_cuda(cudaMemcpy(mh.data(), d_.mh, size_t(c.man) * sizeof(ManagerHeader), cudaMemcpyDeviceToHost), "read");
        uint64_t pts = 0, fl = 0, frows = 0;
        for (auto x : cnt) pts += x;
        for (auto x : found) fl += x;
        for (auto x : lost) fl += x;
        for (const auto& h : mh) frows += 2u * h.anchors;
        out[5] = pts;
        out[10] = frows;
        out[11] = fl;
    }
    void device_view(fyzz_b200_device_view_t* v) {
        ensure_device();
        v->position = d_.b_p; v->orientation = d_.b_q; v->velocity = d_.b_v; v->angular_velocity = d_.b_w;
        v->n_bodies = d_.n_bodies; v->n_shapes = d_.n_shapes; v->stream = stream_;
    }
    uint64_t read_pairs(int which, uint32_t* out, uint64_t cap) {
        if (!uploaded_) return 0;
        const auto c = read_counters();
        const ManagerSet& cur = sets_[last_cur_];
        const ManagerSet& prev = sets_[last_cur_ ^ 1];
        const uint32_t n = which == 2 ? c.prev_pairs : c.pairs;
        std::vector<uint64_t> keys(n);
        std::vector<uint32_t> flag(n, 1u);
        if (n) {
            check_cuda(cudaMemcpy(keys.data(), which == 2 ? prev.key : cur.key, size_t(n) * 8, cudaMemcpyDeviceToHost), "read");
            if (which == 1) check_cuda(cudaMemcpy(flag.data(), d_.found_flag, size_t(n) * 4, cudaMemcpyDeviceToHost), "read");
            if (which == 2) check_cuda(cudaMemcpy(flag.data(), d_.lost_flag, size_t(n) * 4, cudaMemcpyDeviceToHost), "read");
        }
        uint64_t k = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (!flag[i]) continue;
            if (out && k < cap) { out[2 * k] = uint32_t(keys[i] >> 32); out[2 * k + 1] = uint32_t(keys[i]); }
            ++k;
        }
        return k;
    }
    uint64_t read_manifolds(uint32_t* pairs, uint32_t* counts, float* points, uint64_t cap) {
        if (!uploaded_) return 0;
        const auto c = read_counters();
        const ManagerSet& cur = sets_[last_cur_];
        std::vector<uint64_t> keys(c.pairs);
        std::vector<uint32_t> cnt(c.pairs);
        std::vector<ContactPt> pts(size_t(c.pairs) * 4);
        if (c.pairs) {
            check_cuda(cudaMemcpy(keys.data(), cur.key, size_t(c.pairs) * 8, cudaMemcpyDeviceToHost), "read");
            check_cuda(cudaMemcpy(cnt.data(), cur.count, size_t(c.pairs) * 4, cudaMemcpyDeviceToHost), "read");
            check_cuda(cudaMemcpy(pts.data(), d_.pts, size_t(c.pairs) * 4 * sizeof(ContactPt), cudaMemcpyDeviceToHost), "read");
        }
        uint64_t k = 0;
        for (uint32_t i = 0; i < c.pairs; ++i) {
            if (!cnt[i]) continue;
            if (pairs && k < cap) {
                pairs[2 * k] = uint32_t(keys[i] >> 32);
                pairs[2 * k + 1] = uint32_t(keys[i]);
                counts[k] = cnt[i];
                for (uint32_t j = 0; j < 4; ++j) {
                    float* o = points + 28 * k + 7 * j;
                    if (j < cnt[i]) {
                        const ContactPt& p = pts[4 * size_t(i) + j];
                        std::memcpy(o, p.p, 12); std::memcpy(o + 3, p.n, 12); o[6] = p.sep;
                    } else {
                        std::memset(o, 0, 28);
                    }
                }
            }
            ++k;
        }
        return k;
    }
    void read_bounds(uint32_t* out, uint32_t n) {
        if (n != shapes_.size()) throw std::invalid_argument("Shape count mismatch");
        ensure_device();
        std::vector<uint4> lo(n), hi(n);
        check_cuda(cudaMemcpy(lo.data(), d_.s_lo, size_t(n) * 16, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(hi.data(), d_.s_hi, size_t(n) * 16, cudaMemcpyDeviceToHost), "read");
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t* o = out + 6 * size_t(i);
            o[0] = lo[i].x; o[1] = lo[i].y; o[2] = lo[i].z; o[3] = hi[i].x; o[4] = hi[i].y; o[5] = hi[i].z;
        }
    }
    uint64_t read_sorted_min_x(uint32_t scene, uint32_t* values, uint32_t* ids, uint64_t cap) {
        if (scene >= scene_body_begin_.size()) throw std::out_of_range("Unknown scene");
        ensure_device();
        const uint32_t b = h_fbegin_[scene], e = h_fbegin_[scene + 1];
        const uint64_t n = e - b;
        if (values && n) {
            const uint64_t m = std::min<uint64_t>(n, cap);
            check_cuda(cudaMemcpy(values, d_.srt_key + b, m * 4, cudaMemcpyDeviceToHost), "read");
            check_cuda(cudaMemcpy(ids, d_.srt_id + b, m * 4, cudaMemcpyDeviceToHost), "read");
        }
        return n;
    }
    uint64_t read_levels(uint32_t* levels, uint64_t cap) {
        if (!uploaded_) return 0;
        const auto c = read_counters();
        if (levels && c.desc)
            check_cuda(cudaMemcpy(levels, d_.d_level, std::min<uint64_t>(c.desc, cap) * 4, cudaMemcpyDeviceToHost), "read");
        return c.desc;
    }
    // Awake islands of the last step: descriptors and partition levels each.
    uint64_t read_islands(uint32_t* descriptors, uint32_t* levels, uint64_t cap) {
        if (!uploaded_) return 0;
        const auto c = read_counters();
        const uint64_t n = std::min<uint64_t>(c.isl, cap);
        if ((descriptors || levels) && n) {
            std::vector<uint32_t> b(n + 1), e(n);
            check_cuda(cudaMemcpy(b.data(), d_.isl_begin, (n + 1) * 4, cudaMemcpyDeviceToHost), "read");
            check_cuda(cudaMemcpy(e.data(), d_.isl_end, n * 4, cudaMemcpyDeviceToHost), "read");
            for (uint64_t i = 0; i < n; ++i) {
                if (descriptors) descriptors[i] = b[i + 1] - b[i];
                if (levels) levels[i] = e[i];
            }
        }
        return c.isl;
    }
    void read_step_counters(uint32_t* out, uint32_t n) {
        if (n > uint32_t(kCntSlots)) throw std::invalid_argument("At most kCntSlots counters");
        if (!uploaded_) { for (uint32_t i = 0; i < n; ++i) out[i] = 0; return; }
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        check_cuda(cudaMemcpy(out, d_.counters, size_t(n) * 4, cudaMemcpyDeviceToHost), "read");
    }
    uint32_t error_bits() const { return last_err_; }
    uint32_t last_shape() const { return uint32_t(shapes_.size() - 1); }
    size_t n_bodies() const { return bodies_.size(); }

private:
    struct Counters { uint32_t pairs, prev_pairs, man, desc, isl; };
    Counters read_counters() {
        uint32_t h[8] = {};
        check_cuda(cudaStreamSynchronize(stream_), "sync");
        check_cuda(cudaMemcpy(h, d_.counters, sizeof h, cudaMemcpyDeviceToHost), "read");
        uint32_t np = 0, npp = 0, ni = 0;
        check_cuda(cudaMemcpy(&np, sets_[last_cur_].n, 4, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(&npp, sets_[last_cur_ ^ 1].n, 4, cudaMemcpyDeviceToHost), "read");
        check_cuda(cudaMemcpy(&ni, d_.n_isl, 4, cudaMemcpyDeviceToHost), "read");
        return {np, npp, h[kCntMan], h[kCntDesc], ni};
    }
    void pack_host(uint32_t i, float* o) const {
        const HostBody& b = bodies_[i];
        o[0] = b.p[0]; o[1] = b.p[1]; o[2] = b.p[2];
        o[3] = b.v[0]; o[4] = b.v[1]; o[5] = b.v[2];
        o[6] = b.q[0]; o[7] = b.q[1]; o[8] = b.q[2]; o[9] = b.q[3];
        o[10] = b.w[0]; o[11] = b.w[1]; o[12] = b.w[2];
        o[13] = ((b.dynamic || b.kinematic) && (b.sleep & kSleeping)) ? 1.0f : 0.0f;
    }
    DevState view(int parity) const {
        DevState s = d_;
        s.cur = sets_[parity];
        s.prev = sets_[parity ^ 1];
        s.th_cur = th_sets_[parity];
        s.th_prev = th_sets_[parity ^ 1];
        return s;
    }
    uint32_t read_err() {
        check_cuda(cudaMemcpyAsync(host_err_, d_.err, 4, cudaMemcpyDeviceToHost, stream_), "err");
        check_cuda(cudaStreamSynchronize(stream_), "step sync");
        last_err_ = host_err_[0];
        return last_err_;
    }
    void run_steps(float dt, uint32_t steps) {
        if (dt != graph_dt_) {
            for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
            graph_dt_ = dt;
        }
        d_.dt = dt;
        check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "memset");
        for (uint32_t i = 0; i < steps; ++i) {
            if (replay_pending_) {
                // the replayed order is one step's input: launched eagerly,
                // outside the cached step graphs
                DevState s = view(parity_);
                s.replay = true;
                enqueue_broadphase(s, stream_);
                enqueue_narrowphase(s, stream_);
                enqueue_solver(s, stream_, {}, &br_);
                check_cuda(cudaGetLastError(), "replay launch");
                replay_pending_ = false;
                last_cur_ = parity_;
                parity_ ^= 1;
                continue;
            }
            cudaGraphExec_t& exec = graphs_[parity_ + (d_.sleep ? 2 : 0)];
            if (!exec) {
                cudaGraph_t g;
                check_cuda(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "capture");
                const DevState s = view(parity_);
                enqueue_broadphase(s, stream_);
                enqueue_narrowphase(s, stream_);
                enqueue_solver(s, stream_, {}, &br_);
                check_cuda(cudaStreamEndCapture(stream_, &g), "end capture");
                size_t nn = 0;
                check_cuda(cudaGraphGetNodes(g, nullptr, &nn), "graph nodes");
                std::vector<cudaGraphNode_t> nodes(nn);
                check_cuda(cudaGraphGetNodes(g, nodes.data(), &nn), "graph nodes");
                uint32_t kernels = 0;
                for (auto nd : nodes) {
                    cudaGraphNodeType t;
                    if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++kernels;
                }
                kernels_per_step_ = kernels;
                // kernel-node priorities (the largest islands' kernels) are honoured
                check_cuda(cudaGraphInstantiateWithFlags(&exec, g, cudaGraphInstantiateFlagUseNodePriority),
                           "instantiate");
                cudaGraphDestroy(g);
            }
            check_cuda(cudaGraphLaunch(exec, stream_), "graph launch");
            last_cur_ = parity_;
            parity_ ^= 1;
        }
    }
    // Failure atomicity (Scene::step's checkpoint and rollback,
    // scene.cpp:9706-10020, 11013-11016): the bodies and the device
    // counters (the friction-history epoch among them) are saved before each
    // launch.  The contact-manager generation the first step reads is only
    // read by that step; a batch of several steps writes it again from its
    // second step on, so for a batch its live records are saved as well.  A
    // rollback therefore keeps every PCM cache, friction history and touch
    // count, and a retried batch runs exactly as a batch that never failed.
    void snapshot(uint32_t steps) {
        snap_replay_ = replay_pending_;
        const size_t n = size_t(d_.n_bodies) * 16;
        check_cuda(cudaMemcpyAsync(bk_counters_, d_.counters, kCntSlots * 4, cudaMemcpyDeviceToDevice, stream_),
                   "snapshot");
        snap_multi_ = steps > 1;
        if (snap_multi_) {
            if (!bk_set_.key) {
                const size_t cap = d_.pair_cap;
                dalloc(bk_set_.key, cap, pair_owned_); dalloc(bk_set_.cache, cap, pair_owned_);
                dalloc(bk_set_.fric, cap, pair_owned_); dalloc(bk_set_.count, cap, pair_owned_);
                dalloc(bk_set_.n, 1, pair_owned_);
            }
            enqueue_copy_set(bk_set_, sets_[last_cur_], d_.pair_cap, stream_);
            if (d_.thresholds) enqueue_copy_threshold_set(bk_th_, th_sets_[last_cur_], d_.pair_cap, stream_);
        }
        check_cuda(cudaMemcpyAsync(bk_p_, d_.b_p, n, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_q_, d_.b_q, n, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_v_, d_.b_v, n, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_w_, d_.b_w, n, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_wake_, d_.b_wake, n / 4, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_sleep_, d_.b_sleep, n / 4, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        check_cuda(cudaMemcpyAsync(bk_sacc_, d_.b_sacc, 2 * n, cudaMemcpyDeviceToDevice, stream_), "snapshot");
        snap_parity_ = parity_;
        snap_last_ = last_cur_;
    }
    void restore() {
        const size_t n = size_t(d_.n_bodies) * 16;
        check_cuda(cudaMemcpyAsync(d_.b_p, bk_p_, n, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_q, bk_q_, n, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_v, bk_v_, n, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_w, bk_w_, n, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_wake, bk_wake_, n / 4, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_sleep, bk_sleep_, n / 4, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.b_sacc, bk_sacc_, 2 * n, cudaMemcpyDeviceToDevice, stream_), "restore");
        check_cuda(cudaMemcpyAsync(d_.counters, bk_counters_, kCntSlots * 4, cudaMemcpyDeviceToDevice, stream_),
                   "restore");
        // the generation the batch started from, as the reference's journal
        // restores its contact managers
        if (snap_multi_) {
            enqueue_copy_set(sets_[snap_last_], bk_set_, d_.pair_cap, stream_);
            if (d_.thresholds) enqueue_copy_threshold_set(th_sets_[snap_last_], bk_th_, d_.pair_cap, stream_);
        }
        check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "restore");
        check_cuda(cudaStreamSynchronize(stream_), "restore sync");
        replay_pending_ = snap_replay_;
        parity_ = snap_parity_;
        last_cur_ = snap_last_;
    }

    void release_device() {
        release_rollout();
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
        for (void* p : owned_) cudaFree(p);
        owned_.clear();
        d_.j_a = d_.j_b = d_.j_kind = d_.j_row = nullptr;
        d_.j_len = nullptr;
        d_.j_la = d_.j_lb = d_.j_qa = d_.j_qb = nullptr;
        d_.jrow = nullptr;
        joint_cap_ = jrow_cap_ = 0;
        d_.rp_keys = nullptr; d_.rp_pos = nullptr; d_.rp_jrank = nullptr;
        replay_cap_ = replay_jcap_ = 0;
        replay_pending_ = false;
        d_pack_ = nullptr;
        d_vel6_ = nullptr;
        vel_stride_cap_ = 0;
        for (void* p : pair_owned_) cudaFree(p);
        pair_owned_.clear();
        uploaded_ = false;
    }

    void alloc_pairs(uint32_t cap) {
        for (void* p : pair_owned_) cudaFree(p);
        pair_owned_.clear();
        bk_set_ = ManagerSet{};
        bk_th_ = ThresholdSet{};
        th_sets_[0] = th_sets_[1] = ThresholdSet{};
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
        d_.pair_cap = cap;
        d_.desc_cap = cap + d_.n_joints + kJointReserve;
        for (int k = 0; k < 2; ++k) {
            dalloc(sets_[k].key, cap, pair_owned_);
            dalloc(sets_[k].cache, cap, pair_owned_);
            dalloc(sets_[k].fric, cap, pair_owned_);
            // friction records count only with the epoch of the previous
            // step, so unwritten ones must start at epoch 0
            check_cuda(cudaMemsetAsync(sets_[k].fric, 0, size_t(cap) * sizeof(FrictionHist), stream_), "memset");
            dalloc(sets_[k].count, cap, pair_owned_);
            dalloc(sets_[k].n, 1, pair_owned_);
            check_cuda(cudaMemsetAsync(sets_[k].n, 0, 4, stream_), "memset");
        }
        dalloc(d_.prev_idx, cap, pair_owned_);
        dalloc(d_.found_flag, cap, pair_owned_);
        dalloc(d_.lost_flag, cap, pair_owned_);
        dalloc(d_.pts, size_t(cap) * 4, pair_owned_);
        dalloc(d_.gjk_list, cap, pair_owned_);
        // the hull lists and witnesses exist only in worlds with cooked hulls
        const size_t hcap = d_.n_meshes ? size_t(cap) : 1;
        dalloc(d_.cvx_list, hcap, pair_owned_);
        dalloc(d_.cvx_gjk_list, hcap, pair_owned_);
        dalloc(d_.cvx_clip_list, hcap, pair_owned_);
        dalloc(d_.cvx_wit, 3 * hcap, pair_owned_);
        dalloc(d_.cvx_epa_list, hcap, pair_owned_);
        dalloc(d_.cvx_simplex, 12 * hcap, pair_owned_);
        dalloc(d_.man_list, cap, pair_owned_);
        dalloc(d_.mh, cap, pair_owned_);
        dalloc(d_.nrow, size_t(cap) * 4, pair_owned_);
        dalloc(d_.frow, size_t(cap) * 4, pair_owned_);
        const uint32_t dc = d_.desc_cap;
        dalloc(d_.slot_rows, (size_t(dc) + 31u) / 32u * 32u * (kSlotVecPlanes + kSlotScalarPlanes / 4), pair_owned_);
        dalloc(d_.d_key, dc, pair_owned_); dalloc(d_.d_val, dc, pair_owned_);
        dalloc(d_.d_key2, dc, pair_owned_); dalloc(d_.d_val2, dc, pair_owned_);
        dalloc(d_.d_level, dc, pair_owned_);
        dalloc(d_.d_bod, dc, pair_owned_);
        dalloc(d_.d_lbod, dc, pair_owned_);
        dalloc(d_.isl_bod, 2 * size_t(dc) + 2, pair_owned_);
        dalloc(d_.isl_nbod, size_t(dc) + 1, pair_owned_);
        for (int k = 0; k < DevState::kIslLists; ++k)
            dalloc(d_.isl_list[k], size_t(dc) / (kListMinDesc[k] + 1) + 2, pair_owned_);
        dalloc(d_.isl_begin, size_t(dc) + 1, pair_owned_);
        dalloc(d_.isl_end, size_t(dc) + 1, pair_owned_);
        dalloc(d_.tmp_flags, cap, pair_owned_);
        dalloc(d_.tmp_pos, std::max(cap, dc), pair_owned_);
        dalloc(d_.lvl_bound, 2 * size_t(dc) + 2, pair_owned_);
        const uint32_t big = std::max({cap, dc, d_.n_shapes, d_.n_finite, d_.bx_cap, 256u * 64u});
        d_.scan_tmp_words = scan_tmp_words_for(std::max<uint32_t>(big, uint32_t(radix_hist_words(big))));
        dalloc(d_.scan_tmp, d_.scan_tmp_words, pair_owned_);
        check_cuda(cudaMemsetAsync(d_.scan_tmp, 0, d_.scan_tmp_words * 4, stream_), "memset");   // scan epochs start clear
        d_.sort_hist_words = radix_hist_words(big);
        dalloc(d_.sort_hist, d_.sort_hist_words, pair_owned_);
        d_.sort_os_words = onesweep_words(big);
        dalloc(d_.sort_os, d_.sort_os_words, pair_owned_);
        check_cuda(cudaMemsetAsync(d_.sort_os, 0, d_.sort_os_words * 4, stream_), "memset");   // epochs start clear
        if (notify_) alloc_events();
        if (d_.thresholds) alloc_threshold_arrays();
    }
    // The force-threshold stream's generations (both start empty), the
    // batch backup of one, and its per-manager scratch, for the current pair
    // budget.
    void alloc_threshold_arrays() {
        const size_t cap = d_.pair_cap;
        for (auto& t : th_sets_) {
            dalloc(t.key, cap, pair_owned_); dalloc(t.impulse, cap, pair_owned_);
            dalloc(t.thr, cap, pair_owned_); dalloc(t.n, 1, pair_owned_);
            check_cuda(cudaMemsetAsync(t.n, 0, 4, stream_), "memset");
        }
        dalloc(bk_th_.key, cap, pair_owned_); dalloc(bk_th_.impulse, cap, pair_owned_);
        dalloc(bk_th_.thr, cap, pair_owned_); dalloc(bk_th_.n, 1, pair_owned_);
        dalloc(d_.th_hi, cap, pair_owned_); dalloc(d_.th_lo, cap, pair_owned_);
        dalloc(d_.th_sum, cap, pair_owned_); dalloc(d_.th_thr, cap, pair_owned_);
        dalloc(d_.th_k, cap, pair_owned_); dalloc(d_.th_v, cap, pair_owned_);
        dalloc(d_.th_k2, cap, pair_owned_); dalloc(d_.th_v2, cap, pair_owned_);
        dalloc(d_.th_run_sum, cap, pair_owned_); dalloc(d_.th_run_thr, cap, pair_owned_);
        dalloc(d_.th_f0, cap, pair_owned_); dalloc(d_.th_p0, cap, pair_owned_);
        dalloc(d_.th_f1, cap, pair_owned_); dalloc(d_.th_p1, cap, pair_owned_);
        dalloc(reinterpret_cast<ForceThresholdRecord*&>(d_.th_changes), 2 * cap, pair_owned_);
        check_cuda(cudaStreamSynchronize(stream_), "threshold arrays");
    }
    void alloc_events() {
        const size_t cap = d_.pair_cap;
        dalloc(reinterpret_cast<EventRecord*&>(d_.ev), 2 * cap, pair_owned_);
        dalloc(reinterpret_cast<EventPoint*&>(d_.ev_pts), 4 * cap, pair_owned_);
        dalloc(d_.ev_lost_key, cap, pair_owned_);
        dalloc(d_.ev_cnt, cap, pair_owned_);
        dalloc(d_.ev_pt_off, cap + 1, pair_owned_);
    }
    // After a rollback: a larger budget, with the generation the next step
    // reads carried over.
    void grow_pairs(uint32_t cap) {
        uint32_t live[2] = {0, 0};
        for (int k = 0; k < 2; ++k)
            check_cuda(cudaMemcpy(&live[k], sets_[k].n, 4, cudaMemcpyDeviceToHost), "read");
        live[last_cur_ ^ 1] = 0;   // the failed step's partial generation is not kept
        check_cuda(cudaMemsetAsync(sets_[last_cur_ ^ 1].n, 0, 4, stream_), "memset");
        resize_pairs_keeping(cap, live);
    }
    [[noreturn]] void raise_step_error(uint32_t err) {
        const std::string bits = "Device step reported error bits " + std::to_string(err);
        if (err & kErrLogic) throw std::logic_error(bits + " (a bounded device wait gave up)");
        throw std::overflow_error(bits);
    }

    void upload_bodies() {
        const uint32_t nb = uint32_t(bodies_.size());
        std::vector<float4> p(nb), q(nb), v(nb), w(nb), inv(nb), mlp(nb), mlq(nb), acc(2 * size_t(nb)),
            kt(2 * size_t(nb));
        std::vector<float> wake(nb);
        std::vector<uint32_t> sl(nb);
        for (uint32_t i = 0; i < nb; ++i) {
            const HostBody& b = bodies_[i];
            wake[i] = b.wake;
            sl[i] = (b.dynamic || b.kinematic) ? b.sleep : 0u;
            kt[2 * i] = make_float4(b.kp[0], b.kp[1], b.kp[2], 0);
            kt[2 * i + 1] = make_float4(b.kq[0], b.kq[1], b.kq[2], b.kq[3]);
            acc[2 * i] = make_float4(b.sacc[0], b.sacc[1], b.sacc[2], 0);
            acc[2 * i + 1] = make_float4(b.sacc[3], b.sacc[4], b.sacc[5], 0);
            p[i] = make_float4(b.p[0], b.p[1], b.p[2], b.inv_mass);
            q[i] = make_float4(b.q[0], b.q[1], b.q[2], b.q[3]);
            v[i] = make_float4(b.v[0], b.v[1], b.v[2], 0);
            w[i] = make_float4(b.w[0], b.w[1], b.w[2], 0);
            inv[i] = make_float4(b.inv_inertia[0], b.inv_inertia[1], b.inv_inertia[2], b.dynamic ? b.inv_mass : 0.0f);
            mlp[i] = make_float4(b.ml_p[0], b.ml_p[1], b.ml_p[2], 0);
            mlq[i] = make_float4(b.ml_q[0], b.ml_q[1], b.ml_q[2], b.ml_q[3]);
        }
        upload(d_.b_p, p, stream_); upload(d_.b_q, q, stream_); upload(d_.b_v, v, stream_);
        upload(d_.b_w, w, stream_); upload(d_.b_inv, inv, stream_);
        upload(d_.b_ml_p, mlp, stream_); upload(d_.b_ml_q, mlq, stream_);
        upload(d_.b_wake, wake, stream_); upload(d_.b_sleep, sl, stream_); upload(d_.b_sacc, acc, stream_);
        upload(d_.b_ktarget, kt, stream_);
        std::vector<float> thr(nb);
        for (uint32_t i = 0; i < nb; ++i) thr[i] = bodies_[i].report_threshold;
        upload(d_.b_thresh, thr, stream_);
        std::vector<float4> mat(shapes_.size());
        for (size_t i = 0; i < shapes_.size(); ++i)
            mat[i] = make_float4(shapes_[i].mat[0], shapes_[i].mat[1], shapes_[i].mat[2], shapes_[i].mat[3]);
        upload(d_.s_mat, mat, stream_);
        check_cuda(cudaStreamSynchronize(stream_), "upload sync");
        host_authoritative_ = false;
    }

    uint32_t live_joints() const {
        uint32_t n = 0;
        for (const auto& j : joints_) n += j.live ? 1u : 0u;
        return n;
    }
    // The device joint tables: live joints per scene, constraint slot
    // descending (scene.cpp:7153-7162), their rows, and the constraints
    // counted on each dynamic endpoint (scene.cpp:2728-2749).  The tables
    // hold kJointReserve joints (and their rows) beyond the count they were
    // sized for, so joint edits between steps only upload; a table that
    // must grow is freed and allocated again.
    void free_joint_tables() {
        void* tabs[] = {d_.j_a, d_.j_b, d_.j_len, d_.j_kind, d_.j_row, d_.j_la, d_.j_lb, d_.j_qa, d_.j_qb, d_.jrow};
        for (void* p : tabs) {
            if (!p) continue;
            auto it = std::find(owned_.begin(), owned_.end(), p);
            if (it != owned_.end()) owned_.erase(it);
            cudaFree(p);
        }
        d_.j_a = d_.j_b = d_.j_kind = d_.j_row = nullptr;
        d_.j_len = nullptr;
        d_.j_la = d_.j_lb = d_.j_qa = d_.j_qb = nullptr;
        d_.jrow = nullptr;
        joint_cap_ = jrow_cap_ = 0;
    }
    void upload_joints() {
        std::vector<HostJoint> js;
        for (const auto& j : joints_)
            if (j.live) js.push_back(j);
        std::stable_sort(js.begin(), js.end(), [](const HostJoint& a, const HostJoint& b) {
            return a.scene != b.scene ? a.scene < b.scene : a.slot > b.slot;
        });
        const size_t n = js.size();
        std::vector<uint32_t> ja(n), jb(n), jk(n), jr(n);
        std::vector<float> jl(n);
        std::vector<float4> jla(n), jlb(n), jqa(n), jqb(n);
        uint32_t nrows = 0;
        for (size_t i = 0; i < n; ++i) {
            const HostJoint& h = js[i];
            ja[i] = h.a; jb[i] = h.b; jl[i] = h.len; jk[i] = h.kind; jr[i] = nrows;
            nrows += joint_rows(h.kind);
            jla[i] = make_float4(h.la[0], h.la[1], h.la[2], 0);
            jlb[i] = make_float4(h.lb[0], h.lb[1], h.lb[2], 0);
            jqa[i] = make_float4(h.qa[0], h.qa[1], h.qa[2], h.qa[3]);
            jqb[i] = make_float4(h.qb[0], h.qb[1], h.qb[2], h.qb[3]);
        }
        d_.n_joints = uint32_t(n);
        d_.n_jrows = nrows;
        if (n > joint_cap_ || nrows > jrow_cap_ || !d_.j_a) {
            // synchronise before freeing: earlier launches may still read the old tables
            check_cuda(cudaStreamSynchronize(stream_), "joint tables");
            free_joint_tables();
            const size_t jc = n + kJointReserve, rc = size_t(nrows) + 6u * kJointReserve;
            dalloc(d_.j_a, jc, owned_); dalloc(d_.j_b, jc, owned_); dalloc(d_.j_len, jc, owned_);
            dalloc(d_.j_kind, jc, owned_); dalloc(d_.j_row, jc, owned_);
            dalloc(d_.j_la, jc, owned_); dalloc(d_.j_lb, jc, owned_);
            dalloc(d_.j_qa, jc, owned_); dalloc(d_.j_qb, jc, owned_);
            dalloc(d_.jrow, rc, owned_);
            joint_cap_ = uint32_t(jc);
            jrow_cap_ = uint32_t(rc);
        }
        std::vector<uint32_t> jcount(bodies_.size(), 0u);
        for (const auto& j : js) {
            if (bodies_[j.a].dynamic) ++jcount[j.a];
            if (bodies_[j.b].dynamic) ++jcount[j.b];
        }
        upload(d_.b_jcount, jcount, stream_);
        upload(d_.j_a, ja, stream_); upload(d_.j_b, jb, stream_); upload(d_.j_len, jl, stream_);
        upload(d_.j_kind, jk, stream_); upload(d_.j_row, jr, stream_);
        upload(d_.j_la, jla, stream_); upload(d_.j_lb, jlb, stream_);
        upload(d_.j_qa, jqa, stream_); upload(d_.j_qb, jqb, stream_);
    }
    // Joints added or retired after the device state exists: new joint
    // tables, while bodies, pairs, PCM caches and friction histories stay
    // (the reference keeps its contact managers across constraint edits).
    // Descriptor arrays hold kJointReserve joints beyond the built count;
    // past that the device state is rebuilt.
    void refresh_joints() {
        if (live_joints() > d_.desc_cap - d_.pair_cap) {
            build_device();
            return;
        }
        release_rollout();
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
        upload_joints();
        check_cuda(cudaStreamSynchronize(stream_), "joint upload");
    }
    void apply_tuning() {
        d_.isl_thread = tuning_.island_thread;
        d_.isl_warp = tuning_.island_warp;
        d_.isl_mid = tuning_.island_cta;
        d_.radix_bits = int(tuning_.radix_bits);
        d_.elem_block = tuning_.elem_block;
        d_.work_queue = tuning_.work_queue != 0;
        for (auto& g : graphs_) if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        release_segment_graphs();
    }
    void build_device() {
        release_device();
        DevState d;
        const uint32_t nb = uint32_t(bodies_.size()), ns = uint32_t(shapes_.size());
        const uint32_t nsc = uint32_t(scene_body_begin_.size());
        d.n_scenes = nsc;
        d.n_bodies = nb;
        d.n_shapes = ns;
        d.n_joints = live_joints();
        // finite ranks, scene ranges, plane pairs
        std::vector<int32_t> frank(ns, -1), dynrank(ns, -1);
        std::vector<uint32_t> sscene(ns), sbody(ns), stype(ns), static_pairs(ns, 0);
        std::vector<uint32_t> fbegin(nsc + 1, 0);
        std::vector<int32_t> plane(nsc, -1);
        uint32_t nf = 0, n_dyn_finite = 0;
        for (uint32_t sc = 0; sc < nsc; ++sc) {
            fbegin[sc] = nf;
            const uint32_t s0 = scene_shape_begin_[sc];
            const uint32_t s1 = sc + 1 < nsc ? scene_shape_begin_[sc + 1] : ns;
            for (uint32_t i = s0; i < s1; ++i)
                if (shapes_[i].type == kPlane) plane[sc] = int32_t(i);
            uint32_t owned_by_plane = 0;
            for (uint32_t i = s0; i < s1; ++i) {
                const HostShape& s = shapes_[i];
                sscene[i] = sc; sbody[i] = s.body; stype[i] = s.type;
                if (s.type == kPlane) continue;
                frank[i] = int32_t(nf++);
                if (!bodies_[s.body].dynamic || plane[sc] < 0) continue;
                ++n_dyn_finite;
                if (uint32_t(plane[sc]) < i) {
                    dynrank[i] = int32_t(owned_by_plane++);
                    ++static_pairs[uint32_t(plane[sc])];
                } else {
                    ++static_pairs[i];
                }
            }
        }
        fbegin[nsc] = nf;
        d.n_finite = nf;
        h_fbegin_ = fbegin;
        std::vector<uint32_t> small;
        std::vector<int32_t> sc_large(nsc, -1);
        d.n_large = 0;
        uint64_t large_items = 0;
        for (uint32_t sc = 0; sc < nsc; ++sc) {
            const uint32_t n = fbegin[sc + 1] - fbegin[sc];
            if (n == 0) continue;
            if (n <= d.max_small_scene) small.push_back(sc);
            else {
                if (d.n_large >= DevState::kMaxLarge) throw std::logic_error("Too many scenes above the per-CTA sort size");
                sc_large[sc] = int32_t(d.n_large);
                d.large_begin[d.n_large] = fbegin[sc];
                d.large_n[d.n_large] = n;
                ++d.n_large;
                large_items += n;
            }
        }
        d.bx_cap = uint32_t(2 * large_items);   // a shape lies in at most two z bands
        d.n_small = uint32_t(small.size());
        tuning_class_ = d.n_large ? "large_scene" : "many_scenes";
        if (!tuning_explicit_) {
            fyzz_b200_tuning_t t{8, 96, 512, 8, 256, 0};
            fyzz_b200_tuning_t table{};
            if (load_tuning(tuning_class_, table)) {
                try { validate_tuning(table); t = table; } catch (const std::invalid_argument&) {}
            }
            tuning_ = t;
        }
        d.isl_thread = tuning_.island_thread;
        d.isl_warp = tuning_.island_warp;
        d.isl_mid = tuning_.island_cta;
        d.radix_bits = int(tuning_.radix_bits);
        d.elem_block = tuning_.elem_block;
        d.work_queue = tuning_.work_queue != 0;
        d.events = notify_;
        d.sleep = sleep_enabled_;
        d.thresholds = thresholds_;
        d_ = d;
        // allocations
        dalloc(d_.sc_fbegin, nsc + 1, owned_); dalloc(d_.sc_plane, nsc, owned_);
        dalloc(d_.small_scenes, small.size(), owned_);
        dalloc(d_.b_p, nb, owned_); dalloc(d_.b_q, nb, owned_); dalloc(d_.b_v, nb, owned_); dalloc(d_.b_w, nb, owned_);
        dalloc(d_.b_inv, nb, owned_); dalloc(d_.b_ml_p, nb, owned_); dalloc(d_.b_ml_q, nb, owned_);
        dalloc(d_.b_dyn0, nb, owned_); dalloc(d_.b_dyn1, nb, owned_);
        dalloc(d_.b_flags, nb, owned_); dalloc(d_.b_scene, nb, owned_);
        dalloc(d_.b_wake, nb, owned_); dalloc(d_.b_sacc, 2 * size_t(nb), owned_); dalloc(d_.b_sleep, nb, owned_);
        dalloc(d_.b_ktarget, 2 * size_t(nb), owned_);
        dalloc(d_.b_jcount, nb, owned_); dalloc(d_.b_counted, nb, owned_);
        dalloc(d_.sl_act, nb, owned_); dalloc(d_.sl_spec, nb, owned_); dalloc(d_.sl_root, nb, owned_);
        dalloc(bk_p_, nb, owned_); dalloc(bk_q_, nb, owned_); dalloc(bk_v_, nb, owned_); dalloc(bk_w_, nb, owned_);
        dalloc(bk_wake_, nb, owned_); dalloc(bk_sleep_, nb, owned_); dalloc(bk_sacc_, 2 * size_t(nb), owned_);
        dalloc(bk_counters_, kCntSlots, owned_);
        dalloc(d_.b_thresh, nb, owned_);
        dalloc(d_.s_body, ns, owned_); dalloc(d_.s_type, ns, owned_); dalloc(d_.s_scene, ns, owned_);
        dalloc(d_.s_geom, ns, owned_); dalloc(d_.s_lp, ns, owned_); dalloc(d_.s_lq, ns, owned_);
        dalloc(d_.s_mat, ns, owned_); dalloc(d_.s_wp, ns, owned_); dalloc(d_.s_wq, ns, owned_);
        dalloc(d_.s_lo, ns, owned_); dalloc(d_.s_hi, ns, owned_);
        dalloc(d_.s_frank, ns, owned_); dalloc(d_.s_dynrank, ns, owned_); dalloc(d_.s_static_pairs, ns, owned_);
        // the sweep list: x-sorted finite shapes, then the large scenes' z-band entries
        const size_t nsw = size_t(nf) + d_.bx_cap;
        dalloc(d_.srt_key, nsw, owned_); dalloc(d_.srt_id, nsw, owned_);
        dalloc(d_.srt_key2, nf, owned_); dalloc(d_.srt_id2, nf, owned_);
        dalloc(d_.sw_rec, nsw, owned_); dalloc(d_.sw_meta, nsw, owned_);
        dalloc(d_.sw_cache, nsw * DevState::kSweepCache, owned_);
        dalloc(d_.sw_found, nsw, owned_);
        dalloc(d_.sc_large, nsc, owned_);
        if (d_.n_large) {
            dalloc(d_.bd_part, size_t(d_.n_large) * DevState::kBandStatBlocks, owned_);
            dalloc(d_.bd_par, d_.n_large, owned_);
            dalloc(d_.bd_cnt, nf, owned_); dalloc(d_.bd_off, nf, owned_); dalloc(d_.bd_n, 1, owned_);
            dalloc(d_.bd_end, size_t(d_.n_large) * DevState::kBands, owned_);
            dalloc(d_.bx_key, d_.bx_cap, owned_); dalloc(d_.bx_val, d_.bx_cap, owned_);
            dalloc(d_.bx_key2, d_.bx_cap, owned_); dalloc(d_.bx_val2, d_.bx_cap, owned_);
        }
        dalloc(d_.own_cnt, ns, owned_); dalloc(d_.own_off, ns, owned_); dalloc(d_.own_cur, ns, owned_);
        dalloc(d_.prev_bkt, ns, owned_);
        dalloc(d_.sb_dv, nb, owned_); dalloc(d_.sb_dw, nb, owned_); dalloc(d_.sb_mdv, nb, owned_);
        dalloc(d_.sb_mdw, nb, owned_); dalloc(d_.sb_v, nb, owned_); dalloc(d_.sb_w, nb, owned_);
        dalloc(d_.sb_sqrt_i, size_t(nb) * 3, owned_);
        dalloc(d_.uf_parent, nb, owned_);
        dalloc(d_.sb_mask, nb, owned_); dalloc(d_.sb_maxdyn, nb, owned_); dalloc(d_.sb_static, nb, owned_);
        dalloc(d_.sb_earliest, nb, owned_);
        dalloc(d_.n_isl, 1, owned_);
        dalloc(d_.n_man, 1, owned_);
        dalloc(d_.counters, kCntSlots, owned_);
        dalloc(d_.err, 1, owned_);
        check_cuda(cudaMemsetAsync(d_.counters, 0, kCntSlots * 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(d_.err, 0, 4, stream_), "memset");
        check_cuda(cudaMemsetAsync(d_.s_lo, 0, size_t(ns) * 16, stream_), "memset");
        check_cuda(cudaMemsetAsync(d_.s_hi, 0, size_t(ns) * 16, stream_), "memset");
        check_cuda(cudaMemsetAsync(d_.n_isl, 0, 4, stream_), "memset");
        // host tables
        std::vector<float4> dyn0(nb, make_float4(0.0f, 0.05f, 1.0e16f, 100.0f));
        std::vector<float4> dyn1(nb, make_float4(1.0e32f, FLT_MAX, 0.0f, 0.0f));
        std::vector<uint32_t> flags(nb), bscene(nb);
        for (uint32_t i = 0; i < nb; ++i) {
            flags[i] = (bodies_[i].dynamic ? kBodyDynamic : 0u) | (bodies_[i].kinematic ? kBodyKinematic : 0u);
            d_.n_kinematic += bodies_[i].kinematic ? 1u : 0u;
            bscene[i] = bodies_[i].scene;
        }
        std::vector<float4> geom(ns), lp(ns), lq(ns);
        std::vector<uint32_t> smesh(ns);
        for (uint32_t i = 0; i < ns; ++i) {
            const HostShape& s = shapes_[i];
            geom[i] = make_float4(s.half[0], s.half[1], s.half[2], s.radius);
            lp[i] = make_float4(s.lp[0], s.lp[1], s.lp[2], s.contact_offset);
            lq[i] = make_float4(s.lq[0], s.lq[1], s.lq[2], s.lq[3]);
            smesh[i] = s.mesh;
        }
        // cooked hull arenas: every mesh's vertices, faces and loops
        std::vector<uint4> mtab;
        std::vector<float4> mhalf, hv, hf;
        std::vector<uint2> hfr;
        std::vector<uint32_t> hidx;
        for (const auto& m : meshes_) {
            mtab.push_back(make_uint4(uint32_t(hv.size()), uint32_t(m->verts.size()), uint32_t(hf.size()),
                                      uint32_t(m->faces.size())));
            const float ex = m->hi[0] - m->lo[0], ey = m->hi[1] - m->lo[1], ez = m->hi[2] - m->lo[2];
            mhalf.push_back(make_float4(0.5f * ex, 0.5f * ey, 0.5f * ez, 0.5f * std::min({ex, ey, ez})));
            for (const auto& v : m->verts) hv.push_back(make_float4(v[0], v[1], v[2], 0.0f));
            const uint32_t i0 = uint32_t(hidx.size());
            for (const auto& f : m->faces) {
                hf.push_back(make_float4(f.n[0], f.n[1], f.n[2], f.d));
                hfr.push_back(make_uint2(i0 + f.first, f.count));
            }
            hidx.insert(hidx.end(), m->idx.begin(), m->idx.end());
        }
        d_.n_meshes = uint32_t(meshes_.size());
        dalloc(d_.s_mesh, ns, owned_);
        dalloc(d_.m_tab, mtab.size(), owned_); dalloc(d_.m_half, mhalf.size(), owned_);
        dalloc(d_.hv, hv.size(), owned_); dalloc(d_.hf, hf.size(), owned_);
        dalloc(d_.hfr, hfr.size(), owned_); dalloc(d_.hidx, hidx.size(), owned_);
        upload(d_.s_mesh, smesh, stream_);
        upload(d_.m_tab, mtab, stream_); upload(d_.m_half, mhalf, stream_);
        upload(d_.hv, hv, stream_); upload(d_.hf, hf, stream_);
        upload(d_.hfr, hfr, stream_); upload(d_.hidx, hidx, stream_);
        upload_joints();
        upload(d_.sc_fbegin, fbegin, stream_); upload(d_.sc_plane, plane, stream_);
        upload(d_.sc_large, sc_large, stream_);
        upload(d_.small_scenes, small, stream_);
        upload(d_.b_dyn0, dyn0, stream_); upload(d_.b_dyn1, dyn1, stream_);
        upload(d_.b_flags, flags, stream_); upload(d_.b_scene, bscene, stream_);
        upload(d_.s_body, sbody, stream_); upload(d_.s_type, stype, stream_); upload(d_.s_scene, sscene, stream_);
        upload(d_.s_geom, geom, stream_); upload(d_.s_lp, lp, stream_); upload(d_.s_lq, lq, stream_);
        upload(d_.s_frank, frank, stream_); upload(d_.s_dynrank, dynrank, stream_);
        upload(d_.s_static_pairs, static_pairs, stream_);
        uploaded_ = true;
        upload_bodies();
        // pair capacity: every plane pair plus a generous overlap budget
        const uint64_t cap = uint64_t(n_dyn_finite) + 8ull * nf + 4096ull;
        alloc_pairs(uint32_t(std::min<uint64_t>(cap, 0x7fffffffull)));
        parity_ = 0;
        last_cur_ = 1;
        topology_dirty_ = false;
        check_cuda(cudaStreamSynchronize(stream_), "build sync");
    }

    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    Branches br_;
    std::vector<HostBody> bodies_;
    std::vector<HostShape> shapes_;
    std::vector<std::shared_ptr<const CookedMesh>> meshes_;
    std::vector<HostJoint> joints_;
    std::vector<std::vector<uint32_t>> free_joints_;   // per scene: retired slots, most recent last
    bool joints_dirty_ = false;
    static constexpr uint32_t kJointReserve = 256;
    uint32_t joint_cap_ = 0, jrow_cap_ = 0;   // joints / joint rows the device tables hold
    int norm_passes_ = 2;                      // orientation normalisations of authored transforms
    fyzz_b200_tuning_t tuning_{8, 96, 512, 8, 256, 0};
    bool tuning_explicit_ = false;
    std::string tuning_class_ = "many_scenes";
    bool replay_pending_ = false, snap_replay_ = false;   // a replayed descriptor order for the next step
    uint64_t replay_cap_ = 0, replay_jcap_ = 0;
    std::vector<uint32_t> scene_body_begin_, scene_shape_begin_;
    std::vector<bool> scene_has_floor_;
    std::vector<uint32_t> h_fbegin_;
    bool topology_dirty_ = true, mass_dirty_ = false, uploaded_ = false, host_authoritative_ = true;
    DevState d_;
    ManagerSet sets_[2];
    std::vector<void*> owned_, pair_owned_;
    float4 *bk_p_ = nullptr, *bk_q_ = nullptr, *bk_v_ = nullptr, *bk_w_ = nullptr, *bk_sacc_ = nullptr;
    float* bk_wake_ = nullptr;
    float* d_pack_ = nullptr;    // read_bodies records (owned, allocated on first use)
    float* d_vel6_ = nullptr;    // write_velocities records
    uint32_t vel_stride_cap_ = 0; // floats per record d_vel6_ holds
    uint32_t* bk_sleep_ = nullptr;
    uint32_t* bk_counters_ = nullptr;
    ManagerSet bk_set_;          // a batch's starting generation (allocated on the first batch)
    ThresholdSet th_sets_[2];    // force-threshold generations, paired with sets_
    ThresholdSet bk_th_;         // a batch's starting threshold generation
    bool thresholds_ = false;    // some body has had a report threshold
    bool th_device_valid_ = false;
    uint64_t th_fetched_ = ~0ull;
    std::vector<ForceThresholdRecord> h_th_;
    bool snap_multi_ = false;
    bool sleep_enabled_ = true;
    cudaGraphExec_t graphs_[4] = {nullptr, nullptr, nullptr, nullptr};   // [parity + 2 * sleeping]
    float graph_dt_ = -1.0f;
    int parity_ = 0, last_cur_ = 1, snap_parity_ = 0, snap_last_ = 1;
    uint64_t steps_done_ = 0;
    std::vector<void*> roll_owned_;
    std::vector<Slot> ckpt_;
    std::vector<Frame> frames_;
    uint32_t roll_steps_ = 0, roll_every_ = 1, roll_cap_ = 0;
    float roll_dt_ = 1.0f / 120.0f;
    bool roll_done_ = false;
    AdjState adj_;
    struct SegGraph { int parity = 0; uint32_t len = 0; cudaGraphExec_t exec = nullptr; };
    std::vector<SegGraph> seg_graphs_;
    float seg_dt_ = -1.0f;
    bool notify_ = false;
    bool ev_device_valid_ = false;
    uint64_t ev_fetched_ = ~0ull;
    std::vector<EventRecord> h_ev_;
    std::vector<EventPoint> h_ev_pts_;
    uint32_t last_err_ = 0;
    uint32_t* host_err_ = nullptr;
    uint32_t kernels_per_step_ = 0;
};

}  // namespace fyzz::b200

// ------------------------------------------------------------------ C ABI
struct fyzz_b200_world {
    fyzz::b200::World* impl = nullptr;
    std::string error;
};
struct fyzz_b200_convex_mesh {
    std::shared_ptr<const fyzz::b200::CookedMesh> mesh;
};

namespace {
template <class F> int guarded(fyzz_b200_world* w, F&& f) {
    if (!w || !w->impl) return FYZZ_B200_INVALID_ARGUMENT;
    try {
        f(*w->impl);
        w->error.clear();
        return FYZZ_B200_OK;
    } catch (const std::invalid_argument& e) {
        w->error = e.what(); return FYZZ_B200_INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        w->error = e.what(); return FYZZ_B200_INVALID_ARGUMENT;
    } catch (const std::overflow_error& e) {
        w->error = e.what(); return FYZZ_B200_OVERFLOW;
    } catch (const std::logic_error& e) {
        w->error = e.what(); return FYZZ_B200_LOGIC_ERROR;
    } catch (const std::exception& e) {
        w->error = e.what(); return FYZZ_B200_RUNTIME_ERROR;
    }
}
}  // namespace

extern "C" {

int fyzz_b200_create(int device, fyzz_b200_world** out) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    try {
        auto* w = new fyzz_b200_world;
        w->impl = new fyzz::b200::World(device);
        *out = w;
        return FYZZ_B200_OK;
    } catch (const std::exception&) {
        *out = nullptr;
        return FYZZ_B200_RUNTIME_ERROR;
    }
}
int fyzz_b200_destroy(fyzz_b200_world* w) {
    if (!w) return FYZZ_B200_INVALID_ARGUMENT;
    delete w->impl;
    delete w;
    return FYZZ_B200_OK;
}
const char* fyzz_b200_last_error(const fyzz_b200_world* w) { return w ? w->error.c_str() : "null world"; }
int fyzz_b200_error_bits(const fyzz_b200_world* w, uint32_t* bits) {
    if (!w || !w->impl || !bits) return FYZZ_B200_INVALID_ARGUMENT;
    *bits = w->impl->error_bits();
    return FYZZ_B200_OK;
}
int fyzz_b200_begin_scene(fyzz_b200_world* w, uint32_t* out) {
    return guarded(w, [&](auto& W) { const uint32_t s = W.begin_scene(); if (out) *out = s; });
}
int fyzz_b200_add_static_floor(fyzz_b200_world* w, float h, uint32_t* out) {
    return guarded(w, [&](auto& W) { const uint32_t b = W.add_static_floor(h); if (out) *out = b; });
}
int fyzz_b200_create_dynamic_body(fyzz_b200_world* w, const float pose[7], uint32_t* out) {
    if (!pose) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { const uint32_t b = W.create_dynamic_body(pose); if (out) *out = b; });
}
int fyzz_b200_attach_box_shape(fyzz_b200_world* w, uint32_t body, const float half[3], const float local[7], uint32_t* out) {
    if (!half) return FYZZ_B200_INVALID_ARGUMENT;
    static const float identity[7] = {0, 0, 0, 0, 0, 0, 1};
    return guarded(w, [&](auto& W) {
        const uint32_t s = W.attach(body, fyzz::b200::kBox, half, 0.0f, local ? local : identity);
        if (out) *out = s;
    });
}
int fyzz_b200_attach_sphere_shape(fyzz_b200_world* w, uint32_t body, float r, const float local[7], uint32_t* out) {
    static const float identity[7] = {0, 0, 0, 0, 0, 0, 1};
    return guarded(w, [&](auto& W) {
        const float no_half[3] = {0.0f, 0.0f, 0.0f};
        const uint32_t s = W.attach(body, fyzz::b200::kSphere, no_half, r, local ? local : identity);
        if (out) *out = s;
    });
}
int fyzz_b200_update_mass_properties(fyzz_b200_world* w, uint32_t body, float density) {
    return guarded(w, [&](auto& W) { W.update_mass_properties(body, density); });
}
int fyzz_b200_body_mass_properties(const fyzz_b200_world* w, uint32_t body, float out[11]) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(const_cast<fyzz_b200_world*>(w), [&](auto& W) { W.mass_props(body, out); });
}
int fyzz_b200_set_shape_material(fyzz_b200_world* w, uint32_t shape, const fyzz_b200_material* m) {
    if (!m) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_shape_material(shape, *m); });
}
int fyzz_b200_set_body_velocity(fyzz_b200_world* w, uint32_t body, const float v[3]) {
    if (!v) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_velocity(body, v, false); });
}
int fyzz_b200_set_body_angular_velocity(fyzz_b200_world* w, uint32_t body, const float v[3]) {
    if (!v) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_velocity(body, v, true); });
}
int fyzz_b200_add_center_distance_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, float d, uint64_t* out) {
    return guarded(w, [&](auto& W) { const uint64_t id = W.add_distance(a, b, d); if (out) *out = id; });
}
namespace {
thread_local std::string g_cook_error;
}
int fyzz_b200_cook_convex_mesh(const float* verts, uint32_t nv, const uint32_t* tris, uint32_t nt,
                               fyzz_b200_convex_mesh** out) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        auto m = fyzz::b200::cook_convex(verts, nv, tris, nt);
        *out = new fyzz_b200_convex_mesh{std::move(m)};
        g_cook_error.clear();
        return FYZZ_B200_OK;
    } catch (const std::invalid_argument& e) {
        g_cook_error = e.what(); return FYZZ_B200_INVALID_ARGUMENT;
    } catch (const std::overflow_error& e) {
        g_cook_error = e.what(); return FYZZ_B200_OVERFLOW;
    } catch (const std::exception& e) {
        g_cook_error = e.what(); return FYZZ_B200_RUNTIME_ERROR;
    }
}
void fyzz_b200_convex_mesh_release(fyzz_b200_convex_mesh* mesh) { delete mesh; }
const char* fyzz_b200_cook_error(void) { return g_cook_error.c_str(); }
int fyzz_b200_convex_mesh_info(const fyzz_b200_convex_mesh* mesh, uint32_t counts[3], float* faces6,
                               uint32_t* face_indices, double* volume, float* mass18) {
    if (!mesh || !mesh->mesh) return FYZZ_B200_INVALID_ARGUMENT;
    const auto& m = *mesh->mesh;
    if (counts) {
        counts[0] = uint32_t(m.verts.size());
        counts[1] = uint32_t(m.faces.size());
        counts[2] = uint32_t(m.idx.size());
    }
    if (faces6)
        for (size_t i = 0; i < m.faces.size(); ++i) {
            const auto& f = m.faces[i];
            float* o = faces6 + 6 * i;
            o[0] = f.n[0]; o[1] = f.n[1]; o[2] = f.n[2]; o[3] = f.d;
            o[4] = float(f.first); o[5] = float(f.count);
        }
    if (face_indices) std::copy(m.idx.begin(), m.idx.end(), face_indices);
    if (volume) *volume = m.volume;
    if (mass18) {
        for (int k = 0; k < 3; ++k) mass18[k] = m.center[k];
        for (int c = 0; c < 3; ++c)
            for (int k = 0; k < 3; ++k) mass18[3 + 3 * c + k] = m.inertia[c][k];
        for (int k = 0; k < 3; ++k) {
            mass18[12 + k] = m.lo[k];
            mass18[15 + k] = m.hi[k];
        }
    }
    return FYZZ_B200_OK;
}
int fyzz_b200_attach_convex_shape(fyzz_b200_world* w, uint32_t body, const fyzz_b200_convex_mesh* mesh,
                                  const float local[7], uint32_t* out) {
    static const float identity[7] = {0, 0, 0, 0, 0, 0, 1};
    if (!mesh) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) {
        const uint32_t s = W.attach_convex(body, mesh->mesh, local ? local : identity);
        if (out) *out = s;
    });
}
int fyzz_b200_remove_constraint(fyzz_b200_world* w, uint64_t id) {
    return guarded(w, [&](auto& W) { W.remove_joint(id); });
}
int fyzz_b200_add_scene(fyzz_b200_world* w, uint32_t nb, const float* bodies, uint32_t ns,
                        const uint32_t* shape_body, const uint32_t* shape_type, const float* shape_geom,
                        const float* shape_local, const float* shape_mat, uint32_t nj,
                        const uint32_t* joint_bodies, const float* joint_dist, int has_floor,
                        float floor_height, const float* floor_mat, uint32_t* first_body_out) {
    return fyzz_b200_add_scene_ex(w, nb, bodies, ns, shape_body, shape_type, shape_geom, shape_local, shape_mat, nj,
                                  joint_bodies, joint_dist, has_floor, floor_height, floor_mat, 0, nullptr,
                                  first_body_out);
}
int fyzz_b200_add_scene_ex(fyzz_b200_world* w, uint32_t nb, const float* bodies, uint32_t ns,
                           const uint32_t* shape_body, const uint32_t* shape_type, const float* shape_geom,
                           const float* shape_local, const float* shape_mat, uint32_t nj,
                           const uint32_t* joint_bodies, const float* joint_dist, int has_floor,
                           float floor_height, const float* floor_mat, uint32_t n_meshes,
                           fyzz_b200_convex_mesh* const* meshes, uint32_t* first_body_out) {
    if ((nb && !bodies) || (ns && (!shape_body || !shape_type || !shape_geom || !shape_local || !shape_mat)) ||
        (nj && (!joint_bodies || !joint_dist)) || (n_meshes && !meshes))
        return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) {
        W.begin_scene();
        if (has_floor) {
            W.add_static_floor(floor_height);
            if (floor_mat) {
                const fyzz_b200_material m{floor_mat[0], floor_mat[1], floor_mat[2]};
                W.set_shape_material(W.last_shape(), m);
            }
        }
        std::vector<uint32_t> body_id(nb), shape_id(ns);
        uint32_t si = 0;
        for (uint32_t b = 0; b < nb; ++b) {
            const float* r = bodies + 14 * size_t(b);
            body_id[b] = W.create_dynamic_body(r);
            if (b == 0 && first_body_out) *first_body_out = body_id[b];
            while (si < ns && shape_body[si] == b) {
                const float* g = shape_geom + 4 * size_t(si);
                const float* l = shape_local + 7 * size_t(si);
                if (shape_type[si] == 3) {
                    const uint32_t m = static_cast<uint32_t>(g[0]);
                    if (!(g[0] >= 0.0f) || m >= n_meshes || !meshes[m])
                        throw std::invalid_argument("Convex shape names no cooked mesh");
                    shape_id[si] = W.attach_convex(body_id[b], meshes[m]->mesh, l);
                } else {
                    shape_id[si] = shape_type[si] == 0 ? W.attach(body_id[b], fyzz::b200::kBox, g, 0.0f, l)
                                                       : W.attach(body_id[b], fyzz::b200::kSphere, g, g[0], l);
                }
                ++si;
            }
            W.update_mass_properties(body_id[b], r[13]);
        }
        if (si != ns) throw std::invalid_argument("shape_body must be grouped and ascending");
        for (uint32_t i = 0; i < ns; ++i) {
            const fyzz_b200_material m{shape_mat[3 * i], shape_mat[3 * i + 1], shape_mat[3 * i + 2]};
            W.set_shape_material(shape_id[i], m);
        }
        for (uint32_t b = 0; b < nb; ++b) {
            const float* r = bodies + 14 * size_t(b);
            W.set_velocity(body_id[b], r + 7, false);
            W.set_velocity(body_id[b], r + 10, true);
        }
        for (uint32_t j = 0; j < nj; ++j)
            W.add_distance(body_id[joint_bodies[2 * j]], body_id[joint_bodies[2 * j + 1]], joint_dist[j]);
    });
}
int fyzz_b200_step(fyzz_b200_world* w, float dt) {
    return guarded(w, [&](auto& W) { W.step(dt, 1); });
}
int fyzz_b200_step_n(fyzz_b200_world* w, float dt, uint32_t steps) {
    return guarded(w, [&](auto& W) { W.step(dt, steps); });
}
int fyzz_b200_collide(fyzz_b200_world* w) {
    return guarded(w, [&](auto& W) { W.collide(); });
}
int fyzz_b200_synchronize(fyzz_b200_world* w) {
    return guarded(w, [&](auto& W) { W.synchronize(); });
}
int fyzz_b200_profile_step(fyzz_b200_world* w, float dt, float* ms, uint32_t n) {
    if (!ms && n) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.profile_step(dt, ms, n); });
}
int fyzz_b200_kernels_per_step(fyzz_b200_world* w, uint32_t* out) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { *out = W.kernels_per_step(); });
}
int fyzz_b200_body_state(const fyzz_b200_world* w, uint32_t body, fyzz_b200_body_state_t* out) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(const_cast<fyzz_b200_world*>(w), [&](auto& W) { W.body_state(body, out); });
}
int fyzz_b200_read_bodies(fyzz_b200_world* w, float* out, uint32_t n) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.read_bodies(out, n); });
}
int fyzz_b200_write_velocities(fyzz_b200_world* w, const float* v6, uint32_t n) {
    if (!v6) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.write_velocities(v6, n); });
}
int fyzz_b200_write_velocities_strided(fyzz_b200_world* w, const float* records, uint32_t n, uint32_t stride,
                                       uint32_t linear_offset, uint32_t angular_offset) {
    if (!records) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.write_velocities(records, n, stride, linear_offset, angular_offset); });
}
int fyzz_b200_counts(fyzz_b200_world* w, uint64_t out[12]) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.counts(out); });
}
int fyzz_b200_device_view(fyzz_b200_world* w, fyzz_b200_device_view_t* out) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.device_view(out); });
}
uint64_t fyzz_b200_read_pairs(fyzz_b200_world* w, int which, uint32_t* out, uint64_t cap) {
    uint64_t n = 0;
    if (guarded(w, [&](auto& W) { n = W.read_pairs(which, out, cap); })) return 0;
    return n;
}
uint64_t fyzz_b200_read_manifolds(fyzz_b200_world* w, uint32_t* pairs, uint32_t* counts, float* points, uint64_t cap) {
    uint64_t n = 0;
    if (guarded(w, [&](auto& W) { n = W.read_manifolds(pairs, counts, points, cap); })) return 0;
    return n;
}
int fyzz_b200_read_encoded_bounds(fyzz_b200_world* w, uint32_t* out, uint32_t n) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.read_bounds(out, n); });
}
uint64_t fyzz_b200_read_sorted_min_x(fyzz_b200_world* w, uint32_t scene, uint32_t* values, uint32_t* ids, uint64_t cap) {
    uint64_t n = 0;
    if (guarded(w, [&](auto& W) { n = W.read_sorted_min_x(scene, values, ids, cap); })) return 0;
    return n;
}
static int add_joint_abi(fyzz_b200_world* w, uint32_t kind, uint32_t a, uint32_t b, const float* la,
                         const float* lb, float distance, uint64_t* out) {
    if (!la || !lb) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) {
        const uint64_t id = W.add_joint(kind, a, b, la, lb, distance);
        if (out) *out = id;
    });
}
int fyzz_b200_add_anchored_distance_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[3],
                                               const float local_b[3], float distance, uint64_t* id_out) {
    if (!local_a || !local_b) return FYZZ_B200_INVALID_ARGUMENT;
    const float la[7] = {local_a[0], local_a[1], local_a[2], 0, 0, 0, 1};
    const float lb[7] = {local_b[0], local_b[1], local_b[2], 0, 0, 0, 1};
    return add_joint_abi(w, fyzz::b200::kJointAnchored, a, b, la, lb, distance, id_out);
}
int fyzz_b200_add_fixed_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                   const float local_b[7], uint64_t* id_out) {
    return add_joint_abi(w, fyzz::b200::kJointFixed, a, b, local_a, local_b, 0.0f, id_out);
}
int fyzz_b200_add_spherical_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                       const float local_b[7], uint64_t* id_out) {
    return add_joint_abi(w, fyzz::b200::kJointSpherical, a, b, local_a, local_b, 0.0f, id_out);
}
int fyzz_b200_add_revolute_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                      const float local_b[7], uint64_t* id_out) {
    return add_joint_abi(w, fyzz::b200::kJointRevolute, a, b, local_a, local_b, 0.0f, id_out);
}
int fyzz_b200_add_prismatic_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                       const float local_b[7], uint64_t* id_out) {
    return add_joint_abi(w, fyzz::b200::kJointPrismatic, a, b, local_a, local_b, 0.0f, id_out);
}
int fyzz_b200_set_body_kinematic(fyzz_b200_world* w, uint32_t body, int enabled) {
    return guarded(w, [&](auto& W) { W.set_kinematic(body, enabled != 0); });
}
int fyzz_b200_set_body_kinematic_target(fyzz_b200_world* w, uint32_t body, const float pose[7]) {
    if (!pose) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_kinematic_target(body, pose); });
}
int fyzz_b200_set_sleeping(fyzz_b200_world* w, int enabled) {
    return guarded(w, [&](auto& W) { W.set_sleeping(enabled != 0); });
}
int fyzz_b200_read_sleep_state(fyzz_b200_world* w, float* wake, uint32_t* flags, float* motion6,
                               uint32_t* counted, uint32_t n) {
    return guarded(w, [&](auto& W) { W.read_sleep_state(wake, flags, motion6, counted, n); });
}
int fyzz_b200_set_contact_notifications(fyzz_b200_world* w, int enabled) {
    return guarded(w, [&](auto& W) { W.set_contact_notifications(enabled != 0); });
}
int fyzz_b200_contact_events(fyzz_b200_world* w, const fyzz_b200_contact_event_t** events, uint64_t* n_events,
                             const fyzz_b200_contact_event_point_t** points, uint64_t* n_points) {
    static_assert(sizeof(fyzz_b200_contact_event_t) == sizeof(fyzz::b200::EventRecord), "event layout");
    static_assert(sizeof(fyzz_b200_contact_event_point_t) == sizeof(fyzz::b200::EventPoint), "point layout");
    if (!events || !n_events || !points || !n_points) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) {
        const fyzz::b200::EventRecord* e = nullptr;
        const fyzz::b200::EventPoint* p = nullptr;
        W.contact_events(&e, n_events, &p, n_points);
        *events = reinterpret_cast<const fyzz_b200_contact_event_t*>(e);
        *points = reinterpret_cast<const fyzz_b200_contact_event_point_t*>(p);
    });
}
int fyzz_b200_fit_pair_budget(fyzz_b200_world* w, float headroom, uint32_t* budget_out) {
    return guarded(w, [&](auto& W) {
        W.fit_pair_budget(headroom);
        if (budget_out) *budget_out = W.pair_budget();
    });
}
int fyzz_b200_set_body_contact_report_threshold(fyzz_b200_world* w, uint32_t body, float force) {
    return guarded(w, [&](auto& W) { W.set_report_threshold(body, force); });
}
int fyzz_b200_force_threshold_changes(fyzz_b200_world* w, const fyzz_b200_force_threshold_report_t** reports,
                                      uint64_t* n) {
    static_assert(sizeof(fyzz_b200_force_threshold_report_t) == sizeof(fyzz::b200::ForceThresholdRecord),
                  "record layout");
    if (!reports || !n) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) {
        const fyzz::b200::ForceThresholdRecord* r = nullptr;
        W.threshold_changes(&r, n);
        *reports = reinterpret_cast<const fyzz_b200_force_threshold_report_t*>(r);
    });
}
int fyzz_b200_set_caller_validated_transforms(fyzz_b200_world* w, int enabled) {
    return guarded(w, [&](auto& W) { W.set_caller_validated(enabled != 0); });
}
int fyzz_b200_set_descriptor_order(fyzz_b200_world* w, const uint32_t* pairs, uint64_t n_pairs,
                                   const uint64_t* joint_ids, uint64_t n_joint_ids) {
    if ((n_pairs && !pairs) || (n_joint_ids && !joint_ids)) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_descriptor_order(pairs, n_pairs, joint_ids, n_joint_ids); });
}
int fyzz_b200_set_tuning(fyzz_b200_world* w, const fyzz_b200_tuning_t* t) {
    if (!t) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.set_tuning(*t); });
}
int fyzz_b200_get_tuning(fyzz_b200_world* w, fyzz_b200_tuning_t* t) {
    if (!t) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { *t = W.tuning(); });
}
int fyzz_b200_set_pair_budget(fyzz_b200_world* w, uint32_t pairs, uint32_t* budget_out) {
    return guarded(w, [&](auto& W) {
        const uint32_t cap = W.set_pair_budget(pairs);
        if (budget_out) *budget_out = cap;
    });
}
int fyzz_b200_test_scan(fyzz_b200_world* w, uint32_t n, int skip_first_tile, uint32_t* error_bits,
                        uint64_t* mismatches) {
    return guarded(w, [&](auto& W) {
        const uint32_t bits = W.scan_selftest(n, skip_first_tile != 0, mismatches);
        if (error_bits) *error_bits = bits;
        if (bits & fyzz::b200::kErrLogic)
            throw std::logic_error("Scan look-back wait gave up (error bits " + std::to_string(bits) + ")");
    });
}
int fyzz_b200_rollout_begin(fyzz_b200_world* w, uint32_t steps, uint32_t checkpoint_every) {
    return guarded(w, [&](auto& W) { W.rollout_begin(steps, checkpoint_every); });
}
int fyzz_b200_rollout_rewind(fyzz_b200_world* w) {
    return guarded(w, [&](auto& W) { W.rollout_rewind(); });
}
int fyzz_b200_rollout_forward(fyzz_b200_world* w, float seconds) {
    return guarded(w, [&](auto& W) { W.rollout_forward(seconds); });
}
int fyzz_b200_rollout_backward(fyzz_b200_world* w, const float* grad_center, const float* grad_orientation,
                               const float* grad_velocity, const float* grad_angular, float* grad_v0,
                               float* grad_w0, float* grad_mass, float* grad_static_friction,
                               float* grad_dynamic_friction) {
    return guarded(w, [&](auto& W) {
        W.rollout_backward(grad_center, grad_orientation, grad_velocity, grad_angular, grad_v0, grad_w0,
                           grad_mass, grad_static_friction, grad_dynamic_friction);
    });
}
uint64_t fyzz_b200_read_friction_anchors(fyzz_b200_world* w, uint32_t* anchors, float* anchors0,
                                         float* anchors1, uint64_t cap) {
    uint64_t n = 0;
    if (guarded(w, [&](auto& W) { n = W.read_friction_anchors(anchors, anchors0, anchors1, cap); })) return 0;
    return n;
}
int fyzz_b200_read_mass_frames(fyzz_b200_world* w, float* centers, float* orientations) {
    return guarded(w, [&](auto& W) { W.read_mass_frames(centers, orientations); });
}
int fyzz_b200_read_step_counters(fyzz_b200_world* w, uint32_t* out, uint32_t n) {
    if (!out) return FYZZ_B200_INVALID_ARGUMENT;
    return guarded(w, [&](auto& W) { W.read_step_counters(out, n); });
}
uint64_t fyzz_b200_read_islands(fyzz_b200_world* w, uint32_t* descriptors, uint32_t* levels, uint64_t cap) {
    uint64_t n = 0;
    guarded(w, [&](auto& W) { n = W.read_islands(descriptors, levels, cap); });
    return n;
}
uint64_t fyzz_b200_read_levels(fyzz_b200_world* w, uint32_t* levels, uint64_t cap) {
    uint64_t n = 0;
    if (guarded(w, [&](auto& W) { n = W.read_levels(levels, cap); })) return 0;
    return n;
}

}  // extern "C"
