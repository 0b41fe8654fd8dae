// fyzz::WorldBackend over the B200 C ABI; see b200_world_backend.h.
#include "b200_world_backend.h"

#include "fyzz_b200.h"
#include "fyzzxyzzy/convex.h"

#include <cmath>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace fyzz {
namespace {

void pose7(const Transform& t, float out[7]) {
    out[0] = t.position.x; out[1] = t.position.y; out[2] = t.position.z;
    out[3] = t.orientation.x; out[4] = t.orientation.y; out[5] = t.orientation.z; out[6] = t.orientation.w;
}

class B200WorldBackend final : public WorldBackend {
public:
    B200WorldBackend(int device, const WorldOptions& options) {
        const int rc = fyzz_b200_create(device, &w_);
        if (rc) throw std::runtime_error("B200 world: no CUDA device or context (status " + std::to_string(rc) + ")");
        // World has validated and normalised every transform already
        check(fyzz_b200_set_caller_validated_transforms(w_, 1));
        if (options.contact_notifications) check(fyzz_b200_set_contact_notifications(w_, 1));
    }
    ~B200WorldBackend() override {
        for (auto& [mesh, cooked] : meshes_) fyzz_b200_convex_mesh_release(cooked);
        fyzz_b200_destroy(w_);
    }
    B200WorldBackend(const B200WorldBackend&) = delete;
    B200WorldBackend& operator=(const B200WorldBackend&) = delete;

    // ---- actors and shapes ----
    BodyId create_dynamic_body(Transform pose) override {
        float p[7];
        pose7(pose, p);
        uint32_t id = 0;
        check(fyzz_b200_create_dynamic_body(w_, p, &id));
        return id;
    }
    ShapeId attach_box_shape(BodyId body, Vec3 h, Transform local) override {
        const float half[3] = {h.x, h.y, h.z};
        float p[7];
        pose7(local, p);
        uint32_t id = 0;
        check(fyzz_b200_attach_box_shape(w_, body, half, p, &id));
        return id;
    }
    ShapeId attach_sphere_shape(BodyId body, float radius, Transform local) override {
        float p[7];
        pose7(local, p);
        uint32_t id = 0;
        check(fyzz_b200_attach_sphere_shape(w_, body, radius, p, &id));
        return id;
    }
    // The reference's cooked mesh keeps its input triangles; cooking them
    // again on this side gives the same hull bit for bit (cooking follows
    // cooked_convex.cpp), shared by every shape that attaches the mesh.
    ShapeId attach_convex_shape(BodyId body, std::shared_ptr<const ConvexMesh> mesh, Transform local) override {
        if (!mesh) throw std::invalid_argument("Cooked convex geometry is missing");
        auto it = meshes_.find(mesh.get());
        if (it == meshes_.end()) {
            std::vector<float> v;
            for (const Vec3& x : mesh->vertices()) v.insert(v.end(), {x.x, x.y, x.z});
            std::vector<uint32_t> t;
            for (const ConvexTriangle& tri : mesh->triangles()) t.insert(t.end(), {tri[0], tri[1], tri[2]});
            fyzz_b200_convex_mesh* cooked = nullptr;
            if (const int rc = fyzz_b200_cook_convex_mesh(v.data(), uint32_t(v.size() / 3), t.data(),
                                                          uint32_t(t.size() / 3), &cooked))
                raise(rc, fyzz_b200_cook_error());
            it = meshes_.emplace(mesh.get(), cooked).first;
            keep_.push_back(mesh);
        }
        float p[7];
        pose7(local, p);
        uint32_t id = 0;
        check(fyzz_b200_attach_convex_shape(w_, body, it->second, p, &id));
        return id;
    }
    void set_shape_material(ShapeId shape, Material m) override {
        if (m.damping != 0.0f || m.friction_combine != MaterialCombineMode::Average ||
            m.restitution_combine != MaterialCombineMode::Average || m.damping_combine != MaterialCombineMode::Average ||
            m.compliant_acceleration_spring || m.disable_friction || m.disable_strong_friction || m.restitution < 0.0f)
            throw std::logic_error("The B200 backend supports averaged friction and restitution materials only");
        const fyzz_b200_material mat{m.static_friction, m.dynamic_friction, m.restitution};
        check(fyzz_b200_set_shape_material(w_, shape, &mat));
    }
    void update_mass_properties(BodyId body, float density) override {
        check(fyzz_b200_update_mass_properties(w_, body, density));
    }
    BodyMassProperties body_mass_properties(BodyId body) const override {
        float o[11];
        check(fyzz_b200_body_mass_properties(w_, body, o));
        BodyMassProperties m;
        m.inverse_mass = o[0];
        m.inverse_inertia = {o[1], o[2], o[3]};
        m.mass_local_pose.position = {o[4], o[5], o[6]};
        m.mass_local_pose.orientation = {o[7], o[8], o[9], o[10]};
        return m;
    }
    BodyId add_static_box(Vec3, Vec3) override {
        throw std::logic_error("The B200 backend has no static boxes (one static floor per scene)");
    }
    BodyId add_static_floor(float height) override {
        uint32_t id = 0;
        check(fyzz_b200_add_static_floor(w_, height, &id));
        return id;
    }
    BodyId add_dynamic_box(Vec3 half, Vec3 position, float density) override {
        const BodyId b = create_dynamic_body(Transform{position, {}});
        attach_box_shape(b, half, Transform{});
        update_mass_properties(b, density);
        return b;
    }
    BodyId add_dynamic_sphere(float radius, Vec3 position, float density) override {
        const BodyId b = create_dynamic_body(Transform{position, {}});
        attach_sphere_shape(b, radius, Transform{});
        update_mass_properties(b, density);
        return b;
    }

    // ---- constraints ----
    ConstraintId add_center_distance_constraint(BodyId a, BodyId b, float d) override {
        uint64_t id = 0;
        check(fyzz_b200_add_center_distance_constraint(w_, a, b, d, &id));
        return id;
    }
    ConstraintId add_anchored_distance_constraint(BodyId a, BodyId b, Vec3 la, Vec3 lb, float d) override {
        const float pa[3] = {la.x, la.y, la.z}, pb[3] = {lb.x, lb.y, lb.z};
        uint64_t id = 0;
        check(fyzz_b200_add_anchored_distance_constraint(w_, a, b, pa, pb, d, &id));
        return id;
    }
    ConstraintId add_fixed_constraint(BodyId a, BodyId b, Transform la, Transform lb) override {
        return framed(fyzz_b200_add_fixed_constraint, a, b, la, lb);
    }
    ConstraintId add_spherical_constraint(BodyId a, BodyId b, Transform la, Transform lb) override {
        return framed(fyzz_b200_add_spherical_constraint, a, b, la, lb);
    }
    ConstraintId add_revolute_constraint(BodyId a, BodyId b, Transform la, Transform lb) override {
        return framed(fyzz_b200_add_revolute_constraint, a, b, la, lb);
    }
    ConstraintId add_prismatic_constraint(BodyId a, BodyId b, Transform la, Transform lb) override {
        return framed(fyzz_b200_add_prismatic_constraint, a, b, la, lb);
    }
    void remove_constraint(ConstraintId id) override { check(fyzz_b200_remove_constraint(w_, id)); }

    // ---- stepping and results ----
    void step(float seconds) override {
        ++generation_;
        check(fyzz_b200_step(w_, seconds));
    }
    BodyState body_state(BodyId id) const override {
        fyzz_b200_body_state_t s{};
        check(fyzz_b200_body_state(w_, id, &s));
        BodyState out;
        out.position = {s.position[0], s.position[1], s.position[2]};
        out.velocity = {s.velocity[0], s.velocity[1], s.velocity[2]};
        out.orientation = {s.orientation[0], s.orientation[1], s.orientation[2], s.orientation[3]};
        out.angular_velocity = {s.angular_velocity[0], s.angular_velocity[1], s.angular_velocity[2]};
        out.sleeping = s.sleeping != 0;
        return out;
    }
    std::span<const ContactEvent> contact_events() const override {
        refresh_events();
        return events_;
    }
    std::span<const ContactEventPoint> contact_event_points() const override {
        refresh_events();
        return points_;
    }
    std::span<const ForceThresholdReport> force_threshold_changes() const override {
        if (threshold_generation_ != generation_) {
            const fyzz_b200_force_threshold_report_t* r = nullptr;
            uint64_t n = 0;
            check(fyzz_b200_force_threshold_changes(w_, &r, &n));
            thresholds_.resize(n);
            for (uint64_t i = 0; i < n; ++i) {
                ForceThresholdReport& o = thresholds_[i];
                o.key = ForceThresholdKey{r[i].actor0, r[i].actor1, r[i].static_world != 0};
                o.normal_impulse = r[i].normal_impulse;
                o.threshold = r[i].threshold;
                o.change = static_cast<ForceThresholdChange>(r[i].change);
            }
            threshold_generation_ = generation_;
        }
        return thresholds_;
    }

    // ---- body authoring ----
    void set_body_velocity(BodyId id, Vec3 v) override {
        const float a[3] = {v.x, v.y, v.z};
        check(fyzz_b200_set_body_velocity(w_, id, a));
    }
    void set_body_angular_velocity(BodyId id, Vec3 v) override {
        const float a[3] = {v.x, v.y, v.z};
        check(fyzz_b200_set_body_angular_velocity(w_, id, a));
    }
    void set_body_contact_report_threshold(BodyId id, float force) override {
        check(fyzz_b200_set_body_contact_report_threshold(w_, id, force));
    }
    void set_body_kinematic(BodyId id, bool enabled) override {
        check(fyzz_b200_set_body_kinematic(w_, id, enabled ? 1 : 0));
    }
    void set_body_kinematic_target(BodyId id, Vec3 p, Quat q) override {
        const float pose[7] = {p.x, p.y, p.z, q.x, q.y, q.z, q.w};
        check(fyzz_b200_set_body_kinematic_target(w_, id, pose));
    }

private:
    [[noreturn]] static void raise(int rc, const char* msg) {
        const std::string m = msg ? msg : "B200 world error";
        switch (rc) {
            case FYZZ_B200_INVALID_ARGUMENT: throw std::invalid_argument(m);
            case FYZZ_B200_LOGIC_ERROR: throw std::logic_error(m);
            case FYZZ_B200_OVERFLOW: throw std::overflow_error(m);
            default: throw std::runtime_error(m);
        }
    }
    void check(int rc) const {
        if (rc) raise(rc, fyzz_b200_last_error(w_));
    }
    template <class F>
    ConstraintId framed(F f, BodyId a, BodyId b, const Transform& la, const Transform& lb) {
        float pa[7], pb[7];
        pose7(la, pa);
        pose7(lb, pb);
        uint64_t id = 0;
        check(f(w_, a, b, pa, pb, &id));
        return id;
    }
    void refresh_events() const {
        if (event_generation_ == generation_) return;
        const fyzz_b200_contact_event_t* e = nullptr;
        const fyzz_b200_contact_event_point_t* p = nullptr;
        uint64_t ne = 0, np = 0;
        check(fyzz_b200_contact_events(w_, &e, &ne, &p, &np));
        events_.resize(ne);
        for (uint64_t i = 0; i < ne; ++i) {
            ContactEvent& o = events_[i];
            o.body0 = e[i].body0;
            o.body1 = e[i].body1;
            o.kind = static_cast<ContactEventKind>(e[i].kind);
            o.contact_count = static_cast<std::uint8_t>(e[i].contact_count);
            o.point_offset = static_cast<std::size_t>(e[i].point_offset);
            o.normal_impulse = e[i].normal_impulse;
            o.shape0 = e[i].shape0;
            o.shape1 = e[i].shape1;
        }
        points_.resize(np);
        for (uint64_t i = 0; i < np; ++i) {
            ContactEventPoint& o = points_[i];
            o.position = {p[i].position[0], p[i].position[1], p[i].position[2]};
            o.normal = {p[i].normal[0], p[i].normal[1], p[i].normal[2]};
            o.separation = p[i].separation;
            o.normal_impulse = p[i].normal_impulse;
        }
        event_generation_ = generation_;
    }

    fyzz_b200_world* w_ = nullptr;
    std::map<const ConvexMesh*, fyzz_b200_convex_mesh*> meshes_;
    std::vector<std::shared_ptr<const ConvexMesh>> keep_;
    uint64_t generation_ = 0;
    mutable uint64_t event_generation_ = ~0ull, threshold_generation_ = ~0ull;
    mutable std::vector<ContactEvent> events_;
    mutable std::vector<ContactEventPoint> points_;
    mutable std::vector<ForceThresholdReport> thresholds_;
};

}  // namespace

std::unique_ptr<WorldBackend> create_b200_world_backend(int device, WorldOptions options) {
    return std::make_unique<B200WorldBackend>(device, options);
}

World create_b200_world(int device, WorldOptions options) {
    return World(create_b200_world_backend(device, options));
}

}  // namespace fyzz
