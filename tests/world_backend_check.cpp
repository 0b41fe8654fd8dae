// Test infrastructure: drives the reference SDK's own fyzz::World twice on
// the same authored scene -- once over the B200 backend
// (fyzzxyzzy-sdk_b200/integration/b200_world_backend.cpp, World(std::
// unique_ptr<WorldBackend>), world.h:400) and once over the reference's
// NativeCpu backend (World(WorldOptions{NativeCpu})) -- and returns both
// worlds' body states.  Built by oracle/Makefile (target backend) from the
// reference sources where they exist; tests/test_gpu_world_backend.py loads
// it.
#include "b200_world_backend.h"

#include <cstdint>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

fyzz::Transform transform_of(const float* p) {
    fyzz::Transform t;
    t.position = {p[0], p[1], p[2]};
    t.orientation = {p[3], p[4], p[5], p[6]};
    return t;
}

// The seeded-workload record layout (fyzzxyzzy-sdk_b200/scenes.py): per body
// position(3) orientation(4) velocity(3) angular velocity(3) density; per
// shape owner, type (0 box, 1 sphere), geometry(4), local pose(7),
// material(3); center distance joints.  Authored through the public World
// API in the order the reference harness uses.
void author(fyzz::World& w, uint32_t nb, const float* bodies, uint32_t ns, const uint32_t* shape_body,
            const uint32_t* shape_type, const float* geom, const float* local, const float* mat, uint32_t nj,
            const uint32_t* joints, const float* dist, int has_floor, float floor_height, const float* floor_mat) {
    if (has_floor) {
        const fyzz::BodyId f = w.add_static_floor(floor_height);
        (void)f;
        fyzz::Material m;
        m.static_friction = floor_mat[0];
        m.dynamic_friction = floor_mat[1];
        m.restitution = floor_mat[2];
        w.set_shape_material(0, m);
    }
    std::vector<fyzz::BodyId> ids(nb);
    std::vector<fyzz::ShapeId> shapes(ns);
    uint32_t next = 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const float* r = bodies + 14ull * b;
        ids[b] = w.create_dynamic_body(transform_of(r));
        while (next < ns && shape_body[next] == b) {
            const uint32_t i = next++;
            const float* g = geom + 4ull * i;
            shapes[i] = shape_type[i] == 0 ? w.attach_box_shape(ids[b], {g[0], g[1], g[2]}, transform_of(local + 7ull * i))
                                           : w.attach_sphere_shape(ids[b], g[0], transform_of(local + 7ull * i));
        }
        w.update_mass_properties(ids[b], r[13]);
    }
    for (uint32_t i = 0; i < ns; ++i) {
        fyzz::Material m;
        m.static_friction = mat[3 * i];
        m.dynamic_friction = mat[3 * i + 1];
        m.restitution = mat[3 * i + 2];
        w.set_shape_material(shapes[i], m);
    }
    for (uint32_t b = 0; b < nb; ++b) {
        const float* r = bodies + 14ull * b;
        w.set_body_velocity(ids[b], {r[7], r[8], r[9]});
        w.set_body_angular_velocity(ids[b], {r[10], r[11], r[12]});
    }
    for (uint32_t j = 0; j < nj; ++j) w.add_center_distance_constraint(ids[joints[2 * j]], ids[joints[2 * j + 1]], dist[j]);
}

void read(const fyzz::World& w, uint32_t n_actors, float* out) {
    for (uint32_t i = 0; i < n_actors; ++i) {
        const fyzz::BodyState s = w.body_state(i);
        float* o = out + 14ull * i;
        o[0] = s.position.x; o[1] = s.position.y; o[2] = s.position.z;
        o[3] = s.velocity.x; o[4] = s.velocity.y; o[5] = s.velocity.z;
        o[6] = s.orientation.x; o[7] = s.orientation.y; o[8] = s.orientation.z; o[9] = s.orientation.w;
        o[10] = s.angular_velocity.x; o[11] = s.angular_velocity.y; o[12] = s.angular_velocity.z;
        o[13] = s.sleeping ? 1.0f : 0.0f;
    }
}

void put(char* msg, size_t len, const std::string& s) {
    if (!msg || !len) return;
    std::strncpy(msg, s.c_str(), len - 1);
    msg[len - 1] = '\0';
}

}  // namespace

extern "C" int fz_backend_compare(uint32_t nb, const float* bodies, uint32_t ns, const uint32_t* shape_body,
                                  const uint32_t* shape_type, const float* geom, const float* local,
                                  const float* mat, uint32_t nj, const uint32_t* joints, const float* dist,
                                  int has_floor, float floor_height, const float* floor_mat, float dt,
                                  uint32_t steps, float* out_b200, float* out_native, uint32_t* event_counts,
                                  char* msg, size_t msg_len) {
    try {
        fyzz::WorldOptions opts;
        opts.execution = fyzz::ExecutionMode::NativeCpu;
        opts.contact_notifications = true;
        fyzz::World native(opts);
        fyzz::World b200 = fyzz::create_b200_world(0, opts);
        author(native, nb, bodies, ns, shape_body, shape_type, geom, local, mat, nj, joints, dist, has_floor,
               floor_height, floor_mat);
        author(b200, nb, bodies, ns, shape_body, shape_type, geom, local, mat, nj, joints, dist, has_floor,
               floor_height, floor_mat);
        for (uint32_t k = 0; k < steps; ++k) {
            native.step(dt);
            b200.step(dt);
        }
        const uint32_t n_actors = nb + (has_floor ? 1u : 0u);
        read(b200, n_actors, out_b200);
        read(native, n_actors, out_native);
        if (event_counts) {
            event_counts[0] = uint32_t(b200.contact_events().size());
            event_counts[1] = uint32_t(native.contact_events().size());
            event_counts[2] = uint32_t(b200.contact_event_points().size());
            event_counts[3] = uint32_t(native.contact_event_points().size());
        }
        put(msg, msg_len, "");
        return 0;
    } catch (const std::exception& e) {
        put(msg, msg_len, e.what());
        return 1;
    }
}

// The backend's explicit rejections of what the B200 step does not model.
extern "C" int fz_backend_rejects(char* msg, size_t msg_len) {
    fyzz::World w = fyzz::create_b200_world(0);
    int rejected = 0;
    try { w.add_static_box({1, 1, 1}, {0, 0, 0}); } catch (const std::logic_error&) { ++rejected; }
    try { w.create_aggregate(8, false); } catch (const std::logic_error&) { ++rejected; }
    try { (void)w.raycast({0, 1, 0}, {0, -1, 0}, 10.0f); } catch (const std::logic_error&) { ++rejected; }
    try { w.step(-1.0f); } catch (const std::invalid_argument&) { ++rejected; }
    put(msg, msg_len, std::to_string(rejected));
    return rejected;
}
