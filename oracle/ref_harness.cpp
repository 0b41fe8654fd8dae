// Test infrastructure only: a C-ABI shim over the reference SDK's own
// NativeCpu scene (src/native/scene.{h,cpp}), compiled from the reference
// sources by oracle/Makefile into oracle/_ref/libfyzz_ref.so.
//
// Nothing in the product links or loads this file.  Tests, smoke() and
// bench.py's CPU-baseline leg use it as the checker and as the timed
// reference implementation.
//
// Scene construction mirrors what a user of fyzz::World would call for the
// NativeCpu execution mode (include/fyzzxyzzy/world.h:396-510, forwarded
// 1:1 by NativeCpuWorld at src/native/scene.cpp:11158-11240):
//   add_static_floor, create_dynamic_body, attach_box_shape /
//   attach_sphere_shape, update_mass_properties, set_shape_material,
//   set_body_velocity / set_body_angular_velocity,
//   add_center_distance_constraint, step.
// World validates and normalises transforms (src/world.cpp:38-55) before
// the scene sees them; the same arithmetic is applied here.
//
// Internal intermediates (encoded bounds, SAP endpoint order, Dy descriptor
// order) are read through SolverIterationSourceFixture, one of the friend
// fixtures the reference's Scene declares (src/native/scene.h:1082-1089).

#include "native/scene.h"
#include "fyzzxyzzy/convex.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <thread>
#include <vector>

namespace fyzz::native {
struct SolverIterationSourceFixture {
    static const auto& shapes(const Scene& s) { return s.shapes_; }
    static const auto& actors(const Scene& s) { return s.actors_; }
    static const auto& endpoints(const Scene& s, unsigned axis) {
        return s.sap_axis_endpoints_[axis];
    }
    static const auto& indexed_managers(const Scene& s) { return s.indexed_managers_; }
    static const auto& indexed_joints(const Scene& s) { return s.indexed_joints_; }
    static const auto& island_edges(const Scene& s) { return s.island_edges_; }
    static const auto& ordered(const Scene& s) { return s.ordered_constraints_; }
    static const auto& partition_ends(const Scene& s) { return s.partition_ends_; }
    static const auto& tasks(const Scene& s) { return s.solver_tasks_; }
    static const auto& manifolds(const Scene& s) { return s.manifolds_; }
    static bool reversed(const Scene& s, std::uint32_t edge) {
        return s.island_edges_[edge].gu_order_reversed;
    }
};
} // namespace fyzz::native

namespace {
using fyzz::native::Scene;
using Fix = fyzz::native::SolverIterationSourceFixture;
thread_local std::string g_error;

struct Handle {
    std::unique_ptr<Scene> scene;
    std::vector<fyzz::BodyId> bodies;   // dynamic body index -> BodyId
    std::vector<fyzz::ShapeId> shapes;  // shape index -> ShapeId
    std::vector<std::shared_ptr<const fyzz::ConvexMesh>> meshes;  // convex shape_geom[0] -> mesh
    bool has_floor = false;
};

fyzz::Transform transform_of(const float* p) {
    fyzz::Transform t{};
    t.position = {p[0], p[1], p[2]};
    fyzz::Quat q{p[3], p[4], p[5], p[6]};
    // src/world.cpp:38-55 validated_transform: |q| within 1e-2, then divide.
    const float len = std::sqrt(q.x*q.x + q.y*q.y + q.z*q.z + q.w*q.w);
    if (!std::isfinite(len) || std::abs(len - 1.0f) >= 1.0e-2f)
        throw std::invalid_argument("Rigid pose orientation is not sane");
    t.orientation = {q.x/len, q.y/len, q.z/len, q.w/len};
    return t;
}

template <class F> int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument& e) {
        g_error = e.what(); return 1;
    } catch (const std::logic_error& e) {
        g_error = e.what(); return 2;
    } catch (const std::overflow_error& e) {
        g_error = e.what(); return 3;
    } catch (const std::exception& e) {
        g_error = e.what(); return 4;
    }
}
} // namespace

extern "C" {

const char* fz_ref_error(void) { return g_error.c_str(); }

void* fz_ref_create(int contact_notifications) {
    auto* h = new Handle;
    h->scene = std::make_unique<Scene>();
    h->scene->set_contact_notifications(contact_notifications != 0);
    return h;
}

void fz_ref_destroy(void* p) { delete static_cast<Handle*>(p); }

// Bodies: nb records of 14 floats: position(3) orientation xyzw(4)
// linear velocity(3) angular velocity(3) density.  Shapes: shape_body is
// the 0-based dynamic-body index; shape_type 0 = box, 1 = sphere;
// shape_geom 4 floats (half extents or radius); shape_local 7 floats (local
// pose); shape_mat 3 floats (static friction, dynamic friction, restitution).
// The floor, when present, is created first (BodyId 0, ShapeId 0) and takes
// floor_mat (static friction, dynamic friction, restitution) when given.
int fz_ref_build(void* p, uint32_t nb, const float* bodies, uint32_t ns,
                 const uint32_t* shape_body, const uint32_t* shape_type,
                 const float* shape_geom, const float* shape_local,
                 const float* shape_mat, uint32_t nj,
                 const uint32_t* joint_bodies, const float* joint_dist,
                 int has_floor, float floor_height, const float* floor_mat) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] {
        Scene& s = *h->scene;
        if (has_floor) {
            s.add_static_floor(floor_height);
            h->has_floor = true;
            if (floor_mat) {
                fyzz::Material m{};
                m.static_friction = floor_mat[0];
                m.dynamic_friction = floor_mat[1];
                m.restitution = floor_mat[2];
                s.set_attached_shape_material(0, m);
            }
        }
        h->bodies.resize(nb);
        h->shapes.resize(ns);
        uint32_t next_shape = 0;
        for (uint32_t b = 0; b < nb; ++b) {
            const float* r = bodies + 14ull * b;
            h->bodies[b] = s.create_body(transform_of(r), true);
            while (next_shape < ns && shape_body[next_shape] == b) {
                const uint32_t i = next_shape++;
                const auto local = transform_of(shape_local + 7ull * i);
                const float* g = shape_geom + 4ull * i;
                if (shape_type[i] == 0)
                    h->shapes[i] = s.attach_box(h->bodies[b], {g[0], g[1], g[2]}, local);
                else if (shape_type[i] == 3)
                    h->shapes[i] = s.attach_convex(h->bodies[b], h->meshes.at(static_cast<std::size_t>(g[0])), local);
                else
                    h->shapes[i] = s.attach_sphere(h->bodies[b], g[0], local);
            }
            s.update_mass_properties(h->bodies[b], r[13]);
        }
        if (next_shape != ns)
            throw std::invalid_argument("shape_body must be grouped and ascending");
        for (uint32_t i = 0; i < ns; ++i) {
            fyzz::Material m{};
            m.static_friction = shape_mat[3*i+0];
            m.dynamic_friction = shape_mat[3*i+1];
            m.restitution = shape_mat[3*i+2];
            s.set_attached_shape_material(h->shapes[i], m);
        }
        for (uint32_t b = 0; b < nb; ++b) {
            const float* r = bodies + 14ull * b;
            s.set_velocity(h->bodies[b], {r[7], r[8], r[9]});
            s.set_angular_velocity(h->bodies[b], {r[10], r[11], r[12]});
        }
        for (uint32_t j = 0; j < nj; ++j)
            s.create_center_distance_constraint(h->bodies[joint_bodies[2*j]],
                                                h->bodies[joint_bodies[2*j+1]],
                                                joint_dist[j]);
    });
}

// One joint after fz_ref_build, through the Scene members World forwards to
// (scene.cpp:11236-11260) with World's validation applied first
// (src/world.cpp:231-276).  kind: 0 center distance, 1 anchored distance,
// 2 fixed, 3 spherical, 4 revolute, 5 prismatic.  a / b are 0-based dynamic
// body indices, 0xffffffff for the floor; local poses are 7 floats.
int fz_ref_add_joint(void* p, int kind, uint32_t a, uint32_t b, const float* la, const float* lb,
                     float distance, uint64_t* id_out) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] {
        auto body = [&](uint32_t i) -> fyzz::BodyId {
            if (i == 0xffffffffu) {
                if (!h->has_floor) throw std::invalid_argument("no floor");
                return 0;
            }
            return h->bodies.at(i);
        };
        Scene& s = *h->scene;
        const fyzz::BodyId A = body(a), B = body(b);
        fyzz::ConstraintId id{};
        if (kind == 0) {
            id = s.create_center_distance_constraint(A, B, distance);
        } else if (kind == 1) {
            id = s.create_anchored_distance_constraint(A, B, {la[0], la[1], la[2]}, {lb[0], lb[1], lb[2]}, distance);
        } else {
            const fyzz::Transform ta = transform_of(la), tb = transform_of(lb);
            if (kind == 2) id = s.create_fixed_constraint(A, B, ta, tb);
            else if (kind == 3) id = s.create_spherical_constraint(A, B, ta, tb);
            else if (kind == 4) id = s.create_revolute_constraint(A, B, ta, tb);
            else if (kind == 5) id = s.create_prismatic_constraint(A, B, ta, tb);
            else throw std::invalid_argument("joint kind");
        }
        if (id_out) *id_out = static_cast<uint64_t>(id);
    });
}

// World::remove_constraint (src/world.cpp:277-279 -> Scene::retire_constraint).
int fz_ref_remove_joint(void* p, uint64_t id) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] { h->scene->retire_constraint(static_cast<fyzz::ConstraintId>(id)); });
}

// Scene::set_kinematic / set_kinematic_target (scene.cpp:858-1003) for the
// 0-based dynamic body index i; the target is validated as World does
// (src/world.cpp:361-366) and normalised once by the scene.
int fz_ref_set_kinematic(void* p, uint32_t i, int on) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] { h->scene->set_kinematic(h->bodies.at(i), on != 0); });
}
int fz_ref_set_kinematic_target(void* p, uint32_t i, const float* pose) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] {
        const float m = std::sqrt(pose[3]*pose[3] + pose[4]*pose[4] + pose[5]*pose[5] + pose[6]*pose[6]);
        if (!std::isfinite(m) || std::abs(m - 1.0f) >= 1.0e-2f)
            throw std::invalid_argument("Rigid pose orientation is not sane");
        h->scene->set_kinematic_target(h->bodies.at(i), {pose[0], pose[1], pose[2]},
                                       {pose[3], pose[4], pose[5], pose[6]});
    });
}

int fz_ref_step(void* p, float dt, int steps) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] {
        for (int i = 0; i < steps; ++i) h->scene->step(dt);
    });
}

int fz_ref_advance_collision(void* p) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] { h->scene->advance_collision(false); });
}

// [actors, shapes, pairs, found, lost, manifolds, contact points,
//  partitions, ordered descriptors, tasks]
void fz_ref_counts(void* p, uint64_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    out[0] = Fix::actors(s).size();
    out[1] = Fix::shapes(s).size();
    out[2] = s.pairs().size();
    out[3] = s.found_pairs().size();
    out[4] = s.lost_pairs().size();
    out[5] = s.contacts().size();
    uint64_t pts = 0;
    for (const auto& m : s.contacts()) pts += m.count;
    out[6] = pts;
    out[7] = Fix::partition_ends(s).size();
    out[8] = Fix::ordered(s).size();
    out[9] = Fix::tasks(s).size();
}

// Per actor: position(3) velocity(3) orientation(4) angular velocity(3)
// sleeping(1) = 14 floats.
void fz_ref_body_states(void* p, float* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto n = Fix::actors(s).size();
    for (std::size_t i = 0; i < n; ++i) {
        const auto st = s.body_state(static_cast<fyzz::BodyId>(i));
        float* o = out + 14 * i;
        o[0] = st.position.x; o[1] = st.position.y; o[2] = st.position.z;
        o[3] = st.velocity.x; o[4] = st.velocity.y; o[5] = st.velocity.z;
        o[6] = st.orientation.x; o[7] = st.orientation.y;
        o[8] = st.orientation.z; o[9] = st.orientation.w;
        o[10] = st.angular_velocity.x; o[11] = st.angular_velocity.y;
        o[12] = st.angular_velocity.z; o[13] = st.sleeping ? 1.0f : 0.0f;
    }
}

// Per actor: wake counter, sleeping, ready for sleep, counted interactions,
// sleep-filter linear and local angular motion (scene.h:1147-1156) = 10
// floats.
void fz_ref_sleep_state(void* p, float* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& actors = Fix::actors(s);
    for (std::size_t i = 0; i < actors.size(); ++i) {
        const auto& a = actors[i];
        float* o = out + 10 * i;
        o[0] = a.wake_counter;
        o[1] = a.sleeping ? 1.0f : 0.0f;
        o[2] = a.ready_for_sleep ? 1.0f : 0.0f;
        o[3] = static_cast<float>(a.num_counted_interactions);
        o[4] = a.sleep_linear_acc.x; o[5] = a.sleep_linear_acc.y; o[6] = a.sleep_linear_acc.z;
        o[7] = a.sleep_angular_acc.x; o[8] = a.sleep_angular_acc.y; o[9] = a.sleep_angular_acc.z;
    }
}

// Per actor: inverse mass, inverse inertia(3), mass-local position(3),
// mass-local orientation(4) = 11 floats.  Statics are zero-filled.
void fz_ref_mass_props(void* p, float* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& actors = Fix::actors(s);
    for (std::size_t i = 0; i < actors.size(); ++i) {
        float* o = out + 11 * i;
        std::memset(o, 0, 11 * sizeof(float));
        const auto& a = actors[i];
        o[0] = a.inverse_mass;
        o[1] = a.inverse_inertia_local.x; o[2] = a.inverse_inertia_local.y;
        o[3] = a.inverse_inertia_local.z;
        o[4] = a.mass_local_pose.position.x; o[5] = a.mass_local_pose.position.y;
        o[6] = a.mass_local_pose.position.z;
        o[7] = a.mass_local_pose.orientation.x; o[8] = a.mass_local_pose.orientation.y;
        o[9] = a.mass_local_pose.orientation.z; o[10] = a.mass_local_pose.orientation.w;
    }
}

// Per shape: the 6 encoded u32 bounds (min xyz, max xyz) as last published
// by Scene::update_shape_bounds (src/native/scene.cpp:1233-1316).
void fz_ref_encoded_bounds(void* p, uint32_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& shapes = Fix::shapes(s);
    for (std::size_t i = 0; i < shapes.size(); ++i)
        for (int k = 0; k < 6; ++k) out[6 * i + k] = shapes[i].encoded_bounds[k];
}

// Sorted SAP endpoints of one axis: value, shape id, is_max.
uint64_t fz_ref_endpoints(void* p, int axis, uint32_t* values, uint32_t* ids,
                          uint8_t* is_max) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& e = Fix::endpoints(s, static_cast<unsigned>(axis));
    if (values)
        for (std::size_t i = 0; i < e.size(); ++i) {
            values[i] = e[i].value;
            ids[i] = e[i].id;
            is_max[i] = e[i].is_max ? 1 : 0;
        }
    return e.size();
}

// which: 0 = current overlap pairs, 1 = found, 2 = lost.  2 u32 per pair.
uint64_t fz_ref_pairs(void* p, int which, uint32_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    auto span = which == 0 ? s.pairs() : which == 1 ? s.found_pairs() : s.lost_pairs();
    if (out)
        for (std::size_t i = 0; i < span.size(); ++i) {
            out[2*i] = span[i].a;
            out[2*i+1] = span[i].b;
        }
    return span.size();
}

// Published Gu manifolds in pair order: pair(2), count, Gu-order-reversed
// flag, and up to 4 points of position(3) normal(3) separation(1).
uint64_t fz_ref_manifolds(void* p, uint32_t* pairs, uint32_t* counts,
                          uint32_t* reversed, float* points) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto m = s.contacts();
    if (pairs)
        for (std::size_t i = 0; i < m.size(); ++i) {
            pairs[2*i] = m[i].pair.a;
            pairs[2*i+1] = m[i].pair.b;
            counts[i] = m[i].count;
            reversed[i] = Fix::reversed(s, m[i].edge_handle) ? 1u : 0u;
            for (std::size_t k = 0; k < 4; ++k) {
                float* o = points + 28 * i + 7 * k;
                if (k < m[i].count) {
                    const auto& c = m[i].points[k];
                    o[0] = c.position.x; o[1] = c.position.y; o[2] = c.position.z;
                    o[3] = c.normal.x; o[4] = c.normal.y; o[5] = c.normal.z;
                    o[6] = c.separation;
                } else {
                    std::memset(o, 0, 7 * sizeof(float));
                }
            }
        }
    return m.size();
}

// Dy descriptor input order of the last step: manifold indices in the
// order partition_constraints consumed them (scene.cpp:7174-7216), and the
// constraint slots of the 1D joints in their per-task order.
uint64_t fz_ref_manager_order(void* p, uint64_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& v = Fix::indexed_managers(s);
    if (out) for (std::size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return v.size();
}
// The same order as shape pairs (a < b, 2 u32 each).
uint64_t fz_ref_manager_order_pairs(void* p, uint32_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& v = Fix::indexed_managers(s);
    const auto& m = Fix::manifolds(s);
    if (out)
        for (std::size_t i = 0; i < v.size(); ++i) {
            out[2 * i] = m[v[i]].pair.a;
            out[2 * i + 1] = m[v[i]].pair.b;
        }
    return v.size();
}
uint64_t fz_ref_joint_order(void* p, uint64_t* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& v = Fix::indexed_joints(s);
    const auto& edges = Fix::island_edges(s);
    if (out) for (std::size_t i = 0; i < v.size(); ++i) out[i] = edges[v[i]].constraint_id;
    return v.size();
}
// Partitioned descriptors (scene.cpp:7459-7488): index, row0, row1,
// row_count, plus the cumulative partition ends.
uint64_t fz_ref_partitions(void* p, uint32_t* desc, uint64_t* ends) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto& d = Fix::ordered(s);
    const auto& e = Fix::partition_ends(s);
    if (desc)
        for (std::size_t i = 0; i < d.size(); ++i) {
            desc[4*i] = d[i].index; desc[4*i+1] = d[i].row0;
            desc[4*i+2] = d[i].row1; desc[4*i+3] = d[i].row_count;
        }
    if (ends) for (std::size_t i = 0; i < e.size(); ++i) ends[i] = e[i];
    return d.size();
}

uint64_t fz_ref_normal_impulses(void* p, double* out) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto v = s.solved_normal_impulses();
    if (out) for (std::size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    return v.size();
}

// Contact events: body0, body1, kind, count, point offset, shape0, shape1 as
// u32 (7 per event) plus the summed normal impulse.
uint64_t fz_ref_contact_events(void* p, uint32_t* ev, double* impulse) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto e = s.contact_events();
    if (ev)
        for (std::size_t i = 0; i < e.size(); ++i) {
            uint32_t* o = ev + 7 * i;
            o[0] = e[i].body0; o[1] = e[i].body1;
            o[2] = static_cast<uint32_t>(e[i].kind); o[3] = e[i].contact_count;
            o[4] = static_cast<uint32_t>(e[i].point_offset);
            o[5] = e[i].shape0; o[6] = e[i].shape1;
            impulse[i] = e[i].normal_impulse;
        }
    return e.size();
}

// Contact event points: position(3) normal(3) separation as floats plus the
// normal impulse (ContactEventPoint, world.h:194-199).
uint64_t fz_ref_contact_event_points(void* p, float* pts, double* impulse) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto e = s.contact_event_points();
    if (pts)
        for (std::size_t i = 0; i < e.size(); ++i) {
            float* o = pts + 7 * i;
            o[0] = e[i].position.x; o[1] = e[i].position.y; o[2] = e[i].position.z;
            o[3] = e[i].normal.x; o[4] = e[i].normal.y; o[5] = e[i].normal.z;
            o[6] = e[i].separation;
            impulse[i] = e[i].normal_impulse;
        }
    return e.size();
}

// Scene::set_contact_report_threshold (scene.cpp:1148-1161) on an actor
// (BodyId: the floor, when present, is 0).
int fz_ref_set_contact_report_threshold(void* p, uint32_t actor, float force) {
    return guarded([&] { static_cast<Handle*>(p)->scene->set_contact_report_threshold(actor, force); });
}

// Scene::force_threshold_changes (scene.h:853): per report actor0, actor1,
// static_world, change (ForceThresholdChange) as u32, the impulse and the
// threshold.
uint64_t fz_ref_force_threshold_changes(void* p, uint32_t* rows, double* impulse, float* threshold) {
    const Scene& s = *static_cast<Handle*>(p)->scene;
    const auto t = s.force_threshold_changes();
    if (rows)
        for (std::size_t i = 0; i < t.size(); ++i) {
            rows[4 * i] = t[i].key.actor0;
            rows[4 * i + 1] = t[i].key.actor1;
            rows[4 * i + 2] = t[i].key.static_world ? 1u : 0u;
            rows[4 * i + 3] = static_cast<uint32_t>(t[i].change);
            impulse[i] = t[i].normal_impulse;
            threshold[i] = t[i].threshold;
        }
    return t.size();
}

// ---- stateless Gu generators (public free functions of the reference) ----
// ---- cooked convex meshes (include/fyzzxyzzy/convex.h, cooked_convex.cpp) ----
// Cooks through fyzz::cook_convex_mesh.  Outputs, sized by the caller for
// 3 * nt faces and indices: faces as normal(3) distance(1) first(1)
// count(1) floats, the face index stream, counts {nf, ni}, the volume and
// center(3) inertia columns(9) bounds min(3) max(3).
int fz_ref_cook_convex(const float* verts, uint32_t nv, const uint32_t* tris, uint32_t nt,
                       float* faces6, uint32_t* idx, uint32_t* counts, double* volume, float* mass18) {
    return guarded([&] {
        std::vector<fyzz::Vec3> v(nv);
        for (uint32_t i = 0; i < nv; ++i) v[i] = {verts[3*i], verts[3*i+1], verts[3*i+2]};
        std::vector<fyzz::ConvexTriangle> t(nt);
        for (uint32_t i = 0; i < nt; ++i) t[i] = {tris[3*i], tris[3*i+1], tris[3*i+2]};
        const auto m = fyzz::cook_convex_mesh(v, t);
        const auto f = m->faces();
        const auto fi = m->face_indices();
        counts[0] = static_cast<uint32_t>(f.size());
        counts[1] = static_cast<uint32_t>(fi.size());
        for (std::size_t i = 0; i < f.size(); ++i) {
            float* o = faces6 + 6 * i;
            o[0] = f[i].normal.x; o[1] = f[i].normal.y; o[2] = f[i].normal.z; o[3] = f[i].distance;
            o[4] = static_cast<float>(f[i].first_index); o[5] = static_cast<float>(f[i].index_count);
        }
        for (std::size_t i = 0; i < fi.size(); ++i) idx[i] = fi[i];
        const auto& mp = m->mass_properties();
        *volume = mp.volume;
        mass18[0] = mp.center.x; mass18[1] = mp.center.y; mass18[2] = mp.center.z;
        for (int c = 0; c < 3; ++c) {
            mass18[3 + 3*c] = mp.inertia_columns[c].x;
            mass18[4 + 3*c] = mp.inertia_columns[c].y;
            mass18[5 + 3*c] = mp.inertia_columns[c].z;
        }
        const auto lo = m->bounds_min(), hi = m->bounds_max();
        mass18[12] = lo.x; mass18[13] = lo.y; mass18[14] = lo.z;
        mass18[15] = hi.x; mass18[16] = hi.y; mass18[17] = hi.z;
    });
}

// Meshes for fz_ref_build's convex shapes (shape_type 3, mesh index in
// shape_geom[0]); call before fz_ref_build.  Mesh m has mesh_nv[m] vertices
// and mesh_nt[m] triangles, concatenated in mesh order.
int fz_ref_set_meshes(void* p, uint32_t n, const uint32_t* mesh_nv, const float* verts,
                      const uint32_t* mesh_nt, const uint32_t* tris) {
    auto* h = static_cast<Handle*>(p);
    return guarded([&] {
        h->meshes.clear();
        std::size_t vo = 0, to = 0;
        for (uint32_t m = 0; m < n; ++m) {
            std::vector<fyzz::Vec3> v(mesh_nv[m]);
            for (uint32_t i = 0; i < mesh_nv[m]; ++i)
                v[i] = {verts[3*(vo+i)], verts[3*(vo+i)+1], verts[3*(vo+i)+2]};
            std::vector<fyzz::ConvexTriangle> t(mesh_nt[m]);
            for (uint32_t i = 0; i < mesh_nt[m]; ++i)
                t[i] = {tris[3*(to+i)], tris[3*(to+i)+1], tris[3*(to+i)+2]};
            h->meshes.push_back(fyzz::cook_convex_mesh(v, t));
            vo += mesh_nv[m];
            to += mesh_nt[m];
        }
    });
}

// Finite shape descriptors for the convex Gu functions: half extents(3)
// position(3) orientation xyzw(4) sphere radius(1), plus a mesh index into
// the handle's meshes (-1 for none).
static fyzz::native::PcmFiniteShape finite_of(const Handle* h, const float* d, int mesh) {
    fyzz::native::PcmFiniteShape f{};
    f.half_extents = {d[0], d[1], d[2]};
    f.position = {d[3], d[4], d[5]};
    f.orientation = {d[6], d[7], d[8], d[9]};
    f.sphere_radius = d[10];
    if (mesh >= 0) {
        const auto& m = h->meshes.at(static_cast<std::size_t>(mesh));
        f.hull_vertices = m->vertices();
        f.hull_faces = m->faces();
        f.hull_face_indices = m->face_indices();
    }
    return f;
}
static void put_candidate(const fyzz::native::PcmContactCandidate& k, float* o) {
    o[0]=k.local_a.x; o[1]=k.local_a.y; o[2]=k.local_a.z;
    o[3]=k.local_b.x; o[4]=k.local_b.y; o[5]=k.local_b.z;
    o[6]=k.normal_b.x; o[7]=k.normal_b.y; o[8]=k.normal_b.z;
    o[9]=k.separation;
}
int fz_ref_pcm_convex_gjk_epa(void* p, const float* a, int mesh_a, const float* b, int mesh_b,
                              float cd, float* out) {
    const auto* h = static_cast<const Handle*>(p);
    fyzz::native::PcmContactCandidate k{};
    bool ok = false;
    const int rc = guarded([&] {
        ok = fyzz::native::source_pcm_convex_gjk_epa(finite_of(h, a, mesh_a), finite_of(h, b, mesh_b), cd, k,
                                                     nullptr);
    });
    if (rc) return -rc;
    put_candidate(k, out);
    return ok ? 1 : 0;
}
int fz_ref_pcm_convex_face_contacts(void* p, const float* a, int mesh_a, const float* b, int mesh_b,
                                    float cd, const float* witness, float* out) {
    const auto* h = static_cast<const Handle*>(p);
    std::array<fyzz::native::PcmContactCandidate, 4> c{};
    int n = 0;
    const int rc = guarded([&] {
        const float* w = witness;
        const fyzz::native::PcmContactCandidate k{{w[0],w[1],w[2]}, {w[3],w[4],w[5]}, {w[6],w[7],w[8]}, w[9]};
        n = fyzz::native::source_pcm_convex_face_contacts(finite_of(h, a, mesh_a), finite_of(h, b, mesh_b), cd,
                                                          k, c);
    });
    if (rc) return -rc;
    for (int i = 0; i < n; ++i) put_candidate(c[i], out + 10 * i);
    return n;
}

// Shape records: half extents(3) position(3) orientation xyzw(4).
// Candidate records: local_a(3) local_b(3) normal_b(3) separation(1).
int fz_ref_pcm_box_box_candidates(const float* a, const float* b, float cd,
                                  float* out, uint32_t* count) {
    using namespace fyzz;
    std::vector<native::PcmContactCandidate> c(64);
    std::size_t n = 0;
    bool ok = false;
    const int rc = guarded([&] {
        ok = native::source_pcm_box_box_candidates(
            {a[0],a[1],a[2]}, {a[3],a[4],a[5]}, {a[6],a[7],a[8],a[9]},
            {b[0],b[1],b[2]}, {b[3],b[4],b[5]}, {b[6],b[7],b[8],b[9]}, cd, c, n);
    });
    if (rc) return -rc;
    *count = static_cast<uint32_t>(n);
    for (std::size_t i = 0; i < n; ++i) {
        float* o = out + 10 * i;
        const auto& k = c[i];
        o[0]=k.local_a.x; o[1]=k.local_a.y; o[2]=k.local_a.z;
        o[3]=k.local_b.x; o[4]=k.local_b.y; o[5]=k.local_b.z;
        o[6]=k.normal_b.x; o[7]=k.normal_b.y; o[8]=k.normal_b.z;
        o[9]=k.separation;
    }
    return ok ? 1 : 0;
}

int fz_ref_pcm_batch_selection(const float* candidates, uint32_t n, uint8_t* out) {
    using namespace fyzz;
    std::vector<native::PcmContactCandidate> c(n);
    for (uint32_t i = 0; i < n; ++i) {
        const float* k = candidates + 10 * i;
        c[i] = {{k[0],k[1],k[2]}, {k[3],k[4],k[5]}, {k[6],k[7],k[8]}, k[9]};
    }
    std::array<std::uint8_t, 4> sel{};
    const int rc = guarded([&] { sel = native::source_pcm_box_batch_selection(c, 1.0f); });
    if (rc) return -rc;
    for (int i = 0; i < 4; ++i) out[i] = sel[i];
    return 0;
}

int fz_ref_pcm_box_box_gjk_epa(const float* a, const float* b, float cd, float* out) {
    using namespace fyzz;
    native::PcmContactCandidate k{};
    bool ok = false;
    const int rc = guarded([&] {
        ok = native::source_pcm_box_box_gjk_epa(
            {a[0],a[1],a[2]}, {a[3],a[4],a[5]}, {a[6],a[7],a[8],a[9]},
            {b[0],b[1],b[2]}, {b[3],b[4],b[5]}, {b[6],b[7],b[8],b[9]}, cd, k, nullptr);
    });
    if (rc) return -rc;
    out[0]=k.local_a.x; out[1]=k.local_a.y; out[2]=k.local_a.z;
    out[3]=k.local_b.x; out[4]=k.local_b.y; out[5]=k.local_b.z;
    out[6]=k.normal_b.x; out[7]=k.normal_b.y; out[8]=k.normal_b.z;
    out[9]=k.separation;
    return ok ? 1 : 0;
}

// Sphere generators: output position(3) normal(3) separation(1).
int fz_ref_pcm_sphere_sphere(const float* c0, float r0, const float* c1, float r1,
                             float cd, float* out) {
    std::array<fyzz::native::ContactPoint, 1> o{};
    const auto n = fyzz::native::source_pcm_sphere_sphere(
        {c0[0],c0[1],c0[2]}, r0, {c1[0],c1[1],c1[2]}, r1, cd, o);
    const auto& k = o[0];
    out[0]=k.position.x; out[1]=k.position.y; out[2]=k.position.z;
    out[3]=k.normal.x; out[4]=k.normal.y; out[5]=k.normal.z; out[6]=k.separation;
    return n;
}
int fz_ref_pcm_sphere_box(const float* c, float r, const float* box /*h3 p3 q4*/,
                          float cd, float* out) {
    std::array<fyzz::native::ContactPoint, 1> o{};
    const auto n = fyzz::native::source_pcm_sphere_box(
        {c[0],c[1],c[2]}, r, {box[3],box[4],box[5]},
        {box[6],box[7],box[8],box[9]}, {box[0],box[1],box[2]}, cd, o);
    const auto& k = o[0];
    out[0]=k.position.x; out[1]=k.position.y; out[2]=k.position.z;
    out[3]=k.normal.x; out[4]=k.normal.y; out[5]=k.normal.z; out[6]=k.separation;
    return n;
}

// Steps many independent scenes on `threads` host threads: the batched CPU
// baseline (one NativeCpu Scene per batched scene, as the reference has no
// batch API).  Returns 0 or the first error code.
int fz_ref_step_many(void** handles, uint32_t n, float dt, int steps, int threads) {
    if (threads < 1) threads = 1;
    std::vector<int> rc(threads, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&, t] {
            for (uint32_t i = t; i < n; i += threads) {
                const int r = fz_ref_step(handles[i], dt, steps);
                if (r && !rc[t]) rc[t] = r;
            }
        });
    for (auto& th : pool) th.join();
    for (int r : rc) if (r) return r;
    return 0;
}

} // extern "C"
