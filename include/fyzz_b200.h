/* fyzz_b200.h - C ABI of the B200 rigid-body step.
 *
 * A drop-in for the FyzzXYZZY NativePortableGpu step: the entry points mirror
 * fyzz::World / fyzz::WorldBackend (include/fyzzxyzzy/world.h:226-510 of the
 * reference) and its GPU factory create_native_gpu_world
 * (include/fyzzxyzzy/native_gpu_world.h:90-138).  Plain pointers and sizes
 * only; no C++ or torch types cross this boundary.
 *
 * Status codes map 1:1 to the reference's exception types
 * (world.h, src/native/scene.cpp): 1 std::invalid_argument,
 * 2 std::logic_error, 3 std::overflow_error, 4 std::runtime_error.
 *
 * Identifiers.  Body and shape ids are world-global, allocated in creation
 * order like the reference's BodyId / ShapeId (scene.cpp:192-252).  A world
 * holds one scene unless fyzz_b200_begin_scene is called; scenes are
 * independent (no pairs across scenes) and are stepped together.
 *
 * Threading: a world is not thread-safe (reference compute.h:265).
 */
#ifndef FYZZ_B200_H
#define FYZZ_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum {
    FYZZ_B200_OK = 0,
    FYZZ_B200_INVALID_ARGUMENT = 1,
    FYZZ_B200_LOGIC_ERROR = 2,
    FYZZ_B200_OVERFLOW = 3,
    FYZZ_B200_RUNTIME_ERROR = 4
};

typedef struct fyzz_b200_world fyzz_b200_world;

/* fyzz::Material (world.h:78-90): friction / restitution used by the step. */
typedef struct {
    float static_friction;
    float dynamic_friction;
    float restitution;
} fyzz_b200_material;

/* fyzz::BodyState (world.h:201-212). */
typedef struct {
    float position[3];
    float velocity[3];
    float orientation[4]; /* x, y, z, w */
    float angular_velocity[3];
    uint32_t sleeping;
} fyzz_b200_body_state_t;

/* Device pointers of the resident state, for callers that keep their
 * inputs in HBM (float4 records: xyz + pad; see fyzz_b200_read_bodies for
 * the host layout). */
typedef struct {
    void* position;         /* float4 per body, w = inverse mass */
    void* orientation;      /* float4 per body */
    void* velocity;         /* float4 per body */
    void* angular_velocity; /* float4 per body */
    uint32_t n_bodies;
    uint32_t n_shapes;
    void* stream;           /* cudaStream_t the world launches on */
} fyzz_b200_device_view_t;

/* ---- lifecycle: create_native_gpu_world (native_gpu_world.h:90-138) ---- */
int fyzz_b200_create(int device, fyzz_b200_world** out);
int fyzz_b200_destroy(fyzz_b200_world* w);
/* Message of the last failed call on this world (valid until the next call). */
const char* fyzz_b200_last_error(const fyzz_b200_world* w);
/* Device error bits of the last step (source_dy_distance_native.h:1336-1345). */
int fyzz_b200_error_bits(const fyzz_b200_world* w, uint32_t* bits);

/* ---- authoring: WorldBackend (world.h:226-394) ----
 * Transforms are validated and normalised as fyzz::World does before its
 * backend (src/world.cpp:38-55) and once more as the scene does
 * (Scene::validated_pose, src/native/compound.cpp:9-18). */
/* For a caller that is itself fyzz::World (this world behind a
 * WorldBackend): transforms arrive validated, so only the scene's
 * normalisation is applied.  No reference counterpart. */
int fyzz_b200_set_caller_validated_transforms(fyzz_b200_world* w, int enabled);
/* New independent scene; later bodies belong to it.  (No reference
 * counterpart: the reference World holds exactly one scene.) */
int fyzz_b200_begin_scene(fyzz_b200_world* w, uint32_t* scene_out);
/* World::add_static_floor (world.h:424) */
int fyzz_b200_add_static_floor(fyzz_b200_world* w, float height, uint32_t* body_out);
/* World::create_dynamic_body (world.h:409); pose = position(3) + quaternion xyzw(4) */
int fyzz_b200_create_dynamic_body(fyzz_b200_world* w, const float pose[7], uint32_t* body_out);
/* World::attach_box_shape (world.h:410) */
int fyzz_b200_attach_box_shape(fyzz_b200_world* w, uint32_t body, const float half_extents[3],
                               const float local_pose[7], uint32_t* shape_out);
/* World::attach_sphere_shape (world.h:411) */
int fyzz_b200_attach_sphere_shape(fyzz_b200_world* w, uint32_t body, float radius,
                                  const float local_pose[7], uint32_t* shape_out);
/* ---- cooked convex hulls: cook_convex_mesh (include/fyzzxyzzy/convex.h:56-60,
 * src/native/cooked_convex.cpp:41-330) and World::attach_convex_shape
 * (world.h:412-413, scene.cpp:283-340) ---- */
typedef struct fyzz_b200_convex_mesh fyzz_b200_convex_mesh;
/* Cooks an outward-wound, closed, convex, manifold triangle surface
 * (n_vertices x 3 floats, n_triangles x 3 indices).  Coplanar triangles
 * become one polygon face.  Rejected meshes return FYZZ_B200_INVALID_ARGUMENT
 * with the reason in fyzz_b200_cook_error().  The mesh is reference
 * counted: worlds that attach it keep their own reference, so the caller
 * may release it at any time. */
int fyzz_b200_cook_convex_mesh(const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                               uint32_t n_triangles, fyzz_b200_convex_mesh** mesh_out);
void fyzz_b200_convex_mesh_release(fyzz_b200_convex_mesh* mesh);
/* Message of this thread's last failed cook. */
const char* fyzz_b200_cook_error(void);
/* ConvexMesh accessors (convex.h:34-53); any output may be NULL.
 * counts: vertices, faces, face indices.  faces6: per face normal(3),
 * distance, first index, index count.  mass18: centre of mass(3), inertia
 * columns(9) about it for density one, bounds min(3), max(3). */
int fyzz_b200_convex_mesh_info(const fyzz_b200_convex_mesh* mesh, uint32_t counts[3], float* faces6,
                               uint32_t* face_indices, double* volume, float* mass18);
/* World::attach_convex_shape (world.h:412) */
int fyzz_b200_attach_convex_shape(fyzz_b200_world* w, uint32_t body, const fyzz_b200_convex_mesh* mesh,
                                  const float local_pose[7], uint32_t* shape_out);
/* World::update_mass_properties (world.h:420, compound.cpp:113-203) */
int fyzz_b200_update_mass_properties(fyzz_b200_world* w, uint32_t body, float density);
/* World::body_mass_properties (world.h:421): inverse mass, inverse inertia(3),
 * mass-local position(3), mass-local orientation(4). */
int fyzz_b200_body_mass_properties(const fyzz_b200_world* w, uint32_t body, float out[11]);
/* World::set_shape_material (world.h:416) */
int fyzz_b200_set_shape_material(fyzz_b200_world* w, uint32_t shape, const fyzz_b200_material* m);
/* World::set_body_velocity / set_body_angular_velocity (world.h:477-478) */
int fyzz_b200_set_body_velocity(fyzz_b200_world* w, uint32_t body, const float v[3]);
int fyzz_b200_set_body_angular_velocity(fyzz_b200_world* w, uint32_t body, const float v[3]);
/* World::add_center_distance_constraint (world.h:438) */
int fyzz_b200_add_center_distance_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b,
                                             float distance, uint64_t* id_out);
/* World::add_anchored_distance_constraint (world.h:441): equal-limit 1D
 * joint between body-local anchors.  As in the reference, the anchors are
 * applied to the lower and higher BodyId in the order given. */
int fyzz_b200_add_anchored_distance_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[3],
                                               const float local_b[3], float distance, uint64_t* id_out);
/* World::add_fixed_constraint / add_spherical_constraint /
 * add_revolute_constraint / add_prismatic_constraint (world.h:445-457):
 * local frames are position(3) + orientation xyzw(4) in each body's frame.
 * Fixed locks the relative pose (6 rows); spherical makes the frame origins
 * coincide (3 rows); revolute also aligns the local X axes (5 rows, free
 * rotation about X); prismatic keeps the relative orientation and the
 * transverse position (5 rows, free translation along frame A's X). */
int fyzz_b200_add_fixed_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                   const float local_b[7], uint64_t* id_out);
int fyzz_b200_add_spherical_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                       const float local_b[7], uint64_t* id_out);
int fyzz_b200_add_revolute_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                      const float local_b[7], uint64_t* id_out);
int fyzz_b200_add_prismatic_constraint(fyzz_b200_world* w, uint32_t a, uint32_t b, const float local_a[7],
                                       const float local_b[7], uint64_t* id_out);
/* World::remove_constraint (world.h:458, Scene::retire_constraint): the
 * joint leaves the next step; ids are generation << 32 | slot and a
 * retired slot is reused (generation + 1) by the scene's next joint.
 * Unknown or expired ids return FYZZ_B200_INVALID_ARGUMENT.  Joints added
 * or removed between steps keep the contact-manager history. */
int fyzz_b200_remove_constraint(fyzz_b200_world* w, uint64_t id);

/* Bulk authoring of one scene with the seeded-workload record layout:
 * bodies(14 floats: position 3, orientation 4, velocity 3, angular 3,
 * density), per-shape owner / type (0 box, 1 sphere) / geometry(4) /
 * local pose(7) / material(3), distance joints, optional floor (created
 * first, with material floor_mat).  Equivalent to the per-call sequence
 * add_static_floor, create_dynamic_body, attach_*_shape,
 * update_mass_properties, set_shape_material, set_body_velocity,
 * set_body_angular_velocity, add_center_distance_constraint. */
int fyzz_b200_add_scene(fyzz_b200_world* w, uint32_t n_bodies, const float* bodies,
                        uint32_t n_shapes, const uint32_t* shape_body, const uint32_t* shape_type,
                        const float* shape_geom, const float* shape_local, const float* shape_mat,
                        uint32_t n_joints, const uint32_t* joint_bodies, const float* joint_dist,
                        int has_floor, float floor_height, const float* floor_mat,
                        uint32_t* first_body_out);
/* fyzz_b200_add_scene with cooked hulls: shape type 3 attaches
 * meshes[(uint32_t)shape_geom[4 * i]] (World::attach_convex_shape). */
int fyzz_b200_add_scene_ex(fyzz_b200_world* w, uint32_t n_bodies, const float* bodies,
                           uint32_t n_shapes, const uint32_t* shape_body, const uint32_t* shape_type,
                           const float* shape_geom, const float* shape_local, const float* shape_mat,
                           uint32_t n_joints, const uint32_t* joint_bodies, const float* joint_dist,
                           int has_floor, float floor_height, const float* floor_mat,
                           uint32_t n_meshes, fyzz_b200_convex_mesh* const* meshes, uint32_t* first_body_out);

/* ---- stepping: World::step (world.h:459, scene.cpp:10725) ----
 * Failure-atomic like Scene::step (scene.cpp:11013-11016): when the device
 * reports an error the world returns to its state before the call (bodies,
 * sleep state and the contact-manager history: PCM caches, friction
 * histories, touch counts).  A pair-budget overflow grows the budget and
 * runs the steps again; non-finite state returns FYZZ_B200_OVERFLOW and a
 * bounded device wait that gave up FYZZ_B200_LOGIC_ERROR.  Velocities
 * written in bulk (fyzz_b200_write_velocities*) are not checked on the
 * host: a non-finite one makes the next step fail this way. */
int fyzz_b200_step(fyzz_b200_world* w, float seconds);
/* `steps` consecutive steps launched as one captured CUDA graph per step,
 * with a single error check at the end. */
int fyzz_b200_step_n(fyzz_b200_world* w, float seconds, uint32_t steps);
/* Scene::advance_collision (scene.h:819): bounds, pairs and manifolds only. */
int fyzz_b200_collide(fyzz_b200_world* w);
int fyzz_b200_synchronize(fyzz_b200_world* w);
/* One step launched without the graph, with CUDA events on the world's
 * stream at each stage boundary.  stage_ms receives up to n stage times:
 * 0 bounds, 1 endpoint sort, 2 pairs, 3 narrowphase, 4 islands,
 * 5 partitions and row preparation (concurrent graph branches), 6 PGS,
 * 7 integration.  (Counterpart of the reference's
 * Context::profile_batch_gpu_nanoseconds, compute.h:299.) */
int fyzz_b200_profile_step(fyzz_b200_world* w, float seconds, float* stage_ms, uint32_t n);
/* ---- performance parameters (no reference counterpart) ----
 * Choices that change how the step runs, not what it computes: every
 * setting gives bit-identical results.  A world starts from the tuning
 * table next to the library (tuning.txt, written by the package's
 * autotune.py on a B200; FYZZ_B200_TUNING names another file, "none"
 * keeps the defaults below), taking the line of its class: "large_scene"
 * when some scene has more than 2,048 finite shapes, else "many_scenes".
 * fyzz_b200_set_tuning overrides it for the world. */
typedef struct {
    uint32_t island_thread;  /* islands of at most this many descriptors are solved by one thread (0..8; 8) */
    uint32_t island_warp;    /* ... up to this many by one warp (32..96; 96) */
    uint32_t island_cta;     /* ... up to this many by one 128-thread CTA (128..512; 512); larger islands up to
                                4,096 by one 384-thread CTA, beyond that from global memory */
    uint32_t radix_bits;     /* digit width of the device-wide radix sorts (8..11; 8) */
    uint32_t elem_block;     /* threads a block of the elementwise kernels (64..1024, multiple of 32; 256) */
    uint32_t work_queue;     /* warp and CTA solvers take islands round-robin (0) or from a device work
                                queue, the next list entry per worker from a per-step counter (1); 0 */
} fyzz_b200_tuning_t;
int fyzz_b200_set_tuning(fyzz_b200_world* w, const fyzz_b200_tuning_t* tuning);
int fyzz_b200_get_tuning(fyzz_b200_world* w, fyzz_b200_tuning_t* tuning);
/* Kernel launches in one captured step graph (0 before the first step). */
int fyzz_b200_kernels_per_step(fyzz_b200_world* w, uint32_t* out);

/* ---- results ---- */
/* World::body_state (world.h:460) */
int fyzz_b200_body_state(const fyzz_b200_world* w, uint32_t body, fyzz_b200_body_state_t* out);
/* All bodies, 14 floats each: position(3) velocity(3) orientation(4)
 * angular velocity(3) sleeping(1).  Host buffer. */
int fyzz_b200_read_bodies(fyzz_b200_world* w, float* out, uint32_t n_bodies);
/* Overwrite linear(3) + angular(3) velocities of all bodies from a host
 * buffer (6 floats per body; statics ignored). */
int fyzz_b200_write_velocities(fyzz_b200_world* w, const float* v6, uint32_t n_bodies);
/* The same from records of `stride` floats per body with the linear and
 * angular velocity at the given float offsets: a loop that edits the
 * 14-float records of fyzz_b200_read_bodies writes them back as they are
 * (stride 14, offsets 3 and 10).  No reference counterpart. */
int fyzz_b200_write_velocities_strided(fyzz_b200_world* w, const float* records, uint32_t n_bodies,
                                       uint32_t stride, uint32_t linear_offset, uint32_t angular_offset);
/* Counts: [bodies, shapes, scenes, pairs, touching managers, contact points,
 * descriptors, islands, joints, steps, friction rows, found + lost pairs] */
int fyzz_b200_counts(fyzz_b200_world* w, uint64_t out[12]);
int fyzz_b200_device_view(fyzz_b200_world* w, fyzz_b200_device_view_t* out);

/* ---- contact events: World::contact_events / contact_event_points
 *      (world.h:176-199, 466-468; Scene::publish_contact_events,
 *      scene.cpp:9149-9264) ---- */
/* ContactEvent.  kind: 0 Found, 1 Persists, 2 Lost (ContactEventKind).
 * body0 < body1; shape0 belongs to body0.  point_offset indexes the points
 * span; lost events carry no points and zero impulse. */
typedef struct {
    uint32_t body0, body1;
    uint32_t shape0, shape1;
    uint32_t kind;
    uint32_t contact_count;
    uint64_t point_offset;
    double normal_impulse;  /* sum of the points' impulses */
} fyzz_b200_contact_event_t;
/* ContactEventPoint: manifold point with its normal oriented from body0's
 * solver side, and the final normal impulse of its solver row. */
typedef struct {
    float position[3];
    float normal[3];
    float separation;
    uint32_t reserved;
    double normal_impulse;
} fyzz_b200_contact_event_point_t;
/* WorldOptions::contact_notifications (world.h:61); off by default. */
int fyzz_b200_set_contact_notifications(fyzz_b200_world* w, int enabled);
/* Events of the last completed step, in the reference's order (touching
 * contact managers in shape-pair order merged with lost touches).  The
 * first call after a step copies them from the device; the returned arrays
 * are owned by the world and valid until the next step.  Empty while
 * notifications are off or after a step that failed. */
int fyzz_b200_contact_events(fyzz_b200_world* w, const fyzz_b200_contact_event_t** events,
                             uint64_t* n_events, const fyzz_b200_contact_event_point_t** points,
                             uint64_t* n_points);

/* ---- force-threshold stream: World::set_body_contact_report_threshold /
 *      World::force_threshold_changes (world.h:150-173, 472, 493;
 *      Scene::update_threshold_stream, scene.cpp:9391-9508) ----
 * Body pairs whose summed final normal impulse in a step is strictly above
 * threshold * dt.  A pair against the static world is keyed (dynamic body,
 * world) with that body's threshold; any other pair (actor0 < actor1, a
 * kinematic body keeping its own id) with the smaller of the two
 * thresholds.  Only managers the step solved count (a dynamic body awake).
 * Changes against the previous step, in key order: Found (this step's
 * impulse and threshold), Persists (the previous step's impulse and
 * threshold, as the reference reports them), Lost (zero impulse, the
 * previous threshold). */
typedef struct {
    uint32_t actor0, actor1;   /* ForceThresholdKey; actor1 is 0 against the world */
    uint32_t static_world;     /* 1: actor1 is the static world */
    uint32_t change;           /* ForceThresholdChange: 0 Found, 1 Persists, 2 Lost */
    double normal_impulse;
    float threshold;
    uint32_t reserved;
} fyzz_b200_force_threshold_report_t;
/* World::set_body_contact_report_threshold (world.h:493): force >= 0 and
 * finite (FLT_MAX, the default, disables); dynamic or kinematic bodies only
 * (FYZZ_B200_LOGIC_ERROR otherwise). */
int fyzz_b200_set_body_contact_report_threshold(fyzz_b200_world* w, uint32_t body, float force);
/* World::force_threshold_changes (world.h:472): the last completed step's
 * changes; the array is owned by the world and valid until the next step
 * (empty after fyzz_b200_collide or a failed step). */
int fyzz_b200_force_threshold_changes(fyzz_b200_world* w, const fyzz_b200_force_threshold_report_t** reports,
                                      uint64_t* n);

/* ---- kinematic bodies: World::set_body_kinematic / set_body_kinematic_target
 *      (world.h:505-506; Scene::set_kinematic, set_kinematic_target,
 *      scene.cpp:858-1003) ----
 * A kinematic body has infinite mass in contacts and joints and pairs with
 * dynamic bodies only.  Each step it moves to its pending target: contacts
 * see the velocity that carries it there in one step (scene.cpp:2005-2043),
 * and its pose becomes the target after the solve.  Switching a body in or
 * out of kinematic mode rebuilds the device state (the contact-manager
 * history restarts). */
int fyzz_b200_set_body_kinematic(fyzz_b200_world* w, uint32_t body, int enabled);
/* pose: position(3) + orientation xyzw(4), normalised once. */
int fyzz_b200_set_body_kinematic_target(fyzz_b200_world* w, uint32_t body, const float pose[7]);

/* ---- sleeping ----
 * Bodies fall asleep and wake as in the reference scene: the sleep check
 * after integration (scene.cpp:10640-10705), deactivation of touch-graph
 * islands whose bodies are all ready (scene.cpp:6465-6530), waking on new
 * overlaps and touches (scene.cpp:6148-6250) and on authored velocities
 * (World::set_body_velocity / set_body_angular_velocity, world.h:459-460).
 * A sleeping body keeps its pose, reports zero velocity and sleeping = 1 in
 * its body state. */
/* On by default, as in the reference, which has no switch (no counterpart).
 * Turning it off wakes every body; differentiable rollouts always run with
 * it off. */
int fyzz_b200_set_sleeping(fyzz_b200_world* w, int enabled);
/* Per body (n = body count), any pointer may be null: wake counter in
 * seconds, flags (bit 0 asleep, bit 1 ready for sleep), the sleep filter's
 * accumulated linear and body-local angular motion (6 floats) and the
 * counted interactions (overlap pairs plus constraints) of the last step.
 * No reference counterpart (Scene keeps these in its actors). */
int fyzz_b200_read_sleep_state(fyzz_b200_world* w, float* wake, uint32_t* flags, float* motion6,
                               uint32_t* counted, uint32_t n);

/* ---- differentiable rollouts (no counterpart in the reference, which has
 *      no adjoint) ----
 * A rollout of `steps` steps of the current state with a full-state
 * checkpoint every `checkpoint_every` steps; the backward pass re-runs each
 * segment forward from its checkpoint and applies the step adjoints in
 * reverse.  Differentiated model: the step with its discrete structure
 * (pairs, manifolds, partitions, clamp and branch decisions) frozen from
 * the forward run and contact points moving rigidly with their bodies.
 * Gradients are with respect to the initial linear / angular velocities,
 * the body masses (inverse inertia scaling as the inverse mass) and the
 * shapes' static / dynamic friction coefficients.  Step the scene once
 * before rollout_begin so the pair budget is settled. */
int fyzz_b200_rollout_begin(fyzz_b200_world* w, uint32_t steps, uint32_t checkpoint_every);
/* Restores the state the last rollout_forward started from (no reference
 * counterpart), so the rollout can be run again, e.g. with new initial
 * velocities; a rollout_begin with the same steps and interval then reuses
 * its checkpoints, frames and captured graphs. */
int fyzz_b200_rollout_rewind(fyzz_b200_world* w);
/* Re-sizes the pair budget (initially 8 per shape) to the live pairs times
 * headroom (>= 1), keeping the contact-manager history so the trajectory is
 * unchanged; rollouts size their checkpoints and frames by this budget.
 * A later step that needs more pairs grows it again (and a rollout that
 * sees it grow fails with FYZZ_B200_LOGIC_ERROR). */
int fyzz_b200_fit_pair_budget(fyzz_b200_world* w, float headroom, uint32_t* budget_out);
/* Sets the pair budget to `pairs` (raised to the live pairs of both
 * contact-manager generations), keeping the history like
 * fyzz_b200_fit_pair_budget; for callers that size device memory up front.
 * A step that finds more overlap pairs than the budget is rolled back (the
 * contact-manager history included), the budget doubles and the step runs
 * again, with the same result as a step that had room.  No reference
 * counterpart (the reference's GPU owner has a fixed 32,768-pair capacity,
 * native_gpu_world.cpp). */
int fyzz_b200_set_pair_budget(fyzz_b200_world* w, uint32_t pairs, uint32_t* budget_out);
int fyzz_b200_rollout_forward(fyzz_b200_world* w, float seconds);
/* Loss gradients with respect to the final mass-frame centres (3 per body),
 * orientations (4 per body, may be NULL), linear and angular velocities
 * (3 per body; NULL = zero).  Outputs (NULL to skip): per body grad_v0,
 * grad_w0 (3 floats), grad_mass (1); per shape the two friction gradients.
 * Leaves the world at the end of the rollout. */
int fyzz_b200_rollout_backward(fyzz_b200_world* w, const float* grad_center,
                               const float* grad_orientation, const float* grad_velocity,
                               const float* grad_angular, float* grad_v0, float* grad_w0,
                               float* grad_mass, float* grad_static_friction,
                               float* grad_dynamic_friction);
/* Mass-frame centres (3 per body) and orientations (4 per body) of all
 * bodies (either may be NULL). */
int fyzz_b200_read_mass_frames(fyzz_b200_world* w, float* centers, float* orientations);

/* The Gauss-Seidel order of the next step only, in the reference Scene's
 * terms: the input order of partition_constraints (scene.cpp:7153-7216) --
 * joint constraint ids (matched by slot) in order, then the touching
 * managers' shape pairs (a < b) in order; within each island the
 * partition's greedy levels and the solve follow this order.  Managers and
 * joints not named keep canonical order after the named ones.  The
 * reference builds its order from the insertion history of its island
 * graph; with this hook a caller that knows it (a replay of a reference
 * run) reproduces the reference's sweep.  No reference counterpart. */
int fyzz_b200_set_descriptor_order(fyzz_b200_world* w, const uint32_t* pairs, uint64_t n_pairs,
                                   const uint64_t* joint_ids, uint64_t n_joint_ids);
/* Test hook of the step's exclusive scan (no reference counterpart): scans
 * n ones with this world's scan scratch.  skip_first_tile starts the scan's
 * tile ticket at 1, so one block waits for a tile that never publishes; the
 * wait is bounded (2^18 polls), then the scan sets the logic error bit and
 * this call returns FYZZ_B200_LOGIC_ERROR.  error_bits receives the device
 * error bits, mismatches the outputs that differ from their index.  Later
 * scans and steps run normally. */
int fyzz_b200_test_scan(fyzz_b200_world* w, uint32_t n, int skip_first_tile, uint32_t* error_bits,
                        uint64_t* mismatches);

/* ---- broadphase / narrowphase views (Scene::pairs, found_pairs,
 *      lost_pairs, contacts: scene.h:827-833) ---- */
/* which: 0 current pairs, 1 found, 2 lost; 2 u32 (shape a < shape b) each.
 * Returns the count; writes at most cap pairs. */
uint64_t fyzz_b200_read_pairs(fyzz_b200_world* w, int which, uint32_t* out, uint64_t cap);
/* Touching managers in pair order: pair(2), count, and 4 points of
 * position(3) normal(3) separation(1). */
uint64_t fyzz_b200_read_manifolds(fyzz_b200_world* w, uint32_t* pairs, uint32_t* counts,
                                  float* points, uint64_t cap);
/* Encoded AABBs (Shape::encoded_bounds, scene.h:1194): 6 u32 per shape. */
int fyzz_b200_read_encoded_bounds(fyzz_b200_world* w, uint32_t* out, uint32_t n_shapes);
/* Sorted min-x endpoints of one scene (value, shape id), i.e. the minimum
 * endpoints of the reference's axis-0 endpoint order (scene.cpp:1341-1345). */
uint64_t fyzz_b200_read_sorted_min_x(fyzz_b200_world* w, uint32_t scene, uint32_t* values,
                                     uint32_t* ids, uint64_t cap);
/* Friction patch of every touching manager of the last step (pair order):
 * anchor count (bits 0-7; bit 10 + k: anchor k was taken from this step's
 * contact point with index in bits 12 + 2k .. 13 + 2k) and the anchors in
 * the shape0 / shape1 bodies' mass frames (2 x 3 floats each).  Returns the
 * manager count; writes at most cap. */
uint64_t fyzz_b200_read_friction_anchors(fyzz_b200_world* w, uint32_t* anchors, float* anchors0,
                                         float* anchors1, uint64_t cap);
/* Partition level of every descriptor of the last step, in canonical
 * descriptor order (joints then touching managers). */
uint64_t fyzz_b200_read_levels(fyzz_b200_world* w, uint32_t* levels, uint64_t cap);
/* Awake islands of the last step (the solver's units of work): per island
 * its descriptor count and partition level count.  Returns the island
 * count; writes at most cap.  No reference counterpart. */
uint64_t fyzz_b200_read_islands(fyzz_b200_world* w, uint32_t* descriptors, uint32_t* levels, uint64_t cap);
/* Device counters of the last step, n <= 18: 0 touching managers,
 * 1 descriptors, 5 box pairs finished by GJK/EPA, 8-11 islands per size
 * class ((32,512], (96,512], (512,4096], >4096 descriptors), 16 pairs with
 * a cooked hull, 17 of those regenerated through GJK/EPA. */
int fyzz_b200_read_step_counters(fyzz_b200_world* w, uint32_t* out, uint32_t n);

/* ---- allocation-free sweep-and-prune (no counterpart in the reference) ----
 * The overlap-pair set of one scene's finite shapes, computed on the device
 * without allocating any memory: for callers that cannot allocate where they
 * need a pair set (a frame loop sharing the GPU that must not take the
 * device-wide synchronisation of cudaMalloc / cudaFree, or a process held to
 * a device memory budget fixed up front).  The working set lives in one
 * fixed device array of this library (256 KiB), so:
 *  - n_shapes is at most FYZZ_B200_STATIC_SAP_MAX_SHAPES; larger inputs
 *    return FYZZ_B200_INVALID_ARGUMENT and launch nothing;
 *  - all calls on a device share that array: calls whose work may overlap
 *    in time (other streams, other threads) race; order them on one stream;
 *  - the first call on a device (with that device current) resolves the
 *    array's address and the kernel's shared-memory limit; make it before
 *    any stream capture on that device (after a cudaDeviceReset the next
 *    call resolves them again in the new context).
 * Inputs (device pointers): bounds_dev n_shapes x 6 encoded values (min x,
 * y, z, max x, y, z: the layout of fyzz_b200_read_encoded_bounds), body_dev
 * n_shapes values of body id | (1 << 31 if the body is dynamic).  Pairs
 * follow the reference's full sweep (scene.cpp:2635-2704: 3-axis overlap,
 * different bodies, at least one dynamic), are written as (a, b) with a < b
 * in ascending order to pairs_dev (at most pair_cap pairs), and their total
 * to *count_dev.  When the total exceeds pair_cap, only whole owner buckets
 * (all pairs of one lower shape id) that end within pair_cap are written:
 * the written pairs are a prefix of the full list and the rest of pairs_dev
 * is left as it was; call again with pair_cap >= *count_dev for all pairs.
 * Enqueued on stream (a cudaStream_t, NULL = legacy default stream); the
 * results are ready when that stream reaches this point.  message (may be
 * NULL) receives the reason for a non-zero status. */
#define FYZZ_B200_STATIC_SAP_MAX_SHAPES 8192u
int fyzz_b200_sap_pairs_static_scratch(const uint32_t* bounds_dev, const uint32_t* body_dev,
                                       uint32_t n_shapes, uint32_t* pairs_dev, uint32_t pair_cap,
                                       uint32_t* count_dev, void* stream, char* message,
                                       size_t message_len);

#ifdef __cplusplus
}
#endif
#endif
