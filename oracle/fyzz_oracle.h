/* Test infrastructure: C restatement of the reference's rigid-body step
 * (NativeCpu scene, src/native/scene.cpp) used as the parity oracle for the
 * B200 kernels.  Only tests, smoke() and bench.py's CPU-baseline leg use
 * it; the product never links or loads it.
 *
 * Parity is pinned against oracle/_ref (the reference compiled from its own
 * sources): tests/test_oracle_pin.py runs both on the same seeded scenes.
 */
#ifndef FYZZ_ORACLE_H
#define FYZZ_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { FO_BOX = 0, FO_SPHERE = 1, FO_PLANE = 2, FO_CONVEX = 3 };
enum { FO_OK = 0, FO_INVALID = 1, FO_LOGIC = 2, FO_OVERFLOW = 3 };
/* Joint kinds (scene.h:1528 JointKind, plus the two distance authorings). */
enum { FO_JOINT_CENTER = 0, FO_JOINT_ANCHORED = 1, FO_JOINT_FIXED = 2, FO_JOINT_SPHERICAL = 3,
       FO_JOINT_REVOLUTE = 4, FO_JOINT_PRISMATIC = 5 };
#define FO_OVERFLOW_NEG (-3)
#define FO_LOGIC_NEG (-2)

/* PcmContactCandidate / PcmPersistentContact (scene.h:584-587, 1444-1447) */
typedef struct { float la[3], lb[3], nb[3], sep; } fo_candidate;
/* ContactPoint (scene.h:510-514) */
typedef struct { float p[3], n[3], sep; } fo_point;
/* PcmManifoldCache (scene.h:1448-1459) without the write-only GJK warmstart */
typedef struct {
    fo_candidate pts[4];
    float rel_p[3], rel_q[4], qa[4], qb[4];
    uint8_t count, initialized, pad[2];
} fo_pcm_cache;

/* Cooked convex mesh (include/fyzzxyzzy/convex.h:19-53): planar faces
 * (outward normal, plane distance, boundary loop in idx[first, first+count)),
 * density-one volume, centre of mass and inertia columns about it. */
typedef struct { float n[3], d; uint32_t first, count; } fo_face;
typedef struct {
    uint32_t nv, nf, ni;
    float* verts;
    fo_face* faces;
    uint32_t* idx;
    double volume;
    float center[3], inertia[9], lo[3], hi[3];
} fo_mesh;
int fo_cook_convex(const float* verts, uint32_t nv, const uint32_t* tris, uint32_t nt, fo_mesh* out);
void fo_mesh_free(fo_mesh* m);
/* PcmFiniteShape (scene.h:589-599): half extents, pose, sphere radius and
 * an optional cooked hull in the shape's own frame. */
typedef struct { float half[3], p[3], q[4], radius; const fo_mesh* hull; } fo_finite;
int fo_pcm_convex_gjk_epa(const fo_finite* a, const fo_finite* b, float cd, fo_candidate* out);
int fo_pcm_convex_face_contacts(const fo_finite* a, const fo_finite* b, float cd,
                                const fo_candidate* witness, fo_candidate out[4]);
/* Scene::generate_pcm_convex_pair (scene.cpp:3655-3772).  shape_half is the
 * attached shape's half extents (zero for spheres), used by the rotation
 * travel test. */
int fo_generate_pcm_convex_pair(const fo_finite* first, const float* first_shape_half,
                                const fo_finite* second, const float* second_shape_half, float cd,
                                fo_pcm_cache* cache, fo_point out[4]);
/* Scene::generate_pcm_plane_box with a cooked hull (scene.cpp:3774-3972). */
int fo_generate_pcm_plane_convex(const float* plane_p, const float* shape_half, const float* pose7,
                                 const fo_mesh* hull, float cd, fo_pcm_cache* cache, fo_point out[4]);
/* Scene::update_shape_bounds for a cooked hull (scene.cpp:1258-1298). */
int fo_convex_bounds(const float* pose7, const fo_mesh* hull, float contact_offset, uint32_t* out6);

uint32_t fo_encode_min(float v);
uint32_t fo_encode_max(float v);
int fo_shape_bounds(uint32_t type, const float* pose, const float* geom,
                    float contact_offset, uint32_t* out6);
int fo_pcm_box_box_candidates(const float* a, const float* b, float cd,
                              fo_candidate* out, int cap, int* count);
int fo_pcm_batch_selection(const fo_candidate* c, int n, float tol, uint8_t sel[4]);
int fo_pcm_box_box_gjk_epa(const float* a, const float* b, float cd, fo_candidate* out);
int fo_pcm_sphere_sphere(const float* c0, float r0, const float* c1, float r1,
                         float cd, fo_point* out);
int fo_pcm_sphere_plane(const float* c, float r, float plane_h, float cd, fo_point* out);
int fo_pcm_sphere_box(const float* c, float r, const float* box, float cd, fo_point* out);
int fo_generate_pcm_box_box(const float* first, const float* second, float cd,
                            fo_pcm_cache* cache, fo_point out[4]);
int fo_generate_pcm_plane_box(const float* plane_p, const float* box, float cd,
                              fo_pcm_cache* cache, fo_point out[4]);

/* ---- whole-scene stepping ---- */
typedef struct fo_scene fo_scene;
fo_scene* fo_scene_create(uint32_t nb, const float* bodies, uint32_t ns,
                          const uint32_t* shape_body, const uint32_t* shape_type,
                          const float* shape_geom, const float* shape_local,
                          const float* shape_mat, uint32_t nj,
                          const uint32_t* joint_bodies, const float* joint_dist,
                          int has_floor, float floor_height, const float* floor_mat);
/* As fo_scene_create, with cooked convex shapes: shape_type FO_CONVEX takes
 * its mesh index in shape_geom[0]; mesh m has mesh_nv[m] vertices and
 * mesh_nt[m] triangles, concatenated in mesh order in mesh_verts (3 floats
 * each) and mesh_tris (3 indices each, local to the mesh). */
fo_scene* fo_scene_create_ex(uint32_t nb, const float* bodies, uint32_t ns,
                             const uint32_t* shape_body, const uint32_t* shape_type,
                             const float* shape_geom, const float* shape_local,
                             const float* shape_mat, uint32_t nj,
                             const uint32_t* joint_bodies, const float* joint_dist,
                             int has_floor, float floor_height, const float* floor_mat,
                             uint32_t n_meshes, const uint32_t* mesh_nv, const float* mesh_verts,
                             const uint32_t* mesh_nt, const uint32_t* mesh_tris);
void fo_scene_destroy(fo_scene* s);
const char* fo_error(void);
/* One Scene::step.  manager_order / joint_order (optional) replay the
 * reference's Dy descriptor input order: manager_order lists indices into
 * this step's touching-manifold list, joint_order lists constraint slots.
 * NULL selects the canonical order (joints by constraint slot descending,
 * then touching managers in shape-pair order). */
int fo_scene_step(fo_scene* s, float dt, const uint64_t* manager_order, uint64_t n_mgr,
                  const uint64_t* joint_order, uint64_t n_joint);
/* Scene::advance_collision: bounds, pairs and Gu manifolds only. */
int fo_scene_advance_collision(fo_scene* s);
/* Same counters as the reference harness. */
void fo_scene_counts(const fo_scene* s, uint64_t* out10);
void fo_scene_body_states(const fo_scene* s, float* out14);
void fo_scene_set_body_states(fo_scene* s, const float* in14);
void fo_scene_mass_props(const fo_scene* s, float* out11);
void fo_scene_encoded_bounds(const fo_scene* s, uint32_t* out6);
uint64_t fo_scene_pairs(const fo_scene* s, int which, uint32_t* out2);
uint64_t fo_scene_manifolds(const fo_scene* s, uint32_t* pairs, uint32_t* counts,
                            uint32_t* reversed, float* points28);
uint64_t fo_scene_partitions(const fo_scene* s, uint32_t* desc4, uint64_t* ends);
uint64_t fo_scene_normal_impulses(const fo_scene* s, double* out);
uint64_t fo_scene_sorted_min_x(const fo_scene* s, uint32_t* values, uint32_t* ids);
/* Sets joint j's kind and local frames (position 3 + orientation xyzw 4
 * each; orientations are validated and normalised as World and Scene do;
 * the distance kinds use the positions only).  Call before stepping. */
int fo_scene_set_joint(fo_scene* s, uint32_t j, uint32_t kind, const float* local_a7, const float* local_b7);
/* A joint added after creation (kind, 0-based dynamic bodies or 0xffffffff
 * for the floor, local frames, distance): reuses the most recently retired
 * constraint slot; id = generation << 32 | slot. */
int fo_scene_add_joint(fo_scene* s, uint32_t kind, uint32_t a, uint32_t b, const float* local_a7,
                       const float* local_b7, float distance, uint64_t* id_out);
/* Retires a joint by id (World::remove_constraint). */
int fo_scene_remove_joint(fo_scene* s, uint64_t id);
/* Kinematic mode of an actor (before stepping) and its target pose
 * (position 3 + quaternion xyzw 4). */
int fo_scene_set_kinematic(fo_scene* s, uint32_t actor, int on);
int fo_scene_set_kinematic_target(fo_scene* s, uint32_t actor, const float* pose7);
/* Sleeping on (default) or off (wakes every body). */
void fo_scene_set_sleeping(fo_scene* s, int on);
/* Per actor: wake counter, sleeping, ready, counted interactions, linear
 * and local angular sleep-filter motion (10 floats). */
void fo_scene_sleep_state(const fo_scene* s, float* out10);

#ifdef __cplusplus
}
#endif
#endif
