// Device-resident state of a batched rigid-body world and the host entry
// points that enqueue the step's kernels on a stream.
//
// Layout (HBM, structure of arrays, 16-byte records for 128-bit loads):
//   bodies   b_*  one record per actor of every scene (floors included)
//   shapes   s_*  one record per attached shape
//   pairs    two ping-pong generations of sorted broadphase pair keys and
//            the persistent contact-manager records keyed by them
//   solver   per-step rows, island/level ordering and body deltas
// Scenes are contiguous ranges of bodies and shapes; every shape of a scene
// has a larger global index than every shape of the previous scene, so the
// global (shape a, shape b) order equals the per-scene canonical pair order.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include "common.cuh"

namespace fyzz::b200 {

struct ManagerSet {
    uint64_t* key = nullptr;       // sorted pair keys (a << 32 | b)
    PcmCache* cache = nullptr;
    FrictionHist* fric = nullptr;
    uint32_t* count = nullptr;     // published contact count (touch state)
    uint32_t* n = nullptr;         // device-side pair count of this generation
};

// Pairs whose accumulated normal impulse exceeded their report threshold in
// one step (the force-threshold stream's generation): sorted by key
// (actor0 << 33 | static world << 32 | actor1), with the aggregated impulse
// and the pair's threshold.
struct ThresholdSet {
    uint64_t* key = nullptr;
    double* impulse = nullptr;
    float* thr = nullptr;
    uint32_t* n = nullptr;
};

struct DevState {
    // static topology sizes (host-known)
    uint32_t n_scenes = 0, n_bodies = 0, n_shapes = 0, n_finite = 0, n_joints = 0;
    uint32_t pair_cap = 0, desc_cap = 0;
    uint32_t max_small_scene = 2048;   // finite shapes sorted inside one CTA
    // Performance parameters (fyzz_b200_tuning_t; every choice gives the same
    // results): islands of at most isl_thread descriptors are solved by one
    // thread, up to isl_warp by one warp, up to isl_mid by a 128-thread CTA,
    // up to kBigIsland by the 384-thread CTA; radix sorts take digits of
    // radix_bits; elementwise kernels run elem_block threads a block.
    uint32_t isl_thread = 8, isl_warp = 96, isl_mid = 512;
    int radix_bits = 8;
    uint32_t elem_block = 256;
    // Island scheduling of the warp and CTA solvers: false = static (worker
    // w takes list entries w, w + W, ...), true = a work queue (each worker
    // takes the next entry from a per-step device counter).
    bool work_queue = false;
    int pos_iters = 4, vel_iters = 1;
    float dt = 1.0f / 120.0f;
    uint32_t frame = 0;

    // scenes
    uint32_t* sc_fbegin = nullptr;     // S+1, finite-shape ranges (finite-rank space)
    int32_t* sc_plane = nullptr;       // plane shape of each scene or -1
    uint32_t* small_scenes = nullptr;  // scenes sorted inside one CTA
    uint32_t n_small = 0;

    // bodies
    float4 *b_p = nullptr, *b_q = nullptr, *b_v = nullptr, *b_w = nullptr;
    float4 *b_inv = nullptr;           // inverse inertia xyz, w = inverse mass
    float4 *b_ml_p = nullptr, *b_ml_q = nullptr;
    float4 *b_dyn0 = nullptr;          // linear damping, angular damping, max linear, max angular
    float4 *b_dyn1 = nullptr;          // max depenetration, max contact impulse, slop, unused
    uint32_t* b_flags = nullptr;
    uint32_t* b_scene = nullptr;
    // sleep (Dy sleepCheck and the accurate island's deactivation)
    float* b_wake = nullptr;           // wake counter, seconds
    float4* b_sacc = nullptr;          // 2 per body: accumulated linear, local angular motion
    uint32_t* b_sleep = nullptr;       // kSleeping | kReady
    uint32_t* b_jcount = nullptr;      // distance constraints attached (counted interactions)
    uint32_t* b_counted = nullptr;     // per step: overlap pairs + constraints
    uint32_t* sl_act = nullptr;        // per step: activating this step
    uint32_t* sl_spec = nullptr;       // per step: overlap-graph union-find parent (over touch-graph roots)
    uint32_t* sl_root = nullptr;       // per step: flags of the union-find roots
    float4* b_ktarget = nullptr;       // 2 per body: kinematic target position, orientation
    uint32_t n_kinematic = 0;          // kinematic bodies in the world
    bool sleep = true;                 // sleeping enabled for this step

    // shapes
    uint32_t *s_body = nullptr, *s_type = nullptr, *s_scene = nullptr;
    float4 *s_geom = nullptr;          // half extents xyz, radius
    uint32_t* s_mesh = nullptr;        // cooked hull index, ~0u for other shapes
    // cooked hulls: per mesh its vertex and face ranges and the half size of
    // its vertex bounds (w: half the smallest bound extent); the arenas hold
    // every mesh's vertices, face planes (normal, distance), face boundary
    // loops (first index into hidx, count) and the loop indices (local to
    // the mesh's vertex range)
    uint4* m_tab = nullptr;            // vertex offset, vertex count, face offset, face count
    float4* m_half = nullptr;
    float4* hv = nullptr;
    float4* hf = nullptr;
    uint2* hfr = nullptr;
    uint32_t* hidx = nullptr;
    uint32_t n_meshes = 0;
    float4 *s_lp = nullptr;            // local position, w = contact offset
    float4 *s_lq = nullptr;
    float4 *s_mat = nullptr;           // static f, dynamic f, restitution, rest offset
    float4 *s_wp = nullptr, *s_wq = nullptr;
    uint4 *s_lo = nullptr, *s_hi = nullptr;   // encoded bounds (x,y,z,-)
    int32_t* s_frank = nullptr;        // finite rank, -1 for planes
    int32_t* s_dynrank = nullptr;      // rank among the scene's dynamic finite shapes
    uint32_t* s_static_pairs = nullptr;// plane pairs owned by this shape

    // broadphase scratch
    uint32_t *srt_key = nullptr, *srt_id = nullptr;      // sorted min-x endpoints
    uint32_t *srt_key2 = nullptr, *srt_id2 = nullptr;
    uint32_t *own_cnt = nullptr, *own_off = nullptr, *own_cur = nullptr;
    uint2* prev_bkt = nullptr;         // per shape: its bucket in the previous generation's keys
    ManagerSet cur, prev;
    int32_t* prev_idx = nullptr;
    uint32_t* found_flag = nullptr;    // per current pair
    uint32_t* lost_flag = nullptr;     // per previous pair
    ContactPt* pts = nullptr;          // 4 per current pair
    uint32_t* gjk_list = nullptr;      // pairs awaiting the GJK/EPA continuation
    uint32_t* cvx_list = nullptr;      // pairs with a cooked hull (plane or finite partner)
    uint32_t* cvx_gjk_list = nullptr;  // hull pairs whose manifold regenerates (GJK/EPA)
    uint32_t* cvx_clip_list = nullptr; // regenerated hull pairs with a witness to clip faces around
    float4* cvx_wit = nullptr;         // their witnesses: local a, local b, normal, separation (3 per entry)
    uint32_t* cvx_epa_list = nullptr;  // regenerated hull pairs whose GJK ended in EPA
    float4* cvx_simplex = nullptr;     // their GJK simplices (4 supports x 3 float4; count in [11].w)

    // touching managers
    uint32_t* man_list = nullptr;      // current-pair indices, canonical order
    uint32_t* n_man = nullptr;
    ManagerHeader* mh = nullptr;       // per touching manager
    NormalRow* nrow = nullptr;         // 4 per touching manager
    FrictionRow* frow = nullptr;       // 4 per touching manager
    // The island solvers' copy of the rows in placed-descriptor order (slot
    // i = position in d_val2): kSlotVecPlanes float4 planes then
    // kSlotScalarPlanes float planes of desc_cap records.
    float4* slot_rows = nullptr;

    // joints (static, sorted by scene then constraint slot descending)
    uint32_t *j_a = nullptr, *j_b = nullptr;  // descriptor bodies (distance: ordered pair; others: authored)
    uint32_t* j_kind = nullptr;         // kJoint*
    uint32_t* j_row = nullptr;          // first row in jrow (rows in joint order)
    float4 *j_la = nullptr, *j_lb = nullptr;   // local anchor positions
    float4 *j_qa = nullptr, *j_qb = nullptr;   // local frame orientations (fixed .. prismatic)
    float* j_len = nullptr;
    JointRow* jrow = nullptr;           // n_jrows rows
    uint32_t n_jrows = 0;

    // solver bodies
    float4 *sb_dv = nullptr, *sb_dw = nullptr, *sb_mdv = nullptr, *sb_mdw = nullptr;
    float4 *sb_v = nullptr, *sb_w = nullptr;
    float4 *sb_sqrt_i = nullptr;       // 3 per body: columns of R sqrt(I^-1) R^T
    uint32_t* uf_parent = nullptr;

    // descriptors: [0, n_joints) joints, then touching managers
    uint32_t *d_key = nullptr, *d_val = nullptr, *d_key2 = nullptr, *d_val2 = nullptr;
    uint32_t* d_level = nullptr;
    uint32_t *isl_begin = nullptr, *isl_end = nullptr, *n_isl = nullptr;
    uint32_t* sb_mask = nullptr;       // partition masks per body
    uint32_t* sb_maxdyn = nullptr;
    uint32_t* sb_static = nullptr;
    uint32_t* sb_earliest = nullptr;   // per-body earliest undecided descriptor (partition rounds)
    int2* d_bod = nullptr;             // per descriptor: dynamic solver bodies (-1 = static world)
    // Island-local body slots (islands up to kBigIsland descriptors): the
    // island's dynamic bodies are numbered 0..n-1 so PGS can keep their
    // velocity deltas in shared memory.
    uint32_t* d_lbod = nullptr;        // per placed descriptor: local a | local b << 16 (0xffff static)
    int32_t* isl_bod = nullptr;        // island isl's bodies at [isl_begin + isl, + isl_nbod)
    uint32_t* isl_nbod = nullptr;      // per island
    // Islands by size class (descriptors), listed each step by
    // k_island_classes: 0 (32, 512] shared-memory partition, 1 (isl_warp,
    // isl_mid] 128-thread CTA solver, 2 (512, 4096] shared-memory partition,
    // 3 beyond 4096 global-memory paths, 4 (isl_mid, 4096] 384-thread CTA
    // solver, 5 (isl_thread, isl_warp] warp solver.
    static constexpr int kIslLists = 6;
    uint32_t* isl_list[kIslLists] = {};

    // step scratch
    uint4* sw_rec = nullptr;           // sweep y/z bounds in sorted order
    uint2* sw_meta = nullptr;          // sweep max x and body | dynamic bit
    // Partners found by the counting sweep (kSweepCache per sorted shape) and
    // how many each shape found; the filling sweep reuses them instead of
    // scanning the candidates again (it rescans only shapes that overflowed).
    uint32_t* sw_cache = nullptr;
    uint32_t* sw_found = nullptr;
    static constexpr uint32_t kSweepCache = 16;
    uint32_t* tmp_flags = nullptr;     // pair_cap
    uint32_t* tmp_pos = nullptr;       // max(pair_cap, desc_cap)
    uint32_t* lvl_bound = nullptr;     // 2 * desc_cap + 2: per-island partition starts
    // scenes too large for one CTA: sorted with the device-wide radix sort
    static constexpr int kMaxLarge = 64;
    uint32_t n_large = 0;
    uint32_t large_begin[kMaxLarge] = {}, large_n[kMaxLarge] = {};
    // Large scenes are swept in bands of z (every shape in each band its z
    // extent touches, a pair kept in the one band holding the larger of the
    // two min z).  The sweep list is the x-sorted list of every finite shape
    // (large scenes' entries only publish their plane pairs) followed by the
    // large scenes' band entries, sorted by (scene, band) and x within.
    static constexpr uint32_t kBands = 256, kBandStatBlocks = 148;
    int32_t* sc_large = nullptr;       // per scene: large-scene index or -1
    uint4* bd_part = nullptr;          // kMaxLarge x kBandStatBlocks: min z, max z (encoded), max z extent bits
    float4* bd_par = nullptr;          // per large scene: z origin, 1 / band width
    uint32_t* bd_cnt = nullptr;        // per x-sorted finite shape: bands spanned (0 in small scenes)
    uint32_t* bd_off = nullptr;
    uint32_t* bd_n = nullptr;          // band entries this step
    uint32_t* bd_end = nullptr;        // kMaxLarge x kBands: end of each band's entries (entry index)
    uint32_t *bx_key = nullptr, *bx_val = nullptr, *bx_key2 = nullptr, *bx_val2 = nullptr;
    uint32_t* bx_seg = nullptr;        // per band entry: end of its band in the sweep list
    uint32_t bx_cap = 0;               // band entries at most (2 per large-scene shape)

    // scratch for scans / sorts
    uint32_t* scan_tmp = nullptr;
    size_t scan_tmp_words = 0;
    uint32_t* sort_os = nullptr;       // one-sweep radix passes (onesweep_words)
    size_t sort_os_words = 0;
    uint32_t* sort_hist = nullptr;
    size_t sort_hist_words = 0;
    // Impulse tape of a differentiated step (null otherwise): the applied
    // impulse of every row after each PGS pass, [pass][manager][4] for the
    // normal and friction rows and [pass][joint] for the joints.
    float* tape_n = nullptr;
    float* tape_f = nullptr;
    float* tape_j = nullptr;

    // contact events (allocated while notifications are enabled)
    bool events = false;
    void* ev = nullptr;                // EventRecord, 2 per pair
    void* ev_pts = nullptr;            // EventPoint, 4 per pair
    uint64_t* ev_lost_key = nullptr;   // lost touches, pair order
    uint32_t* ev_cnt = nullptr;        // contact count per touching manager
    uint32_t* ev_pt_off = nullptr;     // first event point per touching manager
    uint32_t* counters = nullptr;      // small device counters
    uint32_t* err = nullptr;           // error bits

    // force-threshold stream (arrays exist once some body has a report
    // threshold; World::set_body_contact_report_threshold)
    bool thresholds = false;
    float* b_thresh = nullptr;         // per body; FLT_MAX disables reporting
    ThresholdSet th_cur, th_prev;      // this step's exceeded pairs / the previous step's
    uint32_t *th_hi = nullptr, *th_lo = nullptr;   // per touching manager: key halves
    double* th_sum = nullptr;          // per touching manager: summed normal impulse
    float* th_thr = nullptr;           // per touching manager: pair threshold
    uint32_t *th_k = nullptr, *th_v = nullptr, *th_k2 = nullptr, *th_v2 = nullptr;   // sort keys / rows
    double* th_run_sum = nullptr;      // per sorted row (run heads): aggregated impulse
    float* th_run_thr = nullptr;
    uint32_t *th_f0 = nullptr, *th_p0 = nullptr, *th_f1 = nullptr, *th_p1 = nullptr;   // flags / scans
    void* th_changes = nullptr;        // ForceThresholdRecord, 2 * pair_cap

    // Replayed descriptor order of one step (fyzz_b200_set_descriptor_order):
    // the touching managers' pair keys, sorted, with their positions in the
    // order, and each joint descriptor's rank.  Off (replay = false) in
    // ordinary steps.
    bool replay = false;
    uint64_t* rp_keys = nullptr;
    uint32_t* rp_pos = nullptr;
    uint32_t rp_n = 0;
    uint32_t* rp_jrank = nullptr;
};

// primitives.cu
void scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t n, const uint32_t* n_dev,
                    uint32_t* total, uint32_t* tmp, size_t tmp_words, cudaStream_t st, uint32_t* err = nullptr);
void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt,
                      uint32_t n_cap, const uint32_t* n_dev, int begin_bit, int end_bit,
                      uint32_t* hist, size_t hist_words, uint32_t* scan_tmp, size_t scan_words,
                      cudaStream_t st, uint32_t* err = nullptr, int digit_bits = 8,
                      uint32_t* os_scratch = nullptr, size_t os_words = 0);
constexpr int kRadixMaxBits = 11;   // widest radix digit
size_t radix_hist_words(uint32_t n_cap);
// One-sweep scratch of radix_sort_pairs (8-bit digits); zero when allocated.
size_t onesweep_words(uint32_t n_cap);
void init_primitive_kernels();
size_t scan_tmp_words_for(uint32_t n_cap);

// Stage boundaries of one step, reported to an optional hook (the world uses
// it to bracket stages with CUDA events when profiling).
enum Stage : int {
    kStBounds = 0, kStSort, kStPairs, kStNarrow, kStIslands, kStPrep, kStPgs, kStIntegrate, kStEnd
};
struct StageHook {
    void (*fn)(void* ctx, int stage, cudaStream_t st) = nullptr;
    void* ctx = nullptr;
    void operator()(int stage, cudaStream_t st) const { if (fn) fn(ctx, stage, st); }
};

// Side streams for independent branches of a step.  They fork from and join
// back into the main stream through events, so inside a stream capture they
// become parallel branches of the step's graph.
struct Branches {
    static constexpr int kN = 3;
    cudaStream_t st[kN] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[kN] = {};
};

// Reverse-mode state of a differentiated rollout (adjoint.cu).  Per body,
// the adjoint of the mass-frame state (centre c, orientation Q) and the
// velocities: on entry to a step's reverse pass it refers to the end of
// the step, on exit to its start.  The rest is per-step scratch and the
// parameter gradients accumulated over the rollout.
struct AdjState {
    float4 *c = nullptr, *q = nullptr, *v = nullptr, *w = nullptr;
    float4 *x_c = nullptr, *x_q = nullptr;        // the step's start state (mass frame)
    float4 *dvm = nullptr, *dwm = nullptr;        // adjoints of the position-pass deltas
    float4 *dv = nullptr, *dw = nullptr;          // adjoints of the final deltas (reverse sweep)
    float4 *rdv = nullptr, *rdw = nullptr;        // deltas rebuilt during the reverse sweep
    float4 *v1 = nullptr, *w1 = nullptr;          // adjoints of the pre-integrated velocities
    float4 *C = nullptr;                          // 3 rows per body: sqrt inverse inertia tensor
    float *im = nullptr;                          // inverse mass (this step)
    float *g_im = nullptr;                        // inverse mass, whole rollout
    float4 *iI = nullptr, *g_iI = nullptr;        // inverse principal inertia (step, rollout)
    float *g_fs = nullptr, *g_fd = nullptr;       // per shape: static / dynamic friction
    NormalRow* nrow = nullptr;                    // row adjoints
    FrictionRow* frow = nullptr;
    JointRow* jrow = nullptr;
    float4* hd = nullptr;                         // per manager: ima, imb, sf, df
    float *yn = nullptr, *yf = nullptr, *yj = nullptr;   // applied-impulse adjoints
    uint32_t* mark = nullptr;                     // per body: last step it was visited
    uint32_t* epoch = nullptr;                    // step counter of the reverse pass
};
// Copies the live pairs of a contact-manager generation.
void enqueue_copy_set(const ManagerSet& dst, const ManagerSet& src, uint32_t cap, cudaStream_t st);
// adjoint.cu
void enqueue_adjoint_save_start(const DevState& s, const AdjState& a, cudaStream_t st);
void enqueue_adjoint_step(const DevState& s, const AdjState& a, cudaStream_t st);

// broadphase.cu / narrowphase.cu / solver.cu
void enqueue_broadphase(const DevState& s, cudaStream_t st, const StageHook& hook = {});
void enqueue_narrowphase(const DevState& s, cudaStream_t st, const StageHook& hook = {});
void enqueue_solver(const DevState& s, cudaStream_t st, const StageHook& hook = {},
                    const Branches* br = nullptr);
// events.cu: the step's contact events into s.ev / s.ev_pts (after PGS).
void enqueue_events(const DevState& s, cudaStream_t st);
// thresholds.cu: the step's force-threshold changes into s.th_changes
// (after PGS; s.th_cur becomes this step's exceeded set).
void enqueue_thresholds(const DevState& s, cudaStream_t st);
// Copies the live records of a threshold generation (n from the device).
void enqueue_copy_threshold_set(const ThresholdSet& dst, const ThresholdSet& src, uint32_t cap, cudaStream_t st);
// Per-device kernel attributes (shared-memory limits); call with the device
// current before the first step or capture.
// Wakes every dynamic body (as an authored velocity on each would).
void enqueue_wake_bodies(const DevState& s, cudaStream_t st);
// 14-float body records (position, velocity, orientation, angular
// velocity, sleeping) into out (device memory).
void enqueue_pack_bodies(const DevState& s, float* out, cudaStream_t st);
// 6-float velocity records (device memory) into the bodies; wakes them.
void enqueue_unpack_velocities(const DevState& s, const float* rec, uint32_t stride, uint32_t lin, uint32_t ang,
                               cudaStream_t st);
void init_solver_kernels();
// Island size classes (descriptors per island).
constexpr uint32_t kSmallIsland = 96;     // one warp
constexpr uint32_t kMidIsland = 512;      // one CTA, shared-memory deltas
constexpr uint32_t kBigIsland = 4096;     // one CTA, shared-memory deltas (1 CTA / SM)
// Planes of DevState::slot_rows, desc_cap records each: 25 of float4, then
// 16 of float (the layout is described where the solver stages them).
constexpr uint32_t kSlotVecPlanes = 25, kSlotScalarPlanes = 16;
// counters[] slots
enum : int { kCntMan = 0, kCntDesc = 1, kCntIsl = 2, kCntFrame = 3, kCntLevels = 4, kCntGjk = 5,
             kCntAwake = 6 /* descriptors of awake islands */, kCntSleeping = 7 /* asleep at step start */,
             kCntList = 8 /* 4 island-class list lengths */, kCntLost = 12, kCntEvPts = 13,
             kCntReported = 14 /* touching managers with an event */,
             kCntReady = 15 /* ready for sleep at step start */,
             kCntConvex = 16 /* pairs with a cooked hull */,
             kCntConvexGjk = 17 /* hull pairs regenerated through GJK/EPA */,
             kCntActivating = 18 /* nonzero when some body activates this step */,
             kCntConvexClip = 19 /* regenerated hull pairs whose faces are clipped */,
             kCntConvexEpa = 20 /* regenerated hull pairs continuing in EPA */,
             kCntThRows = 21 /* managers with a reportable impulse */,
             kCntThChanges = 22 /* force-threshold changes of the step */,
             kCntThCommon = 23 /* pairs exceeding in this step and the previous one */,
             kCntList4 = 24 /* length of island list 4 */, kCntList5 = 25 /* length of island list 5 */,
             kCntQueue = 26 /* 3 work-queue tickets: warp, mid CTA, big CTA solvers */, kCntSlots = 29 };
// Counter slot of island list c.
__host__ __device__ constexpr int list_counter(int c) { return c < 4 ? kCntList + c : kCntList4 + (c - 4); }
// Each list holds islands of more than this many descriptors (its capacity
// is descriptors / (bound + 1) + 2).
constexpr uint32_t kListMinDesc[6] = {32, 32, 512, 4096, 128, 0};

// Contact event records in device memory; the layouts of
// fyzz_b200_contact_event_t and fyzz_b200_contact_event_point_t.
struct EventRecord {
    uint32_t body0, body1, shape0, shape1, kind, count;
    uint64_t point_offset;
    double normal_impulse;
};
static_assert(sizeof(EventRecord) == 40, "EventRecord layout");
struct EventPoint {
    float position[3], normal[3], separation;
    uint32_t pad;
    double normal_impulse;
};
static_assert(sizeof(EventPoint) == 40, "EventPoint layout");
// fyzz_b200_force_threshold_report_t.
struct ForceThresholdRecord {
    uint32_t actor0, actor1, static_world, change;
    double normal_impulse;
    float threshold;
    uint32_t pad;
};
static_assert(sizeof(ForceThresholdRecord) == 32, "ForceThresholdRecord layout");

}  // namespace fyzz::b200
