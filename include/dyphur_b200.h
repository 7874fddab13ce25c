/* dyphur_b200.h — C ABI of the B200-native dyphur frame step.
 *
 * The frame step is integrate -> Morton/LBVH broadphase -> (a, b) pair order
 * -> SAT narrowphase -> XPBD contact solve -> FNV-1a state hash, as the
 * reference drives it in examples/stress_test_blocks/main.cpp:264-279.
 *
 * Conventions
 *   - Every pointer inside a view struct is a DEVICE pointer (cudaMalloc or
 *     torch storage) unless the name says host. Counts that the GPU produces
 *     stay on the device (uint32_t* d_*).
 *   - Every entry point returns dyph_status (0 = OK) and never throws.
 *   - Work is queued on the given stream (a cudaStream_t; NULL = legacy
 *     default stream). Nothing synchronises the host unless its name says
 *     "download".
 *   - The view structs have the field order and meaning of the reference's
 *     kernel views, so a BodyView / ShapeView / ContactView can be passed by
 *     reinterpret_cast.
 */
#ifndef DYPHUR_B200_H
#define DYPHUR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* dyph_stream;

typedef enum dyph_status {
    DYPH_OK = 0,
    DYPH_ERR_INVALID = 1,          /* bad argument (null pointer, size, mode) */
    DYPH_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    DYPH_ERR_PAIR_OVERFLOW = 3,    /* more candidate pairs than capacity (sorted prefix kept) */
    DYPH_ERR_CONTACT_OVERFLOW = 4, /* more contacts than capacity (ordered prefix kept) */
    DYPH_ERR_TIMEOUT = 5,          /* a bounded device-side wait gave up */
    DYPH_ERR_NO_DEVICE = 6,        /* no CUDA device / not an sm_100 device */
    DYPH_ERR_NOMEM = 7,            /* device allocation failed */
    DYPH_ERR_NOT_FINITE = 8,       /* NaN / Inf found in body state */
    DYPH_ERR_TOO_LARGE = 9,        /* size above a fixed-scratch entry point's maximum */
    DYPH_ERR_UNSUPPORTED = 10      /* a path the adjoint does not differentiate (see dyph_world_rollout_backward) */
} dyph_status;

/* Mirrors BodyView (core/include/core/body.hpp:30-46). */
typedef struct dyph_bodies {
    float *pos_x, *pos_y, *pos_z;
    float *rot_w, *rot_x, *rot_y, *rot_z;
    float *vel_x, *vel_y, *vel_z;
    float *ang_x, *ang_y, *ang_z;
    float* inv_mass;
    float *iI_xx, *iI_yy, *iI_zz;
    float *iI_xy, *iI_xz, *iI_yz;
    uint32_t* shape;
    uint32_t* flags;
    uint32_t n;
} dyph_bodies;

/* Mirrors ShapeView (core/include/core/shapes.hpp:22-29). type: 0 box, 1 sphere. */
typedef struct dyph_shapes {
    const uint32_t* type;
    const float* half_x;
    const float* half_y;
    const float* half_z;
    const uint32_t* ext_id;
    uint32_t n;
} dyph_shapes;

/* Mirrors ContactView (core/include/core/contact.hpp:8-20). Normal points from B toward A. */
typedef struct dyph_contacts {
    uint32_t* body_a;
    uint32_t* body_b;
    float *pos_x, *pos_y, *pos_z;
    float *norm_x, *norm_y, *norm_z;
    float* depth;
    uint32_t* n; /* device: live contact count */
    uint32_t capacity;
} dyph_contacts;

/* Mirrors AABB (core/include/core/aabb.hpp:7-9). */
typedef struct dyph_aabb {
    float min_x, min_y, min_z, max_x, max_y, max_z;
} dyph_aabb;

/* Mirrors ContactPair (core/include/core/broadphase.hpp:12-14): a < b. */
typedef struct dyph_pair {
    uint32_t a, b;
} dyph_pair;

/* Mirrors NodeBox (core/include/core/broadphase.hpp:21-25): raw fp16 bits. */
typedef struct dyph_node_box {
    uint16_t mn_x, mn_y, mn_z, mx_x, mx_y, mx_z, pad0, pad1;
} dyph_node_box;

/* Mirrors BvhView (core/include/core/broadphase.hpp:30-38), plus the sorted
 * 64-bit Morton keys (morton30 << 32 | body) the tree was built from. */
typedef struct dyph_bvh_view {
    const int32_t* left;
    const int32_t* right;
    const int32_t* parent;
    const int32_t* root;
    const uint32_t* sorted_idx;
    const dyph_node_box* aabb;
    const uint64_t* sorted_keys;
    uint32_t n;
} dyph_bvh_view;

/* Mirrors IntegratorParams (core/include/core/integrator.hpp:7-11). */
typedef struct dyph_integrator_params {
    float gravity[3];
    float dt;
    int32_t n_substeps;
} dyph_integrator_params;

/* Solver order modes. */
typedef enum dyph_solver_mode {
    /* XpbdSolver default (core/src/xpbd_solver.cpp:620-733): sequential order
     * when n_con <= 256, else Jones–Plassmann colours processed in ascending
     * colour order. Bit-identical to the reference. */
    DYPH_SOLVER_REFERENCE = 0,
    /* XpbdSolver::set_force_serial(true) (core/include/core/xpbd_solver.hpp:48):
     * sorted contact order, run as a dependency schedule on per-body contact
     * lists (one block at <= 2048 contacts), bit-identical to the serial loop. */
    DYPH_SOLVER_SEQUENTIAL = 1,
    /* Jones–Plassmann colours at every contact count (no sequential threshold):
     * the fast mode for batched small scenes; its drift against the
     * sequential order is measured, not zero. */
    DYPH_SOLVER_COLORED = 2,
    /* As DYPH_SOLVER_REFERENCE, with the colouring and sweeps run round by
     * round and colour by colour behind grid barriers (the reference's own
     * schedule) instead of the per-contact dataflow schedule. Same results;
     * the coloured modes use this schedule by themselves when a frame has more
     * than 16 contacts per resident thread. */
    DYPH_SOLVER_REFERENCE_ROUNDS = 3
} dyph_solver_mode;

/* ── library ──────────────────────────────────────────────────────────────── */

const char* dyph_status_string(int status);
/* Text of the CUDA runtime error behind the calling thread's last
 * DYPH_ERR_CUDA ("no error" if there was none). */
const char* dyph_last_cuda_error(void);
/* Returns DYPH_OK when a CUDA device of compute capability 10.x is current. */
dyph_status dyph_device_check(void);
/* Sticky device-side error word of the library (DYPH_ERR_TIMEOUT etc.), read
 * and cleared. Blocks on the stream. */
dyph_status dyph_download_device_error(dyph_stream s, uint32_t* out_code);
/* The same, plus where the first error was raised: 1 tile look-back, 2 sort
 * look-back, 3 grid barrier, 5 sequential solve schedule, 6 / 7 tree walk,
 * 8 narrowphase pair index. Both words are cleared. */
dyph_status dyph_download_device_error_site(dyph_stream s, uint32_t* out_code, uint32_t* out_site);
/* Iteration limit of every bounded device wait (look-backs, grid barriers,
 * dataflow polls) on the current device; 0 restores the default (2^24 polls
 * with a back-off, over a second). Synchronous. A wait that reaches the limit
 * raises DYPH_ERR_TIMEOUT in the sticky device error word and its kernel
 * returns. */
dyph_status dyph_set_spin_limit(uint32_t limit);
/* Runs one bounded wait that nothing ends, so the timeout path can be checked
 * without a fault: which 1 = a tile look-back whose predecessor never
 * publishes (error site 1), 3 = a grid barrier waiting for a block that is
 * never launched (site 3). Blocking; afterwards dyph_download_device_error_site
 * reports DYPH_ERR_TIMEOUT and the site. */
dyph_status dyph_wait_selftest(int which, dyph_stream s);
/* Blocking: DYPH_ERR_NOT_FINITE if any body's 13 state floats (pos, rot,
 * vel, ang) hold a NaN or Inf, with the smallest such body index in
 * *out_first_bad (UINT32_MAX and DYPH_OK otherwise). */
dyph_status dyph_bodies_check_finite(const dyph_bodies* bodies, dyph_stream s, uint32_t* out_first_bad);
/* Blocking raw copies between host memory and device memory (the Buffer<T>
 * upload / download of compute/include/compute/buffer.hpp:41-49). */
dyph_status dyph_copy_to_host(void* host_dst, const void* dev_src, size_t bytes, dyph_stream s);
dyph_status dyph_copy_to_device(void* dev_dst, const void* host_src, size_t bytes, dyph_stream s);

/* Host-side BodyStore::add for n bodies (core/src/body_store.cpp:28-69),
 * no device work: fills the host SoA rows of a BodyView — state13 = pos xyz,
 * rot wxyz, vel xyz, ang xyz ([13][n]), inv_mass [n], iI6 = iI_xx, iI_yy,
 * iI_zz, iI_xy, iI_xz, iI_yz ([6][n]) and flags [n]. A body is static when
 * flagged Static or mass <= 0: it gets inv_mass 0, a zero inverse inertia and
 * the Static flag; otherwise the inverse inertia is Mat3::inverse (adjugate /
 * determinant, core/include/core/math/mat3.hpp:61-79) of the body-frame
 * inertia, in float, as the reference computes it. */
void dyph_pack_bodies(uint32_t n, const float* pos, const float* rot, const float* vel, const float* ang,
                      const float* mass, const float* inertia, const uint32_t* flags_in, float* state13,
                      float* inv_mass, float* iI6, uint32_t* flags_out);

/* ── integrate — replaces integrate(Stream&, BodyView, const IntegratorParams&)
 *    (core/include/core/integrator.hpp:25, core/src/integrator.cpp:7-71) ──── */
dyph_status dyph_integrate(const dyph_bodies* bodies, const dyph_integrator_params* params, dyph_stream s);

/* ── sort — replaces sort_by_key<K,V> / sort<K>
 *    (compute/include/compute/sort.hpp:29-137). Ascending, stable LSD radix
 *    sort; unlike the reference n need not be a power of two. ──────────── */
size_t dyph_sort_workspace_bytes(size_t n);
dyph_status dyph_sort_by_key_u64_u32(uint64_t* keys, uint32_t* values, size_t n, void* workspace,
                                     size_t workspace_bytes, dyph_stream s);
dyph_status dyph_sort_u64(uint64_t* keys, size_t n, void* workspace, size_t workspace_bytes, dyph_stream s);
dyph_status dyph_sort_by_key_u32_u32(uint32_t* keys, uint32_t* values, size_t n, int key_bits, void* workspace,
                                     size_t workspace_bytes, dyph_stream s);

/* Sort by key without any device allocation and without a caller workspace.
 * No counterpart in the reference: its sort_by_key (compute/include/compute/
 * sort.hpp:29-80) is an in-place bitonic sort that needs no scratch. This
 * radix sort needs scratch, which dyph_sort_by_key_u64_u32 takes from the
 * caller and this entry point keeps inside the library.
 *
 * For callers that must not allocate device memory while they run — a host
 * engine whose frame callback owns the device memory budget, or a process at
 * its memory limit, where cudaMalloc / cudaFree would fail or synchronise the
 * device in the middle of a frame — and that cannot hand in a workspace.
 * Scratch is a fixed library-owned device array of about 4.2 MB, sized for
 * DYPH_SORT_NOALLOC_MAX_KEYS keys; larger n returns DYPH_ERR_TOO_LARGE and
 * touches nothing. The first call on each device (with that device current)
 * looks the array up and sets the sort kernels' attributes; make that first
 * call before any stream capture. The scratch counters are cleared on the
 * stream at the start of every call.
 *
 * There is one scratch array per device: calls that overlap on a device (two
 * streams, two host threads, or two graph launches in flight together) race
 * on it and give wrong results. Serialise them, e.g. on one stream.
 *
 * The looked-up address is kept per device index for the life of the
 * process: do not call this entry point on a device after cudaDeviceReset
 * has torn down the context it was first called in. */
#define DYPH_SORT_NOALLOC_MAX_KEYS 262144u
dyph_status dyph_sort_by_key_u64_u32_noalloc(uint64_t* keys, uint32_t* values, size_t n, dyph_stream s);

/* ── broadphase — replaces class Broadphase
 *    (core/include/core/broadphase.hpp:50-111, core/src/broadphase.cpp:82-377).
 *    Pairs come out already in ascending (a << 32 | b) order, so
 *    dyph_broadphase_sort_pairs is a no-op kept for the call sequence. ───── */
typedef struct dyph_broadphase dyph_broadphase;
dyph_status dyph_broadphase_create(uint32_t max_bodies, uint32_t max_pairs, dyph_broadphase** out);
void dyph_broadphase_destroy(dyph_broadphase* bp);
dyph_status dyph_broadphase_build_and_query(dyph_broadphase* bp, const dyph_bodies* bodies,
                                            const dyph_shapes* shapes, const dyph_aabb* scene_bounds,
                                            dyph_stream s);
dyph_status dyph_broadphase_sort_pairs(dyph_broadphase* bp, uint32_t n_pairs, dyph_stream s);
/* Blocking: true candidate-pair count of the last build (may exceed max_pairs). */
dyph_status dyph_broadphase_download_count(dyph_broadphase* bp, dyph_stream s, uint32_t* out);
const dyph_pair* dyph_broadphase_pairs(const dyph_broadphase* bp);
/* Device count of pairs stored (min(true count, max_pairs)). */
const uint32_t* dyph_broadphase_count_ptr(const dyph_broadphase* bp);
uint32_t dyph_broadphase_max_pairs(const dyph_broadphase* bp);
dyph_status dyph_broadphase_bvh_view(const dyph_broadphase* bp, uint32_t n_active, dyph_bvh_view* out);
/* Batched scenes (no reference counterpart: the reference steps one scene).
 * Bodies [body_offset[s], body_offset[s+1]) form scene s, which is quantised
 * against scene_bounds[s] and never paired with another scene. Morton keys
 * become (scene << 30 | code) and sort scene-major, so every scene's leaves
 * are contiguous. Each scene's pair list equals the pair list it has alone,
 * shifted by its first body index. At most 4096 scenes and 2^22 bodies. Host
 * arrays; allocates, so call outside stream capture. */
dyph_status dyph_broadphase_set_scenes(dyph_broadphase* bp, uint32_t n_scenes, const uint32_t* body_offset,
                                       const dyph_aabb* scene_bounds);

/* ── narrowphase — replaces class Narrowphase
 *    (core/include/core/narrowphase.hpp:26-73, core/src/narrowphase.cpp:1053-1144).
 *    One thread per pair; contacts are compacted in pair order, which is the
 *    order the reference's (pair_idx << 32 | sub) key sort restores. ────── */
typedef struct dyph_narrowphase dyph_narrowphase;
dyph_status dyph_narrowphase_create(uint32_t max_contacts, dyph_narrowphase** out);
void dyph_narrowphase_destroy(dyph_narrowphase* np);
/* Pair count read from device memory (no host sync). */
dyph_status dyph_narrowphase_run(dyph_narrowphase* np, const dyph_pair* pairs, const uint32_t* d_n_pairs,
                                 const dyph_bodies* bodies, const dyph_shapes* shapes, dyph_stream s);
/* Pair count given on the host. */
dyph_status dyph_narrowphase_run_host_count(dyph_narrowphase* np, const dyph_pair* pairs, uint32_t n_pairs,
                                            const dyph_bodies* bodies, const dyph_shapes* shapes,
                                            dyph_stream s);
dyph_status dyph_narrowphase_contacts(dyph_narrowphase* np, dyph_contacts* out);
dyph_status dyph_narrowphase_download_count(dyph_narrowphase* np, dyph_stream s, uint32_t* stored,
                                            uint32_t* true_count);

/* ── ray query — replaces ray_query(Stream&, BvhView, BodyView, ShapeView,
 *    const Ray*, RayHit*, n_rays) (core/include/core/ray_query.hpp:9-48,
 *    core/src/ray_query.cpp:126-195). Mirrors Ray / RayHit. The closest hit of
 *    each ray (t < t_max; body_idx UINT32_MAX on a miss) over a BVH from
 *    dyph_broadphase_bvh_view after its build: node boxes are slab-tested in
 *    fp32, leaves exactly (sphere quadratic, oriented-box slabs in the body
 *    frame; every non-sphere shape as its box). Same walk order and float
 *    expressions as the reference, so hits and ties are identical. One thread
 *    per ray; d_rays / d_hits are device arrays; asynchronous. ───────────── */
typedef struct dyph_ray {
    float ox, oy, oz; /* origin */
    float dx, dy, dz; /* direction; t is in direction units */
    float t_max;      /* the reference's default is 1e9 */
} dyph_ray;
typedef struct dyph_ray_hit {
    float t;
    uint32_t body_idx;
} dyph_ray_hit;
dyph_status dyph_ray_query(const dyph_bvh_view* bvh, const dyph_bodies* bodies, const dyph_shapes* shapes,
                           const dyph_ray* d_rays, dyph_ray_hit* d_hits, uint32_t n_rays, dyph_stream s);

/* ── contact sensor — replaces class ContactSensor
 *    (core/include/core/contact_sensor.hpp:9-58, core/src/contact_sensor.cpp:6-59):
 *    the contacts whose body a or body b (index < n_bodies) has shape
 *    shape_idx, in store order. The filter runs on the device; only the
 *    matches are copied to the host. d_body_shape is BodyView::shape (device).
 *    _filter enqueues the filter only (device view valid once the stream
 *    reaches it); _query also downloads the matches (blocking) into host
 *    arrays that stay valid until the next query. Buffers grow to the contact
 *    store's capacity on first use (allocates). ────────────────────────── */
typedef struct dyph_contact_sensor dyph_contact_sensor;
dyph_status dyph_contact_sensor_create(uint32_t shape_idx, dyph_contact_sensor** out);
void dyph_contact_sensor_destroy(dyph_contact_sensor* cs);
dyph_status dyph_contact_sensor_filter(dyph_contact_sensor* cs, const dyph_contacts* contacts,
                                       const uint32_t* d_body_shape, uint32_t n_bodies, dyph_stream s);
dyph_status dyph_contact_sensor_query(dyph_contact_sensor* cs, const dyph_contacts* contacts,
                                      const uint32_t* d_body_shape, uint32_t n_bodies, dyph_stream s,
                                      uint32_t* out_count);
uint32_t dyph_contact_sensor_count(const dyph_contact_sensor* cs);
uint32_t dyph_contact_sensor_shape_idx(const dyph_contact_sensor* cs);
/* Host (after _query) or device (after _filter) views of the matches; n
 * points at the match count (host word / device word). */
dyph_status dyph_contact_sensor_host_view(dyph_contact_sensor* cs, dyph_contacts* out);
dyph_status dyph_contact_sensor_device_view(dyph_contact_sensor* cs, dyph_contacts* out);

/* ── XPBD solver — replaces class XpbdSolver : IConstraintSolver
 *    (core/include/core/solver.hpp:11-22, core/include/core/xpbd_solver.hpp:29-70,
 *    core/src/xpbd_solver.cpp:593-733). Contacts only (JointView{} with n = 0). */
typedef struct dyph_xpbd dyph_xpbd;
dyph_status dyph_xpbd_create(int32_t n_iters, uint32_t max_contacts, uint32_t max_bodies, float friction,
                             dyph_xpbd** out);
void dyph_xpbd_destroy(dyph_xpbd* sv);
dyph_status dyph_xpbd_set_mode(dyph_xpbd* sv, dyph_solver_mode mode);
dyph_status dyph_xpbd_solve(dyph_xpbd* sv, const dyph_contacts* contacts, const dyph_bodies* bodies, float dt,
                            dyph_stream s);
/* Colours of the last coloured solve (UINT32_MAX for the sequential path) and
 * the colour count (0 = sequential). Blocking. */
dyph_status dyph_xpbd_download_colors(dyph_xpbd* sv, dyph_stream s, uint32_t* host_colors, uint32_t cap,
                                      uint32_t* n_colors);

/* Blocking: which path the last solve took (0 none / sequential, 1 coloured
 * attempt fell back to sequential, 2 coloured), its colour count and the
 * number of Jones–Plassmann rounds it needed. */
dyph_status dyph_xpbd_download_stats(dyph_xpbd* sv, dyph_stream s, uint32_t* path, uint32_t* n_colors,
                                     uint32_t* rounds);

/* Blocking: durations (ns, device clock) of the last coloured solve's phases:
 * set-up, colouring, grouping by colour, sweeps + renormalisation. */
dyph_status dyph_xpbd_download_phase_ns(dyph_xpbd* sv, dyph_stream s, uint64_t* out4);

/* ── state hash — replaces the host FNV-1a-64 loop
 *    (examples/stress_test_blocks/main.cpp:34-41, 301-311) ───────────────── */
dyph_status dyph_fnv1a64_state(const dyph_bodies* bodies, uint64_t* d_hash, dyph_stream s);

/* ── world: the whole frame step behind one handle. Replaces the open-coded
 *    loop examples/stress_test_blocks/main.cpp:264-279 (integrate,
 *    build_and_query, download_count, sort_pairs, Narrowphase::run,
 *    XpbdSolver::solve) with a sync-free, CUDA-graph-replayed sequence. ─── */
typedef struct dyph_world_desc {
    dyph_bodies bodies;       /* device SoA, updated in place */
    dyph_shapes shapes;       /* device SoA */
    dyph_aabb scene_bounds;
    dyph_integrator_params integrator;
    uint32_t max_pairs;
    uint32_t max_contacts;
    int32_t n_iters;
    float friction;
    dyph_solver_mode mode;
} dyph_world_desc;

typedef struct dyph_world dyph_world;
dyph_status dyph_world_create(const dyph_world_desc* desc, dyph_stream s, dyph_world** out);
void dyph_world_destroy(dyph_world* w);
/* Queue n_frames frame steps (graph-replayed after the first call). */
dyph_status dyph_world_step(dyph_world* w, int32_t n_frames, dyph_stream s);
/* Batched scenes in one world (dyph_broadphase_set_scenes; desc.scene_bounds is
 * then unused). No reference counterpart: the reference steps one scene per
 * solve (core/src/xpbd_solver.cpp:603-733). The solver then runs one thread
 * block per scene over the scene's contiguous run of contacts, with the
 * scene's own contact indices, so in EVERY mode each scene evolves
 * bit-identically to stepping it alone in that mode (a scene without contacts
 * in a frame is not renormalised, as the reference's solve returns at once).
 * When the largest scene also fits the fused frame (about 1,400 bodies), each
 * frame is one kernel launch: every block integrates its scene, finds its
 * candidate pairs by testing every body pair's fp16 leaf boxes (the same set
 * the LBVH traversal returns), runs the narrowphase and the solve, all in
 * shared memory; the BVH is then not built (dyph_broadphase_bvh_view is
 * empty) and the pair / contact lists are compacted on request
 * (dyph_world_sync_lists). Each scene keeps at most 48 n + 64 pairs and
 * 16 n + 64 contacts (n its body count), its capacities when stepped alone.
 * The largest scene's bodies must fit one block's shared memory (about 1,900
 * bodies); otherwise the whole batch is solved as one contact set, which is
 * exact per scene only in DYPH_SOLVER_SEQUENTIAL. Allocates; drops captured
 * graphs. */
dyph_status dyph_world_set_scenes(dyph_world* w, uint32_t n_scenes, const uint32_t* body_offset,
                                  const dyph_aabb* scene_bounds);
/* Batched worlds whose frame runs fused (one kernel launch per frame, one
 * thread block per scene: integrate, pair search, narrowphase and solve in
 * shared memory, see dyph_world_set_scenes) keep each scene's pairs and
 * contacts in per-scene slots. This call compacts the last frame's lists, in
 * the order the per-frame stages produce them, into the broadphase's pair
 * list, the narrowphase's ContactView and the solver's colours (queued on s;
 * no-op for other worlds). Call it before reading those lists. */
dyph_status dyph_world_sync_lists(dyph_world* w, dyph_stream s);
/* Knobs of the fused batched frame (no reference counterpart). Every setting
 * gives the same results bit for bit; they move only where a scene's pair and
 * contact words live (shared memory, or global memory past the cap) and how
 * many blocks fit an SM:
 *   smem_bytes     dynamic shared memory per block: what the largest scene
 *                  needs, or less (smem_cap), down to its bodies plus 64
 *                  contacts' words; with no cap and more scenes than SMs, at
 *                  most what lets two blocks share an SM;
 *   teams          0: every scene takes a block; 1: scenes whose frame fits
 *                  a quarter of that run one per warp, four to a block; 2: also
 *                  scenes that fit half of it on two warps, two to a block;
 *   register_blocks the kernel's register budget: 4, 5 or 6 resident blocks
 *                  per SM (128, 96 or 80 registers a thread; 0 = 4).
 * dyph_world_autotune times `frames` frames of each candidate (smem caps
 * 96/72/56/48/44/40/32 KB below the need and the floor itself, each team
 * policy, each register budget) from the
 * world's current state, keeps the fastest, and puts the state and the
 * statistics back; the choice is cached per device and batch profile (scene
 * sizes, solver mode, iterations, substeps) for the life of the process, so
 * a second world of the same profile takes it without timing (candidates 0).
 * Blocking; drops captured frames. */
typedef struct dyph_fused_config {
    uint32_t smem_bytes;    /* dynamic shared memory per block */
    uint32_t teams;         /* team policy (0, 1, 2) */
    uint32_t warp_scenes;   /* scenes run by one warp */
    uint32_t half_scenes;   /* scenes run by two warps */
    uint32_t block_scenes;  /* scenes run by a whole block */
    uint32_t blocks;        /* thread blocks per frame */
    uint32_t blocks_per_sm; /* resident blocks per SM at smem_bytes and the register budget */
    uint32_t register_blocks; /* the kernel variant's register budget (blocks per SM) */
    float ms_per_frame;     /* the autotuner's measurement (0 when not tuned) */
    uint32_t candidates;    /* configurations the autotuner timed (0: cached or not tuned) */
} dyph_fused_config;
dyph_status dyph_world_fused_config(dyph_world* w, dyph_fused_config* out);
dyph_status dyph_world_set_fused_config(dyph_world* w, uint32_t smem_cap, uint32_t teams, uint32_t register_blocks);
dyph_status dyph_world_autotune(dyph_world* w, int32_t frames, dyph_stream s, dyph_fused_config* out);
/* The reverse kernel of dyph_world_rollout_backward lays out its own work
 * items (same results bit for bit, whatever the setting): smem_bytes of
 * dynamic shared memory per block (0: a third of an SM's; at least the
 * largest scene's bodies plus 64 contacts' words, at most 200 KB)
 * and the same team policies, a scene's need being its bodies plus the words
 * and records of about 2.5 contacts per body (default teams 2). The kernel
 * takes 240 registers a thread, two blocks per SM; its levels are dependent
 * chains with a barrier each, so teams smaller than a block leave fewer warps
 * waiting. dyph_world_adjoint_config reports it in a dyph_fused_config
 * (register_blocks 2, ms_per_frame and candidates 0). */
dyph_status dyph_world_adjoint_config(dyph_world* w, dyph_fused_config* out);
dyph_status dyph_world_set_adjoint_config(dyph_world* w, uint32_t smem_bytes, uint32_t teams);
/* Phase timing of fused batched frames, the per-stage table of the
 * reference's --profile mode (examples/stress_test_blocks/main.cpp:199-254)
 * for a frame that is one kernel: with it on, every scene's team leader adds
 * the device-clock ns of its phases — 0 staging, integrate and leaf boxes,
 * 1 pair search, 2 narrowphase, 3 contact-solve set-up (contact lists,
 * colours or levels, groups), 4 sweep and renormalisation, 5 write-back —
 * summed over scenes (work time, not wall time). Drops captured graphs;
 * invalid for worlds that are not fused. dyph_world_download_phase_ns reads
 * (cap >= 6) and clears the sums (blocking). */
dyph_status dyph_world_set_phase_timing(dyph_world* w, int on);
dyph_status dyph_world_download_phase_ns(dyph_world* w, dyph_stream s, uint64_t* out, uint32_t cap);
/* ── adjoint: gradients through fused batched frames. No reference
 *    counterpart: the reference has no differentiation (its docs defer it). ─
 *
 * dyph_world_rollout steps n_frames frames from the world's current state and
 * stores the state at frames 0, every, 2 every, ... into d_ckpt (device,
 * [ceil(n_frames / every)][13][n] floats, rows pos xyz, rot wxyz, vel xyz,
 * ang xyz, as the BodyView arrays).
 *
 * dyph_world_rollout_backward takes d_grad_final, the adjoint of the state
 * after the rollout ([13][n]), and returns d_grad_init, the adjoint of the
 * state at frame 0 ([13][n]), and d_grad_inv_mass, the adjoint of every
 * body's inverse mass ([n], overwritten; the inverse inertia is held fixed).
 * Each checkpoint segment is recomputed forward once, from its checkpoint, by
 * a recording kernel (one launch per frame) that keeps every frame's contact
 * set, narrowphase branches and pre-solve states and stores the next frame's
 * start state; every frame is then reversed by one launch of the reverse
 * kernel, which applies the hand-written adjoints of the renormalisations,
 * the contact solves (in reverse level order), the narrowphase and the
 * integration. Segment seg - 1 is recorded on a side stream while segment
 * seg is reversed on s (with every = 1, a segment is up to 4 frames, each
 * recorded from its own checkpoint, as many as keep two segments' record
 * sets within 2 GiB; 1 frame when they do not fit the device). The contact set and every branch are those of the
 * forward frames. Static bodies get zero adjoints. Returns
 * DYPH_ERR_UNSUPPORTED (the gradients are then incomplete) when a frame took
 * a path the adjoint does not differentiate: a contact that first acted after
 * a renormalisation (deferred at w_total < 1e-10), more than 8 substeps or 10
 * iterations. Device memory beyond the checkpoints: one record set per frame
 * of two segments (2 min(L, n_frames) sets, L = every, or up to 4 when
 * every = 1, of 4 (36 + 13) bytes per contact slot plus 44 bytes per body)
 * and, when every > 1, 2 (min(every, n_frames) - 1) states. Fused batched worlds only; the world's body state is left as it
 * was. */
dyph_status dyph_world_rollout(dyph_world* w, int32_t n_frames, int32_t every, float* d_ckpt, dyph_stream s);
dyph_status dyph_world_rollout_backward(dyph_world* w, int32_t n_frames, int32_t every, const float* d_ckpt,
                                        const float* d_grad_final, float* d_grad_init, float* d_grad_inv_mass,
                                        dyph_stream s);
/* Blocking: FNV-1a-64 of every scene's pose arrays (one value for a single
 * scene); cap >= number of scenes. */
dyph_status dyph_world_scene_hashes(dyph_world* w, dyph_stream s, uint64_t* host_out, uint32_t cap);
/* dyph_bodies_check_finite over the world's bodies. */
dyph_status dyph_world_check_finite(dyph_world* w, dyph_stream s, uint32_t* out_first_bad);
/* Blocking: peak pair / contact counts and the sticky status of the frames
 * stepped so far (overflow or timeout). */
dyph_status dyph_world_download_stats(dyph_world* w, dyph_stream s, uint32_t* last_pairs,
                                      uint32_t* last_contacts, uint32_t* peak_pairs, uint32_t* peak_contacts,
                                      uint32_t* status);
/* Capture n_frames consecutive frames as one graph (an "episode"); with
 * probe_stage 0..3 (integrate, broadphase, narrowphase, solver) the caller's
 * events ev_start[f] / ev_end[f] (from dyph_event_create) are recorded around
 * that stage of frame f (probe_stage 4: around the solver's dataflow kernel
 * alone) — the per-stage timing of the reference's --profile
 * mode (examples/stress_test_blocks/main.cpp:199-254) without host fences.
 * probe_stage -1 records nothing. */
dyph_status dyph_world_capture_episode(dyph_world* w, int32_t n_frames, int32_t probe_stage,
                                       void* const* ev_start, void* const* ev_end);
dyph_status dyph_world_run_episode(dyph_world* w, dyph_stream s);
/* Timing events (cudaEvent_t behind void*). */
dyph_status dyph_event_create(void** out);
void dyph_event_destroy(void* ev);
dyph_status dyph_event_record(void* ev, dyph_stream s);
/* Blocks until `end` completes. */
dyph_status dyph_event_elapsed_ms(void* start, void* end, float* ms);
/* Blocking: true pair / contact counts of the most recent min(cap, 4096)
 * frames (oldest first) and the number of frames stepped so far. */
dyph_status dyph_world_download_history(dyph_world* w, dyph_stream s, uint32_t* pairs, uint32_t* contacts,
                                        uint32_t cap, uint32_t* frames_total);
/* Trajectory recording: replaces the example loop's download_state() +
 * write_traj_frame() every other frame (examples/stress_test_blocks/
 * main.cpp:182-197, 275-278). While set, after every frame f with
 * f % every == 0 and f / every < max_records, the pose of every body is
 * written to host_dst + (f / every) * 7 * n as n rows of x, y, z, w, qx, qy,
 * qz (the .trajectory row layout). Frames are counted by dyph_world_step from
 * this call on, and within an episode from the episode's first frame (the
 * recording is captured into the episode, so set it before
 * dyph_world_capture_episode; this call drops a captured episode). The copies
 * run on a side stream, overlapped with the next frames, and are complete when
 * the step or episode is. host_dst must be pinned host memory (cudaHostAlloc
 * or cudaHostRegister) of max_records * 7 * n floats; NULL stops recording.
 * Blocking (synchronises the world's streams). */
dyph_status dyph_world_set_trajectory(dyph_world* w, float* host_dst, uint32_t every, uint32_t max_records);
dyph_status dyph_world_broadphase(dyph_world* w, dyph_broadphase** out);
dyph_status dyph_world_narrowphase(dyph_world* w, dyph_narrowphase** out);
dyph_status dyph_world_solver(dyph_world* w, dyph_xpbd** out);

#ifdef __cplusplus
}
#endif
#endif /* DYPHUR_B200_H */
