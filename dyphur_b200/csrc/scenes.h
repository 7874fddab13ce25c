// Synthetic scene builders for the frame-step workloads (host code, C ABI).
//
// A scene set is one or more independent scenes laid out back to back in
// BodyParams-style host arrays (the fields of core/include/core/body.hpp:16-25)
// plus a shape catalogue (core/include/core/shapes.hpp:13-19). Scene s owns
// bodies [body_offset[s], body_offset[s+1]) and shapes
// [shape_offset[s], shape_offset[s+1]); body shape handles are global indices.
#pragma once
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum dyph_scene_kind {
    /* examples/stress_test_blocks/main.cpp:72-166: boxes (h = 0.4 m, 1 kg) on an
     * nx * nz footprint, ny high, at `spacing`, with uniform jitter in
     * [-jitter, jitter] per axis from std::mt19937_64(seed), over a static ground
     * box of half extents (max(20, nx/2 + 2), 0.5, same). a = (nx, ny, nz). */
    DYPH_SCENE_BOX_GRID = 0,
    /* core/tests/sim_determinism_test.cpp:41-97 (ground half width 5, bounds
     * {-20,-2,-20,20,30,20}, pair capacity 32 n + 256). a = (nx, ny, nz). */
    DYPH_SCENE_DETERMINISM = 1,
    /* Random pile: a0 bodies, 70 % boxes (half extents U[0.1,0.5]) and 30 %
     * spheres (r U[0.1,0.4]), density 500 kg/m^3, uniform positions in
     * [-20,20] x [1.5,41.5] x [-20,20], Shoemake-uniform rotations, velocity
     * N(0, 0.5) per axis, static ground of half extents (40, 0.5, 40). */
    DYPH_SCENE_RANDOM_PILE = 2,
    /* a0 independent scenes, dynamic body count log-uniform in [a1, a2]; each
     * scene is a jittered box stack (h 0.4 m, 1 kg) or a sphere pile (r 0.4 m,
     * the box's density) over its own ground box. */
    DYPH_SCENE_BATCH = 3,
    /* a0 scenes of 64 boxes (h 0.2 m, 1 kg) in a 4x4x4 block resting on the
     * ground plus a pusher box (h 0.3 m, 5 kg) starting 0.285 m from the
     * block's face and moving toward it with speed N(2, 0.3) m/s; loss
     * targets for the 64 boxes (zero rows for the pusher and the ground). */
    DYPH_SCENE_PUSH = 4,
    /* a0 independent scenes, counts log-uniform in [a1, a2], bodies drawn as in
     * DYPH_SCENE_RANDOM_PILE inside a footprint scaled to the count. */
    DYPH_SCENE_BATCH_MIXED = 5
} dyph_scene_kind;

typedef struct dyph_scene_set {
    uint32_t n_scenes, n_bodies, n_shapes;
    float* pos;      /* [3 n] */
    float* rot;      /* [4 n] w x y z */
    float* vel;      /* [3 n] */
    float* ang;      /* [3 n] */
    float* mass;     /* [n] */
    float* inertia;  /* [9 n] row-major body-frame inertia */
    uint32_t* shape; /* [n] global shape index */
    uint32_t* flags; /* [n] */
    uint32_t* shape_type; /* [n_shapes] */
    float* shape_half;    /* [3 n_shapes] */
    uint32_t* body_offset;  /* [n_scenes + 1] */
    uint32_t* shape_offset; /* [n_scenes + 1] */
    float* bounds;          /* [6 n_scenes] Morton quantisation bounds */
    float* targets;         /* [3 n] loss targets (DYPH_SCENE_PUSH), else zeros */
    uint32_t max_pairs;     /* capacity per the reference's sizing rule (largest scene) */
    uint32_t max_contacts;
    float dt;
    int32_t n_iters;
    float friction;
} dyph_scene_set;

/* BodyStore::add for n bodies (core/src/body_store.cpp:28-69): fills the
 * host SoA rows of a BodyView — state13 = pos xyz, rot wxyz, vel xyz, ang xyz
 * ([13][n]), inv_mass [n], iI6 = iI_xx, iI_yy, iI_zz, iI_xy, iI_xz, iI_yz
 * ([6][n]) and flags [n]. A body is static when flagged Static or mass <= 0;
 * a static body gets inv_mass 0, a zero inverse inertia and the Static flag;
 * otherwise the inverse inertia is Mat3::inverse (adjugate / determinant,
 * core/include/core/math/mat3.hpp:61-79) of the body-frame inertia. */
void dyph_pack_bodies(uint32_t n, const float* pos, const float* rot, const float* vel, const float* ang,
                      const float* mass, const float* inertia, const uint32_t* flags_in, float* state13,
                      float* inv_mass, float* iI6, uint32_t* flags_out);

/* Returns NULL on a bad kind or size. Free with dyph_scene_free. */
dyph_scene_set* dyph_scene_make(int kind, uint64_t seed, int32_t a0, int32_t a1, int32_t a2, float spacing,
                                float jitter);
void dyph_scene_free(dyph_scene_set* s);

#ifdef __cplusplus
}
#endif
