/* Common C interface of the two CPU checkers in oracle/:
 *
 *   dyo_*  — oracle/dyphur_oracle.c, a plain-C restatement of dyphur's frame
 *            step (scalar, one thread);
 *   dyr_*  — oracle/ref_capi.cpp over the reference's own sources compiled
 *            with the host SYCL shim (oracle/_ref/libdyphur_ref.so, OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline load these libraries as the checker. The shipped library never
 * links them.
 *
 * A world is created from host BodyParams-style arrays (the fields of
 * core/include/core/body.hpp:16-25) and ShapeParams arrays
 * (core/include/core/shapes.hpp:13-19). The frame step is the sequence of
 * examples/stress_test_blocks/main.cpp:264-279.
 */
#ifndef DYPHUR_ORACLE_API_H
#define DYPHUR_ORACLE_API_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dyo_scene {
    uint32_t n_bodies;
    const float* pos;       /* [3n] */
    const float* rot;       /* [4n] w, x, y, z */
    const float* vel;       /* [3n] */
    const float* ang;       /* [3n] */
    const float* mass;      /* [n]  */
    const float* inertia;   /* [9n] row-major body-frame inertia */
    const uint32_t* shape;  /* [n]  */
    const uint32_t* flags;  /* [n]  */
    uint32_t n_shapes;
    const uint32_t* shape_type; /* [n_shapes] 0 box, 1 sphere */
    const float* shape_half;    /* [3 n_shapes] half extents (sphere radius = x) */
    uint32_t max_pairs;
    uint32_t max_contacts;
    int32_t n_iters;
    float friction;
    float bounds[6];        /* min xyz, max xyz */
    float gravity[3];
    float dt;
    int32_t n_substeps;
} dyo_scene;

/* Solver modes. */
#define DYO_SOLVER_REFERENCE 0  /* serial when n_con <= 256, else Jones–Plassmann colouring */
#define DYO_SOLVER_SERIAL 1     /* XpbdSolver::set_force_serial(true) */
#define DYO_SOLVER_COLORED 2    /* colouring at every contact count: the library's coloured mode, no reference
                                 * counterpart (the restatement only drops the n_con <= 256 test) */

/* Stages for *_run_stage. */
#define DYO_STAGE_INTEGRATE 1
#define DYO_STAGE_BROADPHASE 2   /* build_and_query + download_count + sort_pairs */
#define DYO_STAGE_NARROWPHASE 3
#define DYO_STAGE_SOLVE 4

/* Number of float arrays in a body-state snapshot: pos xyz, rot wxyz, vel xyz, ang xyz. */
#define DYO_STATE_ARRAYS 13

#ifdef __cplusplus
}
#endif
#endif
