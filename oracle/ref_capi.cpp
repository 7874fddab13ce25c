// C interface over the reference's own frame-step classes, compiled from the
// reference sources with the host SYCL shim (oracle/sycl_shim). Built by
// oracle/Makefile into oracle/_ref/libdyphur_ref.so.
//
// TEST INFRASTRUCTURE ONLY: the parity checker and the "reference" CPU
// baseline. The step sequence is examples/stress_test_blocks/main.cpp:264-279;
// scene construction goes through BodyStore::add / ShapeStore::add
// (core/src/body_store.cpp:28-69, core/src/shapes.cpp:19-27) exactly as the
// reference's examples do.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <vector>

#include <sycl/sycl.hpp>

// The checker reads a few private buffers (sorted Morton keys, JP colours) that
// the reference keeps inside its classes; no reference behaviour is changed.
#define private public
#include <compute/device.hpp>
#include <core/articulation.hpp>
#include <core/body_store.hpp>
#include <core/broadphase.hpp>
#include <core/contact_sensor.hpp>
#include <core/integrator.hpp>
#include <core/narrowphase.hpp>
#include <core/ray_query.hpp>
#include <core/shape_store.hpp>
#include <core/xpbd_solver.hpp>
#undef private

#include "oracle_api.h"

using namespace dyphur;

namespace {

uint32_t next_pow2_u32(uint32_t n) {
    if (n <= 1u) return 1u;
    --n;
    n |= n >> 1u; n |= n >> 2u; n |= n >> 4u; n |= n >> 8u; n |= n >> 16u;
    return n + 1u;
}

struct RefWorld {
    Device dev;
    Stream s;
    ShapeStore ss;
    BodyStore bs;
    Broadphase bp;
    Narrowphase np;
    XpbdSolver solver;
    IntegratorParams ip;
    AABB bounds{};
    float dt = 1.f / 60.f;
    uint32_t n = 0;
    uint32_t max_pairs = 0;
    uint32_t n_pairs = 0;
    bool colored_last = false;

    explicit RefWorld(const dyo_scene* d)
        : dev(Device::default_cpu()),
          s(dev.make_stream()),
          ss(s, d->n_shapes),
          bs(s, d->n_bodies),
          bp(s, d->n_bodies, d->max_pairs),
          np(s, d->max_contacts),
          solver(s, d->n_iters, d->max_contacts, d->friction) {
        for (uint32_t k = 0; k < d->n_shapes; ++k) {
            ShapeParams sp;
            sp.type = static_cast<ShapeType>(d->shape_type[k]);
            sp.half_x = d->shape_half[3 * k + 0];
            sp.half_y = d->shape_half[3 * k + 1];
            sp.half_z = d->shape_half[3 * k + 2];
            ss.add(sp);
        }
        ss.upload();
        for (uint32_t i = 0; i < d->n_bodies; ++i) {
            BodyParams p;
            p.position = {d->pos[3 * i], d->pos[3 * i + 1], d->pos[3 * i + 2]};
            p.rotation = Quatf(d->rot[4 * i], d->rot[4 * i + 1], d->rot[4 * i + 2], d->rot[4 * i + 3]);
            p.linear_velocity = {d->vel[3 * i], d->vel[3 * i + 1], d->vel[3 * i + 2]};
            p.angular_velocity = {d->ang[3 * i], d->ang[3 * i + 1], d->ang[3 * i + 2]};
            p.mass = d->mass[i];
            const float* I = d->inertia + 9 * i;
            p.inertia = Mat3f(I[0], I[1], I[2], I[3], I[4], I[5], I[6], I[7], I[8]);
            p.shape_handle = d->shape[i];
            p.flags = d->flags[i];
            bs.add(p);
        }
        bs.upload();
        s.wait();
        ip.gravity = {d->gravity[0], d->gravity[1], d->gravity[2]};
        ip.dt = d->dt;
        ip.n_substeps = d->n_substeps;
        dt = d->dt;
        n = d->n_bodies;
        max_pairs = d->max_pairs;
        std::memcpy(&bounds, d->bounds, sizeof(bounds));
    }

    int stage(int st, int mode) {
        // The reference has no always-coloured mode (DYO_SOLVER_COLORED).
        if (mode != DYO_SOLVER_REFERENCE && mode != DYO_SOLVER_SERIAL) return -2;
        BodyView bv = bs.view();
        ShapeView sv = ss.view();
        switch (st) {
            case DYO_STAGE_INTEGRATE:
                integrate(s, bv, ip);
                return 0;
            case DYO_STAGE_BROADPHASE: {
                bp.build_and_query(s, bv, sv, bounds);
                n_pairs = bp.download_count(s);
                // Broadphase::sort_pairs sorts next_pow2(n_pairs) entries in
                // buffers of max_pairs; refuse counts that would run past them.
                if (next_pow2_u32(n_pairs) > max_pairs && n_pairs > 1) return -2;
                bp.sort_pairs(s, n_pairs);
                return 0;
            }
            case DYO_STAGE_NARROWPHASE:
                np.run(s, bp.pairs_ptr(), std::min(n_pairs, max_pairs), bv, sv);
                return np.overflowed() ? -3 : 0;
            case DYO_STAGE_SOLVE: {
                solver.set_force_serial(mode == DYO_SOLVER_SERIAL);
                uint32_t nc = np.download_count(s);
                colored_last = !(mode == DYO_SOLVER_SERIAL || nc <= XpbdSolver::kSerialThreshold);
                solver.solve(s, np.contacts(), JointView{}, bv, dt);
                return 0;
            }
            default:
                return -1;
        }
    }
};

uint64_t fnv1a64(uint64_t h, const void* data, size_t n) {
    const auto* p = static_cast<const uint8_t*>(data);
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 0x00000100000001B3ULL;
    }
    return h;
}

float* state_ptr(BodyView& v, int k) {
    float* arr[DYO_STATE_ARRAYS] = {v.pos_x, v.pos_y, v.pos_z, v.rot_w, v.rot_x, v.rot_y, v.rot_z,
                                    v.vel_x, v.vel_y, v.vel_z, v.ang_x, v.ang_y, v.ang_z};
    return arr[k];
}

}  // namespace

extern "C" {

void* dyr_create(const dyo_scene* d) {
    try {
        return new RefWorld(d);
    } catch (...) {
        return nullptr;
    }
}

void dyr_destroy(void* w) { delete static_cast<RefWorld*>(w); }

int dyr_run_stage(void* w, int stage, int mode) { return static_cast<RefWorld*>(w)->stage(stage, mode); }

int dyr_step(void* w, int n_frames, int mode) {
    auto* rw = static_cast<RefWorld*>(w);
    for (int f = 0; f < n_frames; ++f) {
        for (int st = DYO_STAGE_INTEGRATE; st <= DYO_STAGE_SOLVE; ++st) {
            int rc = rw->stage(st, mode);
            if (rc != 0) return rc;
        }
    }
    return 0;
}

void dyr_get_state(void* w, float* out) {
    auto* rw = static_cast<RefWorld*>(w);
    BodyView v = rw->bs.view();
    for (int k = 0; k < DYO_STATE_ARRAYS; ++k)
        std::memcpy(out + static_cast<size_t>(k) * rw->n, state_ptr(v, k), rw->n * sizeof(float));
}

void dyr_set_state(void* w, const float* in) {
    auto* rw = static_cast<RefWorld*>(w);
    BodyView v = rw->bs.view();
    for (int k = 0; k < DYO_STATE_ARRAYS; ++k)
        std::memcpy(state_ptr(v, k), in + static_cast<size_t>(k) * rw->n, rw->n * sizeof(float));
}

void dyr_get_inv(void* w, float* inv_mass, float* iI6) {
    auto* rw = static_cast<RefWorld*>(w);
    BodyView v = rw->bs.view();
    const uint32_t n = rw->n;
    std::memcpy(inv_mass, v.inv_mass, n * sizeof(float));
    const float* src[6] = {v.iI_xx, v.iI_yy, v.iI_zz, v.iI_xy, v.iI_xz, v.iI_yz};
    for (int k = 0; k < 6; ++k) std::memcpy(iI6 + static_cast<size_t>(k) * n, src[k], n * sizeof(float));
}

uint64_t dyr_hash(void* w) {
    auto* rw = static_cast<RefWorld*>(w);
    BodyView v = rw->bs.view();
    uint64_t h = 0xcbf29ce484222325ULL;
    for (int k = 0; k < 7; ++k) h = fnv1a64(h, state_ptr(v, k), rw->n * sizeof(float));
    return h;
}

uint32_t dyr_get_pairs(void* w, uint32_t* ab, uint32_t cap) {
    auto* rw = static_cast<RefWorld*>(w);
    uint32_t m = std::min({rw->n_pairs, rw->max_pairs, cap});
    const ContactPair* p = rw->bp.pairs_ptr();
    for (uint32_t i = 0; i < m; ++i) {
        ab[2 * i] = p[i].a;
        ab[2 * i + 1] = p[i].b;
    }
    return rw->n_pairs;
}

// Contacts of the last narrowphase in store order: ab[2c], p7[7c] =
// pos xyz, normal xyz, depth.
uint32_t dyr_get_contacts(void* w, uint32_t* ab, float* p7, uint32_t cap) {
    auto* rw = static_cast<RefWorld*>(w);
    ContactView cv = rw->np.contacts();
    uint32_t nc = rw->np.download_count(rw->s);
    uint32_t m = std::min(nc, cap);
    for (uint32_t c = 0; c < m; ++c) {
        ab[2 * c] = cv.body_a[c];
        ab[2 * c + 1] = cv.body_b[c];
        float* o = p7 + 7 * static_cast<size_t>(c);
        o[0] = cv.pos_x[c]; o[1] = cv.pos_y[c]; o[2] = cv.pos_z[c];
        o[3] = cv.norm_x[c]; o[4] = cv.norm_y[c]; o[5] = cv.norm_z[c];
        o[6] = cv.depth[c];
    }
    return nc;
}

// BVH of the last build: sorted 64-bit Morton keys [n], sorted_idx [n],
// left/right [n-1], parent [2n-1], node boxes [2n-1] x 8 halves (raw bits).
void dyr_get_bvh(void* w, uint64_t* keys, uint32_t* sorted_idx, int32_t* left, int32_t* right,
                 int32_t* parent, uint16_t* aabb8) {
    auto* rw = static_cast<RefWorld*>(w);
    const uint32_t n = rw->n;
    std::memcpy(keys, rw->bp.d_morton_.data(), n * sizeof(uint64_t));
    std::memcpy(sorted_idx, rw->bp.d_sorted_idx_.data(), n * sizeof(uint32_t));
    if (n >= 2) {
        std::memcpy(left, rw->bp.d_left_.data(), (n - 1) * sizeof(int32_t));
        std::memcpy(right, rw->bp.d_right_.data(), (n - 1) * sizeof(int32_t));
        std::memcpy(parent, rw->bp.d_parent_.data(), (2 * n - 1) * sizeof(int32_t));
        std::memcpy(aabb8, rw->bp.d_aabb_.data(), (2 * n - 1) * sizeof(NodeBox));
    }
}

// Jones–Plassmann colours of the last coloured solve (UINT32_MAX when the last
// solve took the serial path). Returns the constraint count.
uint32_t dyr_get_colors(void* w, uint32_t* out, uint32_t cap) {
    auto* rw = static_cast<RefWorld*>(w);
    uint32_t nc = rw->np.download_count(rw->s);
    uint32_t m = std::min(nc, cap);
    if (!rw->colored_last) {
        for (uint32_t c = 0; c < m; ++c) out[c] = 0xFFFFFFFFu;
        return nc;
    }
    std::memcpy(out, rw->solver.color_.data(), m * sizeof(uint32_t));
    return nc;
}

// ray_query (core/src/ray_query.cpp:126-195) over the tree of the last
// broadphase stage. rays: [7 n_rays] = origin xyz, direction xyz, t_max.
void dyr_ray_query(void* w, const float* rays, uint32_t n_rays, float* out_t, uint32_t* out_body) {
    auto* rw = static_cast<RefWorld*>(w);
    if (n_rays == 0) return;
    std::vector<Ray> r(n_rays);
    std::vector<RayHit> h(n_rays);
    for (uint32_t q = 0; q < n_rays; ++q) {
        const float* x = rays + 7 * static_cast<size_t>(q);
        r[q] = Ray{x[0], x[1], x[2], x[3], x[4], x[5], x[6]};
    }
    ray_query(rw->s, rw->bp.bvh_view(rw->n), rw->bs.view(), rw->ss.view(), r.data(), h.data(), n_rays);
    rw->s.wait();
    for (uint32_t q = 0; q < n_rays; ++q) {
        out_t[q] = h[q].t;
        out_body[q] = h[q].body_idx;
    }
}

// ContactSensor(shape_idx).query(s, np, bs.body_shapes()) on the contacts of
// the last narrowphase stage (core/src/contact_sensor.cpp:6-59). Writes
// ab[2m], p7[7m]; returns the match count.
uint32_t dyr_contact_sensor(void* w, uint32_t shape_idx, uint32_t* ab, float* p7, uint32_t cap) {
    auto* rw = static_cast<RefWorld*>(w);
    ContactSensor cs(shape_idx);
    uint32_t m = cs.query(rw->s, rw->np, rw->bs.body_shapes());
    for (uint32_t c = 0; c < std::min(m, cap); ++c) {
        ab[2 * c] = cs.body_a()[c];
        ab[2 * c + 1] = cs.body_b()[c];
        float* o = p7 + 7 * static_cast<size_t>(c);
        o[0] = cs.pos_x()[c]; o[1] = cs.pos_y()[c]; o[2] = cs.pos_z()[c];
        o[3] = cs.norm_x()[c]; o[4] = cs.norm_y()[c]; o[5] = cs.norm_z()[c];
        o[6] = cs.depth()[c];
    }
    return m;
}

}  // extern "C"
