/* dyphur_oracle.c — plain-C, single-threaded restatement of dyphur's frame step.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA path is compared
 * against (tests/, __graft_entry__.smoke(), bench.py's CPU baseline leg). The
 * shipped library never links it.
 *
 * Parity is pinned two ways (tests/test_oracle_pins.py):
 *   - against the reference's own sources built here on a host SYCL shim
 *     (oracle/_ref), stage by stage and frame by frame, bit for bit;
 *   - against the reference's published golden vectors: the 8-box / 20-frame
 *     sim hash 0xcbcd209c3665c818 (core/tests/sim_determinism_test.cpp:224) and
 *     the narrowphase / broadphase / integrator / solver KATs of core/tests/.
 *
 * Every float expression keeps the reference's operand order and association,
 * because the goal is bit-identical results: a*b+c is evaluated as two
 * rounded operations (the build uses -ffp-contract=off on x86-64 SSE).
 */
#include "oracle_api.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ── small helpers ─────────────────────────────────────────────────────────── */

#define FLAG_STATIC 1u   /* core/include/core/body.hpp:9 */
#define FLAG_SLEEPING 4u /* core/include/core/body.hpp:11 */
#define SHAPE_BOX 0u
#define SHAPE_SPHERE 1u

static float rsqrt_ref(float x) { return 1.0f / sqrtf(x); } /* sycl::rsqrt on the host device */


/* IEEE binary16 conversion, round to nearest even (sycl::half(float)). */
static uint16_t f32_to_f16(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xFFu;
    uint32_t man = x & 0x7FFFFFu;
    if (exp == 0xFFu) return (uint16_t)(sign | 0x7C00u | (man ? 0x200u : 0u));
    int e = (int)exp - 127 + 15;
    if (e >= 0x1F) return (uint16_t)(sign | 0x7C00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        uint32_t m = man | 0x800000u;
        int shift = 14 - e; /* 24-bit significand down to a subnormal */
        uint32_t half_m = m >> shift;
        uint32_t rem = m & ((1u << shift) - 1u);
        uint32_t halfway = 1u << (shift - 1);
        if (rem > halfway || (rem == halfway && (half_m & 1u))) half_m++;
        return (uint16_t)(sign | half_m);
    }
    uint32_t h = sign | ((uint32_t)e << 10) | (man >> 13);
    uint32_t rem = man & 0x1FFFu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++; /* carry may roll into the exponent */
    return (uint16_t)h;
}

static float f16_to_f32(uint16_t h) {
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1Fu;
    uint32_t man = h & 0x3FFu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) {
            x = sign;
        } else {
            int e = -1;
            do { ++e; man <<= 1; } while (!(man & 0x400u));
            x = sign | ((uint32_t)(127 - 15 - e) << 23) | ((man & 0x3FFu) << 13);
        }
    } else if (exp == 0x1Fu) {
        x = sign | 0x7F800000u | (man << 13);
    } else {
        x = sign | ((exp - 15 + 127) << 23) | (man << 13);
    }
    float f;
    memcpy(&f, &x, 4);
    return f;
}

static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

typedef struct { uint16_t h[8]; } node_box; /* NodeBox, core/include/core/broadphase.hpp:21-25 */

/* ── world ─────────────────────────────────────────────────────────────────── */

typedef struct world {
    uint32_t n, n_shapes, max_pairs, max_contacts;
    int n_iters, n_substeps;
    float mu, dt, gravity[3], bounds[6];
    /* BodyView SoA (core/include/core/body.hpp:30-46) */
    float *px, *py, *pz, *qw, *qx, *qy, *qz, *vx, *vy, *vz, *wx, *wy, *wz;
    float *inv_mass, *iIxx, *iIyy, *iIzz, *iIxy, *iIxz, *iIyz;
    uint32_t *shape, *flags;
    uint32_t* stype;
    float *hx, *hy, *hz;
    /* broadphase */
    uint64_t* keys;
    uint32_t* sorted_idx;
    int32_t *left, *right, *parent;
    int32_t root;
    node_box* aabb;
    uint32_t* pairs; /* 2 * max_pairs */
    uint32_t n_pairs; /* true count of the last build */
    /* contacts (ContactView, core/include/core/contact.hpp:8-20) */
    uint32_t *ca, *cb;
    float *cpx, *cpy, *cpz, *cnx, *cny, *cnz, *cd;
    uint32_t nc, nc_true;
    /* solver */
    float* lambda;
    uint32_t* color;
    int colored_last;
} world;

static void* xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

static float** state_arr(world* w, float** a) {
    a[0] = w->px; a[1] = w->py; a[2] = w->pz; a[3] = w->qw; a[4] = w->qx; a[5] = w->qy; a[6] = w->qz;
    a[7] = w->vx; a[8] = w->vy; a[9] = w->vz; a[10] = w->wx; a[11] = w->wy; a[12] = w->wz;
    return a;
}

/* BodyStore::add (core/src/body_store.cpp:28-69) with Mat3::inverse
 * (core/include/core/math/mat3.hpp:61-79). */
static void add_body(world* w, uint32_t i, const dyo_scene* d) {
    w->px[i] = d->pos[3 * i]; w->py[i] = d->pos[3 * i + 1]; w->pz[i] = d->pos[3 * i + 2];
    w->qw[i] = d->rot[4 * i]; w->qx[i] = d->rot[4 * i + 1]; w->qy[i] = d->rot[4 * i + 2]; w->qz[i] = d->rot[4 * i + 3];
    w->vx[i] = d->vel[3 * i]; w->vy[i] = d->vel[3 * i + 1]; w->vz[i] = d->vel[3 * i + 2];
    w->wx[i] = d->ang[3 * i]; w->wy[i] = d->ang[3 * i + 1]; w->wz[i] = d->ang[3 * i + 2];
    int is_static = (d->flags[i] & FLAG_STATIC) || d->mass[i] <= 0.f;
    w->inv_mass[i] = is_static ? 0.f : 1.f / d->mass[i];
    if (is_static) {
        w->iIxx[i] = w->iIyy[i] = w->iIzz[i] = w->iIxy[i] = w->iIxz[i] = w->iIyz[i] = 0.f;
    } else {
        const float* m = d->inertia + 9 * i;
        float det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                    m[2] * (m[3] * m[7] - m[4] * m[6]);
        w->iIxx[i] = (m[4] * m[8] - m[5] * m[7]) / det;
        w->iIxy[i] = -(m[1] * m[8] - m[2] * m[7]) / det;
        w->iIxz[i] = (m[1] * m[5] - m[2] * m[4]) / det;
        w->iIyy[i] = (m[0] * m[8] - m[2] * m[6]) / det;
        w->iIyz[i] = -(m[0] * m[5] - m[2] * m[3]) / det;
        w->iIzz[i] = (m[0] * m[4] - m[1] * m[3]) / det;
    }
    w->shape[i] = d->shape[i];
    w->flags[i] = is_static ? (d->flags[i] | FLAG_STATIC) : d->flags[i];
}

void* dyo_create(const dyo_scene* d) {
    world* w = (world*)xcalloc(1, sizeof(world));
    if (!w) return NULL;
    uint32_t n = d->n_bodies;
    w->n = n; w->n_shapes = d->n_shapes; w->max_pairs = d->max_pairs; w->max_contacts = d->max_contacts;
    w->n_iters = d->n_iters; w->n_substeps = d->n_substeps; w->mu = d->friction; w->dt = d->dt;
    memcpy(w->gravity, d->gravity, sizeof(w->gravity));
    memcpy(w->bounds, d->bounds, sizeof(w->bounds));
    float** fields[] = {&w->px, &w->py, &w->pz, &w->qw, &w->qx, &w->qy, &w->qz, &w->vx, &w->vy, &w->vz,
                        &w->wx, &w->wy, &w->wz, &w->inv_mass, &w->iIxx, &w->iIyy, &w->iIzz,
                        &w->iIxy, &w->iIxz, &w->iIyz};
    for (size_t k = 0; k < sizeof(fields) / sizeof(fields[0]); ++k) *fields[k] = (float*)xcalloc(n, 4);
    w->shape = (uint32_t*)xcalloc(n, 4);
    w->flags = (uint32_t*)xcalloc(n, 4);
    w->stype = (uint32_t*)xcalloc(d->n_shapes, 4);
    w->hx = (float*)xcalloc(d->n_shapes, 4);
    w->hy = (float*)xcalloc(d->n_shapes, 4);
    w->hz = (float*)xcalloc(d->n_shapes, 4);
    for (uint32_t k = 0; k < d->n_shapes; ++k) {
        w->stype[k] = d->shape_type[k];
        w->hx[k] = d->shape_half[3 * k]; w->hy[k] = d->shape_half[3 * k + 1]; w->hz[k] = d->shape_half[3 * k + 2];
    }
    for (uint32_t i = 0; i < n; ++i) add_body(w, i, d);
    w->keys = (uint64_t*)xcalloc(n, 8);
    w->sorted_idx = (uint32_t*)xcalloc(n, 4);
    w->left = (int32_t*)xcalloc(n, 4);
    w->right = (int32_t*)xcalloc(n, 4);
    w->parent = (int32_t*)xcalloc(2 * (size_t)n, 4);
    w->aabb = (node_box*)xcalloc(2 * (size_t)n, sizeof(node_box));
    w->pairs = (uint32_t*)xcalloc(2 * (size_t)d->max_pairs, 4);
    uint32_t mc = d->max_contacts;
    w->ca = (uint32_t*)xcalloc(mc, 4); w->cb = (uint32_t*)xcalloc(mc, 4);
    w->cpx = (float*)xcalloc(mc, 4); w->cpy = (float*)xcalloc(mc, 4); w->cpz = (float*)xcalloc(mc, 4);
    w->cnx = (float*)xcalloc(mc, 4); w->cny = (float*)xcalloc(mc, 4); w->cnz = (float*)xcalloc(mc, 4);
    w->cd = (float*)xcalloc(mc, 4);
    w->lambda = (float*)xcalloc(mc, 4);
    w->color = (uint32_t*)xcalloc(mc, 4);
    return w;
}

void dyo_destroy(void* p) {
    world* w = (world*)p;
    if (!w) return;
    void* ptrs[] = {w->px, w->py, w->pz, w->qw, w->qx, w->qy, w->qz, w->vx, w->vy, w->vz, w->wx, w->wy,
                    w->wz, w->inv_mass, w->iIxx, w->iIyy, w->iIzz, w->iIxy, w->iIxz, w->iIyz,
                    w->shape, w->flags, w->stype, w->hx, w->hy, w->hz, w->keys, w->sorted_idx,
                    w->left, w->right, w->parent, w->aabb, w->pairs, w->ca, w->cb, w->cpx, w->cpy,
                    w->cpz, w->cnx, w->cny, w->cnz, w->cd, w->lambda, w->color};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); ++k) free(ptrs[k]);
    free(w);
}

/* ── integrate (core/src/integrator.cpp:7-71) ──────────────────────────────── */

static void integrate(world* w) {
    if (w->n == 0) return;
    const float sub_dt = w->dt / (float)w->n_substeps;
    const float gx = w->gravity[0], gy = w->gravity[1], gz = w->gravity[2];
    const float half_dt = 0.5f * sub_dt;
    for (int sub = 0; sub < w->n_substeps; ++sub) {
        for (uint32_t i = 0; i < w->n; ++i) {
            if (w->inv_mass[i] == 0.f) continue;
            if (w->flags[i] & FLAG_SLEEPING) continue;
            float vx = w->vx[i] + gx * sub_dt;
            float vy = w->vy[i] + gy * sub_dt;
            float vz = w->vz[i] + gz * sub_dt;
            w->vx[i] = vx; w->vy[i] = vy; w->vz[i] = vz;
            w->px[i] += vx * sub_dt;
            w->py[i] += vy * sub_dt;
            w->pz[i] += vz * sub_dt;
            const float ox = w->wx[i], oy = w->wy[i], oz = w->wz[i];
            float qw = w->qw[i], qx = w->qx[i], qy = w->qy[i], qz = w->qz[i];
            const float dpw = -(ox * qx + oy * qy + oz * qz);
            const float dpx = (ox * qw + oy * qz - oz * qy);
            const float dpy = (oy * qw + oz * qx - ox * qz);
            const float dpz = (oz * qw + ox * qy - oy * qx);
            qw += half_dt * dpw;
            qx += half_dt * dpx;
            qy += half_dt * dpy;
            qz += half_dt * dpz;
            const float inv_n = rsqrt_ref(qw * qw + qx * qx + qy * qy + qz * qz);
            w->qw[i] = qw * inv_n; w->qx[i] = qx * inv_n; w->qy[i] = qy * inv_n; w->qz[i] = qz * inv_n;
        }
    }
}

/* ── broadphase (core/src/broadphase.cpp) ──────────────────────────────────── */

static uint32_t expand_bits(uint32_t v) { /* broadphase.cpp:22-29 */
    v &= 0x000003ffu;
    v = (v | (v << 16u)) & 0xFF0000FFu;
    v = (v | (v << 8u)) & 0x0F00F00Fu;
    v = (v | (v << 4u)) & 0xC30C30C3u;
    v = (v | (v << 2u)) & 0x49249249u;
    return v;
}

static int delta(int i, int j, const uint64_t* codes, int n) { /* broadphase.cpp:38-41 */
    if (j < 0 || j >= n) return -1;
    return clz64(codes[i] ^ codes[j]);
}

static void find_range(int i, const uint64_t* c, int n, int* lo, int* hi) { /* broadphase.cpp:44-62 */
    int d = (delta(i, i + 1, c, n) - delta(i, i - 1, c, n)) >= 0 ? 1 : -1;
    int delta_min = delta(i, i - d, c, n);
    int l_max = 2;
    while (delta(i, i + l_max * d, c, n) > delta_min) l_max <<= 1;
    int l = 0;
    for (int t = l_max >> 1; t >= 1; t >>= 1)
        if (delta(i, i + (l + t) * d, c, n) > delta_min) l += t;
    int j = i + l * d;
    *lo = d > 0 ? i : j;
    *hi = d > 0 ? j : i;
}

static int find_split(int lo, int hi, const uint64_t* c, int n) { /* broadphase.cpp:66-76 */
    int delta_node = delta(lo, hi, c, n);
    int s = 0, step = hi - lo;
    do {
        step = (step + 1) >> 1;
        if (delta(lo, lo + s + step, c, n) > delta_node) s += step;
    } while (step > 1);
    return lo + s;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

static node_box make_box(float mnx, float mny, float mnz, float mxx, float mxy, float mxz) {
    node_box b;
    b.h[0] = f32_to_f16(mnx); b.h[1] = f32_to_f16(mny); b.h[2] = f32_to_f16(mnz);
    b.h[3] = f32_to_f16(mxx); b.h[4] = f32_to_f16(mxy); b.h[5] = f32_to_f16(mxz);
    b.h[6] = 0; b.h[7] = 0;
    return b;
}

static uint32_t broadphase(world* w) { /* Broadphase::build_and_query, broadphase.cpp:101-346 */
    const uint32_t n = w->n;
    w->n_pairs = 0;
    if (n < 2) return 0;
    const int ni = (int)n;
    const float sx0 = w->bounds[0], sy0 = w->bounds[1], sz0 = w->bounds[2];
    const float sx1 = w->bounds[3], sy1 = w->bounds[4], sz1 = w->bounds[5];
    /* Step 1: Morton keys (:118-147). */
    for (uint32_t i = 0; i < n; ++i) {
        float tx = (w->px[i] - sx0) / (sx1 - sx0);
        float ty = (w->py[i] - sy0) / (sy1 - sy0);
        float tz = (w->pz[i] - sz0) / (sz1 - sz0);
        tx = tx < 0.f ? 0.f : (tx > 1.f ? 1.f : tx);
        ty = ty < 0.f ? 0.f : (ty > 1.f ? 1.f : ty);
        tz = tz < 0.f ? 0.f : (tz > 1.f ? 1.f : tz);
        uint32_t qx = (uint32_t)(tx * 1023.f), qy = (uint32_t)(ty * 1023.f), qz = (uint32_t)(tz * 1023.f);
        uint32_t m = expand_bits(qx) | (expand_bits(qy) << 1u) | (expand_bits(qz) << 2u);
        w->keys[i] = ((uint64_t)m << 32) | (uint64_t)i;
    }
    /* Step 2: sort (:150). Keys are distinct, so any correct sort matches the bitonic order. */
    qsort(w->keys, n, sizeof(uint64_t), cmp_u64);
    for (uint32_t k = 0; k < n; ++k) w->sorted_idx[k] = (uint32_t)(w->keys[k] & 0xFFFFFFFFu);
    /* Step 3-5: Karras tree (:152-192). */
    for (uint32_t k = 0; k < 2 * n - 1; ++k) w->parent[k] = -1;
    for (int i = 0; i < ni - 1; ++i) {
        int lo, hi;
        find_range(i, w->keys, ni, &lo, &hi);
        int gamma = find_split(lo, hi, w->keys, ni);
        int lft = (lo == gamma) ? (ni - 1 + lo) : gamma;
        int rgt = (gamma + 1 == hi) ? (ni - 1 + gamma + 1) : (gamma + 1);
        w->left[i] = lft; w->right[i] = rgt;
        w->parent[lft] = i; w->parent[rgt] = i;
    }
    int root = 0;
    for (int i = 0; i < ni - 1; ++i)
        if (w->parent[i] == -1) root = i;
    w->root = root;
    /* Step 6a: leaf boxes (:216-251). */
    for (int k = 0; k < ni; ++k) {
        uint32_t body = w->sorted_idx[k];
        float px = w->px[body], py = w->py[body], pz = w->pz[body];
        uint32_t sh = w->shape[body], st = w->stype[sh];
        float hx = w->hx[sh];
        float mnx, mny, mnz, mxx, mxy, mxz;
        if (st == SHAPE_SPHERE) {
            mnx = px - hx; mxx = px + hx; mny = py - hx; mxy = py + hx; mnz = pz - hx; mxz = pz + hx;
        } else {
            float qw = w->qw[body], qx = w->qx[body], qy = w->qy[body], qz = w->qz[body];
            float hy = w->hy[sh], hz = w->hz[sh];
            float rxx = 1.f - 2.f * (qy * qy + qz * qz);
            float rxy = 2.f * (qx * qy - qz * qw);
            float rxz = 2.f * (qx * qz + qy * qw);
            float ryx = 2.f * (qx * qy + qz * qw);
            float ryy = 1.f - 2.f * (qx * qx + qz * qz);
            float ryz = 2.f * (qy * qz - qx * qw);
            float rzx = 2.f * (qx * qz - qy * qw);
            float rzy = 2.f * (qy * qz + qx * qw);
            float rzz = 1.f - 2.f * (qx * qx + qy * qy);
            float ex = fabsf(rxx) * hx + fabsf(rxy) * hy + fabsf(rxz) * hz;
            float ey = fabsf(ryx) * hx + fabsf(ryy) * hy + fabsf(ryz) * hz;
            float ez = fabsf(rzx) * hx + fabsf(rzy) * hy + fabsf(rzz) * hz;
            mnx = px - ex; mxx = px + ex; mny = py - ey; mxy = py + ey; mnz = pz - ez; mxz = pz + ez;
        }
        w->aabb[ni - 1 + k] = make_box(mnx, mny, mnz, mxx, mxy, mxz);
    }
    /* Step 6b: refit (:253-287) — children before parents; fp16 min/max is exact,
     * so a post-order walk gives the same boxes as the level-synchronised rounds. */
    {
        int* order = (int*)xcalloc(n, sizeof(int));
        int* stack = (int*)xcalloc(2 * (size_t)n, sizeof(int));
        int top = 0, cnt = 0;
        stack[top++] = root;
        while (top > 0) { /* pre-order, then reverse it */
            int node = stack[--top];
            if (node >= ni - 1) continue;
            order[cnt++] = node;
            stack[top++] = w->left[node];
            stack[top++] = w->right[node];
        }
        for (int k = cnt - 1; k >= 0; --k) {
            int p = order[k];
            node_box bl = w->aabb[w->left[p]], br = w->aabb[w->right[p]], b;
            for (int a = 0; a < 3; ++a) {
                b.h[a] = f32_to_f16(fminf(f16_to_f32(bl.h[a]), f16_to_f32(br.h[a])));
                b.h[3 + a] = f32_to_f16(fmaxf(f16_to_f32(bl.h[3 + a]), f16_to_f32(br.h[3 + a])));
            }
            b.h[6] = 0; b.h[7] = 0;
            w->aabb[p] = b;
        }
        free(order);
        free(stack);
    }
    /* Step 7: traversal (:290-345) with a 64-entry stack per leaf. */
    uint64_t* pk = (uint64_t*)xcalloc(16, 8);
    size_t pk_cap = 16, cnt = 0;
    for (int j = 0; j < ni; ++j) {
        node_box jb = w->aabb[ni - 1 + j];
        float jmnx = f16_to_f32(jb.h[0]), jmxx = f16_to_f32(jb.h[3]);
        float jmny = f16_to_f32(jb.h[1]), jmxy = f16_to_f32(jb.h[4]);
        float jmnz = f16_to_f32(jb.h[2]), jmxz = f16_to_f32(jb.h[5]);
        int stack[64], top = 0;
        stack[top++] = root;
        while (top > 0) {
            int node = stack[--top];
            node_box nb = w->aabb[node];
            if (f16_to_f32(nb.h[0]) > jmxx || f16_to_f32(nb.h[3]) < jmnx || f16_to_f32(nb.h[1]) > jmxy ||
                f16_to_f32(nb.h[4]) < jmny || f16_to_f32(nb.h[2]) > jmxz || f16_to_f32(nb.h[5]) < jmnz)
                continue;
            if (node >= ni - 1) {
                int li = node - (ni - 1);
                if (li < j) {
                    uint32_t a = w->sorted_idx[li], b = w->sorted_idx[j];
                    if (a > b) { uint32_t t = a; a = b; b = t; }
                    if (cnt == pk_cap) { pk_cap *= 2; pk = (uint64_t*)realloc(pk, pk_cap * 8); }
                    pk[cnt++] = ((uint64_t)a << 32) | b;
                }
                continue;
            }
            stack[top++] = w->left[node];
            stack[top++] = w->right[node];
        }
    }
    /* sort_pairs (:348-359): ascending (a << 32 | b). */
    qsort(pk, cnt, 8, cmp_u64);
    uint32_t keep = cnt < w->max_pairs ? (uint32_t)cnt : w->max_pairs;
    for (uint32_t i = 0; i < keep; ++i) {
        w->pairs[2 * i] = (uint32_t)(pk[i] >> 32);
        w->pairs[2 * i + 1] = (uint32_t)(pk[i] & 0xFFFFFFFFu);
    }
    free(pk);
    w->n_pairs = (uint32_t)cnt;
    return (uint32_t)cnt;
}

/* ── narrowphase (core/src/narrowphase.cpp) ────────────────────────────────── */

static int sphere_sphere(float acx, float acy, float acz, float ra, float bcx, float bcy, float bcz,
                         float rb, float* px, float* py, float* pz, float* nx, float* ny, float* nz,
                         float* depth) { /* narrowphase.cpp:46-68 */
    float dx = acx - bcx, dy = acy - bcy, dz = acz - bcz;
    float dist2 = dx * dx + dy * dy + dz * dz;
    float sum_r = ra + rb;
    if (dist2 >= sum_r * sum_r) return 0;
    float dist = sqrtf(dist2);
    if (dist < 1e-8f) { *nx = 0.f; *ny = 1.f; *nz = 0.f; }
    else { float inv = 1.f / dist; *nx = dx * inv; *ny = dy * inv; *nz = dz * inv; }
    *depth = sum_r - dist;
    float sa = acx - *nx * ra, sb = bcx + *nx * rb;
    *px = 0.5f * (sa + sb);
    sa = acy - *ny * ra; sb = bcy + *ny * rb; *py = 0.5f * (sa + sb);
    sa = acz - *nz * ra; sb = bcz + *nz * rb; *pz = 0.5f * (sa + sb);
    return 1;
}

static int sphere_box(float scx, float scy, float scz, float sr, float bcx, float bcy, float bcz,
                      const float E[3][3], float bh0, float bh1, float bh2, float* px, float* py,
                      float* pz, float* nx, float* ny, float* nz, float* depth) { /* narrowphase.cpp:71-127 */
    float e0x = E[0][0], e0y = E[0][1], e0z = E[0][2];
    float e1x = E[1][0], e1y = E[1][1], e1z = E[1][2];
    float e2x = E[2][0], e2y = E[2][1], e2z = E[2][2];
    float dx = scx - bcx, dy = scy - bcy, dz = scz - bcz;
    float q0 = dx * e0x + dy * e0y + dz * e0z;
    float q1 = dx * e1x + dy * e1y + dz * e1z;
    float q2 = dx * e2x + dy * e2y + dz * e2z;
    float c0 = q0 < -bh0 ? -bh0 : (q0 > bh0 ? bh0 : q0);
    float c1 = q1 < -bh1 ? -bh1 : (q1 > bh1 ? bh1 : q1);
    float c2 = q2 < -bh2 ? -bh2 : (q2 > bh2 ? bh2 : q2);
    float lx = q0 - c0, ly = q1 - c1, lz = q2 - c2;
    float dist2 = lx * lx + ly * ly + lz * lz;
    if (dist2 < 1e-12f) {
        float pen0 = bh0 - fabsf(q0), pen1 = bh1 - fabsf(q1), pen2 = bh2 - fabsf(q2);
        if (pen0 <= pen1 && pen0 <= pen2) {
            float s = q0 >= 0.f ? 1.f : -1.f;
            *nx = -(s * e0x); *ny = -(s * e0y); *nz = -(s * e0z);
            *depth = sr + pen0;
        } else if (pen1 <= pen2) {
            float s = q1 >= 0.f ? 1.f : -1.f;
            *nx = -(s * e1x); *ny = -(s * e1y); *nz = -(s * e1z);
            *depth = sr + pen1;
        } else {
            float s = q2 >= 0.f ? 1.f : -1.f;
            *nx = -(s * e2x); *ny = -(s * e2y); *nz = -(s * e2z);
            *depth = sr + pen2;
        }
        *px = scx - *nx * sr; *py = scy - *ny * sr; *pz = scz - *nz * sr;
        return 1;
    }
    if (dist2 >= sr * sr) return 0;
    float dist = sqrtf(dist2);
    float inv_d = 1.f / dist;
    float wx = lx * e0x + ly * e1x + lz * e2x;
    float wy = lx * e0y + ly * e1y + lz * e2y;
    float wz = lx * e0z + ly * e1z + lz * e2z;
    *nx = -wx * inv_d; *ny = -wy * inv_d; *nz = -wz * inv_d;
    *depth = sr - dist;
    *px = bcx + c0 * e0x + c1 * e1x + c2 * e2x;
    *py = bcy + c0 * e0y + c1 * e1y + c2 * e2y;
    *pz = bcz + c0 * e0z + c1 * e1z + c2 * e2z;
    return 1;
}

/* One SAT axis (the SAT_TEST macro, narrowphase.cpp:158-175, and the edge
 * block :192-208 have the same arithmetic). Returns 0 when separated. */
static int sat_axis(float lx, float ly, float lz, const float Ae[3][3], const float Ah[3],
                    const float Be[3][3], const float Bh[3], float dx, float dy, float dz, int type,
                    int i, int j, float* best_ov, int* best_type, int* best_i, int* best_j,
                    float* bnx, float* bny, float* bnz) {
    float rA = Ah[0] * fabsf(lx * Ae[0][0] + ly * Ae[0][1] + lz * Ae[0][2]) +
               Ah[1] * fabsf(lx * Ae[1][0] + ly * Ae[1][1] + lz * Ae[1][2]) +
               Ah[2] * fabsf(lx * Ae[2][0] + ly * Ae[2][1] + lz * Ae[2][2]);
    float rB = Bh[0] * fabsf(lx * Be[0][0] + ly * Be[0][1] + lz * Be[0][2]) +
               Bh[1] * fabsf(lx * Be[1][0] + ly * Be[1][1] + lz * Be[1][2]) +
               Bh[2] * fabsf(lx * Be[2][0] + ly * Be[2][1] + lz * Be[2][2]);
    float t = fabsf(dx * lx + dy * ly + dz * lz);
    float ov = rA + rB - t;
    if (ov <= 0.f) return 0;
    if (ov < *best_ov) {
        *best_ov = ov;
        *best_type = type; *best_i = i; *best_j = j;
        float sgn = (dx * lx + dy * ly + dz * lz) >= 0.f ? -1.f : 1.f;
        *bnx = sgn * lx; *bny = sgn * ly; *bnz = sgn * lz;
    }
    return 1;
}

static int box_box(float acx, float acy, float acz, const float Ae[3][3], const float Ah[3], float bcx,
                   float bcy, float bcz, const float Be[3][3], const float Bh[3], float opx[4],
                   float opy[4], float opz[4], float* onx, float* ony, float* onz,
                   float od[4]) { /* narrowphase.cpp:130-306 */
    const float eps_par = 1e-5f;
    float C[3][3];
    float dx = bcx - acx, dy = bcy - acy, dz = bcz - acz;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i][j] = Ae[i][0] * Be[j][0] + Ae[i][1] * Be[j][1] + Ae[i][2] * Be[j][2];
    float best_ov = 1e30f;
    int best_type = -1, best_i = 0, best_j = 0;
    float bnx = 0.f, bny = 1.f, bnz = 0.f;
    for (int i = 0; i < 3; ++i)
        if (!sat_axis(Ae[i][0], Ae[i][1], Ae[i][2], Ae, Ah, Be, Bh, dx, dy, dz, 0, i, 0, &best_ov,
                      &best_type, &best_i, &best_j, &bnx, &bny, &bnz))
            return 0;
    for (int i = 0; i < 3; ++i)
        if (!sat_axis(Be[i][0], Be[i][1], Be[i][2], Ae, Ah, Be, Bh, dx, dy, dz, 1, i, 0, &best_ov,
                      &best_type, &best_i, &best_j, &bnx, &bny, &bnz))
            return 0;
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) {
            float cx = Ae[i][1] * Be[j][2] - Ae[i][2] * Be[j][1];
            float cy = Ae[i][2] * Be[j][0] - Ae[i][0] * Be[j][2];
            float cz = Ae[i][0] * Be[j][1] - Ae[i][1] * Be[j][0];
            float len2 = cx * cx + cy * cy + cz * cz;
            if (len2 < eps_par * eps_par) continue;
            float inv_l = rsqrt_ref(len2);
            if (!sat_axis(cx * inv_l, cy * inv_l, cz * inv_l, Ae, Ah, Be, Bh, dx, dy, dz, 2, i, j,
                          &best_ov, &best_type, &best_i, &best_j, &bnx, &bny, &bnz))
                return 0;
        }
    }
    *onx = bnx; *ony = bny; *onz = bnz;
    int n_out = 0;
    if (best_type == 0 || best_type == 1) {
        if (best_type == 0) {
            int t0A = (best_i + 1) % 3, t1A = (best_i + 2) % 3;
            int j_best = 0;
            for (int j = 1; j < 3; ++j)
                if (fabsf(C[best_i][j]) > fabsf(C[best_i][j_best])) j_best = j;
            int t0B = (j_best + 1) % 3, t1B = (j_best + 2) % 3;
            if (Bh[t0B] * Bh[t1B] > Ah[t0A] * Ah[t1A]) { best_type = 1; best_i = j_best; }
        }
        int a_is_ref = (best_type == 0);
        int ref_ax = best_i;
        float rcx = a_is_ref ? acx : bcx, rcy = a_is_ref ? acy : bcy;
        const float(*Re)[3] = a_is_ref ? Ae : Be;
        const float* Rh = a_is_ref ? Ah : Bh;
        const float(*Ie)[3] = a_is_ref ? Be : Ae;
        const float* Ih = a_is_ref ? Bh : Ah;
        float icx = a_is_ref ? bcx : acx, icy = a_is_ref ? bcy : acy, icz = a_is_ref ? bcz : acz;
        int t0 = (ref_ax + 1) % 3, t1 = (ref_ax + 2) % 3;
        float rc_dot_n3 = rcx * bnx + rcy * bny + (a_is_ref ? acz : bcz) * bnz;
        float sign_depth = a_is_ref ? 1.f : -1.f;
        for (int k = 0; k < 8; ++k) {
            float sx = (k & 1) ? 1.f : -1.f, sy = (k & 2) ? 1.f : -1.f, sz = (k & 4) ? 1.f : -1.f;
            float vx = icx + sx * Ih[0] * Ie[0][0] + sy * Ih[1] * Ie[1][0] + sz * Ih[2] * Ie[2][0];
            float vy = icy + sx * Ih[0] * Ie[0][1] + sy * Ih[1] * Ie[1][1] + sz * Ih[2] * Ie[2][1];
            float vz = icz + sx * Ih[0] * Ie[0][2] + sy * Ih[1] * Ie[1][2] + sz * Ih[2] * Ie[2][2];
            float v_dot_n = vx * bnx + vy * bny + vz * bnz;
            float dv = Rh[ref_ax] + sign_depth * (v_dot_n - rc_dot_n3);
            if (dv <= 0.f) continue;
            float vx_rel = vx - (a_is_ref ? acx : bcx);
            float vy_rel = vy - (a_is_ref ? acy : bcy);
            float vz_rel = vz - (a_is_ref ? acz : bcz);
            float qt0 = vx_rel * Re[t0][0] + vy_rel * Re[t0][1] + vz_rel * Re[t0][2];
            float qt1 = vx_rel * Re[t1][0] + vy_rel * Re[t1][1] + vz_rel * Re[t1][2];
            if (fabsf(qt0) > Rh[t0] + 1e-3f) continue;
            if (fabsf(qt1) > Rh[t1] + 1e-3f) continue;
            float cpx = vx - sign_depth * dv * bnx;
            float cpy = vy - sign_depth * dv * bny;
            float cpz = vz - sign_depth * dv * bnz;
            if (n_out < 4) {
                opx[n_out] = cpx; opy[n_out] = cpy; opz[n_out] = cpz; od[n_out] = dv;
                ++n_out;
            }
        }
    } else {
        int i = best_i, j = best_j;
        int t0A = (i + 1) % 3, t1A = (i + 2) % 3;
        float s0A = (-bnx * Ae[t0A][0] - bny * Ae[t0A][1] - bnz * Ae[t0A][2]) >= 0.f ? 1.f : -1.f;
        float s1A = (-bnx * Ae[t1A][0] - bny * Ae[t1A][1] - bnz * Ae[t1A][2]) >= 0.f ? 1.f : -1.f;
        float pAx = acx + s0A * Ah[t0A] * Ae[t0A][0] + s1A * Ah[t1A] * Ae[t1A][0];
        float pAy = acy + s0A * Ah[t0A] * Ae[t0A][1] + s1A * Ah[t1A] * Ae[t1A][1];
        float pAz = acz + s0A * Ah[t0A] * Ae[t0A][2] + s1A * Ah[t1A] * Ae[t1A][2];
        int t0B = (j + 1) % 3, t1B = (j + 2) % 3;
        float s0B = (bnx * Be[t0B][0] + bny * Be[t0B][1] + bnz * Be[t0B][2]) >= 0.f ? 1.f : -1.f;
        float s1B = (bnx * Be[t1B][0] + bny * Be[t1B][1] + bnz * Be[t1B][2]) >= 0.f ? 1.f : -1.f;
        float pBx = bcx + s0B * Bh[t0B] * Be[t0B][0] + s1B * Bh[t1B] * Be[t1B][0];
        float pBy = bcy + s0B * Bh[t0B] * Be[t0B][1] + s1B * Bh[t1B] * Be[t1B][1];
        float pBz = bcz + s0B * Bh[t0B] * Be[t0B][2] + s1B * Bh[t1B] * Be[t1B][2];
        float uAx = Ae[i][0], uAy = Ae[i][1], uAz = Ae[i][2];
        float uBx = Be[j][0], uBy = Be[j][1], uBz = Be[j][2];
        float b12 = C[i][j];
        float denom = 1.f - b12 * b12;
        float wx = pAx - pBx, wy = pAy - pBy, wz = pAz - pBz;
        float d1 = wx * uAx + wy * uAy + wz * uAz;
        float d2 = wx * uBx + wy * uBy + wz * uBz;
        float s_t = 0.f, t_t = 0.f;
        if (fabsf(denom) > 1e-6f) {
            s_t = (b12 * d2 - d1) / denom;
            t_t = (d2 - b12 * d1) / denom;
        }
        float qAx = pAx + s_t * uAx, qAy = pAy + s_t * uAy, qAz = pAz + s_t * uAz;
        float qBx = pBx + t_t * uBx, qBy = pBy + t_t * uBy, qBz = pBz + t_t * uBz;
        opx[0] = 0.5f * (qAx + qBx);
        opy[0] = 0.5f * (qAy + qBy);
        opz[0] = 0.5f * (qAz + qBz);
        od[0] = best_ov;
        n_out = 1;
    }
    return n_out;
}

static void make_axes(float qw, float qx, float qy, float qz, float Ae[3][3]) { /* narrowphase.cpp:913-917 */
    Ae[0][0] = 1.f - 2.f * (qy * qy + qz * qz); Ae[0][1] = 2.f * (qx * qy + qz * qw); Ae[0][2] = 2.f * (qx * qz - qy * qw);
    Ae[1][0] = 2.f * (qx * qy - qz * qw); Ae[1][1] = 1.f - 2.f * (qx * qx + qz * qz); Ae[1][2] = 2.f * (qy * qz + qx * qw);
    Ae[2][0] = 2.f * (qx * qz + qy * qw); Ae[2][1] = 2.f * (qy * qz - qx * qw); Ae[2][2] = 1.f - 2.f * (qx * qx + qy * qy);
}

static void emit(world* w, uint32_t ia, uint32_t ib, float px, float py, float pz, float nx, float ny,
                 float nz, float d) {
    uint32_t idx = w->nc_true++;
    if (idx >= w->max_contacts) return;
    w->ca[idx] = ia; w->cb[idx] = ib;
    w->cpx[idx] = px; w->cpy[idx] = py; w->cpz[idx] = pz;
    w->cnx[idx] = nx; w->cny[idx] = ny; w->cnz[idx] = nz;
    w->cd[idx] = d;
}

/* process_pair for box / sphere shapes (narrowphase.cpp:920-1001). Pairs are
 * processed in order, so appends land in the order the reference's
 * (pair_idx, sub) key sort restores (:1077-1127). */
static void process_pair(world* w, uint32_t ia, uint32_t ib) {
    uint32_t sha = w->shape[ia], shb = w->shape[ib];
    uint32_t ta = w->stype[sha], tb = w->stype[shb];
    float px, py, pz, nx, ny, nz, depth;
    if (ta == SHAPE_SPHERE && tb == SHAPE_SPHERE) {
        if (!sphere_sphere(w->px[ia], w->py[ia], w->pz[ia], w->hx[sha], w->px[ib], w->py[ib], w->pz[ib],
                           w->hx[shb], &px, &py, &pz, &nx, &ny, &nz, &depth))
            return;
        emit(w, ia, ib, px, py, pz, nx, ny, nz, depth);
        return;
    }
    if (ta == SHAPE_SPHERE && tb == SHAPE_BOX) {
        float Be[3][3];
        make_axes(w->qw[ib], w->qx[ib], w->qy[ib], w->qz[ib], Be);
        if (!sphere_box(w->px[ia], w->py[ia], w->pz[ia], w->hx[sha], w->px[ib], w->py[ib], w->pz[ib], Be,
                        w->hx[shb], w->hy[shb], w->hz[shb], &px, &py, &pz, &nx, &ny, &nz, &depth))
            return;
        nx = -nx; ny = -ny; nz = -nz;
        emit(w, ia, ib, px, py, pz, nx, ny, nz, depth);
        return;
    }
    if (ta == SHAPE_BOX && tb == SHAPE_SPHERE) {
        float Ae[3][3];
        make_axes(w->qw[ia], w->qx[ia], w->qy[ia], w->qz[ia], Ae);
        if (!sphere_box(w->px[ib], w->py[ib], w->pz[ib], w->hx[shb], w->px[ia], w->py[ia], w->pz[ia], Ae,
                        w->hx[sha], w->hy[sha], w->hz[sha], &px, &py, &pz, &nx, &ny, &nz, &depth))
            return;
        emit(w, ia, ib, px, py, pz, nx, ny, nz, depth);
        return;
    }
    if (ta == SHAPE_BOX && tb == SHAPE_BOX) {
        float Ae[3][3], Be[3][3];
        float Ah[3] = {w->hx[sha], w->hy[sha], w->hz[sha]};
        float Bh[3] = {w->hx[shb], w->hy[shb], w->hz[shb]};
        make_axes(w->qw[ia], w->qx[ia], w->qy[ia], w->qz[ia], Ae);
        make_axes(w->qw[ib], w->qx[ib], w->qy[ib], w->qz[ib], Be);
        float opx[4], opy[4], opz[4], od[4], onx, ony, onz;
        int nc = box_box(w->px[ia], w->py[ia], w->pz[ia], Ae, Ah, w->px[ib], w->py[ib], w->pz[ib], Be, Bh,
                         opx, opy, opz, &onx, &ony, &onz, od);
        if (nc > 0) {
            float cx = 0, cy = 0, cz = 0, cd = 0;
            for (int k = 0; k < nc; ++k) { cx += opx[k]; cy += opy[k]; cz += opz[k]; cd += od[k]; }
            float inv = 1.f / (float)nc;
            emit(w, ia, ib, cx * inv, cy * inv, cz * inv, onx, ony, onz, cd * inv);
        }
    }
}

static void narrowphase(world* w) {
    w->nc = 0; w->nc_true = 0;
    uint32_t np = w->n_pairs < w->max_pairs ? w->n_pairs : w->max_pairs;
    for (uint32_t i = 0; i < np; ++i) process_pair(w, w->pairs[2 * i], w->pairs[2 * i + 1]);
    w->nc = w->nc_true < w->max_contacts ? w->nc_true : w->max_contacts;
}

/* ── XPBD solver (core/src/xpbd_solver.cpp) ────────────────────────────────── */

static void world_inv_inertia(const world* w, uint32_t bi, float vx, float vy, float vz, float* ox,
                              float* oy, float* oz) { /* xpbd_solver.cpp:40-59 */
    float qw = w->qw[bi], qx = w->qx[bi], qy = w->qy[bi], qz = w->qz[bi];
    float R00 = 1.f - 2.f * (qy * qy + qz * qz), R01 = 2.f * (qx * qy + qz * qw), R02 = 2.f * (qx * qz - qy * qw);
    float R10 = 2.f * (qx * qy - qz * qw), R11 = 1.f - 2.f * (qx * qx + qz * qz), R12 = 2.f * (qy * qz + qx * qw);
    float R20 = 2.f * (qx * qz + qy * qw), R21 = 2.f * (qy * qz - qx * qw), R22 = 1.f - 2.f * (qx * qx + qy * qy);
    float lx = R00 * vx + R10 * vy + R20 * vz;
    float ly = R01 * vx + R11 * vy + R21 * vz;
    float lz = R02 * vx + R12 * vy + R22 * vz;
    float ilx = w->iIxx[bi] * lx + w->iIxy[bi] * ly + w->iIxz[bi] * lz;
    float ily = w->iIxy[bi] * lx + w->iIyy[bi] * ly + w->iIyz[bi] * lz;
    float ilz = w->iIxz[bi] * lx + w->iIyz[bi] * ly + w->iIzz[bi] * lz;
    *ox = R00 * ilx + R01 * ily + R02 * ilz;
    *oy = R10 * ilx + R11 * ily + R12 * ilz;
    *oz = R20 * ilx + R21 * ily + R22 * ilz;
}

static void apply_ang_delta(world* w, uint32_t bi, float ax, float ay, float az) { /* :78-87 */
    if (w->inv_mass[bi] == 0.f) return;
    float qw = w->qw[bi], qx = w->qx[bi], qy = w->qy[bi], qz = w->qz[bi];
    w->qw[bi] += 0.5f * (-ax * qx - ay * qy - az * qz);
    w->qx[bi] += 0.5f * (ax * qw + ay * qz - az * qy);
    w->qy[bi] += 0.5f * (-ax * qz + ay * qw + az * qx);
    w->qz[bi] += 0.5f * (ax * qy - ay * qx + az * qw);
}

static void solve_contact(world* w, uint32_t c, float mu, float* lc, float dt) { /* :413-521 */
    uint32_t ia = w->ca[c], ib = w->cb[c];
    float depth = w->cd[c];
    if (depth <= 0.f) return;
    float remaining = depth - lc[c];
    if (remaining <= 1e-6f) return;
    float nx = w->cnx[c], ny = w->cny[c], nz = w->cnz[c];
    float px = w->cpx[c], py = w->cpy[c], pz = w->cpz[c];
    float wa = w->inv_mass[ia], wb = w->inv_mass[ib];
    float rax = px - w->px[ia], ray = py - w->py[ia], raz = pz - w->pz[ia];
    float rbx = px - w->px[ib], rby = py - w->py[ib], rbz = pz - w->pz[ib];
    float raxnx = ray * nz - raz * ny, raxny = raz * nx - rax * nz, raxnz = rax * ny - ray * nx;
    float rbxnx = rby * nz - rbz * ny, rbxny = rbz * nx - rbx * nz, rbxnz = rbx * ny - rby * nx;
    float iIa_x, iIa_y, iIa_z, iIb_x, iIb_y, iIb_z;
    world_inv_inertia(w, ia, raxnx, raxny, raxnz, &iIa_x, &iIa_y, &iIa_z);
    world_inv_inertia(w, ib, rbxnx, rbxny, rbxnz, &iIb_x, &iIb_y, &iIb_z);
    float wa_ang = raxnx * iIa_x + raxny * iIa_y + raxnz * iIa_z;
    float wb_ang = rbxnx * iIb_x + rbxny * iIb_y + rbxnz * iIb_z;
    float w_total = wa + wb + wa_ang + wb_ang;
    if (w_total < 1e-10f) return;
    float dl = remaining / w_total;
    lc[c] += remaining;
    if (wa != 0.f) { w->px[ia] += wa * dl * nx; w->py[ia] += wa * dl * ny; w->pz[ia] += wa * dl * nz; }
    if (wb != 0.f) { w->px[ib] -= wb * dl * nx; w->py[ib] -= wb * dl * ny; w->pz[ib] -= wb * dl * nz; }
    apply_ang_delta(w, ia, dl * iIa_x, dl * iIa_y, dl * iIa_z);
    apply_ang_delta(w, ib, -dl * iIb_x, -dl * iIb_y, -dl * iIb_z);
    float oax = w->wx[ia], oay = w->wy[ia], oaz = w->wz[ia];
    float obx = w->wx[ib], oby = w->wy[ib], obz = w->wz[ib];
    float vcax = w->vx[ia] + oay * raz - oaz * ray;
    float vcay = w->vy[ia] + oaz * rax - oax * raz;
    float vcaz = w->vz[ia] + oax * ray - oay * rax;
    float vcbx = w->vx[ib] + oby * rbz - obz * rby;
    float vcby = w->vy[ib] + obz * rbx - obx * rbz;
    float vcbz = w->vz[ib] + obx * rby - oby * rbx;
    float vrel_x = vcax - vcbx, vrel_y = vcay - vcby, vrel_z = vcaz - vcbz;
    float vrel_n = vrel_x * nx + vrel_y * ny + vrel_z * nz;
    if (vrel_n < 0.f) {
        float j_n = -vrel_n / w_total;
        float doa_x, doa_y, doa_z, dob_x, dob_y, dob_z;
        world_inv_inertia(w, ia, raxnx, raxny, raxnz, &doa_x, &doa_y, &doa_z);
        world_inv_inertia(w, ib, rbxnx, rbxny, rbxnz, &dob_x, &dob_y, &dob_z);
        if (wa != 0.f) {
            w->vx[ia] += wa * j_n * nx; w->vy[ia] += wa * j_n * ny; w->vz[ia] += wa * j_n * nz;
            w->wx[ia] += j_n * doa_x; w->wy[ia] += j_n * doa_y; w->wz[ia] += j_n * doa_z;
        }
        if (wb != 0.f) {
            w->vx[ib] -= wb * j_n * nx; w->vy[ib] -= wb * j_n * ny; w->vz[ib] -= wb * j_n * nz;
            w->wx[ib] -= j_n * dob_x; w->wy[ib] -= j_n * dob_y; w->wz[ib] -= j_n * dob_z;
        }
    }
    if (mu > 0.f) {
        float oax2 = w->wx[ia], oay2 = w->wy[ia], oaz2 = w->wz[ia];
        float obx2 = w->wx[ib], oby2 = w->wy[ib], obz2 = w->wz[ib];
        float vcax2 = w->vx[ia] + oay2 * raz - oaz2 * ray;
        float vcay2 = w->vy[ia] + oaz2 * rax - oax2 * raz;
        float vcaz2 = w->vz[ia] + oax2 * ray - oay2 * rax;
        float vcbx2 = w->vx[ib] + oby2 * rbz - obz2 * rby;
        float vcby2 = w->vy[ib] + obz2 * rbx - obx2 * rbz;
        float vcbz2 = w->vz[ib] + obx2 * rby - oby2 * rbx;
        float rvx = vcax2 - vcbx2, rvy = vcay2 - vcby2, rvz = vcaz2 - vcbz2;
        float rvn = rvx * nx + rvy * ny + rvz * nz;
        float vt_x = rvx - rvn * nx, vt_y = rvy - rvn * ny, vt_z = rvz - rvn * nz;
        float vt2 = vt_x * vt_x + vt_y * vt_y + vt_z * vt_z;
        if (vt2 > 1e-12f) {
            float vt_len = sqrtf(vt2);
            float tx = vt_x / vt_len, ty = vt_y / vt_len, tz = vt_z / vt_len;
            float ratx = ray * tz - raz * ty, raty = raz * tx - rax * tz, ratz = rax * ty - ray * tx;
            float rbtx = rby * tz - rbz * ty, rbty = rbz * tx - rbx * tz, rbtz = rbx * ty - rby * tx;
            float fIa_x, fIa_y, fIa_z, fIb_x, fIb_y, fIb_z;
            world_inv_inertia(w, ia, ratx, raty, ratz, &fIa_x, &fIa_y, &fIa_z);
            world_inv_inertia(w, ib, rbtx, rbty, rbtz, &fIb_x, &fIb_y, &fIb_z);
            float wt = wa + wb + ratx * fIa_x + raty * fIa_y + ratz * fIa_z + rbtx * fIb_x + rbty * fIb_y +
                       rbtz * fIb_z;
            if (wt > 1e-10f) {
                float j_n_static = lc[c] / (dt * w_total);
                float j_t = vt_len / wt;
                j_t = fminf(j_t, mu * j_n_static);
                if (wa != 0.f) {
                    w->vx[ia] -= wa * j_t * tx; w->vy[ia] -= wa * j_t * ty; w->vz[ia] -= wa * j_t * tz;
                    w->wx[ia] -= j_t * fIa_x; w->wy[ia] -= j_t * fIa_y; w->wz[ia] -= j_t * fIa_z;
                }
                if (wb != 0.f) {
                    w->vx[ib] += wb * j_t * tx; w->vy[ib] += wb * j_t * ty; w->vz[ib] += wb * j_t * tz;
                    w->wx[ib] += j_t * fIb_x; w->wy[ib] += j_t * fIb_y; w->wz[ib] += j_t * fIb_z;
                }
            }
        }
    }
}

static void renormalize(world* w) { /* xpbd_solver.cpp:579-584, 726-731 */
    for (uint32_t i = 0; i < w->n; ++i) {
        float qw = w->qw[i], qx = w->qx[i], qy = w->qy[i], qz = w->qz[i];
        float inv_len = rsqrt_ref(qw * qw + qx * qx + qy * qy + qz * qz);
        w->qw[i] = qw * inv_len; w->qx[i] = qx * inv_len; w->qy[i] = qy * inv_len; w->qz[i] = qz * inv_len;
    }
}

static void run_serial(world* w, uint32_t nc) { /* :559-587 (no joints) */
    for (int iter = 0; iter < w->n_iters; ++iter) {
        for (uint32_t c = 0; c < nc; ++c) solve_contact(w, c, w->mu, w->lambda, w->dt);
        renormalize(w);
    }
}

static uint32_t hash_u32(uint32_t x) { /* :31-34 */
    x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;
    return x;
}

/* Jones–Plassmann colouring (:620-694), emulated round by round. Returns the
 * colour count, or 0 when the reference falls back to the serial path. */
static uint32_t jp_color(world* w, uint32_t n_con) {
    const uint32_t UNC = 0xFFFFFFFFu;
    uint64_t* bpri = (uint64_t*)xcalloc(w->n, 8);
    uint64_t* bmask = (uint64_t*)xcalloc(w->n, 8);
    for (uint32_t k = 0; k < n_con; ++k) w->color[k] = UNC;
    uint32_t max_color = 0, overflow = 0, rem = n_con, r = 0;
    while (rem > 0 && r < 256u) {
        for (uint32_t bi = 0; bi < 8u && r < 256u; ++bi, ++r) {
            memset(bpri, 0, w->n * 8);
            for (uint32_t k = 0; k < n_con; ++k) {
                if (w->color[k] != UNC) continue;
                uint32_t a = w->ca[k], b = w->cb[k];
                uint64_t pk = ((uint64_t)hash_u32(k) << 32) | k;
                if (w->inv_mass[a] != 0.f && bpri[a] < pk) bpri[a] = pk;
                if (w->inv_mass[b] != 0.f && bpri[b] < pk) bpri[b] = pk;
            }
            for (uint32_t k = 0; k < n_con; ++k) {
                if (w->color[k] != UNC) continue;
                uint32_t a = w->ca[k], b = w->cb[k];
                int da = w->inv_mass[a] != 0.f, db = w->inv_mass[b] != 0.f;
                uint64_t pk = ((uint64_t)hash_u32(k) << 32) | k;
                if ((da && bpri[a] != pk) || (db && bpri[b] != pk)) continue;
                uint64_t used = (da ? bmask[a] : 0ull) | (db ? bmask[b] : 0ull);
                uint64_t freebits = ~used;
                if (freebits == 0ull) { overflow = 1; continue; }
                uint64_t lowbit = freebits & (0ull - freebits);
                uint32_t col = 63u - (uint32_t)clz64(lowbit);
                w->color[k] = col;
                uint64_t bit = (uint64_t)1 << col;
                if (da) bmask[a] |= bit;
                if (db) bmask[b] |= bit;
                if (col > max_color) max_color = col;
                rem--;
            }
        }
    }
    free(bpri);
    free(bmask);
    if (rem > 0 || overflow) return 0;
    return max_color + 1;
}

static void solve(world* w, int mode) { /* XpbdSolver::solve, :603-733 */
    memset(w->lambda, 0, (size_t)w->max_contacts * 4);
    uint32_t nc = w->nc;
    w->colored_last = 0;
    if (nc == 0) return;
    if (mode == DYO_SOLVER_SERIAL || (mode == DYO_SOLVER_REFERENCE && nc <= 256u)) { run_serial(w, nc); return; }
    uint32_t n_colors = jp_color(w, nc);
    if (n_colors == 0) { run_serial(w, nc); return; }
    w->colored_last = 1;
    for (int iter = 0; iter < w->n_iters; ++iter) {
        for (uint32_t ci = 0; ci < n_colors; ++ci)
            for (uint32_t k = 0; k < nc; ++k)
                if (w->color[k] == ci) solve_contact(w, k, w->mu, w->lambda, w->dt);
        renormalize(w);
    }
}

/* ── C interface (oracle_api.h) ────────────────────────────────────────────── */

int dyo_run_stage(void* p, int stage, int mode) {
    world* w = (world*)p;
    switch (stage) {
        case DYO_STAGE_INTEGRATE: integrate(w); return 0;
        case DYO_STAGE_BROADPHASE: broadphase(w); return 0;
        case DYO_STAGE_NARROWPHASE: narrowphase(w); return w->nc_true > w->max_contacts ? -3 : 0;
        case DYO_STAGE_SOLVE: solve(w, mode); return 0;
        default: return -1;
    }
}

int dyo_step(void* p, int n_frames, int mode) {
    for (int f = 0; f < n_frames; ++f)
        for (int st = DYO_STAGE_INTEGRATE; st <= DYO_STAGE_SOLVE; ++st) {
            int rc = dyo_run_stage(p, st, mode);
            if (rc != 0) return rc;
        }
    return 0;
}

void dyo_get_state(void* p, float* out) {
    world* w = (world*)p;
    float* a[DYO_STATE_ARRAYS];
    state_arr(w, a);
    for (int k = 0; k < DYO_STATE_ARRAYS; ++k) memcpy(out + (size_t)k * w->n, a[k], w->n * 4);
}

void dyo_set_state(void* p, const float* in) {
    world* w = (world*)p;
    float* a[DYO_STATE_ARRAYS];
    state_arr(w, a);
    for (int k = 0; k < DYO_STATE_ARRAYS; ++k) memcpy(a[k], in + (size_t)k * w->n, w->n * 4);
}

void dyo_get_inv(void* p, float* inv_mass, float* iI6) {
    world* w = (world*)p;
    memcpy(inv_mass, w->inv_mass, w->n * 4);
    const float* src[6] = {w->iIxx, w->iIyy, w->iIzz, w->iIxy, w->iIxz, w->iIyz};
    for (int k = 0; k < 6; ++k) memcpy(iI6 + (size_t)k * w->n, src[k], w->n * 4);
}

/* FNV-1a-64 over pos_x … rot_z (examples/stress_test_blocks/main.cpp:34-41, 301-311). */
uint64_t dyo_fnv1a64(const void* data, size_t nbytes, uint64_t h) {
    const uint8_t* q = (const uint8_t*)data;
    for (size_t i = 0; i < nbytes; ++i) { h ^= q[i]; h *= 0x00000100000001B3ULL; }
    return h;
}

uint64_t dyo_hash(void* p) {
    world* w = (world*)p;
    float* a[DYO_STATE_ARRAYS];
    state_arr(w, a);
    uint64_t h = 0xcbf29ce484222325ULL;
    for (int k = 0; k < 7; ++k) h = dyo_fnv1a64(a[k], w->n * 4, h);
    return h;
}

uint32_t dyo_get_pairs(void* p, uint32_t* ab, uint32_t cap) {
    world* w = (world*)p;
    uint32_t m = w->n_pairs < w->max_pairs ? w->n_pairs : w->max_pairs;
    if (m > cap) m = cap;
    memcpy(ab, w->pairs, (size_t)m * 8);
    return w->n_pairs;
}

uint32_t dyo_get_contacts(void* p, uint32_t* ab, float* p7, uint32_t cap) {
    world* w = (world*)p;
    uint32_t m = w->nc < cap ? w->nc : cap;
    for (uint32_t c = 0; c < m; ++c) {
        ab[2 * c] = w->ca[c]; ab[2 * c + 1] = w->cb[c];
        float* o = p7 + 7 * (size_t)c;
        o[0] = w->cpx[c]; o[1] = w->cpy[c]; o[2] = w->cpz[c];
        o[3] = w->cnx[c]; o[4] = w->cny[c]; o[5] = w->cnz[c]; o[6] = w->cd[c];
    }
    return w->nc;
}

void dyo_get_bvh(void* p, uint64_t* keys, uint32_t* sorted_idx, int32_t* left, int32_t* right,
                 int32_t* parent, uint16_t* aabb8) {
    world* w = (world*)p;
    uint32_t n = w->n;
    memcpy(keys, w->keys, (size_t)n * 8);
    memcpy(sorted_idx, w->sorted_idx, (size_t)n * 4);
    if (n >= 2) {
        memcpy(left, w->left, (size_t)(n - 1) * 4);
        memcpy(right, w->right, (size_t)(n - 1) * 4);
        memcpy(parent, w->parent, (size_t)(2 * n - 1) * 4);
        memcpy(aabb8, w->aabb, (size_t)(2 * n - 1) * sizeof(node_box));
    }
}

uint32_t dyo_get_colors(void* p, uint32_t* out, uint32_t cap) {
    world* w = (world*)p;
    uint32_t m = w->nc < cap ? w->nc : cap;
    for (uint32_t c = 0; c < m; ++c) out[c] = w->colored_last ? w->color[c] : 0xFFFFFFFFu;
    return w->nc;
}

/* ── ray query and contact sensor ─────────────────────────────────────────── */

/* Slab test against a node box (core/src/ray_query.cpp:14-33). */
static int ray_node_hit(const float* r, const float* inv, float mnx, float mny, float mnz, float mxx, float mxy,
                        float mxz, float best_t) {
    float t1x = (mnx - r[0]) * inv[0], t2x = (mxx - r[0]) * inv[0];
    float t1y = (mny - r[1]) * inv[1], t2y = (mxy - r[1]) * inv[1];
    float t1z = (mnz - r[2]) * inv[2], t2z = (mxz - r[2]) * inv[2];
    float tmin = t1x < t2x ? t1x : t2x, tmax = t1x < t2x ? t2x : t1x;
    float ylo = t1y < t2y ? t1y : t2y, yhi = t1y < t2y ? t2y : t1y;
    float zlo = t1z < t2z ? t1z : t2z, zhi = t1z < t2z ? t2z : t1z;
    tmin = tmin > ylo ? tmin : ylo;
    tmax = tmax < yhi ? tmax : yhi;
    tmin = tmin > zlo ? tmin : zlo;
    tmax = tmax < zhi ? tmax : zhi;
    return tmax >= 0.f && tmax >= tmin && tmin < best_t;
}

/* v by the conjugate of q (Quat::rotate, core/include/core/math/quat.hpp:39-42). */
static void rot_conj(float qw, float qx, float qy, float qz, const float v[3], float o[3]) {
    float ux = -qx, uy = -qy, uz = -qz;
    float tx = (uy * v[2] - uz * v[1]) * 2.f, ty = (uz * v[0] - ux * v[2]) * 2.f, tz = (ux * v[1] - uy * v[0]) * 2.f;
    o[0] = (v[0] + tx * qw) + (uy * tz - uz * ty);
    o[1] = (v[1] + ty * qw) + (uz * tx - ux * tz);
    o[2] = (v[2] + tz * qw) + (ux * ty - uy * tx);
}

/* Exact leaf test (core/src/ray_query.cpp:37-123). */
static void ray_leaf(const world* w, uint32_t bi, const float* r, float* best_t, uint32_t* best_body) {
    uint32_t sh = w->shape[bi];
    float hx = w->hx[sh], t;
    if (w->stype[sh] == 1u) { /* sphere */
        float ocx = r[0] - w->px[bi], ocy = r[1] - w->py[bi], ocz = r[2] - w->pz[bi];
        float a = r[3] * r[3] + r[4] * r[4] + r[5] * r[5];
        float b = r[3] * ocx + r[4] * ocy + r[5] * ocz;
        float c = ocx * ocx + ocy * ocy + ocz * ocz - hx * hx;
        float disc = b * b - a * c;
        if (disc < 0.f) {
            t = -1.f;
        } else {
            float sq = sqrtf(disc);
            t = (-b - sq) / a;
            if (t < 0.f) t = (-b + sq) / a;
            t = (t >= 0.f && t < *best_t) ? t : -1.f;
        }
    } else { /* box, and every other type as its box */
        float oc[3] = {r[0] - w->px[bi], r[1] - w->py[bi], r[2] - w->pz[bi]}, d[3] = {r[3], r[4], r[5]};
        float lo[3], ld[3];
        rot_conj(w->qw[bi], w->qx[bi], w->qy[bi], w->qz[bi], oc, lo);
        rot_conj(w->qw[bi], w->qx[bi], w->qy[bi], w->qz[bi], d, ld);
        float h[3] = {hx, w->hy[sh], w->hz[sh]};
        float tmin = 0.f, tmax = 0.f;
        for (int k = 0; k < 3; ++k) {
            float inv = 1.f / ld[k];
            float t1 = (-h[k] - lo[k]) * inv, t2 = (h[k] - lo[k]) * inv;
            float l = t1 < t2 ? t1 : t2, u = t1 < t2 ? t2 : t1;
            if (k == 0) {
                tmin = l;
                tmax = u;
            } else {
                tmin = tmin > l ? tmin : l;
                tmax = tmax < u ? tmax : u;
            }
        }
        if (tmax < 0.f || tmin > tmax) {
            t = -1.f;
        } else {
            t = tmin >= 0.f ? tmin : tmax;
            t = (t >= 0.f && t < *best_t) ? t : -1.f;
        }
    }
    if (t >= 0.f) {
        *best_t = t;
        *best_body = bi;
    }
}

/* ray_query (core/src/ray_query.cpp:126-195) over the tree of the last
 * broadphase stage and the current poses. rays: [7 n_rays] = origin xyz,
 * direction xyz, t_max. */
void dyo_ray_query(void* p, const float* rays, uint32_t n_rays, float* out_t, uint32_t* out_body) {
    world* w = (world*)p;
    for (uint32_t q = 0; q < n_rays; ++q) {
        const float* r = rays + 7 * (size_t)q;
        float best_t = r[6];
        uint32_t best_body = 0xFFFFFFFFu;
        float inv[3] = {1.f / r[3], 1.f / r[4], 1.f / r[5]};
        if (w->n == 1) {
            ray_leaf(w, 0u, r, &best_t, &best_body);
        } else if (w->n > 1) {
            int32_t stack[64];
            int top = 0;
            const int32_t n_int = (int32_t)w->n - 1;
            stack[top++] = w->root;
            while (top > 0) {
                int32_t node = stack[--top];
                const node_box* nb = &w->aabb[node];
                if (!ray_node_hit(r, inv, f16_to_f32(nb->h[0]), f16_to_f32(nb->h[1]), f16_to_f32(nb->h[2]),
                                  f16_to_f32(nb->h[3]), f16_to_f32(nb->h[4]), f16_to_f32(nb->h[5]), best_t))
                    continue;
                if (node >= n_int) {
                    ray_leaf(w, w->sorted_idx[node - n_int], r, &best_t, &best_body);
                } else if (top + 1 < 64) {
                    stack[top++] = w->right[node];
                    stack[top++] = w->left[node];
                }
            }
        }
        out_t[q] = best_t;
        out_body[q] = best_body;
    }
}

/* ContactSensor::query (core/src/contact_sensor.cpp:6-59) on the contacts of
 * the last narrowphase stage, with the bodies' shapes as body_shapes. Writes
 * ab[2m], p7[7m] like dyo_get_contacts; returns the match count. */
uint32_t dyo_contact_sensor(void* p, uint32_t shape_idx, uint32_t* ab, float* p7, uint32_t cap) {
    world* w = (world*)p;
    uint32_t m = 0;
    for (uint32_t c = 0; c < w->nc; ++c) {
        uint32_t a = w->ca[c], b = w->cb[c];
        int hit = (a < w->n && w->shape[a] == shape_idx) || (b < w->n && w->shape[b] == shape_idx);
        if (!hit) continue;
        if (m < cap) {
            ab[2 * m] = a;
            ab[2 * m + 1] = b;
            float* o = p7 + 7 * (size_t)m;
            o[0] = w->cpx[c]; o[1] = w->cpy[c]; o[2] = w->cpz[c];
            o[3] = w->cnx[c]; o[4] = w->cny[c]; o[5] = w->cnz[c];
            o[6] = w->cd[c];
        }
        ++m;
    }
    return m;
}

/* Stand-alone helpers for unit KATs. */
uint16_t dyo_f32_to_f16(float f) { return f32_to_f16(f); }
float dyo_f16_to_f32(uint16_t h) { return f16_to_f32(h); }
