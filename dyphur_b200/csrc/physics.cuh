// Per-body / per-pair / per-contact device math of the frame step.
//
// Every function states the formula of the reference source it follows and
// keeps its operand order, so the results match the reference bit for bit
// under --fmad=false (see common.cuh). Functions are templated on a body
// accessor so the same code runs on global SoA arrays (per-scene path) and on
// shared-memory copies (batched path).
#pragma once

#include "common.cuh"

namespace dyph {

// Accessor over the BodyView SoA in global memory.
struct GlobalBodies {
    dyph_bodies v;
    __device__ __forceinline__ float& px(uint32_t i) const { return v.pos_x[i]; }
    __device__ __forceinline__ float& py(uint32_t i) const { return v.pos_y[i]; }
    __device__ __forceinline__ float& pz(uint32_t i) const { return v.pos_z[i]; }
    __device__ __forceinline__ float& qw(uint32_t i) const { return v.rot_w[i]; }
    __device__ __forceinline__ float& qx(uint32_t i) const { return v.rot_x[i]; }
    __device__ __forceinline__ float& qy(uint32_t i) const { return v.rot_y[i]; }
    __device__ __forceinline__ float& qz(uint32_t i) const { return v.rot_z[i]; }
    __device__ __forceinline__ float& vx(uint32_t i) const { return v.vel_x[i]; }
    __device__ __forceinline__ float& vy(uint32_t i) const { return v.vel_y[i]; }
    __device__ __forceinline__ float& vz(uint32_t i) const { return v.vel_z[i]; }
    __device__ __forceinline__ float& wx(uint32_t i) const { return v.ang_x[i]; }
    __device__ __forceinline__ float& wy(uint32_t i) const { return v.ang_y[i]; }
    __device__ __forceinline__ float& wz(uint32_t i) const { return v.ang_z[i]; }
    __device__ __forceinline__ float im(uint32_t i) const { return v.inv_mass[i]; }
    __device__ __forceinline__ float ixx(uint32_t i) const { return v.iI_xx[i]; }
    __device__ __forceinline__ float iyy(uint32_t i) const { return v.iI_yy[i]; }
    __device__ __forceinline__ float izz(uint32_t i) const { return v.iI_zz[i]; }
    __device__ __forceinline__ float ixy(uint32_t i) const { return v.iI_xy[i]; }
    __device__ __forceinline__ float ixz(uint32_t i) const { return v.iI_xz[i]; }
    __device__ __forceinline__ float iyz(uint32_t i) const { return v.iI_yz[i]; }
    __device__ __forceinline__ uint32_t shape(uint32_t i) const { return v.shape[i]; }
};

// Accessor over the ShapeView SoA in global memory (read-only path).
struct GlobalShapes {
    dyph_shapes v;
    __device__ __forceinline__ uint32_t type(uint32_t s) const { return __ldg(v.type + s); }
    __device__ __forceinline__ float hx(uint32_t s) const { return __ldg(v.half_x + s); }
    __device__ __forceinline__ float hy(uint32_t s) const { return __ldg(v.half_y + s); }
    __device__ __forceinline__ float hz(uint32_t s) const { return __ldg(v.half_z + s); }
};

// One contact record (ContactView row).
struct Contact {
    uint32_t a, b;
    float px, py, pz, nx, ny, nz, depth;
};

// ── integrate one body for one substep (core/src/integrator.cpp:18-68) ──────
struct Pose {
    float px, py, pz, qw, qx, qy, qz, vx, vy, vz;
};

__device__ __forceinline__ void integrate_body(Pose& s, float ox, float oy, float oz, float gx, float gy,
                                               float gz, float sub_dt, float half_dt) {
    float vx = s.vx + gx * sub_dt;
    float vy = s.vy + gy * sub_dt;
    float vz = s.vz + gz * sub_dt;
    s.vx = vx; s.vy = vy; s.vz = vz;
    s.px += vx * sub_dt;
    s.py += vy * sub_dt;
    s.pz += vz * sub_dt;
    float qw = s.qw, qx = s.qx, qy = s.qy, qz = s.qz;
    const float dpw = -(ox * qx + oy * qy + oz * qz);
    const float dpx = (ox * qw + oy * qz - oz * qy);
    const float dpy = (oy * qw + oz * qx - ox * qz);
    const float dpz = (oz * qw + ox * qy - oy * qx);
    qw += half_dt * dpw;
    qx += half_dt * dpx;
    qy += half_dt * dpy;
    qz += half_dt * dpz;
    const float inv_n = rsqrt_ieee(qw * qw + qx * qx + qy * qy + qz * qz);
    s.qw = qw * inv_n; s.qx = qx * inv_n; s.qy = qy * inv_n; s.qz = qz * inv_n;
}

// q * rsqrt(|q|^2) (core/src/xpbd_solver.cpp:579-584, 726-731).
__device__ __forceinline__ void renormalize(float& qw, float& qx, float& qy, float& qz) {
    float inv_len = rsqrt_ieee(qw * qw + qx * qx + qy * qy + qz * qz);
    qw = qw * inv_len; qx = qx * inv_len; qy = qy * inv_len; qz = qz * inv_len;
}

// ── Morton code (core/src/broadphase.cpp:21-33, 128-141) ────────────────────
__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v &= 0x000003ffu;
    v = (v | (v << 16u)) & 0xFF0000FFu;
    v = (v | (v << 8u)) & 0x0F00F00Fu;
    v = (v | (v << 4u)) & 0xC30C30C3u;
    v = (v | (v << 2u)) & 0x49249249u;
    return v;
}

__device__ __forceinline__ uint32_t morton_code(float px, float py, float pz, const dyph_aabb& b) {
    float tx = (px - b.min_x) / (b.max_x - b.min_x);
    float ty = (py - b.min_y) / (b.max_y - b.min_y);
    float tz = (pz - b.min_z) / (b.max_z - b.min_z);
    tx = tx < 0.f ? 0.f : (tx > 1.f ? 1.f : tx);
    ty = ty < 0.f ? 0.f : (ty > 1.f ? 1.f : ty);
    tz = tz < 0.f ? 0.f : (tz > 1.f ? 1.f : tz);
    uint32_t qx = static_cast<uint32_t>(tx * 1023.f);
    uint32_t qy = static_cast<uint32_t>(ty * 1023.f);
    uint32_t qz = static_cast<uint32_t>(tz * 1023.f);
    return expand_bits(qx) | (expand_bits(qy) << 1u) | (expand_bits(qz) << 2u);
}

// ── leaf box (core/src/broadphase.cpp:216-251), fp16 round-to-nearest-even ──
__device__ __forceinline__ uint4 leaf_box(uint32_t stype, float px, float py, float pz, float qw, float qx,
                                          float qy, float qz, float hx, float hy, float hz) {
    float mn_x, mn_y, mn_z, mx_x, mx_y, mx_z;
    if (stype == kShapeSphere) {
        mn_x = px - hx; mx_x = px + hx;
        mn_y = py - hx; mx_y = py + hx;
        mn_z = pz - hx; mx_z = pz + hx;
    } else {
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
        mn_x = px - ex; mx_x = px + ex;
        mn_y = py - ey; mx_y = py + ey;
        mn_z = pz - ez; mx_z = pz + ez;
    }
    uint4 r;
    r.x = static_cast<uint32_t>(f2h_bits(mn_x)) | (static_cast<uint32_t>(f2h_bits(mn_y)) << 16);
    r.y = static_cast<uint32_t>(f2h_bits(mn_z)) | (static_cast<uint32_t>(f2h_bits(mx_x)) << 16);
    r.z = static_cast<uint32_t>(f2h_bits(mx_y)) | (static_cast<uint32_t>(f2h_bits(mx_z)) << 16);
    r.w = 0u;  // pad0, pad1 = half(0)
    return r;
}

// Node box as six floats (exact fp16 -> fp32).
struct BoxF {
    float mnx, mny, mnz, mxx, mxy, mxz;
};
__device__ __forceinline__ BoxF unpack_box(uint4 r) {
    BoxF b;
    b.mnx = h2f_bits(static_cast<uint16_t>(r.x & 0xFFFFu));
    b.mny = h2f_bits(static_cast<uint16_t>(r.x >> 16));
    b.mnz = h2f_bits(static_cast<uint16_t>(r.y & 0xFFFFu));
    b.mxx = h2f_bits(static_cast<uint16_t>(r.y >> 16));
    b.mxy = h2f_bits(static_cast<uint16_t>(r.z & 0xFFFFu));
    b.mxz = h2f_bits(static_cast<uint16_t>(r.z >> 16));
    return b;
}
// Internal-node merge: fp16(min/max of the two children) — exact (broadphase.cpp:271-280).
__device__ __forceinline__ uint4 merge_box(uint4 a, uint4 b) {
    BoxF x = unpack_box(a), y = unpack_box(b);
    uint4 r;
    r.x = static_cast<uint32_t>(f2h_bits(fminf(x.mnx, y.mnx))) | (static_cast<uint32_t>(f2h_bits(fminf(x.mny, y.mny))) << 16);
    r.y = static_cast<uint32_t>(f2h_bits(fminf(x.mnz, y.mnz))) | (static_cast<uint32_t>(f2h_bits(fmaxf(x.mxx, y.mxx))) << 16);
    r.z = static_cast<uint32_t>(f2h_bits(fmaxf(x.mxy, y.mxy))) | (static_cast<uint32_t>(f2h_bits(fmaxf(x.mxz, y.mxz))) << 16);
    r.w = 0u;
    return r;
}
// Inclusive overlap test of the traversal (broadphase.cpp:322-325).
__device__ __forceinline__ bool box_overlap(const BoxF& n, const BoxF& q) {
    return !(n.mnx > q.mxx || n.mxx < q.mnx || n.mny > q.mxy || n.mxy < q.mny || n.mnz > q.mxz ||
             n.mxz < q.mnz);
}

// ── narrowphase primitives (core/src/narrowphase.cpp) ───────────────────────

// make_axes (narrowphase.cpp:913-917): row k = body axis k in world space.
__device__ __forceinline__ void make_axes(float qw, float qx, float qy, float qz, float A[3][3]) {
    A[0][0] = 1.f - 2.f * (qy * qy + qz * qz); A[0][1] = 2.f * (qx * qy + qz * qw); A[0][2] = 2.f * (qx * qz - qy * qw);
    A[1][0] = 2.f * (qx * qy - qz * qw); A[1][1] = 1.f - 2.f * (qx * qx + qz * qz); A[1][2] = 2.f * (qy * qz + qx * qw);
    A[2][0] = 2.f * (qx * qz + qy * qw); A[2][1] = 2.f * (qy * qz - qx * qw); A[2][2] = 1.f - 2.f * (qx * qx + qy * qy);
}

// sphere_sphere (narrowphase.cpp:46-68).
// `br` (optional) receives the branch taken: bit 0 set when the centres
// coincide (dist < 1e-8, fixed normal).
__device__ __forceinline__ bool sphere_sphere(float acx, float acy, float acz, float ra, float bcx, float bcy,
                                              float bcz, float rb, Contact& c, uint32_t* br = nullptr) {
    float dx = acx - bcx, dy = acy - bcy, dz = acz - bcz;
    float dist2 = dx * dx + dy * dy + dz * dz;
    float sum_r = ra + rb;
    if (dist2 >= sum_r * sum_r) return false;
    float dist = __fsqrt_rn(dist2);
    if (br) *br = dist < 1e-8f ? 1u : 0u;
    if (dist < 1e-8f) { c.nx = 0.f; c.ny = 1.f; c.nz = 0.f; }
    else { float inv = __fdiv_rn(1.f, dist); c.nx = dx * inv; c.ny = dy * inv; c.nz = dz * inv; }
    c.depth = sum_r - dist;
    float sa = acx - c.nx * ra, sb = bcx + c.nx * rb;
    c.px = 0.5f * (sa + sb);
    sa = acy - c.ny * ra; sb = bcy + c.ny * rb; c.py = 0.5f * (sa + sb);
    sa = acz - c.nz * ra; sb = bcz + c.nz * rb; c.pz = 0.5f * (sa + sb);
    return true;
}

// sphere_box (narrowphase.cpp:71-127); E rows are the box axes. `br`
// (optional) receives the branch taken: bit 0 centre inside the box, then
// bits 1-2 the face axis and bit 3 its sign (s < 0); outside, bits 4 + 2k /
// 5 + 2k mark local coordinate k clamped to -h_k / +h_k.
__device__ __forceinline__ bool sphere_box(float scx, float scy, float scz, float sr, float bcx, float bcy,
                                           float bcz, const float E[3][3], float bh0, float bh1, float bh2,
                                           Contact& c, uint32_t* br = nullptr) {
    const float e0x = E[0][0], e0y = E[0][1], e0z = E[0][2];
    const float e1x = E[1][0], e1y = E[1][1], e1z = E[1][2];
    const float e2x = E[2][0], e2y = E[2][1], e2z = E[2][2];
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
            c.nx = -(s * e0x); c.ny = -(s * e0y); c.nz = -(s * e0z);
            c.depth = sr + pen0;
            if (br) *br = 1u | (0u << 1) | (s < 0.f ? 8u : 0u);
        } else if (pen1 <= pen2) {
            float s = q1 >= 0.f ? 1.f : -1.f;
            c.nx = -(s * e1x); c.ny = -(s * e1y); c.nz = -(s * e1z);
            c.depth = sr + pen1;
            if (br) *br = 1u | (1u << 1) | (s < 0.f ? 8u : 0u);
        } else {
            float s = q2 >= 0.f ? 1.f : -1.f;
            c.nx = -(s * e2x); c.ny = -(s * e2y); c.nz = -(s * e2z);
            c.depth = sr + pen2;
            if (br) *br = 1u | (2u << 1) | (s < 0.f ? 8u : 0u);
        }
        c.px = scx - c.nx * sr; c.py = scy - c.ny * sr; c.pz = scz - c.nz * sr;
        return true;
    }
    if (dist2 >= sr * sr) return false;
    if (br)
        *br = (q0 < -bh0 ? 16u : 0u) | (q0 > bh0 ? 32u : 0u) | (q1 < -bh1 ? 64u : 0u) | (q1 > bh1 ? 128u : 0u) |
              (q2 < -bh2 ? 256u : 0u) | (q2 > bh2 ? 512u : 0u);
    float dist = __fsqrt_rn(dist2);
    float inv_d = __fdiv_rn(1.f, dist);
    float wx = lx * e0x + ly * e1x + lz * e2x;
    float wy = lx * e0y + ly * e1y + lz * e2y;
    float wz = lx * e0z + ly * e1z + lz * e2z;
    c.nx = -wx * inv_d; c.ny = -wy * inv_d; c.nz = -wz * inv_d;
    c.depth = sr - dist;
    c.px = bcx + c0 * e0x + c1 * e1x + c2 * e2x;
    c.py = bcy + c0 * e0y + c1 * e1y + c2 * e2y;
    c.pz = bcz + c0 * e0z + c1 * e1z + c2 * e2z;
    return true;
}

// One SAT axis: the SAT_TEST macro (narrowphase.cpp:158-175) and the edge
// block (:192-208) evaluate the same expressions.
struct SatBest {
    float ov;
    int type, i, j;
    float nx, ny, nz;
};
__device__ __forceinline__ bool sat_axis(float lx, float ly, float lz, const float Ae[3][3], const float Ah[3],
                                         const float Be[3][3], const float Bh[3], float dx, float dy, float dz,
                                         int type, int i, int j, SatBest& best) {
    float rA = Ah[0] * fabsf(lx * Ae[0][0] + ly * Ae[0][1] + lz * Ae[0][2]) +
               Ah[1] * fabsf(lx * Ae[1][0] + ly * Ae[1][1] + lz * Ae[1][2]) +
               Ah[2] * fabsf(lx * Ae[2][0] + ly * Ae[2][1] + lz * Ae[2][2]);
    float rB = Bh[0] * fabsf(lx * Be[0][0] + ly * Be[0][1] + lz * Be[0][2]) +
               Bh[1] * fabsf(lx * Be[1][0] + ly * Be[1][1] + lz * Be[1][2]) +
               Bh[2] * fabsf(lx * Be[2][0] + ly * Be[2][1] + lz * Be[2][2]);
    float t = fabsf(dx * lx + dy * ly + dz * lz);
    float ov = rA + rB - t;
    if (ov <= 0.f) return false;
    if (ov < best.ov) {
        best.ov = ov;
        best.type = type; best.i = i; best.j = j;
        float sgn = (dx * lx + dy * ly + dz * lz) >= 0.f ? -1.f : 1.f;
        best.nx = sgn * lx; best.ny = sgn * ly; best.nz = sgn * lz;
    }
    return true;
}

}  // namespace dyph
