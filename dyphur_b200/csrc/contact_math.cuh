// Box–box SAT, pair dispatch and the XPBD contact solve (device code).
#pragma once

#include "physics.cuh"

namespace dyph {

// Branch word of a box-box contact (filled when box_box_centroid gets `br`):
//   bits 0-1  SAT axis type (0 face of A, 1 face of B, 2 edge pair)
//   bits 2-3  axis i, bits 4-5 axis j (edge pair)
//   bit  7    reference face on B (face case; after the larger-face switch)
//   bits 8-9  reference face axis
//   bits 10-17 incident vertices kept (face case)
//   bits 18-21 edge-point signs s0A, s1A, s0B, s1B negative (edge case)
//   bit  22   edge case with |1 - b12^2| > 1e-6 (closest-point parameters solved)
constexpr uint32_t kBrRefB = 1u << 7;
constexpr uint32_t kBrDenom = 1u << 22;

// box_box (core/src/narrowphase.cpp:130-306) followed by the centroid
// reduction of process_pair (:991-998). Returns false for no contact.
__device__ __forceinline__ bool box_box_centroid(float acx, float acy, float acz, const float Ae[3][3],
                                                 const float Ah[3], float bcx, float bcy, float bcz,
                                                 const float Be[3][3], const float Bh[3], Contact& out,
                                                 uint32_t* br = nullptr) {
    const float eps_par = 1e-5f;
    float C[3][3];
    float dx = bcx - acx, dy = bcy - acy, dz = bcz - acz;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) C[i][j] = Ae[i][0] * Be[j][0] + Ae[i][1] * Be[j][1] + Ae[i][2] * Be[j][2];
    SatBest best{1e30f, -1, 0, 0, 0.f, 1.f, 0.f};
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (!sat_axis(Ae[i][0], Ae[i][1], Ae[i][2], Ae, Ah, Be, Bh, dx, dy, dz, 0, i, 0, best)) return false;
#pragma unroll
    for (int i = 0; i < 3; ++i)
        if (!sat_axis(Be[i][0], Be[i][1], Be[i][2], Ae, Ah, Be, Bh, dx, dy, dz, 1, i, 0, best)) return false;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float cx = Ae[i][1] * Be[j][2] - Ae[i][2] * Be[j][1];
            float cy = Ae[i][2] * Be[j][0] - Ae[i][0] * Be[j][2];
            float cz = Ae[i][0] * Be[j][1] - Ae[i][1] * Be[j][0];
            float len2 = cx * cx + cy * cy + cz * cz;
            if (len2 < eps_par * eps_par) continue;
            float inv_l = rsqrt_ieee(len2);
            if (!sat_axis(cx * inv_l, cy * inv_l, cz * inv_l, Ae, Ah, Be, Bh, dx, dy, dz, 2, i, j, best))
                return false;
        }
    }
    const float bnx = best.nx, bny = best.ny, bnz = best.nz;
    float sx_acc = 0.f, sy_acc = 0.f, sz_acc = 0.f, sd_acc = 0.f;
    int n_out = 0;
    int best_type = best.type, best_i = best.i;
    uint32_t word = static_cast<uint32_t>(best.type) | (static_cast<uint32_t>(best.i) << 2) |
                    (static_cast<uint32_t>(best.j) << 4);
    if (best_type == 0 || best_type == 1) {
        if (best_type == 0) {
            int t0A = (best_i + 1) % 3, t1A = (best_i + 2) % 3;
            int j_best = 0;
            for (int j = 1; j < 3; ++j)
                if (fabsf(C[best_i][j]) > fabsf(C[best_i][j_best])) j_best = j;
            int t0B = (j_best + 1) % 3, t1B = (j_best + 2) % 3;
            if (Bh[t0B] * Bh[t1B] > Ah[t0A] * Ah[t1A]) { best_type = 1; best_i = j_best; }
        }
        const bool a_is_ref = (best_type == 0);
        const int ref_ax = best_i;
        word |= (a_is_ref ? 0u : kBrRefB) | (static_cast<uint32_t>(ref_ax) << 8);
        const float rcx = a_is_ref ? acx : bcx, rcy = a_is_ref ? acy : bcy, rcz = a_is_ref ? acz : bcz;
        float Re[3][3], Ie[3][3], Rh[3], Ih[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                Re[r][q] = a_is_ref ? Ae[r][q] : Be[r][q];
                Ie[r][q] = a_is_ref ? Be[r][q] : Ae[r][q];
            }
            Rh[r] = a_is_ref ? Ah[r] : Bh[r];
            Ih[r] = a_is_ref ? Bh[r] : Ah[r];
        }
        const float icx = a_is_ref ? bcx : acx, icy = a_is_ref ? bcy : acy, icz = a_is_ref ? bcz : acz;
        const int t0 = (ref_ax + 1) % 3, t1 = (ref_ax + 2) % 3;
        const float rc_dot_n3 = rcx * bnx + rcy * bny + rcz * bnz;
        const float sign_depth = a_is_ref ? 1.f : -1.f;
        float Rh_ref = Rh[0], Rh_t0 = Rh[1], Rh_t1 = Rh[2];
        if (ref_ax == 1) { Rh_ref = Rh[1]; Rh_t0 = Rh[2]; Rh_t1 = Rh[0]; }
        if (ref_ax == 2) { Rh_ref = Rh[2]; Rh_t0 = Rh[0]; Rh_t1 = Rh[1]; }
        float Rt0[3], Rt1[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            Rt0[q] = (t0 == 0) ? Re[0][q] : (t0 == 1 ? Re[1][q] : Re[2][q]);
            Rt1[q] = (t1 == 0) ? Re[0][q] : (t1 == 1 ? Re[1][q] : Re[2][q]);
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float sx = (k & 1) ? 1.f : -1.f, sy = (k & 2) ? 1.f : -1.f, sz = (k & 4) ? 1.f : -1.f;
            float vx = icx + sx * Ih[0] * Ie[0][0] + sy * Ih[1] * Ie[1][0] + sz * Ih[2] * Ie[2][0];
            float vy = icy + sx * Ih[0] * Ie[0][1] + sy * Ih[1] * Ie[1][1] + sz * Ih[2] * Ie[2][1];
            float vz = icz + sx * Ih[0] * Ie[0][2] + sy * Ih[1] * Ie[1][2] + sz * Ih[2] * Ie[2][2];
            float v_dot_n = vx * bnx + vy * bny + vz * bnz;
            float dv = Rh_ref + sign_depth * (v_dot_n - rc_dot_n3);
            if (dv <= 0.f) continue;
            float vx_rel = vx - rcx, vy_rel = vy - rcy, vz_rel = vz - rcz;
            float qt0 = vx_rel * Rt0[0] + vy_rel * Rt0[1] + vz_rel * Rt0[2];
            float qt1 = vx_rel * Rt1[0] + vy_rel * Rt1[1] + vz_rel * Rt1[2];
            if (fabsf(qt0) > Rh_t0 + 1e-3f) continue;
            if (fabsf(qt1) > Rh_t1 + 1e-3f) continue;
            if (n_out < 4) {
                word |= 1u << (10 + k);
                // centroid accumulation in the reference's order (cx += opx[k] ...)
                sx_acc += vx - sign_depth * dv * bnx;
                sy_acc += vy - sign_depth * dv * bny;
                sz_acc += vz - sign_depth * dv * bnz;
                sd_acc += dv;
                ++n_out;
            }
        }
    } else {
        const int i = best.i, j = best.j;
        const int t0A = (i + 1) % 3, t1A = (i + 2) % 3;
        const float s0A = (-bnx * Ae[t0A][0] - bny * Ae[t0A][1] - bnz * Ae[t0A][2]) >= 0.f ? 1.f : -1.f;
        const float s1A = (-bnx * Ae[t1A][0] - bny * Ae[t1A][1] - bnz * Ae[t1A][2]) >= 0.f ? 1.f : -1.f;
        float pAx = acx + s0A * Ah[t0A] * Ae[t0A][0] + s1A * Ah[t1A] * Ae[t1A][0];
        float pAy = acy + s0A * Ah[t0A] * Ae[t0A][1] + s1A * Ah[t1A] * Ae[t1A][1];
        float pAz = acz + s0A * Ah[t0A] * Ae[t0A][2] + s1A * Ah[t1A] * Ae[t1A][2];
        const int t0B = (j + 1) % 3, t1B = (j + 2) % 3;
        const float s0B = (bnx * Be[t0B][0] + bny * Be[t0B][1] + bnz * Be[t0B][2]) >= 0.f ? 1.f : -1.f;
        const float s1B = (bnx * Be[t1B][0] + bny * Be[t1B][1] + bnz * Be[t1B][2]) >= 0.f ? 1.f : -1.f;
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
        word |= (s0A < 0.f ? 1u << 18 : 0u) | (s1A < 0.f ? 1u << 19 : 0u) | (s0B < 0.f ? 1u << 20 : 0u) |
                (s1B < 0.f ? 1u << 21 : 0u) | (fabsf(denom) > 1e-6f ? kBrDenom : 0u);
        if (fabsf(denom) > 1e-6f) {
            s_t = __fdiv_rn(b12 * d2 - d1, denom);
            t_t = __fdiv_rn(d2 - b12 * d1, denom);
        }
        float qAx = pAx + s_t * uAx, qAy = pAy + s_t * uAy, qAz = pAz + s_t * uAz;
        float qBx = pBx + t_t * uBx, qBy = pBy + t_t * uBy, qBz = pBz + t_t * uBz;
        sx_acc = 0.f + 0.5f * (qAx + qBx);
        sy_acc = 0.f + 0.5f * (qAy + qBy);
        sz_acc = 0.f + 0.5f * (qAz + qBz);
        sd_acc = 0.f + best.ov;
        n_out = 1;
    }
    if (n_out == 0) return false;
    if (br) *br = word;
    float inv = __fdiv_rn(1.f, static_cast<float>(n_out));
    out.px = sx_acc * inv; out.py = sy_acc * inv; out.pz = sz_acc * inv;
    out.nx = bnx; out.ny = bny; out.nz = bnz;
    out.depth = sd_acc * inv;
    return true;
}

// process_pair for box / sphere shapes (narrowphase.cpp:920-1001).
// Returns true and fills `c` when the pair is in contact.
template <class Bodies, class Shapes>
__device__ __forceinline__ bool process_pair(const Bodies& B, const Shapes& S, uint32_t ia, uint32_t ib, Contact& c,
                                             uint32_t* br = nullptr) {
    const uint32_t sha = B.shape(ia), shb = B.shape(ib);
    const uint32_t ta = S.type(sha), tb = S.type(shb);
    c.a = ia; c.b = ib;
    if (ta == kShapeSphere && tb == kShapeSphere)
        return sphere_sphere(B.px(ia), B.py(ia), B.pz(ia), S.hx(sha), B.px(ib), B.py(ib), B.pz(ib), S.hx(shb), c, br);
    if (ta == kShapeSphere && tb == kShapeBox) {
        float Be[3][3];
        make_axes(B.qw(ib), B.qx(ib), B.qy(ib), B.qz(ib), Be);
        if (!sphere_box(B.px(ia), B.py(ia), B.pz(ia), S.hx(sha), B.px(ib), B.py(ib), B.pz(ib), Be, S.hx(shb),
                        S.hy(shb), S.hz(shb), c, br))
            return false;
        c.nx = -c.nx; c.ny = -c.ny; c.nz = -c.nz;
        return true;
    }
    if (ta == kShapeBox && tb == kShapeSphere) {
        float Ae[3][3];
        make_axes(B.qw(ia), B.qx(ia), B.qy(ia), B.qz(ia), Ae);
        return sphere_box(B.px(ib), B.py(ib), B.pz(ib), S.hx(shb), B.px(ia), B.py(ia), B.pz(ia), Ae, S.hx(sha),
                          S.hy(sha), S.hz(sha), c, br);
    }
    if (ta == kShapeBox && tb == kShapeBox) {
        float Ae[3][3], Be[3][3];
        const float Ah[3] = {S.hx(sha), S.hy(sha), S.hz(sha)};
        const float Bh[3] = {S.hx(shb), S.hy(shb), S.hz(shb)};
        make_axes(B.qw(ia), B.qx(ia), B.qy(ia), B.qz(ia), Ae);
        make_axes(B.qw(ib), B.qx(ib), B.qy(ib), B.qz(ib), Be);
        return box_box_centroid(B.px(ia), B.py(ia), B.pz(ia), Ae, Ah, B.px(ib), B.py(ib), B.pz(ib), Be, Bh, c, br);
    }
    return false;  // convex hulls / meshes are not on this path
}

// ── XPBD contact solve (core/src/xpbd_solver.cpp:40-133, 413-521) ──────────

template <class Bodies>
__device__ __forceinline__ void world_inv_inertia(const Bodies& B, uint32_t bi, float vx, float vy, float vz,
                                                  float& ox, float& oy, float& oz) {
    const float qw = B.qw(bi), qx = B.qx(bi), qy = B.qy(bi), qz = B.qz(bi);
    const float R00 = 1.f - 2.f * (qy * qy + qz * qz), R01 = 2.f * (qx * qy + qz * qw), R02 = 2.f * (qx * qz - qy * qw);
    const float R10 = 2.f * (qx * qy - qz * qw), R11 = 1.f - 2.f * (qx * qx + qz * qz), R12 = 2.f * (qy * qz + qx * qw);
    const float R20 = 2.f * (qx * qz + qy * qw), R21 = 2.f * (qy * qz - qx * qw), R22 = 1.f - 2.f * (qx * qx + qy * qy);
    const float lx = R00 * vx + R10 * vy + R20 * vz;
    const float ly = R01 * vx + R11 * vy + R21 * vz;
    const float lz = R02 * vx + R12 * vy + R22 * vz;
    const float ixx = B.ixx(bi), iyy = B.iyy(bi), izz = B.izz(bi);
    const float ixy = B.ixy(bi), ixz = B.ixz(bi), iyz = B.iyz(bi);
    const float ilx = ixx * lx + ixy * ly + ixz * lz;
    const float ily = ixy * lx + iyy * ly + iyz * lz;
    const float ilz = ixz * lx + iyz * ly + izz * lz;
    ox = R00 * ilx + R01 * ily + R02 * ilz;
    oy = R10 * ilx + R11 * ily + R12 * ilz;
    oz = R20 * ilx + R21 * ily + R22 * ilz;
}

template <class Bodies>
__device__ __forceinline__ void apply_ang_delta(const Bodies& B, uint32_t bi, float ax, float ay, float az) {
    if (B.im(bi) == 0.f) return;
    const float qw = B.qw(bi), qx = B.qx(bi), qy = B.qy(bi), qz = B.qz(bi);
    B.qw(bi) += 0.5f * (-ax * qx - ay * qy - az * qz);
    B.qx(bi) += 0.5f * (ax * qw + ay * qz - az * qy);
    B.qy(bi) += 0.5f * (-ax * qz + ay * qw + az * qx);
    B.qz(bi) += 0.5f * (ax * qy - ay * qx + az * qw);
}

// Result codes of one contact solve.
constexpr int kSolveSkipped = 0;   // depth <= 0 or already resolved
constexpr int kSolveDone = 1;      // correction applied
constexpr int kSolveDeferred = 2;  // w_total < 1e-10: lambda untouched, retried next iteration

// Branch flags of one contact solve (solve_contact's optional `flags`).
constexpr uint32_t kSfActive = 1u;     // position correction applied
constexpr uint32_t kSfNormal = 2u;     // normal velocity impulse (vrel_n < 0)
constexpr uint32_t kSfFriction = 4u;   // friction impulse applied
constexpr uint32_t kSfClamped = 8u;    // friction impulse clamped to mu * j_n_static

template <class Bodies>
__device__ __forceinline__ int solve_contact(const Bodies& B, const Contact& ct, float mu, float& lc, float dt,
                                             uint32_t* flags = nullptr) {
    const uint32_t ia = ct.a, ib = ct.b;
    const float depth = ct.depth;
    if (depth <= 0.f) return kSolveSkipped;
    const float remaining = depth - lc;
    if (remaining <= 1e-6f) return kSolveSkipped;
    const float nx = ct.nx, ny = ct.ny, nz = ct.nz;
    const float px = ct.px, py = ct.py, pz = ct.pz;
    const float wa = B.im(ia), wb = B.im(ib);
    const float rax = px - B.px(ia), ray = py - B.py(ia), raz = pz - B.pz(ia);
    const float rbx = px - B.px(ib), rby = py - B.py(ib), rbz = pz - B.pz(ib);
    const float raxnx = ray * nz - raz * ny, raxny = raz * nx - rax * nz, raxnz = rax * ny - ray * nx;
    const float rbxnx = rby * nz - rbz * ny, rbxny = rbz * nx - rbx * nz, rbxnz = rbx * ny - rby * nx;
    float iIa_x, iIa_y, iIa_z, iIb_x, iIb_y, iIb_z;
    world_inv_inertia(B, ia, raxnx, raxny, raxnz, iIa_x, iIa_y, iIa_z);
    world_inv_inertia(B, ib, rbxnx, rbxny, rbxnz, iIb_x, iIb_y, iIb_z);
    const float wa_ang = raxnx * iIa_x + raxny * iIa_y + raxnz * iIa_z;
    const float wb_ang = rbxnx * iIb_x + rbxny * iIb_y + rbxnz * iIb_z;
    const float w_total = wa + wb + wa_ang + wb_ang;
    if (w_total < 1e-10f) return kSolveDeferred;
    const float dl = __fdiv_rn(remaining, w_total);
    lc += remaining;
    if (flags) *flags = kSfActive;
    if (wa != 0.f) { B.px(ia) += wa * dl * nx; B.py(ia) += wa * dl * ny; B.pz(ia) += wa * dl * nz; }
    if (wb != 0.f) { B.px(ib) -= wb * dl * nx; B.py(ib) -= wb * dl * ny; B.pz(ib) -= wb * dl * nz; }
    apply_ang_delta(B, ia, dl * iIa_x, dl * iIa_y, dl * iIa_z);
    apply_ang_delta(B, ib, -dl * iIb_x, -dl * iIb_y, -dl * iIb_z);
    {
        const float oax = B.wx(ia), oay = B.wy(ia), oaz = B.wz(ia);
        const float obx = B.wx(ib), oby = B.wy(ib), obz = B.wz(ib);
        const float vcax = B.vx(ia) + oay * raz - oaz * ray;
        const float vcay = B.vy(ia) + oaz * rax - oax * raz;
        const float vcaz = B.vz(ia) + oax * ray - oay * rax;
        const float vcbx = B.vx(ib) + oby * rbz - obz * rby;
        const float vcby = B.vy(ib) + obz * rbx - obx * rbz;
        const float vcbz = B.vz(ib) + obx * rby - oby * rbx;
        const float vrel_x = vcax - vcbx, vrel_y = vcay - vcby, vrel_z = vcaz - vcbz;
        const float vrel_n = vrel_x * nx + vrel_y * ny + vrel_z * nz;
        if (vrel_n < 0.f) {
            if (flags) *flags |= kSfNormal;
            const float j_n = __fdiv_rn(-vrel_n, w_total);
            float doa_x, doa_y, doa_z, dob_x, dob_y, dob_z;
            world_inv_inertia(B, ia, raxnx, raxny, raxnz, doa_x, doa_y, doa_z);
            world_inv_inertia(B, ib, rbxnx, rbxny, rbxnz, dob_x, dob_y, dob_z);
            if (wa != 0.f) {
                B.vx(ia) += wa * j_n * nx; B.vy(ia) += wa * j_n * ny; B.vz(ia) += wa * j_n * nz;
                B.wx(ia) += j_n * doa_x; B.wy(ia) += j_n * doa_y; B.wz(ia) += j_n * doa_z;
            }
            if (wb != 0.f) {
                B.vx(ib) -= wb * j_n * nx; B.vy(ib) -= wb * j_n * ny; B.vz(ib) -= wb * j_n * nz;
                B.wx(ib) -= j_n * dob_x; B.wy(ib) -= j_n * dob_y; B.wz(ib) -= j_n * dob_z;
            }
        }
    }
    if (mu > 0.f) {
        const float oax2 = B.wx(ia), oay2 = B.wy(ia), oaz2 = B.wz(ia);
        const float obx2 = B.wx(ib), oby2 = B.wy(ib), obz2 = B.wz(ib);
        const float vcax2 = B.vx(ia) + oay2 * raz - oaz2 * ray;
        const float vcay2 = B.vy(ia) + oaz2 * rax - oax2 * raz;
        const float vcaz2 = B.vz(ia) + oax2 * ray - oay2 * rax;
        const float vcbx2 = B.vx(ib) + oby2 * rbz - obz2 * rby;
        const float vcby2 = B.vy(ib) + obz2 * rbx - obx2 * rbz;
        const float vcbz2 = B.vz(ib) + obx2 * rby - oby2 * rbx;
        const float rvx = vcax2 - vcbx2, rvy = vcay2 - vcby2, rvz = vcaz2 - vcbz2;
        const float rvn = rvx * nx + rvy * ny + rvz * nz;
        const float vt_x = rvx - rvn * nx, vt_y = rvy - rvn * ny, vt_z = rvz - rvn * nz;
        const float vt2 = vt_x * vt_x + vt_y * vt_y + vt_z * vt_z;
        if (vt2 > 1e-12f) {
            const float vt_len = __fsqrt_rn(vt2);
            const float tx = __fdiv_rn(vt_x, vt_len), ty = __fdiv_rn(vt_y, vt_len), tz = __fdiv_rn(vt_z, vt_len);
            const float ratx = ray * tz - raz * ty, raty = raz * tx - rax * tz, ratz = rax * ty - ray * tx;
            const float rbtx = rby * tz - rbz * ty, rbty = rbz * tx - rbx * tz, rbtz = rbx * ty - rby * tx;
            float fIa_x, fIa_y, fIa_z, fIb_x, fIb_y, fIb_z;
            world_inv_inertia(B, ia, ratx, raty, ratz, fIa_x, fIa_y, fIa_z);
            world_inv_inertia(B, ib, rbtx, rbty, rbtz, fIb_x, fIb_y, fIb_z);
            const float wt = wa + wb + ratx * fIa_x + raty * fIa_y + ratz * fIa_z + rbtx * fIb_x + rbty * fIb_y +
                             rbtz * fIb_z;
            if (wt > 1e-10f) {
                const float j_n_static = __fdiv_rn(lc, dt * w_total);
                float j_t = __fdiv_rn(vt_len, wt);
                if (flags) *flags |= kSfFriction | (mu * j_n_static < j_t ? kSfClamped : 0u);
                j_t = fminf(j_t, mu * j_n_static);
                if (wa != 0.f) {
                    B.vx(ia) -= wa * j_t * tx; B.vy(ia) -= wa * j_t * ty; B.vz(ia) -= wa * j_t * tz;
                    B.wx(ia) -= j_t * fIa_x; B.wy(ia) -= j_t * fIa_y; B.wz(ia) -= j_t * fIa_z;
                }
                if (wb != 0.f) {
                    B.vx(ib) += wb * j_t * tx; B.vy(ib) += wb * j_t * ty; B.vz(ib) += wb * j_t * tz;
                    B.wx(ib) += j_t * fIb_x; B.wy(ib) += j_t * fIb_y; B.wz(ib) += j_t * fIb_z;
                }
            }
        }
    }
    return kSolveDone;
}

}  // namespace dyph

namespace dyph {

// The two bodies of one contact held in registers (index 0 = body a, 1 = body
// b), so solve_contact's read-modify-writes stay on chip; only the 13 state
// floats of a dynamic body are written back.
struct LocalPair {
    float p[2][3], q[2][4], v[2][3], w[2][3], m[2], I[2][6];
    __device__ __forceinline__ float& px(uint32_t i) { return p[i][0]; }
    __device__ __forceinline__ float& py(uint32_t i) { return p[i][1]; }
    __device__ __forceinline__ float& pz(uint32_t i) { return p[i][2]; }
    __device__ __forceinline__ float& qw(uint32_t i) { return q[i][0]; }
    __device__ __forceinline__ float& qx(uint32_t i) { return q[i][1]; }
    __device__ __forceinline__ float& qy(uint32_t i) { return q[i][2]; }
    __device__ __forceinline__ float& qz(uint32_t i) { return q[i][3]; }
    __device__ __forceinline__ float& vx(uint32_t i) { return v[i][0]; }
    __device__ __forceinline__ float& vy(uint32_t i) { return v[i][1]; }
    __device__ __forceinline__ float& vz(uint32_t i) { return v[i][2]; }
    __device__ __forceinline__ float& wx(uint32_t i) { return w[i][0]; }
    __device__ __forceinline__ float& wy(uint32_t i) { return w[i][1]; }
    __device__ __forceinline__ float& wz(uint32_t i) { return w[i][2]; }
    __device__ __forceinline__ float im(uint32_t i) const { return m[i]; }
    __device__ __forceinline__ float ixx(uint32_t i) const { return I[i][0]; }
    __device__ __forceinline__ float iyy(uint32_t i) const { return I[i][1]; }
    __device__ __forceinline__ float izz(uint32_t i) const { return I[i][2]; }
    __device__ __forceinline__ float ixy(uint32_t i) const { return I[i][3]; }
    __device__ __forceinline__ float ixz(uint32_t i) const { return I[i][4]; }
    __device__ __forceinline__ float iyz(uint32_t i) const { return I[i][5]; }
};

// LocalPair's accessors are non-const; solve_contact takes `const Bodies&`,
// so it is driven through this thin reference wrapper.
struct LocalPairRef {
    LocalPair* s;
    __device__ __forceinline__ float& px(uint32_t i) const { return s->p[i][0]; }
    __device__ __forceinline__ float& py(uint32_t i) const { return s->p[i][1]; }
    __device__ __forceinline__ float& pz(uint32_t i) const { return s->p[i][2]; }
    __device__ __forceinline__ float& qw(uint32_t i) const { return s->q[i][0]; }
    __device__ __forceinline__ float& qx(uint32_t i) const { return s->q[i][1]; }
    __device__ __forceinline__ float& qy(uint32_t i) const { return s->q[i][2]; }
    __device__ __forceinline__ float& qz(uint32_t i) const { return s->q[i][3]; }
    __device__ __forceinline__ float& vx(uint32_t i) const { return s->v[i][0]; }
    __device__ __forceinline__ float& vy(uint32_t i) const { return s->v[i][1]; }
    __device__ __forceinline__ float& vz(uint32_t i) const { return s->v[i][2]; }
    __device__ __forceinline__ float& wx(uint32_t i) const { return s->w[i][0]; }
    __device__ __forceinline__ float& wy(uint32_t i) const { return s->w[i][1]; }
    __device__ __forceinline__ float& wz(uint32_t i) const { return s->w[i][2]; }
    __device__ __forceinline__ float im(uint32_t i) const { return s->m[i]; }
    __device__ __forceinline__ float ixx(uint32_t i) const { return s->I[i][0]; }
    __device__ __forceinline__ float iyy(uint32_t i) const { return s->I[i][1]; }
    __device__ __forceinline__ float izz(uint32_t i) const { return s->I[i][2]; }
    __device__ __forceinline__ float ixy(uint32_t i) const { return s->I[i][3]; }
    __device__ __forceinline__ float ixz(uint32_t i) const { return s->I[i][4]; }
    __device__ __forceinline__ float iyz(uint32_t i) const { return s->I[i][5]; }
};

__device__ __forceinline__ void load_local(const GlobalBodies& B, uint32_t bi, LocalPair& L, int j) {
    L.p[j][0] = B.px(bi); L.p[j][1] = B.py(bi); L.p[j][2] = B.pz(bi);
    L.q[j][0] = B.qw(bi); L.q[j][1] = B.qx(bi); L.q[j][2] = B.qy(bi); L.q[j][3] = B.qz(bi);
    L.v[j][0] = B.vx(bi); L.v[j][1] = B.vy(bi); L.v[j][2] = B.vz(bi);
    L.w[j][0] = B.wx(bi); L.w[j][1] = B.wy(bi); L.w[j][2] = B.wz(bi);
    L.m[j] = B.im(bi);
    L.I[j][0] = B.ixx(bi); L.I[j][1] = B.iyy(bi); L.I[j][2] = B.izz(bi);
    L.I[j][3] = B.ixy(bi); L.I[j][4] = B.ixz(bi); L.I[j][5] = B.iyz(bi);
}

__device__ __forceinline__ void store_local(const GlobalBodies& B, uint32_t bi, const LocalPair& L, int j) {
    B.px(bi) = L.p[j][0]; B.py(bi) = L.p[j][1]; B.pz(bi) = L.p[j][2];
    B.qw(bi) = L.q[j][0]; B.qx(bi) = L.q[j][1]; B.qy(bi) = L.q[j][2]; B.qz(bi) = L.q[j][3];
    B.vx(bi) = L.v[j][0]; B.vy(bi) = L.v[j][1]; B.vz(bi) = L.v[j][2];
    B.wx(bi) = L.w[j][0]; B.wy(bi) = L.w[j][1]; B.wz(bi) = L.w[j][2];
}

// solve_contact on register copies of the two bodies: the same arithmetic in
// the same order, so the results are bit-identical to the global-memory form.
__device__ __forceinline__ int solve_contact_reg(const GlobalBodies& B, const Contact& ct, float mu, float& lc,
                                                 float dt) {
    if (ct.depth <= 0.f || ct.depth - lc <= 1e-6f) return kSolveSkipped;
    LocalPair L;
    load_local(B, ct.a, L, 0);
    load_local(B, ct.b, L, 1);
    Contact lct = ct;
    lct.a = 0u;
    lct.b = 1u;
    const int res = solve_contact(LocalPairRef{&L}, lct, mu, lc, dt);
    if (res == kSolveDone) {
        if (L.m[0] != 0.f) store_local(B, ct.a, L, 0);
        if (L.m[1] != 0.f) store_local(B, ct.b, L, 1);
    }
    return res;
}

}  // namespace dyph
