// Hand-written reverse-mode adjoints of the frame step's per-body, per-contact
// and per-pair primitives (device code of the adjoint's reverse kernel,
// reverse.cu).
//
// Each *_adj routine takes the primal inputs of one primitive, the branch it
// took in the forward pass (recorded there, so the adjoint differentiates the
// very piece the forward evaluated: the contact set and every branch are held
// fixed), and the adjoint of the primitive's outputs; it returns (adds) the
// adjoints of its inputs. Values the adjoint needs are recomputed from the
// primal inputs. The derivatives follow the primitives:
//   integrate_body          core/src/integrator.cpp:18-68
//   renormalize             core/src/xpbd_solver.cpp:579-584
//   sphere_sphere / sphere_box / box_box_centroid
//                           core/src/narrowphase.cpp:46-306, 991-998
//   solve_contact           core/src/xpbd_solver.cpp:40-133, 413-521
#pragma once

#include "contact_math.cuh"

namespace dyph {

struct F3 {
    float x, y, z;
};
__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ F3 operator+(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ F3 operator-(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 operator-(F3 a) { return F3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ F3 operator*(float s, F3 a) { return F3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ F3& operator+=(F3& a, F3 b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
__device__ __forceinline__ F3& operator-=(F3& a, F3 b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
// Sums of products with explicit fused multiply-adds. The reverse pass is
// compiled without contraction, so the compiler fuses nothing by itself and
// every team layout of a scene rounds alike; the fusions are written here,
// where most of the adjoint's arithmetic is.
__device__ __forceinline__ float fma2(float a0, float b0, float a1, float b1) {
    return __fmaf_rn(a1, b1, a0 * b0);
}
__device__ __forceinline__ float fma3(float a0, float b0, float a1, float b1, float a2, float b2) {
    return __fmaf_rn(a2, b2, __fmaf_rn(a1, b1, a0 * b0));
}
__device__ __forceinline__ float dot(F3 a, F3 b) { return fma3(a.x, b.x, a.y, b.y, a.z, b.z); }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
    return F3{__fmaf_rn(a.y, b.z, -(a.z * b.y)), __fmaf_rn(a.z, b.x, -(a.x * b.z)), __fmaf_rn(a.x, b.y, -(a.y * b.x))};
}
// a + s b, fused per component.
__device__ __forceinline__ F3 fmav(float s, F3 b, F3 a) {
    return F3{__fmaf_rn(s, b.x, a.x), __fmaf_rn(s, b.y, a.y), __fmaf_rn(s, b.z, a.z)};
}
__device__ __forceinline__ float fmav(float s, float b, float a) { return __fmaf_rn(s, b, a); }
// M^T v and M v for a 3x3 M.
__device__ __forceinline__ F3 mtv(const float M[3][3], F3 v) {
    return f3(fma3(M[0][0], v.x, M[1][0], v.y, M[2][0], v.z), fma3(M[0][1], v.x, M[1][1], v.y, M[2][1], v.z),
              fma3(M[0][2], v.x, M[1][2], v.y, M[2][2], v.z));
}
__device__ __forceinline__ F3 mv(const float M[3][3], F3 v) {
    return f3(fma3(M[0][0], v.x, M[0][1], v.y, M[0][2], v.z), fma3(M[1][0], v.x, M[1][1], v.y, M[1][2], v.z),
              fma3(M[2][0], v.x, M[2][1], v.y, M[2][2], v.z));
}
// I v for the symmetric inertia I6 = ixx, iyy, izz, ixy, ixz, iyz.
__device__ __forceinline__ F3 i6v(const float I6[6], F3 v) {
    return f3(fma3(I6[0], v.x, I6[3], v.y, I6[4], v.z), fma3(I6[3], v.x, I6[1], v.y, I6[5], v.z),
              fma3(I6[4], v.x, I6[5], v.y, I6[2], v.z));
}

// Adjoint of the rotation rows A(q) (make_axes; also the matrix of
// world_inv_inertia): q̄ += Σ_ij Ā_ij ∂A_ij/∂q.
__device__ __forceinline__ void rot_adj(const float q[4], const float Ab[3][3], float qb[4]) {
    const float w = q[0], x = q[1], y = q[2], z = q[3];
    // sums of the products, grouped by the quaternion component they multiply
    const float a01 = Ab[0][1] - Ab[1][0], a12 = Ab[1][2] - Ab[2][1], a20 = Ab[2][0] - Ab[0][2];
    const float s01 = Ab[0][1] + Ab[1][0], s12 = Ab[1][2] + Ab[2][1], s20 = Ab[2][0] + Ab[0][2];
    qb[0] += 2.f * fma3(z, a01, x, a12, y, a20);
    qb[1] += 2.f * fma3(y, s01, z, s20, w, a12) - 4.f * x * (Ab[1][1] + Ab[2][2]);
    qb[2] += 2.f * fma3(x, s01, z, s12, w, a20) - 4.f * y * (Ab[0][0] + Ab[2][2]);
    qb[3] += 2.f * fma3(w, a01, x, s20, y, s12) - 4.f * z * (Ab[0][0] + Ab[1][1]);
}

__device__ __forceinline__ void rot_rows(const float q[4], float A[3][3]) { make_axes(q[0], q[1], q[2], q[3], A); }

// y = R I R^T v (world_inv_inertia); I6 = ixx, iyy, izz, ixy, ixz, iyz.
__device__ __forceinline__ F3 winv(const float q[4], const float I6[6], F3 v) {
    float R[3][3];
    rot_rows(q, R);
    return mv(R, i6v(I6, mtv(R, v)));
}

// Adjoint of y = winv(q, I, v): v̄ += W ȳ (W symmetric), q̄ += ∂(W v)/∂q^T ȳ.
__device__ __forceinline__ void winv_adj(const float q[4], const float I6[6], F3 v, F3 yb, F3& vb, float qb[4]) {
    float R[3][3];
    rot_rows(q, R);
    const F3 il = i6v(I6, mtv(R, v));
    // y = R il: il̄ = R^T ȳ, R̄ += ȳ il^T; il = I l: l̄ = I il̄
    const F3 lb = i6v(I6, mtv(R, yb));
    // l = R^T v: v̄ += R l̄, R̄ += v l̄^T
    vb += mv(R, lb);
    const float yv[3] = {yb.x, yb.y, yb.z}, ilv[3] = {il.x, il.y, il.z};
    const float vv[3] = {v.x, v.y, v.z}, lbv[3] = {lb.x, lb.y, lb.z};
    float Rb[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Rb[i][j] = fma2(yv[i], ilv[j], vv[i], lbv[j]);
    rot_adj(q, Rb, qb);
}

// Adjoint of y = q / |q|: q̄ = r ȳ - r^3 (q·ȳ) q.
__device__ __forceinline__ void normalize_adj(const float q[4], const float yb[4], float qb[4]) {
    const float s = __fmaf_rn(q[3], q[3], fma3(q[0], q[0], q[1], q[1], q[2], q[2]));
    const float r = 1.f / sqrtf(s);
    const float qy = __fmaf_rn(q[3], yb[3], fma3(q[0], yb[0], q[1], yb[1], q[2], yb[2]));
    const float r3qy = r * r * r * qy;
#pragma unroll
    for (int k = 0; k < 4; ++k) qb[k] = __fmaf_rn(r, yb[k], -(r3qy * q[k]));
}

// q' = q + h * Ω(a) q with the component formulas of integrate_body /
// apply_ang_delta (Ω(a) q = (-a·q_v, a q_w + a × q_v)): adjoints for q and a.
__device__ __forceinline__ void quat_delta_adj(const float q[4], F3 a, float h, const float gb[4], float qb[4],
                                               F3& ab) {
    const float gw = gb[0], gx = gb[1], gy = gb[2], gz = gb[3];
    qb[0] += __fmaf_rn(h, fma3(a.x, gx, a.y, gy, a.z, gz), gw);
    qb[1] += __fmaf_rn(h, fma3(-a.x, gw, a.z, gy, -a.y, gz), gx);
    qb[2] += __fmaf_rn(h, fma3(-a.y, gw, -a.z, gx, a.x, gz), gy);
    qb[3] += __fmaf_rn(h, fma3(-a.z, gw, a.y, gx, -a.x, gy), gz);
    ab.x += h * __fmaf_rn(q[2], gz, fma3(-q[1], gw, q[0], gx, -q[3], gy));
    ab.y += h * __fmaf_rn(-q[1], gz, fma3(-q[2], gw, q[3], gx, q[0], gy));
    ab.z += h * __fmaf_rn(q[0], gz, fma3(-q[3], gw, -q[2], gx, q[1], gy));
}

// ── integrate (one body, n_substeps substeps of sub_dt) ─────────────────────
// State adjoint in/out: x̄ (3), q̄ (4), v̄ (3), ω̄ (3). Supports n_substeps <= 8.
__device__ __forceinline__ bool integrate_body_adj(const Pose& p0, float ox, float oy, float oz, float gx, float gy,
                                                   float gz, float sub_dt, float half_dt, int n_substeps, F3& xb,
                                                   float qb[4], F3& vb, F3& wb) {
    if (n_substeps > 8) return false;
    Pose st[8];
    Pose p = p0;
    for (int k = 0; k < n_substeps; ++k) {
        st[k] = p;
        integrate_body(p, ox, oy, oz, gx, gy, gz, sub_dt, half_dt);
    }
    const F3 om = f3(ox, oy, oz);
    for (int k = n_substeps - 1; k >= 0; --k) {
        const Pose& s = st[k];
        // q' = q + half_dt * Ω(ω) q, q_out = q' / |q'|
        const float q[4] = {s.qw, s.qx, s.qy, s.qz};
        const float dpw = -(ox * q[1] + oy * q[2] + oz * q[3]);
        const float dpx = (ox * q[0] + oy * q[3] - oz * q[2]);
        const float dpy = (oy * q[0] + oz * q[1] - ox * q[3]);
        const float dpz = (oz * q[0] + ox * q[2] - oy * q[1]);
        const float qp[4] = {q[0] + half_dt * dpw, q[1] + half_dt * dpx, q[2] + half_dt * dpy, q[3] + half_dt * dpz};
        float qpb[4];
        normalize_adj(qp, qb, qpb);
        float qin[4] = {0.f, 0.f, 0.f, 0.f};
        quat_delta_adj(q, om, half_dt, qpb, qin, wb);
        qb[0] = qin[0]; qb[1] = qin[1]; qb[2] = qin[2]; qb[3] = qin[3];
        // v1 = v0 + g dt, x1 = x0 + v1 dt
        vb += sub_dt * xb;
    }
    return true;
}

// ── narrowphase ─────────────────────────────────────────────────────────────

// sphere a (centre ca, radius ra) and sphere b: contact p, n, depth.
__device__ __forceinline__ void sphere_sphere_adj(F3 ca, float ra, F3 cb, float rb, uint32_t br, F3 pb, F3 nb,
                                                  float db, F3& cab, F3& cbb) {
    // p = 0.5 (ca + cb + n (rb - ra)), depth = ra + rb - dist, n = d / dist
    cab += 0.5f * pb;
    cbb += 0.5f * pb;
    nb += (0.5f * (rb - ra)) * pb;
    const F3 d = ca - cb;
    const float dist = sqrtf(dot(d, d));
    float distb = -db;
    F3 dbv = f3(0.f, 0.f, 0.f);
    if (!(br & 1u)) {
        const F3 n = (1.f / dist) * d;
        dbv += (1.f / dist) * nb;
        distb += -dot(nb, n) / dist;
        dbv += (distb / dist) * d;
    } else {
        dbv += (distb / fmaxf(dist, 1e-30f)) * d;
    }
    cab += dbv;
    cbb -= dbv;
}

// sphere (centre sc, radius r) against a box (centre bc, axes E = rows of
// A(qbox), half extents h): adjoints of sc, bc and qbox.
__device__ __forceinline__ void sphere_box_adj(F3 sc, float r, F3 bc, const float qbox[4], const float h[3],
                                               uint32_t br, F3 pb, F3 nb, float dpb, F3& scb, F3& bcb,
                                               float qboxb[4]) {
    float E[3][3];
    rot_rows(qbox, E);
    const F3 Ek[3] = {f3(E[0][0], E[0][1], E[0][2]), f3(E[1][0], E[1][1], E[1][2]), f3(E[2][0], E[2][1], E[2][2])};
    const F3 d = sc - bc;
    float qv[3] = {dot(d, Ek[0]), dot(d, Ek[1]), dot(d, Ek[2])};
    float qbv[3] = {0.f, 0.f, 0.f};
    F3 Eb[3] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
    if (br & 1u) {  // centre inside: n = -s E_k, depth = r + h_k - s q_k, p = sc - n r
        const int k = (br >> 1) & 3u;
        const float s = (br & 8u) ? -1.f : 1.f;
        scb += pb;
        nb += (-r) * pb;
        Eb[k] += (-s) * nb;
        qbv[k] += -s * dpb;
    } else {
        float cl[3], l[3];
        bool clamped[3];
        for (int k = 0; k < 3; ++k) {
            const bool lo = (br >> (4 + 2 * k)) & 1u, hi = (br >> (5 + 2 * k)) & 1u;
            clamped[k] = lo || hi;
            cl[k] = lo ? -h[k] : (hi ? h[k] : qv[k]);
            l[k] = qv[k] - cl[k];
        }
        const F3 wv = l[0] * Ek[0] + l[1] * Ek[1] + l[2] * Ek[2];
        const float dist = sqrtf(l[0] * l[0] + l[1] * l[1] + l[2] * l[2]);
        // p = bc + Σ cl_k E_k
        bcb += pb;
        float clb[3];
        for (int k = 0; k < 3; ++k) {
            clb[k] = dot(pb, Ek[k]);
            Eb[k] += cl[k] * pb;
        }
        // n = -w / dist, depth = r - dist
        const F3 wb = (-1.f / dist) * nb;
        float distb = dot(nb, wv) / (dist * dist) - dpb;
        float lb[3];
        for (int k = 0; k < 3; ++k) {
            lb[k] = dot(wb, Ek[k]) + (distb / dist) * l[k];
            Eb[k] += l[k] * wb;
        }
        for (int k = 0; k < 3; ++k) qbv[k] += clamped[k] ? lb[k] : clb[k];
    }
    // q_k = d · E_k
    F3 dbv = f3(0.f, 0.f, 0.f);
    for (int k = 0; k < 3; ++k) {
        dbv += qbv[k] * Ek[k];
        Eb[k] += qbv[k] * d;
    }
    scb += dbv;
    bcb -= dbv;
    const float Ab[3][3] = {{Eb[0].x, Eb[0].y, Eb[0].z}, {Eb[1].x, Eb[1].y, Eb[1].z}, {Eb[2].x, Eb[2].y, Eb[2].z}};
    rot_adj(qbox, Ab, qboxb);
}

// box a / box b (box_box_centroid): adjoints of both centres and quaternions.
// n is the contact normal the forward produced (its sign against the SAT
// axis is read from it).
__device__ __forceinline__ void box_box_adj(F3 ca, const float qa[4], const float ha[3], F3 cb, const float qb_[4],
                                            const float hb[3], uint32_t br, F3 n, F3 pbar, F3 nbar, float dbar,
                                            F3& cab, float qab[4], F3& cbb, float qbb[4]) {
    float A[3][3], Bm[3][3];
    rot_rows(qa, A);
    rot_rows(qb_, Bm);
    F3 Ar[3], Br[3];
    for (int k = 0; k < 3; ++k) {
        Ar[k] = f3(A[k][0], A[k][1], A[k][2]);
        Br[k] = f3(Bm[k][0], Bm[k][1], Bm[k][2]);
    }
    F3 Arb[3] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
    F3 Brb[3] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
    const int type = br & 3u, ai = (br >> 2) & 3u, aj = (br >> 4) & 3u;
    F3 nb = nbar;
    if (type != 2) {
        // face case: reference face, incident vertices kept, centroid
        const bool refB = br & kBrRefB;
        const F3 rc = refB ? cb : ca;
        const F3 ic = refB ? ca : cb;
        const F3* Ie = refB ? Ar : Br;
        const float* Ih = refB ? ha : hb;
        const float sd = refB ? -1.f : 1.f;
        const uint32_t kept = (br >> 10) & 0xFFu;
        const float nk = static_cast<float>(__popc(kept));
        F3 rcb = f3(0.f, 0.f, 0.f), icb = f3(0.f, 0.f, 0.f);
        F3 Ieb[3] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
        const float Rh_ref = (refB ? hb : ha)[(br >> 8) & 3u];
        for (int k = 0; k < 8; ++k) {
            if (!((kept >> k) & 1u)) continue;
            const float sx = (k & 1) ? 1.f : -1.f, sy = (k & 2) ? 1.f : -1.f, sz = (k & 4) ? 1.f : -1.f;
            const F3 v = ic + (sx * Ih[0]) * Ie[0] + (sy * Ih[1]) * Ie[1] + (sz * Ih[2]) * Ie[2];
            const float dv = Rh_ref + sd * (dot(v, n) - dot(rc, n));
            // point += (v - sd dv n) / nk, depth += dv / nk
            F3 vb = (1.f / nk) * pbar;
            const float dvb = (-sd * dot(pbar, n) + dbar) / nk;
            nb += (-sd * dv / nk) * pbar;
            vb += (sd * dvb) * n;
            nb += (sd * dvb) * (v - rc);
            rcb += (-sd * dvb) * n;
            icb += vb;
            Ieb[0] += (sx * Ih[0]) * vb;
            Ieb[1] += (sy * Ih[1]) * vb;
            Ieb[2] += (sz * Ih[2]) * vb;
        }
        if (refB) {
            cbb += rcb;
            cab += icb;
            for (int k = 0; k < 3; ++k) Arb[k] += Ieb[k];
        } else {
            cab += rcb;
            cbb += icb;
            for (int k = 0; k < 3; ++k) Brb[k] += Ieb[k];
        }
        // n = sgn * axis (face i of the box the SAT chose)
        const F3 axis = type == 0 ? Ar[ai] : Br[ai];
        const float sgn = dot(n, axis) >= 0.f ? 1.f : -1.f;
        if (type == 0) Arb[ai] += sgn * nb;
        else Brb[ai] += sgn * nb;
    } else {
        // edge case: closest points of edge i of A and edge j of B
        const int t0A = (ai + 1) % 3, t1A = (ai + 2) % 3, t0B = (aj + 1) % 3, t1B = (aj + 2) % 3;
        const float s0A = (br >> 18) & 1u ? -1.f : 1.f, s1A = (br >> 19) & 1u ? -1.f : 1.f;
        const float s0B = (br >> 20) & 1u ? -1.f : 1.f, s1B = (br >> 21) & 1u ? -1.f : 1.f;
        const F3 pA = ca + (s0A * ha[t0A]) * Ar[t0A] + (s1A * ha[t1A]) * Ar[t1A];
        const F3 pB = cb + (s0B * hb[t0B]) * Br[t0B] + (s1B * hb[t1B]) * Br[t1B];
        const F3 uA = Ar[ai], uB = Br[aj];
        const float b12 = dot(uA, uB), denom = 1.f - b12 * b12;
        const F3 wv = pA - pB;
        const float d1 = dot(wv, uA), d2 = dot(wv, uB);
        float s_t = 0.f, t_t = 0.f;
        const bool solved = br & kBrDenom;
        if (solved) {
            s_t = (b12 * d2 - d1) / denom;
            t_t = (d2 - b12 * d1) / denom;
        }
        // point = 0.5 (pA + s uA + pB + t uB)
        const F3 qAb = 0.5f * pbar, qBb = 0.5f * pbar;
        F3 pAb = qAb, pBb = qBb;
        const float sb = dot(qAb, uA), tb = dot(qBb, uB);
        F3 uAb = s_t * qAb, uBb = t_t * qBb;
        if (solved) {
            float b12b = sb * d2 / denom - tb * d1 / denom;
            float d1b = -sb / denom - tb * b12 / denom;
            float d2b = sb * b12 / denom + tb / denom;
            const float denb = -sb * s_t / denom - tb * t_t / denom;
            b12b += -2.f * b12 * denb;
            const F3 wb = d1b * uA + d2b * uB;
            uAb += d1b * wv;
            uBb += d2b * wv;
            uAb += b12b * uB;
            uBb += b12b * uA;
            pAb += wb;
            pBb -= wb;
        }
        cab += pAb;
        Arb[t0A] += (s0A * ha[t0A]) * pAb;
        Arb[t1A] += (s1A * ha[t1A]) * pAb;
        cbb += pBb;
        Brb[t0B] += (s0B * hb[t0B]) * pBb;
        Brb[t1B] += (s1B * hb[t1B]) * pBb;
        Arb[ai] += uAb;
        Brb[aj] += uBb;
        // depth = Σ ha_m |l·A_m| + Σ hb_m |l·B_m| - |d·l|, l = c / |c|, c = A_i × B_j, n = sgn l
        const F3 c = cross(uA, uB);
        const float clen = sqrtf(dot(c, c));
        const F3 l = (1.f / clen) * c;
        const float sgn = dot(n, l) >= 0.f ? 1.f : -1.f;
        F3 lb = sgn * nb;
        const F3 d = cb - ca;
        for (int m = 0; m < 3; ++m) {
            const float sa = dot(l, Ar[m]) >= 0.f ? 1.f : -1.f;
            const float sbm = dot(l, Br[m]) >= 0.f ? 1.f : -1.f;
            lb += (dbar * ha[m] * sa) * Ar[m];
            Arb[m] += (dbar * ha[m] * sa) * l;
            lb += (dbar * hb[m] * sbm) * Br[m];
            Brb[m] += (dbar * hb[m] * sbm) * l;
        }
        const float tau = dot(d, l) >= 0.f ? 1.f : -1.f;
        lb += (-dbar * tau) * d;
        const F3 db = (-dbar * tau) * l;
        cbb += db;
        cab -= db;
        // l = c / |c|
        const F3 cb_ = (1.f / clen) * (lb - dot(lb, l) * l);
        // c = uA × uB
        Arb[ai] += cross(uB, cb_);
        Brb[aj] += cross(cb_, uA);
    }
    const float Ab[3][3] = {{Arb[0].x, Arb[0].y, Arb[0].z}, {Arb[1].x, Arb[1].y, Arb[1].z},
                            {Arb[2].x, Arb[2].y, Arb[2].z}};
    const float Bb[3][3] = {{Brb[0].x, Brb[0].y, Brb[0].z}, {Brb[1].x, Brb[1].y, Brb[1].z},
                            {Brb[2].x, Brb[2].y, Brb[2].z}};
    rot_adj(qa, Ab, qab);
    rot_adj(qb_, Bb, qbb);
}

// ── contact solve ───────────────────────────────────────────────────────────

// Adjoint of one body: pose, velocity, spin, and its inverse mass.
struct BodyBar {
    F3 x;
    float q[4];
    F3 v, w;
    float im;
};

// solve_contact on the pair (L body 0 = a, body 1 = b) from its pre-solve
// state, with the branch flags `fl` the forward solve recorded. G0 / G1 hold
// the adjoint of the post-solve state on entry and of the pre-solve state on
// return (im accumulates); pb, nb, db receive the contact geometry's adjoint.
// lc_in is lambda before the solve.
__device__ __forceinline__ void solve_contact_adj(const LocalPair& L, const Contact& ct, float mu, float dt,
                                                  float lc_in, uint32_t fl, BodyBar& G0, BodyBar& G1, F3& pb,
                                                  F3& nb, float& db) {
    if (!(fl & kSfActive)) return;
    const float wa = L.m[0], wb = L.m[1];
    const bool da = wa != 0.f, dbn = wb != 0.f;
    const F3 n = f3(ct.nx, ct.ny, ct.nz), p = f3(ct.px, ct.py, ct.pz);
    const F3 xa = f3(L.p[0][0], L.p[0][1], L.p[0][2]), xb = f3(L.p[1][0], L.p[1][1], L.p[1][2]);
    const F3 va = f3(L.v[0][0], L.v[0][1], L.v[0][2]), vb = f3(L.v[1][0], L.v[1][1], L.v[1][2]);
    const F3 oa = f3(L.w[0][0], L.w[0][1], L.w[0][2]), ob = f3(L.w[1][0], L.w[1][1], L.w[1][2]);
    const float* qa = L.q[0];
    const float* qbq = L.q[1];
    const F3 ra = p - xa, rb = p - xb;
    const F3 ca = cross(ra, n), cb = cross(rb, n);
    const F3 ua = winv(qa, L.I[0], ca), ub = winv(qbq, L.I[1], cb);
    const float w = wa + wb + dot(ca, ua) + dot(cb, ub);
    const float rem = ct.depth - lc_in;
    const float dl = rem / w;
    const float lc_out = lc_in + rem;
    // rotations after the position correction
    float qa1[4] = {qa[0], qa[1], qa[2], qa[3]}, qb1[4] = {qbq[0], qbq[1], qbq[2], qbq[3]};
    const F3 aa = dl * ua, ab = (-dl) * ub;
    if (da) {
        qa1[0] += 0.5f * (-aa.x * qa[1] - aa.y * qa[2] - aa.z * qa[3]);
        qa1[1] += 0.5f * (aa.x * qa[0] + aa.y * qa[3] - aa.z * qa[2]);
        qa1[2] += 0.5f * (-aa.x * qa[3] + aa.y * qa[0] + aa.z * qa[1]);
        qa1[3] += 0.5f * (aa.x * qa[2] - aa.y * qa[1] + aa.z * qa[0]);
    }
    if (dbn) {
        qb1[0] += 0.5f * (-ab.x * qbq[1] - ab.y * qbq[2] - ab.z * qbq[3]);
        qb1[1] += 0.5f * (ab.x * qbq[0] + ab.y * qbq[3] - ab.z * qbq[2]);
        qb1[2] += 0.5f * (-ab.x * qbq[3] + ab.y * qbq[0] + ab.z * qbq[1]);
        qb1[3] += 0.5f * (ab.x * qbq[2] - ab.y * qbq[1] + ab.z * qbq[0]);
    }
    // normal velocity impulse
    const F3 vrel = (va + cross(oa, ra)) - (vb + cross(ob, rb));
    const float vreln = dot(vrel, n);
    float jn = 0.f;
    F3 dA = f3(0.f, 0.f, 0.f), dB = f3(0.f, 0.f, 0.f);
    F3 va1 = va, vb1 = vb, oa1 = oa, ob1 = ob;
    if (fl & kSfNormal) {
        jn = -vreln / w;
        dA = winv(qa1, L.I[0], ca);
        dB = winv(qb1, L.I[1], cb);
        if (da) { va1 += (wa * jn) * n; oa1 += jn * dA; }
        if (dbn) { vb1 -= (wb * jn) * n; ob1 -= jn * dB; }
    }
    // friction
    F3 rv = f3(0.f, 0.f, 0.f), vt = rv, t = rv, ea = rv, eb = rv, fa = rv, fb = rv;
    float rvn = 0.f, Lt = 0.f, wt = 0.f, jt = 0.f, jt_raw = 0.f, jns = 0.f;
    const bool fr = fl & kSfFriction, clamped = fl & kSfClamped;
    if (fr) {
        rv = (va1 + cross(oa1, ra)) - (vb1 + cross(ob1, rb));
        rvn = dot(rv, n);
        vt = rv - rvn * n;
        Lt = sqrtf(dot(vt, vt));
        t = (1.f / Lt) * vt;
        ea = cross(ra, t);
        eb = cross(rb, t);
        fa = winv(qa1, L.I[0], ea);
        fb = winv(qb1, L.I[1], eb);
        wt = wa + wb + dot(ea, fa) + dot(eb, fb);
        jns = lc_out / (dt * w);
        jt_raw = Lt / wt;
        jt = clamped ? mu * jns : jt_raw;
    }
    // ── reverse ──
    float wab = 0.f, wbb = 0.f, wbar = 0.f, remb = 0.f, dlb = 0.f;
    F3 rab = f3(0.f, 0.f, 0.f), rbb = rab, cab = rab, cbb = rab, uab = rab, ubb = rab;
    float qa1b[4] = {G0.q[0], G0.q[1], G0.q[2], G0.q[3]}, qb1b[4] = {G1.q[0], G1.q[1], G1.q[2], G1.q[3]};
    F3 va1b = G0.v, oa1b = G0.w, vb1b = G1.v, ob1b = G1.w;
    if (fr) {
        float jtb = 0.f;
        F3 tb = f3(0.f, 0.f, 0.f), fab = tb, fbb = tb;
        if (da) {
            jtb += -wa * dot(G0.v, t) - dot(G0.w, fa);
            tb = fmav((-wa * jt), G0.v, tb);
            fab = fmav((-jt), G0.w, fab);
            wab += -jt * dot(G0.v, t);
        }
        if (dbn) {
            jtb += wb * dot(G1.v, t) + dot(G1.w, fb);
            tb = fmav((wb * jt), G1.v, tb);
            fbb = fmav(jt, G1.w, fbb);
            wbb += jt * dot(G1.v, t);
        }
        float Ltb = 0.f, wtb = 0.f;
        if (clamped) {
            const float jnsb = mu * jtb;
            remb += jnsb / (dt * w);
            wbar += -jnsb * lc_out / (dt * w * w);
        } else {
            Ltb += jtb / wt;
            wtb = -jtb * jt_raw / wt;
        }
        wab += wtb;
        wbb += wtb;
        F3 eab = wtb * fa, ebb = wtb * fb;
        fab = fmav(wtb, ea, fab);
        fbb = fmav(wtb, eb, fbb);
        winv_adj(qa1, L.I[0], ea, fab, eab, qa1b);
        winv_adj(qb1, L.I[1], eb, fbb, ebb, qb1b);
        rab += cross(t, eab);
        tb += cross(eab, ra);
        rbb += cross(t, ebb);
        tb += cross(ebb, rb);
        F3 vtb = (1.f / Lt) * tb;
        Ltb += -dot(tb, vt) / (Lt * Lt);
        vtb = fmav((Ltb / Lt), vt, vtb);
        const F3 rvb0 = vtb;
        const float rvnb = -dot(vtb, n);
        nb = fmav((-rvn), vtb, nb);
        const F3 rvb = rvb0 + rvnb * n;
        nb = fmav(rvnb, rv, nb);
        va1b += rvb;
        oa1b += cross(ra, rvb);
        rab += cross(rvb, oa1);
        vb1b -= rvb;
        ob1b -= cross(rb, rvb);
        rbb -= cross(rvb, ob1);
    }
    F3 vab = va1b, oab = oa1b, vbb = vb1b, obb = ob1b;
    if (fl & kSfNormal) {
        float jnb = 0.f;
        F3 dAb = f3(0.f, 0.f, 0.f), dBb = dAb;
        if (da) {
            jnb += wa * dot(va1b, n) + dot(oa1b, dA);
            nb = fmav((wa * jn), va1b, nb);
            wab += jn * dot(va1b, n);
            dAb = fmav(jn, oa1b, dAb);
        }
        if (dbn) {
            jnb += -wb * dot(vb1b, n) - dot(ob1b, dB);
            nb = fmav((-wb * jn), vb1b, nb);
            wbb += -jn * dot(vb1b, n);
            dBb = fmav((-jn), ob1b, dBb);
        }
        winv_adj(qa1, L.I[0], ca, dAb, cab, qa1b);
        winv_adj(qb1, L.I[1], cb, dBb, cbb, qb1b);
        const float vrelnb = -jnb / w;
        wbar += -jnb * jn / w;
        const F3 vrelb = vrelnb * n;
        nb = fmav(vrelnb, vrel, nb);
        vab += vrelb;
        oab += cross(ra, vrelb);
        rab += cross(vrelb, oa);
        vbb -= vrelb;
        obb -= cross(rb, vrelb);
        rbb -= cross(vrelb, ob);
    }
    // rotation and position corrections
    float qab[4] = {qa1b[0], qa1b[1], qa1b[2], qa1b[3]}, qbb[4] = {qb1b[0], qb1b[1], qb1b[2], qb1b[3]};
    if (da) {
        F3 aab = f3(0.f, 0.f, 0.f);
        float qin[4] = {0.f, 0.f, 0.f, 0.f};
        quat_delta_adj(qa, aa, 0.5f, qa1b, qin, aab);
        for (int k = 0; k < 4; ++k) qab[k] = qin[k];
        dlb += dot(aab, ua);
        uab = fmav(dl, aab, uab);
        dlb += wa * dot(G0.x, n);
        wab += dl * dot(G0.x, n);
        nb = fmav((wa * dl), G0.x, nb);
    }
    if (dbn) {
        F3 abb = f3(0.f, 0.f, 0.f);
        float qin[4] = {0.f, 0.f, 0.f, 0.f};
        quat_delta_adj(qbq, ab, 0.5f, qb1b, qin, abb);
        for (int k = 0; k < 4; ++k) qbb[k] = qin[k];
        dlb += -dot(abb, ub);
        ubb = fmav((-dl), abb, ubb);
        dlb += -wb * dot(G1.x, n);
        wbb += -dl * dot(G1.x, n);
        nb = fmav((-wb * dl), G1.x, nb);
    }
    remb += dlb / w;
    wbar += -dlb * dl / w;
    wab += wbar;
    wbb += wbar;
    cab = fmav(wbar, ua, cab);
    uab = fmav(wbar, ca, uab);
    cbb = fmav(wbar, ub, cbb);
    ubb = fmav(wbar, cb, ubb);
    winv_adj(qa, L.I[0], ca, uab, cab, qab);
    winv_adj(qbq, L.I[1], cb, ubb, cbb, qbb);
    rab += cross(n, cab);
    nb += cross(cab, ra);
    rbb += cross(n, cbb);
    nb += cross(cbb, rb);
    pb += rab + rbb;
    // outputs: adjoint of the pre-solve state
    G0.x -= rab;
    G1.x -= rbb;
    for (int k = 0; k < 4; ++k) {
        G0.q[k] = qab[k];
        G1.q[k] = qbb[k];
    }
    G0.v = vab;
    G0.w = oab;
    G1.v = vbb;
    G1.w = obb;
    G0.im += wab;
    G1.im += wbb;
    db += remb;
}

}  // namespace dyph
