// dual_oracle.cpp — FP64 forward-mode (dual-number) gradients of the frame
// step, the checker of the library's hand-written adjoint.
//
// TEST INFRASTRUCTURE ONLY: tests/ and bench.py's gradient-error figure load
// it (oracle/_build/libdyphur_dual.so); the shipped library never links it.
//
// Each scalar is a TD: the float value the frame step computes (every float
// expression in the operand order of the reference's sources, as
// dyphur_oracle.c restates them, so this float trajectory is the one the GPU
// and the reference compute bit for bit), an FP64 value of the same
// expression, and FP64 tangents (one per gradient parameter) propagated by the
// chain rule at the FP64 values (or, with at_float, at the float values: the
// FP64 derivative of the float map itself, which stays defined on horizons
// where the FP64 trajectory and the float one part). Every branch — pair overlap, contact /
// no-contact, SAT axis, kept vertices, solver early-outs, friction clamp —
// is decided on the float value, so the FP64 evaluation follows the float
// run's contact set and branches: the derivative this computes is the
// derivative of the same piecewise-smooth map the adjoint differentiates, and
// the FP64 values are the "FP64 re-run" of the frame step along it.
//
// The restated path (sequential solver order, XpbdSolver::set_force_serial):
//   integrate          core/src/integrator.cpp:18-68
//   candidate pairs    fp16 leaf boxes (core/src/broadphase.cpp:216-251) of every
//                      body pair, inclusive overlap (:322-325), ascending (a, b)
//   narrowphase        core/src/narrowphase.cpp:46-306, 920-1001
//   solve              core/src/xpbd_solver.cpp:40-133, 413-521, 559-587
//   colour order       (dyd_fp64_run) Jones–Plassmann colours, :620-733
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Tangents carried (gradient parameters per call). The FP64 re-run library
// (libdyphur_fp64.so, dyd_fp64_run) is this file built with DYD_MAX_T=1.
#ifndef DYD_MAX_T
#define DYD_MAX_T 96
#endif
constexpr int kMaxT = DYD_MAX_T;
int g_nt = 0;              // tangents in use
bool g_at_float = false;   // evaluate the chain-rule coefficients at the float values

struct TD {
    float f;
    double v;
    double d[kMaxT];
};

TD cst(float x) {
    TD r;
    r.f = x;
    r.v = static_cast<double>(x);
    for (int i = 0; i < g_nt; ++i) r.d[i] = 0.0;
    return r;
}

TD operator+(const TD& a, const TD& b) {
    TD r;
    r.f = a.f + b.f;
    r.v = a.v + b.v;
    for (int i = 0; i < g_nt; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
TD operator-(const TD& a, const TD& b) {
    TD r;
    r.f = a.f - b.f;
    r.v = a.v - b.v;
    for (int i = 0; i < g_nt; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
TD operator-(const TD& a) {
    TD r;
    r.f = -a.f;
    r.v = -a.v;
    for (int i = 0; i < g_nt; ++i) r.d[i] = -a.d[i];
    return r;
}
// value at which the chain rule's coefficients are taken
double cv(const TD& a) { return g_at_float ? static_cast<double>(a.f) : a.v; }

TD operator*(const TD& a, const TD& b) {
    TD r;
    r.f = a.f * b.f;
    r.v = a.v * b.v;
    const double av = cv(a), bv = cv(b);
    for (int i = 0; i < g_nt; ++i) r.d[i] = a.d[i] * bv + av * b.d[i];
    return r;
}
TD operator/(const TD& a, const TD& b) {
    TD r;
    r.f = a.f / b.f;
    r.v = a.v / b.v;
    const double bv = cv(b), qv = cv(a) / bv;
    for (int i = 0; i < g_nt; ++i) r.d[i] = (a.d[i] - qv * b.d[i]) / bv;
    return r;
}
TD operator+(const TD& a, float b) { return a + cst(b); }
TD operator+(float a, const TD& b) { return cst(a) + b; }
TD operator-(const TD& a, float b) { return a - cst(b); }
TD operator-(float a, const TD& b) { return cst(a) - b; }
TD operator*(const TD& a, float b) { return a * cst(b); }
TD operator*(float a, const TD& b) { return cst(a) * b; }
TD operator/(float a, const TD& b) { return cst(a) / b; }
TD& operator+=(TD& a, const TD& b) { return a = a + b; }
TD& operator-=(TD& a, const TD& b) { return a = a - b; }

TD tsqrt(const TD& a) {
    TD r;
    r.f = std::sqrt(a.f);
    r.v = std::sqrt(a.v);
    const double rv = g_at_float ? std::sqrt(static_cast<double>(a.f)) : r.v;
    for (int i = 0; i < g_nt; ++i) r.d[i] = a.d[i] / (2.0 * rv);
    return r;
}
// |a| with the sign taken from the float value (the branch the float run took)
TD tabs(const TD& a) { return a.f < 0.f ? -a : a; }
TD tmin(const TD& a, const TD& b) { return (b.f < a.f) ? b : a; }  // fminf
TD rsqrt_ieee(const TD& x) { return 1.f / tsqrt(x); }

uint16_t f32_to_f16(float f) {
    const _Float16 h = static_cast<_Float16>(f);  // round to nearest even
    uint16_t b;
    std::memcpy(&b, &h, 2);
    return b;
}
float f16_to_f32(uint16_t b) {
    _Float16 h;
    std::memcpy(&h, &b, 2);
    return static_cast<float>(h);
}

struct Body {
    TD p[3], q[4], v[3], w[3];
    TD m;         // inverse mass
    float I[6];   // inverse inertia (held fixed)
    uint32_t type, flags;
    float h[3];
};

struct Contact {
    uint32_t a, b;
    TD p[3], n[3], depth;
};

// ── integrate (integrator.cpp:18-68) ──
void integrate(Body& B, float g[3], float sub_dt, float half_dt, int n_sub) {
    if (B.m.f == 0.f || (B.flags & 4u)) return;
    for (int k = 0; k < n_sub; ++k) {
        TD vx = B.v[0] + g[0] * sub_dt, vy = B.v[1] + g[1] * sub_dt, vz = B.v[2] + g[2] * sub_dt;
        B.v[0] = vx; B.v[1] = vy; B.v[2] = vz;
        B.p[0] = B.p[0] + vx * sub_dt;
        B.p[1] = B.p[1] + vy * sub_dt;
        B.p[2] = B.p[2] + vz * sub_dt;
        TD qw = B.q[0], qx = B.q[1], qy = B.q[2], qz = B.q[3];
        const TD &ox = B.w[0], &oy = B.w[1], &oz = B.w[2];
        TD dpw = -(ox * qx + oy * qy + oz * qz);
        TD dpx = (ox * qw + oy * qz - oz * qy);
        TD dpy = (oy * qw + oz * qx - ox * qz);
        TD dpz = (oz * qw + ox * qy - oy * qx);
        qw = qw + half_dt * dpw;
        qx = qx + half_dt * dpx;
        qy = qy + half_dt * dpy;
        qz = qz + half_dt * dpz;
        TD inv = rsqrt_ieee(qw * qw + qx * qx + qy * qy + qz * qz);
        B.q[0] = qw * inv; B.q[1] = qx * inv; B.q[2] = qy * inv; B.q[3] = qz * inv;
    }
}

void renormalize(TD q[4]) {
    TD inv = rsqrt_ieee(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; ++k) q[k] = q[k] * inv;
}

// make_axes (narrowphase.cpp:913-917)
void axes(const TD q[4], TD A[3][3]) {
    const TD &qw = q[0], &qx = q[1], &qy = q[2], &qz = q[3];
    A[0][0] = 1.f - 2.f * (qy * qy + qz * qz); A[0][1] = 2.f * (qx * qy + qz * qw); A[0][2] = 2.f * (qx * qz - qy * qw);
    A[1][0] = 2.f * (qx * qy - qz * qw); A[1][1] = 1.f - 2.f * (qx * qx + qz * qz); A[1][2] = 2.f * (qy * qz + qx * qw);
    A[2][0] = 2.f * (qx * qz + qy * qw); A[2][1] = 2.f * (qy * qz - qx * qw); A[2][2] = 1.f - 2.f * (qx * qx + qy * qy);
}

// leaf box bits (broadphase.cpp:216-251), float only
void leaf_box(const Body& B, float out[6]) {
    const float px = B.p[0].f, py = B.p[1].f, pz = B.p[2].f;
    float mn[3], mx[3];
    if (B.type == 1u) {
        const float r = B.h[0];
        mn[0] = px - r; mx[0] = px + r; mn[1] = py - r; mx[1] = py + r; mn[2] = pz - r; mx[2] = pz + r;
    } else {
        const float qw = B.q[0].f, qx = B.q[1].f, qy = B.q[2].f, qz = B.q[3].f;
        const float hx = B.h[0], hy = B.h[1], hz = B.h[2];
        float rxx = 1.f - 2.f * (qy * qy + qz * qz), rxy = 2.f * (qx * qy - qz * qw), rxz = 2.f * (qx * qz + qy * qw);
        float ryx = 2.f * (qx * qy + qz * qw), ryy = 1.f - 2.f * (qx * qx + qz * qz), ryz = 2.f * (qy * qz - qx * qw);
        float rzx = 2.f * (qx * qz - qy * qw), rzy = 2.f * (qy * qz + qx * qw), rzz = 1.f - 2.f * (qx * qx + qy * qy);
        float ex = std::fabs(rxx) * hx + std::fabs(rxy) * hy + std::fabs(rxz) * hz;
        float ey = std::fabs(ryx) * hx + std::fabs(ryy) * hy + std::fabs(ryz) * hz;
        float ez = std::fabs(rzx) * hx + std::fabs(rzy) * hy + std::fabs(rzz) * hz;
        mn[0] = px - ex; mx[0] = px + ex; mn[1] = py - ey; mx[1] = py + ey; mn[2] = pz - ez; mx[2] = pz + ez;
    }
    for (int k = 0; k < 3; ++k) {
        out[k] = f16_to_f32(f32_to_f16(mn[k]));
        out[3 + k] = f16_to_f32(f32_to_f16(mx[k]));
    }
}
bool overlap(const float n[6], const float q[6]) {
    return !(n[0] > q[3] || n[3] < q[0] || n[1] > q[4] || n[4] < q[1] || n[2] > q[5] || n[5] < q[2]);
}

// sphere_sphere (narrowphase.cpp:46-68)
bool sphere_sphere(const TD a[3], float ra, const TD b[3], float rb, Contact& c) {
    TD dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    TD dist2 = dx * dx + dy * dy + dz * dz;
    float sum_r = ra + rb;
    if (dist2.f >= sum_r * sum_r) return false;
    TD dist = tsqrt(dist2);
    if (dist.f < 1e-8f) { c.n[0] = cst(0.f); c.n[1] = cst(1.f); c.n[2] = cst(0.f); }
    else { TD inv = 1.f / dist; c.n[0] = dx * inv; c.n[1] = dy * inv; c.n[2] = dz * inv; }
    c.depth = cst(sum_r) - dist;
    TD sa = a[0] - c.n[0] * ra, sb = b[0] + c.n[0] * rb;
    c.p[0] = 0.5f * (sa + sb);
    sa = a[1] - c.n[1] * ra; sb = b[1] + c.n[1] * rb; c.p[1] = 0.5f * (sa + sb);
    sa = a[2] - c.n[2] * ra; sb = b[2] + c.n[2] * rb; c.p[2] = 0.5f * (sa + sb);
    return true;
}

// sphere_box (narrowphase.cpp:71-127); E rows are the box axes
bool sphere_box(const TD s[3], float sr, const TD bc[3], TD E[3][3], const float bh[3], Contact& c) {
    TD dx = s[0] - bc[0], dy = s[1] - bc[1], dz = s[2] - bc[2];
    TD q[3];
    for (int k = 0; k < 3; ++k) q[k] = dx * E[k][0] + dy * E[k][1] + dz * E[k][2];
    TD cl[3];
    for (int k = 0; k < 3; ++k) cl[k] = q[k].f < -bh[k] ? cst(-bh[k]) : (q[k].f > bh[k] ? cst(bh[k]) : q[k]);
    TD lx = q[0] - cl[0], ly = q[1] - cl[1], lz = q[2] - cl[2];
    TD dist2 = lx * lx + ly * ly + lz * lz;
    if (dist2.f < 1e-12f) {
        TD pen[3] = {bh[0] - tabs(q[0]), bh[1] - tabs(q[1]), bh[2] - tabs(q[2])};
        int k = 2;
        if (pen[0].f <= pen[1].f && pen[0].f <= pen[2].f) k = 0;
        else if (pen[1].f <= pen[2].f) k = 1;
        const float sg = q[k].f >= 0.f ? 1.f : -1.f;
        c.n[0] = -(sg * E[k][0]); c.n[1] = -(sg * E[k][1]); c.n[2] = -(sg * E[k][2]);
        c.depth = sr + pen[k];
        for (int j = 0; j < 3; ++j) c.p[j] = s[j] - c.n[j] * sr;
        return true;
    }
    if (dist2.f >= sr * sr) return false;
    TD dist = tsqrt(dist2);
    TD inv_d = 1.f / dist;
    TD wx = lx * E[0][0] + ly * E[1][0] + lz * E[2][0];
    TD wy = lx * E[0][1] + ly * E[1][1] + lz * E[2][1];
    TD wz = lx * E[0][2] + ly * E[1][2] + lz * E[2][2];
    c.n[0] = -wx * inv_d; c.n[1] = -wy * inv_d; c.n[2] = -wz * inv_d;
    c.depth = sr - dist;
    for (int j = 0; j < 3; ++j) c.p[j] = bc[j] + cl[0] * E[0][j] + cl[1] * E[1][j] + cl[2] * E[2][j];
    return true;
}

struct Best {
    TD ov;
    int type, i, j;
    TD n[3];
};

// one SAT axis (narrowphase.cpp:158-175, 192-208)
bool sat_axis(const TD l[3], TD A[3][3], const float Ah[3], TD Bm[3][3], const float Bh[3], const TD d[3], int type,
              int i, int j, Best& best) {
    TD rA = Ah[0] * tabs(l[0] * A[0][0] + l[1] * A[0][1] + l[2] * A[0][2]) +
            Ah[1] * tabs(l[0] * A[1][0] + l[1] * A[1][1] + l[2] * A[1][2]) +
            Ah[2] * tabs(l[0] * A[2][0] + l[1] * A[2][1] + l[2] * A[2][2]);
    TD rB = Bh[0] * tabs(l[0] * Bm[0][0] + l[1] * Bm[0][1] + l[2] * Bm[0][2]) +
            Bh[1] * tabs(l[0] * Bm[1][0] + l[1] * Bm[1][1] + l[2] * Bm[1][2]) +
            Bh[2] * tabs(l[0] * Bm[2][0] + l[1] * Bm[2][1] + l[2] * Bm[2][2]);
    TD dl = d[0] * l[0] + d[1] * l[1] + d[2] * l[2];
    TD t = tabs(dl);
    TD ov = rA + rB - t;
    if (ov.f <= 0.f) return false;
    if (ov.f < best.ov.f) {
        best.ov = ov;
        best.type = type; best.i = i; best.j = j;
        const float sgn = dl.f >= 0.f ? -1.f : 1.f;
        for (int k = 0; k < 3; ++k) best.n[k] = sgn * l[k];
    }
    return true;
}

// box_box + centroid reduction (narrowphase.cpp:130-306, 991-998)
bool box_box(const TD a[3], TD A[3][3], const float Ah[3], const TD b[3], TD Bm[3][3], const float Bh[3], Contact& out) {
    const float eps_par = 1e-5f;
    TD C[3][3];
    TD d[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) C[i][j] = A[i][0] * Bm[j][0] + A[i][1] * Bm[j][1] + A[i][2] * Bm[j][2];
    Best best{cst(1e30f), -1, 0, 0, {cst(0.f), cst(1.f), cst(0.f)}};
    for (int i = 0; i < 3; ++i) {
        const TD l[3] = {A[i][0], A[i][1], A[i][2]};
        if (!sat_axis(l, A, Ah, Bm, Bh, d, 0, i, 0, best)) return false;
    }
    for (int i = 0; i < 3; ++i) {
        const TD l[3] = {Bm[i][0], Bm[i][1], Bm[i][2]};
        if (!sat_axis(l, A, Ah, Bm, Bh, d, 1, i, 0, best)) return false;
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            TD cx = A[i][1] * Bm[j][2] - A[i][2] * Bm[j][1];
            TD cy = A[i][2] * Bm[j][0] - A[i][0] * Bm[j][2];
            TD cz = A[i][0] * Bm[j][1] - A[i][1] * Bm[j][0];
            TD len2 = cx * cx + cy * cy + cz * cz;
            if (len2.f < eps_par * eps_par) continue;
            TD inv_l = rsqrt_ieee(len2);
            const TD l[3] = {cx * inv_l, cy * inv_l, cz * inv_l};
            if (!sat_axis(l, A, Ah, Bm, Bh, d, 2, i, j, best)) return false;
        }
    const TD &bnx = best.n[0], &bny = best.n[1], &bnz = best.n[2];
    TD sx = cst(0.f), sy = cst(0.f), sz = cst(0.f), sd = cst(0.f);
    int n_out = 0;
    int best_type = best.type, best_i = best.i;
    if (best_type == 0 || best_type == 1) {
        if (best_type == 0) {
            int t0A = (best_i + 1) % 3, t1A = (best_i + 2) % 3;
            int j_best = 0;
            for (int j = 1; j < 3; ++j)
                if (std::fabs(C[best_i][j].f) > std::fabs(C[best_i][j_best].f)) j_best = j;
            int t0B = (j_best + 1) % 3, t1B = (j_best + 2) % 3;
            if (Bh[t0B] * Bh[t1B] > Ah[t0A] * Ah[t1A]) { best_type = 1; best_i = j_best; }
        }
        const bool a_ref = best_type == 0;
        const int ref_ax = best_i;
        const TD* rc = a_ref ? a : b;
        const TD* ic = a_ref ? b : a;
        TD (*Re)[3] = a_ref ? A : Bm;
        TD (*Ie)[3] = a_ref ? Bm : A;
        const float* Rh = a_ref ? Ah : Bh;
        const float* Ih = a_ref ? Bh : Ah;
        const int t0 = (ref_ax + 1) % 3, t1 = (ref_ax + 2) % 3;
        TD rc_dot_n3 = rc[0] * bnx + rc[1] * bny + rc[2] * bnz;
        const float sign_depth = a_ref ? 1.f : -1.f;
        const float Rh_ref = Rh[ref_ax], Rh_t0 = Rh[t0], Rh_t1 = Rh[t1];
        for (int k = 0; k < 8; ++k) {
            const float sgx = (k & 1) ? 1.f : -1.f, sgy = (k & 2) ? 1.f : -1.f, sgz = (k & 4) ? 1.f : -1.f;
            TD vx = ic[0] + sgx * Ih[0] * Ie[0][0] + sgy * Ih[1] * Ie[1][0] + sgz * Ih[2] * Ie[2][0];
            TD vy = ic[1] + sgx * Ih[0] * Ie[0][1] + sgy * Ih[1] * Ie[1][1] + sgz * Ih[2] * Ie[2][1];
            TD vz = ic[2] + sgx * Ih[0] * Ie[0][2] + sgy * Ih[1] * Ie[1][2] + sgz * Ih[2] * Ie[2][2];
            TD v_dot_n = vx * bnx + vy * bny + vz * bnz;
            TD dv = Rh_ref + sign_depth * (v_dot_n - rc_dot_n3);
            if (dv.f <= 0.f) continue;
            TD rx = vx - rc[0], ry = vy - rc[1], rz = vz - rc[2];
            TD qt0 = rx * Re[t0][0] + ry * Re[t0][1] + rz * Re[t0][2];
            TD qt1 = rx * Re[t1][0] + ry * Re[t1][1] + rz * Re[t1][2];
            if (std::fabs(qt0.f) > Rh_t0 + 1e-3f) continue;
            if (std::fabs(qt1.f) > Rh_t1 + 1e-3f) continue;
            if (n_out < 4) {
                sx += vx - sign_depth * dv * bnx;
                sy += vy - sign_depth * dv * bny;
                sz += vz - sign_depth * dv * bnz;
                sd += dv;
                ++n_out;
            }
        }
    } else {
        const int i = best.i, j = best.j;
        const int t0A = (i + 1) % 3, t1A = (i + 2) % 3;
        const float s0A = (-bnx * A[t0A][0] - bny * A[t0A][1] - bnz * A[t0A][2]).f >= 0.f ? 1.f : -1.f;
        const float s1A = (-bnx * A[t1A][0] - bny * A[t1A][1] - bnz * A[t1A][2]).f >= 0.f ? 1.f : -1.f;
        TD pA[3], pB[3];
        for (int k = 0; k < 3; ++k) pA[k] = a[k] + s0A * Ah[t0A] * A[t0A][k] + s1A * Ah[t1A] * A[t1A][k];
        const int t0B = (j + 1) % 3, t1B = (j + 2) % 3;
        const float s0B = (bnx * Bm[t0B][0] + bny * Bm[t0B][1] + bnz * Bm[t0B][2]).f >= 0.f ? 1.f : -1.f;
        const float s1B = (bnx * Bm[t1B][0] + bny * Bm[t1B][1] + bnz * Bm[t1B][2]).f >= 0.f ? 1.f : -1.f;
        for (int k = 0; k < 3; ++k) pB[k] = b[k] + s0B * Bh[t0B] * Bm[t0B][k] + s1B * Bh[t1B] * Bm[t1B][k];
        TD b12 = C[i][j];
        TD denom = 1.f - b12 * b12;
        TD wx = pA[0] - pB[0], wy = pA[1] - pB[1], wz = pA[2] - pB[2];
        TD d1 = wx * A[i][0] + wy * A[i][1] + wz * A[i][2];
        TD d2 = wx * Bm[j][0] + wy * Bm[j][1] + wz * Bm[j][2];
        TD s_t = cst(0.f), t_t = cst(0.f);
        if (std::fabs(denom.f) > 1e-6f) {
            s_t = (b12 * d2 - d1) / denom;
            t_t = (d2 - b12 * d1) / denom;
        }
        for (int k = 0; k < 3; ++k) {
            TD qA = pA[k] + s_t * A[i][k], qB = pB[k] + t_t * Bm[j][k];
            TD m = 0.f + 0.5f * (qA + qB);
            if (k == 0) sx = m; else if (k == 1) sy = m; else sz = m;
        }
        sd = 0.f + best.ov;
        n_out = 1;
    }
    if (n_out == 0) return false;
    TD inv = 1.f / cst(static_cast<float>(n_out));
    out.p[0] = sx * inv; out.p[1] = sy * inv; out.p[2] = sz * inv;
    out.n[0] = bnx; out.n[1] = bny; out.n[2] = bnz;
    out.depth = sd * inv;
    return true;
}

// process_pair for boxes / spheres (narrowphase.cpp:920-1001)
bool process_pair(std::vector<Body>& Bs, uint32_t ia, uint32_t ib, Contact& c) {
    Body &a = Bs[ia], &b = Bs[ib];
    c.a = ia; c.b = ib;
    if (a.type == 1u && b.type == 1u) return sphere_sphere(a.p, a.h[0], b.p, b.h[0], c);
    if (a.type == 1u && b.type == 0u) {
        TD E[3][3];
        axes(b.q, E);
        if (!sphere_box(a.p, a.h[0], b.p, E, b.h, c)) return false;
        for (int k = 0; k < 3; ++k) c.n[k] = -c.n[k];
        return true;
    }
    if (a.type == 0u && b.type == 1u) {
        TD E[3][3];
        axes(a.q, E);
        return sphere_box(b.p, b.h[0], a.p, E, a.h, c);
    }
    TD A[3][3], Bm[3][3];
    axes(a.q, A);
    axes(b.q, Bm);
    return box_box(a.p, A, a.h, b.p, Bm, b.h, c);
}

// world_inv_inertia (xpbd_solver.cpp:40-70)
void winv(const Body& B, const TD& vx, const TD& vy, const TD& vz, TD& ox, TD& oy, TD& oz) {
    const TD &qw = B.q[0], &qx = B.q[1], &qy = B.q[2], &qz = B.q[3];
    TD R00 = 1.f - 2.f * (qy * qy + qz * qz), R01 = 2.f * (qx * qy + qz * qw), R02 = 2.f * (qx * qz - qy * qw);
    TD R10 = 2.f * (qx * qy - qz * qw), R11 = 1.f - 2.f * (qx * qx + qz * qz), R12 = 2.f * (qy * qz + qx * qw);
    TD R20 = 2.f * (qx * qz + qy * qw), R21 = 2.f * (qy * qz - qx * qw), R22 = 1.f - 2.f * (qx * qx + qy * qy);
    TD lx = R00 * vx + R10 * vy + R20 * vz;
    TD ly = R01 * vx + R11 * vy + R21 * vz;
    TD lz = R02 * vx + R12 * vy + R22 * vz;
    TD ilx = B.I[0] * lx + B.I[3] * ly + B.I[4] * lz;
    TD ily = B.I[3] * lx + B.I[1] * ly + B.I[5] * lz;
    TD ilz = B.I[4] * lx + B.I[5] * ly + B.I[2] * lz;
    ox = R00 * ilx + R01 * ily + R02 * ilz;
    oy = R10 * ilx + R11 * ily + R12 * ilz;
    oz = R20 * ilx + R21 * ily + R22 * ilz;
}

void ang_delta(Body& B, const TD& ax, const TD& ay, const TD& az) {
    if (B.m.f == 0.f) return;
    TD qw = B.q[0], qx = B.q[1], qy = B.q[2], qz = B.q[3];
    B.q[0] = B.q[0] + 0.5f * (-ax * qx - ay * qy - az * qz);
    B.q[1] = B.q[1] + 0.5f * (ax * qw + ay * qz - az * qy);
    B.q[2] = B.q[2] + 0.5f * (-ax * qz + ay * qw + az * qx);
    B.q[3] = B.q[3] + 0.5f * (ax * qy - ay * qx + az * qw);
}

// solve_contact (xpbd_solver.cpp:413-521)
void solve_contact(std::vector<Body>& Bs, const Contact& ct, float mu, TD& lc, float dt) {
    Body &A = Bs[ct.a], &Bb = Bs[ct.b];
    const TD& depth = ct.depth;
    if (depth.f <= 0.f) return;
    TD remaining = depth - lc;
    if (remaining.f <= 1e-6f) return;
    const TD &nx = ct.n[0], &ny = ct.n[1], &nz = ct.n[2];
    const TD &px = ct.p[0], &py = ct.p[1], &pz = ct.p[2];
    TD wa = A.m, wb = Bb.m;
    TD rax = px - A.p[0], ray = py - A.p[1], raz = pz - A.p[2];
    TD rbx = px - Bb.p[0], rby = py - Bb.p[1], rbz = pz - Bb.p[2];
    TD raxnx = ray * nz - raz * ny, raxny = raz * nx - rax * nz, raxnz = rax * ny - ray * nx;
    TD rbxnx = rby * nz - rbz * ny, rbxny = rbz * nx - rbx * nz, rbxnz = rbx * ny - rby * nx;
    TD iIa_x, iIa_y, iIa_z, iIb_x, iIb_y, iIb_z;
    winv(A, raxnx, raxny, raxnz, iIa_x, iIa_y, iIa_z);
    winv(Bb, rbxnx, rbxny, rbxnz, iIb_x, iIb_y, iIb_z);
    TD wa_ang = raxnx * iIa_x + raxny * iIa_y + raxnz * iIa_z;
    TD wb_ang = rbxnx * iIb_x + rbxny * iIb_y + rbxnz * iIb_z;
    TD w_total = wa + wb + wa_ang + wb_ang;
    if (w_total.f < 1e-10f) return;
    TD dl = remaining / w_total;
    lc += remaining;
    if (wa.f != 0.f) { A.p[0] += wa * dl * nx; A.p[1] += wa * dl * ny; A.p[2] += wa * dl * nz; }
    if (wb.f != 0.f) { Bb.p[0] -= wb * dl * nx; Bb.p[1] -= wb * dl * ny; Bb.p[2] -= wb * dl * nz; }
    ang_delta(A, dl * iIa_x, dl * iIa_y, dl * iIa_z);
    ang_delta(Bb, -dl * iIb_x, -dl * iIb_y, -dl * iIb_z);
    {
        TD oax = A.w[0], oay = A.w[1], oaz = A.w[2];
        TD obx = Bb.w[0], oby = Bb.w[1], obz = Bb.w[2];
        TD vcax = A.v[0] + oay * raz - oaz * ray, vcay = A.v[1] + oaz * rax - oax * raz;
        TD vcaz = A.v[2] + oax * ray - oay * rax;
        TD vcbx = Bb.v[0] + oby * rbz - obz * rby, vcby = Bb.v[1] + obz * rbx - obx * rbz;
        TD vcbz = Bb.v[2] + obx * rby - oby * rbx;
        TD vrel_x = vcax - vcbx, vrel_y = vcay - vcby, vrel_z = vcaz - vcbz;
        TD vrel_n = vrel_x * nx + vrel_y * ny + vrel_z * nz;
        if (vrel_n.f < 0.f) {
            TD j_n = -vrel_n / w_total;
            TD dax, day, daz, dbx, dby, dbz;
            winv(A, raxnx, raxny, raxnz, dax, day, daz);
            winv(Bb, rbxnx, rbxny, rbxnz, dbx, dby, dbz);
            if (wa.f != 0.f) {
                A.v[0] += wa * j_n * nx; A.v[1] += wa * j_n * ny; A.v[2] += wa * j_n * nz;
                A.w[0] += j_n * dax; A.w[1] += j_n * day; A.w[2] += j_n * daz;
            }
            if (wb.f != 0.f) {
                Bb.v[0] -= wb * j_n * nx; Bb.v[1] -= wb * j_n * ny; Bb.v[2] -= wb * j_n * nz;
                Bb.w[0] -= j_n * dbx; Bb.w[1] -= j_n * dby; Bb.w[2] -= j_n * dbz;
            }
        }
    }
    if (mu > 0.f) {
        TD oax = A.w[0], oay = A.w[1], oaz = A.w[2];
        TD obx = Bb.w[0], oby = Bb.w[1], obz = Bb.w[2];
        TD vcax = A.v[0] + oay * raz - oaz * ray, vcay = A.v[1] + oaz * rax - oax * raz;
        TD vcaz = A.v[2] + oax * ray - oay * rax;
        TD vcbx = Bb.v[0] + oby * rbz - obz * rby, vcby = Bb.v[1] + obz * rbx - obx * rbz;
        TD vcbz = Bb.v[2] + obx * rby - oby * rbx;
        TD rvx = vcax - vcbx, rvy = vcay - vcby, rvz = vcaz - vcbz;
        TD rvn = rvx * nx + rvy * ny + rvz * nz;
        TD vtx = rvx - rvn * nx, vty = rvy - rvn * ny, vtz = rvz - rvn * nz;
        TD vt2 = vtx * vtx + vty * vty + vtz * vtz;
        if (vt2.f > 1e-12f) {
            TD vt_len = tsqrt(vt2);
            // Where the FP64 slip is exactly zero the float run's slip is
            // rounding noise: the FP64 impulse j_t = |vt| / wt is 0 and the
            // direction is immaterial, so divide by 1 there instead of 0.
            TD dir_len = vt_len;
            if (dir_len.v == 0.0) dir_len.v = 1.0;
            TD tx = vtx / dir_len, ty = vty / dir_len, tz = vtz / dir_len;
            TD ratx = ray * tz - raz * ty, raty = raz * tx - rax * tz, ratz = rax * ty - ray * tx;
            TD rbtx = rby * tz - rbz * ty, rbty = rbz * tx - rbx * tz, rbtz = rbx * ty - rby * tx;
            TD fax, fay, faz, fbx, fby, fbz;
            winv(A, ratx, raty, ratz, fax, fay, faz);
            winv(Bb, rbtx, rbty, rbtz, fbx, fby, fbz);
            TD wt = wa + wb + ratx * fax + raty * fay + ratz * faz + rbtx * fbx + rbty * fby + rbtz * fbz;
            if (wt.f > 1e-10f) {
                TD jns = lc / (dt * w_total);
                TD j_t = vt_len / wt;
                j_t = tmin(j_t, mu * jns);
                if (wa.f != 0.f) {
                    A.v[0] -= wa * j_t * tx; A.v[1] -= wa * j_t * ty; A.v[2] -= wa * j_t * tz;
                    A.w[0] -= j_t * fax; A.w[1] -= j_t * fay; A.w[2] -= j_t * faz;
                }
                if (wb.f != 0.f) {
                    Bb.v[0] += wb * j_t * tx; Bb.v[1] += wb * j_t * ty; Bb.v[2] += wb * j_t * tz;
                    Bb.w[0] += j_t * fbx; Bb.w[1] += j_t * fby; Bb.w[2] += j_t * fbz;
                }
            }
        }
    }
}

}  // namespace

extern "C" {

/* One scene (n bodies) stepped n_frames frames in the sequential order,
 * FP64 tangents for n_params parameters:
 *   kind 0-2 initial velocity x/y/z of body, 3-5 initial spin x/y/z, 6 inverse mass.
 * state13 [13][n] (pos, rot wxyz, vel, ang), inv_mass [n], iI6 [6][n],
 * shape type [n], half extents [3][n], flags [n]. Loss = Σ over bodies with
 * mask[i] of |x_i - target_i|^2. at_float: chain-rule coefficients at the
 * float values instead of the FP64 ones. shift_param >= 0 adds `shift` to
 * that parameter's FP64 value only (central differences of the FP64 re-run
 * along the float run's branches). Outputs: loss (FP64), grad
 * [n_params], final float state [13][n] and FP64 state [13][n]. Returns 0,
 * or -1 when n_params exceeds the tangent limit. */
int dyd_rollout(uint32_t n, const float* state13, const float* inv_mass, const float* iI6, const uint32_t* type,
                const float* half3, const uint32_t* flags, int n_frames, float dt, const float* gravity, int n_sub,
                int n_iters, float mu, int n_params, const int* kind, const uint32_t* body, const float* target3,
                const uint8_t* mask, int at_float, int shift_param, double shift, double* loss, double* grad,
                float* final_f, double* final_v) {
    if (n_params > kMaxT) return -1;
    g_nt = n_params;
    g_at_float = at_float != 0;
    std::vector<Body> Bs(n);
    for (uint32_t i = 0; i < n; ++i) {
        Body& B = Bs[i];
        TD* rows[13] = {&B.p[0], &B.p[1], &B.p[2], &B.q[0], &B.q[1], &B.q[2], &B.q[3],
                        &B.v[0], &B.v[1], &B.v[2], &B.w[0], &B.w[1], &B.w[2]};
        for (int r = 0; r < 13; ++r) *rows[r] = cst(state13[static_cast<size_t>(r) * n + i]);
        B.m = cst(inv_mass[i]);
        for (int k = 0; k < 6; ++k) B.I[k] = iI6[static_cast<size_t>(k) * n + i];
        B.type = type[i];
        B.flags = flags[i];
        for (int k = 0; k < 3; ++k) B.h[k] = half3[static_cast<size_t>(k) * n + i];
    }
    for (int p = 0; p < n_params; ++p) {
        Body& B = Bs[body[p]];
        TD* t = kind[p] < 3 ? &B.v[kind[p]] : (kind[p] < 6 ? &B.w[kind[p] - 3] : &B.m);
        t->d[p] = 1.0;
        if (p == shift_param) t->v += shift;  // FP64 value only: the float path and its branches stay put
    }
    float g[3] = {gravity[0], gravity[1], gravity[2]};
    const float sub_dt = dt / static_cast<float>(n_sub), half_dt = 0.5f * sub_dt;
    std::vector<float> box(6 * n);
    std::vector<Contact> contacts;
    for (int f = 0; f < n_frames; ++f) {
        for (auto& B : Bs) integrate(B, g, sub_dt, half_dt, n_sub);
        for (uint32_t i = 0; i < n; ++i) leaf_box(Bs[i], &box[6 * i]);
        contacts.clear();
        for (uint32_t a = 0; a < n; ++a)
            for (uint32_t b = a + 1; b < n; ++b) {
                if (!overlap(&box[6 * b], &box[6 * a])) continue;
                Contact c;
                if (process_pair(Bs, a, b, c)) contacts.push_back(c);
            }
        if (contacts.empty()) continue;
        std::vector<TD> lam(contacts.size(), cst(0.f));
        for (int it = 0; it < n_iters; ++it) {
            for (size_t c = 0; c < contacts.size(); ++c) solve_contact(Bs, contacts[c], mu, lam[c], dt);
            for (auto& B : Bs) renormalize(B.q);
        }
    }
    TD L = cst(0.f);
    for (uint32_t i = 0; i < n; ++i) {
        if (!mask[i]) continue;
        for (int k = 0; k < 3; ++k) {
            TD e = Bs[i].p[k] - target3[3 * i + k];
            L = L + e * e;
        }
    }
    *loss = L.v;
    for (int p = 0; p < n_params; ++p) grad[p] = L.d[p];
    for (uint32_t i = 0; i < n; ++i) {
        const Body& B = Bs[i];
        const TD* rows[13] = {&B.p[0], &B.p[1], &B.p[2], &B.q[0], &B.q[1], &B.q[2], &B.q[3],
                              &B.v[0], &B.v[1], &B.v[2], &B.w[0], &B.w[1], &B.w[2]};
        for (int r = 0; r < 13; ++r) {
            final_f[static_cast<size_t>(r) * n + i] = rows[r]->f;
            final_v[static_cast<size_t>(r) * n + i] = rows[r]->v;
        }
    }
    return 0;
}

// FP64 re-run of the frame step along the float run's decisions, with the
// solver order of `mode`: 0 the reference's (serial at <= 256 contacts, else
// Jones–Plassmann colours, serial when the colouring fails), 1 serial, 2
// colours at every contact count (core/src/xpbd_solver.cpp:603-733; colours
// from the float run's contact list). Per frame f: err_pos[f] = max over
// bodies of |x_float - x_fp64| (m), err_rot[f] = max over bodies of the
// quaternion component error. With `local`, every frame's FP64 run starts
// from the float state the frame starts from, so err_* is that frame's own
// rounding error; without it the FP64 state is carried and err_* is the
// accumulated error. Final float state and FP64 values as dyd_rollout.
int dyd_fp64_run(uint32_t n, const float* state13, const float* inv_mass, const float* iI6, const uint32_t* type,
                 const float* half3, const uint32_t* flags, int n_frames, float dt, const float* gravity, int n_sub,
                 int n_iters, float mu, int mode, int local, double* err_pos, double* err_rot, float* final_f,
                 double* final_v) {
    g_nt = 0;
    g_at_float = false;
    std::vector<Body> Bs(n);
    for (uint32_t i = 0; i < n; ++i) {
        Body& B = Bs[i];
        TD* rows[13] = {&B.p[0], &B.p[1], &B.p[2], &B.q[0], &B.q[1], &B.q[2], &B.q[3],
                        &B.v[0], &B.v[1], &B.v[2], &B.w[0], &B.w[1], &B.w[2]};
        for (int r = 0; r < 13; ++r) *rows[r] = cst(state13[static_cast<size_t>(r) * n + i]);
        B.m = cst(inv_mass[i]);
        for (int k = 0; k < 6; ++k) B.I[k] = iI6[static_cast<size_t>(k) * n + i];
        B.type = type[i];
        B.flags = flags[i];
        for (int k = 0; k < 3; ++k) B.h[k] = half3[static_cast<size_t>(k) * n + i];
    }
    float g[3] = {gravity[0], gravity[1], gravity[2]};
    const float sub_dt = dt / static_cast<float>(n_sub), half_dt = 0.5f * sub_dt;
    std::vector<float> box(6 * n);
    std::vector<Contact> contacts;
    std::vector<uint32_t> color;
    std::vector<uint64_t> bpri(n), bmask(n);
    for (int f = 0; f < n_frames; ++f) {
        if (local)
            for (auto& B : Bs) {
                TD* rows[13] = {&B.p[0], &B.p[1], &B.p[2], &B.q[0], &B.q[1], &B.q[2], &B.q[3],
                                &B.v[0], &B.v[1], &B.v[2], &B.w[0], &B.w[1], &B.w[2]};
                for (TD* r : rows) r->v = r->f;
            }
        for (auto& B : Bs) integrate(B, g, sub_dt, half_dt, n_sub);
        for (uint32_t i = 0; i < n; ++i) leaf_box(Bs[i], &box[6 * i]);
        contacts.clear();
        for (uint32_t a = 0; a < n; ++a)
            for (uint32_t b = a + 1; b < n; ++b) {
                if (!overlap(&box[6 * b], &box[6 * a])) continue;
                Contact c;
                if (process_pair(Bs, a, b, c)) contacts.push_back(c);
            }
        const uint32_t nc = static_cast<uint32_t>(contacts.size());
        if (nc > 0) {
            // Jones–Plassmann colours of the float run (priorities hash(k) << 32 | k,
            // 8 rounds per batch, at most 256 rounds and 64 colours).
            uint32_t n_colors = 0;
            if (mode == 2 || (mode == 0 && nc > 256u)) {
                const uint32_t UNC = 0xFFFFFFFFu;
                color.assign(nc, UNC);
                std::fill(bmask.begin(), bmask.end(), 0ull);
                uint32_t max_color = 0, rem = nc, r = 0;
                bool overflow = false;
                auto hash_u32 = [](uint32_t x) {
                    x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;
                    return x;
                };
                auto dyn = [&](uint32_t b) { return Bs[b].m.f != 0.f; };
                while (rem > 0 && r < 256u) {
                    for (uint32_t bi = 0; bi < 8u && r < 256u; ++bi, ++r) {
                        std::fill(bpri.begin(), bpri.end(), 0ull);
                        for (uint32_t k = 0; k < nc; ++k) {
                            if (color[k] != UNC) continue;
                            const uint64_t pk = (static_cast<uint64_t>(hash_u32(k)) << 32) | k;
                            const uint32_t a = contacts[k].a, b = contacts[k].b;
                            if (dyn(a) && bpri[a] < pk) bpri[a] = pk;
                            if (dyn(b) && bpri[b] < pk) bpri[b] = pk;
                        }
                        for (uint32_t k = 0; k < nc; ++k) {
                            if (color[k] != UNC) continue;
                            const uint32_t a = contacts[k].a, b = contacts[k].b;
                            const bool da = dyn(a), db = dyn(b);
                            const uint64_t pk = (static_cast<uint64_t>(hash_u32(k)) << 32) | k;
                            if ((da && bpri[a] != pk) || (db && bpri[b] != pk)) continue;
                            const uint64_t used = (da ? bmask[a] : 0ull) | (db ? bmask[b] : 0ull);
                            const uint64_t freebits = ~used;
                            if (freebits == 0ull) {
                                overflow = true;
                                continue;
                            }
                            const uint32_t col = static_cast<uint32_t>(__builtin_ctzll(freebits));
                            color[k] = col;
                            if (da) bmask[a] |= 1ull << col;
                            if (db) bmask[b] |= 1ull << col;
                            max_color = std::max(max_color, col);
                            --rem;
                        }
                    }
                }
                n_colors = (rem > 0 || overflow) ? 0u : max_color + 1u;
            }
            std::vector<TD> lam(nc, cst(0.f));
            for (int it = 0; it < n_iters; ++it) {
                if (n_colors == 0) {
                    for (uint32_t c = 0; c < nc; ++c) solve_contact(Bs, contacts[c], mu, lam[c], dt);
                } else {
                    for (uint32_t ci = 0; ci < n_colors; ++ci)
                        for (uint32_t c = 0; c < nc; ++c)
                            if (color[c] == ci) solve_contact(Bs, contacts[c], mu, lam[c], dt);
                }
                for (auto& B : Bs) renormalize(B.q);
            }
        }
        double ep = 0.0, er = 0.0;
        for (const Body& B : Bs) {
            double d2 = 0.0;
            for (int k = 0; k < 3; ++k) {
                const double d = static_cast<double>(B.p[k].f) - B.p[k].v;
                d2 += d * d;
            }
            ep = std::max(ep, std::sqrt(d2));
            for (int k = 0; k < 4; ++k) er = std::max(er, std::fabs(static_cast<double>(B.q[k].f) - B.q[k].v));
        }
        err_pos[f] = ep;
        err_rot[f] = er;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const Body& B = Bs[i];
        const TD* rows[13] = {&B.p[0], &B.p[1], &B.p[2], &B.q[0], &B.q[1], &B.q[2], &B.q[3],
                              &B.v[0], &B.v[1], &B.v[2], &B.w[0], &B.w[1], &B.w[2]};
        for (int r = 0; r < 13; ++r) {
            final_f[static_cast<size_t>(r) * n + i] = rows[r]->f;
            final_v[static_cast<size_t>(r) * n + i] = rows[r]->v;
        }
    }
    return 0;
}

}  // extern "C"
