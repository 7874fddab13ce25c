// Synthetic scene builders (see scenes.h). Host-only C++20.
#include "scenes.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr float kPi = 3.14159265358979323846f;

struct Builder {
    std::vector<float> pos, rot, vel, ang, mass, inertia, half, bounds, targets;
    std::vector<uint32_t> shape, flags, stype, body_off{0}, shape_off{0};
    uint32_t max_pairs = 0, max_contacts = 0;

    uint32_t add_shape(uint32_t type, float hx, float hy, float hz) {
        stype.push_back(type);
        half.insert(half.end(), {hx, hy, hz});
        return static_cast<uint32_t>(stype.size() - 1);
    }
    void add_body(const float p[3], const float q[4], const float v[3], float m, const float I[3],
                  uint32_t sh, uint32_t fl) {
        pos.insert(pos.end(), p, p + 3);
        rot.insert(rot.end(), q, q + 4);
        vel.insert(vel.end(), v, v + 3);
        ang.insert(ang.end(), {0.f, 0.f, 0.f});
        mass.push_back(m);
        inertia.insert(inertia.end(), {I[0], 0.f, 0.f, 0.f, I[1], 0.f, 0.f, 0.f, I[2]});
        shape.push_back(sh);
        flags.push_back(fl);
        targets.insert(targets.end(), {0.f, 0.f, 0.f});
    }
    void add_ground(uint32_t sh) {
        const float p[3] = {0.f, 0.f, 0.f}, q[4] = {1.f, 0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f};
        const float I[3] = {1.f, 1.f, 1.f};
        add_body(p, q, v, 0.f, I, sh, 1u /* BodyFlag::Static */);
    }
    void end_scene(const float b[6], uint32_t pairs, uint32_t contacts) {
        body_off.push_back(static_cast<uint32_t>(mass.size()));
        shape_off.push_back(static_cast<uint32_t>(stype.size()));
        bounds.insert(bounds.end(), b, b + 6);
        max_pairs = std::max(max_pairs, pairs);
        max_contacts = std::max(max_contacts, contacts);
    }

    template <typename T>
    static T* dup(const std::vector<T>& v) {
        T* p = static_cast<T*>(std::malloc(std::max<size_t>(1, v.size()) * sizeof(T)));
        if (p && !v.empty()) std::memcpy(p, v.data(), v.size() * sizeof(T));
        return p;
    }
    dyph_scene_set* finish(float dt, int32_t n_iters, float mu) {
        auto* s = static_cast<dyph_scene_set*>(std::calloc(1, sizeof(dyph_scene_set)));
        s->n_scenes = static_cast<uint32_t>(body_off.size() - 1);
        s->n_bodies = static_cast<uint32_t>(mass.size());
        s->n_shapes = static_cast<uint32_t>(stype.size());
        s->pos = dup(pos); s->rot = dup(rot); s->vel = dup(vel); s->ang = dup(ang);
        s->mass = dup(mass); s->inertia = dup(inertia); s->shape = dup(shape); s->flags = dup(flags);
        s->shape_type = dup(stype); s->shape_half = dup(half);
        s->body_offset = dup(body_off); s->shape_offset = dup(shape_off);
        s->bounds = dup(bounds); s->targets = dup(targets);
        s->max_pairs = max_pairs; s->max_contacts = max_contacts;
        s->dt = dt; s->n_iters = n_iters; s->friction = mu;
        return s;
    }
};

// Box grid in the reference's loop order (iy outer, ix, iz inner) and formula
// (examples/stress_test_blocks/main.cpp:128-137), scaled by `spacing` and
// jittered per axis (x, y, z draw order).
void grid_positions(int nx, int ny, int nz, int count, float spacing, float base_y, float jitter,
                    std::mt19937_64& rng, std::vector<float>& out) {
    std::uniform_real_distribution<float> U(-jitter, jitter);
    int placed = 0;
    for (int iy = 0; iy < ny && placed < count; ++iy)
        for (int ix = 0; ix < nx && placed < count; ++ix)
            for (int iz = 0; iz < nz && placed < count; ++iz, ++placed) {
                float p[3] = {(ix - nx / 2 + 0.5f) * spacing, base_y + (iy + 1) * spacing,
                              (iz - nz / 2 + 0.5f) * spacing};
                if (jitter > 0.f) {
                    p[0] += U(rng);
                    p[1] += U(rng);
                    p[2] += U(rng);
                }
                out.insert(out.end(), p, p + 3);
            }
}

void shoemake(std::mt19937_64& rng, float q[4]) {
    std::uniform_real_distribution<float> U01(0.f, 1.f);
    float u1 = U01(rng), u2 = U01(rng), u3 = U01(rng);
    float a = std::sqrt(1.f - u1), b = std::sqrt(u1);
    float x = a * std::sin(2.f * kPi * u2), y = a * std::cos(2.f * kPi * u2);
    float z = b * std::sin(2.f * kPi * u3), w = b * std::cos(2.f * kPi * u3);
    float inv = 1.f / std::sqrt(w * w + x * x + y * y + z * z);
    q[0] = w * inv; q[1] = x * inv; q[2] = y * inv; q[3] = z * inv;
}

// One body of the mixed box / sphere distribution (its own shape entry).
void mixed_body(Builder& B, std::mt19937_64& rng, float lo_x, float hi_x, float lo_y, float hi_y, float lo_z,
                float hi_z) {
    std::uniform_real_distribution<float> U01(0.f, 1.f);
    std::normal_distribution<float> N(0.f, 0.5f);
    const float rho = 500.f;
    bool box = U01(rng) < 0.7f;
    float h[3], m, I[3];
    uint32_t sh;
    if (box) {
        std::uniform_real_distribution<float> Uh(0.1f, 0.5f);
        h[0] = Uh(rng); h[1] = Uh(rng); h[2] = Uh(rng);
        m = rho * 8.f * h[0] * h[1] * h[2];
        I[0] = m / 3.f * (h[1] * h[1] + h[2] * h[2]);
        I[1] = m / 3.f * (h[0] * h[0] + h[2] * h[2]);
        I[2] = m / 3.f * (h[0] * h[0] + h[1] * h[1]);
        sh = B.add_shape(0u, h[0], h[1], h[2]);
    } else {
        std::uniform_real_distribution<float> Ur(0.1f, 0.4f);
        float r = Ur(rng);
        m = rho * (4.f / 3.f) * kPi * r * r * r;
        I[0] = I[1] = I[2] = 0.4f * m * r * r;
        sh = B.add_shape(1u, r, r, r);
    }
    std::uniform_real_distribution<float> Ux(lo_x, hi_x), Uy(lo_y, hi_y), Uz(lo_z, hi_z);
    float p[3];
    p[0] = Ux(rng); p[1] = Uy(rng); p[2] = Uz(rng);
    float q[4];
    shoemake(rng, q);
    float v[3];
    v[0] = N(rng); v[1] = N(rng); v[2] = N(rng);
    B.add_body(p, q, v, m, I, sh, 0u);
}

uint32_t log_uniform_count(std::mt19937_64& rng, int lo, int hi) {
    std::uniform_real_distribution<double> U(std::log(double(lo)), std::log(double(hi) + 1.0));
    int n = static_cast<int>(std::floor(std::exp(U(rng))));
    return static_cast<uint32_t>(std::clamp(n, lo, hi));
}

}  // namespace

extern "C" dyph_scene_set* dyph_scene_make(int kind, uint64_t seed, int32_t a0, int32_t a1, int32_t a2,
                                           float spacing, float jitter) {
    Builder B;
    std::mt19937_64 rng(seed);
    const float dt = 1.f / 60.f;
    switch (kind) {
        case DYPH_SCENE_BOX_GRID:
        case DYPH_SCENE_DETERMINISM: {
            const int nx = a0, ny = a1, nz = a2;
            if (nx <= 0 || ny <= 0 || nz <= 0) return nullptr;
            const int n_dyn = nx * ny * nz;
            const bool det = (kind == DYPH_SCENE_DETERMINISM);
            const float BOX_H = 0.4f, GND_HY = 0.5f;
            const float GND_HX = det ? 5.f : std::max(20.f, 0.5f * static_cast<float>(std::max(nx, nz)) + 2.f);
            uint32_t ds = B.add_shape(0u, BOX_H, BOX_H, BOX_H);
            uint32_t gs = B.add_shape(0u, GND_HX, GND_HY, GND_HX);
            const float m = 1.f;
            const float Id = det ? m / 3.f * 2.f * BOX_H * BOX_H : m / 3.f * (BOX_H * BOX_H + BOX_H * BOX_H);
            const float I[3] = {Id, Id, Id};
            std::vector<float> P;
            grid_positions(nx, ny, nz, n_dyn, det ? 1.f : spacing, GND_HY, det ? 0.f : jitter, rng, P);
            const float q[4] = {1.f, 0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f};
            for (int i = 0; i < n_dyn; ++i) B.add_body(&P[3 * i], q, v, m, I, ds, 0u);
            B.add_ground(gs);
            const uint32_t nb = static_cast<uint32_t>(n_dyn + 1);
            if (det) {
                const float b[6] = {-20.f, -2.f, -20.f, 20.f, 30.f, 20.f};
                B.end_scene(b, nb * 32u + 256u, nb * 32u + 256u);
            } else {
                const float bxz = GND_HX + 5.f;
                const float by = std::max(22.f, GND_HY + static_cast<float>(ny) + 5.f);
                const float b[6] = {-bxz, -2.f, -bxz, bxz, by, bxz};
                B.end_scene(b, std::max<uint32_t>(65536u, static_cast<uint32_t>(n_dyn) * 48u),
                            std::max<uint32_t>(16384u, static_cast<uint32_t>(n_dyn) * 16u));
            }
            return B.finish(dt, 10, 0.5f);
        }
        case DYPH_SCENE_RANDOM_PILE: {
            const int n_dyn = a0;
            if (n_dyn <= 0) return nullptr;
            for (int i = 0; i < n_dyn; ++i) mixed_body(B, rng, -20.f, 20.f, 1.5f, 41.5f, -20.f, 20.f);
            B.add_ground(B.add_shape(0u, 40.f, 0.5f, 40.f));
            const float b[6] = {-45.f, -2.f, -45.f, 45.f, 47.f, 45.f};
            B.end_scene(b, std::max<uint32_t>(65536u, static_cast<uint32_t>(n_dyn) * 48u),
                        std::max<uint32_t>(16384u, static_cast<uint32_t>(n_dyn) * 16u));
            return B.finish(dt, 10, 0.5f);
        }
        case DYPH_SCENE_BATCH: {
            const int n_sc = a0;
            if (n_sc <= 0 || a1 <= 0 || a2 < a1) return nullptr;
            std::uniform_real_distribution<float> U01(0.f, 1.f);
            for (int sc = 0; sc < n_sc; ++sc) {
                const int n = static_cast<int>(log_uniform_count(rng, a1, a2));
                const bool boxes = U01(rng) < 0.5f;
                const int k = std::max(1, static_cast<int>(std::lround(std::cbrt(double(n)))));
                const int layers = (n + k * k - 1) / (k * k);
                const float h = 0.4f, sp = 0.85f, gy = 0.5f;
                const float ghx = std::max(3.f, 0.5f * k * sp + 2.f);
                uint32_t ds = boxes ? B.add_shape(0u, h, h, h) : B.add_shape(1u, h, h, h);
                uint32_t gs = B.add_shape(0u, ghx, gy, ghx);
                const float m = boxes ? 1.f : (4.f / 3.f) * kPi * h * h * h / (8.f * h * h * h);
                float I[3];
                if (boxes) I[0] = I[1] = I[2] = m / 3.f * (h * h + h * h);
                else I[0] = I[1] = I[2] = 0.4f * m * h * h;
                std::vector<float> P;
                grid_positions(k, layers, k, n, sp, gy, boxes ? 0.01f : 0.05f, rng, P);
                const float q[4] = {1.f, 0.f, 0.f, 0.f}, v[3] = {0.f, 0.f, 0.f};
                for (int i = 0; i < n; ++i) B.add_body(&P[3 * i], q, v, m, I, ds, 0u);
                B.add_ground(gs);
                const float top = gy + (layers + 1) * sp + 5.f;
                const float b[6] = {-ghx - 5.f, -2.f, -ghx - 5.f, ghx + 5.f, std::max(top, 10.f), ghx + 5.f};
                B.end_scene(b, 48u * n + 64u, 16u * n + 64u);
            }
            return B.finish(dt, 10, 0.5f);
        }
        case DYPH_SCENE_PUSH: {
            const int n_sc = a0;
            if (n_sc <= 0) return nullptr;
            std::normal_distribution<float> N(2.f, 0.3f);
            std::uniform_real_distribution<float> Ut(-0.3f, 0.3f), Uf(0.2f, 1.0f);
            for (int sc = 0; sc < n_sc; ++sc) {
                const float h = 0.2f, sp = 0.41f, gy = 0.5f;
                uint32_t bs = B.add_shape(0u, h, h, h);
                uint32_t ps = B.add_shape(0u, 0.3f, 0.3f, 0.3f);
                uint32_t gs = B.add_shape(0u, 5.f, gy, 5.f);
                const float q[4] = {1.f, 0.f, 0.f, 0.f}, v0[3] = {0.f, 0.f, 0.f};
                const float Ib = 1.f / 3.f * (h * h + h * h);
                const float I[3] = {Ib, Ib, Ib};
                for (int iy = 0; iy < 4; ++iy)
                    for (int ix = 0; ix < 4; ++ix)
                        for (int iz = 0; iz < 4; ++iz) {
                            float p[3] = {(ix - 2 + 0.5f) * sp, gy + h + 0.005f + iy * sp, (iz - 2 + 0.5f) * sp};
                            B.add_body(p, q, v0, 1.f, I, bs, 0u);
                            float* t = &B.targets[B.targets.size() - 3];
                            t[0] = p[0] + Uf(rng);
                            t[1] = p[1] * 0.5f;
                            t[2] = p[2] + Ut(rng);
                        }
                const float Ip = 5.f / 3.f * (0.3f * 0.3f + 0.3f * 0.3f);
                const float Ipv[3] = {Ip, Ip, Ip};
                const float pp[3] = {-1.2f, gy + 0.3f + 0.01f, 0.f};
                const float pv[3] = {N(rng), 0.f, 0.f};
                B.add_body(pp, q, pv, 5.f, Ipv, ps, 0u);
                B.add_ground(gs);
                const float b[6] = {-10.f, -2.f, -10.f, 10.f, 10.f, 10.f};
                B.end_scene(b, 48u * 65u + 64u, 16u * 65u + 64u);
            }
            return B.finish(dt, 10, 0.5f);
        }
        case DYPH_SCENE_BATCH_MIXED: {
            const int n_sc = a0;
            if (n_sc <= 0 || a1 <= 0 || a2 < a1) return nullptr;
            for (int sc = 0; sc < n_sc; ++sc) {
                const int n = static_cast<int>(log_uniform_count(rng, a1, a2));
                const float L = std::max(2.f, static_cast<float>(std::cbrt(double(n))) * 1.2f);
                for (int i = 0; i < n; ++i) mixed_body(B, rng, -0.5f * L, 0.5f * L, 1.5f, 1.5f + L, -0.5f * L, 0.5f * L);
                const float g = 0.5f * L + 2.f;
                B.add_ground(B.add_shape(0u, g, 0.5f, g));
                const float b[6] = {-g - 5.f, -2.f, -g - 5.f, g + 5.f, 1.5f + L + 5.f, g + 5.f};
                B.end_scene(b, 48u * n + 64u, 16u * n + 64u);
            }
            return B.finish(dt, 10, 0.5f);
        }
        default:
            return nullptr;
    }
}

extern "C" void dyph_pack_bodies(uint32_t n, const float* pos, const float* rot, const float* vel,
                                 const float* ang, const float* mass, const float* inertia,
                                 const uint32_t* flags_in, float* st, float* inv_mass, float* iI6,
                                 uint32_t* flags_out) {
    for (uint32_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) st[static_cast<size_t>(k) * n + i] = pos[3 * i + k];
        for (int k = 0; k < 4; ++k) st[static_cast<size_t>(3 + k) * n + i] = rot[4 * i + k];
        for (int k = 0; k < 3; ++k) st[static_cast<size_t>(7 + k) * n + i] = vel[3 * i + k];
        for (int k = 0; k < 3; ++k) st[static_cast<size_t>(10 + k) * n + i] = ang[3 * i + k];
        const bool is_static = (flags_in[i] & 1u) || mass[i] <= 0.f;
        inv_mass[i] = is_static ? 0.f : 1.f / mass[i];
        float out[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (!is_static) {
            const float* d = inertia + 9 * static_cast<size_t>(i);
            const float det = d[0] * (d[4] * d[8] - d[5] * d[7]) - d[1] * (d[3] * d[8] - d[5] * d[6]) +
                              d[2] * (d[3] * d[7] - d[4] * d[6]);
            out[0] = (d[4] * d[8] - d[5] * d[7]) / det;   // (0,0)
            out[1] = (d[0] * d[8] - d[2] * d[6]) / det;   // (1,1)
            out[2] = (d[0] * d[4] - d[1] * d[3]) / det;   // (2,2)
            out[3] = -(d[1] * d[8] - d[2] * d[7]) / det;  // (0,1)
            out[4] = (d[1] * d[5] - d[2] * d[4]) / det;   // (0,2)
            out[5] = -(d[0] * d[5] - d[2] * d[3]) / det;  // (1,2)
        }
        for (int k = 0; k < 6; ++k) iI6[static_cast<size_t>(k) * n + i] = out[k];
        flags_out[i] = is_static ? (flags_in[i] | 1u) : flags_in[i];
    }
}

extern "C" void dyph_scene_free(dyph_scene_set* s) {
    if (!s) return;
    void* p[] = {s->pos, s->rot, s->vel, s->ang, s->mass, s->inertia, s->shape, s->flags, s->shape_type,
                 s->shape_half, s->body_offset, s->shape_offset, s->bounds, s->targets};
    for (void* q : p) std::free(q);
    std::free(s);
}
