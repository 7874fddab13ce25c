// Adjoint of one fused frame of batched scenes (included after
// scene_frame.cuh: by world.cu, whose scene_frame_record_kernel runs
// record_scene, and by reverse.cu, whose scene_frame_reverse_kernel runs
// reverse_scene), in two kernels so that one checkpoint segment's recording
// runs while the next one's reverse pass does (they touch different record
// sets):
//   record:  recompute the frame from its starting state (frame_scene with an
//            AdjRun), recording the pose after integrate, every contact's
//            narrowphase branch, every acting contact's pre-solve body states
//            and the quaternions before the renormalisations — the contact
//            set and all branches are those of the forward frame — keep the
//            scene's contact words (pairs, groups, geometry) in global
//            memory, and store the frame's end state when asked;
//   reverse: reverse the renormalisations, then the contact solves group by
//            group in descending order (a group's contacts share no dynamic
//            body), each with solve_contact_adj on its recorded pre-solve
//            state, then the narrowphase (contact geometry -> the two bodies'
//            poses after integrate) and the integration.
// The adjoint of the state at the frame's end comes in, the adjoint of the
// state at its start goes out, and the inverse masses' adjoints accumulate.
#pragma once

#include "adjoint_math.cuh"

namespace dyph {
namespace {

// process_pair's adjoint: contact (point, normal, depth) adjoints -> adjoints
// of the two bodies' poses. ta / tb are the shape types, br the branch word.
__device__ __forceinline__ void process_pair_adj(uint32_t ta, uint32_t tb, F3 xa, const float qa[4], const float ha[3],
                                                 F3 xb, const float qb[4], const float hb[3], uint32_t br, F3 n,
                                                 F3 pbar, F3 nbar, float dbar, F3& xab, float qab[4], F3& xbb,
                                                 float qbb[4]) {
    if (ta == kShapeSphere && tb == kShapeSphere) {
        sphere_sphere_adj(xa, ha[0], xb, hb[0], br, pbar, nbar, dbar, xab, xbb);
    } else if (ta == kShapeSphere && tb == kShapeBox) {
        sphere_box_adj(xa, ha[0], xb, qb, hb, br, pbar, -nbar, dbar, xab, xbb, qbb);  // normal flipped
    } else if (ta == kShapeBox && tb == kShapeSphere) {
        sphere_box_adj(xb, hb[0], xa, qa, ha, br, pbar, nbar, dbar, xbb, xab, qab);
    } else {
        box_box_adj(xa, qa, ha, xb, qb, hb, br, n, pbar, nbar, dbar, xab, qab, xbb, qbb);
    }
}

struct AdjFrame {
    const float* gin;   // [13][n_stride] adjoint of the state at the frame's end
    float* gout;        // [13][n_stride] adjoint of the state at the frame's start (work array)
    float* gim;         // [n] inverse-mass adjoints, accumulated
};

__device__ __forceinline__ float& grow(float* g, uint32_t stride, int r, uint32_t i) {
    return g[static_cast<size_t>(r) * stride + i];
}

// A recorded frame's contact words and counts, kept for the reverse pass.
struct AdjKeep {
    uint32_t* words;  // [kSceneWords][words_stride], the layout of FrameBufs::words
    uint32_t* mg;     // [2 n_scenes] contacts and groups of every scene
};

// Recomputation of scene s's frame with recording (team T, `smem_bytes` of
// shared memory at smem); F.words is K.words, so a scene whose words spill
// writes them in place and the others copy theirs out.
template <class Team>
__device__ void record_scene(const Team& T, uint32_t s, unsigned char* smem, uint32_t smem_bytes, SceneShared& sh,
                             const SceneBufs& S, const FrameBufs& F, const FrameParams& P_, const AdjRun& A,
                             const AdjKeep& K) {
    FrameOut fo{};
    const bool ok = frame_scene<true>(T, s, smem, smem_bytes, sh, S, F, P_, &A, &fo);
    const uint32_t m = ok ? fo.m : 0u, groups = ok ? fo.groups : 0u;
    const SceneContacts dst{K.words + F.contact_base[s] + s, F.words_stride};
    const SceneContacts& SC = fo.SC;
    if (ok && m > 0 && SC.w != dst.w) {
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            dst.ab(k) = SC.ab(k);
            dst.ent(k) = SC.ent(k);
#pragma unroll
            for (int r = 0; r < 7; ++r) dst.g(r, k) = SC.g(r, k);
        }
        for (uint32_t g = T.rank(); g <= groups; g += T.size()) dst.pa(g) = SC.pa(g);
    }
    if (T.leader()) {
        K.mg[2 * s] = m;
        K.mg[2 * s + 1] = groups;
    }
    T.sync();
}

// The reverse pass of scene s's recorded frame by team T.
template <class Team>
__device__ void reverse_scene(const Team& T, uint32_t s, unsigned char* smem, uint32_t smem_bytes, SceneShared& sh,
                              const SceneBufs& S, const FrameBufs& F, const FrameParams& P_, const AdjRun& A,
                              const AdjKeep& K, const AdjFrame& G) {
    const uint32_t ns = A.n_stride, rs = A.rec_stride;
    const uint32_t b0 = S.body_offset[s], nb = S.body_offset[s + 1] - b0;
    const uint32_t ldb = (nb + 3u) & ~3u;
    float* fb = reinterpret_cast<float*>(smem);
    const SceneBodies SB{fb, ldb};
    const SceneSolverRows R = scene_solver_rows(fb, ldb);
    uint32_t* info = R.cnt + ldb;
    float* half = reinterpret_cast<float*>(info + ldb);
    // the bodies' constant rows, shape types, flags and half extents
    {
        const GlobalBodies B{P_.gb};
        for (uint32_t i = T.rank(); i < nb; i += T.size()) {
            const uint32_t g = b0 + i, sh_i = P_.gb.shape[g];
            fb[13 * ldb + i] = B.im(g);
            fb[14 * ldb + i] = B.ixx(g); fb[15 * ldb + i] = B.iyy(g); fb[16 * ldb + i] = B.izz(g);
            fb[17 * ldb + i] = B.ixy(g); fb[18 * ldb + i] = B.ixz(g); fb[19 * ldb + i] = B.iyz(g);
            info[i] = P_.gs.type[sh_i] | (P_.gb.flags[g] << 8);
            half[i] = P_.gs.half_x[sh_i];
            half[ldb + i] = P_.gs.half_y[sh_i];
            half[2 * ldb + i] = P_.gs.half_z[sh_i];
        }
    }
    // the kept contact words, staged in shared memory after the bodies when
    // they fit (the group loops below read them on their critical path)
    const SceneContacts KC{K.words + F.contact_base[s] + s, F.words_stride};
    const uint32_t m = K.mg[2 * s], n_groups = K.mg[2 * s + 1], cbase = F.contact_base[s];
    const uint32_t ldc = (m + 4u) & ~3u;
    const bool staged = frame_body_bytes(nb) + kSceneWords * 4u * ldc <= smem_bytes;
    const SceneContacts SC = staged ? SceneContacts{reinterpret_cast<uint32_t*>(smem + frame_body_bytes(nb)), ldc} : KC;
    if (staged) {
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            SC.ab(k) = KC.ab(k);
            SC.ent(k) = KC.ent(k);
#pragma unroll
            for (int r = 0; r < 7; ++r) SC.g(r, k) = KC.g(r, k);
        }
        for (uint32_t g = T.rank(); g <= n_groups; g += T.size()) SC.pa(g) = KC.pa(g);
    }
    // The scene's contact records, staged after the contact words when both
    // fit: rows 0-27 and 35 (poses before each solve, geometry, the solve's
    // flags) are read once per contact, one dependency level after another;
    // rows 28-34 and 0-13 are rewritten below and read back from there.
    const uint32_t rec_off = frame_body_bytes(nb) + kSceneWords * 4u * ldc;
    const bool rec_staged = staged && rec_off + kRecWords * 4u * ldc <= smem_bytes;
    float* const recb = rec_staged ? reinterpret_cast<float*>(smem + rec_off) : A.rec + cbase;
    const size_t rst = rec_staged ? ldc : rs;
    if (rec_staged)
        for (uint32_t e = T.rank(); e < 29u * m; e += T.size()) {
            const uint32_t q = e / m, k = e - q * m, row = q < 28u ? q : 35u;
            recb[static_cast<size_t>(row) * ldc + k] = A.rec[cbase + k + static_cast<size_t>(row) * rs];
        }
    T.sync();
    // ── adjoint of the frame's end state ──
    for (uint32_t i = T.rank(); i < nb; i += T.size())
        for (int r = 0; r < 13; ++r) grow(G.gout, ns, r, b0 + i) = G.gin[static_cast<size_t>(r) * ns + b0 + i];
    T.sync();
    if (m > 0) {
        // ── renormalisations: q_end = renorm^n_iters(q_sweeps) ──
        for (uint32_t i = T.rank(); i < nb; i += T.size()) {
            float q[4] = {A.qs[b0 + i], A.qs[ns + b0 + i], A.qs[2ull * ns + b0 + i], A.qs[3ull * ns + b0 + i]};
            float chain[10][4];
            const int n_it = P_.n_iters;
            int kept = 0;
            for (int it = 0; it < n_it && it < 10; ++it) {
                for (int c = 0; c < 4; ++c) chain[it][c] = q[c];
                renormalize(q[0], q[1], q[2], q[3]);
                ++kept;
            }
            if (n_it > 10) atomicOr(A.flag, 2u);
            float g[4] = {grow(G.gout, ns, 3, b0 + i), grow(G.gout, ns, 4, b0 + i), grow(G.gout, ns, 5, b0 + i),
                          grow(G.gout, ns, 6, b0 + i)};
            for (int it = kept - 1; it >= 0; --it) {
                float gi[4];
                normalize_adj(chain[it], g, gi);
                for (int c = 0; c < 4; ++c) g[c] = gi[c];
            }
            for (int c = 0; c < 4; ++c) grow(G.gout, ns, 3 + c, b0 + i) = g[c];
        }
        T.sync();
        // ── contact solves, last group first ──
        for (int g = static_cast<int>(n_groups) - 1; g >= 0; --g) {
            const uint32_t end = SC.pa(g + 1);
            for (uint32_t idx = SC.pa(g) + T.rank(); idx < end; idx += T.size()) {
                const uint32_t k = SC.ent(idx);
                const float* r = recb + k;
                if (r[35ull * rst] == 0.f) continue;  // did not act
                const Contact ct = SC.contact(k);
                const uint32_t ia = ct.a, ib = ct.b;
                LocalPair L;
                for (int j = 0; j < 2; ++j) {
                    const uint32_t bi = j ? ib : ia;
                    const int o = j ? 13 : 0;
                    for (int c = 0; c < 3; ++c) L.p[j][c] = r[static_cast<size_t>(o + c) * rst];
                    for (int c = 0; c < 4; ++c) L.q[j][c] = r[static_cast<size_t>(o + 3 + c) * rst];
                    for (int c = 0; c < 3; ++c) L.v[j][c] = r[static_cast<size_t>(o + 7 + c) * rst];
                    for (int c = 0; c < 3; ++c) L.w[j][c] = r[static_cast<size_t>(o + 10 + c) * rst];
                    L.m[j] = SB.im(bi);
                    L.I[j][0] = SB.ixx(bi); L.I[j][1] = SB.iyy(bi); L.I[j][2] = SB.izz(bi);
                    L.I[j][3] = SB.ixy(bi); L.I[j][4] = SB.ixz(bi); L.I[j][5] = SB.iyz(bi);
                }
                BodyBar G0, G1;
                BodyBar* Gs[2] = {&G0, &G1};
                for (int j = 0; j < 2; ++j) {
                    const uint32_t gi = b0 + (j ? ib : ia);
                    BodyBar& Gj = *Gs[j];
                    Gj.x = f3(grow(G.gout, ns, 0, gi), grow(G.gout, ns, 1, gi), grow(G.gout, ns, 2, gi));
                    for (int c = 0; c < 4; ++c) Gj.q[c] = grow(G.gout, ns, 3 + c, gi);
                    Gj.v = f3(grow(G.gout, ns, 7, gi), grow(G.gout, ns, 8, gi), grow(G.gout, ns, 9, gi));
                    Gj.w = f3(grow(G.gout, ns, 10, gi), grow(G.gout, ns, 11, gi), grow(G.gout, ns, 12, gi));
                    Gj.im = 0.f;
                }
                F3 pb = f3(0.f, 0.f, 0.f), nb3 = pb;
                float db = 0.f;
                solve_contact_adj(L, ct, P_.mu, P_.dt, r[26ull * rst], __float_as_uint(r[35ull * rst]), G0, G1, pb,
                                  nb3, db);
                for (int j = 0; j < 2; ++j) {
                    if (L.m[j] == 0.f) continue;  // a static body's state is not a variable
                    const uint32_t gi = b0 + (j ? ib : ia);
                    const BodyBar& Gj = *Gs[j];
                    grow(G.gout, ns, 0, gi) = Gj.x.x; grow(G.gout, ns, 1, gi) = Gj.x.y;
                    grow(G.gout, ns, 2, gi) = Gj.x.z;
                    for (int c = 0; c < 4; ++c) grow(G.gout, ns, 3 + c, gi) = Gj.q[c];
                    grow(G.gout, ns, 7, gi) = Gj.v.x; grow(G.gout, ns, 8, gi) = Gj.v.y;
                    grow(G.gout, ns, 9, gi) = Gj.v.z;
                    grow(G.gout, ns, 10, gi) = Gj.w.x; grow(G.gout, ns, 11, gi) = Gj.w.y;
                    grow(G.gout, ns, 12, gi) = Gj.w.z;
                    G.gim[gi] += Gj.im;
                }
                float* w = recb + k;
                w[28ull * rst] = pb.x; w[29ull * rst] = pb.y; w[30ull * rst] = pb.z;
                w[31ull * rst] = nb3.x; w[32ull * rst] = nb3.y; w[33ull * rst] = nb3.z;
                w[34ull * rst] = db;
            }
            T.sync();
        }
        // ── narrowphase: geometry adjoints -> poses after integrate ──
        // Each acting contact's adjoints for its two bodies go to its record
        // (rows 0-13, free once the solve's adjoint has run); then every body
        // adds its contacts' adjoints in contact order. Each sum is taken in
        // one fixed order without atomics, so the gradients are the same from
        // run to run, bit for bit, and no barrier is needed per group.
        // Per-body lists of acting contacts (both sides, dynamic bodies):
        // counts, scan, fill, sort; entries in the free pb / done rows.
        auto entry = [&](uint32_t e) -> uint32_t& { return e < m ? SC.pb(e) : SC.done(e - m); };
        for (uint32_t i = T.rank(); i < nb; i += T.size()) R.cnt[i] = 0u;
        T.sync();
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            if (recb[k + 35ull * rst] == 0.f) continue;
            const uint32_t ab = SC.ab(k), a = ab & 0xFFFFu, b = ab >> 16;
            if (SB.im(a) != 0.f) atomicAdd(&R.cnt[a], 1u);
            if (SB.im(b) != 0.f) atomicAdd(&R.cnt[b], 1u);
        }
        if (T.leader()) sh.carry = 0u;
        T.sync();
        for (uint32_t base = 0; base < nb; base += T.size()) {
            const uint32_t i = base + T.rank();
            uint32_t tot;
            const uint32_t ex = T.exclusive_scan(i < nb ? R.cnt[i] : 0u, sh.scan, tot);
            if (i < nb) {
                R.off[i] = sh.carry + ex;
                R.cnt[i] = 0u;
            }
            T.sync();
            if (T.leader()) sh.carry += tot;
            T.sync();
        }
        if (T.leader()) R.off[nb] = sh.carry;
        T.sync();
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            if (recb[k + 35ull * rst] == 0.f) continue;
            const uint32_t ab = SC.ab(k), a = ab & 0xFFFFu, b = ab >> 16;
            if (SB.im(a) != 0.f) entry(R.off[a] + atomicAdd(&R.cnt[a], 1u)) = k;
            if (SB.im(b) != 0.f) entry(R.off[b] + atomicAdd(&R.cnt[b], 1u)) = k;
        }
        T.sync();
        for (uint32_t x = T.rank(); x < nb; x += T.size()) {
            const uint32_t lo = R.off[x], hi = R.off[x + 1];
            for (uint32_t i = lo + 1; i < hi; ++i) {
                const uint32_t v = entry(i);
                uint32_t j = i;
                while (j > lo && entry(j - 1) > v) {
                    entry(j) = entry(j - 1);
                    --j;
                }
                entry(j) = v;
            }
        }
        // the contacts' geometry adjoints, into their records
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            float* r = recb + k;
            if (r[35ull * rst] == 0.f) continue;  // a contact that did not act has no effect
            const Contact ct = SC.contact(k);
            const uint32_t ia = ct.a, ib = ct.b;
            const uint32_t ga = b0 + ia, gbi = b0 + ib;
            const F3 xa = f3(A.pose1[ga], A.pose1[ns + ga], A.pose1[2ull * ns + ga]);
            const F3 xb = f3(A.pose1[gbi], A.pose1[ns + gbi], A.pose1[2ull * ns + gbi]);
            const float qa[4] = {A.pose1[3ull * ns + ga], A.pose1[4ull * ns + ga], A.pose1[5ull * ns + ga],
                                 A.pose1[6ull * ns + ga]};
            const float qb[4] = {A.pose1[3ull * ns + gbi], A.pose1[4ull * ns + gbi], A.pose1[5ull * ns + gbi],
                                 A.pose1[6ull * ns + gbi]};
            const float ha[3] = {half[ia], half[ldb + ia], half[2 * ldb + ia]};
            const float hb[3] = {half[ib], half[ldb + ib], half[2 * ldb + ib]};
            F3 xab = f3(0.f, 0.f, 0.f), xbb = xab;
            float qab[4] = {0.f, 0.f, 0.f, 0.f}, qbb[4] = {0.f, 0.f, 0.f, 0.f};
            process_pair_adj(info[ia] & 0xFFu, info[ib] & 0xFFu, xa, qa, ha, xb, qb, hb,
                             __float_as_uint(r[27ull * rst]), f3(ct.nx, ct.ny, ct.nz),
                             f3(r[28ull * rst], r[29ull * rst], r[30ull * rst]),
                             f3(r[31ull * rst], r[32ull * rst], r[33ull * rst]), r[34ull * rst], xab, qab, xbb, qbb);
            const float out[14] = {xab.x, xab.y, xab.z, qab[0], qab[1], qab[2], qab[3],
                                   xbb.x, xbb.y, xbb.z, qbb[0], qbb[1], qbb[2], qbb[3]};
#pragma unroll
            for (int c = 0; c < 14; ++c) r[static_cast<size_t>(c) * rst] = out[c];
        }
        T.sync();
        // every body's sum over its contacts, in contact order
        for (uint32_t x = T.rank(); x < nb; x += T.size()) {
            const uint32_t lo = R.off[x], hi = R.off[x + 1];
            if (lo == hi) continue;
            const uint32_t gx = b0 + x;
            float acc[7];
#pragma unroll
            for (int c = 0; c < 7; ++c) acc[c] = grow(G.gout, ns, c, gx);
            for (uint32_t e = lo; e < hi; ++e) {
                const uint32_t k = entry(e);
                const uint32_t side = (SC.ab(k) & 0xFFFFu) == x ? 0u : 7u;
                const float* r = recb + k;
#pragma unroll
                for (int c = 0; c < 7; ++c) acc[c] += r[static_cast<size_t>(side + c) * rst];
            }
#pragma unroll
            for (int c = 0; c < 7; ++c) grow(G.gout, ns, c, gx) = acc[c];
        }
        T.sync();
    }
    // ── integration, from the state at the frame's start ──
    const GlobalBodies B0{P_.gb};
    for (uint32_t i = T.rank(); i < nb; i += T.size()) {
        const uint32_t gi = b0 + i;
        if (SB.im(i) == 0.f) {
            for (int r = 0; r < 13; ++r) grow(G.gout, ns, r, gi) = 0.f;
            continue;
        }
        if ((info[i] >> 8) & kFlagSleeping) continue;  // not integrated: identity
        const Pose p0{B0.px(gi), B0.py(gi), B0.pz(gi), B0.qw(gi), B0.qx(gi), B0.qy(gi), B0.qz(gi),
                      B0.vx(gi), B0.vy(gi), B0.vz(gi)};
        F3 xb = f3(grow(G.gout, ns, 0, gi), grow(G.gout, ns, 1, gi), grow(G.gout, ns, 2, gi));
        float qb[4] = {grow(G.gout, ns, 3, gi), grow(G.gout, ns, 4, gi), grow(G.gout, ns, 5, gi),
                       grow(G.gout, ns, 6, gi)};
        F3 vb = f3(grow(G.gout, ns, 7, gi), grow(G.gout, ns, 8, gi), grow(G.gout, ns, 9, gi));
        F3 wb = f3(grow(G.gout, ns, 10, gi), grow(G.gout, ns, 11, gi), grow(G.gout, ns, 12, gi));
        if (!integrate_body_adj(p0, B0.wx(gi), B0.wy(gi), B0.wz(gi), P_.gx, P_.gy, P_.gz, P_.sub_dt, P_.half_dt,
                                P_.n_substeps, xb, qb, vb, wb))
            atomicOr(A.flag, 4u);
        grow(G.gout, ns, 0, gi) = xb.x; grow(G.gout, ns, 1, gi) = xb.y; grow(G.gout, ns, 2, gi) = xb.z;
        for (int c = 0; c < 4; ++c) grow(G.gout, ns, 3 + c, gi) = qb[c];
        grow(G.gout, ns, 7, gi) = vb.x; grow(G.gout, ns, 8, gi) = vb.y; grow(G.gout, ns, 9, gi) = vb.z;
        grow(G.gout, ns, 10, gi) = wb.x; grow(G.gout, ns, 11, gi) = wb.y; grow(G.gout, ns, 12, gi) = wb.z;
    }
    T.sync();
}

// Work items as for scene_frame_kernel: a large scene per block, two
// mid-size scenes on two warps each, or up to four small scenes, one per warp.
template <class Fn>
__device__ __forceinline__ void for_each_item(const uint32_t* items, uint32_t n_items, uint32_t smem_bytes, Fn&& fn) {
    extern __shared__ __align__(16) unsigned char scene_smem[];
    __shared__ SceneShared sh[kSceneThreads / 32];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t share = (smem_bytes / 4u) & ~15u;
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
        const uint32_t kind = items[4 * it + 1];
        if (kind == kItemBlock) {
            fn(BlockTeam{}, items[4 * it], scene_smem, smem_bytes, sh[0]);
        } else if (kind == kItemHalf) {
            const uint32_t half = warp >> 1, s = items[4 * it + 2 * half];
            if (s != kItemEmpty) fn(HalfTeam{half}, s, scene_smem + half * 2u * share, 2u * share, sh[2 * half]);
        } else {
            const uint32_t s = items[4 * it + warp];
            if (s != kItemEmpty) fn(WarpTeam{}, s, scene_smem + warp * share, share, sh[warp]);
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace dyph
