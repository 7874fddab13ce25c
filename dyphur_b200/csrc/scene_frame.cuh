// Batched scenes, fused: one thread block runs a whole frame of one scene —
// integrate, pair search, narrowphase and contact solve — on the scene's
// bodies in shared memory, and writes the bodies back once. Included by
// world.cu (after solver.cu in the library's translation unit).
//
// Every stage is the single-scene stage restated for one block:
//   * integrate: integrate_body per dynamic, awake body (core/src/
//     integrator.cpp:18-68), all substeps in registers;
//   * pairs: the candidate-pair set is the set of body pairs whose fp16 leaf
//     boxes (core/src/broadphase.cpp:216-251) overlap under the traversal's
//     inclusive test (:322-325), because internal nodes merge the leaf boxes
//     exactly. So every (a, b) with a < b is tested directly and the pairs
//     come out in ascending (a << 32 | b) order, as Broadphase::sort_pairs
//     leaves them; a scene keeps the first max_pairs of them, as it does alone;
//   * narrowphase: process_pair (core/src/narrowphase.cpp:920-1001) per pair,
//     contacts compacted in pair order, the first max_contacts kept;
//   * solve: scene_solve (solver_scene.cuh).
// A scene's frame is therefore bit-identical to the frame of the scene
// stepped alone. The frame's pair and contact lists stay in per-scene slots
// and are compacted into the broadphase's / narrowphase's lists on request
// (scene_gather_*).
#pragma once

#include "solver_scene.cuh"

namespace dyph {
namespace {

// Per-body rows the fused frame adds after the solver's rows: shape type and
// flags, half extents (3), leaf box (6 floats).
constexpr uint32_t kFrameBodyRows = 10;

__host__ __device__ __forceinline__ uint32_t frame_body_bytes(uint32_t nb) {
    const uint32_t ldb = (nb + 3u) & ~3u;
    return scene_body_bytes(nb) + kFrameBodyRows * 4u * ldb;
}

// Overlap bits of the candidate-pair search: body a has ceil((nb - 1 - a) /
// 32) words, one per chunk of 32 partners b > a, laid out by ascending a.
// S(t) = sum over u = 1..t of ceil(u / 32) = 16 q (q + 1) + (q + 1) r, t = 32 q + r.
__host__ __device__ __forceinline__ uint32_t chunk_prefix(uint32_t t) {
    const uint32_t q = t >> 5, r = t & 31u;
    return 16u * q * (q + 1u) + (q + 1u) * r;
}
__host__ __device__ __forceinline__ uint32_t overlap_mask_words(uint32_t nb) {
    return nb ? chunk_prefix(nb - 1u) : 0u;
}
__host__ __device__ __forceinline__ uint32_t overlap_mask_base(uint32_t nb, uint32_t a) {
    return chunk_prefix(nb - 1u) - chunk_prefix(nb - 1u - a);
}

struct FrameBufs {
    const uint32_t* pair_base;     // [n_scenes + 1] first pair slot of each scene (capacity 48 n + 64)
    const uint32_t* contact_base;  // [n_scenes + 1] first contact slot of each scene (capacity 16 n + 64)
    uint32_t* pair_raw;            // [total pair slots] a | b << 16 (local indices)
    uint32_t* contact_raw;         // [9][total contact slots] a, b (global), position, normal, depth
    uint32_t* color_raw;           // [total contact slots] colour (UINT32_MAX on the sequential order)
    uint32_t* counts;              // [4 n_scenes] stored pairs, true pairs, stored contacts, true contacts
    uint32_t* words;               // [kSceneWords][words_stride] contact words of scenes too big for shared memory
    uint32_t words_stride;         // total contact slots + n_scenes
    uint32_t contact_slots;        // total contact slots
};

// Shape rows of one scene in shared memory, indexed by local body (each body
// carries its own shape's type and half extents).
struct SceneShapes {
    const uint32_t* info;  // type | flags << 8
    const float* half;     // 3 rows
    uint32_t ld;
    __device__ __forceinline__ uint32_t type(uint32_t i) const { return info[i] & 0xFFu; }
    __device__ __forceinline__ float hx(uint32_t i) const { return half[i]; }
    __device__ __forceinline__ float hy(uint32_t i) const { return half[ld + i]; }
    __device__ __forceinline__ float hz(uint32_t i) const { return half[2 * ld + i]; }
};

struct SceneBodiesShaped : SceneBodies {
    __device__ __forceinline__ uint32_t shape(uint32_t i) const { return i; }
};

// Per-frame parameters of the fused kernel.
struct FrameParams {
    dyph_bodies gb;
    dyph_shapes gs;
    float gx, gy, gz, sub_dt, half_dt, mu, dt;
    int n_substeps, mode, n_iters;
    uint32_t* meta;
    uint32_t* bp_counts;
    uint32_t* np_counts;
    uint32_t* status;
    unsigned long long* phase_ns;  // null, or [kFramePhases] device-clock ns summed over scenes
};

// Phases of a scene's fused frame, timed per scene by its team leader when
// phase_ns is set: 0 staging + integrate + leaf boxes, 1 pair search,
// 2 narrowphase, 3 contact-solve set-up (lists, colours or levels, groups),
// 4 sweep + renormalisation, 5 write-back.
constexpr int kFramePhases = 6;

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

template <class Team>
__device__ __forceinline__ void phase_mark(const Team& T, const FrameParams& P_, int k, uint64_t& t0) {
    if (P_.phase_ns && T.leader()) {
        const uint64_t t = global_ns();
        atomicAdd(&P_.phase_ns[k], static_cast<unsigned long long>(t - t0));
        t0 = t;
    }
}

// Recording for the adjoint pass (frame_scene with `adj`): the frame is
// recomputed from the given state, its branches and intermediates recorded,
// and nothing is reported; the end state goes to `store` when it is set (the
// given state is left as it was).
struct AdjRun {
    float* rec;          // [kRecWords][rec_stride] per-contact records, slot = contact slot of the scene
    uint32_t rec_stride;
    float* pose1;        // [7][n_stride] pose after integrate (x, q)
    float* qs;           // [4][n_stride] quaternions after the sweeps, before the renormalisations
    uint32_t n_stride;
    uint32_t* flag;      // unsupported paths
    float* store;        // [13][n_stride] the frame's end state (x, q, v, w), or null
};

// What the adjoint pass needs of a recomputed frame.
struct FrameOut {
    SceneContacts SC;
    uint32_t m, groups;
};

// One frame of scene s by team T with `smem_bytes` of shared memory at smem.
// Returns false after raising an error. kRecord compiles the adjoint's
// recording in (`adj_in`, `out`); the forward frame is built without it.
template <bool kRecord = false, class Team>
__device__ bool frame_scene(const Team& T, uint32_t s, unsigned char* smem, uint32_t smem_bytes, SceneShared& sh,
                            const SceneBufs& S, const FrameBufs& F, const FrameParams& P_,
                            const AdjRun* adj_in = nullptr, FrameOut* out = nullptr) {
    const AdjRun* const adj = kRecord ? adj_in : nullptr;
    const GlobalBodies B{P_.gb};
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t t0 = P_.phase_ns ? global_ns() : 0u;
    const uint32_t b0 = S.body_offset[s], nb = S.body_offset[s + 1] - b0;
    const uint32_t ldb = (nb + 3u) & ~3u;
    float* fb = reinterpret_cast<float*>(smem);
    const SceneSolverRows R = scene_solver_rows(fb, ldb);
    uint32_t* info = R.cnt + ldb;
    float* half = reinterpret_cast<float*>(info + ldb);
    float* box = half + 3 * ldb;  // rows mnx, mny, mnz, mxx, mxy, mxz
    const SceneBodiesShaped SB{{fb, ldb}};
    const SceneShapes SS{info, half, ldb};
    const uint32_t pcap = F.pair_base[s + 1] - F.pair_base[s];
    const uint32_t ccap = F.contact_base[s + 1] - F.contact_base[s];
    // ── stage and integrate ──
    scene_load_bodies(T, B, b0, nb, fb, ldb);
    for (uint32_t i = T.rank(); i < nb; i += T.size()) {
        const uint32_t g = b0 + i, sh_i = P_.gb.shape[g];
        info[i] = P_.gs.type[sh_i] | (P_.gb.flags[g] << 8);
        half[i] = P_.gs.half_x[sh_i];
        half[ldb + i] = P_.gs.half_y[sh_i];
        half[2 * ldb + i] = P_.gs.half_z[sh_i];
        if (SB.im(i) != 0.f && !((info[i] >> 8) & kFlagSleeping)) {
            Pose p{SB.px(i), SB.py(i), SB.pz(i), SB.qw(i), SB.qx(i), SB.qy(i), SB.qz(i),
                   SB.vx(i), SB.vy(i), SB.vz(i)};
            const float ox = SB.wx(i), oy = SB.wy(i), oz = SB.wz(i);
            for (int k = 0; k < P_.n_substeps; ++k)
                integrate_body(p, ox, oy, oz, P_.gx, P_.gy, P_.gz, P_.sub_dt, P_.half_dt);
            SB.px(i) = p.px; SB.py(i) = p.py; SB.pz(i) = p.pz;
            SB.qw(i) = p.qw; SB.qx(i) = p.qx; SB.qy(i) = p.qy; SB.qz(i) = p.qz;
            SB.vx(i) = p.vx; SB.vy(i) = p.vy; SB.vz(i) = p.vz;
        }
        if (adj) {
            float* r = adj->pose1 + b0 + i;
            const float v[7] = {SB.px(i), SB.py(i), SB.pz(i), SB.qw(i), SB.qx(i), SB.qy(i), SB.qz(i)};
            for (int j = 0; j < 7; ++j) r[static_cast<size_t>(j) * adj->n_stride] = v[j];
        }
        // leaf box from the integrated pose, kept as the exact floats of its fp16 bounds
        const BoxF bx = unpack_box(leaf_box(SS.type(i), SB.px(i), SB.py(i), SB.pz(i), SB.qw(i), SB.qx(i),
                                            SB.qy(i), SB.qz(i), SS.hx(i), SS.hy(i), SS.hz(i)));
        box[i] = bx.mnx; box[ldb + i] = bx.mny; box[2 * ldb + i] = bx.mnz;
        box[3 * ldb + i] = bx.mxx; box[4 * ldb + i] = bx.mxy; box[5 * ldb + i] = bx.mxz;
    }
    T.sync();
    phase_mark(T, P_, 0, t0);
    // ── candidate pairs: per body a, the partners b > a in ascending order ──
    // The count pass keeps each 32-partner chunk's overlap bits at the end of
    // the team's shared memory when they fit there, so the write pass reads
    // them instead of testing the boxes again.
    const uint32_t mask_words = overlap_mask_words(nb);
    const uint32_t mask_off = (smem_bytes - 4u * mask_words) & ~15u;
    const bool keep_masks = 4u * mask_words <= smem_bytes && frame_body_bytes(nb) <= mask_off;
    uint32_t* masks = reinterpret_cast<uint32_t*>(smem + mask_off);
    for (uint32_t a = T.warp(); a < nb; a += T.warps()) {
        const BoxF q{box[a], box[ldb + a], box[2 * ldb + a], box[3 * ldb + a], box[4 * ldb + a], box[5 * ldb + a]};
        uint32_t c = 0, w = overlap_mask_base(nb, a);
        for (uint32_t j0 = a + 1; j0 < nb; j0 += 32u, ++w) {
            const uint32_t j = j0 + lane;
            bool ov = false;
            if (j < nb) {
                const BoxF n{box[j], box[ldb + j], box[2 * ldb + j], box[3 * ldb + j], box[4 * ldb + j],
                             box[5 * ldb + j]};
                ov = box_overlap(n, q);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, ov);
            if (keep_masks && lane == 0) masks[w] = bal;
            c += __popc(bal);
        }
        if (lane == 0) R.cnt[a] = c;
    }
    if (T.leader()) sh.carry = 0u;
    T.sync();
    for (uint32_t base = 0; base < nb; base += T.size()) {
        const uint32_t i = base + T.rank();
        const uint32_t v = i < nb ? R.cnt[i] : 0u;
        uint32_t tot;
        const uint32_t ex = T.exclusive_scan(v, sh.scan, tot);
        if (i < nb) R.off[i] = sh.carry + ex;
        T.sync();
        if (T.leader()) sh.carry += tot;
        T.sync();
    }
    const uint32_t p_true = sh.carry;
    const uint32_t P = min(p_true, pcap);
    // ── layout of the pairs and the contact words: shared memory if they fit ──
    const uint32_t cc = min(P, ccap);
    const uint32_t ldc = (cc + 4u) & ~3u;  // >= cc + 1: group offsets take m + 1 words
    const uint32_t pwords = (P + 3u) & ~3u;
    const uint32_t body_bytes = frame_body_bytes(nb);
    const bool in_smem = body_bytes + 4u * pwords + kSceneWords * 4u * ldc <= smem_bytes;
    uint32_t* pairs = in_smem ? reinterpret_cast<uint32_t*>(smem + body_bytes) : F.pair_raw + F.pair_base[s];
    const SceneContacts SC{in_smem ? reinterpret_cast<uint32_t*>(smem + body_bytes) + pwords
                                   : F.words + F.contact_base[s] + s,
                           in_smem ? ldc : F.words_stride};
    // the masks survive the write pass unless the pairs themselves reach them
    const bool use_masks = keep_masks && (!in_smem || body_bytes + 4u * pwords <= mask_off);
    for (uint32_t a = T.warp(); a < nb; a += T.warps()) {
        const BoxF q{box[a], box[ldb + a], box[2 * ldb + a], box[3 * ldb + a], box[4 * ldb + a], box[5 * ldb + a]};
        uint32_t pos = R.off[a], w = overlap_mask_base(nb, a);
        for (uint32_t j0 = a + 1; j0 < nb && pos < P; j0 += 32u, ++w) {
            const uint32_t j = j0 + lane;
            unsigned bal;
            if (use_masks) {
                bal = masks[w];
            } else {
                bool ov = false;
                if (j < nb) {
                    const BoxF n{box[j], box[ldb + j], box[2 * ldb + j], box[3 * ldb + j], box[4 * ldb + j],
                                 box[5 * ldb + j]};
                    ov = box_overlap(n, q);
                }
                bal = __ballot_sync(0xffffffffu, ov);
            }
            const bool ov = (bal >> lane) & 1u;
            const uint32_t at = pos + __popc(bal & ((1u << lane) - 1u));
            if (ov && at < P) pairs[at] = a | (j << 16);
            pos += __popc(bal);
        }
    }
    T.sync();
    if (in_smem && !adj)
        for (uint32_t p = T.rank(); p < P; p += T.size()) F.pair_raw[F.pair_base[s] + p] = pairs[p];
    phase_mark(T, P_, 1, t0);
    // ── narrowphase: contacts in pair order ──
    for (uint32_t i = T.rank(); i < nb; i += T.size()) R.cnt[i] = 0u;
    if (T.leader()) sh.carry = 0u;
    T.sync();
    const uint32_t cbase = F.contact_base[s];
    for (uint32_t base = 0; base < P; base += T.size()) {
        const uint32_t p = base + T.rank();
        Contact c{};
        bool hit = false;
        uint32_t br = 0u;
        if (p < P) {
            const uint32_t ab = pairs[p];
            hit = process_pair(SB, SS, ab & 0xFFFFu, ab >> 16, c, adj ? &br : nullptr);
        }
        uint32_t tot;
        const uint32_t ex = T.exclusive_scan(hit ? 1u : 0u, sh.scan, tot);
        const uint32_t k = sh.carry + ex;
        if (hit && k < cc) {
            SC.ab(k) = c.a | (c.b << 16);
            SC.lam(k) = 0.f;
            SC.pb(k) = kSceneNone;
            SC.g(0, k) = c.px; SC.g(1, k) = c.py; SC.g(2, k) = c.pz;
            SC.g(3, k) = c.nx; SC.g(4, k) = c.ny; SC.g(5, k) = c.nz;
            SC.g(6, k) = c.depth;
            if (SB.im(c.b) != 0.f) atomicAdd(&R.cnt[c.b], 1u);
            const uint32_t slot = cbase + k, st = F.contact_slots;
            if (adj) {
                adj->rec[27ull * adj->rec_stride + slot] = __uint_as_float(br);
            } else {
                F.contact_raw[slot] = b0 + c.a;
                F.contact_raw[st + slot] = b0 + c.b;
                F.contact_raw[2 * st + slot] = __float_as_uint(c.px);
                F.contact_raw[3 * st + slot] = __float_as_uint(c.py);
                F.contact_raw[4 * st + slot] = __float_as_uint(c.pz);
                F.contact_raw[5 * st + slot] = __float_as_uint(c.nx);
                F.contact_raw[6 * st + slot] = __float_as_uint(c.ny);
                F.contact_raw[7 * st + slot] = __float_as_uint(c.nz);
                F.contact_raw[8 * st + slot] = __float_as_uint(c.depth);
            }
        }
        T.sync();
        if (T.leader()) sh.carry += tot;
        T.sync();
    }
    const uint32_t m_true = sh.carry, m = min(m_true, cc);
    T.sync();  // every thread has read the count before scene_solve reuses sh.carry
    if (T.leader() && !adj) {
        F.counts[4 * s + 0] = P;
        F.counts[4 * s + 1] = p_true;
        F.counts[4 * s + 2] = m;
        F.counts[4 * s + 3] = m_true;
        atomicAdd(&P_.bp_counts[0], P);
        atomicAdd(&P_.bp_counts[1], p_true);
        atomicAdd(&P_.np_counts[0], m);
        atomicAdd(&P_.np_counts[1], m_true);
        // a scene past its own capacity keeps its ordered prefix, as it does alone
        if (p_true > pcap) atomicCAS(P_.status, 0u, static_cast<uint32_t>(DYPH_ERR_PAIR_OVERFLOW));
        if (m_true > ccap) atomicCAS(P_.status, 0u, static_cast<uint32_t>(DYPH_ERR_CONTACT_OVERFLOW));
    }
    phase_mark(T, P_, 2, t0);
    // ── contact solve (none without contacts, as the reference's solve returns) ──
    bool colored = false;
    uint32_t n_colors = 0, rounds = 0, groups = 0;
    if (m > 0) {
        SolveRecord rec{};
        if (adj) rec = SolveRecord{adj->rec, adj->rec_stride, cbase, adj->qs, adj->n_stride, b0, adj->flag};
        uint64_t t_sweep = 0;
        if (!scene_solve<kRecord>(T, nb, m, SB, R, SC, P_.mode, P_.n_iters, P_.mu, P_.dt, sh, colored, n_colors, rounds,
                         adj ? &rec : nullptr, &groups, P_.phase_ns ? &t_sweep : nullptr))
            return false;
        if (P_.phase_ns && T.leader()) {
            atomicAdd(&P_.phase_ns[3], static_cast<unsigned long long>(t_sweep - t0));
            t0 = t_sweep;
        }
        if (!adj) {
            for (uint32_t k = T.rank(); k < m; k += T.size())
                F.color_raw[cbase + k] = colored ? SC.done(k) : kUncolored;
            scene_stats(T, P_.meta, colored, n_colors, rounds);
        }
    }
    if (out) *out = FrameOut{SC, m, groups};
    phase_mark(T, P_, 4, t0);
    if (!adj) {
        scene_store_bodies(T, B, b0, nb, SB);
    } else if (adj->store) {
        for (uint32_t i = T.rank(); i < nb; i += T.size()) {
            const float v[13] = {SB.px(i), SB.py(i), SB.pz(i), SB.qw(i), SB.qx(i), SB.qy(i), SB.qz(i),
                                 SB.vx(i), SB.vy(i), SB.vz(i), SB.wx(i), SB.wy(i), SB.wz(i)};
#pragma unroll
            for (int r = 0; r < 13; ++r) adj->store[static_cast<size_t>(r) * adj->n_stride + b0 + i] = v[r];
        }
    }
    T.sync();
    phase_mark(T, P_, 5, t0);
    return true;
}

// Work item i: items[4 i] a large scene solved by the whole block when
// items[4 i + 1] == kItemBlock; two mid-size scenes items[4 i] and
// items[4 i + 2], two warps and half the block's shared memory each, when
// items[4 i + 1] == kItemHalf; otherwise up to four small scenes, one per
// warp, each with a quarter of the shared memory. kItemEmpty marks an unused
// team.
constexpr uint32_t kItemEmpty = 0xFFFFFFFFu;
constexpr uint32_t kItemBlock = 0xFFFFFFFEu;
constexpr uint32_t kItemHalf = 0xFFFFFFFDu;

// kMinBlocks is the register budget: 4 resident blocks per SM (128
// registers a thread), 5 (96) or 6 (80, a few bytes spilled). Which one runs
// best depends on the batch (dyph_world_autotune picks it with the shared
// memory cap); all three compute the same frames.
template <int kMinBlocks>
__global__ void __launch_bounds__(kSceneThreads, kMinBlocks) scene_frame_kernel(SceneBufs S, FrameBufs F,
                                                                                FrameParams P_,
                                                                                const uint32_t* __restrict__ items,
                                                                                uint32_t n_items) {
    extern __shared__ __align__(16) unsigned char scene_smem[];
    __shared__ SceneShared sh[kSceneThreads / 32];
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t share = (S.smem_bytes / 4u) & ~15u;
    for (uint32_t it = blockIdx.x; it < n_items; it += gridDim.x) {
        const uint32_t kind = items[4 * it + 1];
        if (kind == kItemBlock) {
            frame_scene(BlockTeam{}, items[4 * it], scene_smem, S.smem_bytes, sh[0], S, F, P_);
        } else if (kind == kItemHalf) {
            const uint32_t half = warp >> 1, s = items[4 * it + 2 * half];
            if (s != kItemEmpty)
                frame_scene(HalfTeam{half}, s, scene_smem + half * 2u * share, 2u * share, sh[2 * half], S, F, P_);
        } else {
            const uint32_t s = items[4 * it + warp];
            if (s != kItemEmpty) frame_scene(WarpTeam{}, s, scene_smem + warp * share, share, sh[warp], S, F, P_);
        }
        __syncthreads();
    }
}

// Exclusive scans of the scenes' stored pair / contact counts (one block):
// pos[2 s] / pos[2 s + 1] = first compacted pair / contact of scene s, and the
// totals into the broadphase / narrowphase stored-count words.
__global__ void __launch_bounds__(1024) scene_gather_scan_kernel(const uint32_t* __restrict__ counts,
                                                                 uint32_t n_scenes, uint32_t* __restrict__ pos,
                                                                 uint32_t* __restrict__ bp_counts,
                                                                 uint32_t* __restrict__ np_counts) {
    __shared__ uint32_t s_scan[32];
    __shared__ uint32_t carry[2];
    if (threadIdx.x < 2) carry[threadIdx.x] = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < n_scenes; base += blockDim.x) {
        const uint32_t s = base + threadIdx.x;
        for (int w = 0; w < 2; ++w) {
            const uint32_t v = s < n_scenes ? counts[4 * s + 2 * w] : 0u;
            uint32_t tot;
            const uint32_t ex = block_exclusive_scan<1024>(v, s_scan, tot);
            if (s < n_scenes) pos[2 * s + w] = carry[w] + ex;
            __syncthreads();
            if (threadIdx.x == 0) carry[w] += tot;
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        bp_counts[0] = carry[0];
        np_counts[0] = carry[1];
    }
}

// Copy every scene's pairs (as global body indices), contacts and colours to
// their compacted positions (one block per scene).
__global__ void scene_gather_copy_kernel(SceneBufs S, FrameBufs F, const uint32_t* __restrict__ pos,
                                         dyph_pair* __restrict__ pairs, dyph_contacts cv,
                                         uint32_t* __restrict__ color) {
    const uint32_t s = blockIdx.x;
    if (s >= S.n_scenes) return;
    const uint32_t b0 = S.body_offset[s];
    const uint32_t np_ = F.counts[4 * s + 0], nc = F.counts[4 * s + 2];
    const uint32_t p0 = pos[2 * s], c0 = pos[2 * s + 1];
    for (uint32_t p = threadIdx.x; p < np_; p += blockDim.x) {
        const uint32_t ab = F.pair_raw[F.pair_base[s] + p];
        pairs[p0 + p] = dyph_pair{b0 + (ab & 0xFFFFu), b0 + (ab >> 16)};
    }
    const uint32_t st = F.contact_slots, cb = F.contact_base[s];
    float* rows[7] = {cv.pos_x, cv.pos_y, cv.pos_z, cv.norm_x, cv.norm_y, cv.norm_z, cv.depth};
    for (uint32_t k = threadIdx.x; k < nc; k += blockDim.x) {
        cv.body_a[c0 + k] = F.contact_raw[cb + k];
        cv.body_b[c0 + k] = F.contact_raw[st + cb + k];
#pragma unroll
        for (int r = 0; r < 7; ++r) rows[r][c0 + k] = __uint_as_float(F.contact_raw[(2 + r) * st + cb + k]);
        color[c0 + k] = F.color_raw[cb + k];
    }
}

}  // namespace
}  // namespace dyph
