// Batched scenes (included by solver.cu): one thread block solves one scene,
// the scene's bodies staged in shared memory.
//
// The reference solves one scene per XpbdSolver::solve (xpbd_solver.cpp:
// 603-733). A batch is many independent scenes, so each block takes one scene
// and runs exactly that solve on it:
//   * the scene's contacts are a contiguous run of the contact list (pairs are
//     sorted by body a and a scene's bodies are contiguous), local contact
//     index k = global index - first index;
//   * a scene without contacts is left alone (the reference returns before
//     any renormalisation when n_con == 0);
//   * sequential order (set_force_serial, or n_con <= 256 in the reference
//     mode, or a colouring that needs more than 64 colours or 256 rounds):
//     contacts are solved in waves, contact k as soon as the previous contact
//     of each of its dynamic bodies (in contact order) is solved — the serial
//     loop's per-body order, so the result is bit-identical to it;
//   * coloured order: Jones–Plassmann rounds with the priorities
//     hash(k) << 32 | k of the local index (:645-688), then colour by colour;
//   * every iteration renormalises every body of the scene (:579-584,
//     :726-731); a contact deferred at w_total < 1e-10 is retried by the next
//     iteration's sweep, as in the reference.
// Each scene therefore evolves bit for bit as it does stepped alone in the
// same mode. Waves and rounds are separated by block barriers; a scene whose
// chain of dependent contacts is d long takes d waves.
#pragma once

#include "solver_common.cuh"

namespace dyph {
namespace {

constexpr int kSceneThreads = 128;
constexpr uint32_t kSceneNone = 0xFFFFFFFFu;
constexpr uint32_t kSceneWords = 13;         // per-contact words (see SceneContacts)
constexpr uint32_t kSceneMaxBodies = 65535;  // local body indices are 16 bits

// Shared-memory bytes of a scene's body part (see the layout in scene_solve_kernel).
__host__ __device__ __forceinline__ uint32_t scene_body_bytes(uint32_t nb) {
    const uint32_t ldb = (nb + 3u) & ~3u;
    return 20u * 4u * ldb + 2u * 8u * ldb + 4u * (ldb + 4u) + 4u * ldb;
}

struct SceneBufs {
    const uint32_t* body_offset;  // [n_scenes + 1] first body of each scene
    const uint32_t* scene_of;     // [n] scene of each body
    const uint32_t* order;        // [n_scenes] scenes by descending body count (largest first)
    uint32_t* range;              // [2 n_scenes] first / one-past-last contact of each scene
    uint32_t* scratch;            // [kSceneWords][scratch_stride] per-contact words of scenes too big for shared memory
    uint32_t scratch_stride;      // max contacts + n_scenes (one extra word per scene)
    uint32_t n_scenes;
    uint32_t smem_bytes;          // dynamic shared memory of one block
};

// First and one-past-last contact of every scene (range cleared to 0 first).
__global__ void scene_range_kernel(dyph_contacts cv, SceneBufs S) {
    const uint32_t nc = contact_count(cv);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += gridDim.x * blockDim.x) {
        const uint32_t s = S.scene_of[cv.body_a[c]];
        if (c == 0 || S.scene_of[cv.body_a[c - 1]] != s) S.range[2 * s] = c;
        if (c + 1 == nc || S.scene_of[cv.body_a[c + 1]] != s) S.range[2 * s + 1] = c + 1;
    }
}

// Body rows of one scene in shared memory: row r of local body i at f[r * ld + i].
// Rows 0-12 state, 13 inverse mass, 14-19 inverse inertia.
struct SceneBodies {
    float* f;
    uint32_t ld;
    __device__ __forceinline__ float& px(uint32_t i) const { return f[0 * ld + i]; }
    __device__ __forceinline__ float& py(uint32_t i) const { return f[1 * ld + i]; }
    __device__ __forceinline__ float& pz(uint32_t i) const { return f[2 * ld + i]; }
    __device__ __forceinline__ float& qw(uint32_t i) const { return f[3 * ld + i]; }
    __device__ __forceinline__ float& qx(uint32_t i) const { return f[4 * ld + i]; }
    __device__ __forceinline__ float& qy(uint32_t i) const { return f[5 * ld + i]; }
    __device__ __forceinline__ float& qz(uint32_t i) const { return f[6 * ld + i]; }
    __device__ __forceinline__ float& vx(uint32_t i) const { return f[7 * ld + i]; }
    __device__ __forceinline__ float& vy(uint32_t i) const { return f[8 * ld + i]; }
    __device__ __forceinline__ float& vz(uint32_t i) const { return f[9 * ld + i]; }
    __device__ __forceinline__ float& wx(uint32_t i) const { return f[10 * ld + i]; }
    __device__ __forceinline__ float& wy(uint32_t i) const { return f[11 * ld + i]; }
    __device__ __forceinline__ float& wz(uint32_t i) const { return f[12 * ld + i]; }
    __device__ __forceinline__ float im(uint32_t i) const { return f[13 * ld + i]; }
    __device__ __forceinline__ float ixx(uint32_t i) const { return f[14 * ld + i]; }
    __device__ __forceinline__ float iyy(uint32_t i) const { return f[15 * ld + i]; }
    __device__ __forceinline__ float izz(uint32_t i) const { return f[16 * ld + i]; }
    __device__ __forceinline__ float ixy(uint32_t i) const { return f[17 * ld + i]; }
    __device__ __forceinline__ float ixz(uint32_t i) const { return f[18 * ld + i]; }
    __device__ __forceinline__ float iyz(uint32_t i) const { return f[19 * ld + i]; }
};

// Per-contact words of one scene (shared memory, or the global scratch for
// a scene with too many contacts): row r of local contact k at w[r * ld + k].
//   0 a | b << 16 (local body indices)   1 predecessor on a   2 predecessor on b
//   3 wave solved in / colour            4 b-side list entry   5 lambda
//   6-12 position xyz, normal xyz, depth (copied from the contact list)
struct SceneContacts {
    uint32_t* w;
    uint32_t ld;
    __device__ __forceinline__ uint32_t& ab(uint32_t k) const { return w[k]; }
    __device__ __forceinline__ uint32_t& pa(uint32_t k) const { return w[1 * ld + k]; }
    __device__ __forceinline__ uint32_t& pb(uint32_t k) const { return w[2 * ld + k]; }
    __device__ __forceinline__ uint32_t& done(uint32_t k) const { return w[3 * ld + k]; }
    __device__ __forceinline__ uint32_t& ent(uint32_t k) const { return w[4 * ld + k]; }
    __device__ __forceinline__ float& lam(uint32_t k) const { return reinterpret_cast<float*>(w)[5 * ld + k]; }
    __device__ __forceinline__ float& g(int r, uint32_t k) const { return reinterpret_cast<float*>(w)[(6 + r) * ld + k]; }
    __device__ __forceinline__ Contact contact(uint32_t k) const {
        Contact ct;
        const uint32_t ab_k = ab(k);
        ct.a = ab_k & 0xFFFFu;
        ct.b = ab_k >> 16;
        ct.px = g(0, k); ct.py = g(1, k); ct.pz = g(2, k);
        ct.nx = g(3, k); ct.ny = g(4, k); ct.nz = g(5, k);
        ct.depth = g(6, k);
        return ct;
    }
};

// A team of threads that runs one scene: the whole block (big scenes) or one
// warp (small scenes, several to a block).
struct BlockTeam {
    __device__ __forceinline__ uint32_t rank() const { return threadIdx.x; }
    __device__ __forceinline__ uint32_t size() const { return kSceneThreads; }
    __device__ __forceinline__ uint32_t warp() const { return threadIdx.x >> 5; }
    __device__ __forceinline__ uint32_t warps() const { return kSceneThreads / 32; }
    __device__ __forceinline__ bool leader() const { return threadIdx.x == 0; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    __device__ __forceinline__ bool any(bool p) const { return __syncthreads_or(p) != 0; }
    __device__ __forceinline__ uint32_t exclusive_scan(uint32_t v, uint32_t* scratch, uint32_t& total) const {
        return block_exclusive_scan<kSceneThreads>(v, scratch, total);
    }
};

struct WarpTeam {
    __device__ __forceinline__ uint32_t rank() const { return threadIdx.x & 31u; }
    __device__ __forceinline__ uint32_t size() const { return 32u; }
    __device__ __forceinline__ uint32_t warp() const { return 0u; }
    __device__ __forceinline__ uint32_t warps() const { return 1u; }
    __device__ __forceinline__ bool leader() const { return (threadIdx.x & 31u) == 0u; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    __device__ __forceinline__ bool any(bool p) const { return __any_sync(0xffffffffu, p) != 0; }
    __device__ __forceinline__ uint32_t exclusive_scan(uint32_t v, uint32_t*, uint32_t& total) const {
        const uint32_t lane = threadIdx.x & 31u;
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= static_cast<uint32_t>(d)) x += y;
        }
        total = __shfl_sync(0xffffffffu, x, 31);
        return x - v;
    }
};

// Two warps of a block (half 0: warps 0-1, half 1: warps 2-3), synchronised
// on named barrier 1 + half; the block's own __syncthreads uses barrier 0.
struct HalfTeam {
    uint32_t half;
    __device__ __forceinline__ uint32_t rank() const { return threadIdx.x & 63u; }
    __device__ __forceinline__ uint32_t size() const { return 64u; }
    __device__ __forceinline__ uint32_t warp() const { return (threadIdx.x >> 5) & 1u; }
    __device__ __forceinline__ uint32_t warps() const { return 2u; }
    __device__ __forceinline__ bool leader() const { return (threadIdx.x & 63u) == 0u; }
    // Immediate barrier ids (the branch is uniform over the team), so the
    // kernel reserves barriers 0-2 only.
    __device__ __forceinline__ void sync() const {
        if (half)
            asm volatile("bar.sync 2, 64;" ::: "memory");
        else
            asm volatile("bar.sync 1, 64;" ::: "memory");
    }
    __device__ __forceinline__ bool any(bool p) const {
        uint32_t r;
        if (half)
            asm volatile(
                "{\n\t.reg .pred pin, pout;\n\t"
                "setp.ne.u32 pin, %1, 0;\n\t"
                "bar.red.or.pred pout, 2, 64, pin;\n\t"
                "selp.u32 %0, 1, 0, pout;\n\t}"
                : "=r"(r)
                : "r"(static_cast<uint32_t>(p))
                : "memory");
        else
            asm volatile(
                "{\n\t.reg .pred pin, pout;\n\t"
                "setp.ne.u32 pin, %1, 0;\n\t"
                "bar.red.or.pred pout, 1, 64, pin;\n\t"
                "selp.u32 %0, 1, 0, pout;\n\t}"
                : "=r"(r)
                : "r"(static_cast<uint32_t>(p))
                : "memory");
        return r != 0u;
    }
    __device__ __forceinline__ uint32_t exclusive_scan(uint32_t v, uint32_t* scratch, uint32_t& total) const {
        const uint32_t lane = threadIdx.x & 31u, w = warp();
        uint32_t x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= static_cast<uint32_t>(d)) x += y;
        }
        if (lane == 31u) scratch[w] = x;
        sync();
        const uint32_t t0 = scratch[0], t1 = scratch[1];
        total = t0 + t1;
        sync();  // the scratch words are free again for the next scan
        return (w ? t0 : 0u) + x - v;
    }
};

// Levels of the sequential order on one scene: level(k) = 1 + the larger
// level of k's predecessors on its two dynamic bodies. Contacts of one level
// share no dynamic body, and solving the levels in ascending order gives
// every body its contacts in contact order: the serial loop's result, bit for
// bit. Levels go to SC.done (1-based); returns the level count, or 0 if the
// predecessor links were inconsistent (they cannot be: every predecessor has a
// lower index).
template <class Team>
__device__ uint32_t scene_levels(const Team& T, uint32_t m, const SceneContacts& SC, uint32_t* s_max) {
    for (uint32_t k = T.rank(); k < m; k += T.size()) SC.done(k) = 0u;
    if (T.leader()) *s_max = 0u;
    T.sync();
    uint32_t my_max = 0;
    for (uint32_t pass = 0;; ++pass) {
        int pending = 0;
        // A level, once written, is final, so a pass may use levels written
        // by other threads during the same pass.
        for (uint32_t k = T.rank(); k < m; k += T.size()) {
            if (SC.done(k) != 0u) continue;
            const uint32_t pa = SC.pa(k), pb = SC.pb(k);
            const uint32_t la = pa == kSceneNone ? 0u : SC.done(pa);
            const uint32_t lb = pb == kSceneNone ? 0u : SC.done(pb);
            if ((pa != kSceneNone && la == 0u) || (pb != kSceneNone && lb == 0u)) {
                pending = 1;
                continue;
            }
            const uint32_t l = max(la, lb) + 1u;
            SC.done(k) = l;
            my_max = max(my_max, l);
        }
        if (!T.any(pending)) break;
        if (pass > m) return 0u;
    }
    atomicMax(s_max, my_max);
    T.sync();
    const uint32_t levels = *s_max;
    T.sync();
    return levels;
}

// Counting sort of the scene's contacts by group done(k) - base (a level or a
// colour) into SC.ent; group g is SC.ent[SC.pa(g), SC.pa(g + 1)). The
// predecessor rows are free once the groups are known.
template <class Team>
__device__ void scene_group(const Team& T, uint32_t m, uint32_t groups, uint32_t base, const SceneContacts& SC,
                            uint32_t* s_scan, uint32_t* s_carry) {
    for (uint32_t g = T.rank(); g <= groups; g += T.size()) SC.pa(g) = 0u;
    if (T.leader()) *s_carry = 0u;
    T.sync();
    for (uint32_t k = T.rank(); k < m; k += T.size()) atomicAdd(&SC.pa(SC.done(k) - base), 1u);
    T.sync();
    for (uint32_t g0 = 0; g0 <= groups; g0 += T.size()) {
        const uint32_t g = g0 + T.rank();
        const uint32_t v = g <= groups ? SC.pa(g) : 0u;
        uint32_t tot;
        const uint32_t ex = T.exclusive_scan(v, s_scan, tot);
        if (g <= groups) {
            SC.pa(g) = *s_carry + ex;
            SC.pb(g) = *s_carry + ex;  // fill cursor
        }
        T.sync();
        if (T.leader()) *s_carry += tot;
        T.sync();
    }
    for (uint32_t k = T.rank(); k < m; k += T.size()) SC.ent(atomicAdd(&SC.pb(SC.done(k) - base), 1u)) = k;
    T.sync();
}

// What the adjoint pass records of a scene's solve (solve_record): for every
// contact that acts, both bodies' state before its solve and lambda; the
// quaternions before the renormalisations.
constexpr int kRecWords = 36;  // per-contact record rows (see SolveRecord)
struct SolveRecord {
    // rows r of contact k at rec[r * stride + base + k]: 0-12 body a state,
    // 13-25 body b state, 26 lambda before, 27 narrowphase branch word,
    // 28-34 contact geometry adjoint (point, normal, depth), 35 the solve's
    // branch flags (bits of a float; 0 when the contact did not act)
    float* rec;
    uint32_t stride, base;
    float* qs;           // [4][qs_stride] quaternions after the sweeps, at body b0 + i
    uint32_t qs_stride, b0;
    uint32_t* flag;      // set when the solve took a path the adjoint does not cover
};

__device__ __forceinline__ void record_state(float* r, uint32_t stride, const SceneBodies& SB, uint32_t i,
                                             int row0) {
    const float v[13] = {SB.px(i), SB.py(i), SB.pz(i), SB.qw(i), SB.qx(i), SB.qy(i), SB.qz(i),
                         SB.vx(i), SB.vy(i), SB.vz(i), SB.wx(i), SB.wy(i), SB.wz(i)};
#pragma unroll
    for (int j = 0; j < 13; ++j) r[static_cast<size_t>(row0 + j) * stride] = v[j];
}

// One sweep over the groups in ascending order, one contact per thread at a
// time inside a group (no two of a group share a dynamic body). kRecord
// compiles the recording in; without it `rec` is ignored.
template <bool kRecord, class Team>
__device__ void scene_sweep(const Team& T, uint32_t groups, const SceneBodies& SB, const SceneContacts& SC, float mu,
                            float dt, int* s_flag, const SolveRecord* rec_in = nullptr, int iter = 0) {
    const SolveRecord* const rec = kRecord ? rec_in : nullptr;
    for (uint32_t g = 0; g < groups; ++g) {
        const uint32_t end = SC.pa(g + 1);
        for (uint32_t i = SC.pa(g) + T.rank(); i < end; i += T.size()) {
            const uint32_t k = SC.ent(i);
            const Contact ct = SC.contact(k);
            float lc = SC.lam(k);
            if (rec) {
                // The pre-solve state of the first sweep, the one the adjoint
                // differentiates, marked as acted only if it did. A later sweep
                // (after a deferral) must not overwrite it: it re-solves only the
                // deferred contacts, and one of those that acts there is
                // reported as a path the adjoint does not cover.
                float* r = rec->rec + rec->base + k;
                const float lc0 = lc;
                if (iter == 0) {
                    record_state(r, rec->stride, SB, ct.a, 0);
                    record_state(r, rec->stride, SB, ct.b, 13);
                }
                uint32_t fl = 0u;
                if (solve_contact(SB, ct, mu, lc, dt, &fl) == kSolveDeferred) *s_flag = 1;
                if (fl & kSfActive) {
                    r[26ull * rec->stride] = lc0;
                    r[35ull * rec->stride] = __uint_as_float(fl);
                    if (iter > 0) atomicOr(rec->flag, 1u);  // acted after a renormalisation
                } else if (iter == 0) {
                    r[35ull * rec->stride] = 0.f;
                }
            } else if (solve_contact(SB, ct, mu, lc, dt) == kSolveDeferred) {
                *s_flag = 1;
            }
            SC.lam(k) = lc;
        }
        T.sync();
    }
}

// Block-shared scalars of one scene's solve.
struct SceneShared {
    uint32_t scan[kSceneThreads / 32];
    uint32_t carry, rem, over, maxcol;
    int flag;
};

// The solver's per-body rows after the 20 body rows (see scene_body_bytes).
struct SceneSolverRows {
    uint64_t* pri;   // [ldb] JP priorities
    uint64_t* mask;  // [ldb] JP colour masks
    uint32_t* off;   // [ldb + 4] b-side list offsets
    uint32_t* cnt;   // [ldb] counts / fill cursors / last b-side contact
};

__device__ __forceinline__ SceneSolverRows scene_solver_rows(float* fb, uint32_t ldb) {
    SceneSolverRows R;
    R.pri = reinterpret_cast<uint64_t*>(fb + 20 * ldb);
    R.mask = R.pri + ldb;
    R.off = reinterpret_cast<uint32_t*>(R.mask + ldb);
    R.cnt = R.off + ldb + 4;
    return R;
}

template <class Team>
__device__ __forceinline__ void scene_load_bodies(const Team& T, const GlobalBodies& B, uint32_t b0, uint32_t nb,
                                                  float* fb, uint32_t ldb) {
    const SceneBodies SB{fb, ldb};
    for (uint32_t i = T.rank(); i < nb; i += T.size()) {
        const uint32_t g = b0 + i;
        SB.px(i) = B.px(g); SB.py(i) = B.py(g); SB.pz(i) = B.pz(g);
        SB.qw(i) = B.qw(g); SB.qx(i) = B.qx(g); SB.qy(i) = B.qy(g); SB.qz(i) = B.qz(g);
        SB.vx(i) = B.vx(g); SB.vy(i) = B.vy(g); SB.vz(i) = B.vz(g);
        SB.wx(i) = B.wx(g); SB.wy(i) = B.wy(g); SB.wz(i) = B.wz(g);
        fb[13 * ldb + i] = B.im(g);
        fb[14 * ldb + i] = B.ixx(g); fb[15 * ldb + i] = B.iyy(g); fb[16 * ldb + i] = B.izz(g);
        fb[17 * ldb + i] = B.ixy(g); fb[18 * ldb + i] = B.ixz(g); fb[19 * ldb + i] = B.iyz(g);
    }
}

template <class Team>
__device__ __forceinline__ void scene_store_bodies(const Team& T, const GlobalBodies& B, uint32_t b0, uint32_t nb,
                                                   const SceneBodies& SB) {
    for (uint32_t i = T.rank(); i < nb; i += T.size()) {
        const uint32_t g = b0 + i;
        B.px(g) = SB.px(i); B.py(g) = SB.py(i); B.pz(g) = SB.pz(i);
        B.qw(g) = SB.qw(i); B.qx(g) = SB.qx(i); B.qy(g) = SB.qy(i); B.qz(g) = SB.qz(i);
        B.vx(g) = SB.vx(i); B.vy(g) = SB.vy(i); B.vz(g) = SB.vz(i);
        B.wx(g) = SB.wx(i); B.wy(g) = SB.wy(i); B.wz(g) = SB.wz(i);
    }
}

// XpbdSolver::solve on one scene whose m >= 1 contacts sit in SC (rows ab,
// lambda = 0, geometry; pb = none) with R.cnt[b] = the b-side contact count of
// every dynamic body b. Leaves the bodies solved and renormalised in SB and
// the colours (or UINT32_MAX) in SC.done. Returns false after raising an error.
template <bool kRecord = false, class Team>
__device__ bool scene_solve(const Team& T, uint32_t nb, uint32_t m, const SceneBodies& SB, const SceneSolverRows& R,
                            const SceneContacts& SC, int mode, int n_iters, float mu, float dt, SceneShared& sh,
                            bool& colored_out, uint32_t& n_colors_out, uint32_t& rounds_out,
                            const SolveRecord* rec_in = nullptr, uint32_t* groups_out = nullptr,
                            uint64_t* sweep_start = nullptr) {
    const SolveRecord* const rec = kRecord ? rec_in : nullptr;
    // ── predecessors in contact order: b-side lists (scan, fill, sort) ──
    if (T.leader()) {
        sh.carry = 0u;
        sh.flag = 0;
    }
    T.sync();
    for (uint32_t base = 0; base < nb; base += T.size()) {
        const uint32_t i = base + T.rank();
        const uint32_t v = i < nb ? R.cnt[i] : 0u;
        uint32_t tot;
        const uint32_t ex = T.exclusive_scan(v, sh.scan, tot);
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
        const uint32_t b = SC.ab(k) >> 16;
        if (SB.im(b) != 0.f) SC.ent(R.off[b] + atomicAdd(&R.cnt[b], 1u)) = k;
    }
    T.sync();
    for (uint32_t x = T.rank(); x < nb; x += T.size()) {
        const uint32_t lo = R.off[x], hi = R.off[x + 1];
        for (uint32_t i = lo + 1; i < hi; ++i) {
            const uint32_t v = SC.ent(i);
            uint32_t j = i;
            while (j > lo && SC.ent(j - 1) > v) {
                SC.ent(j) = SC.ent(j - 1);
                --j;
            }
            SC.ent(j) = v;
        }
        for (uint32_t i = lo + 1; i < hi; ++i) SC.pb(SC.ent(i)) = SC.ent(i - 1);
        R.cnt[x] = hi > lo ? SC.ent(hi - 1) : kSceneNone;  // last b-side contact of x
    }
    T.sync();
    for (uint32_t k = T.rank(); k < m; k += T.size()) {
        const uint32_t a = SC.ab(k) & 0xFFFFu;
        uint32_t p = kSceneNone;
        if (SB.im(a) != 0.f) p = (k > 0 && (SC.ab(k - 1) & 0xFFFFu) == a) ? k - 1 : R.cnt[a];
        SC.pa(k) = p;
    }
    // ── colouring (reference mode above 256 contacts, coloured mode always) ──
    bool colored = mode == DYPH_SOLVER_COLORED ||
                   ((mode == DYPH_SOLVER_REFERENCE || mode == DYPH_SOLVER_REFERENCE_ROUNDS) && m > kSerialThreshold);
    uint32_t n_colors = 0, rounds = 0;
    if (colored) {
        for (uint32_t k = T.rank(); k < m; k += T.size()) SC.done(k) = kUncolored;
        for (uint32_t i = T.rank(); i < nb; i += T.size()) R.mask[i] = 0ull;
        if (T.leader()) {
            sh.rem = m;
            sh.over = 0u;
            sh.maxcol = 0u;
        }
        T.sync();
        while (sh.rem > 0u && rounds < kMaxRounds) {
            for (uint32_t i = T.rank(); i < nb; i += T.size()) R.pri[i] = 0ull;
            T.sync();
            for (uint32_t k = T.rank(); k < m; k += T.size()) {
                if (SC.done(k) != kUncolored) continue;
                const uint32_t a = SC.ab(k) & 0xFFFFu, b = SC.ab(k) >> 16;
                const unsigned long long pk = (static_cast<unsigned long long>(hash_u32(k)) << 32) | k;
                if (SB.im(a) != 0.f) atomicMax(reinterpret_cast<unsigned long long*>(&R.pri[a]), pk);
                if (SB.im(b) != 0.f) atomicMax(reinterpret_cast<unsigned long long*>(&R.pri[b]), pk);
            }
            T.sync();
            for (uint32_t k = T.rank(); k < m; k += T.size()) {
                if (SC.done(k) != kUncolored) continue;
                const uint32_t a = SC.ab(k) & 0xFFFFu, b = SC.ab(k) >> 16;
                const bool da = SB.im(a) != 0.f, db = SB.im(b) != 0.f;
                const uint64_t pk = (static_cast<uint64_t>(hash_u32(k)) << 32) | k;
                if ((da && R.pri[a] != pk) || (db && R.pri[b] != pk)) continue;  // not a local maximum
                const uint64_t used = (da ? R.mask[a] : 0ull) | (db ? R.mask[b] : 0ull);
                if (~used == 0ull) {  // > 64 colours: the reference falls back to the serial order
                    sh.over = 1u;
                    continue;
                }
                const uint32_t col = static_cast<uint32_t>(__ffsll(static_cast<long long>(~used)) - 1);
                SC.done(k) = col;
                const unsigned long long bit = 1ull << col;
                if (da) atomicOr(reinterpret_cast<unsigned long long*>(&R.mask[a]), bit);
                if (db) atomicOr(reinterpret_cast<unsigned long long*>(&R.mask[b]), bit);
                atomicMax(&sh.maxcol, col);
                atomicSub(&sh.rem, 1u);
            }
            T.sync();
            ++rounds;
        }
        colored = sh.rem == 0u && sh.over == 0u;
        n_colors = sh.maxcol + 1u;
        T.sync();
    }
    // ── groups: colours, or the levels of the sequential order ──
    uint32_t groups = n_colors, base = 0u;
    if (!colored) {
        groups = scene_levels(T, m, SC, &sh.maxcol);
        base = 1u;
        if (groups == 0u) {
            if (T.leader()) raise_error(DYPH_ERR_TIMEOUT, 11u);
            return false;
        }
    }
    scene_group(T, m, groups, base, SC, sh.scan, &sh.carry);
    if (sweep_start && T.leader()) {
        uint64_t t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        *sweep_start = t;
    }
    // ── sweeps and renormalisation ──
    bool deferred = false;
    if (groups_out) *groups_out = groups;
    for (int iter = 0; iter < n_iters; ++iter) {
        if (iter == 0 || deferred) {
            scene_sweep<kRecord>(T, groups, SB, SC, mu, dt, &sh.flag, rec, iter);
            deferred = sh.flag != 0;
        }
        if (rec && iter == 0)
            for (uint32_t i = T.rank(); i < nb; i += T.size()) {
                float* q = rec->qs + rec->b0 + i;
                q[0] = SB.qw(i);
                q[rec->qs_stride] = SB.qx(i);
                q[2ull * rec->qs_stride] = SB.qy(i);
                q[3ull * rec->qs_stride] = SB.qz(i);
            }
        const int times = deferred ? 1 : n_iters - iter;
        for (uint32_t i = T.rank(); i < nb; i += T.size()) {
            float qw = SB.qw(i), qx = SB.qx(i), qy = SB.qy(i), qz = SB.qz(i);
            for (int t = 0; t < times; ++t) renormalize(qw, qx, qy, qz);
            SB.qw(i) = qw; SB.qx(i) = qx; SB.qy(i) = qy; SB.qz(i) = qz;
        }
        T.sync();
        if (!deferred) break;
    }
    colored_out = colored;
    n_colors_out = n_colors;
    rounds_out = rounds;
    return true;
}

template <class Team>
__device__ __forceinline__ void scene_stats(const Team& T, uint32_t* meta, bool colored, uint32_t n_colors,
                                            uint32_t rounds) {
    if (T.leader()) {
        if (colored) {
            atomicMax(&meta[kMetaMaxColor], n_colors - 1u);
            meta[kMetaSceneColored] = 1u;
        }
        atomicMax(&meta[kMetaRounds], rounds);
        meta[kMetaDecision] = kDecisionScenes;
    }
}

__global__ void __launch_bounds__(kSceneThreads, 4) scene_solve_kernel(dyph_contacts cv, dyph_bodies gb,
                                                                       SceneBufs S, int mode, int n_iters,
                                                                       float mu, float dt,
                                                                       uint32_t* __restrict__ color,
                                                                       uint32_t* __restrict__ meta) {
    extern __shared__ __align__(16) unsigned char scene_smem[];
    __shared__ SceneShared sh;
    const GlobalBodies B{gb};
    const BlockTeam T;
    for (uint32_t t = blockIdx.x; t < S.n_scenes; t += gridDim.x) {
        const uint32_t s = S.order[t];
        const uint32_t b0 = S.body_offset[s], nb = S.body_offset[s + 1] - b0;
        const uint32_t k0 = S.range[2 * s], m = S.range[2 * s + 1] - k0;
        if (m == 0) continue;  // no contacts: the reference's solve returns at once
        // ── layout: bodies, then (if they fit) the contact words ──
        const uint32_t ldb = (nb + 3u) & ~3u;
        float* fb = reinterpret_cast<float*>(scene_smem);
        const SceneSolverRows R = scene_solver_rows(fb, ldb);
        const uint32_t body_bytes = scene_body_bytes(nb);
        const uint32_t ldc = (m + 4u) & ~3u;  // >= m + 1: group offsets take m + 1 words
        const bool in_smem = body_bytes + kSceneWords * 4u * ldc <= S.smem_bytes;
        const SceneBodies SB{fb, ldb};
        // (in the scratch, scene s owns words [k0 + s, k0 + s + m] of each row: m + 1 words)
        const SceneContacts SC{in_smem ? reinterpret_cast<uint32_t*>(scene_smem + body_bytes) : S.scratch + k0 + s,
                               in_smem ? ldc : S.scratch_stride};
        // ── stage the scene's bodies and contacts ──
        scene_load_bodies(T, B, b0, nb, fb, ldb);
        for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) R.cnt[i] = 0u;
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) {
            const uint32_t a = cv.body_a[k0 + k] - b0, b = cv.body_b[k0 + k] - b0;
            SC.ab(k) = a | (b << 16);
            SC.lam(k) = 0.f;
            const uint32_t c = k0 + k;
            SC.g(0, k) = cv.pos_x[c]; SC.g(1, k) = cv.pos_y[c]; SC.g(2, k) = cv.pos_z[c];
            SC.g(3, k) = cv.norm_x[c]; SC.g(4, k) = cv.norm_y[c]; SC.g(5, k) = cv.norm_z[c];
            SC.g(6, k) = cv.depth[c];
            SC.pb(k) = kSceneNone;
            if (SB.im(b) != 0.f) atomicAdd(&R.cnt[b], 1u);
        }
        __syncthreads();
        bool colored = false;
        uint32_t n_colors = 0, rounds = 0;
        if (!scene_solve(T, nb, m, SB, R, SC, mode, n_iters, mu, dt, sh, colored, n_colors, rounds)) return;
        // ── write back, colours and statistics ──
        scene_store_bodies(T, B, b0, nb, SB);
        for (uint32_t k = threadIdx.x; k < m; k += blockDim.x) color[k0 + k] = colored ? SC.done(k) : kUncolored;
        scene_stats(T, meta, colored, n_colors, rounds);
        __syncthreads();
    }
}

}  // namespace
}  // namespace dyph
