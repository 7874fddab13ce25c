// Coloured XPBD path (included by solver.cu): Jones–Plassmann colouring and
// colour-ordered Gauss–Seidel sweeps in one cooperative kernel.
//
// Rounds and sweeps shrink fast: most contacts take a colour in the first few
// rounds and the late colours hold few contacts. So the kernel keeps a
// work-list of the still-uncoloured contacts (losers append themselves with a
// warp-aggregated atomic), and once a round's list, or every remaining colour,
// fits in one thread block, block 0 finishes alone with block barriers while
// the other blocks wait at one grid barrier.
#pragma once

namespace dyph {
namespace {

constexpr int kColorThreads = 512;
constexpr uint32_t kTail = kColorThreads;

// Priority of contact k in round r: the round in the top 8 bits, then the
// murmur3 hash (xpbd_solver.cpp:31-34), then k (k < 2^24). Inside a round the
// order is the reference's (hash << 32 | k); a value left from an earlier
// round is smaller than any current one, so the two priority buffers
// (read this round / post the next) are cleared once per solve, not per round.
__device__ __forceinline__ uint64_t jp_tag(uint32_t r, uint32_t k) {
    return (static_cast<uint64_t>(r) << 56) | (static_cast<uint64_t>(hash_u32(k)) << 24) | k;
}

struct JpCtx {
    dyph_contacts cv;
    GlobalBodies B;
    uint32_t* color;
    uint64_t* bpri;  // [2 nb]
    uint64_t* bmask;
    uint32_t* meta;
    uint32_t nb;
};

// Selection of contact k in round r (xpbd_solver.cpp:664-684); a contact that
// stays uncoloured posts its round r+1 priority. Returns true if uncoloured.
__device__ __forceinline__ bool jp_step(const JpCtx& X, uint32_t r, uint32_t k) {
    const uint64_t* pri = X.bpri + static_cast<size_t>(r & 1u) * X.nb;
    uint64_t* pri_next = X.bpri + static_cast<size_t>((r + 1u) & 1u) * X.nb;
    const uint32_t a = X.cv.body_a[k], b = X.cv.body_b[k];
    const bool da = X.B.im(a) != 0.f, db = X.B.im(b) != 0.f;
    const uint64_t tag = jp_tag(r, k);
    // L2 loads: the priorities were posted with atomics
    bool won = !((da && __ldcg(&pri[a]) != tag) || (db && __ldcg(&pri[b]) != tag));
    if (won) {
        const uint64_t used = (da ? __ldcg(&X.bmask[a]) : 0ull) | (db ? __ldcg(&X.bmask[b]) : 0ull);
        const uint64_t freebits = ~used;
        if (freebits == 0ull) {
            X.meta[kMetaOverflow] = 1u;  // > 64 colours at a body: the caller falls back to serial
            won = false;
        } else {
            const uint32_t col = static_cast<uint32_t>(__ffsll(static_cast<long long>(freebits)) - 1);
            X.color[k] = col;
            const uint64_t bit = 1ull << col;
            if (da) atomicOr(reinterpret_cast<unsigned long long*>(&X.bmask[a]), bit);
            if (db) atomicOr(reinterpret_cast<unsigned long long*>(&X.bmask[b]), bit);
            atomicMax(&X.meta[kMetaMaxColor], col);
        }
    }
    if (!won) {
        const uint64_t nt = jp_tag(r + 1u, k);
        if (da) atomicMax(reinterpret_cast<unsigned long long*>(&pri_next[a]), nt);
        if (db) atomicMax(reinterpret_cast<unsigned long long*>(&pri_next[b]), nt);
    }
    return !won;
}

// Phase timestamps of the coloured solve (thread 0 of block 0): start, after
// set-up, after colouring, after grouping, end (dyph_xpbd_download_phase_ns).
__device__ __forceinline__ void stamp(uint32_t* meta, uint32_t gtid, int i) {
    if (gtid != 0) return;
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    meta[kMetaTime + 2 * i] = static_cast<uint32_t>(t);
    meta[kMetaTime + 2 * i + 1] = static_cast<uint32_t>(t >> 32);
}

__device__ __forceinline__ void solve_one(const dyph_contacts& cv, const GlobalBodies& B, float* lambda,
                                          uint32_t* meta, uint32_t k, float mu, float dt) {
    const Contact ct = load_contact(cv, k);
    float lc = lambda[k];
    const int res = solve_contact(B, ct, mu, lc, dt);
    lambda[k] = lc;
    if (res == kSolveDeferred) meta[kMetaDeferred] = 1u;
}

__global__ void __launch_bounds__(kColorThreads) color_solve_kernel(dyph_contacts cv, GlobalBodies B, int mode,
                                                                    int n_iters, float mu, float dt,
                                                                    float* __restrict__ lambda,
                                                                    uint32_t* __restrict__ color,
                                                                    uint32_t* __restrict__ order,
                                                                    uint32_t* __restrict__ lists,
                                                                    uint64_t* __restrict__ bpri,
                                                                    uint64_t* __restrict__ bmask,
                                                                    uint32_t* __restrict__ meta) {
    __shared__ uint32_t s_off[65];
    __shared__ uint32_t s_list[2][kTail];
    __shared__ uint32_t s_len[2];
    __shared__ uint32_t s_wbase[kColorThreads / 32];
    const uint32_t nc = contact_count(cv);
    if (nc == 0 || wants_sequential(mode, nc)) return;
    // Runs when asked for, or when the dataflow kernel had too many contacts per thread.
    if (mode != DYPH_SOLVER_REFERENCE_ROUNDS && ld_acquire(&meta[kMetaDecision]) != 3u) return;
    const uint32_t nb = B.v.n;
    const uint32_t nblk = gridDim.x;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gstride = gridDim.x * blockDim.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t* bar = meta + kMetaBarrier;
    uint32_t* list_len = meta + kMetaListLen;  // [3], round r reads [r % 3], appends to [(r+1) % 3]
    const JpCtx X{cv, B, color, bpri, bmask, meta, nb};
    stamp(meta, gtid, 0);

    for (uint32_t k = gtid; k < nc; k += gstride) {
        lambda[k] = 0.f;
        color[k] = kUncolored;
        lists[k] = k;
    }
    for (uint32_t i = gtid; i < 2 * nb; i += gstride) bpri[i] = 0ull;
    for (uint32_t i = gtid; i < nb; i += gstride) bmask[i] = 0ull;
    if (gtid == 0) {
        list_len[0] = nc;
        list_len[1] = 0u;
        list_len[2] = 0u;
    }
    if (!grid_barrier(bar, nblk)) return;
    for (uint32_t k = gtid; k < nc; k += gstride) {  // round 0 priorities
        const uint32_t a = cv.body_a[k], b = cv.body_b[k];
        const uint64_t t0 = jp_tag(0u, k);
        if (B.im(a) != 0.f) atomicMax(reinterpret_cast<unsigned long long*>(&bpri[a]), t0);
        if (B.im(b) != 0.f) atomicMax(reinterpret_cast<unsigned long long*>(&bpri[b]), t0);
    }
    if (!grid_barrier(bar, nblk)) return;
    stamp(meta, gtid, 1);

    // ── Jones–Plassmann rounds (xpbd_solver.cpp:645-688) ──
    uint32_t r = 0, remaining = nc;
    while (true) {
        uint32_t* cur = lists + static_cast<size_t>(r & 1u) * cv.capacity;
        uint32_t* nxt = lists + static_cast<size_t>((r + 1u) & 1u) * cv.capacity;
        remaining = ld_acquire(&list_len[r % 3u]);
        if (remaining == 0u || ld_acquire(&meta[kMetaOverflow]) != 0u || r >= kMaxRounds) break;
        if (remaining <= kTail) {
            if (blockIdx.x == 0) {  // block-local tail rounds
                if (threadIdx.x < remaining) s_list[0][threadIdx.x] = __ldcg(&cur[threadIdx.x]);
                if (threadIdx.x == 0) s_len[0] = remaining;
                __syncthreads();
                uint32_t c = 0;
                while (s_len[c] > 0u && r < kMaxRounds && *reinterpret_cast<volatile uint32_t*>(&meta[kMetaOverflow]) == 0u) {
                    if (threadIdx.x == 0) s_len[c ^ 1u] = 0u;
                    __syncthreads();
                    const uint32_t len = s_len[c];
                    if (threadIdx.x < len) {
                        const uint32_t k = s_list[c][threadIdx.x];
                        if (jp_step(X, r, k)) s_list[c ^ 1u][atomicAdd(&s_len[c ^ 1u], 1u)] = k;
                    }
                    __syncthreads();
                    c ^= 1u;
                    ++r;
                }
                if (threadIdx.x == 0) meta[kMetaTailRemaining] = s_len[c];
                __syncthreads();
            }
            if (!grid_barrier(bar, nblk)) return;
            remaining = ld_acquire(&meta[kMetaTailRemaining]);
            break;
        }
        if (gtid == 0) list_len[(r + 2u) % 3u] = 0u;
        for (uint32_t base = blockIdx.x * blockDim.x; base < remaining; base += gstride) {
            const uint32_t idx = base + threadIdx.x;
            bool keep = false;
            uint32_t k = 0;
            if (idx < remaining) {
                k = __ldcg(&cur[idx]);
                keep = jp_step(X, r, k);
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (m) {  // warp-aggregated append of the losers
                if (lane == 0) s_wbase[warp] = atomicAdd(&list_len[(r + 1u) % 3u], static_cast<uint32_t>(__popc(m)));
                __syncwarp();
                if (keep) nxt[s_wbase[warp] + __popc(m & ((1u << lane) - 1u))] = k;
                __syncwarp();
            }
        }
        if (!grid_barrier(bar, nblk)) return;
        ++r;
    }
    if (gtid == 0) meta[kMetaRounds] = r;
    if (remaining != 0u || ld_acquire(&meta[kMetaOverflow]) != 0u) {  // serial fallback (xpbd_solver.cpp:690-693)
        if (gtid == 0) meta[kMetaDecision] = 1u;
        return;
    }
    stamp(meta, gtid, 2);
    const uint32_t n_colors = ld_acquire(&meta[kMetaMaxColor]) + 1u;

    // ── group contacts by colour (order inside a colour is irrelevant) ──
    for (uint32_t k = gtid; k < nc; k += gstride) atomicAdd(&meta[kMetaColorCount + color[k]], 1u);
    if (!grid_barrier(bar, nblk)) return;
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (uint32_t c = 0; c < n_colors; ++c) {
            s_off[c] = acc;
            acc += ld_acquire(&meta[kMetaColorCount + c]);
        }
        s_off[n_colors] = acc;
    }
    __syncthreads();
    for (uint32_t k = gtid; k < nc; k += gstride) {
        const uint32_t c = color[k];
        order[s_off[c] + atomicAdd(&meta[kMetaColorCursor + c], 1u)] = k;
    }
    // first colour from which every colour fits in one block
    uint32_t c_tail = n_colors;
    while (c_tail > 0 && s_off[c_tail] - s_off[c_tail - 1] <= kTail) --c_tail;
    if (!grid_barrier(bar, nblk)) return;
    stamp(meta, gtid, 3);

    // ── Gauss–Seidel across colours, parallel within a colour (xpbd_solver.cpp:718-732) ──
    bool deferred_any = false;
    for (int iter = 0; iter < n_iters; ++iter) {
        if (iter == 0 || deferred_any) {
            const uint32_t c_grid_end = (iter == 0) ? c_tail : n_colors;
            for (uint32_t ci = 0; ci < c_grid_end; ++ci) {
                for (uint32_t idx = s_off[ci] + gtid; idx < s_off[ci + 1]; idx += gstride)
                    solve_one(cv, B, lambda, meta, __ldcg(&order[idx]), mu, dt);
                if (!grid_barrier(bar, nblk)) return;
            }
            if (c_grid_end < n_colors) {
                if (blockIdx.x == 0) {
                    for (uint32_t ci = c_grid_end; ci < n_colors; ++ci) {
                        const uint32_t idx = s_off[ci] + threadIdx.x;
                        if (idx < s_off[ci + 1]) solve_one(cv, B, lambda, meta, __ldcg(&order[idx]), mu, dt);
                        __syncthreads();
                    }
                }
                if (!grid_barrier(bar, nblk)) return;
            }
            deferred_any = ld_acquire(&meta[kMetaDeferred]) != 0u;
        }
        if (!deferred_any) {
            // Remaining iterations only renormalise: apply them all now.
            for (uint32_t i = gtid; i < nb; i += gstride) renorm_body(B, i, n_iters - iter);
            break;
        }
        for (uint32_t i = gtid; i < nb; i += gstride) renorm_body(B, i, 1);
        if (!grid_barrier(bar, nblk)) return;
    }
    stamp(meta, gtid, 4);
    if (gtid == 0) meta[kMetaDecision] = 2u;
}

}  // namespace
}  // namespace dyph
