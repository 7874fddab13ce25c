// Dataflow XPBD path (included by solver.cu): the reference's Jones–Plassmann
// colouring and colour-ordered Gauss–Seidel sweep, scheduled per contact
// instead of per round / per colour.
//
// Facts it rests on (xpbd_solver.cpp:645-732):
//   * priorities hash(k) << 32 | k are distinct and fixed across rounds, and a
//     contact wins a round exactly when every uncoloured contact sharing one of
//     its dynamic bodies has a lower priority. So every higher-priority
//     neighbour is coloured before it and no lower-priority one is: its colour
//     is the lowest colour unused by its higher-priority neighbours (greedy
//     colouring in priority order), and its round is the longest chain of
//     higher-priority neighbours ending at it.
//   * the sweep solves the contacts of one body in ascending colour order, and
//     contacts that share no dynamic body commute exactly.
// So each dynamic body gets its contact list sorted by priority (colouring) and
// then by colour (sweep), and a contact waits only for its predecessor on the
// lists of its two bodies. Published cells are write-once (0 = not yet), so
// the colouring polls them with relaxed loads; the sweep hands body state on
// with release / acquire. Every thread works through its own contacts in
// priority (then colour) order, all threads are co-resident (cooperative
// launch) and a warp never blocks on one lane, so the highest-priority
// (lowest-colour) unfinished contact can always run: no deadlock.
#pragma once

namespace dyph {
namespace {

constexpr int kFlowThreads = 256;
constexpr int kFlowItems = 16;     // contacts per thread; more -> the round-synchronous kernel
constexpr int kBodySlots = 64;     // list slots per body: a body with more contacts needs > 64 colours
constexpr uint32_t kNoLink = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t ld_relaxed_u64(const unsigned long long* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u32(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// With a relaxed load that saw a release store before it, this fence makes the
// writer's earlier stores visible to the loads after it (acquire pattern).
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

struct FlowBufs {
    uint32_t* body_cnt;          // [nb] contacts on each dynamic body
    // [nb * kBodySlots] (key << 32 | entry), entry = contact << 1 | side; the
    // key half is 0 until the colouring writes the contact's colour there.
    unsigned long long* body_list;
    uint32_t* slot;              // [2 nc] list slot of each entry
    uint32_t* link;              // [2 nc] predecessor entry of each entry on its body's list
    unsigned long long* cmask;   // [2 nc] colours used on the entry's body up to and including it
    uint32_t* cround;            // [nc] JP round + 1 of each contact
    // [2 cap][16] body state handed along each body's colour-ordered list: the
    // 13 state floats of the entry's body after the contact, each word
    // (tag << 32 | float bits), tag = the sweep pass's number.
    unsigned long long* hand;
    uint32_t hand_cap;           // entries the records were allocated for (2 max contacts)
    uint32_t* tail;              // [nb] last entry of each body's colour-ordered list
    uint32_t* tag;               // [1] last sweep-pass number used (kept across solves)
    // Sequential order: every dynamic body's entries in one array (any count).
    uint32_t* csr_off;           // [nb + 1] first entry of each body
    uint32_t* csr_cur;           // [nb] fill cursors
    uint32_t* csr;               // [2 nc] entries
    uint32_t* partial;           // [kFlowMaxBlocks] per-block sums of the offset scan
};

constexpr uint32_t kSeqOneBlock = 2048;  // sequential order up to this many contacts: the one-block kernel
constexpr int kFlowMaxBlocks = 4096;

constexpr int kHandWords = 16;  // record stride (13 words used): 128 bytes

__device__ __forceinline__ uint64_t hand_word(uint32_t tag, float v) {
    return (static_cast<uint64_t>(tag) << 32) | __float_as_uint(v);
}

// Load a record into body slot j of L; true when all 13 words carry `tag`.
// The last word is written last, so it is polled alone first: a waiting
// contact then costs one 8-byte load per pass, not thirteen.
__device__ __forceinline__ bool load_hand(const unsigned long long* r, uint32_t tag, LocalPair& L, int j) {
    if (static_cast<uint32_t>(ld_relaxed_u64(r + 12) >> 32) != tag) return false;
    uint64_t w[13];
#pragma unroll
    for (int i = 0; i < 13; ++i) w[i] = ld_relaxed_u64(r + i);
    bool ok = true;
#pragma unroll
    for (int i = 0; i < 13; ++i) ok = ok && static_cast<uint32_t>(w[i] >> 32) == tag;
    L.p[j][0] = __uint_as_float(static_cast<uint32_t>(w[0]));
    L.p[j][1] = __uint_as_float(static_cast<uint32_t>(w[1]));
    L.p[j][2] = __uint_as_float(static_cast<uint32_t>(w[2]));
    L.q[j][0] = __uint_as_float(static_cast<uint32_t>(w[3]));
    L.q[j][1] = __uint_as_float(static_cast<uint32_t>(w[4]));
    L.q[j][2] = __uint_as_float(static_cast<uint32_t>(w[5]));
    L.q[j][3] = __uint_as_float(static_cast<uint32_t>(w[6]));
    L.v[j][0] = __uint_as_float(static_cast<uint32_t>(w[7]));
    L.v[j][1] = __uint_as_float(static_cast<uint32_t>(w[8]));
    L.v[j][2] = __uint_as_float(static_cast<uint32_t>(w[9]));
    L.w[j][0] = __uint_as_float(static_cast<uint32_t>(w[10]));
    L.w[j][1] = __uint_as_float(static_cast<uint32_t>(w[11]));
    L.w[j][2] = __uint_as_float(static_cast<uint32_t>(w[12]));
    return ok;
}

__device__ __forceinline__ void store_hand(unsigned long long* r, uint32_t tag, const LocalPair& L, int j) {
    const float f[13] = {L.p[j][0], L.p[j][1], L.p[j][2], L.q[j][0], L.q[j][1], L.q[j][2], L.q[j][3],
                         L.v[j][0], L.v[j][1], L.v[j][2], L.w[j][0], L.w[j][1], L.w[j][2]};
#pragma unroll
    for (int i = 0; i < 13; ++i) st_relaxed_u64(r + i, hand_word(tag, f[i]));
}

// The 13 state floats of body bi from the SoA arrays.
__device__ __forceinline__ void load_state(const GlobalBodies& B, uint32_t bi, LocalPair& L, int j) {
    L.p[j][0] = B.px(bi); L.p[j][1] = B.py(bi); L.p[j][2] = B.pz(bi);
    L.q[j][0] = B.qw(bi); L.q[j][1] = B.qx(bi); L.q[j][2] = B.qy(bi); L.q[j][3] = B.qz(bi);
    L.v[j][0] = B.vx(bi); L.v[j][1] = B.vy(bi); L.v[j][2] = B.vz(bi);
    L.w[j][0] = B.wx(bi); L.w[j][1] = B.wy(bi); L.w[j][2] = B.wz(bi);
}

// Sort a thread's items (at most kFlowItems) by key, ascending.
__device__ __forceinline__ void sort_items(uint32_t* item, uint32_t* key, int n) {
    for (int i = 1; i < n; ++i) {
        const uint32_t v = item[i], kv = key[i];
        int j = i;
        while (j > 0 && key[j - 1] > kv) {
            item[j] = item[j - 1];
            key[j] = key[j - 1];
            --j;
        }
        item[j] = v;
        key[j] = kv;
    }
}

// Link every entry to its predecessor on its body's list in ascending key
// order, key = ~hash (descending priority) or the colour. One thread per
// contact scans its bodies' lists (at most kBodySlots entries each).
template <bool BY_COLOR>
__device__ __forceinline__ void link_lists(const FlowBufs& F, const dyph_contacts& cv, const GlobalBodies& B,
                                           uint32_t nc, const uint32_t* color, uint32_t gtid, uint32_t gstride) {
    for (uint32_t k = gtid; k < nc; k += gstride) {
        const uint32_t mykey = BY_COLOR ? color[k] : ~hash_u32(k);
        for (uint32_t side = 0; side < 2u; ++side) {
            const uint32_t x = side ? cv.body_b[k] : cv.body_a[k];
            if (B.im(x) == 0.f) continue;
            const uint32_t e = 2u * k + side;
            const uint32_t m = min(F.body_cnt[x], static_cast<uint32_t>(kBodySlots));
            const unsigned long long* L = F.body_list + static_cast<size_t>(x) * kBodySlots;
            uint32_t best = kNoLink, best_key = 0;
            bool last = true;
            for (uint32_t i = 0; i < m; ++i) {
                const uint64_t v = L[i];
                const uint32_t e2 = static_cast<uint32_t>(v);
                const uint32_t key2 = BY_COLOR ? static_cast<uint32_t>(v >> 32) : ~hash_u32(e2 >> 1);
                if (e2 != e && key2 < mykey && (best == kNoLink || key2 > best_key)) {
                    best = e2;
                    best_key = key2;
                }
                last = last && !(e2 != e && key2 > mykey);
            }
            F.link[e] = best;
            if (BY_COLOR && last) F.tail[x] = e;
        }
    }
}

__device__ __forceinline__ uint32_t block_max(uint32_t v, uint32_t* smem) {
    for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, d));
    if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t r = 0;
    for (int w = 0; w < kFlowThreads / 32; ++w) r = max(r, smem[w]);
    __syncthreads();
    return r;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t* smem) {
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    if ((threadIdx.x & 31) == 0) smem[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t r = 0;
    for (int w = 0; w < kFlowThreads / 32; ++w) r += smem[w];
    __syncthreads();
    return r;
}

// Sequential order (XpbdSolver::run_serial, xpbd_solver.cpp:559-587): each
// dynamic body's contacts in one exact-size list, each entry linked to the
// body's previous contact in contact order. Four grid phases.
__device__ __forceinline__ bool link_sequential(const FlowBufs& F, const dyph_contacts& cv, const GlobalBodies& B,
                                                uint32_t nc, uint32_t nb, uint32_t* bar, uint32_t* s_red,
                                                uint32_t* s_scan, uint32_t gtid, uint32_t gstride) {
    const uint32_t nblk = gridDim.x;
    const uint32_t chunk = (nb + nblk - 1) / nblk;
    const uint32_t lo = min(blockIdx.x * chunk, nb), hi = min(lo + chunk, nb);
    uint32_t sum = 0;
    for (uint32_t x = lo + threadIdx.x; x < hi; x += blockDim.x) sum += F.body_cnt[x];
    sum = block_sum(sum, s_red);
    if (threadIdx.x == 0) F.partial[blockIdx.x] = sum;
    if (!grid_barrier(bar, nblk)) return false;
    uint32_t pre = 0;
    for (uint32_t i = threadIdx.x; i < blockIdx.x; i += blockDim.x) pre += F.partial[i];
    uint32_t carry = block_sum(pre, s_red);
    for (uint32_t base = lo; base < hi; base += blockDim.x) {
        const uint32_t x = base + threadIdx.x;
        const uint32_t v = x < hi ? F.body_cnt[x] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kFlowThreads>(v, s_scan, tot);
        if (x < hi) {
            F.csr_off[x] = carry + ex;
            F.csr_cur[x] = 0u;
        }
        carry += tot;
    }
    if (blockIdx.x == nblk - 1 && threadIdx.x == 0) F.csr_off[nb] = carry;
    if (!grid_barrier(bar, nblk)) return false;
    for (uint32_t k = gtid; k < nc; k += gstride) {
        for (uint32_t side = 0; side < 2u; ++side) {
            const uint32_t x = side ? cv.body_b[k] : cv.body_a[k];
            if (B.im(x) == 0.f) continue;
            F.csr[F.csr_off[x] + atomicAdd(&F.csr_cur[x], 1u)] = 2u * k + side;
        }
    }
    if (!grid_barrier(bar, nblk)) return false;
    for (uint32_t k = gtid; k < nc; k += gstride) {
        for (uint32_t side = 0; side < 2u; ++side) {
            const uint32_t x = side ? cv.body_b[k] : cv.body_a[k];
            if (B.im(x) == 0.f) continue;
            const uint32_t e = 2u * k + side;
            uint32_t best = kNoLink, best_k = 0;
            bool last = true;
            for (uint32_t i = F.csr_off[x], end = F.csr_off[x + 1]; i < end; ++i) {
                const uint32_t e2 = F.csr[i], k2 = e2 >> 1;
                if (k2 < k && (best == kNoLink || k2 > best_k)) {
                    best = e2;
                    best_k = k2;
                }
                last = last && k2 <= k;
            }
            F.link[e] = best;
            if (last) F.tail[x] = e;
        }
    }
    return grid_barrier(bar, nblk);
}

__global__ void __launch_bounds__(kFlowThreads) flow_solve_kernel(dyph_contacts cv, GlobalBodies B, int mode,
                                                                  int n_iters, float mu, float dt,
                                                                  float* __restrict__ lambda,
                                                                  uint32_t* __restrict__ color, FlowBufs F,
                                                                  uint32_t* __restrict__ meta) {
    __shared__ uint32_t s_red[kFlowThreads / 32];
    __shared__ uint32_t s_scan[kFlowThreads / 32];
    const uint32_t nc = contact_count(cv);
    if (nc == 0) return;
    const bool seq_wanted = wants_sequential(mode, nc);
    if (mode == DYPH_SOLVER_REFERENCE_ROUNDS && !seq_wanted) return;  // the round-synchronous kernel
    if (seq_wanted && nc <= kSeqOneBlock) return;                     // the one-block sequential kernel
    const uint32_t gstride = gridDim.x * blockDim.x;
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    if (nc > static_cast<uint32_t>(kFlowItems) * gstride) {  // too many contacts per thread
        if (gtid == 0) meta[kMetaDecision] = seq_wanted ? 1u : 3u;
        return;
    }
    const uint32_t nb = B.v.n;
    const uint32_t nblk = gridDim.x;
    uint32_t* bar = meta + kMetaBarrier;
    stamp(meta, gtid, 0);
    // Sweep passes are numbered on from the last solve's, so a record left by
    // an earlier pass never carries the current tag and nothing is cleared.
    // Before the 32-bit numbers could wrap, every record is cleared once.
    uint32_t tag_base = *F.tag;
    if (tag_base > 0x7FFFFFFFu) {
        for (size_t i = gtid; i < static_cast<size_t>(F.hand_cap) * kHandWords; i += gstride) F.hand[i] = 0ull;
        tag_base = 0u;
    }

    // ── set-up: clear, then put every contact on its dynamic bodies' lists ──
    for (uint32_t x = gtid; x < nb; x += gstride) F.body_cnt[x] = 0u;
    for (uint32_t k = gtid; k < nc; k += gstride) {
        F.cmask[2 * k] = 0ull;
        F.cmask[2 * k + 1] = 0ull;
        F.cround[k] = 0u;
        lambda[k] = 0.f;
        color[k] = kUncolored;
    }
    if (!grid_barrier(bar, nblk)) return;
    for (uint32_t k = gtid; k < nc; k += gstride) {
        const uint32_t a = cv.body_a[k], b = cv.body_b[k];
        if (B.im(a) != 0.f) {
            const uint32_t s = atomicAdd(&F.body_cnt[a], 1u);
            if (s < static_cast<uint32_t>(kBodySlots)) {
                F.body_list[static_cast<size_t>(a) * kBodySlots + s] = 2u * k;
                F.slot[2 * k] = s;
            } else {
                meta[kMetaOverflow] = 1u;  // > 64 contacts on a body: > 64 colours
            }
        }
        if (B.im(b) != 0.f) {
            const uint32_t s = atomicAdd(&F.body_cnt[b], 1u);
            if (s < static_cast<uint32_t>(kBodySlots)) {
                F.body_list[static_cast<size_t>(b) * kBodySlots + s] = 2u * k + 1u;
                F.slot[2 * k + 1] = s;
            } else {
                meta[kMetaOverflow] = 1u;
            }
        }
    }
    if (!grid_barrier(bar, nblk)) return;
    // More than 64 contacts on a body means more than 64 colours: the
    // reference's serial fallback (xpbd_solver.cpp:690-693).
    bool seq = seq_wanted || ld_acquire(&meta[kMetaOverflow]) != 0u;
    uint32_t item[kFlowItems], key[kFlowItems];
    int n_items = 0;
    if (!seq) {
    link_lists<false>(F, cv, B, nc, color, gtid, gstride);
    if (!grid_barrier(bar, nblk)) return;
    stamp(meta, gtid, 1);

    // ── colouring: greedy in priority order, each contact after its list predecessors ──
    // Lanes of a warp take contacts far apart (position lane * warps + warp),
    // so they rarely wait on one another. The warp polls in lock step: every
    // pass each lane checks its current contact once and finishes it if its
    // predecessors are published, so no lane ever blocks its warp.
    const uint32_t n_warps = gstride / 32u;
    const uint32_t pos = (threadIdx.x & 31u) * n_warps + (gtid >> 5);
    for (uint32_t k = pos; k < nc; k += gstride) {
        item[n_items] = k;
        key[n_items] = ~hash_u32(k);
        ++n_items;
    }
    sort_items(item, key, n_items);
    uint32_t my_max_color = 0, my_rounds = 0;
    {
        int cur = 0;
        bool have = false;
        uint32_t k = 0, a = 0, b = 0, la = kNoLink, lb = kNoLink, ra = 0, rb = 0;
        bool da = false, db = false;
        uint64_t ma = 0, mb = 0;
        uint32_t idle = 0;
        while (__any_sync(0xffffffffu, cur < n_items)) {
            bool progressed = false;
            if (cur < n_items) {
                if (!have) {
                    k = item[cur];
                    a = cv.body_a[k];
                    b = cv.body_b[k];
                    da = B.im(a) != 0.f;
                    db = B.im(b) != 0.f;
                    la = da ? F.link[2 * k] : kNoLink;
                    lb = db ? F.link[2 * k + 1] : kNoLink;
                    ma = mb = 0;
                    ra = rb = 0;
                    have = true;
                }
                if (la != kNoLink) {
                    if (ma == 0) ma = ld_relaxed_u64(&F.cmask[la]);
                    if (ra == 0) ra = ld_relaxed_u32(&F.cround[la >> 1]);
                }
                if (lb != kNoLink) {
                    if (mb == 0) mb = ld_relaxed_u64(&F.cmask[lb]);
                    if (rb == 0) rb = ld_relaxed_u32(&F.cround[lb >> 1]);
                }
                if ((la == kNoLink || (ma != 0 && ra != 0)) && (lb == kNoLink || (mb != 0 && rb != 0))) {
                    const uint64_t used = ma | mb;
                    uint64_t bit;
                    if (~used == 0ull) {
                        bit = ~0ull;  // > 64 colours at a body: publish anyway so the lists drain
                        meta[kMetaOverflow] = 1u;
                    } else {
                        const uint32_t col = static_cast<uint32_t>(__ffsll(static_cast<long long>(~used)) - 1);
                        bit = 1ull << col;
                        color[k] = col;
                        my_max_color = max(my_max_color, col);
                        // the colour is the key of the sweep's list order
                        if (da)
                            reinterpret_cast<uint32_t*>(F.body_list + static_cast<size_t>(a) * kBodySlots +
                                                        F.slot[2 * k])[1] = col;
                        if (db)
                            reinterpret_cast<uint32_t*>(F.body_list + static_cast<size_t>(b) * kBodySlots +
                                                        F.slot[2 * k + 1])[1] = col;
                    }
                    const uint32_t round = max(ra, rb);  // predecessors store round + 1
                    my_rounds = max(my_rounds, round + 1u);
                    st_relaxed_u32(&F.cround[k], round + 1u);
                    if (da) st_relaxed_u64(&F.cmask[2 * k], ma | bit);
                    if (db) st_relaxed_u64(&F.cmask[2 * k + 1], mb | bit);
                    ++cur;
                    have = false;
                    progressed = true;
                }
            }
            if (__any_sync(0xffffffffu, progressed)) {
                idle = 0;
            } else {
                if (++idle > spin_limit()) {
                    raise_error(DYPH_ERR_TIMEOUT, 9u);
                    break;
                }
                if ((idle & 1023u) == 0u && ld_relaxed_u32(&g_device_error) == DYPH_ERR_TIMEOUT) break;
                __nanosleep(32);
            }
        }
    }
    {
        const uint32_t bm = block_max(my_max_color, s_red);
        const uint32_t br = block_max(my_rounds, s_red);
        if (threadIdx.x == 0) {
            atomicMax(&meta[kMetaMaxColor], bm);
            atomicMax(&meta[kMetaRounds], br);
        }
    }
    if (!grid_barrier(bar, nblk)) return;
    // JP stops after MAX_ROUNDS rounds (xpbd_solver.cpp:645): a contact whose
    // round index reaches it is left uncoloured -> serial fallback.
    // (A colouring wait that gave up also takes the sequential order.)
    seq = ld_acquire(&meta[kMetaOverflow]) != 0u || ld_acquire(&meta[kMetaRounds]) > kMaxRounds ||
          ld_relaxed_u32(&g_device_error) == DYPH_ERR_TIMEOUT;
    stamp(meta, gtid, 2);
    if (!seq) {
        link_lists<true>(F, cv, B, nc, color, gtid, gstride);
        for (int i = 0; i < n_items; ++i) key[i] = color[item[i]];
        sort_items(item, key, n_items);
        if (!grid_barrier(bar, nblk)) return;
    }
    }  // !seq
    if (seq) {
        // Contact order: each thread's contacts ascending, lists linked by index.
        if (seq_wanted) {
            stamp(meta, gtid, 1);
            stamp(meta, gtid, 2);
        }
        n_items = 0;
        for (uint32_t k = gtid; k < nc; k += gstride) item[n_items++] = k;
        if (!link_sequential(F, cv, B, nc, nb, bar, s_red, s_scan, gtid, gstride)) return;
    }
    stamp(meta, gtid, 3);

    // ── sweeps: each contact after the lower-colour contacts of its two bodies ──
    // A contact takes each dynamic body's state from its list predecessor's
    // record (or from the arrays when it is first), solves on registers, and
    // publishes the two bodies' new states in its own records. A record is
    // complete when all its words carry the pass's tag: no flag, no fence.
    bool deferred_any = false;
    for (int iter = 0; iter < n_iters; ++iter) {
        if (iter == 0 || deferred_any) {
            const uint32_t tag = tag_base + static_cast<uint32_t>(iter) + 1u;
            int cur = 0;
            bool have = false, got_a = false, got_b = false;
            uint32_t k = 0, la = kNoLink, lb = kNoLink;
            bool da = false, db = false;
            float lc = 0.f;
            Contact ct{};
            LocalPair L;
            uint32_t idle = 0;
            while (__any_sync(0xffffffffu, cur < n_items)) {
                bool progressed = false;
                if (cur < n_items) {
                    if (!have) {
                        k = item[cur];
                        ct = load_contact(cv, k);
                        L.m[0] = B.im(ct.a);
                        L.m[1] = B.im(ct.b);
                        da = L.m[0] != 0.f;
                        db = L.m[1] != 0.f;
                        L.I[0][0] = B.ixx(ct.a); L.I[0][1] = B.iyy(ct.a); L.I[0][2] = B.izz(ct.a);
                        L.I[0][3] = B.ixy(ct.a); L.I[0][4] = B.ixz(ct.a); L.I[0][5] = B.iyz(ct.a);
                        L.I[1][0] = B.ixx(ct.b); L.I[1][1] = B.iyy(ct.b); L.I[1][2] = B.izz(ct.b);
                        L.I[1][3] = B.ixy(ct.b); L.I[1][4] = B.ixz(ct.b); L.I[1][5] = B.iyz(ct.b);
                        la = da ? F.link[2 * k] : kNoLink;
                        lb = db ? F.link[2 * k + 1] : kNoLink;
                        got_a = la == kNoLink;
                        got_b = lb == kNoLink;
                        if (got_a) load_state(B, ct.a, L, 0);
                        if (got_b) load_state(B, ct.b, L, 1);
                        lc = lambda[k];
                        have = true;
                    }
                    if (!got_a) got_a = load_hand(F.hand + static_cast<size_t>(la) * kHandWords, tag, L, 0);
                    if (!got_b) got_b = load_hand(F.hand + static_cast<size_t>(lb) * kHandWords, tag, L, 1);
                    if (got_a && got_b) {
                        if (ct.depth > 0.f && ct.depth - lc > 1e-6f) {
                            Contact lct = ct;
                            lct.a = 0u;
                            lct.b = 1u;
                            if (solve_contact(LocalPairRef{&L}, lct, mu, lc, dt) == kSolveDeferred)
                                meta[kMetaDeferred] = 1u;
                            lambda[k] = lc;
                        }
                        if (da) store_hand(F.hand + static_cast<size_t>(2 * k) * kHandWords, tag, L, 0);
                        if (db) store_hand(F.hand + static_cast<size_t>(2 * k + 1) * kHandWords, tag, L, 1);
                        ++cur;
                        have = false;
                        progressed = true;
                    }
                }
                if (__any_sync(0xffffffffu, progressed)) {
                    idle = 0;
                } else {
                    if (++idle > spin_limit()) {
                        raise_error(DYPH_ERR_TIMEOUT, 10u);
                        break;
                    }
                    if ((idle & 1023u) == 0u && ld_relaxed_u32(&g_device_error) == DYPH_ERR_TIMEOUT) break;
                    __nanosleep(32);
                }
            }
            if (!grid_barrier(bar, nblk)) return;
            deferred_any = ld_acquire(&meta[kMetaDeferred]) != 0u;
            // Each body's final state is its list tail's record.
            for (uint32_t x = gtid; x < nb; x += gstride) {
                if (B.im(x) == 0.f || F.body_cnt[x] == 0u) continue;
                LocalPair T;
                load_hand(F.hand + static_cast<size_t>(F.tail[x]) * kHandWords, tag, T, 0);
                store_local(B, x, T, 0);
            }
        }
        if (!deferred_any) {
            // Remaining iterations only renormalise: apply them all now.
            for (uint32_t i = gtid; i < nb; i += gstride) renorm_body(B, i, n_iters - iter);
            break;
        }
        for (uint32_t i = gtid; i < nb; i += gstride) renorm_body(B, i, 1);
        if (!grid_barrier(bar, nblk)) return;
    }
    if (gtid == 0) *F.tag = tag_base + static_cast<uint32_t>(n_iters > 0 ? n_iters : 0) + 1u;
    stamp(meta, gtid, 4);
    if (gtid == 0) {
        meta[kMetaFlowPath] = 1u;
        // 2 coloured; 4 serial fallback and 5 sequential order, both finished here
        meta[kMetaDecision] = !seq ? 2u : (seq_wanted ? 5u : 4u);
    }
}

}  // namespace
}  // namespace dyph
