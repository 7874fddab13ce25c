// LBVH broadphase: Morton codes -> radix sort -> one-pass bottom-up Karras
// tree with fp16 boxes -> stackless traversal emitting (a, b) pairs already in
// ascending (a << 32 | b) order.
//
// Replaces Broadphase::build_and_query / sort_pairs (core/src/broadphase.cpp:
// 101-359). The tree is the reference's Karras tree node for node (same
// left / right / parent / NodeBox arrays, broadphase.cpp:158-288); it is built
// in a single kernel by letting each leaf walk up and the second child to
// arrive at a node merge the boxes (atomic rendezvous with release / acquire
// fences), instead of the reference's host-synchronised refit rounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "internal.cuh"

namespace dyph {
namespace {

constexpr int kBpThreads = 256;
constexpr int kMaxPartners = 32;  // per-thread sorted partner window (larger lists take extra passes)
constexpr int kFrontier = 128;     // pass 1a hands subtrees of at most this many leaves to pass 1b
constexpr int kFrontierItems = 16; // subtrees one query may hand on (more are walked in place)
constexpr int kQueuePerBody = 16;  // pass 1b queue capacity per body (overflow is walked in place)

// Single scene: 30-bit codes against the scene bounds. Batched scenes
// (codes64 != null): (scene << 30 | code) against each body's scene bounds,
// so every scene's leaves are contiguous after the sort.
__global__ void __launch_bounds__(kBpThreads) morton_kernel(GlobalBodies B, uint32_t n, dyph_aabb bounds,
                                                            uint32_t* __restrict__ codes,
                                                            uint32_t* __restrict__ sorted_idx,
                                                            uint32_t* __restrict__ counts,
                                                            uint32_t* __restrict__ tstatus, uint32_t n_tiles,
                                                            uint32_t* __restrict__ bucket_cnt,
                                                            uint64_t* __restrict__ codes64,
                                                            const uint32_t* __restrict__ scene_of,
                                                            const dyph_aabb* __restrict__ scene_bounds) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = tid; i < n; i += stride) {
        if (codes64) {
            const uint32_t sc = scene_of[i];
            codes64[i] = (static_cast<uint64_t>(sc) << 30) |
                         morton_code(B.px(i), B.py(i), B.pz(i), scene_bounds[sc]);
        } else {
            codes[i] = morton_code(B.px(i), B.py(i), B.pz(i), bounds);
        }
        sorted_idx[i] = i;
        bucket_cnt[i] = 0u;
    }
    for (uint32_t t = tid; t < n_tiles; t += stride) tstatus[t] = 0u;
    if (tid == 0) {
        counts[0] = 0u;
        counts[1] = 0u;
        counts[2] = 0u;
        counts[3] = 0u;  // pass 1b queue length
    }
}

// (code << 32 | body) as in the reference; batched: (scene << 52 | code << 22 | body).
__device__ __forceinline__ uint64_t key64(const uint32_t* codes, const uint64_t* codes64, const uint32_t* si, int i) {
    if (codes64) return (codes64[i] << 22) | static_cast<uint64_t>(si[i]);
    return (static_cast<uint64_t>(codes[i]) << 32) | static_cast<uint64_t>(si[i]);
}

// Common-prefix length between sorted positions i and i+1 (lbvh_delta,
// broadphase.cpp:38-41); -1 outside [0, n-1).
__device__ __forceinline__ int boundary_delta(const uint32_t* codes, const uint64_t* codes64, const uint32_t* si, int i,
                                              int n) {
    if (i < 0 || i >= n - 1) return -1;
    return __clzll(static_cast<long long>(key64(codes, codes64, si, i) ^ key64(codes, codes64, si, i + 1)));
}

__global__ void __launch_bounds__(kBpThreads) build_kernel(GlobalBodies B, GlobalShapes S, uint32_t n_u,
                                                           const uint32_t* __restrict__ codes,
                                                           const uint32_t* __restrict__ si, BvhBuffers T) {
    const int n = static_cast<int>(n_u);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t body = si[k];
    const uint64_t* codes64 = T.codes64;
    T.sorted_keys[k] = key64(codes, codes64, si, k);
    T.inv_sorted[body] = static_cast<uint32_t>(k);
    const uint32_t sh = B.shape(body);
    uint4 box = leaf_box(S.type(sh), B.px(body), B.py(body), B.pz(body), B.qw(body), B.qx(body), B.qy(body),
                         B.qz(body), S.hx(sh), S.hy(sh), S.hz(sh));
    int node = n - 1 + k;
    T.aabb[node] = box;
    // Static bodies (grounds, walls) are "large": pairs with them are found
    // from the other body's side, so no single thread walks the whole tree.
    uint32_t big = B.im(body) == 0.f ? 1u : 0u;
    T.big[node] = big;
    if (k == 0) {
        T.parent[0] = -1;
        T.root[0] = 0;
    }
    if (n == 1) {
        T.parent[0] = -1;
        return;
    }
    int l = k, r = k;
    while (true) {
        if (l == 0 && r == n - 1) return;  // this thread completed the root
        const int dl = boundary_delta(codes, codes64, si, l - 1, n);
        const int dr = boundary_delta(codes, codes64, si, r, n);
        const bool is_left = dr > dl;  // merge across boundary r: we are the left child
        const int s = is_left ? r : l - 1;
        // Publish our far end (left child: slot 2s, right child: slot 2s+1) and
        // box, then rendezvous at split s.
        T.slot[2 * s + (is_left ? 0 : 1)] = static_cast<uint32_t>(is_left ? l : r);
        // One acq_rel atomic: releases this child's slot / box / big writes and,
        // for the second arrival, acquires the sibling's.
        const uint32_t old = atom_add_acq_rel(&T.flags[s], 1u);
        if ((old & 1u) == 0u) return;  // first arrival: the sibling carries on
        // L2 loads (ld.global.cg): the sibling's writes were made on another SM.
        const int other = static_cast<int>(__ldcg(&T.slot[2 * s + (is_left ? 1 : 0)]));
        const int L = is_left ? l : other;
        const int R = is_left ? other : r;
        const int lidx = (L == s) ? (n - 1 + L) : s;
        const int ridx = (s + 1 == R) ? (n - 1 + R) : (s + 1);
        int pidx;
        if (L == 0 && R == n - 1) {
            pidx = 0;
        } else {
            const int pdl = boundary_delta(codes, codes64, si, L - 1, n);
            const int pdr = boundary_delta(codes, codes64, si, R, n);
            pidx = (pdr > pdl) ? R : L;
        }
        const uint4 sib = __ldcg(&T.aabb[is_left ? ridx : lidx]);
        box = is_left ? merge_box(box, sib) : merge_box(sib, box);
        big |= __ldcg(&T.big[is_left ? ridx : lidx]);
        T.big[pidx] = big;
        T.aabb[pidx] = box;
        T.left[pidx] = lidx;
        T.right[pidx] = ridx;
        T.parent[lidx] = pidx;
        T.parent[ridx] = pidx;
        T.range_lo[pidx] = L;
        T.range_hi[pidx] = R;
        T.rsplit[s] = ridx;
        l = L;
        r = R;
        node = pidx;
    }
}

struct Partners {
    uint32_t v[kMaxPartners];
    int m;
};

__device__ __forceinline__ void partner_insert(Partners& p, uint32_t b) {
    int pos = p.m;
    if (pos == kMaxPartners) {
        if (b >= p.v[kMaxPartners - 1]) return;
        pos = kMaxPartners - 1;
    } else {
        p.m++;
    }
    while (pos > 0 && p.v[pos - 1] > b) {
        p.v[pos] = p.v[pos - 1];
        --pos;
    }
    p.v[pos] = b;
}

// Batched scenes: first and last sorted leaf of every scene.
__global__ void __launch_bounds__(kBpThreads) scene_range_kernel(uint32_t n, const uint64_t* __restrict__ codes64,
                                                                 uint32_t* __restrict__ first,
                                                                 uint32_t* __restrict__ last) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t sc = static_cast<uint32_t>(codes64[k] >> 30);
    if (k == 0 || static_cast<uint32_t>(codes64[k - 1] >> 30) != sc) first[sc] = k;
    if (k == n - 1 || static_cast<uint32_t>(codes64[k + 1] >> 30) != sc) last[sc] = k;
}

// Traversal record of every node (32 bytes): box + left child / body, then
// lo, hi and the escape node — the right child of the internal node whose
// split is hi (the next node in pre-order once this subtree is skipped), or -1
// when hi is the last leaf.
__global__ void __launch_bounds__(kBpThreads) finalize_nodes_kernel(uint32_t n_u, BvhBuffers T) {
    const int n = static_cast<int>(n_u);
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 2 * n - 1) return;
    const uint4 box = T.aabb[j];
    int lo, hi, w;
    if (j >= n - 1) {
        lo = hi = j - (n - 1);
        w = static_cast<int>(T.sorted_idx[lo]);
    } else {
        lo = T.range_lo[j];
        hi = T.range_hi[j];
        w = T.left[j];
    }
    const int esc = (hi >= n - 1) ? -1 : T.rsplit[hi];
    T.trav[2 * j] = make_uint4(box.x, box.y, box.z, static_cast<uint32_t>(w));
    T.trav[2 * j + 1] = make_uint4(static_cast<uint32_t>(lo), static_cast<uint32_t>(hi), static_cast<uint32_t>(esc),
                                   T.big[j]);
}

// Pair search of leaf k (pass 1). Every overlapping pair must be found exactly
// once: a pair of two small leaves from the larger leaf index, a pair with a
// large (static) leaf from the small side, a pair of two large leaves from the
// larger index. So a small query visits leaves i < k plus large leaves i > k,
// and a large query visits only large leaves i < k.
//
// The walk covers the subtree at `start` (pre-order: it ends at the first node
// whose leaf range starts past `end_leaf`). `frontier(node)` is offered every
// wanted, overlapping internal node covering at most kFrontier leaves; when it
// returns true the walk hands that subtree on instead of descending into it.
template <typename F, typename G>
__device__ __forceinline__ void walk_pairs(const BvhBuffers& T, int n, const BoxF& q, int k, bool me_big, int start,
                                           int begin_leaf, int end_leaf, F&& visit, G&& frontier) {
    int node = start;
    int budget = 2 * n;
    while (node >= 0) {
        if (node >= 2 * n - 1 || --budget < 0) {
            raise_error(DYPH_ERR_INVALID, 6u);
            return;
        }
        const uint4 r0 = __ldg(&T.trav[2 * node]);
        const uint4 r1 = __ldg(&T.trav[2 * node + 1]);
        if (static_cast<int>(r1.x) > end_leaf) return;
        if (static_cast<int>(r1.y) < begin_leaf) {  // subtree before the query's scene
            node = static_cast<int>(r1.z);
            continue;
        }
        const bool before = static_cast<int>(r1.x) < k;
        const bool has_big = r1.w != 0u;
        const bool wanted = me_big ? (has_big && before) : (before || has_big);
        if (!wanted) {
            if (me_big && !before) return;  // pre-order lo never decreases
            node = static_cast<int>(r1.z);
            continue;
        }
        if (box_overlap(unpack_box(r0), q)) {
            if (node >= n - 1) {
                visit(r0.w);
            } else if (!(static_cast<int>(r1.y - r1.x) < kFrontier && frontier(node))) {
                node = static_cast<int>(r0.w);
                continue;
            }
        }
        node = static_cast<int>(r1.z);
    }
}

// Stackless pre-order traversal over the traversal records: on a hit at an
// internal node go to its left child, otherwise take the escape link. Visits
// only nodes whose leaf range starts below `leaf_end` (pre-order lo values
// never decrease, so the walk stops at the first node that starts at or past
// it). `visit(body)` is called for every overlapping leaf.
template <typename F>
__device__ __forceinline__ void walk(const BvhBuffers& T, int n, const BoxF& q, int leaf_begin, int leaf_end,
                                     F&& visit) {
    int node = 0;
    // A well-formed tree visits each node at most once; anything longer (or an
    // index outside the tree) is reported instead of followed.
    int budget = 2 * n;
    while (node >= 0) {
        if (node >= 2 * n - 1 || --budget < 0) {
            raise_error(DYPH_ERR_INVALID, 7u);
            return;
        }
        const uint4 r0 = __ldg(&T.trav[2 * node]);
        const uint4 r1 = __ldg(&T.trav[2 * node + 1]);
        if (static_cast<int>(r1.x) >= leaf_end) return;
        if (static_cast<int>(r1.y) < leaf_begin) {
            node = static_cast<int>(r1.z);
            continue;
        }
        const BoxF nb = unpack_box(r0);
        if (box_overlap(nb, q)) {
            if (node >= n - 1) {
                visit(r0.w);
            } else {
                node = static_cast<int>(r0.w);
                continue;
            }
        }
        node = static_cast<int>(r1.z);
    }
}

// All overlapping partners b > lo of a query box, smallest kMaxPartners kept.
__device__ __forceinline__ uint32_t traverse(const BvhBuffers& T, int n, const BoxF& q, uint32_t a, uint32_t lo,
                                             Partners& p, int leaf_begin, int leaf_end) {
    uint32_t count = 0;
    p.m = 0;
    walk(T, n, q, leaf_begin, leaf_end, [&](uint32_t b) {
        if (b > lo && b != a) {
            ++count;
            partner_insert(p, b);
        }
    });
    return count;
}

// Sorted-leaf range [begin, end] of the scene of leaf k (the whole tree for a
// single scene).
__device__ __forceinline__ void scene_leaves(const BvhBuffers& T, int n, int k, int& begin, int& end) {
    if (!T.codes64) {
        begin = 0;
        end = n;
        return;
    }
    const uint32_t sc = static_cast<uint32_t>(T.codes64[k] >> 30);
    begin = static_cast<int>(T.scene_first[sc]);
    end = static_cast<int>(T.scene_last[sc]);
}

__device__ __forceinline__ void bucket_pair(const BvhBuffers& T, uint32_t me, uint32_t other) {
    const uint32_t a = me < other ? me : other;
    const uint32_t b = me < other ? other : me;
    const uint32_t slot = atomicAdd(&T.bucket_cnt[a], 1u);
    if (slot < static_cast<uint32_t>(kBucket)) T.bucket[static_cast<size_t>(a) * kBucket + slot] = b;
}

// Pass 1a, one thread per leaf in Morton order (neighbouring threads walk the
// same part of the tree): walk the tree above subtrees of at most kFrontier
// leaves and queue (leaf, subtree) items for pass 1b, so each query's work is
// spread over several threads. Leaf k tests only leaves i < k (plus static
// leaves from the small side), so every overlapping pair is found once; the
// pair goes to the bucket of its smaller body index.
__global__ void __launch_bounds__(kBpThreads) pair_find_kernel(uint32_t n_u, BvhBuffers T, uint2* __restrict__ queue,
                                                               uint32_t queue_cap, uint32_t* __restrict__ queue_len) {
    const int n = static_cast<int>(n_u);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t items[kFrontierItems];
    uint32_t m = 0;
    if (k < n) {
        const uint4 r0 = __ldg(&T.trav[2 * (n - 1 + k)]);
        const uint4 r1 = __ldg(&T.trav[2 * (n - 1 + k) + 1]);
        const BoxF q = unpack_box(r0);
        const uint32_t me = r0.w;
        const bool me_big = r1.w != 0u;
        int sb, se;
        scene_leaves(T, n, k, sb, se);
        walk_pairs(
            T, n, q, k, me_big, 0, sb, se, [&](uint32_t other) { bucket_pair(T, me, other); },
            [&](int node) {
                if (m < static_cast<uint32_t>(kFrontierItems)) {
                    items[m++] = static_cast<uint32_t>(node);
                    return true;
                }
                return false;  // local list full: descend here instead
            });
    }
    // Warp-aggregated append of the items.
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t incl = m;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= static_cast<uint32_t>(d)) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    uint32_t base = 0;
    if (lane == 31 && total) base = atomicAdd(queue_len, total);
    base = __shfl_sync(0xffffffffu, base, 31);
    if (m == 0) return;
    const uint32_t first = base + incl - m;
    const BoxF q = unpack_box(__ldg(&T.trav[2 * (n - 1 + k)]));
    const uint32_t me = __ldg(&T.trav[2 * (n - 1 + k)]).w;
    const bool me_big = __ldg(&T.trav[2 * (n - 1 + k) + 1]).w != 0u;
    int sb, se;
    scene_leaves(T, n, k, sb, se);
    for (uint32_t i = 0; i < m; ++i) {
        if (first + i < queue_cap) {
            queue[first + i] = make_uint2(static_cast<uint32_t>(k), items[i]);
        } else {  // queue full: walk the subtree here
            const int f = static_cast<int>(items[i]);
            const int end_leaf = min(static_cast<int>(__ldg(&T.trav[2 * f + 1]).y), se);
            walk_pairs(
                T, n, q, k, me_big, f, sb, end_leaf, [&](uint32_t other) { bucket_pair(T, me, other); },
                [](int) { return false; });
        }
    }
}

// Pass 1b, one thread per queued (leaf, subtree) item.
__global__ void __launch_bounds__(kBpThreads) pair_subtree_kernel(uint32_t n_u, BvhBuffers T,
                                                                  const uint2* __restrict__ queue, uint32_t queue_cap,
                                                                  const uint32_t* __restrict__ queue_len) {
    const int n = static_cast<int>(n_u);
    const uint32_t len = min(*queue_len, queue_cap);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x) {
        const uint2 it = queue[i];
        const int k = static_cast<int>(it.x), f = static_cast<int>(it.y);
        const uint4 r0 = __ldg(&T.trav[2 * (n - 1 + k)]);
        const bool me_big = __ldg(&T.trav[2 * (n - 1 + k) + 1]).w != 0u;
        const BoxF q = unpack_box(r0);
        const uint32_t me = r0.w;
        int sb, se;
        scene_leaves(T, n, k, sb, se);
        const int end_leaf = min(static_cast<int>(__ldg(&T.trav[2 * f + 1]).y), se);
        walk_pairs(
            T, n, q, k, me_big, f, sb, end_leaf, [&](uint32_t other) { bucket_pair(T, me, other); },
            [](int) { return false; });
    }
}

// Pass 2, one thread per body in body order: place each body's pairs with a
// block scan + decoupled look-back (the counts are final after pass 1, so
// every tile publishes its aggregate at once), then write them sorted by b.
// Buckets go to a block queue and each warp ranks one bucket at a time
// (coalesced loads and stores); buckets that overflowed are rebuilt by a full
// traversal from the body's own leaf.
__global__ void __launch_bounds__(kBpThreads) pair_write_kernel(uint32_t n_u, BvhBuffers T, uint2* __restrict__ pairs,
                                                                uint32_t max_pairs, uint32_t* __restrict__ counts,
                                                                uint32_t* __restrict__ tstatus) {
    __shared__ uint32_t s_tile, s_excl, s_nbig;
    __shared__ uint32_t s_scan[kBpThreads / 32];
    __shared__ uint32_t s_big[kBpThreads], s_big_off[kBpThreads], s_big_cnt[kBpThreads];
    const int n = static_cast<int>(n_u);
    if (threadIdx.x == 0) {
        s_tile = atomicAdd(&counts[2], 1u);
        s_nbig = 0u;
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t a = tile * kBpThreads + threadIdx.x;
    const uint32_t cnt = a < n_u ? T.bucket_cnt[a] : 0u;
    uint32_t total;
    const uint32_t excl_block = block_exclusive_scan<kBpThreads>(cnt, s_scan, total);
    if (threadIdx.x < 32) {
        const uint32_t e = lookback_warp(tstatus, tile, total);
        if (threadIdx.x == 0) {
            s_excl = e;
            const uint32_t last_tile = (n_u - 1) / kBpThreads;
            if (tile == last_tile) {
                const uint32_t all = e + total;
                counts[1] = all;
                counts[0] = all < max_pairs ? all : max_pairs;
            }
        }
    }
    __syncthreads();
    const uint32_t off = s_excl + excl_block;
    if (cnt != 0u && cnt <= static_cast<uint32_t>(kBucket)) {
        const uint32_t qi = atomicAdd(&s_nbig, 1u);
        s_big[qi] = a;
        s_big_off[qi] = off;
        s_big_cnt[qi] = cnt;
    } else if (cnt > static_cast<uint32_t>(kBucket)) {
        Partners P;
        const uint32_t leaf = __ldg(&T.inv_sorted[a]);
        const BoxF q = unpack_box(__ldg(&T.trav[2 * (n - 1 + static_cast<int>(leaf))]));
        int sb, se;
        scene_leaves(T, n, static_cast<int>(leaf), sb, se);
        traverse(T, n, q, a, a, P, sb, se + 1);
        uint32_t written = 0;
        while (true) {
            for (int i = 0; i < P.m; ++i) {
                const uint32_t pos = off + written + static_cast<uint32_t>(i);
                if (pos < max_pairs) pairs[pos] = make_uint2(a, P.v[i]);
            }
            written += static_cast<uint32_t>(P.m);
            if (written >= cnt || P.m == 0) break;
            traverse(T, n, q, a, P.v[P.m - 1], P, sb, se + 1);
        }
    }
    __syncthreads();
    // Warp-ranked buckets: lane l holds elements l, l+32, ...; each element's
    // place is the number of smaller partners (the partners are distinct).
    const uint32_t lane = threadIdx.x & 31u;
    constexpr int kPer = kBucket / 32;
    for (uint32_t q = threadIdx.x >> 5; q < s_nbig; q += kBpThreads / 32) {
        const uint32_t ab = s_big[q], base = s_big_off[q], mb = s_big_cnt[q];
        uint32_t v[kPer], rank[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t i = lane + 32u * j;
            v[j] = i < mb ? T.bucket[static_cast<size_t>(ab) * kBucket + i] : 0xFFFFFFFFu;
            rank[j] = 0u;
        }
#pragma unroll
        for (int jj = 0; jj < kPer; ++jj) {
            for (uint32_t l = 0; l < 32u; ++l) {
                if (32u * jj + l >= mb) break;  // warp-uniform
                const uint32_t w = __shfl_sync(0xffffffffu, v[jj], l);
#pragma unroll
                for (int j = 0; j < kPer; ++j) rank[j] += (w < v[j]) ? 1u : 0u;
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const uint32_t i = lane + 32u * j;
            const uint32_t pos = base + rank[j];
            if (i < mb && pos < max_pairs) pairs[pos] = make_uint2(ab, v[j]);
        }
    }
}

int subtree_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        blocks = sms * 8;
    }
    return blocks;
}

template <typename T>
cudaError_t dev_alloc(T** p, size_t count) {
    return cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
}

}  // namespace

dyph_status broadphase_build(dyph_broadphase* bp, const dyph_bodies* bodies, const dyph_shapes* shapes,
                             const dyph_aabb* bounds, cudaStream_t s) {
    if (!bp || !bodies || !shapes || !bounds) return DYPH_ERR_INVALID;
    const uint32_t n = bodies->n;
    if (n > bp->max_bodies) return DYPH_ERR_INVALID;
    const uint32_t n_tiles = (std::max(n, 1u) + kBpThreads - 1) / kBpThreads;
    GlobalBodies B{*bodies};
    GlobalShapes S{*shapes};
    const uint32_t mblocks = std::max(1u, std::min((n + kBpThreads - 1) / kBpThreads, 2048u));
    morton_kernel<<<mblocks, kBpThreads, 0, s>>>(B, n, *bounds, bp->codes, bp->bvh.sorted_idx, bp->counts,
                                                 bp->tstatus, n_tiles, bp->bvh.bucket_cnt, bp->bvh.codes64,
                                                 bp->bvh.scene_of, bp->scene_bounds);
    DYPH_CUDA_TRY(cudaGetLastError());
    bp->last_n = n;
    if (n < 2) return DYPH_OK;
    dyph_status st = bp->bvh.codes64
                         ? sort_u64_u32(bp->bvh.codes64, bp->bvh.sorted_idx, n, 30 + bp->scene_bits, bp->sort_ws,
                                        bp->sort_ws_bytes, s)
                         : sort_u32_u32(bp->codes, bp->bvh.sorted_idx, n, 30, bp->sort_ws, bp->sort_ws_bytes, s);
    if (st != DYPH_OK) return st;
    if (bp->bvh.codes64) {
        scene_range_kernel<<<(n + kBpThreads - 1) / kBpThreads, kBpThreads, 0, s>>>(
            n, bp->bvh.codes64, bp->bvh.scene_first, bp->bvh.scene_last);
        DYPH_CUDA_TRY(cudaGetLastError());
    }
    const uint32_t leaf_blocks = (n + kBpThreads - 1) / kBpThreads;
    build_kernel<<<leaf_blocks, kBpThreads, 0, s>>>(B, S, n, bp->codes, bp->bvh.sorted_idx, bp->bvh);
    DYPH_CUDA_TRY(cudaGetLastError());
    finalize_nodes_kernel<<<(2 * n - 1 + kBpThreads - 1) / kBpThreads, kBpThreads, 0, s>>>(n, bp->bvh);
    DYPH_CUDA_TRY(cudaGetLastError());
    const uint32_t queue_cap = bp->max_bodies * static_cast<uint32_t>(kQueuePerBody);
    pair_find_kernel<<<leaf_blocks, kBpThreads, 0, s>>>(n, bp->bvh, bp->queue, queue_cap, bp->counts + 3);
    DYPH_CUDA_TRY(cudaGetLastError());
    pair_subtree_kernel<<<subtree_blocks(), kBpThreads, 0, s>>>(n, bp->bvh, bp->queue, queue_cap, bp->counts + 3);
    DYPH_CUDA_TRY(cudaGetLastError());
    pair_write_kernel<<<n_tiles, kBpThreads, 0, s>>>(n, bp->bvh, reinterpret_cast<uint2*>(bp->pairs), bp->max_pairs,
                                                     bp->counts, bp->tstatus);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

dyph_status broadphase_create(uint32_t max_bodies, uint32_t max_pairs, dyph_broadphase** out) {
    if (!out || max_bodies == 0 || max_pairs == 0 || max_bodies >= (1u << 30)) return DYPH_ERR_INVALID;
    auto* bp = new (std::nothrow) dyph_broadphase();
    if (!bp) return DYPH_ERR_NOMEM;
    bp->max_bodies = max_bodies;
    bp->max_pairs = max_pairs;
    const size_t nb = max_bodies, ni = max_bodies > 1 ? max_bodies - 1 : 1, nn = 2 * nb - 1;
    bool ok = dev_alloc(&bp->codes, nb) == cudaSuccess && dev_alloc(&bp->bvh.sorted_idx, nb) == cudaSuccess &&
              dev_alloc(&bp->bvh.sorted_keys, nb) == cudaSuccess &&
              dev_alloc(&bp->bvh.inv_sorted, nb) == cudaSuccess && dev_alloc(&bp->bvh.left, ni) == cudaSuccess &&
              dev_alloc(&bp->bvh.right, ni) == cudaSuccess && dev_alloc(&bp->bvh.parent, nn) == cudaSuccess &&
              dev_alloc(&bp->bvh.root, 1) == cudaSuccess && dev_alloc(&bp->bvh.aabb, nn) == cudaSuccess &&
              dev_alloc(&bp->bvh.range_hi, ni) == cudaSuccess && dev_alloc(&bp->bvh.rsplit, ni) == cudaSuccess &&
              dev_alloc(&bp->bvh.slot, 2 * ni) == cudaSuccess && dev_alloc(&bp->bvh.flags, ni) == cudaSuccess &&
              dev_alloc(&bp->pairs, max_pairs) == cudaSuccess && dev_alloc(&bp->counts, 4) == cudaSuccess &&
              dev_alloc(&bp->tstatus, (nb + kBpThreads - 1) / kBpThreads) == cudaSuccess &&
              dev_alloc(&bp->bvh.range_lo, ni) == cudaSuccess && dev_alloc(&bp->bvh.trav, 2 * nn) == cudaSuccess &&
              dev_alloc(&bp->bvh.bucket_cnt, nb) == cudaSuccess && dev_alloc(&bp->bvh.big, nn) == cudaSuccess &&
              dev_alloc(&bp->bvh.bucket, nb * kBucket) == cudaSuccess &&
              dev_alloc(&bp->queue, nb * kQueuePerBody) == cudaSuccess;
    if (ok) {
        bp->sort_ws_bytes = sort_workspace_bytes(nb, 4);
        ok = cudaMalloc(&bp->sort_ws, bp->sort_ws_bytes) == cudaSuccess;
    }
    // Arrival counters start even; every build adds exactly two per internal node.
    if (ok) ok = cudaMemset(bp->bvh.flags, 0, ni * sizeof(uint32_t)) == cudaSuccess;
    if (ok) ok = cudaMemset(bp->counts, 0, 4 * sizeof(uint32_t)) == cudaSuccess;
    if (ok) ok = sort_prepare() == DYPH_OK;
    if (!ok) {
        broadphase_destroy(bp);
        return DYPH_ERR_NOMEM;
    }
    *out = bp;
    return DYPH_OK;
}

dyph_status broadphase_set_scenes(dyph_broadphase* bp, uint32_t n_scenes, const uint32_t* h_body_offset,
                                  const dyph_aabb* h_scene_bounds) {
    if (!bp || n_scenes == 0 || !h_body_offset || !h_scene_bounds) return DYPH_ERR_INVALID;
    // Keys are (scene << 52 | code << 22 | body): at most 4096 scenes of a
    // tree of at most 2^22 bodies.
    if (n_scenes > 4096u || bp->max_bodies > (1u << 22) || h_body_offset[0] != 0u ||
        h_body_offset[n_scenes] > bp->max_bodies)
        return DYPH_ERR_INVALID;
    for (uint32_t i = 0; i < n_scenes; ++i)
        if (h_body_offset[i + 1] <= h_body_offset[i]) return DYPH_ERR_INVALID;  // every scene has a body
    const uint32_t n = h_body_offset[n_scenes];
    int bits = 0;
    while ((1u << bits) < n_scenes) ++bits;
    bool ok = true;
    if (!bp->bvh.codes64) ok = dev_alloc(&bp->bvh.codes64, bp->max_bodies) == cudaSuccess &&
                                 dev_alloc(&bp->bvh.scene_of, bp->max_bodies) == cudaSuccess;
    if (bp->scene_bounds) cudaFree(bp->scene_bounds);
    if (bp->bvh.scene_first) cudaFree(bp->bvh.scene_first);
    if (bp->bvh.scene_last) cudaFree(bp->bvh.scene_last);
    if (bp->body_offset) cudaFree(bp->body_offset);
    bp->scene_bounds = nullptr;
    bp->bvh.scene_first = bp->bvh.scene_last = bp->body_offset = nullptr;
    ok = ok && dev_alloc(&bp->scene_bounds, n_scenes) == cudaSuccess &&
         dev_alloc(&bp->bvh.scene_first, n_scenes) == cudaSuccess &&
         dev_alloc(&bp->bvh.scene_last, n_scenes) == cudaSuccess &&
         dev_alloc(&bp->body_offset, n_scenes + 1) == cudaSuccess;
    if (!ok) return DYPH_ERR_NOMEM;
    std::vector<uint32_t> scene_of(n);
    for (uint32_t sc = 0; sc < n_scenes; ++sc)
        for (uint32_t i = h_body_offset[sc]; i < h_body_offset[sc + 1]; ++i) scene_of[i] = sc;
    DYPH_CUDA_TRY(cudaMemcpy(bp->bvh.scene_of, scene_of.data(), n * 4, cudaMemcpyHostToDevice));
    DYPH_CUDA_TRY(cudaMemcpy(bp->scene_bounds, h_scene_bounds, n_scenes * sizeof(dyph_aabb), cudaMemcpyHostToDevice));
    DYPH_CUDA_TRY(cudaMemcpy(bp->body_offset, h_body_offset, (n_scenes + 1) * 4, cudaMemcpyHostToDevice));
    const size_t ws = sort_workspace_bytes(bp->max_bodies, 8);
    if (ws > bp->sort_ws_bytes) {
        if (bp->sort_ws) cudaFree(bp->sort_ws);
        bp->sort_ws = nullptr;
        bp->sort_ws_bytes = 0;
        if (cudaMalloc(&bp->sort_ws, ws) != cudaSuccess) return DYPH_ERR_NOMEM;
        bp->sort_ws_bytes = ws;
    }
    bp->n_scenes = n_scenes;
    bp->scene_bits = bits;
    return DYPH_OK;
}

void broadphase_destroy(dyph_broadphase* bp) {
    if (!bp) return;
    void* ptrs[] = {bp->codes, bp->bvh.sorted_idx, bp->bvh.sorted_keys, bp->bvh.inv_sorted, bp->bvh.left,
                    bp->bvh.right, bp->bvh.parent, bp->bvh.root, bp->bvh.aabb, bp->bvh.range_hi, bp->bvh.rsplit,
                    bp->bvh.slot, bp->bvh.flags, bp->pairs, bp->counts, bp->tstatus, bp->sort_ws,
                    bp->bvh.range_lo, bp->bvh.trav, bp->bvh.bucket_cnt, bp->bvh.bucket, bp->bvh.big, bp->queue,
                    bp->bvh.codes64, bp->bvh.scene_of, bp->bvh.scene_first, bp->bvh.scene_last,
                    bp->scene_bounds, bp->body_offset};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete bp;
}

}  // namespace dyph

using namespace dyph;

extern "C" dyph_status dyph_broadphase_create(uint32_t max_bodies, uint32_t max_pairs, dyph_broadphase** out) {
    return broadphase_create(max_bodies, max_pairs, out);
}

extern "C" void dyph_broadphase_destroy(dyph_broadphase* bp) { broadphase_destroy(bp); }

extern "C" dyph_status dyph_broadphase_build_and_query(dyph_broadphase* bp, const dyph_bodies* bodies,
                                                       const dyph_shapes* shapes, const dyph_aabb* bounds,
                                                       dyph_stream s) {
    return broadphase_build(bp, bodies, shapes, bounds, reinterpret_cast<cudaStream_t>(s));
}

extern "C" dyph_status dyph_broadphase_sort_pairs(dyph_broadphase* bp, uint32_t, dyph_stream) {
    return bp ? DYPH_OK : DYPH_ERR_INVALID;  // pairs are emitted in sorted order
}

extern "C" dyph_status dyph_broadphase_download_count(dyph_broadphase* bp, dyph_stream s, uint32_t* out) {
    if (!bp || !out) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaMemcpyAsync(out, bp->counts + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

extern "C" const dyph_pair* dyph_broadphase_pairs(const dyph_broadphase* bp) { return bp ? bp->pairs : nullptr; }
extern "C" const uint32_t* dyph_broadphase_count_ptr(const dyph_broadphase* bp) { return bp ? bp->counts : nullptr; }
extern "C" uint32_t dyph_broadphase_max_pairs(const dyph_broadphase* bp) { return bp ? bp->max_pairs : 0u; }

extern "C" dyph_status dyph_broadphase_bvh_view(const dyph_broadphase* bp, uint32_t n_active, dyph_bvh_view* out) {
    if (!bp || !out) return DYPH_ERR_INVALID;
    out->left = bp->bvh.left;
    out->right = bp->bvh.right;
    out->parent = bp->bvh.parent;
    out->root = bp->bvh.root;
    out->sorted_idx = bp->bvh.sorted_idx;
    out->aabb = reinterpret_cast<const dyph_node_box*>(bp->bvh.aabb);
    out->sorted_keys = bp->bvh.sorted_keys;
    out->n = n_active;
    return DYPH_OK;
}

extern "C" dyph_status dyph_broadphase_set_scenes(dyph_broadphase* bp, uint32_t n_scenes, const uint32_t* body_offset,
                                                  const dyph_aabb* scene_bounds) {
    return dyph::broadphase_set_scenes(bp, n_scenes, body_offset, scene_bounds);
}
