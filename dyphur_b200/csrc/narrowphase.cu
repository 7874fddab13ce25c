// Narrowphase: one thread per candidate pair, contacts compacted in pair order.
//
// Replaces Narrowphase::run (core/src/narrowphase.cpp:1077-1144). For box and
// sphere shapes every pair yields 0 or 1 contact, so the reference's
// append -> (pair_idx << 32 | sub) key sort -> gather is an order-preserving
// stream compaction: each 256-pair tile counts its contacts, finds its output
// offset by decoupled look-back, and writes the ContactView rows directly.
// The pair count is read from device memory, so no host sync is needed.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>

#include "internal.cuh"

namespace dyph {
namespace {

constexpr int kNpThreads = 256;

__global__ void __launch_bounds__(kNpThreads) narrowphase_kernel(const uint2* __restrict__ pairs,
                                                                 const uint32_t* __restrict__ d_n_pairs,
                                                                 uint32_t pair_cap, GlobalBodies B, GlobalShapes S,
                                                                 dyph_contacts out, uint32_t* __restrict__ counts,
                                                                 uint32_t* __restrict__ status) {
    __shared__ uint32_t s_tile, s_excl;
    __shared__ uint32_t s_scan[kNpThreads / 32];
    const uint32_t np_ = min(*d_n_pairs, pair_cap);
    const uint32_t n_tiles = (np_ + kNpThreads - 1) / kNpThreads;
    if (np_ == 0) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            counts[0] = 0u;
            counts[1] = 0u;
        }
        return;
    }
    while (true) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&counts[2], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= n_tiles) break;
        const uint32_t i = tile * kNpThreads + threadIdx.x;
        Contact c;
        bool has = false;
        if (i < np_) {
            const uint2 p = __ldg(&pairs[i]);
            if (p.x < B.v.n && p.y < B.v.n) has = process_pair(B, S, p.x, p.y, c);
            else raise_error(DYPH_ERR_INVALID, 8u);
        }
        uint32_t total;
        const uint32_t excl = block_exclusive_scan<kNpThreads>(has ? 1u : 0u, s_scan, total);
        if (threadIdx.x < 32) {
            const uint32_t e = lookback_warp(status, tile, total);
            if (threadIdx.x == 0) {
                s_excl = e;
                if (tile == n_tiles - 1) {
                    const uint32_t all = e + total;
                    counts[1] = all;
                    counts[0] = all < out.capacity ? all : out.capacity;
                }
            }
        }
        __syncthreads();
        if (has) {
            const uint32_t pos = s_excl + excl;
            if (pos < out.capacity) {
                out.body_a[pos] = c.a;
                out.body_b[pos] = c.b;
                out.pos_x[pos] = c.px;
                out.pos_y[pos] = c.py;
                out.pos_z[pos] = c.pz;
                out.norm_x[pos] = c.nx;
                out.norm_y[pos] = c.ny;
                out.norm_z[pos] = c.nz;
                out.depth[pos] = c.depth;
            }
        }
        __syncthreads();
    }
}

int persistent_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 148, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, narrowphase_kernel, kNpThreads, 0);
        blocks = sms * std::max(1, std::min(per_sm, 8));
    }
    return blocks;
}

}  // namespace

dyph_status narrowphase_create(uint32_t max_contacts, dyph_narrowphase** out) {
    if (!out || max_contacts == 0) return DYPH_ERR_INVALID;
    auto* np = new (std::nothrow) dyph_narrowphase();
    if (!np) return DYPH_ERR_NOMEM;
    np->max_contacts = max_contacts;
    void** bufs[] = {reinterpret_cast<void**>(&np->view.body_a), reinterpret_cast<void**>(&np->view.body_b),
                     reinterpret_cast<void**>(&np->view.pos_x),  reinterpret_cast<void**>(&np->view.pos_y),
                     reinterpret_cast<void**>(&np->view.pos_z),  reinterpret_cast<void**>(&np->view.norm_x),
                     reinterpret_cast<void**>(&np->view.norm_y), reinterpret_cast<void**>(&np->view.norm_z),
                     reinterpret_cast<void**>(&np->view.depth)};
    bool ok = true;
    for (void** b : bufs) ok = ok && cudaMalloc(b, static_cast<size_t>(max_contacts) * 4) == cudaSuccess;
    if (ok) ok = cudaMalloc(&np->counts, 4 * sizeof(uint32_t)) == cudaSuccess;
    if (ok) ok = cudaMemset(np->counts, 0, 4 * sizeof(uint32_t)) == cudaSuccess;
    if (!ok) {
        narrowphase_destroy(np);
        return DYPH_ERR_NOMEM;
    }
    np->view.n = np->counts;
    np->view.capacity = max_contacts;
    persistent_blocks();
    *out = np;
    return DYPH_OK;
}

void narrowphase_destroy(dyph_narrowphase* np) {
    if (!np) return;
    void* ptrs[] = {np->view.body_a, np->view.body_b, np->view.pos_x, np->view.pos_y, np->view.pos_z,
                    np->view.norm_x, np->view.norm_y, np->view.norm_z, np->view.depth, np->counts, np->status};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete np;
}

dyph_status narrowphase_reserve(dyph_narrowphase* np, uint32_t max_pairs) {
    const uint32_t tiles = (max_pairs + kNpThreads - 1) / kNpThreads;
    if (tiles <= np->status_words) return DYPH_OK;
    if (np->status) cudaFree(np->status);
    np->status = nullptr;
    np->status_words = 0;
    if (cudaMalloc(&np->status, std::max<size_t>(tiles, 1) * 4) != cudaSuccess) return DYPH_ERR_NOMEM;
    np->status_words = tiles;
    return DYPH_OK;
}

dyph_status narrowphase_run(dyph_narrowphase* np, const dyph_pair* pairs, const uint32_t* d_n_pairs,
                            uint32_t max_pairs, const dyph_bodies* bodies, const dyph_shapes* shapes,
                            cudaStream_t s) {
    if (!np || !pairs || !d_n_pairs || !bodies || !shapes) return DYPH_ERR_INVALID;
    const uint32_t tiles = (max_pairs + kNpThreads - 1) / kNpThreads;
    dyph_status rs = narrowphase_reserve(np, max_pairs);
    if (rs != DYPH_OK) return rs;
    DYPH_CUDA_TRY(cudaMemsetAsync(np->status, 0, std::max<size_t>(tiles, 1) * 4, s));
    DYPH_CUDA_TRY(cudaMemsetAsync(np->counts + 2, 0, sizeof(uint32_t), s));
    narrowphase_kernel<<<persistent_blocks(), kNpThreads, 0, s>>>(
        reinterpret_cast<const uint2*>(pairs), d_n_pairs, max_pairs, GlobalBodies{*bodies}, GlobalShapes{*shapes},
        np->view, np->counts, np->status);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

}  // namespace dyph

using namespace dyph;

extern "C" dyph_status dyph_narrowphase_create(uint32_t max_contacts, dyph_narrowphase** out) {
    return narrowphase_create(max_contacts, out);
}
extern "C" void dyph_narrowphase_destroy(dyph_narrowphase* np) { narrowphase_destroy(np); }

extern "C" dyph_status dyph_narrowphase_run(dyph_narrowphase* np, const dyph_pair* pairs, const uint32_t* d_n_pairs,
                                            const dyph_bodies* bodies, const dyph_shapes* shapes, dyph_stream s) {
    // Without a capacity the pair count itself is trusted; size the tile
    // status for the largest count the caller can have produced.
    if (!np) return DYPH_ERR_INVALID;
    uint32_t cap = std::max<uint32_t>(np->status_words * kNpThreads, 16u * np->max_contacts);
    return narrowphase_run(np, pairs, d_n_pairs, cap, bodies, shapes, reinterpret_cast<cudaStream_t>(s));
}

extern "C" dyph_status dyph_narrowphase_run_host_count(dyph_narrowphase* np, const dyph_pair* pairs,
                                                       uint32_t n_pairs, const dyph_bodies* bodies,
                                                       const dyph_shapes* shapes, dyph_stream s) {
    if (!np) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    // The count travels through the handle's spare counter word.
    DYPH_CUDA_TRY(cudaMemcpyAsync(np->counts + 3, &n_pairs, sizeof(uint32_t), cudaMemcpyHostToDevice, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return narrowphase_run(np, pairs, np->counts + 3, std::max(n_pairs, 1u), bodies, shapes, cs);
}

extern "C" dyph_status dyph_narrowphase_contacts(dyph_narrowphase* np, dyph_contacts* out) {
    if (!np || !out) return DYPH_ERR_INVALID;
    *out = np->view;
    return DYPH_OK;
}

extern "C" dyph_status dyph_narrowphase_download_count(dyph_narrowphase* np, dyph_stream s, uint32_t* stored,
                                                       uint32_t* true_count) {
    if (!np) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t h[2] = {0, 0};
    DYPH_CUDA_TRY(cudaMemcpyAsync(h, np->counts, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    if (stored) *stored = h[0];
    if (true_count) *true_count = h[1];
    return DYPH_OK;
}
