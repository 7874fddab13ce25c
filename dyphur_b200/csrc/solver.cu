// XPBD contact solver: Jones–Plassmann colouring + coloured Gauss–Seidel
// sweeps (one cooperative kernel), and the sequential-order path (one thread
// block running a level schedule that reproduces the serial order bit for bit).
//
// Replaces XpbdSolver::solve (core/src/xpbd_solver.cpp:603-733) for contacts.
// Facts the schedule relies on:
//   * solve_contact (:413-521) writes only its two bodies and never a body with
//     inv_mass == 0, so two contacts sharing no dynamic body commute exactly;
//   * lambda starts at 0 and a solved contact stores lambda = depth, so every
//     later iteration returns at `remaining <= 1e-6` — only a contact that
//     returned at `w_total < 1e-10` can act again, and that case is tracked;
//   * every iteration ends with a renormalisation of every body, so the
//     quaternion update q * rsqrt(|q|^2) is applied n_iters times per frame;
//   * with no contacts at all nothing (not even the renormalisation) runs.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "internal.cuh"
#include "solver_common.cuh"

#include "solver_color.cuh"
#include "solver_flow.cuh"
#include "solver_scene.cuh"

namespace dyph {
namespace {

// ── sequential path (one block) ─────────────────────────────────────────────
// Predecessors: contacts are sorted by (a, b), so the contacts touching body x
// are its b-side contacts (a < x, scattered) followed by its a-side run
// (a == x, contiguous). pred_a(c) is c-1 inside an a-run, else the last b-side
// contact of a; pred_b(c) is the previous b-side contact of b.
__global__ void __launch_bounds__(kSeqThreads) sequential_solve_kernel(
    dyph_contacts cv, GlobalBodies B, int mode, int n_iters, float mu, float dt, float* __restrict__ lambda,
    uint32_t* __restrict__ pred, uint32_t* __restrict__ entries, uint32_t* __restrict__ done,
    uint32_t* __restrict__ bcnt, uint32_t* __restrict__ boff, uint32_t* __restrict__ meta) {
    __shared__ uint32_t s_scan[kSeqThreads / 32];
    __shared__ uint32_t s_carry;
    __shared__ int s_deferred;
    const uint32_t nc = contact_count(cv);
    if (nc == 0) return;
    // Small sequential-order frames, or a fallback the other kernels handed on.
    if (!(wants_sequential(mode, nc) && nc <= kSeqOneBlock) && ld_acquire(&meta[kMetaDecision]) != 1u) return;
    const uint32_t nb = B.v.n;
    const uint32_t t = threadIdx.x;
    uint32_t* pred_a = pred;
    uint32_t* pred_b = pred + cv.capacity;
    // 1. b-side CSR: counts
    for (uint32_t i = t; i < nb; i += kSeqThreads) bcnt[i] = 0u;
    if (t == 0) s_deferred = 0;
    __syncthreads();
    for (uint32_t c = t; c < nc; c += kSeqThreads) {
        const uint32_t b = cv.body_b[c];
        if (B.im(b) != 0.f) atomicAdd(&bcnt[b], 1u);
    }
    __syncthreads();
    // 2. exclusive scan of counts -> boff
    if (t == 0) s_carry = 0u;
    __syncthreads();
    for (uint32_t base = 0; base < nb; base += kSeqThreads) {
        const uint32_t i = base + t;
        const uint32_t v = i < nb ? bcnt[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<kSeqThreads>(v, s_scan, tot);
        if (i < nb) {
            boff[i] = s_carry + ex;
            bcnt[i] = 0u;  // reused as the fill cursor
        }
        __syncthreads();
        if (t == 0) s_carry += tot;
        __syncthreads();
    }
    if (t == 0) boff[nb] = s_carry;
    __syncthreads();
    // 3. fill (unordered), 4. sort each body's list and link predecessors
    for (uint32_t c = t; c < nc; c += kSeqThreads) {
        const uint32_t b = cv.body_b[c];
        if (B.im(b) != 0.f) entries[boff[b] + atomicAdd(&bcnt[b], 1u)] = c;
        pred_b[c] = kNone;
    }
    __syncthreads();
    for (uint32_t x = t; x < nb; x += kSeqThreads) {
        const uint32_t lo = boff[x], hi = boff[x + 1];
        for (uint32_t i = lo + 1; i < hi; ++i) {
            uint32_t v = entries[i], j = i;
            while (j > lo && entries[j - 1] > v) {
                entries[j] = entries[j - 1];
                --j;
            }
            entries[j] = v;
        }
        for (uint32_t i = lo + 1; i < hi; ++i) pred_b[entries[i]] = entries[i - 1];
        bcnt[x] = (hi > lo) ? entries[hi - 1] : kNone;  // last b-side contact of x
    }
    __syncthreads();
    for (uint32_t c = t; c < nc; c += kSeqThreads) {
        const uint32_t a = cv.body_a[c];
        uint32_t p = kNone;
        if (B.im(a) != 0.f) p = (c > 0 && cv.body_a[c - 1] == a) ? c - 1 : bcnt[a];
        pred_a[c] = p;
    }
    __syncthreads();
    // 5. level-scheduled sweeps; done[c] = wave (>= 1) in which c was solved.
    bool deferred = false;
    for (int iter = 0; iter < n_iters; ++iter) {
        if (iter == 0 || deferred) {
            for (uint32_t c = t; c < nc; c += kSeqThreads) {
                done[c] = 0u;
                if (iter == 0) lambda[c] = 0.f;
            }
            __syncthreads();
            const uint32_t mine = (nc > t) ? (nc - t + kSeqThreads - 1) / kSeqThreads : 0u;
            uint32_t cursor = 0;
            uint32_t wave = 1;
            while (true) {
                int left = cursor < mine;
                if (!__syncthreads_or(left)) break;
                for (uint32_t j = cursor; j < mine && j < cursor + kSeqWindow; ++j) {
                    const uint32_t c = t + j * kSeqThreads;
                    if (done[c] != 0u) continue;
                    const uint32_t pa = pred_a[c], pb = pred_b[c];
                    const uint32_t da = (pa == kNone) ? 1u : done[pa];
                    const uint32_t db = (pb == kNone) ? 1u : done[pb];
                    const bool ready = (pa == kNone || (da != 0u && da < wave)) && (pb == kNone || (db != 0u && db < wave));
                    if (!ready) continue;
                    const Contact ct = load_contact(cv, c);
                    float lc = lambda[c];
                    if (solve_contact(B, ct, mu, lc, dt) == kSolveDeferred) s_deferred = 1;
                    lambda[c] = lc;
                    done[c] = wave;
                }
                while (cursor < mine && done[t + cursor * kSeqThreads] != 0u) ++cursor;
                __syncthreads();
                ++wave;
                // The smallest unsolved contact is always ready, so a correct
                // schedule needs at most nc waves.
                if (wave > nc + 2u) {
                    raise_error(DYPH_ERR_TIMEOUT, 5u);
                    return;
                }
            }
            __syncthreads();
            deferred = s_deferred != 0;
        }
        if (!deferred) {
            for (uint32_t i = t; i < nb; i += kSeqThreads) renorm_body(B, i, n_iters - iter);
            break;
        }
        for (uint32_t i = t; i < nb; i += kSeqThreads) renorm_body(B, i, 1);
        __syncthreads();
    }
}

int coop_block_count() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 148, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, color_solve_kernel, kColorThreads, 0);
        blocks = sms * std::max(1, std::min(per_sm, 1));
    }
    return blocks;
}

// Co-resident blocks of the dataflow kernel: as many as fit, at most 4 per SM
// (more threads -> fewer contacts per thread; more blocks -> dearer barriers).
int flow_block_count() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 148, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, flow_solve_kernel, kFlowThreads, 0);
        blocks = std::min(sms * std::max(1, std::min(per_sm, 4)), kFlowMaxBlocks);
    }
    return blocks;
}

}  // namespace

dyph_status xpbd_create(int32_t n_iters, uint32_t max_contacts, uint32_t max_bodies, float friction,
                        dyph_xpbd** out) {
    // Contact indices must fit the 24-bit field of the colouring priorities.
    if (!out || n_iters < 0 || max_contacts == 0 || max_contacts >= (1u << 24) || max_bodies == 0)
        return DYPH_ERR_INVALID;
    auto* sv = new (std::nothrow) dyph_xpbd();
    if (!sv) return DYPH_ERR_NOMEM;
    sv->n_iters = n_iters;
    sv->friction = friction;
    sv->max_contacts = max_contacts;
    sv->max_bodies = max_bodies;
    const size_t mc = max_contacts, mb = max_bodies;
    bool ok = cudaMalloc(&sv->lambda, mc * 4) == cudaSuccess && cudaMalloc(&sv->color, mc * 4) == cudaSuccess &&
              cudaMalloc(&sv->order, mc * 4) == cudaSuccess && cudaMalloc(&sv->pred, 2 * mc * 4) == cudaSuccess &&
              cudaMalloc(&sv->done, mc * 4) == cudaSuccess && cudaMalloc(&sv->bpri, 3 * mb * 8) == cudaSuccess &&
              cudaMalloc(&sv->bmask, mb * 8) == cudaSuccess && cudaMalloc(&sv->blast, 2 * (mb + 1) * 4) == cudaSuccess &&
              cudaMalloc(&sv->meta, kMetaWords * 4) == cudaSuccess &&
              cudaMalloc(&sv->body_list, mb * kBodySlots * 8) == cudaSuccess &&
              cudaMalloc(&sv->slot, 2 * mc * 4) == cudaSuccess &&
              cudaMalloc(&sv->link, 2 * mc * 4) == cudaSuccess && cudaMalloc(&sv->cmask, 2 * mc * 8) == cudaSuccess &&
              cudaMalloc(&sv->hand, 2 * mc * kHandWords * 8) == cudaSuccess &&
              cudaMemset(sv->hand, 0, 2 * mc * kHandWords * 8) == cudaSuccess &&
              cudaMalloc(&sv->tail, mb * 4) == cudaSuccess && cudaMalloc(&sv->sweep_tag, 4) == cudaSuccess &&
              cudaMalloc(&sv->csr_off, (mb + 1) * 4) == cudaSuccess && cudaMalloc(&sv->csr_cur, mb * 4) == cudaSuccess &&
              cudaMalloc(&sv->csr, 2 * mc * 4) == cudaSuccess &&
              cudaMalloc(&sv->partial, kFlowMaxBlocks * 4) == cudaSuccess &&
              cudaMemset(sv->sweep_tag, 0, 4) == cudaSuccess;
    if (!ok) {
        xpbd_destroy(sv);
        return DYPH_ERR_NOMEM;
    }
    sv->coop_blocks = coop_block_count();
    sv->flow_blocks = flow_block_count();
    *out = sv;
    return DYPH_OK;
}

void xpbd_destroy(dyph_xpbd* sv) {
    if (!sv) return;
    void* ptrs[] = {sv->lambda, sv->color, sv->order, sv->pred, sv->done, sv->bpri, sv->bmask, sv->blast, sv->meta,
                    sv->body_list, sv->slot, sv->link, sv->cmask, sv->hand, sv->tail, sv->sweep_tag,
                    sv->csr_off, sv->csr_cur, sv->csr, sv->partial, sv->scene_range, sv->scene_order,
                    sv->scene_scratch};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    delete sv;
}

dyph_status xpbd_set_scenes(dyph_xpbd* sv, uint32_t n_scenes, const uint32_t* h_body_offset,
                            const uint32_t* d_body_offset, const uint32_t* d_scene_of) {
    if (!sv || !h_body_offset || !d_body_offset || !d_scene_of || n_scenes == 0) return DYPH_ERR_INVALID;
    sv->scene_n = 0;
    // Largest scenes first: blocks are dispatched in index order, so the long
    // scenes start early and the short ones fill in behind them.
    std::vector<uint32_t> order(n_scenes);
    uint32_t max_nb = 0;
    for (uint32_t i = 0; i < n_scenes; ++i) {
        order[i] = i;
        max_nb = std::max(max_nb, h_body_offset[i + 1] - h_body_offset[i]);
    }
    std::stable_sort(order.begin(), order.end(), [h_body_offset](uint32_t x, uint32_t y) {
        return h_body_offset[x + 1] - h_body_offset[x] > h_body_offset[y + 1] - h_body_offset[y];
    });
    constexpr uint32_t kMaxSmem = 200u * 1024u;
    const uint32_t body_bytes = scene_body_bytes(max_nb);
    if (max_nb > kSceneMaxBodies || body_bytes + kSceneWords * 4u * 64u > kMaxSmem) return DYPH_ERR_TOO_LARGE;
    // Room for about three contacts per body of the largest scene next to its
    // bodies; a scene with more keeps its contact words in the global scratch.
    const uint32_t smem = std::min(kMaxSmem, body_bytes + kSceneWords * 4u * std::max(256u, 3u * max_nb));
    // The attribute is per device and per function, shared by every solver:
    // set it on the current device every time, to the most any solver takes,
    // so that no solver lowers it under another's launches.
    DYPH_CUDA_TRY(cudaFuncSetAttribute(scene_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(kMaxSmem)));
    if (sv->scene_range) cudaFree(sv->scene_range);
    if (sv->scene_order) cudaFree(sv->scene_order);
    sv->scene_range = sv->scene_order = nullptr;
    if (cudaMalloc(&sv->scene_range, 2ull * n_scenes * 4) != cudaSuccess ||
        cudaMalloc(&sv->scene_order, static_cast<size_t>(n_scenes) * 4) != cudaSuccess)
        return DYPH_ERR_NOMEM;
    DYPH_CUDA_TRY(cudaMemcpy(sv->scene_order, order.data(), static_cast<size_t>(n_scenes) * 4, cudaMemcpyHostToDevice));
    if (sv->scene_scratch) cudaFree(sv->scene_scratch);
    sv->scene_scratch = nullptr;
    sv->scene_stride = sv->max_contacts + n_scenes;
    if (cudaMalloc(&sv->scene_scratch, static_cast<size_t>(kSceneWords) * sv->scene_stride * 4) != cudaSuccess)
        return DYPH_ERR_NOMEM;
    sv->scene_offset = d_body_offset;
    sv->scene_of = d_scene_of;
    sv->scene_smem = smem;
    sv->scene_n = n_scenes;
    // The whole-batch kernels' buffers are not used again (a world never
    // leaves the batched form): give them back.
    void** unused[] = {reinterpret_cast<void**>(&sv->order), reinterpret_cast<void**>(&sv->pred),
                       reinterpret_cast<void**>(&sv->done), reinterpret_cast<void**>(&sv->bpri),
                       reinterpret_cast<void**>(&sv->bmask), reinterpret_cast<void**>(&sv->blast),
                       reinterpret_cast<void**>(&sv->body_list), reinterpret_cast<void**>(&sv->slot),
                       reinterpret_cast<void**>(&sv->link), reinterpret_cast<void**>(&sv->cmask),
                       reinterpret_cast<void**>(&sv->hand), reinterpret_cast<void**>(&sv->tail),
                       reinterpret_cast<void**>(&sv->csr_off), reinterpret_cast<void**>(&sv->csr_cur),
                       reinterpret_cast<void**>(&sv->csr), reinterpret_cast<void**>(&sv->partial)};
    DYPH_CUDA_TRY(cudaDeviceSynchronize());
    for (void** p : unused) {
        if (*p) cudaFree(*p);
        *p = nullptr;
    }
    return DYPH_OK;
}

dyph_status xpbd_solve(dyph_xpbd* sv, const dyph_contacts* contacts, const dyph_bodies* bodies, float dt,
                       cudaStream_t s) {
    if (!sv || !contacts || !bodies) return DYPH_ERR_INVALID;
    if (bodies->n > sv->max_bodies || contacts->capacity > sv->max_contacts) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaMemsetAsync(sv->meta, 0, kMetaWords * 4, s));
    dyph_contacts cv = *contacts;
    GlobalBodies B{*bodies};
    int mode = static_cast<int>(sv->mode);
    int n_iters = sv->n_iters;
    float mu = sv->friction;
    if (sv->scene_n > 0) {
        // Batched scenes: one block per scene.
        SceneBufs S{sv->scene_offset, sv->scene_of, sv->scene_order, sv->scene_range, sv->scene_scratch,
                    sv->scene_stride, sv->scene_n, sv->scene_smem};
        DYPH_CUDA_TRY(cudaMemsetAsync(sv->scene_range, 0, 2ull * sv->scene_n * 4, s));
        scene_range_kernel<<<std::max(1u, std::min((cv.capacity + 255u) / 256u, 4096u)), 256, 0, s>>>(cv, S);
        if (sv->probe_flow[0])
            DYPH_CUDA_TRY(cudaEventRecordWithFlags(static_cast<cudaEvent_t>(sv->probe_flow[0]), s,
                                                   cudaEventRecordExternal));
        scene_solve_kernel<<<sv->scene_n, kSceneThreads, sv->scene_smem, s>>>(cv, *bodies, S, mode, n_iters, mu, dt,
                                                                              sv->color, sv->meta);
        if (sv->probe_flow[1])
            DYPH_CUDA_TRY(cudaEventRecordWithFlags(static_cast<cudaEvent_t>(sv->probe_flow[1]), s,
                                                   cudaEventRecordExternal));
        DYPH_CUDA_TRY(cudaGetLastError());
        return DYPH_OK;
    }
    // Per-body contact counts live in `blast`, JP rounds in `order`: the
    // kernels that also use them run only after this one declined the frame.
    FlowBufs F{sv->blast, reinterpret_cast<unsigned long long*>(sv->body_list), sv->slot, sv->link,
               reinterpret_cast<unsigned long long*>(sv->cmask), sv->order,
               reinterpret_cast<unsigned long long*>(sv->hand), 2u * sv->max_contacts, sv->tail, sv->sweep_tag,
               sv->csr_off, sv->csr_cur, sv->csr, sv->partial};
    void* fargs[] = {&cv, &B, &mode, &n_iters, &mu, &dt, &sv->lambda, &sv->color, &F, &sv->meta};
    if (sv->probe_flow[0])
        DYPH_CUDA_TRY(cudaEventRecordWithFlags(static_cast<cudaEvent_t>(sv->probe_flow[0]), s, cudaEventRecordExternal));
    DYPH_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(flow_solve_kernel), dim3(sv->flow_blocks),
                                              dim3(kFlowThreads), fargs, 0, s));
    if (sv->probe_flow[1])
        DYPH_CUDA_TRY(cudaEventRecordWithFlags(static_cast<cudaEvent_t>(sv->probe_flow[1]), s, cudaEventRecordExternal));
    void* args[] = {&cv, &B, &mode, &n_iters, &mu, &dt, &sv->lambda, &sv->color, &sv->order, &sv->pred,
                    &sv->bpri, &sv->bmask, &sv->meta};
    DYPH_CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(color_solve_kernel), dim3(sv->coop_blocks),
                                              dim3(kColorThreads), args, 0, s));
    // b-side list entries reuse `order`; per-body counts and offsets live in `blast`.
    sequential_solve_kernel<<<1, kSeqThreads, 0, s>>>(cv, B, mode, n_iters, mu, dt, sv->lambda, sv->pred,
                                                      sv->order, sv->done, sv->blast,
                                                      sv->blast + sv->max_bodies + 1, sv->meta);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

}  // namespace dyph

using namespace dyph;

extern "C" dyph_status dyph_xpbd_create(int32_t n_iters, uint32_t max_contacts, uint32_t max_bodies, float friction,
                                        dyph_xpbd** out) {
    return xpbd_create(n_iters, max_contacts, max_bodies, friction, out);
}
extern "C" void dyph_xpbd_destroy(dyph_xpbd* sv) { xpbd_destroy(sv); }
extern "C" dyph_status dyph_xpbd_set_mode(dyph_xpbd* sv, dyph_solver_mode mode) {
    if (!sv || (mode != DYPH_SOLVER_REFERENCE && mode != DYPH_SOLVER_SEQUENTIAL && mode != DYPH_SOLVER_COLORED &&
                mode != DYPH_SOLVER_REFERENCE_ROUNDS))
        return DYPH_ERR_INVALID;
    sv->mode = mode;
    return DYPH_OK;
}
extern "C" dyph_status dyph_xpbd_solve(dyph_xpbd* sv, const dyph_contacts* contacts, const dyph_bodies* bodies,
                                       float dt, dyph_stream s) {
    return xpbd_solve(sv, contacts, bodies, dt, reinterpret_cast<cudaStream_t>(s));
}
