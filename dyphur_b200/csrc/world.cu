// The whole frame step behind one handle, replayed as a CUDA graph.
//
// One frame is the reference's loop body (examples/stress_test_blocks/
// main.cpp:264-279): integrate, build_and_query, sort_pairs (already sorted),
// Narrowphase::run, XpbdSolver::solve. Every count stays on the device, so a
// frame has no host round trip; the first step captures one frame into a CUDA
// graph and every later frame replays it. A one-thread kernel at the end of
// the frame folds the pair / contact counts into peak and overflow words.
#include <cuda_runtime.h>

#include <new>

#include "internal.cuh"

struct dyph_world {
    dyph_world_desc desc{};
    dyph_broadphase* bp = nullptr;
    dyph_narrowphase* np = nullptr;
    dyph_xpbd* sv = nullptr;
    uint32_t* stats = nullptr;  // [0] last pairs, [1] last contacts, [2] peak pairs, [3] peak contacts, [4] status
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph = nullptr;
};

namespace dyph {
namespace {

__global__ void frame_stats_kernel(const uint32_t* __restrict__ bp_counts, const uint32_t* __restrict__ np_counts,
                                   uint32_t max_pairs, uint32_t max_contacts, uint32_t* __restrict__ stats) {
    const uint32_t p = bp_counts[1], c = np_counts[1];
    stats[0] = p;
    stats[1] = c;
    stats[2] = max(stats[2], p);
    stats[3] = max(stats[3], c);
    if (p > max_pairs) atomicCAS(&stats[4], 0u, static_cast<uint32_t>(DYPH_ERR_PAIR_OVERFLOW));
    if (c > max_contacts) atomicCAS(&stats[4], 0u, static_cast<uint32_t>(DYPH_ERR_CONTACT_OVERFLOW));
}

dyph_status enqueue_frame(dyph_world* w, cudaStream_t s) {
    const dyph_world_desc& d = w->desc;
    dyph_status st = integrate_launch(&d.bodies, &d.integrator, s);
    if (st != DYPH_OK) return st;
    st = broadphase_build(w->bp, &d.bodies, &d.shapes, &d.scene_bounds, s);
    if (st != DYPH_OK) return st;
    st = narrowphase_run(w->np, w->bp->pairs, w->bp->counts, w->bp->max_pairs, &d.bodies, &d.shapes, s);
    if (st != DYPH_OK) return st;
    st = xpbd_solve(w->sv, &w->np->view, &d.bodies, d.integrator.dt, s);
    if (st != DYPH_OK) return st;
    frame_stats_kernel<<<1, 1, 0, s>>>(w->bp->counts, w->np->counts, w->bp->max_pairs, w->np->max_contacts,
                                       w->stats);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

}  // namespace
}  // namespace dyph

using namespace dyph;

extern "C" void dyph_world_destroy(dyph_world* w) {
    if (!w) return;
    if (w->graph) cudaGraphExecDestroy(w->graph);
    if (w->ev_in) cudaEventDestroy(w->ev_in);
    if (w->ev_out) cudaEventDestroy(w->ev_out);
    if (w->stream) cudaStreamDestroy(w->stream);
    if (w->stats) cudaFree(w->stats);
    broadphase_destroy(w->bp);
    narrowphase_destroy(w->np);
    xpbd_destroy(w->sv);
    delete w;
}

extern "C" dyph_status dyph_world_create(const dyph_world_desc* desc, dyph_stream, dyph_world** out) {
    if (!desc || !out || desc->bodies.n == 0 || desc->integrator.n_substeps <= 0) return DYPH_ERR_INVALID;
    dyph_status dc = dyph_device_check();
    if (dc != DYPH_OK) return dc;
    auto* w = new (std::nothrow) dyph_world();
    if (!w) return DYPH_ERR_NOMEM;
    w->desc = *desc;
    dyph_status st = broadphase_create(desc->bodies.n, desc->max_pairs, &w->bp);
    if (st == DYPH_OK) st = narrowphase_create(desc->max_contacts, &w->np);
    if (st == DYPH_OK) st = narrowphase_reserve(w->np, desc->max_pairs);
    if (st == DYPH_OK) st = xpbd_create(desc->n_iters, desc->max_contacts, desc->bodies.n, desc->friction, &w->sv);
    if (st == DYPH_OK) {
        w->sv->mode = desc->mode;
        if (cudaMalloc(&w->stats, 8 * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemset(w->stats, 0, 8 * sizeof(uint32_t)) != cudaSuccess ||
            cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&w->ev_in, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&w->ev_out, cudaEventDisableTiming) != cudaSuccess)
            st = DYPH_ERR_CUDA;
    }
    if (st != DYPH_OK) {
        dyph_world_destroy(w);
        return st;
    }
    *out = w;
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_step(dyph_world* w, int32_t n_frames, dyph_stream s) {
    if (!w || n_frames < 0) return DYPH_ERR_INVALID;
    if (n_frames == 0) return DYPH_OK;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_in, cs));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(w->stream, w->ev_in, 0));
    if (!w->graph) {
        cudaGraph_t g = nullptr;
        DYPH_CUDA_TRY(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
        dyph_status st = enqueue_frame(w, w->stream);
        cudaError_t ce = cudaStreamEndCapture(w->stream, &g);
        if (st != DYPH_OK) {
            if (g) cudaGraphDestroy(g);
            return st;
        }
        if (ce != cudaSuccess) return DYPH_ERR_CUDA;
        ce = cudaGraphInstantiate(&w->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) {
            w->graph = nullptr;
            return DYPH_ERR_CUDA;
        }
    }
    for (int32_t f = 0; f < n_frames; ++f) DYPH_CUDA_TRY(cudaGraphLaunch(w->graph, w->stream));
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_out, w->stream));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->ev_out, 0));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_download_stats(dyph_world* w, dyph_stream s, uint32_t* last_pairs,
                                                 uint32_t* last_contacts, uint32_t* peak_pairs,
                                                 uint32_t* peak_contacts, uint32_t* status) {
    if (!w) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t h[5] = {0, 0, 0, 0, 0};
    DYPH_CUDA_TRY(cudaMemcpyAsync(h, w->stats, sizeof(h), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    if (last_pairs) *last_pairs = h[0];
    if (last_contacts) *last_contacts = h[1];
    if (peak_pairs) *peak_pairs = h[2];
    if (peak_contacts) *peak_contacts = h[3];
    if (status) *status = h[4];
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_broadphase(dyph_world* w, dyph_broadphase** out) {
    if (!w || !out) return DYPH_ERR_INVALID;
    *out = w->bp;
    return DYPH_OK;
}
extern "C" dyph_status dyph_world_narrowphase(dyph_world* w, dyph_narrowphase** out) {
    if (!w || !out) return DYPH_ERR_INVALID;
    *out = w->np;
    return DYPH_OK;
}
extern "C" dyph_status dyph_world_solver(dyph_world* w, dyph_xpbd** out) {
    if (!w || !out) return DYPH_ERR_INVALID;
    *out = w->sv;
    return DYPH_OK;
}
