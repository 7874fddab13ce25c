// The whole frame step behind one handle, replayed as a CUDA graph.
//
// One frame is the reference's loop body (examples/stress_test_blocks/
// main.cpp:264-279): integrate, build_and_query, sort_pairs (already sorted),
// Narrowphase::run, XpbdSolver::solve. Every count stays on the device, so a
// frame has no host round trip; the first step captures one frame into a CUDA
// graph and every later frame replays it. A one-thread kernel at the end of
// the frame folds the pair / contact counts into peak and overflow words.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "internal.cuh"
#include "scene_frame.cuh"
#include "scene_adjoint.cuh"

struct dyph_world {
    dyph_world_desc desc{};
    dyph_broadphase* bp = nullptr;
    dyph_narrowphase* np = nullptr;
    dyph_xpbd* sv = nullptr;
    uint32_t* stats = nullptr;  // [0] last pairs, [1] last contacts, [2] peak pairs, [3] peak contacts, [4] status
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaGraphExec_t episode = nullptr;  // n_frames frames in one graph (dyph_world_capture_episode)
    int32_t episode_frames = 0;
    uint64_t* scene_hash = nullptr;  // [n_scenes] per-scene FNV-1a results
    // Trajectory recording (dyph_world_set_trajectory): pose rows packed on
    // the frame's stream into one of two device staging buffers, copied to the
    // caller's pinned host buffer on a side stream.
    float* traj_host = nullptr;
    uint32_t traj_every = 0, traj_max = 0;
    uint64_t traj_frame = 0;              // frames stepped by dyph_world_step since the last set-up
    float* traj_stage[2] = {nullptr, nullptr};
    cudaStream_t traj_stream = nullptr;
    cudaEvent_t traj_packed[2] = {nullptr, nullptr};
    cudaEvent_t traj_copied[2] = {nullptr, nullptr};
    bool traj_pending = false;            // a copy on the side stream not yet joined
    bool traj_live[2] = {false, false};   // traj_copied[k] was last recorded outside a capture
    // Batched scenes with the whole frame fused into one kernel (one block per scene).
    bool fused = false;
    uint32_t frame_smem = 0;
    uint32_t* f_pair_base = nullptr;     // [n_scenes + 1]
    uint32_t* f_contact_base = nullptr;  // [n_scenes + 1]
    uint32_t* f_pair_raw = nullptr;
    uint32_t* f_contact_raw = nullptr;
    uint32_t* f_color_raw = nullptr;
    uint32_t* f_counts = nullptr;        // [4 n_scenes]
    uint32_t* f_words = nullptr;
    uint32_t* f_pos = nullptr;           // [2 n_scenes] gather positions
    uint32_t* f_items = nullptr;         // [4 f_n_items] work items of the fused kernel
    uint32_t f_n_items = 0;
    unsigned long long* f_phase = nullptr;  // [kFramePhases] phase timing of fused frames (null = off)
    // Adjoint of fused frames (dyph_world_rollout_backward), allocated on first use.
    // Record sets, one per frame of two checkpoint segments: contact records,
    // poses after integrate, quaternions before renormalisation, contact
    // words, counts.
    std::vector<float*> a_rec;       // [kRecWords][f_contact_slots]
    std::vector<float*> a_pose1;     // [7][n]
    std::vector<float*> a_qs;        // [4][n]
    std::vector<uint32_t*> a_words;  // [kSceneWords][f_words_stride]
    std::vector<uint32_t*> a_mg;     // [2 n_scenes]
    float* a_g[2] = {nullptr, nullptr};  // [13][n] adjoint ping-pong
    float* a_seg[2] = {nullptr, nullptr};  // [a_seg_frames][13][n] states of frames 1.. of a segment (double buffer)
    uint32_t a_seg_frames = 0;
    uint32_t* a_pairs = nullptr;         // pair slots of spilled scenes, the recording's own
    cudaStream_t a_stream = nullptr;     // records the next checkpoint segment while this one is reversed
    cudaEvent_t a_seg_ready = nullptr, a_rtail = nullptr, a_rev_done = nullptr;
    uint32_t* a_flag = nullptr;
    uint32_t a_sized[4] = {0, 0, 0, 0};  // contact slots, words stride, pair slots, scenes the sets were made for
    uint32_t f_words_stride = 0, f_contact_slots = 0, f_pair_slots = 0;
    // Knobs of the fused kernel (dyph_world_set_fused_config / dyph_world_autotune).
    std::vector<uint32_t> h_body_offset;  // host copy of the scenes' body ranges
    uint32_t f_smem_cap = 0;              // shared memory cap per block (0 = what the largest scene needs)
    uint32_t f_teams = 2;                 // 0 blocks only, 1 + small scenes one per warp, 2 + mid-size two warps
    uint32_t f_variant = 0;               // register budget: 4 (0), 5 (1) or 6 (2) blocks per SM
    uint32_t f_warp_scenes = 0, f_half_scenes = 0, f_block_scenes = 0;
    // Work items of the adjoint's reverse kernel, laid out on their own: its
    // levels are long dependent chains with a barrier each, which favours
    // one-warp teams over the forward frame's choice.
    uint32_t* r_items = nullptr;
    uint32_t r_n_items = 0, r_smem = 0;
    uint32_t r_smem_cap = 0;              // 0: a third of an SM's shared memory
    uint32_t r_teams = 2;
    uint32_t r_warp_scenes = 0, r_half_scenes = 0, r_block_scenes = 0;
    float f_tuned_ms = 0.f;
    uint32_t f_tuned_candidates = 0;
};

namespace dyph {
namespace {

constexpr uint32_t kHistory = 4096;

// Frame f's recomputation with recording for the adjoint (record_scene), on
// the fused kernel's work items.
__global__ void __launch_bounds__(kSceneThreads, 4) scene_frame_record_kernel(SceneBufs S, FrameBufs F,
                                                                              FrameParams P_, AdjRun A, AdjKeep K,
                                                                              const uint32_t* __restrict__ items,
                                                                              uint32_t n_items) {
    for_each_item(items, n_items, S.smem_bytes,
                  [&](const auto& T, uint32_t s, unsigned char* smem, uint32_t bytes, SceneShared& sh) {
                      record_scene(T, s, smem, bytes, sh, S, F, P_, A, K);
                  });
}
constexpr size_t kStatsWords = 8 + 2 * kHistory;

__global__ void frame_stats_kernel(const uint32_t* __restrict__ bp_counts, const uint32_t* __restrict__ np_counts,
                                   uint32_t max_pairs, uint32_t max_contacts, uint32_t* __restrict__ stats) {
    const uint32_t p = bp_counts[1], c = np_counts[1];
    stats[0] = p;
    stats[1] = c;
    stats[2] = max(stats[2], p);
    stats[3] = max(stats[3], c);
    // per-frame history ring: [8 + 2 k] pairs, [9 + 2 k] contacts of frame k mod kHistory
    const uint32_t f = stats[5]++;
    stats[8 + 2 * (f % kHistory)] = p;
    stats[9 + 2 * (f % kHistory)] = c;
    if (p > max_pairs) atomicCAS(&stats[4], 0u, static_cast<uint32_t>(DYPH_ERR_PAIR_OVERFLOW));
    if (c > max_contacts) atomicCAS(&stats[4], 0u, static_cast<uint32_t>(DYPH_ERR_CONTACT_OVERFLOW));
}

// Pose rows of every body, interleaved per body as the .trajectory row
// (x, y, z, w, qx, qy, qz), examples/stress_test_blocks/main.cpp:191-197.
__global__ void pack_pose_kernel(GlobalBodies B, float* __restrict__ out) {
    const uint32_t n = B.v.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float* r = out + 7ull * i;
        r[0] = B.px(i); r[1] = B.py(i); r[2] = B.pz(i);
        r[3] = B.qw(i); r[4] = B.qx(i); r[5] = B.qy(i); r[6] = B.qz(i);
    }
}

// Queue trajectory record `rec` (the pose rows after the frame just queued on
// s): pack into staging buffer rec % 2 once that buffer's previous copy is
// done (when `wait_prev`), then copy it to the host on the side stream.
dyph_status enqueue_trajectory_record(dyph_world* w, cudaStream_t s, uint64_t rec, bool wait_prev) {
    const uint32_t n = w->desc.bodies.n;
    const int k = static_cast<int>(rec & 1u);
    if (wait_prev) DYPH_CUDA_TRY(cudaStreamWaitEvent(s, w->traj_copied[k], 0));
    pack_pose_kernel<<<(n + 255) / 256, 256, 0, s>>>(GlobalBodies{w->desc.bodies}, w->traj_stage[k]);
    DYPH_CUDA_TRY(cudaGetLastError());
    DYPH_CUDA_TRY(cudaEventRecord(w->traj_packed[k], s));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(w->traj_stream, w->traj_packed[k], 0));
    DYPH_CUDA_TRY(cudaMemcpyAsync(w->traj_host + rec * 7ull * n, w->traj_stage[k], 7ull * n * sizeof(float),
                                  cudaMemcpyDeviceToHost, w->traj_stream));
    DYPH_CUDA_TRY(cudaEventRecord(w->traj_copied[k], w->traj_stream));
    w->traj_pending = true;
    return DYPH_OK;
}

// Order every queued trajectory copy before the work that follows on s.
dyph_status join_trajectory(dyph_world* w, cudaStream_t s, uint64_t last_rec) {
    if (!w->traj_pending) return DYPH_OK;
    DYPH_CUDA_TRY(cudaStreamWaitEvent(s, w->traj_copied[last_rec & 1u], 0));
    w->traj_pending = false;
    return DYPH_OK;
}

bool trajectory_frame(const dyph_world* w, uint64_t frame) {
    return w->traj_host && frame % w->traj_every == 0 && frame / w->traj_every < w->traj_max;
}

// Records an event inside a stream capture as a real timestamp node.
dyph_status probe_record(void* ev, cudaStream_t s) {
    if (!ev) return DYPH_OK;
    DYPH_CUDA_TRY(cudaEventRecordWithFlags(static_cast<cudaEvent_t>(ev), s, cudaEventRecordExternal));
    return DYPH_OK;
}

// One frame; when probe_stage matches a stage (0 integrate, 1 broadphase,
// 2 narrowphase, 3 solver) the events are recorded around it; probe_stage 4
// records them around the solver's dataflow kernel alone.
dyph_status enqueue_frame(dyph_world* w, cudaStream_t s, int probe_stage = -1, void* ev0 = nullptr,
                          void* ev1 = nullptr) {
    const dyph_world_desc& d = w->desc;
    dyph_status st;
    if (w->fused) {
        // One launch per frame: every scene's integrate, pairs, narrowphase and solve.
        DYPH_CUDA_TRY(cudaMemsetAsync(w->bp->counts, 0, 4 * sizeof(uint32_t), s));
        DYPH_CUDA_TRY(cudaMemsetAsync(w->np->counts, 0, 4 * sizeof(uint32_t), s));
        DYPH_CUDA_TRY(cudaMemsetAsync(w->sv->meta, 0, 16 * sizeof(uint32_t), s));
        if (probe_stage >= 0 && (st = probe_record(ev0, s)) != DYPH_OK) return st;
        const dyph_integrator_params& ip = d.integrator;
        const float sub_dt = ip.dt / static_cast<float>(ip.n_substeps);
        SceneBufs S{w->bp->body_offset, w->bp->bvh.scene_of, w->sv->scene_order, nullptr, nullptr, 0,
                    w->bp->n_scenes, w->frame_smem};
        FrameBufs F{w->f_pair_base, w->f_contact_base, w->f_pair_raw, w->f_contact_raw, w->f_color_raw,
                    w->f_counts, w->f_words, w->f_words_stride, w->f_contact_slots};
        FrameParams P{d.bodies, d.shapes, ip.gravity[0], ip.gravity[1], ip.gravity[2], sub_dt, 0.5f * sub_dt,
                      w->sv->friction, ip.dt, ip.n_substeps, static_cast<int>(w->sv->mode), w->sv->n_iters,
                      w->sv->meta, w->bp->counts, w->np->counts, w->stats + 4, w->f_phase};
        switch (w->f_variant) {
            case 1:
                scene_frame_kernel<5><<<w->f_n_items, kSceneThreads, w->frame_smem, s>>>(S, F, P, w->f_items,
                                                                                       w->f_n_items);
                break;
            case 2:
                scene_frame_kernel<6><<<w->f_n_items, kSceneThreads, w->frame_smem, s>>>(S, F, P, w->f_items,
                                                                                       w->f_n_items);
                break;
            default:
                scene_frame_kernel<4><<<w->f_n_items, kSceneThreads, w->frame_smem, s>>>(S, F, P, w->f_items,
                                                                                       w->f_n_items);
        }
        DYPH_CUDA_TRY(cudaGetLastError());
        if (probe_stage >= 0 && (st = probe_record(ev1, s)) != DYPH_OK) return st;
        frame_stats_kernel<<<1, 1, 0, s>>>(w->bp->counts, w->np->counts, w->bp->max_pairs, w->np->max_contacts,
                                           w->stats);
        DYPH_CUDA_TRY(cudaGetLastError());
        return DYPH_OK;
    }
    w->sv->probe_flow[0] = probe_stage == 4 ? ev0 : nullptr;
    w->sv->probe_flow[1] = probe_stage == 4 ? ev1 : nullptr;
    for (int stage = 0; stage < 4; ++stage) {
        if (stage == probe_stage && (st = probe_record(ev0, s)) != DYPH_OK) return st;
        switch (stage) {
            case 0: st = integrate_launch(&d.bodies, &d.integrator, s); break;
            case 1: st = broadphase_build(w->bp, &d.bodies, &d.shapes, &d.scene_bounds, s); break;
            case 2:
                st = narrowphase_run(w->np, w->bp->pairs, w->bp->counts, w->bp->max_pairs, &d.bodies, &d.shapes, s);
                break;
            default: st = xpbd_solve(w->sv, &w->np->view, &d.bodies, d.integrator.dt, s); break;
        }
        if (st != DYPH_OK) break;
        if (stage == probe_stage && (st = probe_record(ev1, s)) != DYPH_OK) break;
    }
    w->sv->probe_flow[0] = w->sv->probe_flow[1] = nullptr;
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
    if (w->episode) cudaGraphExecDestroy(w->episode);
    if (w->ev_in) cudaEventDestroy(w->ev_in);
    if (w->ev_out) cudaEventDestroy(w->ev_out);
    if (w->stream) cudaStreamDestroy(w->stream);
    if (w->stats) cudaFree(w->stats);
    if (w->scene_hash) cudaFree(w->scene_hash);
    if (w->traj_stream) cudaStreamSynchronize(w->traj_stream);
    for (int k = 0; k < 2; ++k) {
        if (w->traj_stage[k]) cudaFree(w->traj_stage[k]);
        if (w->traj_packed[k]) cudaEventDestroy(w->traj_packed[k]);
        if (w->traj_copied[k]) cudaEventDestroy(w->traj_copied[k]);
    }
    if (w->traj_stream) cudaStreamDestroy(w->traj_stream);
    void* fb[] = {w->f_pair_base, w->f_contact_base, w->f_pair_raw, w->f_contact_raw, w->f_color_raw, w->f_counts,
                  w->f_words, w->f_pos, w->f_items, w->r_items, w->f_phase, w->a_g[0], w->a_g[1], w->a_seg[0],
                  w->a_seg[1], w->a_flag, w->a_pairs};
    for (void* p : fb)
        if (p) cudaFree(p);
    for (size_t k = 0; k < w->a_rec.size(); ++k) {
        void* pk[] = {w->a_rec[k], w->a_pose1[k], w->a_qs[k], w->a_words[k], w->a_mg[k]};
        for (void* p : pk)
            if (p) cudaFree(p);
    }
    if (w->a_stream) cudaStreamDestroy(w->a_stream);
    if (w->a_seg_ready) cudaEventDestroy(w->a_seg_ready);
    if (w->a_rtail) cudaEventDestroy(w->a_rtail);
    if (w->a_rev_done) cudaEventDestroy(w->a_rev_done);
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
        if (cudaMalloc(&w->stats, kStatsWords * sizeof(uint32_t)) != cudaSuccess ||
            cudaMemset(w->stats, 0, kStatsWords * sizeof(uint32_t)) != cudaSuccess ||
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
    uint64_t last_rec = 0;
    for (int32_t f = 0; f < n_frames; ++f) {
        DYPH_CUDA_TRY(cudaGraphLaunch(w->graph, w->stream));
        if (trajectory_frame(w, w->traj_frame)) {
            last_rec = w->traj_frame / w->traj_every;
            const int k = static_cast<int>(last_rec & 1u);
            dyph_status st = enqueue_trajectory_record(w, w->stream, last_rec, w->traj_live[k]);
            if (st != DYPH_OK) return st;
            w->traj_live[k] = true;
        }
        ++w->traj_frame;
    }
    dyph_status jst = join_trajectory(w, w->stream, last_rec);
    if (jst != DYPH_OK) return jst;
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_out, w->stream));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->ev_out, 0));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_capture_episode(dyph_world* w, int32_t n_frames, int32_t probe_stage,
                                                  void* const* ev_start, void* const* ev_end) {
    if (!w || n_frames <= 0 || probe_stage < -1 || probe_stage > 4) return DYPH_ERR_INVALID;
    if (probe_stage >= 0 && (!ev_start || !ev_end)) return DYPH_ERR_INVALID;
    if (w->episode) {
        cudaGraphExecDestroy(w->episode);
        w->episode = nullptr;
    }
    cudaGraph_t g = nullptr;
    DYPH_CUDA_TRY(cudaStreamBeginCapture(w->stream, cudaStreamCaptureModeThreadLocal));
    dyph_status st = DYPH_OK;
    uint64_t last_rec = 0;
    for (int32_t f = 0; f < n_frames && st == DYPH_OK; ++f) {
        st = enqueue_frame(w, w->stream, probe_stage, probe_stage >= 0 ? ev_start[f] : nullptr,
                           probe_stage >= 0 ? ev_end[f] : nullptr);
        if (st == DYPH_OK && trajectory_frame(w, static_cast<uint64_t>(f))) {
            last_rec = static_cast<uint64_t>(f) / w->traj_every;
            st = enqueue_trajectory_record(w, w->stream, last_rec, last_rec >= 2);
        }
    }
    if (st == DYPH_OK) st = join_trajectory(w, w->stream, last_rec);
    w->traj_pending = false;
    cudaError_t ce = cudaStreamEndCapture(w->stream, &g);
    if (st != DYPH_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (ce != cudaSuccess) return DYPH_ERR_CUDA;
    ce = cudaGraphInstantiate(&w->episode, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        w->episode = nullptr;
        return DYPH_ERR_CUDA;
    }
    w->episode_frames = n_frames;
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_run_episode(dyph_world* w, dyph_stream s) {
    if (!w || !w->episode) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_in, cs));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(w->stream, w->ev_in, 0));
    DYPH_CUDA_TRY(cudaGraphLaunch(w->episode, w->stream));
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_out, w->stream));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->ev_out, 0));
    return DYPH_OK;
}

extern "C" dyph_status dyph_event_create(void** out) {
    if (!out) return DYPH_ERR_INVALID;
    cudaEvent_t e = nullptr;
    DYPH_CUDA_TRY(cudaEventCreate(&e));
    *out = e;
    return DYPH_OK;
}

extern "C" void dyph_event_destroy(void* ev) {
    if (ev) cudaEventDestroy(static_cast<cudaEvent_t>(ev));
}

extern "C" dyph_status dyph_event_record(void* ev, dyph_stream s) {
    if (!ev) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaEventRecord(static_cast<cudaEvent_t>(ev), reinterpret_cast<cudaStream_t>(s)));
    return DYPH_OK;
}

extern "C" dyph_status dyph_event_elapsed_ms(void* start, void* end, float* ms) {
    if (!start || !end || !ms) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaEventSynchronize(static_cast<cudaEvent_t>(end)));
    DYPH_CUDA_TRY(cudaEventElapsedTime(ms, static_cast<cudaEvent_t>(start), static_cast<cudaEvent_t>(end)));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_check_finite(dyph_world* w, dyph_stream s, uint32_t* out_first_bad) {
    if (!w) return DYPH_ERR_INVALID;
    return dyph_bodies_check_finite(&w->desc.bodies, s, out_first_bad);
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

extern "C" dyph_status dyph_world_download_history(dyph_world* w, dyph_stream s, uint32_t* pairs,
                                                   uint32_t* contacts, uint32_t cap, uint32_t* frames_total) {
    if (!w) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    static thread_local uint32_t h[kStatsWords];
    DYPH_CUDA_TRY(cudaMemcpyAsync(h, w->stats, sizeof(h), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    const uint32_t total = h[5];
    if (frames_total) *frames_total = total;
    // most recent min(cap, total, kHistory) frames, oldest first
    uint32_t m = total < kHistory ? total : kHistory;
    if (m > cap) m = cap;
    for (uint32_t i = 0; i < m; ++i) {
        const uint32_t f = total - m + i;
        if (pairs) pairs[i] = h[8 + 2 * (f % kHistory)];
        if (contacts) contacts[i] = h[9 + 2 * (f % kHistory)];
    }
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

namespace {

// Fused frames for batched scenes: per-scene pair / contact slots sized as the
// scene's own capacities when stepped alone (48 n + 64 pairs, 16 n + 64
// contacts), and one block's shared memory for the largest scene's bodies
// plus about two contacts per body.
// Shared memory a block needs for the largest scene's bodies plus its pair
// and contact words, and the least it can run with (bodies plus 64 contacts'
// words; pair and contact lists then live in global memory).
constexpr uint32_t kMaxSmem = 200u * 1024u;

uint32_t fused_smem_need(uint32_t max_nb) {
    return std::min(kMaxSmem, frame_body_bytes(max_nb) + (4u + kSceneWords * 4u) * 2u * std::max(64u, max_nb));
}
uint32_t fused_smem_floor(uint32_t max_nb) { return frame_body_bytes(max_nb) + 56u * 64u; }

// Work items, largest scenes first: a scene whose estimated shared-memory
// need fits a quarter of the block's (`share`) runs on one warp, four such
// scenes to a block (teams >= 1); one that fits half of it on two warps, two
// to a block (teams == 2); larger scenes take the whole block.
template <class Est>
void build_items(const uint32_t* body_offset, uint32_t n_scenes, uint32_t share, uint32_t teams, Est est,
                 std::vector<uint32_t>& items, uint32_t& n_small, uint32_t& n_mid) {
    std::vector<uint32_t> order(n_scenes);
    for (uint32_t i = 0; i < n_scenes; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [body_offset](uint32_t x, uint32_t y) {
        return body_offset[x + 1] - body_offset[x] > body_offset[y + 1] - body_offset[y];
    });
    items.clear();
    std::vector<uint32_t> small, mid;
    for (uint32_t s : order) {
        const uint32_t e = est(body_offset[s + 1] - body_offset[s]);
        if (teams >= 1 && e <= share) {
            small.push_back(s);
        } else if (teams >= 2 && e <= 2u * share) {
            mid.push_back(s);
        } else {
            items.insert(items.end(), {s, kItemBlock, kItemEmpty, kItemEmpty});
        }
    }
    for (size_t i = 0; i < mid.size(); i += 2)
        items.insert(items.end(), {mid[i], kItemHalf, i + 1 < mid.size() ? mid[i + 1] : kItemEmpty, kItemHalf});
    for (size_t i = 0; i < small.size(); i += 4)
        for (size_t j = 0; j < 4; ++j) items.push_back(i + j < small.size() ? small[i + j] : kItemEmpty);
    n_small = static_cast<uint32_t>(small.size());
    n_mid = static_cast<uint32_t>(mid.size());
}

// The fused kernels may take up to kMaxSmem of dynamic shared memory, set
// once per device: the attribute belongs to the kernel, not to a world, so a
// world that lowered it would make another world's launches fail.
constexpr int kFusedMaxDevices = 64;
std::mutex g_fused_smem_mu;
bool g_fused_smem[kFusedMaxDevices] = {};

dyph_status fused_smem_prepare() {
    int dev = 0;
    DYPH_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kFusedMaxDevices) return DYPH_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_fused_smem_mu);
    if (g_fused_smem[dev]) return DYPH_OK;
    for (const void* k : {reinterpret_cast<const void*>(scene_frame_kernel<4>),
                          reinterpret_cast<const void*>(scene_frame_kernel<5>),
                          reinterpret_cast<const void*>(scene_frame_kernel<6>),
                          reinterpret_cast<const void*>(scene_frame_record_kernel),
                          reverse_kernel()})
        DYPH_CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kMaxSmem)));
    g_fused_smem[dev] = true;
    return DYPH_OK;
}

// Dynamic shared memory per block with which `blocks` blocks of `kernel`
// share an SM, as the occupancy calculator counts it (static shared memory
// and the per-block reservation included): the SM's share for one block,
// lowered in 128-byte steps until that many blocks fit.
uint32_t smem_for_blocks(const void* kernel, int blocks) {
    int dev = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0u;
    }
    uint32_t bytes = std::min(kMaxSmem, static_cast<uint32_t>(per_sm / blocks)) & ~127u;
    for (; bytes >= 128u; bytes -= 128u) {
        int fit = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, kSceneThreads, bytes) != cudaSuccess) {
            cudaGetLastError();
            return 0u;
        }
        if (fit >= blocks) return bytes;
    }
    return 0u;
}

// Dynamic shared memory per block when `blocks` blocks of `kernel` split an
// SM's shared memory (its static shared memory and the per-block reservation
// counted), whatever its registers allow.
uint32_t smem_share(const void* kernel, uint32_t blocks) {
    int dev = 0, per_sm = 0, reserved = 0;
    cudaFuncAttributes fa{};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, kernel) != cudaSuccess) {
        cudaGetLastError();
        return 0u;
    }
    const int64_t bytes = static_cast<int64_t>(per_sm) / blocks - reserved - static_cast<int64_t>(fa.sharedSizeBytes);
    return bytes > 0 ? std::min(kMaxSmem, static_cast<uint32_t>(bytes) & ~127u) : 0u;
}

// The reverse kernel's items and shared memory: per scene its bodies' rows
// plus the contact words and records of about 2.5 contacts per body (a scene
// with more reads them from global memory).
dyph_status setup_reverse(dyph_world* w) {
    const uint32_t n_scenes = static_cast<uint32_t>(w->h_body_offset.size() - 1);
    const uint32_t* off = w->h_body_offset.data();
    uint32_t max_nb = 0;
    for (uint32_t i = 0; i < n_scenes; ++i) max_nb = std::max(max_nb, off[i + 1] - off[i]);
    // Default: a third of an SM's shared memory. The kernel's registers allow
    // two blocks per SM; the smaller blocks leave shared memory to the
    // recording kernel that runs beside it. At least the largest scene's
    // bodies plus 64 contacts' words.
    uint32_t smem = w->r_smem_cap ? std::min(kMaxSmem, w->r_smem_cap & ~15u) : smem_share(reverse_kernel(), 3u);
    smem = std::max(smem, frame_body_bytes(max_nb) + kSceneWords * 4u * 64u);
    if (smem > kMaxSmem) return DYPH_ERR_TOO_LARGE;
    std::vector<uint32_t> items;
    uint32_t n_small = 0, n_mid = 0;
    build_items(off, n_scenes, (smem / 4u) & ~15u, w->r_teams,
                [](uint32_t nb) { return frame_body_bytes(nb) + (kSceneWords + kRecWords) * 10u * nb; }, items,
                n_small, n_mid);
    if (w->r_items) cudaFree(w->r_items);
    w->r_items = nullptr;
    if (cudaMalloc(&w->r_items, items.size() * 4) != cudaSuccess) return DYPH_ERR_NOMEM;
    DYPH_CUDA_TRY(cudaMemcpy(w->r_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice));
    w->r_n_items = static_cast<uint32_t>(items.size() / 4);
    w->r_smem = smem;
    w->r_warp_scenes = n_small;
    w->r_half_scenes = n_mid;
    w->r_block_scenes = n_scenes - n_small - n_mid;
    return DYPH_OK;
}

dyph_status setup_fused(dyph_world* w, uint32_t n_scenes, const uint32_t* body_offset) {
    w->fused = false;
    w->h_body_offset.assign(body_offset, body_offset + n_scenes + 1);
    uint32_t max_nb = 0;
    std::vector<uint32_t> pb(n_scenes + 1, 0u), cb(n_scenes + 1, 0u);
    for (uint32_t i = 0; i < n_scenes; ++i) {
        const uint32_t nb = body_offset[i + 1] - body_offset[i];
        max_nb = std::max(max_nb, nb);
        pb[i + 1] = pb[i] + std::max(64u, 48u * nb + 64u);
        cb[i + 1] = cb[i] + std::max(64u, 16u * nb + 64u);
    }
    if (fused_smem_floor(max_nb) > kMaxSmem) return DYPH_ERR_TOO_LARGE;
    dyph_status prep = fused_smem_prepare();
    if (prep != DYPH_OK) return prep;
    uint32_t smem = fused_smem_need(max_nb);
    const void* variant = w->f_variant == 1   ? reinterpret_cast<const void*>(scene_frame_kernel<5>)
                          : w->f_variant == 2 ? reinterpret_cast<const void*>(scene_frame_kernel<6>)
                                              : reinterpret_cast<const void*>(scene_frame_kernel<4>);
    if (w->f_smem_cap) {
        smem = std::max(fused_smem_floor(max_nb), std::min(smem, w->f_smem_cap & ~15u));
    } else {
        // With more scenes than SMs, a block that leaves room for a second one
        // on its SM beats one that holds the largest scene whole.
        int dev = 0, sms = 0;
        DYPH_CUDA_TRY(cudaGetDevice(&dev));
        DYPH_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const uint32_t two = smem_for_blocks(variant, 2);
        if (n_scenes > static_cast<uint32_t>(sms) && smem > two && two >= fused_smem_floor(max_nb)) smem = two;
    }
    uint32_t** bufs[] = {&w->f_pair_base, &w->f_contact_base, &w->f_pair_raw, &w->f_contact_raw, &w->f_color_raw,
                         &w->f_counts, &w->f_words, &w->f_pos};
    for (uint32_t** b : bufs) {
        if (*b) cudaFree(*b);
        *b = nullptr;
    }
    if (w->f_items) cudaFree(w->f_items);
    w->f_items = nullptr;
    const size_t pslots = pb[n_scenes], cslots = cb[n_scenes];
    w->f_contact_slots = static_cast<uint32_t>(cslots);
    w->f_pair_slots = static_cast<uint32_t>(pslots);
    w->f_words_stride = static_cast<uint32_t>(cslots + n_scenes);
    const size_t sizes[] = {n_scenes + 1ull, n_scenes + 1ull, pslots, 9 * cslots, cslots, 4ull * n_scenes,
                            static_cast<size_t>(kSceneWords) * w->f_words_stride, 2ull * n_scenes};
    for (int k = 0; k < 8; ++k)
        if (cudaMalloc(bufs[k], sizes[k] * sizeof(uint32_t)) != cudaSuccess) return DYPH_ERR_NOMEM;
    // Work items: a scene's frame is expected to need its bodies' rows plus
    // about 4 pairs and 2.5 contacts per body.
    std::vector<uint32_t> items;
    uint32_t n_small = 0, n_mid = 0;
    build_items(body_offset, n_scenes, (smem / 4u) & ~15u, w->f_teams,
                [](uint32_t nb) { return frame_body_bytes(nb) + 146u * nb; }, items, n_small, n_mid);
    w->f_n_items = static_cast<uint32_t>(items.size() / 4);
    if (cudaMalloc(&w->f_items, items.size() * 4) != cudaSuccess) return DYPH_ERR_NOMEM;
    DYPH_CUDA_TRY(cudaMemcpy(w->f_items, items.data(), items.size() * 4, cudaMemcpyHostToDevice));
    DYPH_CUDA_TRY(cudaMemcpy(w->f_pair_base, pb.data(), pb.size() * 4, cudaMemcpyHostToDevice));
    DYPH_CUDA_TRY(cudaMemcpy(w->f_contact_base, cb.data(), cb.size() * 4, cudaMemcpyHostToDevice));
    DYPH_CUDA_TRY(cudaMemset(w->f_counts, 0, 4ull * n_scenes * sizeof(uint32_t)));
    w->frame_smem = smem;
    w->f_warp_scenes = n_small;
    w->f_half_scenes = n_mid;
    w->f_block_scenes = n_scenes - n_small - n_mid;
    dyph_status st = setup_reverse(w);
    if (st != DYPH_OK) return st;
    w->fused = true;
    return DYPH_OK;
}

void drop_graphs(dyph_world* w) {
    if (w->graph) cudaGraphExecDestroy(w->graph);
    if (w->episode) cudaGraphExecDestroy(w->episode);
    w->graph = w->episode = nullptr;
    w->episode_frames = 0;
}

void fused_report(const dyph_world* w, dyph_fused_config* out) {
    *out = dyph_fused_config{};
    if (!w->fused) return;
    int per_sm = 0;
    const void* k = w->f_variant == 1   ? reinterpret_cast<const void*>(scene_frame_kernel<5>)
                    : w->f_variant == 2 ? reinterpret_cast<const void*>(scene_frame_kernel<6>)
                                        : reinterpret_cast<const void*>(scene_frame_kernel<4>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kSceneThreads, w->frame_smem);
    out->smem_bytes = w->frame_smem;
    out->teams = w->f_teams;
    out->warp_scenes = w->f_warp_scenes;
    out->half_scenes = w->f_half_scenes;
    out->block_scenes = w->f_block_scenes;
    out->blocks = w->f_n_items;
    out->blocks_per_sm = static_cast<uint32_t>(per_sm);
    out->register_blocks = 4u + w->f_variant;
    out->ms_per_frame = w->f_tuned_ms;
    out->candidates = w->f_tuned_candidates;
}

// Tuned configurations, per device and batch profile (scene sizes, solver
// settings), for the life of the process.
struct TunedConfig {
    uint32_t smem_cap;
    uint32_t teams;
    uint32_t variant;
    float ms;
};
std::mutex g_tuned_mu;
std::map<uint64_t, TunedConfig> g_tuned;

uint64_t tune_key(const dyph_world* w) {
    int dev = 0;
    cudaGetDevice(&dev);
    uint64_t h = 0xcbf29ce484222325ull;
    auto mix = [&h](uint64_t v) {
        for (int b = 0; b < 8; ++b) {
            h ^= (v >> (8 * b)) & 0xFFu;
            h *= 0x100000001b3ull;
        }
    };
    mix(static_cast<uint64_t>(dev));
    mix(static_cast<uint64_t>(w->sv->mode));
    mix(static_cast<uint64_t>(w->sv->n_iters));
    mix(static_cast<uint64_t>(w->desc.integrator.n_substeps));
    for (uint32_t v : w->h_body_offset) mix(v);
    return h;
}

}  // namespace

extern "C" dyph_status dyph_world_sync_lists(dyph_world* w, dyph_stream s) {
    if (!w) return DYPH_ERR_INVALID;
    if (!w->fused) return DYPH_OK;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_in, cs));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(w->stream, w->ev_in, 0));
    const uint32_t n = w->bp->n_scenes;
    scene_gather_scan_kernel<<<1, 1024, 0, w->stream>>>(w->f_counts, n, w->f_pos, w->bp->counts, w->np->counts);
    SceneBufs S{w->bp->body_offset, w->bp->bvh.scene_of, w->sv->scene_order, nullptr, nullptr, 0, n, 0};
    FrameBufs F{w->f_pair_base, w->f_contact_base, w->f_pair_raw, w->f_contact_raw, w->f_color_raw, w->f_counts,
                w->f_words, w->f_words_stride, w->f_contact_slots};
    scene_gather_copy_kernel<<<n, 256, 0, w->stream>>>(S, F, w->f_pos, w->bp->pairs, w->np->view, w->sv->color);
    DYPH_CUDA_TRY(cudaGetLastError());
    DYPH_CUDA_TRY(cudaEventRecord(w->ev_out, w->stream));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->ev_out, 0));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_fused_config(dyph_world* w, dyph_fused_config* out) {
    if (!w || !out) return DYPH_ERR_INVALID;
    fused_report(w, out);
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_set_fused_config(dyph_world* w, uint32_t smem_cap, uint32_t teams,
                                                   uint32_t register_blocks) {
    if (!w || !w->fused || teams > 2u || (register_blocks != 0 && (register_blocks < 4 || register_blocks > 6)))
        return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    w->f_smem_cap = smem_cap;
    w->f_teams = teams;
    w->f_variant = register_blocks ? register_blocks - 4u : 0u;
    const std::vector<uint32_t> off = w->h_body_offset;
    dyph_status st = setup_fused(w, static_cast<uint32_t>(off.size() - 1), off.data());
    drop_graphs(w);
    return st;
}

extern "C" dyph_status dyph_world_adjoint_config(dyph_world* w, dyph_fused_config* out) {
    if (!w || !out) return DYPH_ERR_INVALID;
    *out = dyph_fused_config{};
    if (!w->fused) return DYPH_OK;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reverse_kernel(), kSceneThreads, w->r_smem);
    out->smem_bytes = w->r_smem;
    out->teams = w->r_teams;
    out->warp_scenes = w->r_warp_scenes;
    out->half_scenes = w->r_half_scenes;
    out->block_scenes = w->r_block_scenes;
    out->blocks = w->r_n_items;
    out->blocks_per_sm = static_cast<uint32_t>(per_sm);
    out->register_blocks = 2u;
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_set_adjoint_config(dyph_world* w, uint32_t smem_bytes, uint32_t teams) {
    if (!w || !w->fused || teams > 2u) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    w->r_smem_cap = smem_bytes;
    w->r_teams = teams;
    return setup_reverse(w);
}

extern "C" dyph_status dyph_world_autotune(dyph_world* w, int32_t frames, dyph_stream s, dyph_fused_config* out) {
    if (!w || !w->fused || frames <= 0) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    const uint64_t key = tune_key(w);
    {
        std::lock_guard<std::mutex> lock(g_tuned_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            dyph_status st =
                dyph_world_set_fused_config(w, it->second.smem_cap, it->second.teams, 4u + it->second.variant);
            w->f_tuned_ms = it->second.ms;
            w->f_tuned_candidates = 0;  // taken from the cache
            if (out) fused_report(w, out);
            return st;
        }
    }
    const size_t n = w->desc.bodies.n;
    uint32_t max_nb = 0;
    for (size_t k = 0; k + 1 < w->h_body_offset.size(); ++k)
        max_nb = std::max(max_nb, w->h_body_offset[k + 1] - w->h_body_offset[k]);
    // The state, the statistics and the phase timer are put back after the trials.
    float* saved = nullptr;
    uint32_t saved_stats[5];
    if (cudaMalloc(&saved, 13 * n * sizeof(float)) != cudaSuccess) return DYPH_ERR_NOMEM;
    float* rows[13] = {w->desc.bodies.pos_x, w->desc.bodies.pos_y, w->desc.bodies.pos_z, w->desc.bodies.rot_w,
                       w->desc.bodies.rot_x, w->desc.bodies.rot_y, w->desc.bodies.rot_z, w->desc.bodies.vel_x,
                       w->desc.bodies.vel_y, w->desc.bodies.vel_z, w->desc.bodies.ang_x, w->desc.bodies.ang_y,
                       w->desc.bodies.ang_z};
    auto copy_rows = [&](bool save) -> cudaError_t {
        for (int r = 0; r < 13; ++r) {
            cudaError_t e = save ? cudaMemcpyAsync(saved + r * n, rows[r], n * 4, cudaMemcpyDeviceToDevice, w->stream)
                                 : cudaMemcpyAsync(rows[r], saved + r * n, n * 4, cudaMemcpyDeviceToDevice, w->stream);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    };
    dyph_status st = DYPH_OK;
    unsigned long long* phase = w->f_phase;
    w->f_phase = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    const uint32_t need = fused_smem_need(max_nb), floor_ = fused_smem_floor(max_nb);
    // caps below the need down to the floor itself (the least a block can hold)
    std::vector<uint32_t> caps = {need};
    for (uint32_t c : {96u << 10, 72u << 10, 56u << 10, 48u << 10, 44u << 10, 40u << 10, 32u << 10})
        if (c < need && c >= floor_) caps.push_back(c);
    if (floor_ < need && std::find(caps.begin(), caps.end(), floor_) == caps.end()) caps.push_back(floor_);
    TunedConfig best{need, 2u, 0u, 1e30f};
    uint32_t tried = 0;
    const uint32_t cap0 = w->f_smem_cap, variant0 = w->f_variant;
    const uint32_t teams0 = w->f_teams;
    do {
        if (cudaMemcpyAsync(saved_stats, w->stats, sizeof(saved_stats), cudaMemcpyDeviceToHost, w->stream) !=
                cudaSuccess ||
            copy_rows(true) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
            cudaEventCreate(&e1) != cudaSuccess) {
            st = DYPH_ERR_CUDA;
            break;
        }
        for (uint32_t cap : caps) {
            for (uint32_t combo = 0; combo < 9u && st == DYPH_OK; ++combo) {
                const uint32_t teams = 2u - combo / 3u;
                const uint32_t variant = combo % 3u;
                w->f_smem_cap = cap;
                w->f_teams = teams;
                w->f_variant = variant;
                st = setup_fused(w, static_cast<uint32_t>(w->h_body_offset.size() - 1), w->h_body_offset.data());
                if (st != DYPH_OK) break;
                // one untimed frame, then the timed ones, each trial from the saved state
                for (int f = 0; f <= frames && st == DYPH_OK; ++f) {
                    if (f == 1 && cudaEventRecord(e0, w->stream) != cudaSuccess) st = DYPH_ERR_CUDA;
                    if (st == DYPH_OK) st = enqueue_frame(w, w->stream);
                }
                if (st == DYPH_OK && cudaEventRecord(e1, w->stream) != cudaSuccess) st = DYPH_ERR_CUDA;
                if (st == DYPH_OK && (copy_rows(false) != cudaSuccess || cudaStreamSynchronize(w->stream) != cudaSuccess))
                    st = DYPH_ERR_CUDA;
                float ms = 0.f;
                if (st == DYPH_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) st = DYPH_ERR_CUDA;
                if (st != DYPH_OK) break;
                ++tried;
                ms /= static_cast<float>(frames);
                if (ms < best.ms) best = TunedConfig{cap, teams, variant, ms};
            }
            if (st != DYPH_OK) break;
        }
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    w->f_phase = phase;
    if (st == DYPH_OK) {
        w->f_smem_cap = best.smem_cap;
        w->f_teams = best.teams;
        w->f_variant = best.variant;
    } else {
        w->f_smem_cap = cap0;
        w->f_teams = teams0;
        w->f_variant = variant0;
    }
    const dyph_status st2 = setup_fused(w, static_cast<uint32_t>(w->h_body_offset.size() - 1), w->h_body_offset.data());
    drop_graphs(w);
    if (st == DYPH_OK && st2 == DYPH_OK) {
        if (cudaMemcpyAsync(w->stats, saved_stats, sizeof(saved_stats), cudaMemcpyHostToDevice, w->stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(w->stream) != cudaSuccess)
            st = DYPH_ERR_CUDA;
        w->f_tuned_ms = best.ms;
        w->f_tuned_candidates = tried;
        std::lock_guard<std::mutex> lock(g_tuned_mu);
        g_tuned[key] = best;
    }
    cudaFree(saved);
    if (out) fused_report(w, out);
    return st != DYPH_OK ? st : st2;
}

extern "C" dyph_status dyph_world_set_scenes(dyph_world* w, uint32_t n_scenes, const uint32_t* body_offset,
                                             const dyph_aabb* scene_bounds) {
    if (!w || !body_offset || n_scenes == 0 || body_offset[n_scenes] != w->desc.bodies.n) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    dyph_status st = broadphase_set_scenes(w->bp, n_scenes, body_offset, scene_bounds);
    if (st != DYPH_OK) return st;
    // One block per scene when the largest scene fits a block; otherwise the
    // whole-batch kernels solve the batch.
    st = xpbd_set_scenes(w->sv, n_scenes, body_offset, w->bp->body_offset, w->bp->bvh.scene_of);
    if (st != DYPH_OK && st != DYPH_ERR_TOO_LARGE) return st;
    if (st == DYPH_OK) {
        st = setup_fused(w, n_scenes, body_offset);
        if (st != DYPH_OK && st != DYPH_ERR_TOO_LARGE) return st;
    }
    // Captured frames launch the single-scene form: record them again.
    if (w->graph) cudaGraphExecDestroy(w->graph);
    if (w->episode) cudaGraphExecDestroy(w->episode);
    w->graph = nullptr;
    w->episode = nullptr;
    w->episode_frames = 0;
    if (w->scene_hash) cudaFree(w->scene_hash);
    w->scene_hash = nullptr;
    if (cudaMalloc(&w->scene_hash, n_scenes * sizeof(uint64_t)) != cudaSuccess) return DYPH_ERR_NOMEM;
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_scene_hashes(dyph_world* w, dyph_stream s, uint64_t* host_out, uint32_t cap) {
    if (!w || !host_out) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    const uint32_t n = w->bp->n_scenes ? w->bp->n_scenes : 1u;
    if (cap < n) return DYPH_ERR_INVALID;
    if (!w->scene_hash && cudaMalloc(&w->scene_hash, sizeof(uint64_t)) != cudaSuccess) return DYPH_ERR_NOMEM;
    dyph_status st = fnv_state(&w->desc.bodies, w->bp->n_scenes ? w->bp->body_offset : nullptr, n, w->scene_hash, cs);
    if (st != DYPH_OK) return st;
    DYPH_CUDA_TRY(cudaMemcpyAsync(host_out, w->scene_hash, n * sizeof(uint64_t), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_set_trajectory(dyph_world* w, float* host_dst, uint32_t every,
                                                 uint32_t max_records) {
    if (!w || (host_dst && (every == 0 || max_records == 0))) return DYPH_ERR_INVALID;
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    if (w->traj_stream) DYPH_CUDA_TRY(cudaStreamSynchronize(w->traj_stream));
    // A captured episode has the old recording baked in.
    if (w->episode) {
        cudaGraphExecDestroy(w->episode);
        w->episode = nullptr;
        w->episode_frames = 0;
    }
    w->traj_host = host_dst;
    w->traj_every = every;
    w->traj_max = max_records;
    w->traj_frame = 0;
    w->traj_pending = false;
    w->traj_live[0] = w->traj_live[1] = false;
    if (!host_dst) return DYPH_OK;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, host_dst) != cudaSuccess || attr.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        w->traj_host = nullptr;
        return DYPH_ERR_INVALID;  // pageable memory: the copies could not run asynchronously or be captured
    }
    const size_t bytes = 7ull * w->desc.bodies.n * sizeof(float);
    for (int k = 0; k < 2; ++k) {
        if (!w->traj_stage[k] && cudaMalloc(&w->traj_stage[k], bytes) != cudaSuccess) return DYPH_ERR_NOMEM;
        if (!w->traj_packed[k]) DYPH_CUDA_TRY(cudaEventCreateWithFlags(&w->traj_packed[k], cudaEventDisableTiming));
        if (!w->traj_copied[k]) DYPH_CUDA_TRY(cudaEventCreateWithFlags(&w->traj_copied[k], cudaEventDisableTiming));
    }
    if (!w->traj_stream) DYPH_CUDA_TRY(cudaStreamCreateWithFlags(&w->traj_stream, cudaStreamNonBlocking));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_set_phase_timing(dyph_world* w, int on) {
    if (!w) return DYPH_ERR_INVALID;
    if (!w->fused) return on ? DYPH_ERR_INVALID : DYPH_OK;
    DYPH_CUDA_TRY(cudaStreamSynchronize(w->stream));
    // captured frames hold the old setting
    if (w->graph) cudaGraphExecDestroy(w->graph);
    if (w->episode) cudaGraphExecDestroy(w->episode);
    w->graph = w->episode = nullptr;
    w->episode_frames = 0;
    if (!on) {
        if (w->f_phase) cudaFree(w->f_phase);
        w->f_phase = nullptr;
        return DYPH_OK;
    }
    if (!w->f_phase && cudaMalloc(&w->f_phase, kFramePhases * sizeof(unsigned long long)) != cudaSuccess)
        return DYPH_ERR_NOMEM;
    DYPH_CUDA_TRY(cudaMemset(w->f_phase, 0, kFramePhases * sizeof(unsigned long long)));
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_download_phase_ns(dyph_world* w, dyph_stream s, uint64_t* out, uint32_t cap) {
    if (!w || !out || cap < static_cast<uint32_t>(kFramePhases) || !w->f_phase) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaMemcpyAsync(out, w->f_phase, kFramePhases * sizeof(uint64_t), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaMemsetAsync(w->f_phase, 0, kFramePhases * sizeof(uint64_t), cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

namespace dyph {
namespace {

// State rows (pos xyz, rot wxyz, vel xyz, ang xyz) of every body to / from a
// [13][n] buffer.
__global__ void pack_state_kernel(GlobalBodies B, float* __restrict__ out) {
    const uint32_t n = B.v.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float v[13] = {B.px(i), B.py(i), B.pz(i), B.qw(i), B.qx(i), B.qy(i), B.qz(i),
                             B.vx(i), B.vy(i), B.vz(i), B.wx(i), B.wy(i), B.wz(i)};
        for (int r = 0; r < 13; ++r) out[static_cast<size_t>(r) * n + i] = v[r];
    }
}

__global__ void unpack_state_kernel(const float* __restrict__ in, GlobalBodies B) {
    const uint32_t n = B.v.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = in + i;
        B.px(i) = r[0]; B.py(i) = r[n]; B.pz(i) = r[2ull * n];
        B.qw(i) = r[3ull * n]; B.qx(i) = r[4ull * n]; B.qy(i) = r[5ull * n]; B.qz(i) = r[6ull * n];
        B.vx(i) = r[7ull * n]; B.vy(i) = r[8ull * n]; B.vz(i) = r[9ull * n];
        B.wx(i) = r[10ull * n]; B.wy(i) = r[11ull * n]; B.wz(i) = r[12ull * n];
    }
}

dyph_status pack_state(const dyph_world* w, float* out, cudaStream_t s) {
    const uint32_t n = w->desc.bodies.n;
    pack_state_kernel<<<(n + 255) / 256, 256, 0, s>>>(GlobalBodies{w->desc.bodies}, out);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

dyph_status unpack_state(const dyph_world* w, const float* in, cudaStream_t s) {
    const uint32_t n = w->desc.bodies.n;
    unpack_state_kernel<<<(n + 255) / 256, 256, 0, s>>>(in, GlobalBodies{w->desc.bodies});
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

// A BodyView over a [13][n] state buffer, with the world's constant rows.
dyph_bodies state_view(const dyph_world* w, float* st) {
    dyph_bodies v = w->desc.bodies;
    const size_t n = v.n;
    float** rows[13] = {&v.pos_x, &v.pos_y, &v.pos_z, &v.rot_w, &v.rot_x, &v.rot_y, &v.rot_z,
                        &v.vel_x, &v.vel_y, &v.vel_z, &v.ang_x, &v.ang_y, &v.ang_z};
    for (int r = 0; r < 13; ++r) *rows[r] = st + r * n;
    return v;
}

// Frames per recorded segment of a backward pass with a checkpoint at every
// frame: enough to record the next segment while one is reversed, with one
// wait between the two streams per segment; fewer when the two segments'
// record sets would pass kRecordBudget bytes.
constexpr int32_t kRecordGroup = 4;
constexpr size_t kRecordBudget = size_t(2) << 30;

// Bytes of one record set (records, poses after integrate, quaternions before
// renormalisation, contact words, counts).
size_t record_set_bytes(const dyph_world* w) {
    return 4 * (static_cast<size_t>(kRecWords) * w->f_contact_slots + 11ull * w->desc.bodies.n +
                static_cast<size_t>(kSceneWords) * w->f_words_stride + 2ull * std::max(w->bp->n_scenes, 1u));
}

// The adjoint's buffers: `sets` record sets and two segment buffers of
// `seg_states` states each. The record sets and the recording's pair slots
// are sized by the scenes' slots, so they are made again after the scenes
// change (dyph_world_set_scenes).
dyph_status adjoint_buffers(dyph_world* w, uint32_t sets, uint32_t seg_states) {
    const size_t n = w->desc.bodies.n;
    const uint32_t n_sc = std::max(w->bp->n_scenes, 1u);
    if (!w->a_g[0]) {
        const bool ok = cudaMalloc(&w->a_g[0], 13 * n * 4) == cudaSuccess &&
                        cudaMalloc(&w->a_g[1], 13 * n * 4) == cudaSuccess && cudaMalloc(&w->a_flag, 4) == cudaSuccess;
        if (!ok) return DYPH_ERR_NOMEM;
        DYPH_CUDA_TRY(cudaStreamCreateWithFlags(&w->a_stream, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&w->a_seg_ready, &w->a_rtail, &w->a_rev_done})
            DYPH_CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    const uint32_t sized[4] = {w->f_contact_slots, w->f_words_stride, w->f_pair_slots, n_sc};
    if (!std::equal(sized, sized + 4, w->a_sized)) {
        for (size_t k = 0; k < w->a_rec.size(); ++k) {
            void* pk[] = {w->a_rec[k], w->a_pose1[k], w->a_qs[k], w->a_words[k], w->a_mg[k]};
            for (void* p : pk)
                if (p) cudaFree(p);
        }
        w->a_rec.clear();
        w->a_pose1.clear();
        w->a_qs.clear();
        w->a_words.clear();
        w->a_mg.clear();
        if (w->a_pairs) cudaFree(w->a_pairs);
        w->a_pairs = nullptr;
        std::fill(w->a_sized, w->a_sized + 4, 0u);
        if (cudaMalloc(&w->a_pairs, static_cast<size_t>(std::max(w->f_pair_slots, 1u)) * 4) != cudaSuccess)
            return DYPH_ERR_NOMEM;
        std::copy(sized, sized + 4, w->a_sized);
    }
    while (w->a_rec.size() < sets) {
        float *rec = nullptr, *pose1 = nullptr, *qs = nullptr;
        uint32_t *words = nullptr, *mg = nullptr;
        const bool ok =
            cudaMalloc(&rec, static_cast<size_t>(kRecWords) * w->f_contact_slots * 4) == cudaSuccess &&
            cudaMalloc(&pose1, 7 * n * 4) == cudaSuccess && cudaMalloc(&qs, 4 * n * 4) == cudaSuccess &&
            cudaMalloc(&words, static_cast<size_t>(kSceneWords) * w->f_words_stride * 4) == cudaSuccess &&
            cudaMalloc(&mg, 2ull * n_sc * 4) == cudaSuccess;
        if (!ok) {
            void* pk[] = {rec, pose1, qs, words, mg};
            for (void* p : pk)
                if (p) cudaFree(p);
            return DYPH_ERR_NOMEM;
        }
        w->a_rec.push_back(rec);
        w->a_pose1.push_back(pose1);
        w->a_qs.push_back(qs);
        w->a_words.push_back(words);
        w->a_mg.push_back(mg);
    }
    if (seg_states > w->a_seg_frames) {
        for (float*& b : w->a_seg) {
            if (b) cudaFree(b);
            b = nullptr;
        }
        w->a_seg_frames = 0;
        for (float*& b : w->a_seg)
            if (cudaMalloc(&b, static_cast<size_t>(seg_states) * 13 * n * 4) != cudaSuccess) return DYPH_ERR_NOMEM;
        w->a_seg_frames = seg_states;
    }
    return DYPH_OK;
}

}  // namespace
}  // namespace dyph

extern "C" dyph_status dyph_world_rollout(dyph_world* w, int32_t n_frames, int32_t every, float* d_ckpt,
                                          dyph_stream s) {
    if (!w || !w->fused || n_frames <= 0 || every <= 0 || !d_ckpt) return DYPH_ERR_INVALID;
    const size_t n = w->desc.bodies.n;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    for (int32_t f = 0; f < n_frames; ++f) {
        if (f % every == 0) {
            dyph_status st = pack_state(w, d_ckpt + static_cast<size_t>(f / every) * 13 * n, cs);
            if (st != DYPH_OK) return st;
        }
        dyph_status st = dyph_world_step(w, 1, s);
        if (st != DYPH_OK) return st;
    }
    return DYPH_OK;
}

extern "C" dyph_status dyph_world_rollout_backward(dyph_world* w, int32_t n_frames, int32_t every,
                                                   const float* d_ckpt, const float* d_grad_final,
                                                   float* d_grad_init, float* d_grad_inv_mass, dyph_stream s) {
    if (!w || !w->fused || n_frames <= 0 || every <= 0 || !d_ckpt || !d_grad_final || !d_grad_init ||
        !d_grad_inv_mass)
        return DYPH_ERR_INVALID;
    // Frames are recorded in segments on a_stream, one record set per frame;
    // sets alternate between two segments, so segment seg - 1 is recorded
    // while segment seg is reversed on the caller's stream, last frame first.
    // With checkpoints every `every` > 1 frames a segment is a checkpoint's
    // frames, each recorded from the state the one before stored; with a
    // checkpoint at every frame it is up to kRecordGroup frames, each recorded
    // from its own checkpoint (one frame when that many sets do not fit).
    int32_t group = every;
    if (every == 1) {
        const size_t sets = kRecordBudget / (2 * record_set_bytes(w));
        group = static_cast<int32_t>(std::max<size_t>(1, std::min<size_t>(kRecordGroup, sets)));
    }
    dyph_status st = DYPH_ERR_NOMEM;
    for (;;) {
        const uint32_t seg_frames = static_cast<uint32_t>(std::min(group, n_frames));
        st = adjoint_buffers(w, 2u * seg_frames, every > 1 ? seg_frames - 1u : 0u);
        if (st != DYPH_ERR_NOMEM || every > 1 || group == 1) break;
        cudaGetLastError();  // the failed allocation
        group = 1;
    }
    if (st != DYPH_OK) return st;
    const int32_t seg_frames = std::min(group, n_frames);
    const int32_t n_seg = (n_frames + group - 1) / group;
    const size_t n = w->desc.bodies.n;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaMemsetAsync(w->a_flag, 0, 4, cs));
    DYPH_CUDA_TRY(cudaMemsetAsync(d_grad_inv_mass, 0, n * 4, cs));
    DYPH_CUDA_TRY(cudaMemcpyAsync(w->a_g[0], d_grad_final, 13 * n * 4, cudaMemcpyDeviceToDevice, cs));
    const dyph_world_desc& d = w->desc;
    const dyph_integrator_params& ip = d.integrator;
    const float sub_dt = ip.dt / static_cast<float>(ip.n_substeps);
    SceneBufs S{w->bp->body_offset, w->bp->bvh.scene_of, w->sv->scene_order, nullptr, nullptr, 0, w->bp->n_scenes,
                w->frame_smem};
    SceneBufs S_rev = S;
    S_rev.smem_bytes = w->r_smem;
    auto seg_len = [&](int32_t seg) { return std::min(group, n_frames - seg * group); };
    auto ckpt = [&](int32_t c) { return d_ckpt + static_cast<size_t>(c) * 13 * n; };
    // Frame f's start state: its segment's checkpoint, or the state its
    // predecessor's recording stored. The record and reverse kernels only
    // read it, so a checkpoint serves directly.
    auto state = [&](int32_t f) {
        const int32_t seg = f / every, j = f % every;
        return j == 0 ? const_cast<float*>(ckpt(seg)) : w->a_seg[seg & 1] + static_cast<size_t>(j - 1) * 13 * n;
    };
    auto set_of = [&](int32_t f) { return static_cast<size_t>(((f / group) & 1) * seg_frames + f % group); };
    auto params = [&](int32_t f) {
        return FrameParams{state_view(w, state(f)), d.shapes, ip.gravity[0], ip.gravity[1], ip.gravity[2], sub_dt,
                           0.5f * sub_dt, w->sv->friction, ip.dt, ip.n_substeps, static_cast<int>(w->sv->mode),
                           w->sv->n_iters, w->sv->meta, w->bp->counts, w->np->counts, w->stats + 4, nullptr};
    };
    auto adj = [&](int32_t f, float* store) {
        const size_t k = set_of(f);
        return AdjRun{w->a_rec[k], w->f_contact_slots, w->a_pose1[k], w->a_qs[k], static_cast<uint32_t>(n),
                      w->a_flag, store};
    };
    auto keep = [&](int32_t f) { return AdjKeep{w->a_words[set_of(f)], w->a_mg[set_of(f)]}; };
    auto frame_bufs = [&](int32_t f) {
        return FrameBufs{w->f_pair_base, w->f_contact_base, w->a_pairs, w->f_contact_raw, w->f_color_raw,
                         w->f_counts, w->a_words[set_of(f)], w->f_words_stride, w->f_contact_slots};
    };
    // The recordings spill into their own pair slots and keep their contact
    // words; each but a segment's last stores the next frame's start state.
    auto record_segment = [&](int32_t seg) -> dyph_status {
        const int32_t f0 = seg * group, len = seg_len(seg);
        for (int32_t j = 0; j < len; ++j) {
            const int32_t f = f0 + j;
            float* store = every > 1 && j + 1 < len ? state(f + 1) : nullptr;
            scene_frame_record_kernel<<<w->f_n_items, kSceneThreads, w->frame_smem, w->a_stream>>>(
                S, frame_bufs(f), params(f), adj(f, store), keep(f), w->f_items, w->f_n_items);
            DYPH_CUDA_TRY(cudaGetLastError());
        }
        DYPH_CUDA_TRY(cudaEventRecord(w->a_seg_ready, w->a_stream));
        return DYPH_OK;
    };
    // everything below starts after the caller's stream
    DYPH_CUDA_TRY(cudaEventRecord(w->a_rtail, cs));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(w->a_stream, w->a_rtail, 0));
    if ((st = record_segment(n_seg - 1)) != DYPH_OK) return st;
    int cur = 0;
    for (int32_t seg = n_seg - 1; seg >= 0; --seg) {
        DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->a_seg_ready, 0));
        if (seg > 0) {
            // segment seg - 1's sets and states were last read by segment
            // seg + 1's reverse passes, queued on cs before this point
            if (seg + 1 < n_seg) DYPH_CUDA_TRY(cudaStreamWaitEvent(w->a_stream, w->a_rev_done, 0));
            if ((st = record_segment(seg - 1)) != DYPH_OK) return st;
        }
        for (int32_t f = seg * group + seg_len(seg) - 1; f >= seg * group; --f) {
            AdjFrame G{w->a_g[cur], w->a_g[cur ^ 1], d_grad_inv_mass};
            FrameBufs fb = frame_bufs(f);
            FrameParams pf = params(f);
            AdjRun af = adj(f, nullptr);
            AdjKeep kf = keep(f);
            void* args[] = {&S_rev, &fb, &pf, &af, &kf, &G, &w->r_items, &w->r_n_items};
            DYPH_CUDA_TRY(
                cudaLaunchKernel(reverse_kernel(), dim3(w->r_n_items), dim3(kSceneThreads), args, w->r_smem, cs));
            cur ^= 1;
        }
        DYPH_CUDA_TRY(cudaEventRecord(w->a_rev_done, cs));
    }
    // the side stream ends before the caller's stream goes on
    DYPH_CUDA_TRY(cudaEventRecord(w->a_rtail, w->a_stream));
    DYPH_CUDA_TRY(cudaStreamWaitEvent(cs, w->a_rtail, 0));
    DYPH_CUDA_TRY(cudaMemcpyAsync(d_grad_init, w->a_g[cur], 13 * n * 4, cudaMemcpyDeviceToDevice, cs));
    uint32_t flag = 0;
    DYPH_CUDA_TRY(cudaMemcpyAsync(&flag, w->a_flag, 4, cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return flag ? DYPH_ERR_UNSUPPORTED : DYPH_OK;
}
