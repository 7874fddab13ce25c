// Constants and small device helpers of the contact solver, shared by
// solver.cu and the solver headers it includes (solver_color.cuh,
// solver_flow.cuh, solver_scene.cuh), and by reverse.cu through
// solver_scene.cuh.
#pragma once

#include "internal.cuh"

namespace dyph {
namespace {

constexpr int kSeqThreads = 1024;
constexpr int kSeqWindow = 4;
constexpr uint32_t kUncolored = 0xFFFFFFFFu;
constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kSerialThreshold = 256u;  // XpbdSolver::kSerialThreshold (xpbd_solver.hpp:43)
constexpr uint32_t kMaxRounds = 256u;        // MAX_ROUNDS (xpbd_solver.cpp:645)

// meta words
constexpr int kMetaDecision = 0;  // 1 = sequential fallback requested, 2 = coloured path finished
constexpr int kMetaRemaining = 1;
constexpr int kMetaOverflow = 2;
constexpr int kMetaMaxColor = 3;
constexpr int kMetaBarrier = 4;   // [4] count, [5] generation
constexpr int kMetaDeferred = 6;
constexpr int kMetaRounds = 7;    // JP rounds of the last coloured solve (diagnostic)
constexpr int kMetaListLen = 8;   // [8, 11) work-list lengths of the JP rounds
constexpr int kMetaTailRemaining = 11;
constexpr int kMetaFlowPath = 12;  // 1 when the last coloured solve ran the dataflow kernel
constexpr int kMetaSceneColored = 13;  // batched scenes: 1 when some scene took the coloured order
constexpr uint32_t kDecisionScenes = 6u;  // decision word: the per-scene kernel solved the batch
constexpr int kMetaTime = 144;    // [144, 154) phase timestamps (ns) of the coloured solve
constexpr int kMetaColorCount = 16;   // [16, 80)
constexpr int kMetaColorCursor = 80;  // [80, 144)
constexpr int kMetaWords = 160;

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {  // xpbd_solver.cpp:31-34
    x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;
    return x;
}

__device__ __forceinline__ Contact load_contact(const dyph_contacts& cv, uint32_t c) {
    Contact ct;
    ct.a = cv.body_a[c]; ct.b = cv.body_b[c];
    ct.px = cv.pos_x[c]; ct.py = cv.pos_y[c]; ct.pz = cv.pos_z[c];
    ct.nx = cv.norm_x[c]; ct.ny = cv.norm_y[c]; ct.nz = cv.norm_z[c];
    ct.depth = cv.depth[c];
    return ct;
}

__device__ __forceinline__ uint32_t contact_count(const dyph_contacts& cv) {
    uint32_t nc = *cv.n;
    return nc < cv.capacity ? nc : cv.capacity;
}

__device__ __forceinline__ bool wants_sequential(int mode, uint32_t nc) {
    return mode == DYPH_SOLVER_SEQUENTIAL ||
           ((mode == DYPH_SOLVER_REFERENCE || mode == DYPH_SOLVER_REFERENCE_ROUNDS) && nc <= kSerialThreshold);
}

__device__ __forceinline__ void renorm_body(const GlobalBodies& B, uint32_t i, int times) {
    float qw = B.qw(i), qx = B.qx(i), qy = B.qy(i), qz = B.qz(i);
    for (int t = 0; t < times; ++t) renormalize(qw, qx, qy, qz);
    B.qw(i) = qw; B.qx(i) = qx; B.qy(i) = qy; B.qz(i) = qz;
}

}  // namespace
}  // namespace dyph
