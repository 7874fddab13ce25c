// Handle layouts and cross-file entry points of the native library.
#pragma once

#include <cuda_runtime.h>

#include "contact_math.cuh"
#include "sort.cuh"

namespace dyph {

// Device arrays of one LBVH (Karras indexing: internal nodes [0, n-2], leaf k
// at n-1+k; core/include/core/broadphase.hpp:95-106).
struct BvhBuffers {
    uint32_t* sorted_idx;   // leaf k -> body
    uint64_t* sorted_keys;  // (morton30 << 32 | body) of leaf k
    uint32_t* inv_sorted;   // body -> leaf k
    int32_t* left;          // [n-1]
    int32_t* right;         // [n-1]
    int32_t* parent;        // [2n-1]
    int32_t* root;          // [1] (always 0 for distinct keys)
    uint4* aabb;            // [2n-1] NodeBox (6 x fp16 + 2 pad)
    int32_t* range_hi;      // [n-1] last leaf covered by internal node i
    int32_t* rsplit;        // [n-1] right child of the node whose split is s
    uint32_t* slot;         // [2(n-1)] build rendezvous: far end of the left / right child
    uint32_t* flags;        // [n-1] build arrival counters (two per build)
    int32_t* range_lo;      // [n-1] first leaf covered by internal node i
    // Traversal record per node, 32 bytes = one sector: [2j] = fp16 box (12 B) +
    // left child (internal) or body (leaf); [2j+1] = lo, hi, escape node, 0.
    uint4* trav;            // [2(2n-1)]
    uint32_t* big;          // [2n-1] 1 when the subtree holds a static body's leaf
    uint32_t* bucket_cnt;   // [n] candidate partners b > a found for body a
    uint32_t* bucket;       // [n * kBucket] first kBucket partners of body a (unordered)
    // Batched scenes only (null for one scene):
    uint64_t* codes64;      // [n] (scene << 30 | Morton code), sorted in place
    uint32_t* scene_of;     // [n] scene of each body
    uint32_t* scene_first;  // [n_scenes] first sorted leaf of each scene
    uint32_t* scene_last;   // [n_scenes] last sorted leaf of each scene
};

// Partners kept per body by the Morton-order pass (a multiple of 32); bodies
// with more take a second, body-order traversal.
constexpr int kBucket = 128;

}  // namespace dyph

struct dyph_broadphase {
    uint32_t max_bodies = 0, max_pairs = 0, last_n = 0;
    uint32_t* codes = nullptr;   // Morton codes, sorted in place
    dyph::BvhBuffers bvh{};
    dyph_pair* pairs = nullptr;  // [max_pairs]
    uint32_t* counts = nullptr;  // [0] stored pairs, [1] true pairs, [2] tile counter, [3] subtree queue length
    uint2* queue = nullptr;      // [16 max_bodies] (leaf, subtree) items of the pair search's second pass
    uint32_t* tstatus = nullptr; // traversal look-back status, one word per 256 bodies
    void* sort_ws = nullptr;
    size_t sort_ws_bytes = 0;
    uint32_t n_scenes = 0;              // 0: one scene (bounds passed per build)
    int scene_bits = 0;                 // bits of a scene index
    dyph_aabb* scene_bounds = nullptr;  // [n_scenes] Morton bounds of each scene
    uint32_t* body_offset = nullptr;    // [n_scenes + 1] first body of each scene
};

struct dyph_narrowphase {
    uint32_t max_contacts = 0;
    dyph_contacts view{};         // store (count = stored contacts)
    uint32_t* counts = nullptr;   // [0] stored (== view.n), [1] true count, [2] tile counter
    uint32_t* status = nullptr;   // look-back status per 256-pair tile
    uint32_t status_words = 0;    // words cleared before a run
    uint32_t max_pairs_seen = 0;  // status capacity in tiles * 256
};

struct dyph_xpbd {
    int32_t n_iters = 10;
    float friction = 0.5f;
    uint32_t max_contacts = 0, max_bodies = 0;
    dyph_solver_mode mode = DYPH_SOLVER_REFERENCE;
    float* lambda = nullptr;        // [max_contacts]
    uint32_t* color = nullptr;      // [max_contacts]
    uint32_t* order = nullptr;      // [max_contacts] contacts grouped by colour / level
    uint32_t* pred = nullptr;       // [2 max_contacts] predecessor contact on body a / b
    uint32_t* done = nullptr;       // [max_contacts] wave in which a contact was solved
    uint64_t* bpri = nullptr;       // [3 max_bodies] JP priorities (read / post / clear buffers)
    uint64_t* bmask = nullptr;      // [max_bodies] JP used-colour masks
    uint32_t* blast = nullptr;      // [max_bodies] last contact seen per body (sequential path)
    uint32_t* meta = nullptr;       // solver control words (see solver.cu)
    uint64_t* body_list = nullptr;  // [64 max_bodies] dataflow path: (key, entry) lists of each body
    uint32_t* slot = nullptr;       // [2 max_contacts] dataflow path: list slot of each entry
    uint32_t* link = nullptr;       // [2 max_contacts] dataflow path: list predecessor of each entry
    uint64_t* cmask = nullptr;      // [2 max_contacts] dataflow path: published colour masks
    uint64_t* hand = nullptr;       // [2 max_contacts][16] dataflow path: tagged body-state records
    uint32_t* tail = nullptr;       // [max_bodies] dataflow path: last entry of each body's list
    uint32_t* sweep_tag = nullptr;  // [1] dataflow path: last sweep-pass number (kept across solves)
    uint32_t* csr_off = nullptr;    // [max_bodies + 1] dataflow sequential order: list offsets
    uint32_t* csr_cur = nullptr;    // [max_bodies] dataflow sequential order: fill cursors
    uint32_t* csr = nullptr;        // [2 max_contacts] dataflow sequential order: list entries
    uint32_t* partial = nullptr;    // [4096] dataflow sequential order: per-block sums
    int coop_blocks = 0;            // co-resident blocks of the round-synchronous coloured kernel
    int flow_blocks = 0;            // co-resident blocks of the dataflow kernel
    void* probe_flow[2] = {nullptr, nullptr};  // events recorded around the dataflow kernel (timing probe)
    // Batched scenes solved one scene per block (xpbd_set_scenes); 0 = off.
    uint32_t scene_n = 0;
    const uint32_t* scene_offset = nullptr;  // [scene_n + 1] device, owned by the broadphase
    const uint32_t* scene_of = nullptr;      // [bodies] device, owned by the broadphase
    uint32_t* scene_range = nullptr;         // [2 scene_n] first / end contact of each scene
    uint32_t* scene_order = nullptr;         // [scene_n] scenes by descending body count
    uint32_t* scene_scratch = nullptr;       // [13][scene_stride] per-contact words of large scenes
    uint32_t scene_stride = 0;               // max_contacts + scene_n
    uint32_t scene_smem = 0;                 // dynamic shared memory per block
};

namespace dyph {

dyph_status broadphase_create(uint32_t max_bodies, uint32_t max_pairs, dyph_broadphase** out);
void broadphase_destroy(dyph_broadphase* bp);
dyph_status broadphase_build(dyph_broadphase* bp, const dyph_bodies* bodies, const dyph_shapes* shapes,
                             const dyph_aabb* bounds, cudaStream_t s);
// Switch the broadphase to batched scenes (allocates; call outside graph capture).
dyph_status broadphase_set_scenes(dyph_broadphase* bp, uint32_t n_scenes, const uint32_t* h_body_offset,
                                  const dyph_aabb* h_scene_bounds);

dyph_status narrowphase_create(uint32_t max_contacts, dyph_narrowphase** out);
void narrowphase_destroy(dyph_narrowphase* np);
// Size the tile-status buffer for up to max_pairs pairs (allocates; call outside graph capture).
dyph_status narrowphase_reserve(dyph_narrowphase* np, uint32_t max_pairs);
dyph_status narrowphase_run(dyph_narrowphase* np, const dyph_pair* pairs, const uint32_t* d_n_pairs,
                            uint32_t max_pairs, const dyph_bodies* bodies, const dyph_shapes* shapes,
                            cudaStream_t s);

dyph_status xpbd_create(int32_t n_iters, uint32_t max_contacts, uint32_t max_bodies, float friction,
                        dyph_xpbd** out);
void xpbd_destroy(dyph_xpbd* sv);
dyph_status xpbd_solve(dyph_xpbd* sv, const dyph_contacts* contacts, const dyph_bodies* bodies, float dt,
                       cudaStream_t s);
// Solve batched scenes one scene per thread block (device arrays of the
// broadphase's scene set; allocates, call outside graph capture). Returns
// DYPH_ERR_TOO_LARGE, and leaves the whole-batch kernels in charge, when the
// largest scene's bodies do not fit one block's shared memory.
dyph_status xpbd_set_scenes(dyph_xpbd* sv, uint32_t n_scenes, const uint32_t* h_body_offset,
                            const uint32_t* d_body_offset, const uint32_t* d_scene_of);

// Pre-set kernel attributes of the sort (call once, outside graph capture).
dyph_status sort_prepare();

// The adjoint's reverse kernel (reverse.cu, its own translation unit), for
// cudaLaunchKernel with the argument list (SceneBufs, FrameBufs, FrameParams,
// AdjRun, AdjKeep, AdjFrame, const uint32_t* items, uint32_t n_items).
const void* reverse_kernel();

dyph_status integrate_launch(const dyph_bodies* bodies, const dyph_integrator_params* p, cudaStream_t s);

}  // namespace dyph
