// The adjoint's reverse kernel, the library's second translation unit.
//
// It is compiled with contracted multiply-adds and approximate division and
// square root, unlike every other kernel (dyphur_b200.cu keeps each float
// operation correctly rounded and uncontracted, which the bit-exact forward
// frame and its recording need). The reverse pass only follows the branches
// the recording fixed (contact set, narrowphase features, solve flags, clamp
// bits); the signs it recomputes are of quantities that are zero by
// construction (their terms cancel) or far from zero, and its gradients are
// checked against the FP64 dual-number oracle within 1e-3 relative. The
// straight-line adjoint code then runs without the correctly rounded
// division's and square root's slow-path branches on each level's
// dependency chain.
//
// world.cu launches it through reverse_kernel() with cudaLaunchKernel: its
// argument structs come from the same headers in both translation units.
#define DYPH_DEVICE_GLOBAL static __device__

#include "internal.cuh"
#include "scene_frame.cuh"
#include "scene_adjoint.cuh"

namespace dyph {
namespace {

__global__ void __launch_bounds__(kSceneThreads, 2) scene_frame_reverse_kernel(SceneBufs S, FrameBufs F,
                                                                               FrameParams P_, AdjRun A, AdjKeep K,
                                                                               AdjFrame G,
                                                                               const uint32_t* __restrict__ items,
                                                                               uint32_t n_items) {
    for_each_item(items, n_items, S.smem_bytes,
                  [&](const auto& T, uint32_t s, unsigned char* smem, uint32_t bytes, SceneShared& sh) {
                      reverse_scene(T, s, smem, bytes, sh, S, F, P_, A, K, G);
                  });
}

}  // namespace

__attribute__((visibility("hidden"))) const void* reverse_kernel() {
    return reinterpret_cast<const void*>(scene_frame_reverse_kernel);
}

}  // namespace dyph
