// FNV-1a-64 of the pose arrays (examples/stress_test_blocks/main.cpp:34-41,
// 301-311): h = 0xcbf29ce484222325; for every byte of pos_x[n], pos_y, pos_z,
// rot_w, rot_x, rot_y, rot_z (little-endian float bytes): h ^= byte, h *= prime.
// FNV is byte-serial, so one thread hashes one scene; batched scenes hash in
// parallel (one thread per scene).
#include <cuda_runtime.h>

#include "internal.cuh"

namespace dyph {
namespace {

__device__ __forceinline__ uint64_t fnv_word(uint64_t h, uint32_t w) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
        h ^= (w >> (8 * b)) & 0xFFu;
        h *= 0x00000100000001B3ULL;
    }
    return h;
}

__global__ void fnv_state_kernel(GlobalBodies B, const uint32_t* __restrict__ offsets, uint32_t n_scenes,
                                 uint64_t* __restrict__ out) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_scenes) return;
    const uint32_t b0 = offsets ? offsets[s] : 0u;
    const uint32_t b1 = offsets ? offsets[s + 1] : B.v.n;
    const float* arr[7] = {B.v.pos_x, B.v.pos_y, B.v.pos_z, B.v.rot_w, B.v.rot_x, B.v.rot_y, B.v.rot_z};
    uint64_t h = 0xcbf29ce484222325ULL;
    for (int k = 0; k < 7; ++k)
        for (uint32_t i = b0; i < b1; ++i) h = fnv_word(h, __float_as_uint(arr[k][i]));
    out[s] = h;
}

}  // namespace

dyph_status fnv_state(const dyph_bodies* bodies, const uint32_t* d_offsets, uint32_t n_scenes, uint64_t* d_out,
                      cudaStream_t s) {
    if (!bodies || !d_out || n_scenes == 0) return DYPH_ERR_INVALID;
    fnv_state_kernel<<<(n_scenes + 127) / 128, 128, 0, s>>>(GlobalBodies{*bodies}, d_offsets, n_scenes, d_out);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

}  // namespace dyph

extern "C" dyph_status dyph_fnv1a64_state(const dyph_bodies* bodies, uint64_t* d_hash, dyph_stream s) {
    return dyph::fnv_state(bodies, nullptr, 1u, d_hash, reinterpret_cast<cudaStream_t>(s));
}

extern "C" dyph_status dyph_xpbd_download_stats(dyph_xpbd* sv, dyph_stream s, uint32_t* path, uint32_t* n_colors,
                                                uint32_t* rounds) {
    if (!sv) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t meta[16] = {};
    DYPH_CUDA_TRY(cudaMemcpyAsync(meta, sv->meta, sizeof(meta), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    // decision word: 2 coloured; 4 fallback / 5 sequential order run by the dataflow kernel;
    // 6 batched scenes, one per block (coloured when some scene was: word 13)
    const bool colored = meta[0] == 2u || (meta[0] == 6u && meta[13] != 0u);
    if (path) *path = meta[0] == 4u ? 1u : (meta[0] == 5u || meta[0] == 6u ? (colored ? 2u : 0u) : meta[0]);
    if (n_colors) *n_colors = colored ? meta[3] + 1u : 0u;
    if (rounds) *rounds = meta[7];
    return DYPH_OK;
}

extern "C" dyph_status dyph_xpbd_download_phase_ns(dyph_xpbd* sv, dyph_stream s, uint64_t* out4) {
    if (!sv || !out4) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t t[10];
    DYPH_CUDA_TRY(cudaMemcpyAsync(t, sv->meta + 144, sizeof(t), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    uint64_t ts[5];
    for (int i = 0; i < 5; ++i) ts[i] = static_cast<uint64_t>(t[2 * i]) | (static_cast<uint64_t>(t[2 * i + 1]) << 32);
    for (int i = 0; i < 4; ++i) out4[i] = (ts[i + 1] >= ts[i]) ? ts[i + 1] - ts[i] : 0u;
    return DYPH_OK;
}

extern "C" dyph_status dyph_xpbd_download_colors(dyph_xpbd* sv, dyph_stream s, uint32_t* host_colors, uint32_t cap,
                                                 uint32_t* n_colors) {
    if (!sv) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t meta[16] = {};
    DYPH_CUDA_TRY(cudaMemcpyAsync(meta, sv->meta, sizeof(meta), cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    // the coloured path finished, or batched scenes of which some were coloured
    // (the others' entries hold UINT32_MAX)
    const bool colored = meta[0] == 2u || (meta[0] == 6u && meta[13] != 0u);
    if (n_colors) *n_colors = colored ? meta[3] + 1u : 0u;
    if (host_colors && cap) {
        if (colored) {
            DYPH_CUDA_TRY(cudaMemcpyAsync(host_colors, sv->color, static_cast<size_t>(cap) * 4,
                                          cudaMemcpyDeviceToHost, cs));
            DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
        } else {
            for (uint32_t i = 0; i < cap; ++i) host_colors[i] = 0xFFFFFFFFu;
        }
    }
    return DYPH_OK;
}
