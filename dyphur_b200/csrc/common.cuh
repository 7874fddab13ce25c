// Shared device helpers for the sm_100a frame-step kernels.
//
// Numerics: the library is compiled with --fmad=false, -prec-div=true and
// -prec-sqrt=true, so every a*b+c is two correctly rounded operations and
// division / square root are IEEE. That makes each kernel's float results
// identical to the reference's host build for the same inputs.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dyphur_b200.h"

namespace dyph {

constexpr uint32_t kFlagStatic = 1u;    // BodyFlag::Static (core/include/core/body.hpp:9)
constexpr uint32_t kFlagSleeping = 4u;  // BodyFlag::Sleeping (core/include/core/body.hpp:11)
constexpr uint32_t kShapeBox = 0u;
constexpr uint32_t kShapeSphere = 1u;

// Default iteration limit for every device-side spin (look-back, grid
// barrier, dataflow polls). With the nanosleep back-off this is well over a
// second of waiting. The limit in force is the device variable g_spin_limit
// (dyph_set_spin_limit), so a test can make a wait give up quickly.
constexpr uint32_t kSpinLimit = 1u << 24;

// The device words below belong to dyphur_b200.cu, the library's main
// translation unit (its kernels share them without relocatable device code).
// reverse.cu, the second one, defines DYPH_DEVICE_GLOBAL as `static
// __device__`: it gets private copies, which its one kernel never touches.
#ifndef DYPH_DEVICE_GLOBAL
#define DYPH_DEVICE_GLOBAL __device__
#endif

// Sticky device error word (DYPH_ERR_TIMEOUT ...), read by dyph_download_device_error.
DYPH_DEVICE_GLOBAL uint32_t g_device_error = 0u;

// Where the first error was raised (1 look-back, 2 sort look-back, 3 grid
// barrier, 5 sequential schedule, 6 / 7 tree walk, 8 narrowphase pair index).
DYPH_DEVICE_GLOBAL uint32_t g_device_error_site = 0u;

// Iteration limit of the bounded waits in force (the default unless a
// caller of dyph_set_spin_limit changed it).
DYPH_DEVICE_GLOBAL uint32_t g_spin_limit = kSpinLimit;

__device__ __forceinline__ uint32_t spin_limit() { return __ldg(&g_spin_limit); }

__device__ __forceinline__ void raise_error(uint32_t code, uint32_t site = 0u) {
    if (atomicCAS(&g_device_error, 0u, code) == 0u) g_device_error_site = site;
}

__device__ __forceinline__ float rsqrt_ieee(float x) { return __fdiv_rn(1.0f, __fsqrt_rn(x)); }

__device__ __forceinline__ uint16_t f2h_bits(float f) { return __half_as_ushort(__float2half_rn(f)); }
__device__ __forceinline__ float h2f_bits(uint16_t h) { return __half2float(__ushort_as_half(h)); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ── block-wide exclusive scan of one uint32 per thread ──────────────────────
// BLOCK threads; `smem` holds BLOCK/32 words. Returns the exclusive prefix and
// writes the block total.
template <int BLOCK>
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        constexpr int NW = BLOCK / 32;
        uint32_t w = lane < NW ? smem[lane] : 0u;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w += y;
        }
        if (lane < NW) smem[lane] = w;
    }
    __syncthreads();
    uint32_t warp_prefix = warp > 0 ? smem[warp - 1] : 0u;
    total = smem[BLOCK / 32 - 1];
    __syncthreads();
    return warp_prefix + x - v;
}

// ── decoupled look-back over tiles ──────────────────────────────────────────
// status[t]: 0 = not ready, (1 << 30) | v = tile aggregate v,
// (2 << 30) | v = inclusive prefix v. Values must stay below 2^30.
constexpr uint32_t kLbAgg = 1u << 30;
constexpr uint32_t kLbPrefix = 2u << 30;
constexpr uint32_t kLbMask = (1u << 30) - 1u;

// Called by one full warp. Publishes the tile aggregate, looks back, publishes
// the inclusive prefix and returns the exclusive prefix (valid in all lanes).
// On a timeout it raises DYPH_ERR_TIMEOUT and returns 0.
__device__ __forceinline__ uint32_t lookback_warp(uint32_t* status, uint32_t tile, uint32_t aggregate) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_release(&status[0], kLbPrefix | aggregate);
        return 0u;
    }
    if (lane == 0) st_release(&status[tile], kLbAgg | aggregate);
    uint32_t exclusive = 0;
    int64_t base = static_cast<int64_t>(tile) - 1;
    uint32_t spins = 0;
    const uint32_t limit = spin_limit();
    while (true) {
        int64_t t = base - lane;
        uint32_t s = (t >= 0) ? ld_acquire(&status[t]) : kLbPrefix;
        uint32_t flag = s & ~kLbMask;
        // Lane j looks at tile base - j. Everything from lane 0 up to the
        // closest tile holding an inclusive prefix must be ready.
        unsigned not_ready = __ballot_sync(0xffffffffu, flag == 0u);
        unsigned is_prefix = __ballot_sync(0xffffffffu, flag == kLbPrefix);
        unsigned first_prefix = is_prefix ? static_cast<unsigned>(__ffs(is_prefix) - 1) : 32u;
        unsigned need = (first_prefix >= 31u) ? 0xffffffffu : ((1u << (first_prefix + 1u)) - 1u);
        if (not_ready & need) {
            if (++spins > limit) {
                raise_error(DYPH_ERR_TIMEOUT, 1u);
                return 0u;
            }
            __nanosleep(32);
            continue;
        }
        uint32_t contrib = (static_cast<unsigned>(lane) <= first_prefix) ? (s & kLbMask) : 0u;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) contrib += __shfl_xor_sync(0xffffffffu, contrib, d);
        exclusive += contrib;
        if (first_prefix < 32) break;
        base -= 32;
    }
    if (lane == 0) st_release(&status[tile], kLbPrefix | ((exclusive + aggregate) & kLbMask));
    return exclusive;
}

// ── bounded grid barrier for cooperative launches ───────────────────────────
// bar[0] = arrival count, bar[1] = generation. Returns false (and raises
// DYPH_ERR_TIMEOUT) if the wait gave up; the caller must then leave the kernel.
// The block's writes are ordered before thread 0's arrival by __syncthreads;
// the arrival is an acq_rel atomic (release of the block's writes, acquire of
// the earlier arrivals'), and the release store of the generation word with
// the acquire spin on it carries the rest, so no separate fences are needed.
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ bool grid_barrier(uint32_t* bar, uint32_t n_blocks) {
    __shared__ int ok_flag;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const uint32_t gen = ld_acquire(&bar[1]);
        const uint32_t arrived = atom_add_acq_rel(&bar[0], 1u);
        if (arrived == n_blocks - 1) {
            bar[0] = 0u;
            st_release(&bar[1], gen + 1u);
        } else {
            uint32_t spins = 0;
            const uint32_t limit = spin_limit();
            while (ld_acquire(&bar[1]) == gen) {
                if (++spins > limit) {
                    raise_error(DYPH_ERR_TIMEOUT, 3u);
                    ok = 0;
                    break;
                }
                if ((spins & 1023u) == 0u && ld_acquire(&g_device_error) == DYPH_ERR_TIMEOUT) {
                    ok = 0;
                    break;
                }
                // back-off keeps hundreds of pollers from starving the arrivals
                __nanosleep(32);
            }
        }
        ok_flag = ok;
    }
    __syncthreads();
    return ok_flag != 0;
}

}  // namespace dyph

namespace dyph {
// The CUDA error behind the calling thread's last DYPH_ERR_CUDA
// (dyph_last_cuda_error).
inline thread_local cudaError_t t_last_cuda_error = cudaSuccess;
}  // namespace dyph

#define DYPH_CUDA_TRY(expr)                                   \
    do {                                                      \
        cudaError_t _e = (expr);                              \
        if (_e != cudaSuccess) {                              \
            dyph::t_last_cuda_error = _e;                     \
            return DYPH_ERR_CUDA;                             \
        }                                                     \
    } while (0)
