// Stable LSD radix sort by key (8-bit digits), replacing the reference's
// bitonic sort_by_key / sort (compute/include/compute/sort.hpp:29-137).
//
// Large inputs: one histogram kernel for all digit passes, then one onesweep
// pass kernel per digit: each 2048-key tile ranks its keys with warp
// match-any, finds its global offset per digit by decoupled look-back over the
// preceding tiles, and scatters. Small inputs (<= 4096 keys): one thread
// block sorts in shared memory with all passes in one launch.
//
// Keys of the frame step are distinct, so the stable ascending order equals
// the reference's bitonic order element for element.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "sort.cuh"

namespace dyph {
namespace {

constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;  // 2048
constexpr int kWarps = kThreads / 32;
constexpr int kMaxPasses = 8;

constexpr int kSmallThreads = 1024;
constexpr int kSmallItems = 4;
constexpr int kSmallMax = kSmallThreads * kSmallItems;  // 4096
constexpr int kSmallWarps = kSmallThreads / 32;

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
    return static_cast<uint32_t>((k >> shift) & static_cast<K>(0xFF));
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename K>
__global__ void __launch_bounds__(kThreads) histogram_kernel(const K* __restrict__ keys, size_t n, int passes,
                                                             uint32_t* __restrict__ hist) {
    __shared__ uint32_t sh[kMaxPasses * 256];
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) sh[i] = 0u;
    __syncthreads();
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        K k = keys[i];
        for (int p = 0; p < passes; ++p) atomicAdd(&sh[p * 256 + digit_of(k, 8 * p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Thread-level decoupled look-back for one digit column.
__device__ __forceinline__ uint32_t lookback_column(uint32_t* status, uint32_t tile, uint32_t col, uint32_t agg) {
    if (tile == 0) {
        st_release(&status[col], kLbPrefix | agg);
        return 0u;
    }
    st_release(&status[static_cast<size_t>(tile) * 256 + col], kLbAgg | agg);
    uint32_t excl = 0;
    int64_t t = static_cast<int64_t>(tile) - 1;
    uint32_t spins = 0;
    while (t >= 0) {
        uint32_t s = ld_acquire(&status[static_cast<size_t>(t) * 256 + col]);
        uint32_t flag = s & ~kLbMask;
        if (flag == 0u) {
            if (++spins > spin_limit()) {
                raise_error(DYPH_ERR_TIMEOUT, 2u);
                return 0u;
            }
            __nanosleep(32);
            continue;
        }
        excl += s & kLbMask;
        if (flag == kLbPrefix) break;
        --t;
    }
    st_release(&status[static_cast<size_t>(tile) * 256 + col], kLbPrefix | ((excl + agg) & kLbMask));
    return excl;
}

template <typename K, bool HAS_VAL>
__global__ void __launch_bounds__(kThreads) onesweep_kernel(const K* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                            K* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            size_t n, int shift, const uint32_t* __restrict__ hist,
                                                            uint32_t* status, uint32_t* tile_ctr) {
    __shared__ uint32_t s_warp[kWarps][256];
    __shared__ uint32_t s_base[256];
    __shared__ uint32_t s_scan[kWarps];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(tile_ctr, 1u);
    for (int i = tid; i < kWarps * 256; i += kThreads) (&s_warp[0][0])[i] = 0u;
    __syncthreads();
    const uint32_t tile = s_tile;
    const size_t base = static_cast<size_t>(tile) * kTile + static_cast<size_t>(warp) * 32 * kItems;

    K k[kItems];
    uint32_t v[kItems], d[kItems], rank[kItems];
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        size_t idx = base + static_cast<size_t>(i) * 32 + lane;
        bool ok = idx < n;
        k[i] = ok ? kin[idx] : K(0);
        if (HAS_VAL) v[i] = ok ? vin[idx] : 0u;
        d[i] = ok ? digit_of(k[i], shift) : 0xFFFFFFFFu;
    }
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        uint32_t peers = __match_any_sync(0xffffffffu, d[i]);
        if (d[i] != 0xFFFFFFFFu) {
            uint32_t before = s_warp[warp][d[i]];
            rank[i] = before + __popc(peers & lt);
            __syncwarp(peers);
            if ((peers & lt) == 0u) s_warp[warp][d[i]] = before + __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    // Per digit: exclusive scan across warps, tile aggregate, look-back.
    {
        const uint32_t dg = static_cast<uint32_t>(tid);  // kThreads == 256 digits
        uint32_t sum = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            uint32_t c = s_warp[w][dg];
            s_warp[w][dg] = sum;
            sum += c;
        }
        uint32_t excl_tiles = lookback_column(status, tile, dg, sum);
        uint32_t total;
        uint32_t gexcl = block_exclusive_scan<kThreads>(hist[dg], s_scan, total);
        s_base[dg] = gexcl + excl_tiles;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kItems; ++i) {
        if (d[i] == 0xFFFFFFFFu) continue;
        uint32_t pos = s_base[d[i]] + s_warp[warp][d[i]] + rank[i];
        kout[pos] = k[i];
        if (HAS_VAL) vout[pos] = v[i];
    }
}

// Single-block sort for n <= kSmallMax. Dynamic shared memory:
// 2 key buffers, 2 value buffers, per-warp digit counters.
template <typename K, bool HAS_VAL>
__global__ void __launch_bounds__(kSmallThreads) small_sort_kernel(K* __restrict__ keys, uint32_t* __restrict__ vals,
                                                                   uint32_t n, int passes) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K* kb0 = reinterpret_cast<K*>(smem_raw);
    K* kb1 = kb0 + kSmallMax;
    uint32_t* vb0 = reinterpret_cast<uint32_t*>(kb1 + kSmallMax);
    uint32_t* vb1 = vb0 + (HAS_VAL ? kSmallMax : 0);
    uint32_t* cnt = vb1 + (HAS_VAL ? kSmallMax : 0);  // [kSmallWarps][256]
    __shared__ uint32_t s_scan[kSmallWarps];
    __shared__ uint32_t s_digit_base[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (uint32_t i = tid; i < n; i += kSmallThreads) {
        kb0[i] = keys[i];
        if (HAS_VAL) vb0[i] = vals[i];
    }
    __syncthreads();
    K* kin = kb0; K* kout = kb1;
    uint32_t* vin = vb0; uint32_t* vout = vb1;
    const uint32_t lt = lanemask_lt();
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        for (int i = tid; i < kSmallWarps * 256; i += kSmallThreads) cnt[i] = 0u;
        __syncthreads();
        K k[kSmallItems];
        uint32_t v[kSmallItems], d[kSmallItems], rank[kSmallItems];
#pragma unroll
        for (int i = 0; i < kSmallItems; ++i) {
            uint32_t idx = static_cast<uint32_t>(warp) * 32 * kSmallItems + i * 32 + lane;
            bool ok = idx < n;
            k[i] = ok ? kin[idx] : K(0);
            if (HAS_VAL) v[i] = ok ? vin[idx] : 0u;
            d[i] = ok ? digit_of(k[i], shift) : 0xFFFFFFFFu;
        }
#pragma unroll
        for (int i = 0; i < kSmallItems; ++i) {
            uint32_t peers = __match_any_sync(0xffffffffu, d[i]);
            if (d[i] != 0xFFFFFFFFu) {
                uint32_t before = cnt[warp * 256 + d[i]];
                rank[i] = before + __popc(peers & lt);
                __syncwarp(peers);
                if ((peers & lt) == 0u) cnt[warp * 256 + d[i]] = before + __popc(peers);
            }
            __syncwarp();
        }
        __syncthreads();
        uint32_t total_d = 0;
        if (tid < 256) {
            uint32_t sum = 0;
            for (int w = 0; w < kSmallWarps; ++w) {
                uint32_t c = cnt[w * 256 + tid];
                cnt[w * 256 + tid] = sum;
                sum += c;
            }
            total_d = sum;
        }
        uint32_t tot;
        uint32_t ex = block_exclusive_scan<kSmallThreads>(tid < 256 ? total_d : 0u, s_scan, tot);
        if (tid < 256) s_digit_base[tid] = ex;
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kSmallItems; ++i) {
            if (d[i] == 0xFFFFFFFFu) continue;
            uint32_t pos = s_digit_base[d[i]] + cnt[warp * 256 + d[i]] + rank[i];
            kout[pos] = k[i];
            if (HAS_VAL) vout[pos] = v[i];
        }
        __syncthreads();
        K* tk = kin; kin = kout; kout = tk;
        uint32_t* tv = vin; vin = vout; vout = tv;
    }
    for (uint32_t i = tid; i < n; i += kSmallThreads) {
        keys[i] = kin[i];
        if (HAS_VAL) vals[i] = vin[i];
    }
}

template <typename K, bool HAS_VAL>
size_t small_smem_bytes() {
    return 2 * kSmallMax * sizeof(K) + (HAS_VAL ? 2 * kSmallMax * 4 : 0) + kSmallWarps * 256 * 4;
}

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

template <typename K>
size_t ws_bytes(size_t n, int passes) {
    size_t tiles = (n + kTile - 1) / kTile;
    size_t b = align256(kMaxPasses * 256 * 4) + align256(kMaxPasses * 4) + align256(passes * tiles * 256 * 4);
    b += align256(n * sizeof(K)) + align256(n * 4);
    return b;
}

template <typename K, bool HAS_VAL>
dyph_status radix_sort(K* keys, uint32_t* vals, size_t n, int key_bits, void* ws, size_t ws_size,
                       cudaStream_t s) {
    if (n <= 1) return DYPH_OK;
    if (!keys || (HAS_VAL && !vals) || key_bits <= 0 || key_bits > 8 * static_cast<int>(sizeof(K)))
        return DYPH_ERR_INVALID;
    if (n >= (static_cast<size_t>(1) << 30)) return DYPH_ERR_INVALID;
    const int passes = (key_bits + 7) / 8;
    if (n <= static_cast<size_t>(kSmallMax)) {
        size_t smem = small_smem_bytes<K, HAS_VAL>();
        dyph_status ps = sort_prepare();
        if (ps != DYPH_OK) return ps;
        small_sort_kernel<K, HAS_VAL><<<1, kSmallThreads, smem, s>>>(keys, vals, static_cast<uint32_t>(n), passes);
        DYPH_CUDA_TRY(cudaGetLastError());
        return DYPH_OK;
    }
    if (!ws || ws_size < ws_bytes<K>(n, passes)) return DYPH_ERR_INVALID;
    const size_t tiles = (n + kTile - 1) / kTile;
    unsigned char* p = static_cast<unsigned char*>(ws);
    uint32_t* hist = reinterpret_cast<uint32_t*>(p);
    p += align256(kMaxPasses * 256 * 4);
    uint32_t* ctr = reinterpret_cast<uint32_t*>(p);
    p += align256(kMaxPasses * 4);
    uint32_t* status = reinterpret_cast<uint32_t*>(p);
    p += align256(passes * tiles * 256 * 4);
    K* kalt = reinterpret_cast<K*>(p);
    p += align256(n * sizeof(K));
    uint32_t* valt = reinterpret_cast<uint32_t*>(p);
    const size_t zero_bytes = static_cast<size_t>(reinterpret_cast<unsigned char*>(kalt) -
                                                  static_cast<unsigned char*>(ws));
    DYPH_CUDA_TRY(cudaMemsetAsync(ws, 0, zero_bytes, s));
    int hist_blocks = static_cast<int>(std::min<size_t>((n + 4095) / 4096, 592));
    histogram_kernel<K><<<hist_blocks, kThreads, 0, s>>>(keys, n, passes, hist);
    DYPH_CUDA_TRY(cudaGetLastError());
    K* ksrc = keys; K* kdst = kalt;
    uint32_t* vsrc = vals; uint32_t* vdst = valt;
    for (int pz = 0; pz < passes; ++pz) {
        onesweep_kernel<K, HAS_VAL><<<static_cast<unsigned>(tiles), kThreads, 0, s>>>(
            ksrc, vsrc, kdst, vdst, n, 8 * pz, hist + pz * 256, status + static_cast<size_t>(pz) * tiles * 256,
            ctr + pz);
        DYPH_CUDA_TRY(cudaGetLastError());
        std::swap(ksrc, kdst);
        std::swap(vsrc, vdst);
    }
    if (ksrc != keys) {
        DYPH_CUDA_TRY(cudaMemcpyAsync(keys, ksrc, n * sizeof(K), cudaMemcpyDeviceToDevice, s));
        if (HAS_VAL) DYPH_CUDA_TRY(cudaMemcpyAsync(vals, vsrc, n * 4, cudaMemcpyDeviceToDevice, s));
    }
    return DYPH_OK;
}

}  // namespace

// The dynamic shared memory opt-in of the one-block sorts, set once per
// device (a function attribute is per device).
constexpr int kSortMaxDevices = 64;
bool g_sort_configured[kSortMaxDevices] = {};
std::mutex g_sort_configured_mu;

dyph_status sort_prepare() {
    int dev = 0;
    DYPH_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kSortMaxDevices) return DYPH_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_sort_configured_mu);
    if (g_sort_configured[dev]) return DYPH_OK;
    DYPH_CUDA_TRY(cudaFuncSetAttribute(small_sort_kernel<uint32_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(small_smem_bytes<uint32_t, true>())));
    DYPH_CUDA_TRY(cudaFuncSetAttribute(small_sort_kernel<uint64_t, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(small_smem_bytes<uint64_t, true>())));
    DYPH_CUDA_TRY(cudaFuncSetAttribute(small_sort_kernel<uint64_t, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(small_smem_bytes<uint64_t, false>())));
    g_sort_configured[dev] = true;
    return DYPH_OK;
}

size_t sort_workspace_bytes(size_t n, int key_bytes) {
    return key_bytes == 8 ? ws_bytes<uint64_t>(n, 8) : ws_bytes<uint32_t>(n, 4);
}

dyph_status sort_u32_u32(uint32_t* keys, uint32_t* vals, size_t n, int key_bits, void* ws, size_t ws_size,
                         cudaStream_t s) {
    return radix_sort<uint32_t, true>(keys, vals, n, key_bits, ws, ws_size, s);
}

dyph_status sort_u64_u32(uint64_t* keys, uint32_t* vals, size_t n, int key_bits, void* ws, size_t ws_size,
                         cudaStream_t s) {
    return radix_sort<uint64_t, true>(keys, vals, n, key_bits, ws, ws_size, s);
}

}  // namespace dyph

extern "C" size_t dyph_sort_workspace_bytes(size_t n) { return dyph::sort_workspace_bytes(n, 8); }

extern "C" dyph_status dyph_sort_by_key_u64_u32(uint64_t* keys, uint32_t* values, size_t n, void* ws,
                                                size_t ws_bytes, dyph_stream s) {
    return dyph::radix_sort<uint64_t, true>(keys, values, n, 64, ws, ws_bytes, reinterpret_cast<cudaStream_t>(s));
}

extern "C" dyph_status dyph_sort_u64(uint64_t* keys, size_t n, void* ws, size_t ws_bytes, dyph_stream s) {
    return dyph::radix_sort<uint64_t, false>(keys, nullptr, n, 64, ws, ws_bytes, reinterpret_cast<cudaStream_t>(s));
}

extern "C" dyph_status dyph_sort_by_key_u32_u32(uint32_t* keys, uint32_t* values, size_t n, int key_bits,
                                                void* ws, size_t ws_bytes, dyph_stream s) {
    return dyph::radix_sort<uint32_t, true>(keys, values, n, key_bits, ws, ws_bytes,
                                            reinterpret_cast<cudaStream_t>(s));
}

// ── sort with library-owned scratch ─────────────────────────────────────────
// The scratch is a file-scope device array sized for DYPH_SORT_NOALLOC_MAX_KEYS
// 64-bit keys with 32-bit values: histograms, pass counters and look-back
// status (cleared on the stream by every call), then the alternate key and
// value buffers. Nothing here calls cudaMalloc or cudaFree.
namespace dyph {
namespace {

constexpr size_t kNoAllocMaxKeys = DYPH_SORT_NOALLOC_MAX_KEYS;
constexpr size_t round256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }
constexpr size_t kNoAllocTiles = (kNoAllocMaxKeys + kTile - 1) / kTile;
constexpr size_t kNoAllocScratchBytes = round256(kMaxPasses * 256 * 4) + round256(kMaxPasses * 4) +
                                        round256(kMaxPasses * kNoAllocTiles * 256 * 4) +
                                        round256(kNoAllocMaxKeys * 8) + round256(kNoAllocMaxKeys * 4);

static __device__ __align__(256) unsigned char g_sort_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
void* g_sort_scratch_ptr[kNoAllocMaxDevices] = {};
std::mutex g_sort_scratch_mu;

// Per-device set-up, done by the first call with that device current: the
// array's device address and the small-sort kernel's shared-memory attribute.
dyph_status noalloc_scratch(void** out) {
    int dev = 0;
    DYPH_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return DYPH_ERR_INVALID;
    std::lock_guard<std::mutex> lock(g_sort_scratch_mu);
    if (!g_sort_scratch_ptr[dev]) {
        void* p = nullptr;
        DYPH_CUDA_TRY(cudaGetSymbolAddress(&p, g_sort_scratch));
        DYPH_CUDA_TRY(cudaFuncSetAttribute(small_sort_kernel<uint64_t, true>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           static_cast<int>(small_smem_bytes<uint64_t, true>())));
        g_sort_scratch_ptr[dev] = p;
    }
    *out = g_sort_scratch_ptr[dev];
    return DYPH_OK;
}

}  // namespace
}  // namespace dyph

extern "C" dyph_status dyph_sort_by_key_u64_u32_noalloc(uint64_t* keys, uint32_t* values, size_t n, dyph_stream s) {
    if (n > dyph::kNoAllocMaxKeys) return DYPH_ERR_TOO_LARGE;
    if (n <= 1) return DYPH_OK;
    if (!keys || !values) return DYPH_ERR_INVALID;
    void* scratch = nullptr;
    const dyph_status st = dyph::noalloc_scratch(&scratch);
    if (st != DYPH_OK) return st;
    if (dyph::ws_bytes<uint64_t>(n, 8) > dyph::kNoAllocScratchBytes) return DYPH_ERR_TOO_LARGE;
    return dyph::radix_sort<uint64_t, true>(keys, values, n, 64, scratch, dyph::kNoAllocScratchBytes,
                                            reinterpret_cast<cudaStream_t>(s));
}
