// Symplectic Euler integration (core/src/integrator.cpp:7-71) and the
// library-level C entry points (status strings, device check, error word).
#include <algorithm>

#include <cuda_runtime.h>

#include "internal.cuh"

namespace dyph {
namespace {

constexpr int kIntThreads = 256;

// One body per thread; the substep loop stays in registers, which gives the
// same values as the reference's one launch per substep.
__global__ void __launch_bounds__(kIntThreads) integrate_kernel(GlobalBodies B, float gx, float gy, float gz,
                                                                float sub_dt, float half_dt, int n_substeps) {
    const uint32_t n = B.v.n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (B.im(i) == 0.f) continue;
        if (B.v.flags[i] & kFlagSleeping) continue;
        Pose s{B.px(i), B.py(i), B.pz(i), B.qw(i), B.qx(i), B.qy(i), B.qz(i), B.vx(i), B.vy(i), B.vz(i)};
        const float ox = B.wx(i), oy = B.wy(i), oz = B.wz(i);
        for (int k = 0; k < n_substeps; ++k) integrate_body(s, ox, oy, oz, gx, gy, gz, sub_dt, half_dt);
        B.px(i) = s.px; B.py(i) = s.py; B.pz(i) = s.pz;
        B.qw(i) = s.qw; B.qx(i) = s.qx; B.qy(i) = s.qy; B.qz(i) = s.qz;
        B.vx(i) = s.vx; B.vy(i) = s.vy; B.vz(i) = s.vz;
    }
}

}  // namespace

dyph_status integrate_launch(const dyph_bodies* bodies, const dyph_integrator_params* p, cudaStream_t s) {
    if (!bodies || !p || p->n_substeps <= 0) return DYPH_ERR_INVALID;
    if (bodies->n == 0) return DYPH_OK;
    const float sub_dt = p->dt / static_cast<float>(p->n_substeps);
    const float half_dt = 0.5f * sub_dt;
    const unsigned blocks = (bodies->n + kIntThreads - 1) / kIntThreads;
    integrate_kernel<<<blocks, kIntThreads, 0, s>>>(GlobalBodies{*bodies}, p->gravity[0], p->gravity[1],
                                                    p->gravity[2], sub_dt, half_dt, p->n_substeps);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

// ── diagnostics ─────────────────────────────────────────────────────────────

// Smallest index of a body with a NaN / Inf in its 13 state floats.
__global__ void finite_kernel(dyph_bodies b, uint32_t* __restrict__ first_bad) {
    const float* rows[13] = {b.pos_x, b.pos_y, b.pos_z, b.rot_w, b.rot_x, b.rot_y, b.rot_z,
                             b.vel_x, b.vel_y, b.vel_z, b.ang_x, b.ang_y, b.ang_z};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < b.n; i += gridDim.x * blockDim.x) {
        bool ok = true;
#pragma unroll
        for (int r = 0; r < 13; ++r) ok = ok && isfinite(rows[r][i]);
        if (!ok) atomicMin(first_bad, i);
    }
}

// A wait that nothing ends: which 1 = the look-back of tile 1 on a tile 0 that
// never publishes (site 1), which 3 = a grid barrier of two blocks launched
// as one (site 3). Each gives up after the spin limit and the kernel returns.
__device__ uint32_t g_selftest_words[4];

__global__ void wait_selftest_kernel(int which) {
    if (which == 1) {
        if (threadIdx.x < 32) lookback_warp(g_selftest_words, 1u, 7u);
    } else {
        grid_barrier(g_selftest_words + 2, 2u);
    }
}

}  // namespace dyph

extern "C" dyph_status dyph_set_spin_limit(uint32_t limit) {
    const uint32_t v = limit ? limit : dyph::kSpinLimit;
    DYPH_CUDA_TRY(cudaMemcpyToSymbol(dyph::g_spin_limit, &v, sizeof(v)));
    return DYPH_OK;
}

extern "C" dyph_status dyph_wait_selftest(int which, dyph_stream s) {
    if (which != 1 && which != 3) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    void* words = nullptr;
    DYPH_CUDA_TRY(cudaGetSymbolAddress(&words, dyph::g_selftest_words));
    DYPH_CUDA_TRY(cudaMemsetAsync(words, 0, 4 * sizeof(uint32_t), cs));
    dyph::wait_selftest_kernel<<<1, 32, 0, cs>>>(which);
    DYPH_CUDA_TRY(cudaGetLastError());
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

extern "C" dyph_status dyph_bodies_check_finite(const dyph_bodies* bodies, dyph_stream s, uint32_t* out_first_bad) {
    if (!bodies) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t first = 0xFFFFFFFFu;
    if (bodies->n > 0) {
        uint32_t* d = nullptr;
        DYPH_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&d), sizeof(uint32_t), cs));
        DYPH_CUDA_TRY(cudaMemsetAsync(d, 0xFF, sizeof(uint32_t), cs));
        const uint32_t blocks = std::min<uint32_t>((bodies->n + 255) / 256, 148u * 8u);
        dyph::finite_kernel<<<blocks, 256, 0, cs>>>(*bodies, d);
        DYPH_CUDA_TRY(cudaGetLastError());
        DYPH_CUDA_TRY(cudaMemcpyAsync(&first, d, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs));
        DYPH_CUDA_TRY(cudaFreeAsync(d, cs));
        DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    }
    if (out_first_bad) *out_first_bad = first;
    return first == 0xFFFFFFFFu ? DYPH_OK : DYPH_ERR_NOT_FINITE;
}

extern "C" dyph_status dyph_integrate(const dyph_bodies* bodies, const dyph_integrator_params* params,
                                      dyph_stream s) {
    return dyph::integrate_launch(bodies, params, reinterpret_cast<cudaStream_t>(s));
}

extern "C" const char* dyph_status_string(int status) {
    switch (status) {
        case DYPH_OK: return "ok";
        case DYPH_ERR_INVALID: return "invalid argument";
        case DYPH_ERR_CUDA: return "CUDA runtime error";
        case DYPH_ERR_PAIR_OVERFLOW: return "candidate pairs exceeded capacity";
        case DYPH_ERR_CONTACT_OVERFLOW: return "contacts exceeded capacity";
        case DYPH_ERR_TIMEOUT: return "bounded device wait timed out";
        case DYPH_ERR_NO_DEVICE: return "no sm_100 CUDA device";
        case DYPH_ERR_NOMEM: return "device allocation failed";
        case DYPH_ERR_NOT_FINITE: return "non-finite body state";
        case DYPH_ERR_TOO_LARGE: return "size exceeds the fixed scratch of a no-allocation entry point";
        case DYPH_ERR_UNSUPPORTED: return "a frame took a path the adjoint does not differentiate";
        default: return "unknown status";
    }
}

extern "C" const char* dyph_last_cuda_error(void) {
    return cudaGetErrorString(dyph::t_last_cuda_error);
}

extern "C" dyph_status dyph_device_check(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return DYPH_ERR_NO_DEVICE;
    }
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DYPH_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess)
        return DYPH_ERR_NO_DEVICE;
    return major == 10 ? DYPH_OK : DYPH_ERR_NO_DEVICE;
}

extern "C" dyph_status dyph_copy_to_host(void* host_dst, const void* dev_src, size_t bytes, dyph_stream s) {
    if (bytes == 0) return DYPH_OK;
    if (!host_dst || !dev_src) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaMemcpyAsync(host_dst, dev_src, bytes, cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

extern "C" dyph_status dyph_copy_to_device(void* dev_dst, const void* host_src, size_t bytes, dyph_stream s) {
    if (bytes == 0) return DYPH_OK;
    if (!dev_dst || !host_src) return DYPH_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    DYPH_CUDA_TRY(cudaMemcpyAsync(dev_dst, host_src, bytes, cudaMemcpyHostToDevice, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    return DYPH_OK;
}

extern "C" dyph_status dyph_download_device_error_site(dyph_stream s, uint32_t* out_code, uint32_t* out_site) {
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(s);
    uint32_t h[2] = {0, 0};
    const uint32_t zero = 0;
    DYPH_CUDA_TRY(cudaMemcpyFromSymbolAsync(&h[0], dyph::g_device_error, sizeof(uint32_t), 0, cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaMemcpyFromSymbolAsync(&h[1], dyph::g_device_error_site, sizeof(uint32_t), 0,
                                            cudaMemcpyDeviceToHost, cs));
    DYPH_CUDA_TRY(cudaMemcpyToSymbolAsync(dyph::g_device_error_site, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, cs));
    DYPH_CUDA_TRY(cudaMemcpyToSymbolAsync(dyph::g_device_error, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, cs));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs));
    if (out_code) *out_code = h[0];
    if (out_site) *out_site = h[1];
    return DYPH_OK;
}

extern "C" dyph_status dyph_download_device_error(dyph_stream s, uint32_t* out_code) {
    return dyph_download_device_error_site(s, out_code, nullptr);
}
