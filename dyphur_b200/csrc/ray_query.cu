// Queries over the frame's products: batched ray casts against the LBVH and
// the per-shape contact filter.
//
//   dyph_ray_query      ray_query (core/src/ray_query.cpp:126-195): closest
//                       hit of each ray, LBVH walk over the fp16 node boxes,
//                       exact sphere / oriented-box test at the leaves.
//   dyph_contact_sensor ContactSensor::query (core/src/contact_sensor.cpp:6-59):
//                       the contacts whose body a or b has a given shape, in
//                       store order. The filter runs on the device (one pass,
//                       tile look-back compaction) and only the matches cross
//                       to the host.
//
// The ray walk keeps the reference's visiting order (a 64-entry stack, right
// child pushed before left, node box tested when popped) and its float
// expressions, so hits and tie-breaks are identical, not just close.
#include <algorithm>
#include <new>

#include "common.cuh"

namespace dyph {
namespace {

constexpr int kRayThreads = 128;
constexpr int kRayStack = 64;  // ray_query.cpp:173

// Slab test against a node box (ray_query.cpp:14-33).
__device__ __forceinline__ bool ray_node_hit(float ox, float oy, float oz, float ix, float iy, float iz,
                                             float mnx, float mny, float mnz, float mxx, float mxy, float mxz,
                                             float best_t) {
    const float t1x = (mnx - ox) * ix, t2x = (mxx - ox) * ix;
    const float t1y = (mny - oy) * iy, t2y = (mxy - oy) * iy;
    const float t1z = (mnz - oz) * iz, t2z = (mxz - oz) * iz;
    float tmin = t1x < t2x ? t1x : t2x;
    float tmax = t1x < t2x ? t2x : t1x;
    const float ylo = t1y < t2y ? t1y : t2y, yhi = t1y < t2y ? t2y : t1y;
    tmin = tmin > ylo ? tmin : ylo;
    tmax = tmax < yhi ? tmax : yhi;
    const float zlo = t1z < t2z ? t1z : t2z, zhi = t1z < t2z ? t2z : t1z;
    tmin = tmin > zlo ? tmin : zlo;
    tmax = tmax < zhi ? tmax : zhi;
    return tmax >= 0.f && tmax >= tmin && tmin < best_t;
}

// v rotated by the conjugate of (w, x, y, z): t = 2 (u x v), v + w t + u x t
// with u = (-x, -y, -z) (Quat::rotate, core/include/core/math/quat.hpp:39-42).
__device__ __forceinline__ void rotate_conj(float w, float x, float y, float z, float vx, float vy, float vz,
                                            float& rx, float& ry, float& rz) {
    const float ux = -x, uy = -y, uz = -z;
    const float tx = (uy * vz - uz * vy) * 2.f;
    const float ty = (uz * vx - ux * vz) * 2.f;
    const float tz = (ux * vy - uy * vx) * 2.f;
    rx = (vx + tx * w) + (uy * tz - uz * ty);
    ry = (vy + ty * w) + (uz * tx - ux * tz);
    rz = (vz + tz * w) + (ux * ty - uy * tx);
}

// Oriented box in the body frame; t or -1 (ray_query.cpp:37-73).
__device__ __forceinline__ float ray_box(float ox, float oy, float oz, float dx, float dy, float dz, float px,
                                         float py, float pz, float qw, float qx, float qy, float qz, float hx,
                                         float hy, float hz, float best_t) {
    float lox, loy, loz, ldx, ldy, ldz;
    rotate_conj(qw, qx, qy, qz, ox - px, oy - py, oz - pz, lox, loy, loz);
    rotate_conj(qw, qx, qy, qz, dx, dy, dz, ldx, ldy, ldz);
    const float ix = 1.f / ldx, iy = 1.f / ldy, iz = 1.f / ldz;
    const float t1x = (-hx - lox) * ix, t2x = (hx - lox) * ix;
    const float t1y = (-hy - loy) * iy, t2y = (hy - loy) * iy;
    const float t1z = (-hz - loz) * iz, t2z = (hz - loz) * iz;
    float tmin = t1x < t2x ? t1x : t2x;
    float tmax = t1x < t2x ? t2x : t1x;
    const float ylo = t1y < t2y ? t1y : t2y, yhi = t1y < t2y ? t2y : t1y;
    tmin = tmin > ylo ? tmin : ylo;
    tmax = tmax < yhi ? tmax : yhi;
    const float zlo = t1z < t2z ? t1z : t2z, zhi = t1z < t2z ? t2z : t1z;
    tmin = tmin > zlo ? tmin : zlo;
    tmax = tmax < zhi ? tmax : zhi;
    if (tmax < 0.f || tmin > tmax) return -1.f;
    const float t = tmin >= 0.f ? tmin : tmax;
    return (t >= 0.f && t < best_t) ? t : -1.f;
}

// Sphere by the quadratic; t or -1 (ray_query.cpp:76-91).
__device__ __forceinline__ float ray_sphere(float ox, float oy, float oz, float dx, float dy, float dz, float cx,
                                            float cy, float cz, float r, float best_t) {
    const float ocx = ox - cx, ocy = oy - cy, ocz = oz - cz;
    const float a = dx * dx + dy * dy + dz * dz;
    const float b = dx * ocx + dy * ocy + dz * ocz;
    const float c = ocx * ocx + ocy * ocy + ocz * ocz - r * r;
    const float disc = b * b - a * c;
    if (disc < 0.f) return -1.f;
    const float sq = __fsqrt_rn(disc);
    float t = (-b - sq) / a;
    if (t < 0.f) t = (-b + sq) / a;
    return (t >= 0.f && t < best_t) ? t : -1.f;
}

struct RayScene {
    dyph_bodies b;
    dyph_shapes sh;
};

__device__ __forceinline__ void ray_leaf(const RayScene& S, uint32_t bi, const dyph_ray& r, float& best_t,
                                         uint32_t& best_body) {
    const uint32_t shape = __ldg(&S.b.shape[bi]);
    const float hx = __ldg(&S.sh.half_x[shape]);
    float t;
    if (__ldg(&S.sh.type[shape]) == kShapeSphere) {
        t = ray_sphere(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, S.b.pos_x[bi], S.b.pos_y[bi], S.b.pos_z[bi], hx, best_t);
    } else {
        // Every other shape type is cast as its box (ray_query.cpp:113-118).
        t = ray_box(r.ox, r.oy, r.oz, r.dx, r.dy, r.dz, S.b.pos_x[bi], S.b.pos_y[bi], S.b.pos_z[bi], S.b.rot_w[bi],
                    S.b.rot_x[bi], S.b.rot_y[bi], S.b.rot_z[bi], hx, __ldg(&S.sh.half_y[shape]),
                    __ldg(&S.sh.half_z[shape]), best_t);
    }
    if (t >= 0.f) {
        best_t = t;
        best_body = bi;
    }
}

__global__ void __launch_bounds__(kRayThreads) ray_query_kernel(dyph_bvh_view bvh, RayScene S,
                                                                const dyph_ray* __restrict__ rays,
                                                                dyph_ray_hit* __restrict__ hits, uint32_t n_rays) {
    const uint32_t idx = blockIdx.x * kRayThreads + threadIdx.x;
    if (idx >= n_rays) return;
    const dyph_ray r = rays[idx];
    float best_t = r.t_max;
    uint32_t best_body = 0xFFFFFFFFu;
    const float ix = 1.f / r.dx, iy = 1.f / r.dy, iz = 1.f / r.dz;
    if (bvh.n == 1u) {
        // A one-body build has no tree (broadphase.cpp returns early): body 0.
        ray_leaf(S, 0u, r, best_t, best_body);
    } else if (bvh.n > 1u) {
        int32_t stack[kRayStack];
        int top = 0;
        stack[top++] = __ldg(bvh.root);
        const int32_t n_int = static_cast<int32_t>(bvh.n - 1u);
        const uint4* boxes = reinterpret_cast<const uint4*>(bvh.aabb);
        while (top > 0) {
            const int32_t node = stack[--top];
            const uint4 nb = __ldg(&boxes[node]);
            if (!ray_node_hit(r.ox, r.oy, r.oz, ix, iy, iz, h2f_bits(nb.x & 0xFFFFu), h2f_bits(nb.x >> 16),
                              h2f_bits(nb.y & 0xFFFFu), h2f_bits(nb.y >> 16), h2f_bits(nb.z & 0xFFFFu),
                              h2f_bits(nb.z >> 16), best_t))
                continue;
            if (node >= n_int) {
                ray_leaf(S, __ldg(&bvh.sorted_idx[node - n_int]), r, best_t, best_body);
            } else if (top + 1 < kRayStack) {
                stack[top++] = __ldg(&bvh.right[node]);
                stack[top++] = __ldg(&bvh.left[node]);
            }
        }
    }
    hits[idx] = dyph_ray_hit{best_t, best_body};
}

// ── contact sensor ──────────────────────────────────────────────────────────

constexpr int kSensorThreads = 256;
constexpr int kSensorRows = 9;  // body_a, body_b, pos xyz, normal xyz, depth

__global__ void __launch_bounds__(kSensorThreads) sensor_filter_kernel(dyph_contacts in,
                                                                       const uint32_t* __restrict__ body_shape,
                                                                       uint32_t n_bodies, uint32_t shape_idx,
                                                                       uint32_t* __restrict__ out, uint32_t cap,
                                                                       uint32_t* __restrict__ counts,
                                                                       uint32_t* __restrict__ status) {
    __shared__ uint32_t s_tile, s_excl;
    __shared__ uint32_t s_scan[kSensorThreads / 32];
    const uint32_t nc = min(*in.n, in.capacity);
    const uint32_t n_tiles = (nc + kSensorThreads - 1) / kSensorThreads;
    if (nc == 0u) {
        if (blockIdx.x == 0 && threadIdx.x == 0) counts[0] = 0u;
        return;
    }
    while (true) {
        if (threadIdx.x == 0) s_tile = atomicAdd(&counts[1], 1u);
        __syncthreads();
        const uint32_t tile = s_tile;
        if (tile >= n_tiles) break;
        const uint32_t i = tile * kSensorThreads + threadIdx.x;
        bool keep = false;
        uint32_t a = 0, b = 0;
        if (i < nc) {
            a = in.body_a[i];
            b = in.body_b[i];
            keep = (a < n_bodies && __ldg(&body_shape[a]) == shape_idx) ||
                   (b < n_bodies && __ldg(&body_shape[b]) == shape_idx);
        }
        uint32_t total;
        const uint32_t excl = block_exclusive_scan<kSensorThreads>(keep ? 1u : 0u, s_scan, total);
        if (threadIdx.x < 32) {
            const uint32_t e = lookback_warp(status, tile, total);
            if (threadIdx.x == 0) {
                s_excl = e;
                if (tile == n_tiles - 1) counts[0] = e + total;
            }
        }
        __syncthreads();
        if (keep) {
            const uint32_t pos = s_excl + excl;
            if (pos < cap) {
                const float row[7] = {in.pos_x[i], in.pos_y[i], in.pos_z[i], in.norm_x[i],
                                      in.norm_y[i], in.norm_z[i], in.depth[i]};
                out[pos] = a;
                out[static_cast<size_t>(cap) + pos] = b;
#pragma unroll
                for (int k = 0; k < 7; ++k) out[static_cast<size_t>(2 + k) * cap + pos] = __float_as_uint(row[k]);
            }
        }
        __syncthreads();
    }
}

int sensor_blocks() {
    static int blocks = 0;
    if (blocks == 0) {
        int dev = 0, sms = 148, per_sm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sensor_filter_kernel, kSensorThreads, 0);
        blocks = sms * std::max(1, std::min(per_sm, 8));
    }
    return blocks;
}

}  // namespace
}  // namespace dyph

struct dyph_contact_sensor {
    uint32_t shape_idx = 0;
    uint32_t cap = 0;             // rows of the device and host match buffers
    uint32_t* d_rows = nullptr;   // [9][cap] matches in store order
    uint32_t* counts = nullptr;   // [0] matches, [1] tile counter
    uint32_t* status = nullptr;   // look-back status per 256-contact tile
    uint32_t status_words = 0;
    uint32_t* h_rows = nullptr;   // pinned host copy of the matches
    uint32_t count = 0;           // matches of the last query
};

using namespace dyph;

extern "C" dyph_status dyph_ray_query(const dyph_bvh_view* bvh, const dyph_bodies* bodies, const dyph_shapes* shapes,
                                      const dyph_ray* d_rays, dyph_ray_hit* d_hits, uint32_t n_rays, dyph_stream s) {
    if (n_rays == 0) return DYPH_OK;
    if (!bvh || !bodies || !shapes || !d_rays || !d_hits) return DYPH_ERR_INVALID;
    if (bvh->n > 1u && (!bvh->root || !bvh->left || !bvh->right || !bvh->sorted_idx || !bvh->aabb))
        return DYPH_ERR_INVALID;
    if (bvh->n > bodies->n) return DYPH_ERR_INVALID;
    const uint32_t grid = (n_rays + kRayThreads - 1) / kRayThreads;
    ray_query_kernel<<<grid, kRayThreads, 0, reinterpret_cast<cudaStream_t>(s)>>>(*bvh, RayScene{*bodies, *shapes},
                                                                                   d_rays, d_hits, n_rays);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

extern "C" dyph_status dyph_contact_sensor_create(uint32_t shape_idx, dyph_contact_sensor** out) {
    if (!out) return DYPH_ERR_INVALID;
    auto* cs = new (std::nothrow) dyph_contact_sensor();
    if (!cs) return DYPH_ERR_NOMEM;
    cs->shape_idx = shape_idx;
    if (cudaMalloc(&cs->counts, 2 * sizeof(uint32_t)) != cudaSuccess) {
        delete cs;
        return DYPH_ERR_NOMEM;
    }
    *out = cs;
    return DYPH_OK;
}

extern "C" void dyph_contact_sensor_destroy(dyph_contact_sensor* cs) {
    if (!cs) return;
    if (cs->d_rows) cudaFree(cs->d_rows);
    if (cs->counts) cudaFree(cs->counts);
    if (cs->status) cudaFree(cs->status);
    if (cs->h_rows) cudaFreeHost(cs->h_rows);
    delete cs;
}

namespace {
dyph_status sensor_reserve(dyph_contact_sensor* cs, uint32_t capacity) {
    const uint32_t tiles = (capacity + kSensorThreads - 1) / kSensorThreads;
    if (tiles > cs->status_words) {
        if (cs->status) cudaFree(cs->status);
        cs->status = nullptr;
        cs->status_words = 0;
        if (cudaMalloc(&cs->status, std::max<size_t>(tiles, 1) * 4) != cudaSuccess) return DYPH_ERR_NOMEM;
        cs->status_words = tiles;
    }
    if (capacity > cs->cap) {
        if (cs->d_rows) cudaFree(cs->d_rows);
        if (cs->h_rows) cudaFreeHost(cs->h_rows);
        cs->d_rows = cs->h_rows = nullptr;
        cs->cap = 0;
        const size_t bytes = static_cast<size_t>(capacity) * kSensorRows * 4;
        if (cudaMalloc(&cs->d_rows, bytes) != cudaSuccess) return DYPH_ERR_NOMEM;
        if (cudaMallocHost(&cs->h_rows, bytes) != cudaSuccess) return DYPH_ERR_NOMEM;
        cs->cap = capacity;
    }
    return DYPH_OK;
}
}  // namespace

extern "C" dyph_status dyph_contact_sensor_filter(dyph_contact_sensor* cs, const dyph_contacts* contacts,
                                                  const uint32_t* d_body_shape, uint32_t n_bodies, dyph_stream s) {
    if (!cs || !contacts || !contacts->n || (n_bodies && !d_body_shape)) return DYPH_ERR_INVALID;
    const uint32_t capacity = std::max(contacts->capacity, 1u);
    dyph_status rs = sensor_reserve(cs, capacity);
    if (rs != DYPH_OK) return rs;
    cudaStream_t cs_ = reinterpret_cast<cudaStream_t>(s);
    const uint32_t tiles = (capacity + kSensorThreads - 1) / kSensorThreads;
    DYPH_CUDA_TRY(cudaMemsetAsync(cs->status, 0, static_cast<size_t>(tiles) * 4, cs_));
    DYPH_CUDA_TRY(cudaMemsetAsync(cs->counts, 0, 2 * sizeof(uint32_t), cs_));
    sensor_filter_kernel<<<sensor_blocks(), kSensorThreads, 0, cs_>>>(*contacts, d_body_shape, n_bodies,
                                                                       cs->shape_idx, cs->d_rows, cs->cap,
                                                                       cs->counts, cs->status);
    DYPH_CUDA_TRY(cudaGetLastError());
    return DYPH_OK;
}

extern "C" dyph_status dyph_contact_sensor_query(dyph_contact_sensor* cs, const dyph_contacts* contacts,
                                                 const uint32_t* d_body_shape, uint32_t n_bodies, dyph_stream s,
                                                 uint32_t* out_count) {
    dyph_status rs = dyph_contact_sensor_filter(cs, contacts, d_body_shape, n_bodies, s);
    if (rs != DYPH_OK) return rs;
    cudaStream_t cs_ = reinterpret_cast<cudaStream_t>(s);
    uint32_t m = 0;
    DYPH_CUDA_TRY(cudaMemcpyAsync(&m, cs->counts, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs_));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs_));
    m = std::min(m, cs->cap);
    // Nine row copies of the matches only (one stream, one wait).
    for (int k = 0; k < kSensorRows && m > 0; ++k)
        DYPH_CUDA_TRY(cudaMemcpyAsync(cs->h_rows + static_cast<size_t>(k) * cs->cap,
                                      cs->d_rows + static_cast<size_t>(k) * cs->cap, static_cast<size_t>(m) * 4,
                                      cudaMemcpyDeviceToHost, cs_));
    DYPH_CUDA_TRY(cudaStreamSynchronize(cs_));
    cs->count = m;
    if (out_count) *out_count = m;
    return DYPH_OK;
}

extern "C" uint32_t dyph_contact_sensor_count(const dyph_contact_sensor* cs) { return cs ? cs->count : 0u; }
extern "C" uint32_t dyph_contact_sensor_shape_idx(const dyph_contact_sensor* cs) { return cs ? cs->shape_idx : 0u; }

namespace {
void sensor_view(uint32_t* rows, uint32_t cap, uint32_t* n, dyph_contacts* out) {
    auto row = [&](int k) { return rows ? rows + static_cast<size_t>(k) * cap : nullptr; };
    out->body_a = row(0);
    out->body_b = row(1);
    out->pos_x = reinterpret_cast<float*>(row(2));
    out->pos_y = reinterpret_cast<float*>(row(3));
    out->pos_z = reinterpret_cast<float*>(row(4));
    out->norm_x = reinterpret_cast<float*>(row(5));
    out->norm_y = reinterpret_cast<float*>(row(6));
    out->norm_z = reinterpret_cast<float*>(row(7));
    out->depth = reinterpret_cast<float*>(row(8));
    out->n = n;
    out->capacity = cap;
}
}  // namespace

extern "C" dyph_status dyph_contact_sensor_host_view(dyph_contact_sensor* cs, dyph_contacts* out) {
    if (!cs || !out) return DYPH_ERR_INVALID;
    sensor_view(cs->h_rows, cs->cap, &cs->count, out);
    return DYPH_OK;
}

extern "C" dyph_status dyph_contact_sensor_device_view(dyph_contact_sensor* cs, dyph_contacts* out) {
    if (!cs || !out) return DYPH_ERR_INVALID;
    sensor_view(cs->d_rows, cs->cap, cs->counts, out);
    return DYPH_OK;
}
