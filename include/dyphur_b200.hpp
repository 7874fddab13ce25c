// C++20 class layer over the C ABI, mirroring the reference's compute/ and
// core/ surface so host code written against it keeps compiling:
//   Device / Stream / Event / Buffer<T>      compute/include/compute/{device,stream,buffer}.hpp
//   sort_by_key / sort                       compute/include/compute/sort.hpp:29,88
//   BodyStore / ShapeStore                   core/include/core/{body_store,shape_store}.hpp
//   integrate                                core/include/core/integrator.hpp:25
//   Broadphase / Narrowphase / XpbdSolver    core/include/core/{broadphase,narrowphase,xpbd_solver}.hpp
// The views (BodyView, ShapeView, ContactView, ContactPair, AABB) are the C
// ABI's structs, which have the reference's field order. Errors throw
// std::runtime_error where the reference throws (SYCL exceptions, no GPU);
// there is no CPU device. Link with libdyphur_b200.so and the CUDA runtime.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dyphur_b200.h"

namespace dyphur {

inline void check(dyph_status st, const char* what) {
    if (st != DYPH_OK) throw std::runtime_error(std::string(what) + ": " + dyph_status_string(st));
}
inline void check_cuda(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

using BodyView = dyph_bodies;
using ShapeView = dyph_shapes;
using ContactView = dyph_contacts;
using ContactPair = dyph_pair;
using AABB = dyph_aabb;
using BvhView = dyph_bvh_view;

// ── compute ─────────────────────────────────────────────────────────────────

class Event {
public:
    Event() = default;
    explicit Event(cudaStream_t s) {
        check_cuda(cudaEventCreateWithFlags(&e_, cudaEventDisableTiming), "cudaEventCreate");
        check_cuda(cudaEventRecord(e_, s), "cudaEventRecord");
    }
    ~Event() {
        if (e_) cudaEventDestroy(e_);
    }
    Event(const Event&) = delete;
    Event& operator=(const Event&) = delete;
    Event(Event&& o) noexcept : e_(std::exchange(o.e_, nullptr)) {}
    Event& operator=(Event&& o) noexcept {
        std::swap(e_, o.e_);
        return *this;
    }
    void wait() {
        if (e_) check_cuda(cudaEventSynchronize(e_), "Event::wait");
    }

private:
    cudaEvent_t e_ = nullptr;
};

// In-order queue of one device (the reference's in-order sycl::queue).
class Stream {
public:
    explicit Stream(int device) : dev_(device) {
        check_cuda(cudaSetDevice(device), "cudaSetDevice");
        check_cuda(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "cudaStreamCreate");
    }
    ~Stream() {
        if (s_) cudaStreamDestroy(s_);
    }
    Stream(const Stream&) = delete;
    Stream& operator=(const Stream&) = delete;
    Stream(Stream&& o) noexcept : dev_(o.dev_), s_(std::exchange(o.s_, nullptr)) {}
    void wait() { check_cuda(cudaStreamSynchronize(s_), "Stream::wait"); }
    cudaStream_t native() const noexcept { return s_; }
    dyph_stream abi() const noexcept { return reinterpret_cast<dyph_stream>(s_); }
    int device() const noexcept { return dev_; }

private:
    int dev_ = 0;
    cudaStream_t s_ = nullptr;
};

class Device {
public:
    explicit Device(int ordinal) : dev_(ordinal) {}
    // Throws when no sm_100 device is present (the reference throws from its selector).
    static Device default_gpu() {
        check(dyph_device_check(), "Device::default_gpu");
        int d = 0;
        check_cuda(cudaGetDevice(&d), "cudaGetDevice");
        return Device(d);
    }
    // There is no CPU device: the name is kept so host code written against
    // the reference compiles and runs unchanged, and it selects the default GPU.
    static Device default_cpu() { return default_gpu(); }
    static Device preferred() { return default_gpu(); }
    std::string name() const {
        cudaDeviceProp p{};
        check_cuda(cudaGetDeviceProperties(&p, dev_), "cudaGetDeviceProperties");
        return p.name;
    }
    bool is_gpu() const { return true; }
    bool is_cpu() const { return false; }
    size_t max_compute_units() const {
        int v = 0;
        check_cuda(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev_), "attribute");
        return static_cast<size_t>(v);
    }
    size_t global_mem_bytes() const {
        cudaDeviceProp p{};
        check_cuda(cudaGetDeviceProperties(&p, dev_), "cudaGetDeviceProperties");
        return p.totalGlobalMem;
    }
    Stream make_stream() const { return Stream(dev_); }
    int ordinal() const noexcept { return dev_; }

private:
    int dev_ = 0;
};

// Move-only device array (compute/include/compute/buffer.hpp:10-55).
template <typename T>
class Buffer {
public:
    Buffer() = default;
    Buffer(Stream& s, size_t n) : s_(&s), n_(n) {
        if (n > 0) check_cuda(cudaMalloc(reinterpret_cast<void**>(&data_), n * sizeof(T)), "Buffer");
    }
    ~Buffer() {
        if (data_) cudaFree(data_);
    }
    Buffer(const Buffer&) = delete;
    Buffer& operator=(const Buffer&) = delete;
    Buffer(Buffer&& o) noexcept : s_(o.s_), n_(std::exchange(o.n_, 0)), data_(std::exchange(o.data_, nullptr)) {}
    Buffer& operator=(Buffer&& o) noexcept {
        if (this != &o) {
            if (data_) cudaFree(data_);
            s_ = o.s_;
            n_ = std::exchange(o.n_, 0);
            data_ = std::exchange(o.data_, nullptr);
        }
        return *this;
    }
    T* data() noexcept { return data_; }
    const T* data() const noexcept { return data_; }
    size_t size() const noexcept { return n_; }
    bool empty() const noexcept { return n_ == 0; }
    Event upload(const T* src, size_t count = 0) {
        check_cuda(cudaMemcpyAsync(data_, src, (count ? count : n_) * sizeof(T), cudaMemcpyHostToDevice,
                                   s_->native()),
                   "Buffer::upload");
        return Event(s_->native());
    }
    void download(T* dst, size_t count = 0) const {
        check(dyph_copy_to_host(dst, data_, (count ? count : n_) * sizeof(T), s_->abi()), "Buffer::download");
    }

private:
    Stream* s_ = nullptr;
    size_t n_ = 0;
    T* data_ = nullptr;
};

// Stable ascending sorts; unlike the reference, n need not be a power of two.
inline void sort_by_key(Stream& s, uint64_t* keys, uint32_t* values, size_t n) {
    Buffer<uint8_t> ws(s, dyph_sort_workspace_bytes(n));
    check(dyph_sort_by_key_u64_u32(keys, values, n, ws.data(), ws.size(), s.abi()), "sort_by_key");
    s.wait();  // the workspace is freed on return
}
inline void sort_by_key(Stream& s, uint32_t* keys, uint32_t* values, size_t n) {
    Buffer<uint8_t> ws(s, dyph_sort_workspace_bytes(n));
    check(dyph_sort_by_key_u32_u32(keys, values, n, 32, ws.data(), ws.size(), s.abi()), "sort_by_key");
    s.wait();
}
inline void sort(Stream& s, uint64_t* keys, size_t n) {
    Buffer<uint8_t> ws(s, dyph_sort_workspace_bytes(n));
    check(dyph_sort_u64(keys, n, ws.data(), ws.size(), s.abi()), "sort");
    s.wait();
}

// ── core ────────────────────────────────────────────────────────────────────

constexpr uint32_t kBodyStatic = 1u;  // BodyFlag::Static (core/include/core/body.hpp:9)

// BodyParams (core/include/core/body.hpp:16-25) with plain arrays for the math types.
struct BodyParams {
    float position[3] = {0.f, 0.f, 0.f};
    float rotation[4] = {1.f, 0.f, 0.f, 0.f};  // w, x, y, z
    float linear_velocity[3] = {0.f, 0.f, 0.f};
    float angular_velocity[3] = {0.f, 0.f, 0.f};
    float mass = 1.f;
    float inertia[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};  // row-major, body frame
    uint32_t shape_handle = 0;
    uint32_t flags = 0;
};

// core/include/core/body_store.hpp:21-73. add() inverts the inertia on the
// host in float exactly as the reference's Mat3::inverse does.
class BodyStore {
public:
    BodyStore(Stream& s, uint32_t capacity) : s_(&s), cap_(capacity), d_f_(s, size_t(20) * capacity),
                                             d_u_(s, size_t(2) * capacity) {}
    uint32_t add(const BodyParams& p) {
        if (count_ >= cap_) throw std::runtime_error("BodyStore::add: capacity exceeded");
        h_.push_back(p);
        h_shape_.push_back(p.shape_handle);
        return count_++;
    }
    // Shape index of every body added so far (body_store.hpp:48).
    const std::vector<uint32_t>& body_shapes() const noexcept { return h_shape_; }
    // Blocking copies of the 13 state rows (pos xyz, rot wxyz, vel xyz, ang
    // xyz), [13][count] floats, out of / into the device arrays.
    void download_state(float* host13) {
        for (int r = 0; r < 13; ++r)
            check(dyph_copy_to_host(host13 + size_t(r) * count_, d_f_.data() + size_t(r) * cap_, count_ * 4,
                                    s_->abi()),
                  "BodyStore::download_state");
    }
    void upload_state(const float* host13) {
        for (int r = 0; r < 13; ++r)
            check(dyph_copy_to_device(d_f_.data() + size_t(r) * cap_, host13 + size_t(r) * count_, count_ * 4,
                                      s_->abi()),
                  "BodyStore::upload_state");
    }
    // The 20 float rows ([20][capacity]: state, inverse mass, inverse inertia).
    float* device_rows() noexcept { return d_f_.data(); }
    void upload() {
        const uint32_t n = count_;
        std::vector<float> pos(3 * n), rot(4 * n), vel(3 * n), ang(3 * n), mass(n), inertia(9 * n);
        std::vector<uint32_t> flags(n), shape(n), flags_out(n);
        for (uint32_t i = 0; i < n; ++i) {
            const BodyParams& p = h_[i];
            for (int k = 0; k < 3; ++k) {
                pos[3 * i + k] = p.position[k];
                vel[3 * i + k] = p.linear_velocity[k];
                ang[3 * i + k] = p.angular_velocity[k];
            }
            for (int k = 0; k < 4; ++k) rot[4 * i + k] = p.rotation[k];
            for (int k = 0; k < 9; ++k) inertia[9 * i + k] = p.inertia[k];
            mass[i] = p.mass;
            flags[i] = p.flags;
            shape[i] = p.shape_handle;
        }
        // rows 0..12 state, 13 inverse mass, 14..19 inverse inertia, each `cap` long
        std::vector<float> st(size_t(13) * n), im(n), ii(size_t(6) * n);
        dyph_pack_bodies(n, pos.data(), rot.data(), vel.data(), ang.data(), mass.data(), inertia.data(),
                         flags.data(), st.data(), im.data(), ii.data(), flags_out.data());
        for (int r = 0; r < 13; ++r) copy_row(r, st.data() + size_t(r) * n, n);
        copy_row(13, im.data(), n);
        for (int r = 0; r < 6; ++r) copy_row(14 + r, ii.data() + size_t(r) * n, n);
        check_cuda(cudaMemcpyAsync(d_u_.data(), shape.data(), n * 4, cudaMemcpyHostToDevice, s_->native()), "upload");
        check_cuda(cudaMemcpyAsync(d_u_.data() + cap_, flags_out.data(), n * 4, cudaMemcpyHostToDevice,
                                   s_->native()),
                   "upload");
        s_->wait();
    }
    BodyView view() noexcept {
        float* f = d_f_.data();
        auto row = [&](int r) { return f + size_t(r) * cap_; };
        return BodyView{row(0),  row(1),  row(2),  row(3),  row(4),  row(5),  row(6),
                        row(7),  row(8),  row(9),  row(10), row(11), row(12), row(13),
                        row(14), row(15), row(16), row(17), row(18), row(19), d_u_.data(),
                        d_u_.data() + cap_, count_};
    }
    uint32_t count() const noexcept { return count_; }
    uint32_t capacity() const noexcept { return cap_; }

private:
    void copy_row(int r, const float* src, uint32_t n) {
        check_cuda(cudaMemcpyAsync(d_f_.data() + size_t(r) * cap_, src, n * 4, cudaMemcpyHostToDevice, s_->native()),
                   "upload");
    }
    Stream* s_;
    uint32_t cap_, count_ = 0;
    Buffer<float> d_f_;
    Buffer<uint32_t> d_u_;
    std::vector<BodyParams> h_;
    std::vector<uint32_t> h_shape_;
};

// ShapeParams / ShapeStore (core/include/core/shapes.hpp, shape_store.hpp):
// boxes (half extents) and spheres (radius in half_x).
enum class ShapeType : uint32_t { Box = 0, Sphere = 1 };
struct ShapeParams {
    ShapeType type = ShapeType::Box;
    float half_x = 0.5f, half_y = 0.5f, half_z = 0.5f;
};

class ShapeStore {
public:
    ShapeStore(Stream& s, uint32_t capacity)
        : s_(&s), cap_(capacity), d_type_(s, capacity), d_half_(s, size_t(3) * capacity), d_ext_(s, capacity) {}
    uint32_t add(const ShapeParams& p) {
        if (count_ >= cap_) throw std::runtime_error("ShapeStore::add: capacity exceeded");
        h_.push_back(p);
        return count_++;
    }
    void upload() {
        std::vector<uint32_t> type(count_), ext(count_, 0u);
        std::vector<float> half(size_t(3) * cap_, 0.f);
        for (uint32_t i = 0; i < count_; ++i) {
            type[i] = static_cast<uint32_t>(h_[i].type);
            half[i] = h_[i].half_x;
            half[cap_ + i] = h_[i].half_y;
            half[2 * size_t(cap_) + i] = h_[i].half_z;
        }
        if (count_) {
            d_type_.upload(type.data(), count_);
            d_ext_.upload(ext.data(), count_);
        }
        d_half_.upload(half.data());
        s_->wait();
    }
    ShapeView view() noexcept {
        return ShapeView{d_type_.data(), d_half_.data(), d_half_.data() + cap_, d_half_.data() + 2 * size_t(cap_),
                         d_ext_.data(), count_};
    }
    uint32_t count() const noexcept { return count_; }
    uint32_t capacity() const noexcept { return cap_; }

private:
    Stream* s_;
    uint32_t cap_, count_ = 0;
    Buffer<uint32_t> d_type_;
    Buffer<float> d_half_;
    Buffer<uint32_t> d_ext_;
    std::vector<ShapeParams> h_;
};

struct IntegratorParams {
    float gravity[3] = {0.f, -9.81f, 0.f};
    float dt = 1.f / 60.f;
    int32_t n_substeps = 1;
};

inline void integrate(Stream& s, BodyView bodies, const IntegratorParams& p) {
    const dyph_integrator_params c{{p.gravity[0], p.gravity[1], p.gravity[2]}, p.dt, p.n_substeps};
    check(dyph_integrate(&bodies, &c, s.abi()), "integrate");
}

class Broadphase {
public:
    Broadphase(Stream& s, uint32_t max_bodies, uint32_t max_pairs) {
        (void)s;
        check(dyph_broadphase_create(max_bodies, max_pairs, &h_), "Broadphase");
    }
    ~Broadphase() { dyph_broadphase_destroy(h_); }
    Broadphase(const Broadphase&) = delete;
    Broadphase& operator=(const Broadphase&) = delete;
    void build_and_query(Stream& s, const BodyView& bodies, const ShapeView& shapes, const AABB& scene_bounds) {
        check(dyph_broadphase_build_and_query(h_, &bodies, &shapes, &scene_bounds, s.abi()), "build_and_query");
    }
    const ContactPair* pairs_ptr() const noexcept { return dyph_broadphase_pairs(h_); }
    const uint32_t* count_ptr() const noexcept { return dyph_broadphase_count_ptr(h_); }
    uint32_t max_pairs() const noexcept { return dyph_broadphase_max_pairs(h_); }
    void sort_pairs(Stream& s, uint32_t n_pairs) { check(dyph_broadphase_sort_pairs(h_, n_pairs, s.abi()), "sort_pairs"); }
    uint32_t download_count(Stream& s) const {
        uint32_t n = 0;
        check(dyph_broadphase_download_count(h_, s.abi(), &n), "download_count");
        return n;
    }
    BvhView bvh_view(uint32_t n_active) const {
        BvhView v{};
        check(dyph_broadphase_bvh_view(h_, n_active, &v), "bvh_view");
        return v;
    }

private:
    dyph_broadphase* h_ = nullptr;
};

class Narrowphase {
public:
    Narrowphase(Stream& s, uint32_t max_contacts) : cap_(max_contacts) {
        (void)s;
        check(dyph_narrowphase_create(max_contacts, &h_), "Narrowphase");
    }
    ~Narrowphase() { dyph_narrowphase_destroy(h_); }
    Narrowphase(const Narrowphase&) = delete;
    Narrowphase& operator=(const Narrowphase&) = delete;
    void run(Stream& s, const ContactPair* d_pairs, uint32_t n_pairs, const BodyView& bodies, const ShapeView& shapes) {
        check(dyph_narrowphase_run_host_count(h_, d_pairs, n_pairs, &bodies, &shapes, s.abi()), "Narrowphase::run");
        uint32_t stored = 0;
        check(dyph_narrowphase_download_count(h_, s.abi(), &stored, &last_count_), "download_count");
    }
    void run(Stream& s, const ContactPair* d_pairs, const uint32_t* d_n_pairs, const BodyView& bodies,
             const ShapeView& shapes) {
        check(dyph_narrowphase_run(h_, d_pairs, d_n_pairs, &bodies, &shapes, s.abi()), "Narrowphase::run");
    }
    ContactView contacts() const {
        ContactView v{};
        check(dyph_narrowphase_contacts(h_, &v), "contacts");
        return v;
    }
    uint32_t download_count(Stream& s) const {
        uint32_t stored = 0, total = 0;
        check(dyph_narrowphase_download_count(h_, s.abi(), &stored, &total), "download_count");
        return stored;
    }
    uint32_t last_contact_count() const noexcept { return last_count_; }
    bool overflowed() const noexcept { return last_count_ > cap_; }

private:
    dyph_narrowphase* h_ = nullptr;
    uint32_t cap_ = 0, last_count_ = 0;
};

class XpbdSolver {
public:
    static constexpr uint32_t kSerialThreshold = 256;  // xpbd_solver.hpp:43
    explicit XpbdSolver(Stream& s, int n_iters = 10, uint32_t max_contacts = 16384, float friction = 0.5f,
                        uint32_t max_bodies = 1u << 16) {
        (void)s;
        check(dyph_xpbd_create(n_iters, max_contacts, max_bodies, friction, &h_), "XpbdSolver");
    }
    ~XpbdSolver() { dyph_xpbd_destroy(h_); }
    XpbdSolver(const XpbdSolver&) = delete;
    XpbdSolver& operator=(const XpbdSolver&) = delete;
    // IConstraintSolver::solve (core/include/core/solver.hpp:17-21); no joints on this path.
    void solve(Stream& s, const ContactView& contacts, BodyView bodies, float dt) {
        check(dyph_xpbd_solve(h_, &contacts, &bodies, dt, s.abi()), "XpbdSolver::solve");
    }
    void set_force_serial(bool v) {
        check(dyph_xpbd_set_mode(h_, v ? DYPH_SOLVER_SEQUENTIAL : DYPH_SOLVER_REFERENCE), "set_force_serial");
    }

private:
    dyph_xpbd* h_ = nullptr;
};

// ── queries ─────────────────────────────────────────────────────────────────

// Ray / RayHit (core/include/core/ray_query.hpp:9-20), layout-identical to the C ABI's.
struct Ray {
    float ox = 0.f, oy = 0.f, oz = 0.f;
    float dx = 1.f, dy = 0.f, dz = 0.f;
    float t_max = 1e9f;
};
struct RayHit {
    float t;
    uint32_t body_idx;  // UINT32_MAX on a miss
};
static_assert(sizeof(Ray) == sizeof(dyph_ray) && sizeof(RayHit) == sizeof(dyph_ray_hit));

// ray_query (core/include/core/ray_query.hpp:34-40); d_rays / d_hits on the device.
inline void ray_query(Stream& s, const BvhView& bvh, const BodyView& bodies, const ShapeView& shapes,
                      const Ray* d_rays, RayHit* d_hits, uint32_t n_rays) {
    check(dyph_ray_query(&bvh, &bodies, &shapes, reinterpret_cast<const dyph_ray*>(d_rays),
                         reinterpret_cast<dyph_ray_hit*>(d_hits), n_rays, s.abi()),
          "ray_query");
}

// ContactSensor (core/include/core/contact_sensor.hpp:20-58). The filter runs
// on the device; query() blocks and leaves the matches in host arrays.
class ContactSensor {
public:
    explicit ContactSensor(uint32_t shape_idx) { check(dyph_contact_sensor_create(shape_idx, &h_), "ContactSensor"); }
    ~ContactSensor() { dyph_contact_sensor_destroy(h_); }
    ContactSensor(const ContactSensor&) = delete;
    ContactSensor& operator=(const ContactSensor&) = delete;
    uint32_t query(Stream& s, const Narrowphase& np, const std::vector<uint32_t>& body_shapes) {
        const uint32_t n = static_cast<uint32_t>(body_shapes.size());
        if (n > shapes_.size()) shapes_ = Buffer<uint32_t>(s, n);
        if (n) shapes_.upload(body_shapes.data(), n);
        ContactView cv = np.contacts();
        uint32_t m = 0;
        check(dyph_contact_sensor_query(h_, &cv, shapes_.data(), n, s.abi(), &m), "ContactSensor::query");
        check(dyph_contact_sensor_host_view(h_, &host_), "ContactSensor::query");
        return m;
    }
    uint32_t count() const noexcept { return dyph_contact_sensor_count(h_); }
    uint32_t shape_idx() const noexcept { return dyph_contact_sensor_shape_idx(h_); }
    const uint32_t* body_a() const noexcept { return host_.body_a; }
    const uint32_t* body_b() const noexcept { return host_.body_b; }
    const float* pos_x() const noexcept { return host_.pos_x; }
    const float* pos_y() const noexcept { return host_.pos_y; }
    const float* pos_z() const noexcept { return host_.pos_z; }
    const float* norm_x() const noexcept { return host_.norm_x; }
    const float* norm_y() const noexcept { return host_.norm_y; }
    const float* norm_z() const noexcept { return host_.norm_z; }
    const float* depth() const noexcept { return host_.depth; }

private:
    dyph_contact_sensor* h_ = nullptr;
    Buffer<uint32_t> shapes_;
    ContactView host_{};
};

// ── the whole frame step ────────────────────────────────────────────────────

// One scene (or a batch of scenes) stepped as examples/stress_test_blocks/
// main.cpp:264-279 does it, graph-replayed, over a BodyStore's device arrays.
class World {
public:
    World(Stream& s, BodyStore& bodies, ShapeStore& shapes, const AABB& scene_bounds,
          const IntegratorParams& ip = {}, uint32_t max_pairs = 0, uint32_t max_contacts = 0, int n_iters = 10,
          float friction = 0.5f, dyph_solver_mode mode = DYPH_SOLVER_REFERENCE)
        : bodies_(&bodies), initial_(s, size_t(13) * bodies.capacity()) {
        const uint32_t n = bodies.count();
        dyph_world_desc d{};
        d.bodies = bodies.view();
        d.shapes = shapes.view();
        d.scene_bounds = scene_bounds;
        d.integrator = dyph_integrator_params{{ip.gravity[0], ip.gravity[1], ip.gravity[2]}, ip.dt, ip.n_substeps};
        d.max_pairs = max_pairs ? max_pairs : 48 * n + 64;
        d.max_contacts = max_contacts ? max_contacts : 16 * n + 64;
        d.n_iters = n_iters;
        d.friction = friction;
        d.mode = mode;
        check(dyph_world_create(&d, s.abi(), &h_), "World");
        check_cuda(cudaMemcpyAsync(initial_.data(), bodies.device_rows(), initial_.size() * 4,
                                   cudaMemcpyDeviceToDevice, s.native()),
                   "World");
        s.wait();
    }
    ~World() { dyph_world_destroy(h_); }
    World(const World&) = delete;
    World& operator=(const World&) = delete;
    // Batched scenes: bodies [body_offset[k], body_offset[k+1]) form scene k.
    void set_scenes(const std::vector<uint32_t>& body_offset, const std::vector<AABB>& bounds) {
        if (body_offset.size() != bounds.size() + 1) throw std::runtime_error("World::set_scenes: sizes");
        check(dyph_world_set_scenes(h_, static_cast<uint32_t>(bounds.size()), body_offset.data(), bounds.data()),
              "World::set_scenes");
    }
    void step(Stream& s, int n_frames) { check(dyph_world_step(h_, n_frames, s.abi()), "World::step"); }
    // Checkpointed rollout and its adjoint (dyph_world_rollout / _backward).
    void rollout(Stream& s, int n_frames, int every, float* d_ckpt) {
        check(dyph_world_rollout(h_, n_frames, every, d_ckpt, s.abi()), "World::rollout");
    }
    void rollout_backward(Stream& s, int n_frames, int every, const float* d_ckpt, const float* d_grad_final,
                          float* d_grad_init, float* d_grad_inv_mass) {
        check(dyph_world_rollout_backward(h_, n_frames, every, d_ckpt, d_grad_final, d_grad_init, d_grad_inv_mass,
                                          s.abi()),
              "World::rollout_backward");
    }
    std::vector<uint64_t> scene_hashes(Stream& s, uint32_t n_scenes) {
        std::vector<uint64_t> out(n_scenes);
        check(dyph_world_scene_hashes(h_, s.abi(), out.data(), n_scenes), "World::scene_hashes");
        return out;
    }
    // Knobs of the fused batched frame (dyph_world_set_fused_config /
    // dyph_world_autotune); every setting gives the same frames.
    dyph_fused_config fused_config() {
        dyph_fused_config c{};
        check(dyph_world_fused_config(h_, &c), "World::fused_config");
        return c;
    }
    void set_fused_config(uint32_t smem_cap, uint32_t teams = 2, uint32_t register_blocks = 0) {
        check(dyph_world_set_fused_config(h_, smem_cap, teams, register_blocks), "World::set_fused_config");
    }
    dyph_fused_config autotune(Stream& s, int frames = 16) {
        dyph_fused_config c{};
        check(dyph_world_autotune(h_, frames, s.abi(), &c), "World::autotune");
        return c;
    }
    // The adjoint's reverse kernel layout (dyph_world_set_adjoint_config).
    dyph_fused_config adjoint_config() {
        dyph_fused_config c{};
        check(dyph_world_adjoint_config(h_, &c), "World::adjoint_config");
        return c;
    }
    void set_adjoint_config(uint32_t smem_bytes, uint32_t teams = 2) {
        check(dyph_world_set_adjoint_config(h_, smem_bytes, teams), "World::set_adjoint_config");
    }
    // State rows at creation ([13][capacity], device), the start of rollouts.
    const float* initial_rows() const noexcept { return initial_.data(); }
    BodyStore& bodies() noexcept { return *bodies_; }
    dyph_world* handle() noexcept { return h_; }

private:
    dyph_world* h_ = nullptr;
    BodyStore* bodies_;
    Buffer<float> initial_;
};

// FNV-1a-64 over pos_x..rot_z (examples/stress_test_blocks/main.cpp:34-41, 301-311).
inline uint64_t state_hash(Stream& s, const BodyView& bodies) {
    Buffer<uint64_t> h(s, 1);
    check(dyph_fnv1a64_state(&bodies, h.data(), s.abi()), "state_hash");
    uint64_t out = 0;
    h.download(&out, 1);
    return out;
}

}  // namespace dyphur
