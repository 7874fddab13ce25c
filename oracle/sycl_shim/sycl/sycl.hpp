// Host-only stand-in for the subset of SYCL 2020 used by dyphur's frame-step
// sources (core/src/{body_store,shapes,contact_store,integrator,broadphase,
// narrowphase,xpbd_solver}.cpp and compute/include/compute/*.hpp).
//
// TEST INFRASTRUCTURE ONLY. This header exists so that the reference's own
// sources can be compiled unmodified with g++/OpenMP into oracle/_ref/, where
// they serve as the parity checker and as the timed CPU baseline. Nothing in
// the shipped library includes it.
//
// Semantics chosen to match a SYCL CPU device:
//   * queue is in-order and synchronous: every submission has completed when
//     the call returns, so event::wait() is a no-op.
//   * parallel_for(range) runs as an OpenMP parallel loop.
//   * device::is_gpu() is false, so compute/sort.hpp takes its multi-launch
//     bitonic path (the work-group-local path is never executed here).
//   * sycl::half is _Float16; float -> half conversion rounds to nearest even.
//   * rsqrt(x) = 1 / sqrt(x) with both operations correctly rounded.
#pragma once

#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace sycl {

using half = _Float16;

namespace access {
enum class address_space { global_space, local_space, constant_space, private_space, generic_space };
enum class fence_space { local_space, global_space, global_and_local };
}  // namespace access

enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };

template <int D = 1>
struct id {
    size_t v[D > 0 ? D : 1]{};
    id() = default;
    id(size_t i) { v[0] = i; }
    size_t operator[](int i) const { return v[i]; }
    operator size_t() const { return v[0]; }
};

template <int D = 1>
struct range {
    size_t v[D > 0 ? D : 1]{};
    range(size_t n) { v[0] = n; }
    size_t operator[](int i) const { return v[i]; }
    size_t size() const { return v[0]; }
};

template <int D = 1>
struct nd_range {
    range<D> global, local;
    nd_range(range<D> g, range<D> l) : global(g), local(l) {}
};

struct group_t {
    size_t idx = 0;
    operator size_t() const { return idx; }
};

template <int D = 1>
struct nd_item {
    size_t gid = 0, lid = 0, grp = 0;
    size_t get_global_id(int) const { return gid; }
    size_t get_local_id(int) const { return lid; }
    size_t get_group(int) const { return grp; }
    group_t get_group() const { return group_t{grp}; }
    void barrier(access::fence_space = access::fence_space::global_and_local) const {}
};

inline void group_barrier(group_t) {}

class event {
public:
    void wait() {}
    void wait_and_throw() {}
};

namespace info {
namespace device {
struct name {};
struct max_compute_units {};
struct global_mem_size {};
}  // namespace device
}  // namespace info

struct gpu_selector_t {};
struct cpu_selector_t {};
inline constexpr gpu_selector_t gpu_selector_v{};
inline constexpr cpu_selector_t cpu_selector_v{};

class device {
public:
    device() = default;
    explicit device(cpu_selector_t) {}
    explicit device(gpu_selector_t) { throw std::runtime_error("host SYCL shim: no GPU device"); }
    bool is_gpu() const { return false; }
    bool is_cpu() const { return true; }
    template <typename Param>
    auto get_info() const {
        if constexpr (std::is_same_v<Param, info::device::name>) {
            return std::string("host-shim-openmp");
        } else if constexpr (std::is_same_v<Param, info::device::max_compute_units>) {
            return size_t(1);
        } else {
            return size_t(0);
        }
    }
};

namespace property {
namespace queue {
struct in_order {};
}  // namespace queue
}  // namespace property

template <typename T, int D = 1>
class local_accessor {
public:
    template <typename H>
    local_accessor(range<D> r, H&) : data_(std::make_shared<std::vector<T>>(r.size())) {}
    T& operator[](size_t i) const { return (*data_)[i]; }

private:
    std::shared_ptr<std::vector<T>> data_;
};

class handler {
public:
    // The nd_range form is only reached on a GPU device (work-group-local
    // bitonic sort) or by reduce_sum, neither of which the frame step uses on
    // this host device. Running it without real barriers would be wrong, so
    // refuse loudly instead.
    template <int D, typename K>
    void parallel_for(nd_range<D>, K) {
        throw std::runtime_error("host SYCL shim: nd_range kernels are not supported");
    }
    template <typename K>
    void parallel_for(range<1> r, K k) {
        const long long n = static_cast<long long>(r.size());
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < n; ++i) k(id<1>(static_cast<size_t>(i)));
    }
};

class queue {
public:
    queue() = default;
    queue(const device& d, property::queue::in_order) : dev_(d) {}
    explicit queue(const device& d) : dev_(d) {}

    event memcpy(void* dst, const void* src, size_t bytes) {
        if (bytes) std::memcpy(dst, src, bytes);
        return {};
    }
    event memset(void* dst, int v, size_t bytes) {
        if (bytes) std::memset(dst, v, bytes);
        return {};
    }
    template <typename K>
    event parallel_for(range<1> r, K k) {
        const long long n = static_cast<long long>(r.size());
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < n; ++i) k(id<1>(static_cast<size_t>(i)));
        return {};
    }
    template <typename F>
    event submit(F f) {
        handler h;
        f(h);
        return {};
    }
    device get_device() const { return dev_; }
    void wait() {}
    void wait_and_throw() {}

private:
    device dev_;
};

template <typename T>
T* malloc_device(size_t n, const queue&) {
    size_t bytes = (n * sizeof(T) + 63) / 64 * 64;
    if (bytes == 0) bytes = 64;
    return static_cast<T*>(std::aligned_alloc(64, bytes));
}
inline void free(void* p, const queue&) { std::free(p); }

template <typename T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::global_space>
class atomic_ref {
public:
    explicit atomic_ref(T& r) : p_(&r) {}
    T fetch_add(T v) const { return __atomic_fetch_add(p_, v, __ATOMIC_SEQ_CST); }
    T fetch_sub(T v) const { return __atomic_fetch_sub(p_, v, __ATOMIC_SEQ_CST); }
    T fetch_or(T v) const { return __atomic_fetch_or(p_, v, __ATOMIC_SEQ_CST); }
    T fetch_max(T v) const {
        T cur = __atomic_load_n(p_, __ATOMIC_SEQ_CST);
        while (cur < v && !__atomic_compare_exchange_n(p_, &cur, v, false, __ATOMIC_SEQ_CST,
                                                       __ATOMIC_SEQ_CST)) {
        }
        return cur;
    }
    T load() const { return __atomic_load_n(p_, __ATOMIC_SEQ_CST); }
    void store(T v) const { __atomic_store_n(p_, v, __ATOMIC_SEQ_CST); }

private:
    T* p_;
};

// ── math ─────────────────────────────────────────────────────────────────────
inline float fabs(float x) { return std::fabs(x); }
inline float fmin(float a, float b) { return std::fmin(a, b); }
inline float fmax(float a, float b) { return std::fmax(a, b); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float atan(float x) { return std::atan(x); }
inline float atan2(float y, float x) { return std::atan2(y, x); }
inline double fabs(double x) { return std::fabs(x); }
inline double sqrt(double x) { return std::sqrt(x); }

inline uint64_t clz(uint64_t x) { return x ? static_cast<uint64_t>(__builtin_clzll(x)) : 64u; }
inline uint32_t clz(uint32_t x) { return x ? static_cast<uint32_t>(__builtin_clz(x)) : 32u; }
inline int64_t clz(int64_t x) { return static_cast<int64_t>(clz(static_cast<uint64_t>(x))); }
inline int32_t clz(int32_t x) { return static_cast<int32_t>(clz(static_cast<uint32_t>(x))); }

}  // namespace sycl
