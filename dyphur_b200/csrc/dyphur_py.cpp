// dyphur_py: the Python module of the reference's bindings
// (bindings/python/dyphur_py.cpp:29-163: Device, Stream, AABB, ShapeType,
// ShapeParams, ShapeStore, BodyParams, BodyStore, Broadphase, Narrowphase,
// ContactSensor) with the same class, method and argument names, built with
// pybind11 over the C++ layer of include/dyphur_b200.hpp. Added beyond the
// reference's surface: Device.default_gpu, ray_query, integrate, XpbdSolver,
// World (step, scene hashes, rollout and its adjoint) and zero-copy device
// views (__cuda_array_interface__) that torch.as_tensor wraps without a copy;
// dyphur_b200.autograd builds the differentiable rollout on them.
//
// Every array the sensor returns is a numpy view of its host buffer (no copy),
// kept alive by the sensor, as the reference's nanobind views are.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstdint>
#include <vector>

#include "dyphur_b200.hpp"

namespace py = pybind11;
using namespace pybind11::literals;
using namespace dyphur;

namespace {

// Device memory exposed through __cuda_array_interface__ (version 3).
struct DeviceArray {
    uintptr_t ptr = 0;
    std::vector<size_t> shape;
    std::string typestr;
    py::dict interface() const {
        py::dict d;
        d["shape"] = py::tuple(py::cast(shape));
        d["typestr"] = typestr;
        d["data"] = py::make_tuple(ptr, false);
        d["version"] = 3;
        d["strides"] = py::none();
        d["stream"] = py::none();
        return d;
    }
};

template <typename T>
py::array_t<T> host_view(const T* ptr, size_t n, py::handle owner) {
    return py::array_t<T>({n}, {sizeof(T)}, ptr, owner);
}

// Host (n, 7) rays -> device, query, device -> host (t, body).
py::tuple ray_query_host(Stream& s, const BvhView& bvh, const BodyView& bodies, const ShapeView& shapes,
                         py::array_t<float, py::array::c_style | py::array::forcecast> rays) {
    if (rays.ndim() != 2 || rays.shape(1) != 7) throw std::invalid_argument("rays must have shape (n, 7)");
    const uint32_t n = static_cast<uint32_t>(rays.shape(0));
    py::array_t<float> t(n);
    py::array_t<uint32_t> body(n);
    if (n == 0) return py::make_tuple(t, body);
    Buffer<Ray> d_rays(s, n);
    Buffer<RayHit> d_hits(s, n);
    d_rays.upload(reinterpret_cast<const Ray*>(rays.data()), n);
    ray_query(s, bvh, bodies, shapes, d_rays.data(), d_hits.data(), n);
    std::vector<RayHit> h(n);
    d_hits.download(h.data(), n);
    auto tt = t.mutable_unchecked<1>();
    auto bb = body.mutable_unchecked<1>();
    for (uint32_t k = 0; k < n; ++k) {
        tt(k) = h[k].t;
        bb(k) = h[k].body_idx;
    }
    return py::make_tuple(t, body);
}

}  // namespace

PYBIND11_MODULE(dyphur_py, m) {
    m.doc() = "dyphur rigid-body frame step on B200 (sm_100a): the reference's Python surface over libdyphur_b200";

    // ── device memory views ─────────────────────────────────────────────────
    py::class_<DeviceArray>(m, "DeviceArray")
        .def_readonly("ptr", &DeviceArray::ptr)
        .def_property_readonly("__cuda_array_interface__", &DeviceArray::interface);

    // ── Device / Stream ─────────────────────────────────────────────────────
    py::class_<Device>(m, "Device")
        .def_static("default_cpu", &Device::default_cpu,
                    "There is no CPU device: kept for scripts written against the reference; the default GPU.")
        .def_static("default_gpu", &Device::default_gpu)
        .def("make_stream", &Device::make_stream)
        .def("name", &Device::name)
        .def("is_gpu", &Device::is_gpu)
        .def("is_cpu", &Device::is_cpu)
        .def("max_compute_units", &Device::max_compute_units)
        .def("global_mem_bytes", &Device::global_mem_bytes);

    py::class_<Stream>(m, "Stream")
        .def("wait", &Stream::wait)
        .def_property_readonly("cuda_stream", [](const Stream& s) { return reinterpret_cast<uintptr_t>(s.native()); });

    // ── AABB ────────────────────────────────────────────────────────────────
    py::class_<AABB>(m, "AABB")
        .def(py::init([](float a, float b, float c, float d, float e, float f) { return AABB{a, b, c, d, e, f}; }),
             "min_x"_a, "min_y"_a, "min_z"_a, "max_x"_a, "max_y"_a, "max_z"_a)
        .def_readwrite("min_x", &AABB::min_x)
        .def_readwrite("min_y", &AABB::min_y)
        .def_readwrite("min_z", &AABB::min_z)
        .def_readwrite("max_x", &AABB::max_x)
        .def_readwrite("max_y", &AABB::max_y)
        .def_readwrite("max_z", &AABB::max_z);

    // ── Shape ───────────────────────────────────────────────────────────────
    py::enum_<ShapeType>(m, "ShapeType")
        .value("Box", ShapeType::Box)
        .value("Sphere", ShapeType::Sphere)
        .export_values();

    py::class_<ShapeParams>(m, "ShapeParams")
        .def(py::init<>())
        .def_readwrite("type", &ShapeParams::type)
        .def_readwrite("half_x", &ShapeParams::half_x)
        .def_readwrite("half_y", &ShapeParams::half_y)
        .def_readwrite("half_z", &ShapeParams::half_z);

    py::class_<ShapeView>(m, "ShapeView").def_readonly("n", &ShapeView::n);

    py::class_<ShapeStore>(m, "ShapeStore")
        .def(py::init<Stream&, uint32_t>(), "s"_a, "capacity"_a, py::keep_alive<1, 2>())
        .def("add", &ShapeStore::add)
        .def("upload", &ShapeStore::upload)
        .def("count", &ShapeStore::count)
        .def("view", &ShapeStore::view);

    // ── Body ────────────────────────────────────────────────────────────────
    py::class_<BodyParams>(m, "BodyParams")
        .def(py::init<>())
        .def("set_position", [](BodyParams& p, float x, float y, float z) {
            p.position[0] = x; p.position[1] = y; p.position[2] = z;
        }, "x"_a, "y"_a, "z"_a)
        .def("set_velocity", [](BodyParams& p, float vx, float vy, float vz) {
            p.linear_velocity[0] = vx; p.linear_velocity[1] = vy; p.linear_velocity[2] = vz;
        }, "vx"_a, "vy"_a, "vz"_a)
        .def("set_rotation", [](BodyParams& p, float w, float x, float y, float z) {
            p.rotation[0] = w; p.rotation[1] = x; p.rotation[2] = y; p.rotation[3] = z;
        }, "w"_a, "x"_a, "y"_a, "z"_a)
        .def("set_angular_velocity", [](BodyParams& p, float wx, float wy, float wz) {
            p.angular_velocity[0] = wx; p.angular_velocity[1] = wy; p.angular_velocity[2] = wz;
        }, "wx"_a, "wy"_a, "wz"_a)
        .def("set_inertia", [](BodyParams& p, const std::vector<float>& rows) {
            if (rows.size() != 9) throw std::invalid_argument("inertia takes 9 row-major values");
            for (int k = 0; k < 9; ++k) p.inertia[k] = rows[k];
        }, "rows"_a)
        .def_readwrite("mass", &BodyParams::mass)
        .def_readwrite("shape_handle", &BodyParams::shape_handle)
        .def_readwrite("flags", &BodyParams::flags);

    py::class_<BodyView>(m, "BodyView").def_readonly("n", &BodyView::n);

    py::class_<BodyStore>(m, "BodyStore")
        .def(py::init<Stream&, uint32_t>(), "s"_a, "capacity"_a, py::keep_alive<1, 2>())
        .def("add", &BodyStore::add)
        .def("upload", &BodyStore::upload)
        .def("count", &BodyStore::count)
        .def("view", &BodyStore::view)
        .def("body_shapes", &BodyStore::body_shapes)
        .def("state", [](BodyStore& b) {
            py::array_t<float> out({size_t(13), size_t(b.count())});
            if (b.count()) b.download_state(out.mutable_data());
            return out;
        }, "The 13 state rows (pos xyz, rot wxyz, vel xyz, ang xyz), (13, n) float32, blocking.")
        .def("set_state", [](BodyStore& b, py::array_t<float, py::array::c_style | py::array::forcecast> st) {
            if (st.size() != py::ssize_t(13) * b.count()) throw std::invalid_argument("state must be (13, n)");
            if (b.count()) b.upload_state(st.data());
        })
        .def("device_rows", [](BodyStore& b) {
            return DeviceArray{reinterpret_cast<uintptr_t>(b.device_rows()), {20, b.capacity()}, "<f4"};
        }, py::keep_alive<0, 1>(),
           "The (20, capacity) float32 device rows: state, inverse mass, inverse inertia (zero-copy).");

    // ── integrate / Broadphase / Narrowphase / XpbdSolver ───────────────────
    py::class_<IntegratorParams>(m, "IntegratorParams")
        .def(py::init<>())
        .def("set_gravity", [](IntegratorParams& p, float x, float y, float z) {
            p.gravity[0] = x; p.gravity[1] = y; p.gravity[2] = z;
        })
        .def_readwrite("dt", &IntegratorParams::dt)
        .def_readwrite("n_substeps", &IntegratorParams::n_substeps);
    m.def("integrate", &integrate, "s"_a, "bodies"_a, "params"_a);

    py::class_<BvhView>(m, "BvhView").def_readonly("n", &BvhView::n);

    py::class_<Broadphase>(m, "Broadphase")
        .def(py::init<Stream&, uint32_t, uint32_t>(), "s"_a, "max_bodies"_a, "max_pairs"_a)
        .def("build_and_query", &Broadphase::build_and_query, "s"_a, "bodies"_a, "shapes"_a, "scene_bounds"_a)
        .def("download_count", &Broadphase::download_count)
        .def("sort_pairs", &Broadphase::sort_pairs, "s"_a, "n_pairs"_a)
        .def("bvh_view", &Broadphase::bvh_view, "n_active"_a, py::keep_alive<0, 1>())
        .def("pairs", [](const Broadphase& bp, Stream& s) {
            const uint32_t n = std::min(bp.download_count(s), bp.max_pairs());
            py::array_t<uint32_t> out({size_t(n), size_t(2)});
            if (n) check(dyph_copy_to_host(out.mutable_data(), bp.pairs_ptr(), size_t(n) * 8, s.abi()), "pairs");
            return out;
        });

    py::class_<Narrowphase>(m, "Narrowphase")
        .def(py::init<Stream&, uint32_t>(), "s"_a, "max_contacts"_a)
        .def("run", [](Narrowphase& np, Stream& s, const Broadphase& bp, uint32_t n_pairs, BodyView bv,
                       ShapeView sv) { np.run(s, bp.pairs_ptr(), n_pairs, bv, sv); },
             "s"_a, "bp"_a, "n_pairs"_a, "bodies"_a, "shapes"_a)
        .def("download_count", &Narrowphase::download_count)
        .def("overflowed", &Narrowphase::overflowed);

    py::class_<XpbdSolver>(m, "XpbdSolver")
        .def(py::init<Stream&, int, uint32_t, float, uint32_t>(), "s"_a, "n_iters"_a = 10,
             "max_contacts"_a = 16384, "friction"_a = 0.5f, "max_bodies"_a = 1u << 16)
        .def("solve", [](XpbdSolver& sv, Stream& s, const Narrowphase& np, BodyView bodies, float dt) {
            sv.solve(s, np.contacts(), bodies, dt);
        }, "s"_a, "np"_a, "bodies"_a, "dt"_a)
        .def("set_force_serial", &XpbdSolver::set_force_serial);

    // ── queries ─────────────────────────────────────────────────────────────
    m.def("ray_query", &ray_query_host, "s"_a, "bvh"_a, "bodies"_a, "shapes"_a, "rays"_a,
          "Closest hit per ray. rays: (n, 7) float32 origin xyz, direction xyz, t_max. Returns (t, body_idx); "
          "body_idx is 0xFFFFFFFF on a miss.");

    py::class_<ContactSensor>(m, "ContactSensor")
        .def(py::init<uint32_t>(), "shape_idx"_a, "Subscribe to contacts involving the given shape index.")
        .def("query", &ContactSensor::query, "s"_a, "np"_a, "body_shapes"_a,
             "Filter the narrowphase's contacts on the device and download the matches. Returns the count.")
        .def("count", &ContactSensor::count)
        .def("shape_idx", &ContactSensor::shape_idx)
        .def("body_a", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.body_a(), cs.count(), self);
        }, "Body-A indices (numpy uint32, zero-copy view).")
        .def("body_b", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.body_b(), cs.count(), self);
        })
        .def("pos_x", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.pos_x(), cs.count(), self);
        })
        .def("pos_y", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.pos_y(), cs.count(), self);
        })
        .def("pos_z", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.pos_z(), cs.count(), self);
        })
        .def("norm_x", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.norm_x(), cs.count(), self);
        })
        .def("norm_y", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.norm_y(), cs.count(), self);
        })
        .def("norm_z", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.norm_z(), cs.count(), self);
        })
        .def("depth", [](py::object self) {
            const auto& cs = self.cast<const ContactSensor&>();
            return host_view(cs.depth(), cs.count(), self);
        }, "Penetration depths (numpy float32, zero-copy view).");

    // ── the whole frame step ────────────────────────────────────────────────
    py::enum_<dyph_solver_mode>(m, "SolverMode")
        .value("Reference", DYPH_SOLVER_REFERENCE)
        .value("Sequential", DYPH_SOLVER_SEQUENTIAL)
        .value("Colored", DYPH_SOLVER_COLORED)
        .value("ReferenceRounds", DYPH_SOLVER_REFERENCE_ROUNDS);

    py::class_<dyph_fused_config>(m, "FusedConfig")
        .def_readonly("smem_bytes", &dyph_fused_config::smem_bytes)
        .def_readonly("teams", &dyph_fused_config::teams)
        .def_readonly("warp_scenes", &dyph_fused_config::warp_scenes)
        .def_readonly("half_scenes", &dyph_fused_config::half_scenes)
        .def_readonly("block_scenes", &dyph_fused_config::block_scenes)
        .def_readonly("blocks", &dyph_fused_config::blocks)
        .def_readonly("blocks_per_sm", &dyph_fused_config::blocks_per_sm)
        .def_readonly("register_blocks", &dyph_fused_config::register_blocks)
        .def_readonly("ms_per_frame", &dyph_fused_config::ms_per_frame)
        .def_readonly("candidates", &dyph_fused_config::candidates);

    py::class_<World>(m, "World")
        .def(py::init<Stream&, BodyStore&, ShapeStore&, const AABB&, const IntegratorParams&, uint32_t, uint32_t,
                      int, float, dyph_solver_mode>(),
             "s"_a, "bodies"_a, "shapes"_a, "scene_bounds"_a, "params"_a = IntegratorParams{}, "max_pairs"_a = 0,
             "max_contacts"_a = 0, "n_iters"_a = 10, "friction"_a = 0.5f, "mode"_a = DYPH_SOLVER_REFERENCE,
             py::keep_alive<1, 2>(), py::keep_alive<1, 3>(), py::keep_alive<1, 4>())
        .def("set_scenes", &World::set_scenes, "body_offset"_a, "bounds"_a)
        .def("step", &World::step, "s"_a, "n_frames"_a = 1)
        .def("fused_config", &World::fused_config)
        .def("set_fused_config", &World::set_fused_config, "smem_cap"_a, "teams"_a = 2, "register_blocks"_a = 0)
        .def("autotune", &World::autotune, "s"_a, "frames"_a = 16)
        .def("adjoint_config", &World::adjoint_config)
        .def("set_adjoint_config", &World::set_adjoint_config, "smem_bytes"_a = 0, "teams"_a = 2)
        .def("hash", [](World& w, Stream& s) { return state_hash(s, w.bodies().view()); })
        .def("scene_hashes", &World::scene_hashes, "s"_a, "n_scenes"_a)
        .def("count", [](World& w) { return w.bodies().count(); })
        .def("device_rows", [](World& w) {
            BodyStore& b = w.bodies();
            return DeviceArray{reinterpret_cast<uintptr_t>(b.device_rows()), {20, b.capacity()}, "<f4"};
        }, py::keep_alive<0, 1>())
        .def("initial_rows", [](World& w) {
            return DeviceArray{reinterpret_cast<uintptr_t>(w.initial_rows()), {13, w.bodies().capacity()}, "<f4"};
        }, py::keep_alive<0, 1>())
        .def("rollout_raw", [](World& w, int n_frames, int every, uintptr_t d_ckpt, uintptr_t stream) {
            check(dyph_world_rollout(w.handle(), n_frames, every, reinterpret_cast<float*>(d_ckpt),
                                     reinterpret_cast<dyph_stream>(stream)),
                  "World::rollout");
        }, "n_frames"_a, "every"_a, "d_ckpt"_a, "stream"_a)
        .def("rollout_backward_raw", [](World& w, int n_frames, int every, uintptr_t d_ckpt, uintptr_t g_final,
                                        uintptr_t g_init, uintptr_t g_inv_mass, uintptr_t stream) {
            check(dyph_world_rollout_backward(w.handle(), n_frames, every, reinterpret_cast<const float*>(d_ckpt),
                                              reinterpret_cast<const float*>(g_final),
                                              reinterpret_cast<float*>(g_init), reinterpret_cast<float*>(g_inv_mass),
                                              reinterpret_cast<dyph_stream>(stream)),
                  "World::rollout_backward");
        }, "n_frames"_a, "every"_a, "d_ckpt"_a, "grad_final"_a, "grad_init"_a, "grad_inv_mass"_a, "stream"_a);

    m.def("rollout", [](py::args args, py::kwargs kwargs) {
        return py::module_::import("dyphur_b200.autograd").attr("rollout")(*args, **kwargs);
    }, "rollout(world, vel, ang, inv_mass, frames, every=10, initial=None) -> final state (13, n): the "
       "differentiable rollout (a torch.autograd.Function over World.rollout_raw / rollout_backward_raw).");

    m.def("status_string", [](int st) { return std::string(dyph_status_string(st)); });
}
