// The reference's frame loop (examples/stress_test_blocks/main.cpp:264-279)
// written against the C++ class layer (include/dyphur_b200.hpp): stores,
// integrate -> build_and_query -> download_count -> sort_pairs ->
// Narrowphase::run -> XpbdSolver::solve, then the FNV-1a state hash.
//
//   frame_loop <scene kind> <a0> <a1> <a2> <spacing> <jitter> <seed> <frames> <force_serial>
//
// Prints "hash 0x... pairs N contacts M".
#include <cinttypes>
#include <cstdio>
#include <cstdlib>

#include "../../dyphur_b200/csrc/scenes.h"
#include "../../include/dyphur_b200.hpp"

int main(int argc, char** argv) {
    if (argc != 10) {
        std::fprintf(stderr, "usage: frame_loop kind a0 a1 a2 spacing jitter seed frames force_serial\n");
        return 2;
    }
    const int kind = std::atoi(argv[1]);
    dyph_scene_set* sc = dyph_scene_make(kind, std::strtoull(argv[7], nullptr, 10), std::atoi(argv[2]),
                                         std::atoi(argv[3]), std::atoi(argv[4]), std::strtof(argv[5], nullptr),
                                         std::strtof(argv[6], nullptr));
    if (!sc) return 2;
    const int frames = std::atoi(argv[8]);
    try {
        dyphur::Device dev = dyphur::Device::default_gpu();
        dyphur::Stream s = dev.make_stream();
        dyphur::ShapeStore shapes(s, sc->n_shapes);
        for (uint32_t i = 0; i < sc->n_shapes; ++i)
            shapes.add({static_cast<dyphur::ShapeType>(sc->shape_type[i]), sc->shape_half[3 * i],
                        sc->shape_half[3 * i + 1], sc->shape_half[3 * i + 2]});
        shapes.upload();
        dyphur::BodyStore bodies(s, sc->n_bodies);
        for (uint32_t i = 0; i < sc->n_bodies; ++i) {
            dyphur::BodyParams p;
            for (int k = 0; k < 3; ++k) {
                p.position[k] = sc->pos[3 * i + k];
                p.linear_velocity[k] = sc->vel[3 * i + k];
                p.angular_velocity[k] = sc->ang[3 * i + k];
            }
            for (int k = 0; k < 4; ++k) p.rotation[k] = sc->rot[4 * i + k];
            for (int k = 0; k < 9; ++k) p.inertia[k] = sc->inertia[9 * i + k];
            p.mass = sc->mass[i];
            p.shape_handle = sc->shape[i];
            p.flags = sc->flags[i];
            bodies.add(p);
        }
        bodies.upload();
        const dyphur::AABB bounds{sc->bounds[0], sc->bounds[1], sc->bounds[2],
                                  sc->bounds[3], sc->bounds[4], sc->bounds[5]};
        dyphur::Broadphase bp(s, sc->n_bodies, sc->max_pairs);
        dyphur::Narrowphase np(s, sc->max_contacts);
        dyphur::XpbdSolver solver(s, sc->n_iters, sc->max_contacts, sc->friction, sc->n_bodies);
        solver.set_force_serial(std::atoi(argv[9]) != 0);
        dyphur::IntegratorParams ip;
        ip.dt = sc->dt;
        uint32_t n_pairs = 0, n_contacts = 0;
        for (int f = 0; f < frames; ++f) {
            dyphur::integrate(s, bodies.view(), ip);
            bp.build_and_query(s, bodies.view(), shapes.view(), bounds);
            n_pairs = bp.download_count(s);
            bp.sort_pairs(s, n_pairs);
            np.run(s, bp.pairs_ptr(), std::min(n_pairs, bp.max_pairs()), bodies.view(), shapes.view());
            n_contacts = np.download_count(s);
            solver.solve(s, np.contacts(), bodies.view(), ip.dt);
        }
        const uint64_t h = dyphur::state_hash(s, bodies.view());
        std::printf("hash 0x%016" PRIx64 " pairs %u contacts %u\n", h, n_pairs, n_contacts);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        dyph_scene_free(sc);
        return 1;
    }
    dyph_scene_free(sc);
    return 0;
}
