// Test driver of the drop-in shim (gpu_world.h): one body built twice through the reference's own builder API
// (SoftBody::add_node / add_beam / finalize, softbody.cpp:8-110), one copy stepped by the reference's
// World::step_substeps, the other through GpuWorld; both end states returned for comparison (tests/test_shim.py).
#include "gpu_world.h"

#include <cstring>
#include <memory>

using namespace bl;
using namespace bl::phys;

namespace {
std::unique_ptr<SoftBody> make_body(int n_nodes, const float* pos, const float* vel, const float* mass, int n_beams, const uint32_t* ab,
                                    const float* k, const float* d, const float* strength, const float* deform) {
    auto b = std::make_unique<SoftBody>();
    for (int i = 0; i < n_nodes; i++) b->add_node(vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), mass[i]);
    for (int j = 0; j < n_beams; j++) b->add_beam(ab[2 * j], ab[2 * j + 1], k[j], d[j], strength[j], deform[j]);
    b->finalize();
    for (int i = 0; i < n_nodes; i++) b->nodes[i].v = vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    return b;
}
} // namespace

extern "C" int shim_step_compare(int n_nodes, const float* pos, const float* vel, const float* mass, int n_beams, const uint32_t* ab,
                                 const float* k, const float* d, const float* strength, const float* deform, float ground_y, int frames,
                                 int substeps, float* ref_nodes, float* gpu_nodes, float* ref_beams, float* gpu_beams) {
    try {
        World w;
        w.settings.sleeping = false;
        w.settings.multithreaded = false; // (the reference's results do not depend on its thread count; no job threads to end)
        w.statics.add_box(vec3(0, ground_y - 1.0f, 0), vec3(100, 1, 100), quat(), 0);
        w.statics.build_grid();
        SoftBody* ref = w.add_body(make_body(n_nodes, pos, vel, mass, n_beams, ab, k, d, strength, deform));
        std::unique_ptr<SoftBody> mine = make_body(n_nodes, pos, vel, mass, n_beams, ab, k, d, strength, deform);
        GpuWorld g(w.settings);
        g.set_statics(w.statics);
        const int id = g.add_body(*mine);
        for (int f = 0; f < frames; f++) w.step_substeps(substeps), g.step_substeps(substeps);
        g.pull(id, *mine);
        std::memcpy(ref_nodes, ref->nodes.data(), sizeof(Node) * n_nodes);
        std::memcpy(gpu_nodes, mine->nodes.data(), sizeof(Node) * n_nodes);
        std::memcpy(ref_beams, ref->beams.data(), sizeof(Beam) * n_beams);
        std::memcpy(gpu_beams, mine->beams.data(), sizeof(Beam) * n_beams);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}
