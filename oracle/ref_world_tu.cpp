// Test infrastructure only: the reference's src/phys/world.cpp, compiled from where it lies as this translation unit
// (in place of compiling it on its own), with its private members open, so that the checker can read an island's
// contact pairs (World::Island::nt, a type private to world.cpp). Nothing of world.cpp's code changes: the same file,
// the same flags; the product never links this.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "core/jobs.h"
#include "core/profiler.h"
#include "core/util.h"
#define private public
#include "phys/world.h"
#include "phys/world.cpp"
#undef private

// The node-triangle contact pairs of every island that searched for pairs in the last frame (Island::nt after
// rebuild_pairs + near_pairs, world.cpp:3466-3475), islands in order: 4 int32 a pair (the node's body and node, the
// triangle's body and triangle; bodies as indices of World::bodies()). Returns the count; writes at most cap.
extern "C" int ref_world_pairs(void* world, int32_t* out, int cap) {
    bl::phys::World& w = *static_cast<bl::phys::World*>(world);
    std::unordered_map<const bl::phys::SoftBody*, int> index;
    for (size_t i = 0; i < w.m_bodies.size(); i++) index[w.m_bodies[i].get()] = (int)i;
    int n = 0;
    for (int k = 0; k < w.m_num_islands; k++) {
        const bl::phys::World::Island& isl = *w.m_islands[k];
        if (!isl.needs_pairs) continue;
        for (const auto& p : isl.nt) {
            if (n < cap) {
                out[4 * n] = index[isl.bodies[p.bn]], out[4 * n + 1] = (int32_t)p.node;
                out[4 * n + 2] = index[isl.bodies[p.bt]], out[4 * n + 3] = (int32_t)p.tri;
            }
            n++;
        }
    }
    return n;
}
