// Test infrastructure only: a C-ABI driver over the reference's own physics (BeamLab `src/phys`, `src/core`),
// compiled from the reference's sources where they lie (oracle/Makefile). It lets tests, the golden-fixture script and
// the CPU-baseline leg of bench.py build the same synthetic rigs through the reference's builder API and step them with
// the reference's `World::step_substeps`, then read the state back.
//
// Nothing of the product links this file. Every call mirrors one reference entry point:
//   ref_world_new / ref_step_substeps   -> bl::phys::World, World::step_substeps   (src/phys/world.h:150-168)
//   ref_set_terrain                     -> Heightfield::create + has_terrain + update_bounds (src/phys/static_world.h:52-90)
//   ref_add_box / ref_build_grid        -> StaticWorld::add_box / build_grid        (src/phys/static_world.h:193-195)
//   ref_add_body                        -> SoftBody::add_node / add_beam / finalize (src/phys/softbody.h:953-973)
//   ref_jobs_init                       -> JobSystem::get().init                   (src/core/jobs.h:22)
#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "core/jobs.h"
// (the FEM frame's solver pattern - ordering, blocks, updates - is private to FemFrame; the checker reads it)
#define private public
#include "phys/fem_shell.h"
#include "phys/world.h"
#undef private

using namespace bl;
using namespace bl::phys;

struct RefWorld {
    World w;
    std::vector<SoftBody*> bodies;
    std::map<int, std::vector<std::pair<uint32_t, vec3>>> loads; // the constant node loads of each body
    std::map<int, std::map<int, std::pair<float, float>>> drives; // each body's wheels' torque and brake (N m)
};

// a body's one pre_substep (the controller hook, world.cpp:3261): its wheels' torque and brake set, its loads added
static void install_pre_substep(RefWorld* r, int body) {
    const std::vector<std::pair<uint32_t, vec3>> all = r->loads[body];
    const std::map<int, std::pair<float, float>> drv = r->drives[body];
    r->bodies[body]->pre_substep = [all, drv](SoftBody& sb, float) {
        for (const auto& [k, tb] : drv)
            if (k < (int)sb.wheels.size()) sb.wheels[k].torque = tb.first, sb.wheels[k].brake = tb.second;
        for (const auto& [nd, f] : all)
            if (nd < sb.force.size()) sb.force[nd] += f;
    };
}

// per-body knobs of SoftBody that the GPU path supports (softbody.h:650-700)
struct RefBodyParams {
    float ground_friction;
    float bounce;
    float contact_push_max;
    float contact_slop;
    float collision_radius;
    int32_t allow_deform;
    int32_t allow_break;
    int32_t ductile;
    int32_t can_sleep;
    float sleep_speed;
    // contacts with other bodies (softbody.h:614-721)
    float contact_friction;
    float hull_depth;
    float face_skin;
    int32_t faces_only;
    int32_t collision_group;
};

extern "C" {

void ref_jobs_init(int workers) { JobSystem::get().init(workers); }
void ref_jobs_shutdown() { JobSystem::get().shutdown(); }
int ref_jobs_threads() { return JobSystem::get().num_threads(); }

RefWorld* ref_world_new() { return new RefWorld(); }
void ref_world_free(RefWorld* r) { delete r; }

void ref_world_settings(RefWorld* r, float gx, float gy, float gz, float dt, int sleeping, int multithreaded, int inter_body, float sleep_speed,
                        float sleep_time) {
    WorldSettings& s = r->w.settings;
    s.gravity = vec3(gx, gy, gz);
    s.dt = dt;
    s.sleeping = sleeping != 0;
    s.multithreaded = multithreaded != 0;
    s.inter_body_collisions = inter_body != 0;
    s.sleep_speed = sleep_speed;
    s.sleep_time = sleep_time;
}

// WorldSettings::tyre_grip (world.h:55): the factor on the tyres' friction
void ref_set_tyre_grip(RefWorld* r, float g) { r->w.settings.tyre_grip = g; }

// heights / surfaces: nz rows of nx samples, x fastest
void ref_set_terrain(RefWorld* r, int nx, int nz, float cell, float ox, float oz, const float* heights, const uint8_t* surfaces) {
    StaticWorld& st = r->w.statics;
    st.terrain.create(nx, nz, cell, vec2(ox, oz));
    for (int z = 0; z < nz; z++)
        for (int x = 0; x < nx; x++) {
            st.terrain.h(x, z) = heights[(size_t)z * nx + x];
            if (surfaces) st.terrain.surf(x, z) = surfaces[(size_t)z * nx + x];
        }
    st.has_terrain = true;
    st.terrain.update_bounds();
}

void ref_add_box(RefWorld* r, float cx, float cy, float cz, float hx, float hy, float hz, float qx, float qy, float qz, float qw, int surface,
                 float max_force) {
    r->w.statics.add_box(vec3(cx, cy, cz), vec3(hx, hy, hz), quat(qx, qy, qz, qw), (uint8_t)surface);
    r->w.statics.boxes.back().max_force = max_force;
}

void ref_add_cylinder(RefWorld* r, float bx, float by, float bz, float radius, float height, int surface) {
    StaticCylinder c;
    c.base = vec3(bx, by, bz);
    c.radius = radius;
    c.height = height;
    c.surface = (uint8_t)surface;
    r->w.statics.cylinders.push_back(c);
}

void ref_build_grid(RefWorld* r) { r->w.statics.build_grid(); }
void ref_set_kill_y(RefWorld* r, float y) { r->w.statics.kill_y = y; }

// Builds one body through the reference's builder calls, in this order: add_node (and its velocity, friction, radius),
// add_beam, add_triangle, finalize; then World::add_body. Returns the body's index in this driver.
int ref_add_body(RefWorld* r, int n_nodes, const float* pos, const float* vel, const float* mass, const uint16_t* nflags, const float* friction,
                 const float* radius, int n_beams, const uint32_t* ab, const float* k, const float* d, const float* strength, const float* deform,
                 const uint8_t* btype, const uint8_t* bflags, int n_tris, const uint32_t* tri, const RefBodyParams* p) {
    auto b = std::make_unique<SoftBody>();
    b->name = "body" + std::to_string(r->bodies.size());
    for (int i = 0; i < n_nodes; i++) {
        const uint32_t id = b->add_node(vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), mass[i], nflags[i]);
        b->nodes[id].v = vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        b->info[id].friction = friction[i];
        b->info[id].radius = radius[i];
    }
    for (int j = 0; j < n_beams; j++) b->add_beam(ab[2 * j], ab[2 * j + 1], k[j], d[j], strength[j], deform[j], btype[j], bflags[j]);
    for (int t = 0; t < n_tris; t++) b->add_triangle(tri[3 * t], tri[3 * t + 1], tri[3 * t + 2]);
    b->ground_friction = p->ground_friction;
    b->bounce = p->bounce;
    b->contact_push_max = p->contact_push_max;
    b->contact_slop = p->contact_slop;
    b->collision_radius = p->collision_radius;
    b->allow_deform = p->allow_deform != 0;
    b->allow_break = p->allow_break != 0;
    b->ductile = p->ductile != 0;
    b->can_sleep = p->can_sleep != 0;
    b->sleep_speed = p->sleep_speed;
    b->contact_friction = p->contact_friction;
    b->hull_depth = p->hull_depth;
    b->face_skin = p->face_skin;
    b->faces_only = p->faces_only != 0;
    b->collision_group = p->collision_group;
    b->finalize();
    r->bodies.push_back(r->w.add_body(std::move(b)));
    return (int)r->bodies.size() - 1;
}

void ref_step_substeps(RefWorld* r, int n) { r->w.step_substeps(n); }

// Triangle::two_sided of a body's collision triangles (0: a hull triangle), set before its first step
void ref_set_tri_sides(RefWorld* r, int body, const uint8_t* two_sided) {
    SoftBody& b = *r->bodies[body];
    for (size_t t = 0; t < b.tris.size(); t++) b.tris[t].two_sided = two_sided[t] != 0;
    b.hull_count = -1;
}

// the islands' contact pairs of the last pair search (ref_world_tu.cpp)
int ref_world_pairs(void* world, int32_t* out, int cap);
int ref_get_pairs(RefWorld* r, int32_t* out, int cap) { return ref_world_pairs(&r->w, out, cap); }

// ---- FEM shell plates (ShellMesher::grid, fem_shell.cpp:34-50) ----
// A plate body of n x n cells: origin + du * i + dv * j, triangle elements of one shell section (E, nu, rho, t,
// yield, damping, drill as given), the nodes of row j = 0 anchored (NF_FIXED) when clamp_edge, gravity on. Its nodes
// carry node_flags. Returns the body index.
int ref_add_plate(RefWorld* r, int n, float ox, float oy, float oz, float dux, float duy, float duz, float dvx, float dvy, float dvz, float E, float nu,
                  float rho, float t, float yield, float damping, float drill, int clamp_edge, int node_flags) {
    auto b = std::make_unique<SoftBody>();
    b->name = "plate" + std::to_string(r->bodies.size());
    b->can_sleep = false;
    ShellSection s = make_shell_section("Steel", t);
    s.E = E, s.nu = nu, s.rho = rho, s.t = t, s.yield = yield, s.damping = damping, s.drill = drill;
    s.pattern = ShellPattern::None;
    s.max_level = 0;
    const uint16_t sec = b->fem.add_shell_section(s);
    ShellMesher m(*b, (uint16_t)node_flags);
    const std::vector<uint32_t> ids = m.grid(vec3(ox, oy, oz), vec3(dux, duy, duz), vec3(dvx, dvy, dvz), n, n, sec, false);
    if (clamp_edge)
        for (int i = 0; i <= n; i++) b->info[ids[i]].flags |= NF_FIXED;
    m.finish();
    b->finalize();
    SoftBody* bp = r->w.add_body(std::move(b));
    bp->fem.finalize(*bp); // (what its first step would do: FemFrame::begin_forces, frame_fem.cpp:1860)
    r->bodies.push_back(bp);
    return (int)r->bodies.size() - 1;
}

// A body with a FEM frame of members and triangles (FemFrame::add_section / add_shell_section / add_element /
// add_tri, frame_fem.cpp:190-222; then finalize as a first step would): its nodes (SoftBody::add_node); the shell
// sections (7 floats each: E nu rho t yield damping drill, on make_shell_section's defaults with no pattern), the
// triangles (a, b, c, section; the mass they put on their corners); the frame sections (16 floats each: E G rho A
// Iy Iz J As_y As_z damping axial joint_k Np Mp Tp hardening), the members (ends, section, joints, mass); tris_first: the
// add_tri calls before the add_element calls (the frame nodes numbered in the calls' order)
int ref_add_fem_body(RefWorld* r, int n_nodes, const float* pos, const float* vel, const float* mass, const uint16_t* nflags, int n_ssec,
                     const float* ssec, int n_tris, const uint32_t* tri, const uint16_t* tsec, const float* tmass, int n_fsec, const float* fsec,
                     int n_members, const uint32_t* ab, const uint16_t* msec, const uint8_t* ends, const float* mmass, int tris_first) {
    auto b = std::make_unique<SoftBody>();
    b->name = "fem" + std::to_string(r->bodies.size());
    b->can_sleep = false;
    for (int i = 0; i < n_nodes; i++) {
        const uint32_t id = b->add_node(vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]), mass[i], nflags[i]);
        b->nodes[id].v = vec3(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
    }
    for (int k = 0; k < n_ssec; k++) {
        const float* f = ssec + 7 * k;
        ShellSection s = make_shell_section("Steel", f[3]);
        s.E = f[0], s.nu = f[1], s.rho = f[2], s.t = f[3], s.yield = f[4], s.damping = f[5], s.drill = f[6];
        s.pattern = ShellPattern::None;
        s.max_level = 0;
        b->fem.add_shell_section(s);
    }
    for (int k = 0; k < n_fsec; k++) {
        const float* f = fsec + 16 * k;
        FrameSection s;
        s.E = f[0], s.G = f[1], s.rho = f[2], s.A = f[3], s.Iy = f[4], s.Iz = f[5], s.J = f[6], s.As_y = f[7], s.As_z = f[8];
        s.damping = f[9], s.axial = f[10], s.joint_k = f[11], s.Np = f[12], s.Mp = f[13], s.Tp = f[14], s.hardening = f[15];
        b->fem.add_section(s);
    }
    auto add_tris = [&]() {
        for (int t = 0; t < n_tris; t++) {
            const uint32_t id = b->fem.add_tri(tri[3 * t], tri[3 * t + 1], tri[3 * t + 2], tsec[t]);
            b->fem.tris[id].mass = tmass[t];
        }
    };
    if (tris_first) add_tris();
    for (int e = 0; e < n_members; e++) {
        const uint32_t id = b->fem.add_element(ab[2 * e], ab[2 * e + 1], msec[e], ends[2 * e], ends[2 * e + 1]);
        b->fem.elems[id].mass = mmass[e];
    }
    if (!tris_first) add_tris();
    b->finalize();
    SoftBody* bp = r->w.add_body(std::move(b));
    bp->fem.finalize(*bp);
    r->bodies.push_back(bp);
    return (int)r->bodies.size() - 1;
}

// SoftBody::air_drag and aero_cda of a body (RoR's per-node drag against its part's mean velocity, and Cd A)
void ref_set_drag(RefWorld* r, int body, float air_drag, float aero_cda) {
    r->bodies[body]->air_drag = air_drag;
    r->bodies[body]->aero_cda = aero_cda;
}

// A shock on one of a body's beams (Shock, softbody.h:88-101; the beam carries BF_SHOCK): type, soft bump, then 20
// floats: spring damp spring_in damp_in prog_spring_in prog_damp_in spring_out damp_out prog_spring_out prog_damp_out
// damp_in_slow split_in damp_in_fast damp_out_slow split_out damp_out_fast short_bound long_bound bound_spring bound_damp
void ref_add_shock(RefWorld* r, int body, uint32_t beam, int type, int soft_bump, const float* f) {
    Shock s;
    s.beam = beam, s.type = (uint8_t)type, s.soft_bump = soft_bump != 0;
    s.spring = f[0], s.damp = f[1], s.spring_in = f[2], s.damp_in = f[3], s.prog_spring_in = f[4], s.prog_damp_in = f[5];
    s.spring_out = f[6], s.damp_out = f[7], s.prog_spring_out = f[8], s.prog_damp_out = f[9];
    s.damp_in_slow = f[10], s.split_in = f[11], s.damp_in_fast = f[12], s.damp_out_slow = f[13], s.split_out = f[14], s.damp_out_fast = f[15];
    s.short_bound = f[16], s.long_bound = f[17], s.bound_spring = f[18], s.bound_damp = f[19];
    r->bodies[body]->shocks.push_back(s);
}

// SoftBody::allow_deform and allow_break of a body (softbody.h:711-712)
void ref_set_body_flags(RefWorld* r, int body, int allow_deform, int allow_break) {
    r->bodies[body]->allow_deform = allow_deform != 0;
    r->bodies[body]->allow_break = allow_break != 0;
}

// A wheel of tyre nodes on a body (Wheel, softbody.h:468-498): its hubs, its tyre nodes (even: axle0's side), radius,
// width, mass, propulsion (0 none, 1 forward, 2 backward) and arm (the reaction torque's arm node and its nearer axle
// node; -1: none), as the vehicle builder fills them
void ref_add_wheel(RefWorld* r, int body, uint32_t axle0, uint32_t axle1, const uint32_t* nodes, int n, float radius, float width, float mass,
                   int propulsed, int arm, int near_attach) {
    Wheel w;
    w.axle0 = axle0, w.axle1 = axle1;
    w.nodes.assign(nodes, nodes + n);
    w.radius = radius, w.width = width, w.mass = mass;
    w.propulsed = propulsed, w.arm = arm, w.near_attach = near_attach;
    r->bodies[body]->wheels.push_back(w);
}

// A constant force on one node of a body, applied every substep right after gravity (the SoftBody::pre_substep hook,
// world.cpp:3261)
void ref_set_point_load(RefWorld* r, int body, int node, float fx, float fy, float fz) {
    // (every load of the body in one callback: a body has one pre_substep)
    r->loads[body].push_back({(uint32_t)node, vec3(fx, fy, fz)});
    install_pre_substep(r, body);
}

// A wheel's drive torque and brake torque (N m), set by the controller hook every substep from now on (a vehicle
// controller's differential output and brake, as the truck controller sets Wheel::torque and brake)
void ref_set_wheel_drive(RefWorld* r, int body, int wheel, float torque, float brake) {
    r->drives[body][wheel] = {torque, brake};
    install_pre_substep(r, body);
}

// the frame's pattern sizes: [frame nodes, tris, components, off-diagonal blocks, block updates, solve failures, clamps]
void ref_fem_info(RefWorld* r, int body, long long* out) {
    const FemFrame& f = r->bodies[body]->fem;
    out[0] = (long long)f.node.size(), out[1] = (long long)f.tris.size(), out[2] = f.components(), out[3] = (long long)f.row_.size();
    out[4] = (long long)f.upd_.size(), out[5] = f.solve_failures, out[6] = f.clamps;
    out[7] = f.passes_; // (the systems assembled and factored: more than one a step where a re-pass ran)
}

// the pattern itself: perm (n), col_ptr (n + 1), row (blocks), upd as (pi, pj, target) triples
void ref_fem_pattern(RefWorld* r, int body, int* perm, int* col_ptr, int* row, int* upd) {
    const FemFrame& f = r->bodies[body]->fem;
    std::copy(f.perm_.begin(), f.perm_.end(), perm);
    std::copy(f.col_ptr_.begin(), f.col_ptr_.end(), col_ptr);
    std::copy(f.row_.begin(), f.row_.end(), row);
    for (size_t u = 0; u < f.upd_.size(); u++) upd[3 * u] = f.upd_[u].pi, upd[3 * u + 1] = f.upd_[u].pj, upd[3 * u + 2] = f.upd_[u].target;
}

// the frame nodes' state: body node, double positions (3), orientation (x y z w), angular velocity (3)
void ref_fem_nodes(RefWorld* r, int body, int* node, double* xd, float* q, float* w) {
    const FemFrame& f = r->bodies[body]->fem;
    for (size_t i = 0; i < f.node.size(); i++) {
        node[i] = (int)f.node[i];
        xd[3 * i] = f.xd[3 * i], xd[3 * i + 1] = f.xd[3 * i + 1], xd[3 * i + 2] = f.xd[3 * i + 2];
        q[4 * i] = f.q[i].x, q[4 * i + 1] = f.q[i].y, q[4 * i + 2] = f.q[i].z, q[4 * i + 3] = f.q[i].w;
        w[3 * i] = f.w[i].x, w[3 * i + 1] = f.w[i].y, w[3 * i + 2] = f.w[i].z;
    }
}

// the triangles: nodes (frame nodes, 3), rest shape X (6), rest frames r0 (12), mass, area0
void ref_fem_tris(RefWorld* r, int body, int* n, float* X, float* r0, float* mass, float* area0) {
    const FemFrame& f = r->bodies[body]->fem;
    for (size_t t = 0; t < f.tris.size(); t++) {
        const FrameTri& tr = f.tris[t];
        for (int i = 0; i < 3; i++) {
            n[3 * t + i] = (int)tr.n[i];
            X[6 * t + 2 * i] = tr.X[i][0], X[6 * t + 2 * i + 1] = tr.X[i][1];
            r0[12 * t + 4 * i] = tr.r0[i].x, r0[12 * t + 4 * i + 1] = tr.r0[i].y, r0[12 * t + 4 * i + 2] = tr.r0[i].z, r0[12 * t + 4 * i + 3] = tr.r0[i].w;
        }
        mass[t] = tr.mass, area0[t] = tr.area0;
    }
}

// each wheel's Wheel::speed and avg_speed
void ref_wheel_state(RefWorld* r, int body, float* speed, float* avg_speed) {
    const SoftBody* b = r->bodies[body];
    for (size_t k = 0; k < b->wheels.size(); k++) speed[k] = b->wheels[k].speed, avg_speed[k] = b->wheels[k].avg_speed;
}

// SoftBody::wheel_speed, wheel_spin
void ref_body_wheel_speed(RefWorld* r, int body, float* out) { out[0] = r->bodies[body]->wheel_speed, out[1] = r->bodies[body]->wheel_spin; }

// FrameTri::dmg of each triangle (the plastic stretch reached)
void ref_fem_tri_dmg(RefWorld* r, int body, float* dmg) {
    const FemFrame& f = r->bodies[body]->fem;
    for (size_t t = 0; t < f.tris.size(); t++) dmg[t] = f.tris[t].dmg;
}

int ref_body_nodes(RefWorld* r, int body) { return (int)r->bodies[body]->nodes.size(); }
int ref_body_beams(RefWorld* r, int body) { return (int)r->bodies[body]->beams.size(); }

// pos, vel: 3 floats a node; inv_mass, mass: 1
void ref_get_nodes(RefWorld* r, int body, float* pos, float* vel, float* inv_mass, float* mass) {
    const SoftBody& b = *r->bodies[body];
    for (size_t i = 0; i < b.nodes.size(); i++) {
        const Node& x = b.nodes[i];
        std::memcpy(pos + 3 * i, &x.p, 12);
        std::memcpy(vel + 3 * i, &x.v, 12);
        if (inv_mass) inv_mass[i] = x.inv_mass;
        if (mass) mass[i] = x.mass;
    }
}

void ref_set_nodes(RefWorld* r, int body, const float* pos, const float* vel) {
    SoftBody& b = *r->bodies[body];
    for (size_t i = 0; i < b.nodes.size(); i++) {
        std::memcpy(&b.nodes[i].p, pos + 3 * i, 12);
        std::memcpy(&b.nodes[i].v, vel + 3 * i, 12);
    }
}

// the beams' state: rest length, yield limits, strength, last force, flags
void ref_get_beams(RefWorld* r, int body, float* L, float* max_pos, float* max_neg, float* strength, float* stress, uint8_t* flags) {
    const SoftBody& b = *r->bodies[body];
    for (size_t j = 0; j < b.beams.size(); j++) {
        const Beam& bm = b.beams[j];
        L[j] = bm.L, max_pos[j] = bm.max_pos, max_neg[j] = bm.max_neg, strength[j] = bm.strength, stress[j] = bm.stress, flags[j] = bm.flags;
    }
}

// out[0..5] aabb min/max, out[6] max_speed, out[7] sleeping, out[8] static_contacts (last frame), out[9] broken beams,
// out[10] sleep_timer
void ref_get_body(RefWorld* r, int body, float* out) {
    const SoftBody& b = *r->bodies[body];
    out[0] = b.aabb.mn.x, out[1] = b.aabb.mn.y, out[2] = b.aabb.mn.z;
    out[3] = b.aabb.mx.x, out[4] = b.aabb.mx.y, out[5] = b.aabb.mx.z;
    out[6] = b.max_speed;
    out[7] = b.sleeping ? 1.0f : 0.0f;
    out[8] = (float)b.static_contacts;
    out[9] = (float)b.stats.broken_beams;
    out[10] = b.sleep_timer;
}

} // extern "C"
