// The drop-in as a BeamLab maintainer would add it: a GpuWorld that steps a bl::phys::World's bodies through
// libbeamlab_b200.so's C ABI (include/beamlab_gpu.h). Compiled against the reference's own headers by the tests
// (tests/test_shim.py), so the record layouts the boundary relies on are checked by the compiler, field by field.
#pragma once

#include "beamlab_gpu.h"
#include "phys/world.h"

#include <cstddef>
#include <stdexcept>
#include <vector>

// Node, NodeInfo, Beam and Triangle cross the boundary as they are (a SoftBody's vectors passed by pointer): every
// field at the same offset with the same size (softbody.h:43-58, 71-85, 138-147).
#define BL_SAME_FIELD(R, B, f) static_assert(offsetof(R, f) == offsetof(B, f) && sizeof(R::f) == sizeof(B::f), #R "::" #f)
static_assert(sizeof(bl::phys::Node) == sizeof(bl_node) && alignof(bl::phys::Node) >= alignof(bl_node), "Node");
BL_SAME_FIELD(bl::phys::Node, bl_node, p);
BL_SAME_FIELD(bl::phys::Node, bl_node, inv_mass);
BL_SAME_FIELD(bl::phys::Node, bl_node, v);
BL_SAME_FIELD(bl::phys::Node, bl_node, mass);
static_assert(sizeof(bl::phys::NodeInfo) == sizeof(bl_node_info), "NodeInfo");
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, flags);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, surface);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, pad);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, friction);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, radius);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, frame);
BL_SAME_FIELD(bl::phys::NodeInfo, bl_node_info, ror_id);
static_assert(sizeof(bl::phys::Beam) == sizeof(bl_beam), "Beam");
BL_SAME_FIELD(bl::phys::Beam, bl_beam, a);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, b);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, L);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, k);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, d);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, max_pos);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, max_neg);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, strength);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, plastic);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, stress);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, L0);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, support_limit);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, type);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, flags);
BL_SAME_FIELD(bl::phys::Beam, bl_beam, group);
static_assert(sizeof(bl::phys::Triangle) == sizeof(bl_tri), "Triangle");
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, a);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, b);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, c);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, surface);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, two_sided);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, torn);
BL_SAME_FIELD(bl::phys::Triangle, bl_tri, rest_edge2);
// the flag values the two sides share (NodeFlag, BeamType, BeamFlag: softbody.h:29-69)
static_assert(bl::phys::NF_GROUND == BL_NF_GROUND && bl::phys::NF_FIXED == BL_NF_FIXED && bl::phys::NF_TYRE == BL_NF_TYRE &&
              bl::phys::NF_RIM == BL_NF_RIM && bl::phys::NF_CONTACTER == BL_NF_CONTACTER && bl::phys::NF_FRAME == BL_NF_FRAME &&
              bl::phys::NF_LOAD == BL_NF_LOAD && bl::phys::NF_NO_MOUSE == BL_NF_NO_MOUSE && bl::phys::NF_SELF_COLL == BL_NF_SELF_COLL,
              "NodeFlag");
static_assert(bl::phys::BT_NORMAL == BL_BT_NORMAL && bl::phys::BT_ROPE == BL_BT_ROPE && bl::phys::BT_SUPPORT == BL_BT_SUPPORT, "BeamType");
static_assert(bl::phys::BF_BROKEN == BL_BF_BROKEN && bl::phys::BF_INVISIBLE == BL_BF_INVISIBLE && bl::phys::BF_NO_DEFORM == BL_BF_NO_DEFORM &&
              bl::phys::BF_NO_BREAK == BL_BF_NO_BREAK && bl::phys::BF_WHEEL == BL_BF_WHEEL && bl::phys::BF_HYDRO == BL_BF_HYDRO &&
              bl::phys::BF_SHOCK == BL_BF_SHOCK,
              "BeamFlag");
#undef BL_SAME_FIELD

namespace bl::phys {

class GpuWorld {
public:
    explicit GpuWorld(const WorldSettings& s, int device = 0) {
        bl_gpu_config c;
        bl_gpu_default_config(&c);
        c.gravity[0] = s.gravity.x, c.gravity[1] = s.gravity.y, c.gravity[2] = s.gravity.z;
        c.dt = s.dt, c.sleeping = s.sleeping, c.sleep_speed = s.sleep_speed, c.sleep_time = s.sleep_time;
        c.collision_hz = s.collision_hz, c.inter_body_collisions = s.inter_body_collisions, c.tyre_grip = s.tyre_grip;
        c.device = device;
        check(bl_gpu_create(&c, &ctx_));
    }
    ~GpuWorld() { bl_gpu_destroy(ctx_); }
    GpuWorld(const GpuWorld&) = delete;
    GpuWorld& operator=(const GpuWorld&) = delete;

    // the static world: its terrain (tile by tile into one row-major grid), its boxes, then the grid. A box's
    // orientation crosses as the quaternion of its rotation matrix (exact for axis-aligned boxes).
    void set_statics(const StaticWorld& st) {
        if (st.has_terrain) {
            const Heightfield& t = st.terrain;
            std::vector<float> h((size_t)t.nx() * t.nz());
            std::vector<uint8_t> sf(h.size());
            for (int z = 0; z < t.nz(); z++)
                for (int x = 0; x < t.nx(); x++) h[(size_t)z * t.nx() + x] = t.h(x, z), sf[(size_t)z * t.nx() + x] = t.surf(x, z);
            check(bl_gpu_set_terrain(ctx_, t.nx(), t.nz(), t.cell(), t.origin().x, t.origin().y, h.data(), sf.data()));
        }
        for (const StaticBox& b : st.boxes) {
            const quat q = from_mat3(b.rot);
            const float c[3] = {b.center.x, b.center.y, b.center.z}, hf[3] = {b.half.x, b.half.y, b.half.z}, qq[4] = {q.x, q.y, q.z, q.w};
            check(bl_gpu_add_box(ctx_, c, hf, qq, b.surface, b.max_force));
        }
        check(bl_gpu_set_kill_y(ctx_, st.kill_y));
        check(bl_gpu_build_grid(ctx_));
    }

    // a finalized SoftBody of nodes, beams and collision triangles (the features bl_body_desc carries); its vectors
    // cross as they are
    int add_body(const SoftBody& b) {
        bl_body_desc d{};
        d.n_nodes = (int)b.nodes.size(), d.nodes = (const bl_node*)b.nodes.data(), d.info = (const bl_node_info*)b.info.data();
        d.n_beams = (int)b.beams.size(), d.beams = (const bl_beam*)b.beams.data();
        d.ground_friction = b.ground_friction, d.bounce = b.bounce, d.contact_push_max = b.contact_push_max;
        d.contact_slop = b.contact_slop, d.allow_deform = b.allow_deform, d.allow_break = b.allow_break;
        d.ductile = b.ductile, d.can_sleep = b.can_sleep, d.sleep_speed = b.sleep_speed;
        d.max_speed = b.max_speed, d.sleeping = b.sleeping;
        d.n_tris = (int)b.tris.size(), d.tris = (const bl_tri*)b.tris.data();
        d.collision_radius = b.collision_radius, d.contact_friction = b.contact_friction;
        d.hull_depth = b.hull_depth, d.face_skin = b.face_skin, d.faces_only = b.faces_only;
        d.collision_group = b.collision_group, d.self_collision = b.self_collision;
        d.air_drag = b.air_drag, d.aero_cda = b.aero_cda;
        int id = -1;
        check(bl_gpu_add_body(ctx_, &d, &id));
        return id;
    }
    void step_substeps(int n, void* stream = nullptr) { check(bl_gpu_step_substeps(ctx_, n, stream)); }
    // the body's nodes and beams back into its SoftBody
    void pull(int id, SoftBody& b) {
        check(bl_gpu_download_nodes(ctx_, id, (bl_node*)b.nodes.data()));
        check(bl_gpu_download_beams(ctx_, id, (bl_beam*)b.beams.data()));
    }

private:
    static void check(int rc) {
        if (rc) throw std::runtime_error(bl_gpu_error_string(rc));
    }
    bl_gpu_ctx* ctx_ = nullptr;
};

} // namespace bl::phys
