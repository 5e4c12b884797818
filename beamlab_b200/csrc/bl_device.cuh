// Device-side data layout and math of the explicit soft-body substep.
//
// Every floating-point expression below is written in the reference's operation order (src/core/math.h vector ops,
// src/phys/softbody.cpp, src/phys/static_world.cpp, src/phys/world.cpp) and the library is compiled with
// --fmad=false and IEEE division / square root, so each operation rounds once, as in the reference built without FMA
// contraction: a node's state after any number of substeps is bitwise the reference's, given the same exp and pow
// (bl_math.cuh).
#pragma once

#include <cstdint>

#include "bl_math.cuh"

namespace blg {

constexpr int kMaxCand = 64;               // BL_GPU_MAX_CANDIDATES
constexpr uint32_t kBeamAsleep = 1u << 31; // Beam meta: the beam's body sleeps (not stepped)
constexpr float kMaxNodeSpeed = 400.0f;    // softbody.h:153
// a beam's force scalar when it does not push this substep (a NaN no arithmetic makes: the GPU's NaNs are 0x7fffffff)
#define kNoPush __uint_as_float(0x7fc0beefu)
constexpr int kSurfCount = 11;

enum : uint32_t { NF_GROUND = 1, NF_FIXED = 2, NF_TYRE = 4, NF_RIM = 8, NF_CONTACTER = 16 };
enum : uint32_t { BT_NORMAL = 0, BT_ROPE = 1, BT_SUPPORT = 2 };
enum : uint32_t { BF_BROKEN = 1, BF_NO_DEFORM = 4, BF_NO_BREAK = 8, BF_SHOCK = 64 };
// body bits kept in each beam's meta word (bits 16-18): the body's allow_deform / allow_break / ductile
enum : uint32_t { BB_DEFORM = 1u << 16, BB_BREAK = 1u << 17, BB_DUCTILE = 1u << 18 };
enum : uint32_t { DEVERR_CANDIDATES = 1, DEVERR_NONFINITE = 2, DEVERR_TIMEOUT = 1u << 6 };

// Ground model (GroundModel, static_world.h:18-31): the values of ground_models() (static_world.cpp:85-114)
struct GroundModel {
    float va, ms, mc, t2, vs, alpha, strength, soft_depth, fluid_drag, fluid_density;
};

struct Box {      // StaticBox (static_world.h:121-131): no hull planes
    float cx, cy, cz, hx, hy, hz;
    float r[9];   // columns: local axes in world space (to_mat3 of its quaternion, math.h:166-174)
    float mnx, mny, mnz, mxx, mxy, mxz; // aabb
    int surface;
    float max_force;
};

struct Cyl {      // StaticCylinder (static_world.h:133-137)
    float bx, by, bz, radius, height;
    int surface;
};

// The static world as the kernels see it (by value as a kernel parameter)
struct Statics {
    int has_terrain, hnx, hnz, bx, bz;
    float cell, ox, oz;
    const float* h;          // nz x nx heights
    const uint8_t* surf;     // nz x nx surfaces
    const float* block_max;  // bz x bx maxima over 16 x 16 cells (Heightfield::update_bounds)
    float kill_y;
    int nboxes, ncyls;
    const Box* boxes;
    const Cyl* cyls;
    int gx, gz, nbig;        // box grid (StaticWorld::build_grid)
    float gox, goz, grid_cell;
    const int* cell_ptr;
    const int* cell_items;
    const int* big;
};

// A body on the device. The first 64 bytes are what the node kernel reads for every node.
struct alignas(64) Body {
    // hot: node kernel
    float fric;              // SoftBody::ground_friction (x rest_friction when resting: rest damping is not supported)
    float bounce, push_max, slop;
    float terrain_max;       // this frame's terrain culling height (World::Island::terrain_max)
    int sleeping;
    int nbox, ncyl;          // this frame's static candidates (-1: more than kMaxCand)
    int node0, nnodes, beam0, nbeams;
    int can_sleep;
    float sleep_speed;
    float max_speed, sleep_timer;
    // frame accumulators (atomics of the node kernel)
    float acc_mn[3], acc_mx[3];
    float acc_v2;
    int acc_contacts;
    // per frame results
    float aabb_mn[3], aabb_mx[3];
    int static_contacts, broken_beams, repaired;
    int fell_asleep, needs_repair;
    int is_fem;              // the body has a FEM frame: its nodes are integrated after the frame's implicit step
    int has_ext;             // constant node forces (bl_gpu_set_node_force) are added after gravity
    int box_ids[kMaxCand];
    int cyl_ids[kMaxCand];
    // contacts with other bodies (bl_contacts.cuh)
    int tri0, ntris;         // its collision triangles
    float crad;              // SoftBody::collision_radius
    float cfric;             // SoftBody::contact_friction
    float hull_depth;        // SoftBody::hull_depth
    float face_skin;         // SoftBody::face_skin
    int faces_only;          // SoftBody::faces_only
    int hull;                // it has hull (one-sided) triangles: SoftBody::hull_reach() = hull_depth
    int group;               // SoftBody::collision_group
    int contacters;          // it has NF_CONTACTER nodes
    int island;              // this frame: the first body of its island (-1: its island sleeps)
    int pairs;               // this frame: its island has contact pairs (its nodes finish after the contacts)
    int wake_request;        // SoftBody::wake_request
    int body_contacts;       // SoftBody::body_contacts (this frame)
    // air drag (SoftBody::clear_forces with air_drag / aero_cda, softbody.cpp:334-378)
    int drag;                // air_drag > 0 or aero_cda > 0
    float air_drag, aero_cda;
    int part_count;          // its parts (SoftBody::part_labels; 0: not labelled yet)
    int part_age;            // SoftBody::part_age_
    int part_key;            // the broken-beam count the labels were made at (the part key's only changing input here)
    int has_wheels;          // SoftBody::wheels (node tyres): their tyre patches share grip (k_tyres)
    int has_shocks;          // SoftBody::shocks: added after its beams (k_shocks, k_force)
};

// ------------------------------------------------------------------------------------------ math in the reference's order
struct v3 {
    float x, y, z;
};
__device__ __forceinline__ v3 V(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ v3 operator*(v3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float length(v3 a) { return sqrtf(dot(a, a)); }
// vec3 / float: times the reciprocal (math.h:56)
__device__ __forceinline__ v3 divs(v3 a, float s) {
    const float i = 1.0f / s;
    return {a.x * i, a.y * i, a.z * i};
}
__device__ __forceinline__ v3 normalize(v3 a) {
    const float l = length(a);
    return l > 1e-12f ? a * (1.0f / l) : V(0, 0, 0);
}
// std::min / std::max as evaluated by the reference
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }
__device__ __forceinline__ float clampf(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ float signf(float v) { return v < 0.0f ? -1.0f : 1.0f; }
__device__ __forceinline__ v3 vabs(v3 a) { return {fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }

// float atomics through the integer order of IEEE floats (no NaN)
__device__ __forceinline__ void atomic_min_f(float* a, float v) {
    if (v >= 0.0f) atomicMin((int*)a, __float_as_int(v));
    else atomicMax((unsigned int*)a, __float_as_uint(v));
}
__device__ __forceinline__ void atomic_max_f(float* a, float v) {
    if (v >= 0.0f) atomicMax((int*)a, __float_as_int(v));
    else atomicMin((unsigned int*)a, __float_as_uint(v));
}

__device__ __constant__ GroundModel c_ground[kSurfCount];

} // namespace blg
