/* beamlab_gpu.h - the C ABI of the B200-native soft-body substep.
 *
 * It replaces, for the bodies it holds, the stepping of BeamLab's `bl::phys::World` (src/phys/world.h:150-171):
 * gravity, RoR beam spring-dampers with plastic yield and breaking (SoftBody::compute_beam_forces,
 * src/phys/softbody.cpp:412-470), static contacts against the heightfield, boxes and cylinders
 * (World::collide_static, src/phys/world.cpp:781-899; StaticWorld::collide_point, src/phys/static_world.cpp:364-474;
 * primitive_collision, src/phys/static_world.cpp:8-51) and symplectic Euler integration
 * (SoftBody::integrate_nodes, src/phys/softbody.cpp:769-795), frame by frame as World::step_substeps
 * (src/phys/world.cpp:368-585) runs them, with the per-frame static candidate query, top speed and sleep.
 *
 * Plain C: pointers, sizes and POD records only. The node, node-info and beam records have the byte layout of the
 * reference's `Node` (softbody.h:43-48), `NodeInfo` (softbody.h:50-58) and `Beam` (softbody.h:71-85), so a host shim
 * can pass a SoftBody's vectors as they are.
 *
 * Threading: one context is used by one host thread at a time (as World is). Calls on a context are ordered on its
 * CUDA stream; bl_gpu_step_substeps is asynchronous, the download/stat calls synchronise that stream.
 *
 * Errors: every call returns BL_GPU_OK (0) or a negative BL_GPU_E* code; bl_gpu_error_string names it. The
 * reference's step has no return code (its failures show up as counters, src/phys/frame_fem.h:342-344 and
 * src/phys/world.h:111); those counters are in bl_world_stats. */
#ifndef BEAMLAB_GPU_H
#define BEAMLAB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BL_GPU_ABI_VERSION 7

enum {
    BL_GPU_OK = 0,
    BL_GPU_EINVAL = -1,       /* a bad argument (null pointer, index out of range, inconsistent sizes) */
    BL_GPU_ENOMEM = -2,       /* device or host allocation failed */
    BL_GPU_ECUDA = -3,        /* a CUDA call failed; bl_gpu_last_cuda_error has its code */
    BL_GPU_EUNSUPPORTED = -4, /* the body uses a feature this path does not step (shocks, joints, wheels, sheets ...) */
    BL_GPU_ELIMIT = -5,       /* a fixed capacity was exceeded (see the call's comment) */
    BL_GPU_ENODEVICE = -6,    /* no CUDA device of compute capability 10.0 */
    BL_GPU_ESTATE = -7        /* the call is not valid in the context's current state */
};

/* node flags (NodeFlag, softbody.h:29-39), beam types and flags (BeamType / BeamFlag, softbody.h:60-69) */
enum {
    BL_NF_GROUND = 1 << 0, BL_NF_FIXED = 1 << 1, BL_NF_TYRE = 1 << 2, BL_NF_RIM = 1 << 3, BL_NF_CONTACTER = 1 << 4,
    BL_NF_FRAME = 1 << 5, BL_NF_LOAD = 1 << 6, BL_NF_NO_MOUSE = 1 << 7, BL_NF_SELF_COLL = 1 << 8
};
enum { BL_BT_NORMAL = 0, BL_BT_ROPE = 1, BL_BT_SUPPORT = 2 };
enum {
    BL_BF_BROKEN = 1 << 0, BL_BF_INVISIBLE = 1 << 1, BL_BF_NO_DEFORM = 1 << 2, BL_BF_NO_BREAK = 1 << 3,
    BL_BF_WHEEL = 1 << 4, BL_BF_HYDRO = 1 << 5, BL_BF_SHOCK = 1 << 6
};

/* World settings the path reads (WorldSettings, src/phys/world.h:24-77) plus the device to run on */
typedef struct {
    float gravity[3];          /* m/s^2; the reference's default {0, -9.81, 0} */
    float dt;                  /* substep (s); default 0.0005 (2 kHz) */
    int32_t sleeping;          /* bodies at rest fall asleep (WorldSettings::sleeping) */
    float sleep_speed;         /* m/s (WorldSettings::sleep_speed) */
    float sleep_time;          /* s (WorldSettings::sleep_time) */
    int32_t device;            /* CUDA device ordinal */
    int32_t deterministic;     /* 1: every node sums its forces in the reference's order (bitwise equal results);
                                  the only mode of this version */
    float collision_hz;        /* WorldSettings::collision_hz (120): the contact pairs are searched again every
                                  ceil(1 / (collision_hz dt)) substeps and at each frame's start */
    int32_t inter_body_collisions; /* WorldSettings::inter_body_collisions (1) */
    int32_t max_pairs;         /* capacity of the contact pair list of all islands (default 2^21); more pairs in one
                                  search raise BL_GPU_DEVERR_PAIRS and that island's contacts are skipped. The search's
                                  triangle queries (a triangle against a hash or a fast body's grid) hold at least as
                                  many, and 8 x the collision triangles + 65,536: more - a pile-up of many fast bodies
                                  all in reach of one another - raise BL_GPU_DEVERR_PAIRS the same way */
    /* the FEM frames' implicit step (no counterpart in the reference, which always factors): */
    int32_t fem_solver;        /* BL_GPU_FEM_CHOLESKY (default: the reference's block Cholesky), BL_GPU_FEM_PCG (conjugate
                                  gradients, block-Jacobi, from zero), BL_GPU_FEM_PCG_LEARNED (from the energy-norm best
                                  combination of the learned per-node guess and the last solution, the preconditioner
                                  scaled by the learned 3x3 blocks), BL_GPU_FEM_PCG_PREVIOUS (from the last solution,
                                  scaled alike: the warm start without the network); a PCG solve that misses pcg_tol
                                  within pcg_max_iters falls back to the Cholesky for that substep */
    int32_t pcg_max_iters;     /* default 200 */
    float pcg_tol;             /* relative residual |A dv - rhs| / |rhs| to reach; default 1e-6 */
    int32_t fem_check_residual; /* 1: keep a copy of each assembled system and measure the residual of the solution the
                                   step took (bl_gpu_fem_stats); costs a copy of the system a substep */
    int32_t pcg_learned_scale; /* BL_GPU_FEM_PCG_LEARNED: 1 the learned 3x3 scale of the block preconditioner, 0 (default)
                                  none - measured on the plates, the scale as trained costs iterations */
    int32_t graphs;            /* 1 (default): a frame of n substeps is captured once as a CUDA graph and replayed; 0: its
                                  kernels are launched one by one every call (the plain path, one launch per kernel) */
    int32_t beam_kernel;       /* 0 (default): the beams' kernel streams the beam arrays through shared memory by bulk
                                  (TMA) copies and the nodes' kernel reads 4-byte incidences where the rig allows; 1:
                                  plain loads and 8-byte incidences. Results are the same. */
    int32_t fem_dense_front;   /* how the FEM step factors its system (the same pattern and fill as the reference's):
                                  3 (default): 1 while the frames' factorization makes at most 8 M block updates, 2 above;
                                  2: multifrontal - the columns grouped into dense fronts (supernodes of the elimination
                                  tree, small ones amalgamated), each factored by dense tiled kernels, level by level of the
                                  front tree; 1: block column by block column, with the top chain of the elimination tree
                                  (levels of one column each) as one dense front; 0: block column by block column in the
                                  reference's order of sums throughout. 2 and 1 differ from 0 in the order of the
                                  floating-point sums only. */
    /* launch shapes (results do not depend on them; beamlab_b200/autotune.py measures them for a device and workload): */
    int32_t force_block;       /* the nodes' force kernel's block size: 64, 128 or 256; 0 (default): 256 */
    int32_t integrate_block;   /* the integration kernel's block size: 64, 128 or 256; 0 (default): 256 */
    int32_t beams_per_sm;      /* the beams' persistent kernel's blocks an SM (at most what fits); 0 (default): what fits */
    float tyre_grip;           /* WorldSettings::tyre_grip (1): a factor on the tyres' friction (tyre_contact) */
    float bulk_wait_s;         /* (no counterpart in the reference) the beams kernel's bound on a wait for its own bulk
                                  copies, in seconds (default 1, at most 10): one that runs out raises
                                  BL_GPU_DEVERR_TIMEOUT, lets the copies in flight land and ends the block's work for that
                                  substep; 0 makes every such wait report as run out (for tests of that path) */
    int32_t contact_whole_max; /* (no counterpart in the reference) an island's contacts run whole - their order found
                                  over the island - up to this many (default and most: 6144); more run 512 at a time. The
                                  same results either way; 0 runs every island 512 at a time (for tests of that path) */
} bl_gpu_config;

enum { BL_GPU_FEM_CHOLESKY = 0, BL_GPU_FEM_PCG = 1, BL_GPU_FEM_PCG_LEARNED = 2, BL_GPU_FEM_PCG_PREVIOUS = 3 };

/* == bl::phys::Node (softbody.h:43-48): 32 bytes */
typedef struct {
    float p[3];
    float inv_mass;
    float v[3];
    float mass;
} bl_node;

/* == bl::phys::NodeInfo (softbody.h:50-58): 20 bytes */
typedef struct {
    uint16_t flags;
    uint8_t surface;
    uint8_t pad;
    float friction;
    float radius;
    int32_t frame;
    int32_t ror_id;
} bl_node_info;

/* == bl::phys::Beam (softbody.h:71-85): 52 bytes */
typedef struct {
    uint32_t a, b;
    float L, k, d;
    float max_pos, max_neg, strength, plastic, stress, L0, support_limit;
    uint8_t type, flags;
    uint16_t group;
} bl_beam;

/* == the fields of bl::phys::ShellSection (frame_fem.h:114-150) the shell step reads */
typedef struct {
    float E, nu, rho, t;       /* Young's modulus (Pa), Poisson's ratio, density (kg/m3), thickness (m) */
    float yield;               /* yield stress (Pa; 0: elastic): on a body with allow_deform its triangles flow
                                  (membrane and bending, eval_tris); with allow_break too BL_GPU_EUNSUPPORTED (its
                                  tears and bisections are topology events this path does not make) */
    float damping;             /* stiffness-proportional damping (s) */
    float drill;               /* the corners' drilling spring, a share of G t A */
} bl_shell_section;

/* == bl::phys::Triangle (softbody.h:138-147): 20 bytes. A collision triangle between three of the body's nodes
 * (SoftBody::add_triangle, softbody.h:958; rest_edge2 as SoftBody::finalize sets it, softbody.cpp:80). */
typedef struct {
    uint32_t a, b, c;
    uint8_t surface;
    uint8_t two_sided;         /* 0: a hull triangle - one-sided, its winding faces out */
    uint8_t torn;              /* stretched past 2.5x its longest rest edge: no collision */
    uint8_t pad;
    float rest_edge2;          /* longest rest edge, squared */
} bl_tri;

/* A triangle element between three body nodes, as FemFrame::add_tri makes it (frame_fem.cpp:201-209), and the mass
 * it put on its corners (ShellMesher::tri, fem_shell.cpp:17-31; <= 0: its section's areal mass) */
typedef struct {
    uint32_t a, b, c;
    uint16_t section;
    uint16_t pad;
    float mass;
} bl_fem_tri;

/* == the fields of bl::phys::FrameSection (frame_fem.h:90-112) the member step reads */
typedef struct {
    float E, G, rho;           /* Young's and shear moduli (Pa), density (kg/m3) */
    float A, Iy, Iz, J;        /* area (m2), second moments about the local y and z axes, torsion constant (m4) */
    float As_y, As_z;          /* shear areas along y and z (Timoshenko; 0: none) */
    float damping;             /* stiffness-proportional damping (s) */
    float axial;               /* a factor on the axial stiffness (1) */
    float joint_k;             /* BL_FJ_ELASTIC joints: rotational stiffness (N m/rad) */
    float Np, Mp, Tp;          /* plastic axial force (N), moment and torque (N m); Np 0: elastic. On a body with
                                  allow_deform the member yields (axial and Euler buckling, twist, radial-return hinges
                                  at its ends, the unload re-pass); with allow_break too BL_GPU_EUNSUPPORTED (its splits
                                  and tears are topology events this path does not make). A joint's damping and a
                                  mount's break force have no fields. */
    float hardening;           /* the plastic moment's growth over a hinge's first radian (0.25) */
} bl_frame_section;

/* the joints at a member's ends (FrameJoint, frame_fem.h:182-193) */
enum { BL_FJ_RIGID = 0, BL_FJ_BALL = 1, BL_FJ_HINGE_V = 2, BL_FJ_HINGE_H = 3, BL_FJ_SWIVEL = 4, BL_FJ_ELASTIC = 5 };

/* A member between two body nodes, as FemFrame::add_element makes it (frame_fem.cpp:211-222); mass: the mass it put on
 * its nodes (already in their masses; <= 0: its section's rho A L0), which sets the nodes' rotational inertia */
typedef struct {
    uint32_t a, b;
    uint16_t section;          /* into bl_fem_desc.frame_sections */
    uint8_t end_a, end_b;      /* BL_FJ_* */
    float mass;
} bl_fem_member;

/* A body's FEM frame (FemFrame, frame_fem.h:330-815): its add_element calls (the members) and its add_tri calls (the
 * triangles) - the frame nodes are numbered as those calls meet them, the members' first unless tris_first; no mounts
 * or springs. The
 * library does what the reference's FemFrame::finalize and analyse do (rest frames and shapes, inertias, the
 * minimum-degree ordering and the factor's pattern) and steps it implicitly every substep (FemFrame::solve,
 * frame_fem.cpp:2512-3027). */
typedef struct {
    int32_t n_sections;
    const bl_shell_section* sections;
    int32_t n_tris;
    const bl_fem_tri* tris;
    float theta;               /* WorldSettings::frame_theta (0.5) */
    float dissipation;         /* SoftBody::fem_dissipation, else WorldSettings::frame_dissipation (0.02) */
    int32_t n_frame_sections;
    const bl_frame_section* frame_sections;
    int32_t n_members;
    const bl_fem_member* members;
    int32_t tris_first;        /* 1: the add_tri calls came before the add_element calls */
} bl_fem_desc;

/* A wheel of tyre nodes (Wheel, softbody.h:468-498): its hub (axle0 on the side of the even tyre nodes, axle1) and its
 * tyre contact nodes (even: the ring on axle0's side, odd: the other), as the reference's vehicle builder makes them.
 * Its drive and brake torques come from bl_gpu_set_wheel_drive (0: free rolling). A ring tyre (Wheel::ring) is not
 * on this path. A node lies on one wheel once (else BL_GPU_EUNSUPPORTED). */
typedef struct bl_wheel {
    uint32_t axle0, axle1;
    int32_t n_nodes;
    const uint32_t* nodes;
    float radius, width;
    float mass;                /* its tyre nodes' mass (the brake's stop torque and the drive's reaction read it) */
    int32_t propulsed;         /* 0 none, 1 forward, 2 backward (the tangent turned round) */
    int32_t arm, near_attach;  /* the node the drive's reaction torque acts on and its nearer axle node (-1: none) */
} bl_wheel;

/* A shock (Shock, softbody.h:88-101) on one of the body's beams, which carries BL_BF_SHOCK: its force model (type 1:
 * shocks and bounded beams, 2: shocks2 with progressive rates and soft bump stops, 3: shocks3 with split damping) in
 * place of the beam's, added to the ends after all the beams' forces, in the order of the shocks (softbody.cpp:
 * 472-566). Every BL_BF_SHOCK beam has exactly one shock. */
typedef struct bl_shock {
    uint32_t beam;
    uint8_t type;
    uint8_t soft_bump;
    uint16_t pad;
    float spring, damp;
    float spring_in, damp_in, prog_spring_in, prog_damp_in;
    float spring_out, damp_out, prog_spring_out, prog_damp_out;
    float damp_in_slow, split_in, damp_in_fast, damp_out_slow, split_out, damp_out_fast;
    float short_bound, long_bound;   /* fractions of the beam's rest length */
    float bound_spring, bound_damp;  /* the bump stops' stiffness and damping */
} bl_shock;

/* One body: a SoftBody after finalize (softbody.cpp:76-83) - its arrays and the knobs of the explicit path
 * (softbody.h:650-700), its node wheels and shocks, and optionally its FEM frame of members and triangle elements.
 * Bodies with joints, ring tyres, driven or braked wheels, slide nodes, sheets, FEM mounts or grab are
 * rejected by the caller's shim (this record has no fields for them); BL_GPU_EUNSUPPORTED here: a FEM frame of
 * triangles whose nodes collide with the static world (NF_GROUND; a frame of members takes its nodes' static
 * contacts), tyre nodes on a body with a frame, beams on frame nodes, yielding sections on a body that breaks, a frame with collision
 * triangles, air drag, wheels or shocks, self collision, a node on two wheels. */
typedef struct {
    int32_t n_nodes;
    const bl_node* nodes;
    const bl_node_info* info;
    int32_t n_beams;
    const bl_beam* beams;
    float ground_friction;     /* SoftBody::ground_friction */
    float bounce;              /* SoftBody::bounce (-1: RoR's 80% of the approach) */
    float contact_push_max;    /* SoftBody::contact_push_max */
    float contact_slop;        /* SoftBody::contact_slop */
    int32_t allow_deform;      /* SoftBody::allow_deform */
    int32_t allow_break;       /* SoftBody::allow_break */
    int32_t ductile;           /* SoftBody::ductile */
    int32_t can_sleep;         /* SoftBody::can_sleep */
    float sleep_speed;         /* SoftBody::sleep_speed (0: the world's) */
    float max_speed;           /* SoftBody::max_speed at upload (the first frame's static query margin) */
    int32_t sleeping;          /* SoftBody::sleeping at upload */
    const bl_fem_desc* fem;    /* NULL: no FEM frame */
    /* contacts with other bodies' nodes (World::rebuild_pairs / collide_pairs): node-triangle pairs */
    int32_t n_tris;            /* SoftBody::tris (none on a body with a FEM frame) */
    const bl_tri* tris;
    float collision_radius;    /* SoftBody::collision_radius (0.05) */
    float contact_friction;    /* SoftBody::contact_friction (1) */
    float hull_depth;          /* SoftBody::hull_depth (0.3) */
    float face_skin;           /* SoftBody::face_skin (0.002) */
    int32_t faces_only;        /* SoftBody::faces_only */
    int32_t collision_group;   /* SoftBody::collision_group (0: none) */
    int32_t self_collision;    /* SoftBody::self_collision: not supported (BL_GPU_EUNSUPPORTED when set) */
    float air_drag;            /* SoftBody::air_drag (0: none): RoR's per-node drag on the velocity against its part's
                                  mean (softbody.cpp:334-378); a body with a FEM frame takes none */
    float aero_cda;            /* SoftBody::aero_cda (0: none): Cd A (m2) on each part's mean velocity, shared by mass */
    int32_t n_wheels;          /* SoftBody::wheels of node tyres (Wheel, softbody.h:468-498); their tyre nodes (NF_TYRE) */
    const struct bl_wheel* wheels; /* share each patch's grip */
    int32_t n_shocks;          /* SoftBody::shocks (none on a body with a FEM frame) */
    const struct bl_shock* shocks;
} bl_body_desc;

/* A body's runtime state (SoftBody::aabb, max_speed, sleeping, static_contacts, stats.broken_beams, sleep_timer) */
typedef struct {
    float aabb_min[3];
    float aabb_max[3];
    float max_speed;
    int32_t sleeping;
    int32_t static_contacts;   /* over the last frame's substeps */
    int32_t broken_beams;      /* since upload */
    float sleep_timer;
    int32_t repaired_nodes;    /* nodes World::repair_nodes reset, since upload */
    int32_t fem_failures;      /* FemFrame::solve_failures: failed factorizations and non-finite velocity changes */
    int32_t fem_clamps;        /* FemFrame::clamps: velocity changes cut to the safety limits */
    int32_t body_contacts;     /* SoftBody::body_contacts: contacts with other bodies over the last frame */
    int32_t wake_request;      /* SoftBody::wake_request: a moving body touched it while it slept */
} bl_body_state;

/* WorldStats (world.h:79-132), the fields this path fills, and the device's error word */
typedef struct {
    int32_t substeps;          /* of the last bl_gpu_step_substeps */
    int32_t active_bodies, sleeping_bodies, active_nodes, active_beams;
    int64_t total_substeps;    /* since the context was made */
    int64_t kernel_launches;   /* kernels this library launched since the context was made */
    uint32_t device_errors;    /* BL_GPU_DEVERR_* bits raised by the kernels */
    int64_t contacts;          /* contacts between bodies applied since the context was made */
    int64_t pair_searches;     /* an island's pair search (World::rebuild_pairs + near_pairs) counts one */
    int32_t pairs;             /* candidate pairs of all islands after the last search */
    int32_t islands;           /* islands of the last frame with contact pairs */
} bl_world_stats;

enum {
    BL_GPU_DEVERR_CANDIDATES = 1 << 0, /* a body's static candidate list overflowed BL_GPU_MAX_CANDIDATES */
    BL_GPU_DEVERR_NONFINITE = 1 << 1,  /* a body needed the repair of non-finite / runaway nodes */
    BL_GPU_DEVERR_PAIRS = 1 << 2,      /* the contact pair list (or the search's queries) overflowed bl_gpu_config.max_pairs */
    BL_GPU_DEVERR_ISLAND = 1 << 3,     /* an island with contact pairs held more than BL_GPU_MAX_ISLAND_BODIES bodies */
    BL_GPU_DEVERR_CONTACT_UNSUPPORTED = 1 << 5, /* a body with a FEM frame met another body's triangles (not stepped) */
    BL_GPU_DEVERR_TIMEOUT = 1 << 6     /* a kernel's bounded wait on its own bulk copies ran out (bulk_wait_s): the
                                          substep's beams were not all stepped */
};
#define BL_GPU_MAX_ISLAND_BODIES 256
#define BL_GPU_MAX_CANDIDATES 64

typedef struct bl_gpu_ctx bl_gpu_ctx;

/* Defaults of the reference's WorldSettings (world.h:25-60) into *cfg. */
void bl_gpu_default_config(bl_gpu_config* cfg);

/* A world on cfg->device (World::World). The context owns a CUDA stream unless one is given to each call. */
int bl_gpu_create(const bl_gpu_config* cfg, bl_gpu_ctx** out);
int bl_gpu_destroy(bl_gpu_ctx* ctx);

/* Statics, before the first step (StaticWorld, static_world.h:182-201). heights/surfaces: nz rows of nx samples,
 * x fastest (Heightfield::create + h()/surf(), static_world.h:52-70); surfaces may be NULL (grass). */
int bl_gpu_set_terrain(bl_gpu_ctx* ctx, int32_t nx, int32_t nz, float cell, float origin_x, float origin_z, const float* heights,
                       const uint8_t* surfaces);
/* StaticWorld::add_box(center, half, rot = quaternion x,y,z,w, surface); max_force as StaticBox::max_force (0: rigid) */
int bl_gpu_add_box(bl_gpu_ctx* ctx, const float center[3], const float half[3], const float quat[4], int32_t surface, float max_force);
/* a vertical cylinder (StaticCylinder, static_world.h:133-137) */
int bl_gpu_add_cylinder(bl_gpu_ctx* ctx, const float base[3], float radius, float height, int32_t surface);
/* StaticWorld::build_grid (static_world.cpp:308-338): without it boxes are never candidates, as in the reference */
int bl_gpu_build_grid(bl_gpu_ctx* ctx);
/* StaticWorld::kill_y (nodes below are frozen) */
int bl_gpu_set_kill_y(bl_gpu_ctx* ctx, float y);

/* World::add_body (world.cpp:283-289): copies the body in; *body_id is its index (0, 1, ... in order). */
int bl_gpu_add_body(bl_gpu_ctx* ctx, const bl_body_desc* desc, int32_t* body_id);

/* A constant force (N) on one node of a body, added every substep right after gravity - what a SoftBody::pre_substep
 * controller that pushes a node does (world.cpp:3261). Zero removes it. */
int bl_gpu_set_node_force(bl_gpu_ctx* ctx, int32_t body, int32_t node, const float force[3]);

/* A wheel's drive torque and brake torque (N m) from the next substep on, every substep - what a vehicle controller
 * that sets Wheel::torque and brake in its pre_substep hook does (compute_wheel_forces, softbody.cpp:691-767: the
 * torque spread over the tyre nodes along their tangents, the brake's stop torque, the reaction on the arm). */
int bl_gpu_set_wheel_drive(bl_gpu_ctx* ctx, int32_t body, int32_t wheel, float torque, float brake);

/* A body's wheels' Wheel::speed (the tread's tangential speed, m/s) and avg_speed; n the wheel count. Synchronous. */
int bl_gpu_download_wheels(bl_gpu_ctx* ctx, int32_t body, int32_t* n, float* speed, float* avg_speed);

/* SoftBody::wheel_speed and wheel_spin (softbody.cpp:723-766): the mean tread speed (m/s) and spin (rad/s) of the
 * body's forward-propelled wheels, for its drivetrain. A body with none reads 0: the reference starts both at 0
 * (softbody.h:1112-1113) and keeps the last value while no forward-propelled wheel steps, and this path's set of such
 * wheels never changes (detached wheels, which the reference skips, are not modelled: a shim keeps a body that detaches
 * a wheel on the reference's CPU path), so the two agree. Synchronous. */
int bl_gpu_wheel_speed(bl_gpu_ctx* ctx, int32_t body, float* wheel_speed, float* wheel_spin);

/* A body's FEM frame nodes (FemFrame::node / xd / q / w, frame_fem.h:331-350): body node, double position (3),
 * orientation (x y z w), angular velocity (3); n the frame node count (0: none). Any pointer may be NULL. */
int bl_gpu_download_fem(bl_gpu_ctx* ctx, int32_t body, int32_t* n, int32_t* node, double* xd, float* q, float* w);

/* A body's FEM triangles' plastic state (FrameTri::X, r0, dmg, frame_fem.h:153-181): the rest shape (6: the corners in
 * the element's plane, as a yielding membrane flowed it), the rest frames (12: x y z w per corner, the bending's
 * plastic rotations baked in), the plastic stretch reached; n the triangle count (0: none). Any pointer may be NULL. */
int bl_gpu_download_fem_tris(bl_gpu_ctx* ctx, int32_t body, int32_t* n, float* rest, float* frames, float* plastic_stretch);

/* World::step_substeps(n) (world.cpp:368-585): one frame of n substeps of every awake body, enqueued on `stream`
 * (a cudaStream_t; NULL: the context's own). Asynchronous. */
int bl_gpu_step_substeps(bl_gpu_ctx* ctx, int32_t n, void* stream);

/* Whole-body state transfers (synchronous on the context's stream): nodes in bl_node records, beams in bl_beam. */
int bl_gpu_download_nodes(bl_gpu_ctx* ctx, int32_t body, bl_node* out);
int bl_gpu_upload_nodes(bl_gpu_ctx* ctx, int32_t body, const bl_node* nodes);
int bl_gpu_download_beams(bl_gpu_ctx* ctx, int32_t body, bl_beam* out);
int bl_gpu_body_state(bl_gpu_ctx* ctx, int32_t body, bl_body_state* out);
int bl_gpu_stats(bl_gpu_ctx* ctx, bl_world_stats* out);
/* waits for everything enqueued on the context's stream */
int bl_gpu_synchronize(bl_gpu_ctx* ctx);

/* The nodes of all bodies back to back, in bl_node records (body after body, as added), asynchronous on `stream`
 * (NULL: the context's): one copy each way - the caller's buffer should be pinned, and is not to be touched until the
 * stream has passed the copy. n must be the total node count (bl_gpu_device_nodes). These are what a host shim that
 * keeps the reference's SoftBody arrays in step moves each frame. */
int bl_gpu_upload_all_nodes(bl_gpu_ctx* ctx, const bl_node* nodes, int32_t n, void* stream);
int bl_gpu_download_all_nodes(bl_gpu_ctx* ctx, bl_node* out, int32_t n, void* stream);

/* The device-resident node array (bl_node records of all bodies back to back, 16-byte aligned) and its length, for
 * callers that keep their own data on the GPU; each body's first node and beam. Valid until the next bl_gpu_add_body. */
int bl_gpu_device_nodes(bl_gpu_ctx* ctx, void** nodes, int32_t* total_nodes);
int bl_gpu_body_range(bl_gpu_ctx* ctx, int32_t body, int32_t* first_node, int32_t* n_nodes, int32_t* first_beam, int32_t* n_beams);

/* The implicit FEM step's solver counters (all frames of the context as one system) */
typedef struct {
    int64_t pcg_solves;        /* PCG solves run (fem_solver >= 1) */
    int64_t pcg_fallbacks;     /* of those, the ones that missed pcg_tol and were factored instead */
    int64_t pcg_iterations;    /* CG iterations over all solves */
    int32_t last_iterations;   /* of the last solve */
    int32_t pad;
    double last_pcg_residual;  /* relative residual the last PCG solve reached */
    double max_residual;       /* fem_check_residual: the largest relative residual of a solution the step took */
    double last_residual;      /* fem_check_residual: that of the last substep */
    int64_t columns;           /* the factor of all frames: block columns (frame nodes), */
    int64_t blocks;            /* off-diagonal 6 x 6 blocks, */
    int64_t updates;           /* block updates of a factorization (432 flops each), */
    int64_t levels;            /* elimination-tree levels */
    int64_t repasses;          /* unload re-passes: the steps' systems assembled and factored again where the step
                                  unloaded a flowing hinge, bar or twist of a yielding member */
    int64_t fronts;            /* fem_dense_front == 2: the multifrontal factorization's dense fronts (0 otherwise); */
    double factor_flops;       /* the flops of one factorization as this path runs it (multiplies and adds counted
                                  apart; the multifrontal's dense fronts include their explicit zeros) */
} bl_fem_stats;
int bl_gpu_fem_stats(bl_gpu_ctx* ctx, bl_fem_stats* out);

/* The learned warm start (BL_GPU_FEM_PCG_LEARNED; no counterpart in the reference): a per-frame-node MLP
 * 36 -> 64 -> 64 -> 64 -> 12 (ReLU), BF16 weights with FP32 accumulation, whose outputs are the PCG's initial dv guess
 * (3) and a 3 x 3 scale of its block preconditioner's translational part (9). Its features and targets are described
 * in beamlab_b200/csrc/bl_mlp.cuh. Parameters: one float vector of BL_GPU_MLP_PARAMS - W1 (64 x 36, row = output), b1,
 * W2 (64 x 64), b2, W3 (64 x 64), b3, W4 (12 x 64), b4. Every context starts with the weights of seed 1. */
#define BL_GPU_MLP_PARAMS 11468
#define BL_GPU_MLP_INPUTS 36
#define BL_GPU_MLP_OUTPUTS 12
int bl_gpu_mlp_init(bl_gpu_ctx* ctx, uint64_t seed);                    /* He-uniform weights, zero biases */
int bl_gpu_mlp_set_weights(bl_gpu_ctx* ctx, const float* w, int32_t n); /* n == BL_GPU_MLP_PARAMS; resets Adam */
int bl_gpu_mlp_get_weights(bl_gpu_ctx* ctx, float* w, int32_t n);
/* capacity > 0: from the next frame on, every substep's solve records one training sample per frame node (features,
 * targets from the solution the step took) into a ring of `capacity` samples (older ones are overwritten);
 * capacity 0: stop recording (the samples stay for bl_gpu_mlp_train). The frames' graphs are captured again. */
int bl_gpu_mlp_record(bl_gpu_ctx* ctx, int32_t capacity);
int bl_gpu_mlp_samples(bl_gpu_ctx* ctx, int32_t* n);
/* Adam (beta 0.9 / 0.999) on the recorded samples, shuffled each epoch (seeded), minibatches of `batch`; *loss: the
 * mean sample loss over the last epoch. Synchronous. */
int bl_gpu_mlp_train(bl_gpu_ctx* ctx, int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss);
/* The network on n samples (x: n x 36, y: n x 12; host memory), and the gradient of the loss
 * sum_s sum_o w_so (y_so - t_so)^2 / (2 n) over n samples with respect to the parameters (the BF16 values the
 * forward uses), and that loss. Synchronous; for checks against a CPU restatement. */
int bl_gpu_mlp_forward(bl_gpu_ctx* ctx, const float* x, int32_t n, float* y);
int bl_gpu_mlp_gradient(bl_gpu_ctx* ctx, const float* x, const float* t, const float* w, int32_t n, float* grad, float* loss);

/* The contact pairs (node, triangle) of the last pair search, island after island (islands in the order of their
 * first body, each island's pairs in the reference's order: World::Island::nt after rebuild_pairs + near_pairs,
 * world.cpp:1851-2598): 4 int32 a pair - the node's body, the node, the triangle's body, the triangle. Writes at most
 * `capacity` pairs; *n_pairs = all of them. Waits for the device. */
int bl_gpu_download_pairs(bl_gpu_ctx* ctx, int32_t* pairs, int32_t capacity, int32_t* n_pairs);

/* One frame of n substeps, like bl_gpu_step_substeps, with a timing event between its kernels; waits for it and
 * returns the GPU time of each kind of kernel (summed over the frame's substeps). */
typedef struct {
    int32_t substeps;
    float frame_ms;            /* the whole frame */
    float begin_ms;            /* the frame's start (static candidates per body) */
    float beams_ms;            /* the beams' forces, all substeps */
    float nodes_ms;            /* force_ms + contacts_ms + integrate_ms + fem_ms (search_ms apart) */
    float finish_ms;           /* the frame's end (bounds, repair, sleep) */
    float force_ms;            /* the nodes' forces (gravity, beams; the FEM frames' gather), all substeps */
    float contacts_ms;         /* the contacts between bodies (narrow phase, response) */
    float integrate_ms;        /* static contacts and integration */
    float fem_ms;              /* the FEM frames' implicit step */
    float search_ms;           /* the contacts' wake requests and pair searches (World::rebuild_pairs), all substeps */
} bl_frame_profile;
int bl_gpu_profile_frame(bl_gpu_ctx* ctx, int32_t n, void* stream, bl_frame_profile* out);

/* The symbolic phase of a FEM frame, on the host, no GPU needed: what bl_gpu_add_body computes for the frame of `fem`
 * over the body's nodes - FemFrame::analyse's exact minimum-degree order and factor pattern (frame_fem.cpp:544-860)
 * and FemFrame::finalize's rest shapes and inertias (frame_fem.cpp:224-260, 3075-3086). sizes[0..3] receive the frame
 * nodes, off-diagonal blocks, block updates and components; any array may be NULL (call once with NULLs for sizes):
 * perm (frame nodes), col_ptr (frame nodes + 1), row (blocks), upd (3 per update: pi, pj, target as the reference
 * stores them), rest (6 per triangle: its corners in its plane), inertia (frame nodes). */
int bl_fem_pattern(const bl_node* nodes, const bl_node_info* info, int32_t n_nodes, const bl_fem_desc* fem, int32_t sizes[4], int32_t* perm,
                   int32_t* col_ptr, int32_t* row, int32_t* upd, float* rest, float* inertia);

/* One substep - gravity, the beams' spring-dampers with yield and breaking, symplectic Euler - of one body whose
 * device buffers the caller owns, for callers that cannot let the library allocate GPU memory: their memory belongs to
 * another allocator (an engine's or a framework's pool), or they step where allocation is forbidden (a real-time frame
 * loop, a CUDA stream capture). No counterpart in the reference: it is the body part of bl_gpu_step_substeps without
 * a context, without statics and without the frame's bookkeeping. Only a plain beam body gets the node and beam states
 * bl_gpu_step_substeps gives it: gravity and beams (normal, rope, support) alone - no shocks (a BL_BF_SHOCK beam is
 * stepped as a beam with no force), no wheels or tyres, no air drag, no FEM frame, no contacts.
 * nodes / beams: device arrays of bl_node / bl_beam (in and out); inc_ptr (n_nodes + 1) / inc (2 n_beams): device
 * arrays listing each node's beams in beam order, a beam's index with bit 31 set where the node is its b end.
 * The caller guarantees every index: each beam's ends below n_nodes, each inc entry's beam below n_beams, inc_ptr
 * ascending within [0, 2 n_beams]; nothing on the GPU checks them.
 * Allocates nothing: its per-beam scratch is a fixed device array of BL_GPU_NOALLOC_MAX_BEAMS entries (16 MiB, held by
 * every GPU that loads the library until exit), so more beams return BL_GPU_ELIMIT. That array's address belongs to a
 * CUDA context: it is looked up on every call whose stream is not capturing and kept per context for calls made during
 * a capture, so the first call in a context should come before any stream capture. Calls whose kernels overlap on the
 * GPU share the scratch and race; order them on one stream. Asynchronous on `stream` (NULL: the legacy default
 * stream). */
#define BL_GPU_NOALLOC_MAX_BEAMS (1 << 20)
int bl_gpu_substep_noalloc(bl_node* nodes, int32_t n_nodes, bl_beam* beams, int32_t n_beams, const int32_t* inc_ptr, const int32_t* inc,
                           const float gravity[3], float dt, int32_t allow_deform, int32_t allow_break, int32_t ductile, void* stream);

const char* bl_gpu_error_string(int code);
int bl_gpu_last_cuda_error(bl_gpu_ctx* ctx);
int bl_gpu_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif
