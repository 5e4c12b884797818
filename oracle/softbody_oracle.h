/* Test infrastructure only (the checker, never the product): a plain-C restatement of BeamLab's explicit soft-body
 * substep - gravity, RoR beam spring-dampers with plastic yield and breaking, static contacts against a heightfield,
 * boxes and vertical cylinders, symplectic Euler integration - and of the per-frame bookkeeping around it (static
 * candidate query, top speed, sleep). Each function cites the reference file:line it restates. Parity with the reference
 * is pinned by tests that step the same rigs through this code and through the reference compiled from its sources
 * (oracle/Makefile) and require bitwise equal node states.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library. */
#ifndef BEAMLAB_SOFTBODY_ORACLE_H
#define BEAMLAB_SOFTBODY_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OrcWorld OrcWorld;

/* per-body knobs (SoftBody fields, softbody.h:650-700) - same layout as the reference driver's RefBodyParams */
typedef struct {
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
} OrcBodyParams;

OrcWorld* orc_world_new(void);
void orc_world_free(OrcWorld* w);
void orc_world_settings(OrcWorld* w, float gx, float gy, float gz, float dt, int sleeping, int multithreaded, int inter_body, float sleep_speed,
                        float sleep_time);
void orc_set_terrain(OrcWorld* w, int nx, int nz, float cell, float ox, float oz, const float* heights, const uint8_t* surfaces);
void orc_add_box(OrcWorld* w, float cx, float cy, float cz, float hx, float hy, float hz, float qx, float qy, float qz, float qw, int surface,
                 float max_force);
void orc_add_cylinder(OrcWorld* w, float bx, float by, float bz, float radius, float height, int surface);
void orc_build_grid(OrcWorld* w);
void orc_set_kill_y(OrcWorld* w, float y);
int orc_add_body(OrcWorld* w, int n_nodes, const float* pos, const float* vel, const float* mass, const uint16_t* nflags, const float* friction,
                 const float* radius, int n_beams, const uint32_t* ab, const float* k, const float* d, const float* strength, const float* deform,
                 const uint8_t* btype, const uint8_t* bflags, int n_tris, const uint32_t* tri, const OrcBodyParams* p);
void orc_step_substeps(OrcWorld* w, int n);
int orc_body_nodes(OrcWorld* w, int body);
int orc_body_beams(OrcWorld* w, int body);
void orc_get_nodes(OrcWorld* w, int body, float* pos, float* vel, float* inv_mass, float* mass);
void orc_set_nodes(OrcWorld* w, int body, const float* pos, const float* vel);
void orc_get_beams(OrcWorld* w, int body, float* L, float* max_pos, float* max_neg, float* strength, float* stress, uint8_t* flags);
void orc_get_body(OrcWorld* w, int body, float* out);

/* single ground-contact response (static_world.cpp:8-51) for unit tests of the formula */
void orc_primitive_collision(const float* F, const float* vel, float mass, const float* normal, float dt, int surface, float pen, float friction_coef,
                             float push_max, float slop, float restitution, float* out);

/* the oracle's portable exp and pow (orc_math.h) */
float orc_math_exp(float x);
float orc_math_pow(float x, float y);

#ifdef __cplusplus
}
#endif
#endif
