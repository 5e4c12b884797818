/* Test infrastructure only: the CPU restatement of BeamLab's explicit substep. See softbody_oracle.h.
 *
 * Built with -ffp-contract=off: every float operation below happens in the reference's order, one rounding each, as the
 * reference's parity build does. Citations are to files of the reference project (zenkovich/beamlab). */
#include "softbody_oracle.h"
#include "orc_math.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ small vector math (src/core/math.h:46-80) */
typedef struct { float x, y, z; } v3;
static inline v3 V(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float vlen(v3 a) { return sqrtf(vdot(a, a)); }
/* vec3 / float multiplies by the reciprocal (math.h:56) */
static inline v3 vdivs(v3 a, float s) { float i = 1.0f / s; return V(a.x * i, a.y * i, a.z * i); }
static inline v3 vnormalize(v3 a) { float l = vlen(a); return l > 1e-12f ? vmul(a, 1.0f / l) : V(0, 0, 0); }
/* std::min / std::max as the reference's calls evaluate them */
static inline float fmin_(float a, float b) { return (b < a) ? b : a; }
static inline float fmax_(float a, float b) { return (a < b) ? b : a; }
static inline v3 vmin_(v3 a, v3 b) { return V(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)); }
static inline v3 vmax_(v3 a, v3 b) { return V(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z)); }
static inline v3 vabs_(v3 a) { return V(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
static inline float clampf_(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline float signf_(float v) { return v < 0.0f ? -1.0f : 1.0f; }
static inline int isfinite3(v3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }

typedef struct { v3 c[3]; } m3; /* column-major (math.h:105) */
static inline v3 m3mul(const m3* m, v3 v) { return vadd(vadd(vmul(m->c[0], v.x), vmul(m->c[1], v.y)), vmul(m->c[2], v.z)); }

typedef struct { v3 mn, mx; } aabb_t;
static inline aabb_t aabb_empty(void) { aabb_t a = {{1e30f, 1e30f, 1e30f}, {-1e30f, -1e30f, -1e30f}}; return a; }
static inline int aabb_overlaps(const aabb_t* a, const aabb_t* b) {
    return a->mn.x <= b->mx.x && a->mx.x >= b->mn.x && a->mn.y <= b->mx.y && a->mx.y >= b->mn.y && a->mn.z <= b->mx.z && a->mx.z >= b->mn.z;
}
static inline void aabb_expand(aabb_t* a, float r) { a->mn = vsub(a->mn, V(r, r, r)); a->mx = vadd(a->mx, V(r, r, r)); }

/* ------------------------------------------------------------------ constants */
enum { NF_GROUND = 1, NF_FIXED = 2, NF_TYRE = 4, NF_RIM = 8, NF_CONTACTER = 16 };            /* softbody.h:29-39 */
enum { BT_NORMAL = 0, BT_ROPE = 1, BT_SUPPORT = 2 };                                           /* softbody.h:60 */
enum { BF_BROKEN = 1, BF_NO_DEFORM = 4, BF_NO_BREAK = 8, BF_SHOCK = 64 };                      /* softbody.h:61-69 */
static const float kMaxNodeSpeed = 400.0f;                                                     /* softbody.h:153 */
#define SURF_COUNT 11

/* ground models (static_world.cpp:85-114): va, ms, mc, t2, vs, alpha, strength, soft_depth, fluid_drag, fluid_density */
typedef struct { float va, ms, mc, t2, vs, alpha, strength, soft_depth, fluid_drag, fluid_density; } gm_t;
static const gm_t kGround[SURF_COUNT] = {
    {3, 0.80f, 0.55f, 0.005f, 7, 2, 1, 0, 0, 0},           /* grass */
    {3, 0.80f, 0.58f, 0.006f, 4, 2, 1, 0, 0, 0},           /* dirt */
    {3, 1.20f, 0.75f, 0.010f, 6, 2, 1, 0, 0, 0},           /* asphalt */
    {3, 1.20f, 0.75f, 0.010f, 6, 2, 1, 0, 0, 0},           /* concrete */
    {3, 0.85f, 0.60f, 0.006f, 3, 2, 1, 0, 0, 0},           /* gravel */
    {2, 0.50f, 0.35f, 0.004f, 3, 2, 1, 0.12f, 60, 1500},   /* mud */
    {3, 0.70f, 0.55f, 0.0001f, 9, 2, 1, 0.03f, 20, 1600},  /* sand */
    {3, 0.95f, 0.70f, 0.007f, 8, 2, 1, 0, 0, 0},           /* rock */
    {3, 0.90f, 0.60f, 0.005f, 5, 2, 1, 0, 0, 0},           /* wood */
    {3, 0.70f, 0.40f, 0.001f, 3, 2, 1, 0, 0, 0},           /* metal */
    {1, 0.30f, 0.20f, 0.0001f, 3, 2, 1, 0, 0, 0},          /* ice */
};

/* ------------------------------------------------------------------ world state */
typedef struct {
    v3 center, half;
    m3 rot;
    uint8_t surface;
    float max_force;
    aabb_t aabb;
} box_t;
typedef struct { v3 base; float radius, height; uint8_t surface; } cyl_t;

typedef struct {
    int n_nodes, n_beams;
    v3 *p, *v, *force;
    float *inv_mass, *mass;
    uint16_t* flags;
    float *friction, *radius;
    uint32_t *a, *b;
    float *L, *k, *d, *max_pos, *max_neg, *strength, *plastic, *stress, *L0, *support_limit;
    uint8_t *btype, *bflags;
    OrcBodyParams prm;
    aabb_t aabb;
    float max_speed, sleep_timer;
    int sleeping, static_contacts, broken_beams;
    /* per frame: static candidates (World::Island::box_ids / cyl_ids / terrain_max, world.cpp:740-753) */
    int *box_ids, nbox, *cyl_ids, ncyl;
    float terrain_max;
} body_t;

struct OrcWorld {
    v3 gravity;
    float dt, sleep_speed, sleep_time;
    int sleeping;
    /* heightfield (static_world.h:52-110) */
    int has_terrain, hnx, hnz, bx, bz;
    float cell, ox, oz;
    float* h;
    uint8_t* surf;
    float* block_max;
    float kill_y;
    box_t* boxes;
    int nboxes;
    cyl_t* cyls;
    int ncyls;
    /* box grid (static_world.cpp:308-338) */
    float grid_cell, gox, goz;
    int gx, gz;
    int *cell_ptr, *cell_items, *big, nbig;
    body_t* bodies;
    int nbodies;
};

OrcWorld* orc_world_new(void) {
    OrcWorld* w = (OrcWorld*)calloc(1, sizeof(OrcWorld));
    w->gravity = V(0, -9.81f, 0);
    w->dt = 0.0005f;
    w->sleeping = 1;
    w->sleep_speed = 0.06f;
    w->sleep_time = 1.0f;
    w->kill_y = -200.0f;
    w->grid_cell = 16.0f;
    return w;
}

static void free_body(body_t* b) {
    void* ptrs[] = {b->p, b->v, b->force, b->inv_mass, b->mass, b->flags, b->friction, b->radius, b->a, b->b, b->L, b->k, b->d, b->max_pos, b->max_neg,
                    b->strength, b->plastic, b->stress, b->L0, b->support_limit, b->btype, b->bflags, b->box_ids, b->cyl_ids};
    for (size_t i = 0; i < sizeof(ptrs) / sizeof(ptrs[0]); i++) free(ptrs[i]);
}

void orc_world_free(OrcWorld* w) {
    if (!w) return;
    for (int i = 0; i < w->nbodies; i++) free_body(&w->bodies[i]);
    free(w->bodies);
    free(w->h), free(w->surf), free(w->block_max), free(w->boxes), free(w->cyls);
    free(w->cell_ptr), free(w->cell_items), free(w->big);
    free(w);
}

void orc_world_settings(OrcWorld* w, float gx, float gy, float gz, float dt, int sleeping, int multithreaded, int inter_body, float sleep_speed,
                        float sleep_time) {
    (void)multithreaded, (void)inter_body;
    w->gravity = V(gx, gy, gz);
    w->dt = dt;
    w->sleeping = sleeping;
    w->sleep_speed = sleep_speed;
    w->sleep_time = sleep_time;
}

void orc_set_kill_y(OrcWorld* w, float y) { w->kill_y = y; }

/* ------------------------------------------------------------------ heightfield */
static inline float hf_h(const OrcWorld* w, int x, int z) { return w->h[(size_t)z * w->hnx + x]; }

/* Heightfield::create + update_bounds (static_world.cpp:147-184): the block maxima over 16 x 16 cells, a vertex counting
 * for every block it borders */
void orc_set_terrain(OrcWorld* w, int nx, int nz, float cell, float ox, float oz, const float* heights, const uint8_t* surfaces) {
    free(w->h), free(w->surf), free(w->block_max);
    w->hnx = nx, w->hnz = nz, w->cell = cell, w->ox = ox, w->oz = oz;
    w->h = (float*)malloc(sizeof(float) * (size_t)nx * nz);
    w->surf = (uint8_t*)malloc((size_t)nx * nz);
    memcpy(w->h, heights, sizeof(float) * (size_t)nx * nz);
    if (surfaces) memcpy(w->surf, surfaces, (size_t)nx * nz);
    else memset(w->surf, 0, (size_t)nx * nz);
    const int kBlock = 16;
    w->bx = (nx - 1 + kBlock - 1) / kBlock;
    w->bz = (nz - 1 + kBlock - 1) / kBlock;
    w->block_max = (float*)malloc(sizeof(float) * (size_t)(w->bx > 0 ? w->bx : 1) * (w->bz > 0 ? w->bz : 1));
    for (int i = 0; i < w->bx * w->bz; i++) w->block_max[i] = -1e30f;
    for (int z = 0; z < nz; z++)
        for (int x = 0; x < nx; x++) {
            const float v = hf_h(w, x, z);
            int bx0 = (x - 1) / kBlock, bx1 = x / kBlock, bz0 = (z - 1) / kBlock, bz1 = z / kBlock;
            if (bx0 < 0) bx0 = 0;
            if (bz0 < 0) bz0 = 0;
            if (bx1 > w->bx - 1) bx1 = w->bx - 1;
            if (bz1 > w->bz - 1) bz1 = w->bz - 1;
            for (int bz = bz0; bz <= bz1; bz++)
                for (int bx = bx0; bx <= bx1; bx++) {
                    float* m = &w->block_max[(size_t)bz * w->bx + bx];
                    *m = fmax_(*m, v);
                }
        }
    w->has_terrain = 1;
}

/* Heightfield::sample (static_world.cpp:189-205): bilinear on the quad split along its (0,0)-(1,1) diagonal */
static int hf_sample(const OrcWorld* w, float x, float z, float* out_h, v3* n) {
    const float lx = (x - w->ox) / w->cell, lz = (z - w->oz) / w->cell;
    if (!(lx >= 0 && lz >= 0 && lx < w->hnx - 1 && lz < w->hnz - 1)) return 0;
    const int ix = (int)lx, iz = (int)lz;
    const float fx = lx - ix, fz = lz - iz;
    const float h00 = hf_h(w, ix, iz), h10 = hf_h(w, ix + 1, iz), h01 = hf_h(w, ix, iz + 1), h11 = hf_h(w, ix + 1, iz + 1);
    if (fmin_(fmin_(h00, h10), fmin_(h01, h11)) < -1e29f) return 0;
    if (fx > fz) {
        *out_h = h00 + (h10 - h00) * fx + (h11 - h10) * fz;
        *n = vnormalize(V(-(h10 - h00) / w->cell, 1.0f, -(h11 - h10) / w->cell));
    } else {
        *out_h = h00 + (h11 - h01) * fx + (h01 - h00) * fz;
        *n = vnormalize(V(-(h11 - h01) / w->cell, 1.0f, -(h01 - h00) / w->cell));
    }
    return 1;
}

/* Heightfield::surface_at (static_world.cpp:213-218) */
static uint8_t hf_surface_at(const OrcWorld* w, float x, float z) {
    int ix = (int)lroundf((x - w->ox) / w->cell), iz = (int)lroundf((z - w->oz) / w->cell);
    ix = ix < 0 ? 0 : (ix > w->hnx - 1 ? w->hnx - 1 : ix);
    iz = iz < 0 ? 0 : (iz > w->hnz - 1 ? w->hnz - 1 : iz);
    return w->surf[(size_t)iz * w->hnx + ix];
}

/* Heightfield::max_height (static_world.cpp:220-231); C's integer division truncates as C++'s does */
static float hf_max_height(const OrcWorld* w, float x0, float z0, float x1, float z1) {
    const int kBlock = 16;
    int bx0 = (int)floorf((x0 - w->ox) / w->cell) / kBlock, bx1 = (int)floorf((x1 - w->ox) / w->cell) / kBlock;
    int bz0 = (int)floorf((z0 - w->oz) / w->cell) / kBlock, bz1 = (int)floorf((z1 - w->oz) / w->cell) / kBlock;
    if (bx0 < 0) bx0 = 0;
    if (bz0 < 0) bz0 = 0;
    if (bx1 > w->bx - 1) bx1 = w->bx - 1;
    if (bz1 > w->bz - 1) bz1 = w->bz - 1;
    float m = -1e30f;
    for (int bz = bz0; bz <= bz1; bz++)
        for (int bx = bx0; bx <= bx1; bx++) m = fmax_(m, w->block_max[(size_t)bz * w->bx + bx]);
    return m;
}

/* ------------------------------------------------------------------ boxes, cylinders, grid */
/* to_mat3 (math.h:166-174) */
static m3 quat_to_m3(float x, float y, float z, float w) {
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
    m3 m;
    m.c[0] = V(1 - 2 * (yy + zz), 2 * (xy + wz), 2 * (xz - wy));
    m.c[1] = V(2 * (xy - wz), 1 - 2 * (xx + zz), 2 * (yz + wx));
    m.c[2] = V(2 * (xz + wy), 2 * (yz - wx), 1 - 2 * (xx + yy));
    return m;
}

/* StaticWorld::add_box + StaticBox::update_aabb (static_world.cpp:242-246, 298-306); max_force: StaticBox::max_force */
void orc_add_box(OrcWorld* w, float cx, float cy, float cz, float hx, float hy, float hz, float qx, float qy, float qz, float qw, int surface,
                 float max_force) {
    w->boxes = (box_t*)realloc(w->boxes, sizeof(box_t) * (size_t)(w->nboxes + 1));
    box_t* b = &w->boxes[w->nboxes++];
    b->center = V(cx, cy, cz);
    b->half = V(hx, hy, hz);
    b->rot = quat_to_m3(qx, qy, qz, qw);
    b->surface = (uint8_t)surface;
    b->max_force = max_force;
    const v3 e = vadd(vadd(vmul(vabs_(b->rot.c[0]), b->half.x), vmul(vabs_(b->rot.c[1]), b->half.y)), vmul(vabs_(b->rot.c[2]), b->half.z));
    b->aabb.mn = vsub(b->center, e);
    b->aabb.mx = vadd(b->center, e);
}

void orc_add_cylinder(OrcWorld* w, float bx, float by, float bz, float radius, float height, int surface) {
    w->cyls = (cyl_t*)realloc(w->cyls, sizeof(cyl_t) * (size_t)(w->ncyls + 1));
    cyl_t* c = &w->cyls[w->ncyls++];
    c->base = V(bx, by, bz), c->radius = radius, c->height = height, c->surface = (uint8_t)surface;
}

/* StaticWorld::build_grid (static_world.cpp:308-338): 16 m cells over the boxes' bounds; a box over more than 64 cells
 * is kept in the list of big boxes */
void orc_build_grid(OrcWorld* w) {
    free(w->cell_ptr), free(w->cell_items), free(w->big);
    w->cell_ptr = w->cell_items = w->big = NULL;
    w->nbig = 0;
    aabb_t all = aabb_empty();
    for (int i = 0; i < w->nboxes; i++) all.mn = vmin_(all.mn, w->boxes[i].aabb.mn), all.mx = vmax_(all.mx, w->boxes[i].aabb.mx);
    for (int i = 0; i < w->ncyls; i++) {
        const cyl_t* c = &w->cyls[i];
        const v3 lo = vsub(c->base, V(c->radius, 0, c->radius)), hi = vadd(c->base, V(c->radius, c->height, c->radius));
        all.mn = vmin_(all.mn, lo), all.mx = vmax_(all.mx, lo);
        all.mn = vmin_(all.mn, hi), all.mx = vmax_(all.mx, hi);
    }
    if (!(all.mn.x <= all.mx.x)) {
        w->gx = w->gz = 0;
        return;
    }
    w->gox = all.mn.x, w->goz = all.mn.z;
    int gx = (int)ceilf((all.mx.x - all.mn.x) / w->grid_cell) + 1, gz = (int)ceilf((all.mx.z - all.mn.z) / w->grid_cell) + 1;
    w->gx = gx < 1 ? 1 : gx, w->gz = gz < 1 ? 1 : gz;
    const int ncell = w->gx * w->gz;
    int* cnt = (int*)calloc((size_t)ncell + 1, sizeof(int));
    w->big = (int*)malloc(sizeof(int) * (size_t)(w->nboxes + 1));
    /* two passes: count, then fill in box order (each cell's list in box order, as push_back makes it) */
    for (int pass = 0; pass < 2; pass++) {
        for (int i = 0; i < w->nboxes; i++) {
            const aabb_t* a = &w->boxes[i].aabb;
            const int x0 = (int)((a->mn.x - w->gox) / w->grid_cell), x1 = (int)((a->mx.x - w->gox) / w->grid_cell);
            const int z0 = (int)((a->mn.z - w->goz) / w->grid_cell), z1 = (int)((a->mx.z - w->goz) / w->grid_cell);
            if ((x1 - x0 + 1) * (z1 - z0 + 1) > 64) {
                if (pass == 0) w->big[w->nbig++] = i;
                continue;
            }
            for (int z = z0; z <= z1; z++)
                for (int x = x0; x <= x1; x++) {
                    if (pass == 0) cnt[z * w->gx + x + 1]++;
                    else w->cell_items[cnt[z * w->gx + x]++] = i;
                }
        }
        if (pass == 0) {
            for (int c = 0; c < ncell; c++) cnt[c + 1] += cnt[c];
            w->cell_ptr = (int*)malloc(sizeof(int) * ((size_t)ncell + 1));
            memcpy(w->cell_ptr, cnt, sizeof(int) * ((size_t)ncell + 1));
            w->cell_items = (int*)malloc(sizeof(int) * (size_t)(cnt[ncell] + 1));
        }
    }
    free(cnt);
}

/* StaticWorld::query (static_world.cpp:340-362): the big boxes, then the grid cells' boxes without repeats, then every
 * cylinder; appended in that order */
static void statics_query(const OrcWorld* w, const aabb_t* b, int** boxes_out, int* nbox, int** cyl_out, int* ncyl) {
    int cap = w->nboxes + 1, n = 0;
    int* out = (int*)malloc(sizeof(int) * (size_t)cap);
    for (int k = 0; k < w->nbig; k++)
        if (aabb_overlaps(&w->boxes[w->big[k]].aabb, b)) out[n++] = w->big[k];
    if (w->gx > 0) {
        int x0 = (int)((b->mn.x - w->gox) / w->grid_cell), x1 = (int)((b->mx.x - w->gox) / w->grid_cell);
        int z0 = (int)((b->mn.z - w->goz) / w->grid_cell), z1 = (int)((b->mx.z - w->goz) / w->grid_cell);
        x0 = x0 < 0 ? 0 : x0, z0 = z0 < 0 ? 0 : z0;
        x1 = x1 > w->gx - 1 ? w->gx - 1 : x1, z1 = z1 > w->gz - 1 ? w->gz - 1 : z1;
        if (b->mx.x >= w->gox && b->mx.z >= w->goz)
            for (int z = z0; z <= z1; z++)
                for (int x = x0; x <= x1; x++)
                    for (int q = w->cell_ptr[z * w->gx + x]; q < w->cell_ptr[z * w->gx + x + 1]; q++) {
                        const int i = w->cell_items[q];
                        if (!aabb_overlaps(&w->boxes[i].aabb, b)) continue;
                        int dup = 0;
                        for (int k = 0; k < n; k++)
                            if (out[k] == i) { dup = 1; break; }
                        if (!dup) out[n++] = i;
                    }
    }
    int* co = (int*)malloc(sizeof(int) * (size_t)(w->ncyls + 1));
    int nc = 0;
    for (int i = 0; i < w->ncyls; i++) {
        const cyl_t* c = &w->cyls[i];
        if (b->mx.x >= c->base.x - c->radius && b->mn.x <= c->base.x + c->radius && b->mx.z >= c->base.z - c->radius && b->mn.z <= c->base.z + c->radius &&
            b->mx.y >= c->base.y && b->mn.y <= c->base.y + c->height)
            co[nc++] = i;
    }
    free(*boxes_out), free(*cyl_out);
    *boxes_out = out, *nbox = n, *cyl_out = co, *ncyl = nc;
}

/* ------------------------------------------------------------------ contacts */
typedef struct { v3 normal; float depth; uint8_t surface; float max_force; } contact_t;

/* StaticWorld::collide_point (static_world.cpp:364-474): the deepest contact of a sphere over the terrain, the listed
 * boxes and cylinders (a later one only if strictly deeper) */
static int collide_point(const OrcWorld* w, v3 p, float r, const int* box_ids, int nbox, const int* cyl_ids, int ncyl, int test_terrain, contact_t* out) {
    int hit = 0;
    out->depth = 0;
    out->max_force = 0;
    if (test_terrain && w->has_terrain) {
        float th;
        v3 n;
        if (hf_sample(w, p.x, p.z, &th, &n)) {
            const float dd = (th - p.y) * n.y + r;
            if (dd > 0) {
                out->depth = dd;
                out->normal = n;
                out->surface = hf_surface_at(w, p.x, p.z);
                hit = 1;
            }
        }
    }
    for (int k = 0; k < nbox; k++) {
        const box_t* b = &w->boxes[box_ids[k]];
        if (p.x < b->aabb.mn.x - r || p.x > b->aabb.mx.x + r || p.y < b->aabb.mn.y - r || p.y > b->aabb.mx.y + r || p.z < b->aabb.mn.z - r ||
            p.z > b->aabb.mx.z + r)
            continue;
        const v3 rel = vsub(p, b->center);
        const v3 l = V(vdot(rel, b->rot.c[0]), vdot(rel, b->rot.c[1]), vdot(rel, b->rot.c[2]));
        const v3 q = V(clampf_(l.x, -b->half.x, b->half.x), clampf_(l.y, -b->half.y, b->half.y), clampf_(l.z, -b->half.z, b->half.z));
        const v3 dvec = vsub(l, q);
        const float dist2 = vdot(dvec, dvec);
        float depth;
        v3 nl;
        if (dist2 > 1e-12f) {
            if (dist2 >= r * r) continue;
            const float dist = sqrtf(dist2);
            depth = r - dist;
            nl = vdivs(dvec, dist);
        } else {
            const v3 pen = vsub(b->half, vabs_(l));
            if (pen.x <= pen.y && pen.x <= pen.z) depth = pen.x, nl = V(signf_(l.x), 0, 0);
            else if (pen.y <= pen.z) depth = pen.y, nl = V(0, signf_(l.y), 0);
            else depth = pen.z, nl = V(0, 0, signf_(l.z));
            depth += r;
        }
        if (depth > out->depth) {
            out->depth = depth;
            out->normal = m3mul(&b->rot, nl);
            out->surface = b->surface;
            out->max_force = b->max_force;
            hit = 1;
        }
    }
    for (int k = 0; k < ncyl; k++) {
        const cyl_t* c = &w->cyls[cyl_ids[k]];
        const v3 rel = vsub(p, c->base);
        if (rel.y < -r || rel.y > c->height + r) continue;
        if (fabsf(rel.x) >= c->radius + r || fabsf(rel.z) >= c->radius + r) continue;
        const float dxz = sqrtf(rel.x * rel.x + rel.z * rel.z);
        const float side = c->radius + r - dxz;
        const float top = c->height + r - rel.y;
        if (side <= 0) continue;
        float depth;
        v3 n;
        if (top < side && rel.y > c->height * 0.5f) depth = top, n = V(0, 1, 0);
        else depth = side, n = dxz > 1e-6f ? V(rel.x / dxz, 0, rel.z / dxz) : V(1, 0, 0);
        if (depth > out->depth) {
            out->depth = depth;
            out->normal = n;
            out->surface = c->surface;
            hit = 1;
        }
    }
    return hit;
}

/* primitive_collision (static_world.cpp:8-51): RoR's ground response - cancel the normal force, take 80% of the approach
 * speed and a fifth of the penetration (capped), then adhesion or Stribeck friction */
static v3 primitive_collision(v3 F, v3 vel, float mass, v3 normal, float dt, const gm_t* gm, float pen, float friction_coef, float push_max, float slop,
                              float restitution) {
    v3 out = V(0, 0, 0);
    const float Vn = vdot(vel, normal);
    const float Fn = vdot(F, normal);
    const float sgl = gm->soft_depth;
    if (sgl > 0 && pen >= 0) {
        out = vadd(out, vmul(vel, -gm->fluid_drag * fmin_(1.0f, pen / sgl + 0.2f)));
        float Fb = gm->fluid_density * fmin_(pen, sgl) * 9.807f * 0.02f;
        if (Vn >= 0 && Fn < 0 && Fb > -Fn) Fb = -Fn;
        out = vadd(out, vmul(normal, Fb));
    }
    if (pen >= sgl) {
        float R = -Fn;
        const float take = restitution >= 0 ? 1.0f + fmin_(restitution, 0.95f) : 0.8f;
        if (Vn < 0) R -= (take * Vn - fmin_(0.2f * fmax_(0.0f, pen - sgl - slop) / dt, push_max)) * mass / dt;
        if (R > 0) {
            const v3 slipF = vsub(F, vmul(normal, Fn));
            v3 slip = vsub(vel, vmul(normal, Vn));
            const float sv = vlen(slip);
            if (sv > 1e-9f) slip = vdivs(slip, sv);
            else slip = V(0, 0, 0);
            const float G = R * gm->strength * friction_coef;
            const float stop = mass * sv / dt;
            if (sv < gm->va && G > 0 && vlen(slipF) <= gm->ms * G) {
                out = vadd(out, vsub(vsub(vmul(normal, R), vmul(slip, fmin_(gm->ms * G * (1.0f - orc_expf(-sv / gm->va)), stop))), slipF));
            } else {
                const float g = gm->mc + (gm->ms - gm->mc) * orc_expf(-orc_powf(sv / gm->vs, gm->alpha));
                out = vadd(out, vsub(vmul(normal, R), vmul(slip, fmin_((g + fmin_(gm->t2 * sv, 5.0f)) * G, fmax_(0.0f, stop + vdot(slipF, slip))))));
            }
        }
    }
    return out;
}

void orc_primitive_collision(const float* F, const float* vel, float mass, const float* normal, float dt, int surface, float pen, float friction_coef,
                             float push_max, float slop, float restitution, float* out) {
    const v3 r = primitive_collision(V(F[0], F[1], F[2]), V(vel[0], vel[1], vel[2]), mass, V(normal[0], normal[1], normal[2]), dt,
                                     &kGround[surface < SURF_COUNT ? surface : 0], pen, friction_coef, push_max, slop, restitution);
    out[0] = r.x, out[1] = r.y, out[2] = r.z;
}

/* ------------------------------------------------------------------ bodies */
#define ALLOC(ptr, n) ptr = calloc((size_t)(n) + 1, sizeof(*(ptr)))

/* SoftBody::add_node / add_beam / finalize / compute_aabb (softbody.cpp:8-40, 76-83, 271-275) */
int orc_add_body(OrcWorld* w, int n_nodes, const float* pos, const float* vel, const float* mass, const uint16_t* nflags, const float* friction,
                 const float* radius, int n_beams, const uint32_t* ab, const float* k, const float* d, const float* strength, const float* deform,
                 const uint8_t* btype, const uint8_t* bflags, int n_tris, const uint32_t* tri, const OrcBodyParams* p) {
    (void)n_tris, (void)tri;
    w->bodies = (body_t*)realloc(w->bodies, sizeof(body_t) * (size_t)(w->nbodies + 1));
    body_t* b = &w->bodies[w->nbodies];
    memset(b, 0, sizeof(*b));
    b->n_nodes = n_nodes, b->n_beams = n_beams;
    ALLOC(b->p, n_nodes), ALLOC(b->v, n_nodes), ALLOC(b->force, n_nodes), ALLOC(b->inv_mass, n_nodes), ALLOC(b->mass, n_nodes);
    ALLOC(b->flags, n_nodes), ALLOC(b->friction, n_nodes), ALLOC(b->radius, n_nodes);
    ALLOC(b->a, n_beams), ALLOC(b->b, n_beams), ALLOC(b->L, n_beams), ALLOC(b->k, n_beams), ALLOC(b->d, n_beams), ALLOC(b->max_pos, n_beams);
    ALLOC(b->max_neg, n_beams), ALLOC(b->strength, n_beams), ALLOC(b->plastic, n_beams), ALLOC(b->stress, n_beams), ALLOC(b->L0, n_beams);
    ALLOC(b->support_limit, n_beams), ALLOC(b->btype, n_beams), ALLOC(b->bflags, n_beams);
    for (int i = 0; i < n_nodes; i++) {
        b->p[i] = V(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        b->v[i] = V(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        b->mass[i] = mass[i];
        b->inv_mass[i] = (nflags[i] & NF_FIXED) || mass[i] <= 0 ? 0.0f : 1.0f / mass[i];
        b->flags[i] = nflags[i], b->friction[i] = friction[i], b->radius[i] = radius[i];
    }
    for (int j = 0; j < n_beams; j++) {
        b->a[j] = ab[2 * j], b->b[j] = ab[2 * j + 1];
        const float len = vlen(vsub(b->p[b->a[j]], b->p[b->b[j]]));
        b->L[j] = b->L0[j] = fmax_(1e-3f, len); /* finalize's rest length (softbody.cpp:77-79) */
        b->k[j] = k[j], b->d[j] = d[j];
        b->max_pos[j] = deform[j], b->max_neg[j] = -deform[j], b->strength[j] = strength[j];
        b->plastic[j] = 0, b->stress[j] = 0, b->support_limit[j] = 4.0f;
        b->btype[j] = btype[j], b->bflags[j] = bflags[j];
    }
    b->prm = *p;
    b->aabb = aabb_empty();
    for (int i = 0; i < n_nodes; i++) b->aabb.mn = vmin_(b->aabb.mn, b->p[i]), b->aabb.mx = vmax_(b->aabb.mx, b->p[i]);
    return w->nbodies++;
}

/* SoftBody::compute_beam_forces (softbody.cpp:412-470), after clear_forces' gravity (softbody.cpp:330-377, no drag) */
static void beam_forces(const OrcWorld* w, body_t* b) {
    for (int i = 0; i < b->n_nodes; i++) b->force[i] = vmul(w->gravity, b->mass[i]);
    const int deform = b->prm.allow_deform, brk = b->prm.allow_break;
    for (int j = 0; j < b->n_beams; j++) {
        if (b->bflags[j] & (BF_BROKEN | BF_SHOCK)) continue;
        const uint32_t ia = b->a[j], ib = b->b[j];
        const v3 dis = vsub(b->p[ia], b->p[ib]);
        const float len2 = vdot(dis, dis);
        if (len2 < 1e-12f) continue;
        const float inv_len = 1.0f / sqrtf(len2);
        const float len = len2 * inv_len;
        const float diff = len - b->L[j];
        const v3 dv = vsub(b->v[ia], b->v[ib]);
        float kk = b->k[j], dd = b->d[j];
        if (b->btype[j] == BT_ROPE) {
            if (diff < 0) kk = 0, dd *= 0.1f;
        } else if (b->btype[j] == BT_SUPPORT) {
            if (diff > 0) {
                kk = 0;
                dd *= 0.1f;
                if (brk && diff > b->L[j] * b->support_limit[j]) {
                    b->bflags[j] |= BF_BROKEN;
                    b->broken_beams++;
                    continue;
                }
            }
        }
        float slen = -kk * diff - dd * vdot(dv, dis) * inv_len;
        if (deform && !(b->bflags[j] & BF_NO_DEFORM) && kk != 0) {
            if (slen > b->max_pos[j] && diff < 0) {
                const float yield_len = b->max_pos[j] / kk;
                const float def = diff + yield_len * (1.0f - b->plastic[j]);
                const float Lold = b->L[j];
                b->L[j] = fmax_(fmin_(0.1f, 0.3f * b->L0[j]), b->L[j] + def);
                slen = slen - (slen - b->max_pos[j]) * 0.5f;
                if (b->L[j] < Lold) b->max_pos[j] *= Lold / b->L[j];
            } else if (slen < b->max_neg[j] && diff > 0) {
                const float yield_len = b->max_neg[j] / kk;
                const float def = diff + yield_len * (1.0f - b->plastic[j]);
                const float Lold = b->L[j];
                b->L[j] = b->L[j] + def;
                slen = slen - (slen - b->max_neg[j]) * 0.5f;
                if (Lold > 0 && b->L[j] > Lold) b->max_neg[j] *= b->L[j] / Lold;
                if (!b->prm.ductile) b->strength[j] -= def * kk;
            }
        }
        if (brk && fabsf(slen) > b->strength[j] && !(b->bflags[j] & BF_NO_BREAK)) {
            b->bflags[j] |= BF_BROKEN;
            b->broken_beams++;
            continue;
        }
        b->stress[j] = slen;
        const v3 fv = vmul(dis, slen * inv_len);
        b->force[ia] = vadd(b->force[ia], fv);
        b->force[ib] = vsub(b->force[ib], fv);
    }
}

/* World::collide_static for plain nodes (world.cpp:781-870; no tyres, plates or yielding obstacles' frames) */
static void collide_static(const OrcWorld* w, body_t* b, float dt, int* contacts) {
    const float fric_body = b->prm.ground_friction * 1.0f; /* resting needs rest damping: off */
    for (int i = 0; i < b->n_nodes; i++) {
        if (!(b->flags[i] & NF_GROUND) || b->inv_mass[i] <= 0) continue;
        if (b->p[i].y < w->kill_y) {
            b->v[i] = V(0, 0, 0);
            b->inv_mass[i] = 0;
            continue;
        }
        const float r = b->radius[i];
        const v3 p = b->p[i];
        const int near_terrain = w->has_terrain && p.y - r <= b->terrain_max + 0.05f;
        if (!near_terrain && b->nbox == 0 && b->ncyl == 0) continue;
        int bids[16], cids[16];
        const int *bp = b->box_ids, *cp = b->cyl_ids;
        int nb = b->nbox, nc = b->ncyl;
        if (b->nbox <= 16 && b->ncyl <= 16) {
            nb = nc = 0;
            const float rr = r + 0.01f;
            for (int q = 0; q < b->nbox; q++) {
                const aabb_t* a = &w->boxes[b->box_ids[q]].aabb;
                if (p.x >= a->mn.x - rr && p.x <= a->mx.x + rr && p.y >= a->mn.y - rr && p.y <= a->mx.y + rr && p.z >= a->mn.z - rr && p.z <= a->mx.z + rr)
                    bids[nb++] = b->box_ids[q];
            }
            for (int q = 0; q < b->ncyl; q++) {
                const cyl_t* cy = &w->cyls[b->cyl_ids[q]];
                const float cr = cy->radius + rr;
                if (fabsf(p.x - cy->base.x) <= cr && fabsf(p.z - cy->base.z) <= cr && p.y >= cy->base.y - rr && p.y <= cy->base.y + cy->height + rr)
                    cids[nc++] = b->cyl_ids[q];
            }
            bp = bids, cp = cids;
            if (!near_terrain && nb == 0 && nc == 0) continue;
        }
        contact_t c = {{0, 0, 0}, 0, 0, 0};
        if (!collide_point(w, p, r, bp, nb, cp, nc, near_terrain, &c)) continue;
        (*contacts)++;
        const gm_t* gm = &kGround[c.surface < SURF_COUNT ? c.surface : 0];
        const float fc = b->friction[i] * fric_body;
        if (c.max_force > 0) {
            v3 f = primitive_collision(b->force[i], b->v[i], b->mass[i], c.normal, dt, gm, c.depth, fc, b->prm.contact_push_max, b->prm.contact_slop, -1.0f);
            const float fl = vlen(f);
            if (fl > c.max_force) f = vmul(f, c.max_force / fl);
            b->force[i] = vadd(b->force[i], f);
        } else {
            const v3 f = primitive_collision(b->force[i], b->v[i], b->mass[i], c.normal, dt, gm, c.depth, fc, b->prm.contact_push_max, b->prm.contact_slop,
                                             b->prm.bounce);
            b->force[i] = vadd(b->force[i], f);
        }
    }
}

/* SoftBody::integrate_nodes (softbody.cpp:769-795) */
static void integrate(body_t* b, float dt, aabb_t* box, float* max_v2_out) {
    float max_v2 = *max_v2_out;
    v3 mn = box->mn, mx = box->mx;
    for (int i = 0; i < b->n_nodes; i++) {
        if (b->inv_mass[i] > 0) {
            v3 v = vadd(b->v[i], vmul(b->force[i], b->inv_mass[i] * dt));
            float v2 = vdot(v, v);
            if (v2 > kMaxNodeSpeed * kMaxNodeSpeed) {
                v = vmul(v, kMaxNodeSpeed / sqrtf(v2));
                v2 = kMaxNodeSpeed * kMaxNodeSpeed;
            } else if (!(v2 >= 0.0f)) {
                v = V(0, 0, 0);
                v2 = 0;
            }
            b->v[i] = v;
            b->p[i] = vadd(b->p[i], vmul(v, dt));
            max_v2 = v2 > max_v2 ? v2 : max_v2;
        }
        mn = vmin_(mn, b->p[i]);
        mx = vmax_(mx, b->p[i]);
    }
    box->mn = mn, box->mx = mx;
    *max_v2_out = max_v2;
}

static int cmp_float(const void* x, const void* y) {
    const float a = *(const float*)x, b = *(const float*)y;
    return (a > b) - (a < b);
}

/* World::repair_nodes (world.cpp:4022-4111) for bodies of nodes and beams: bad nodes (not finite, too fast, flung
 * 300 m from the body's median) take their good beam neighbours' mean, isolated ones the median at rest */
static int repair_nodes(body_t* b) {
    const int n = b->n_nodes;
    float* xs = (float*)malloc(sizeof(float) * (size_t)(n + 1));
    float* ys = (float*)malloc(sizeof(float) * (size_t)(n + 1));
    float* zs = (float*)malloc(sizeof(float) * (size_t)(n + 1));
    int m = 0;
    for (int i = 0; i < n; i++)
        if (isfinite3(b->p[i])) xs[m] = b->p[i].x, ys[m] = b->p[i].y, zs[m] = b->p[i].z, m++;
    if (m == 0) {
        free(xs), free(ys), free(zs);
        return -1;
    }
    qsort(xs, (size_t)m, sizeof(float), cmp_float);
    qsort(ys, (size_t)m, sizeof(float), cmp_float);
    qsort(zs, (size_t)m, sizeof(float), cmp_float);
    const v3 med = V(xs[m / 2], ys[m / 2], zs[m / 2]);
    free(xs), free(ys), free(zs);
    const float reach = 300.0f;
    uint8_t* bad = (uint8_t*)calloc((size_t)n + 1, 1);
    int nbad = 0;
    for (int i = 0; i < n; i++) {
        const int finite = isfinite3(b->p[i]) && isfinite3(b->v[i]);
        const float lim = 0.9f * kMaxNodeSpeed;
        if (!finite || vdot(b->v[i], b->v[i]) > lim * lim || vlen(vsub(b->p[i], med)) > reach) bad[i] = 1, nbad++;
    }
    if (nbad == 0 || nbad * 2 > n) {
        free(bad);
        return nbad == 0 ? 0 : -1;
    }
    const int reset = nbad;
    v3* sp = (v3*)malloc(sizeof(v3) * (size_t)(n + 1));
    v3* sv = (v3*)malloc(sizeof(v3) * (size_t)(n + 1));
    int* cnt = (int*)malloc(sizeof(int) * (size_t)(n + 1));
    for (int pass = 0; pass < 8 && nbad > 0; pass++) {
        for (int i = 0; i < n; i++) sp[i] = sv[i] = V(0, 0, 0), cnt[i] = 0;
        for (int j = 0; j < b->n_beams; j++) {
            if (b->bflags[j] & BF_BROKEN) continue;
            const uint32_t x = b->a[j], y = b->b[j];
            if (bad[x] && !bad[y]) sp[x] = vadd(sp[x], b->p[y]), sv[x] = vadd(sv[x], b->v[y]), cnt[x]++;
            else if (bad[y] && !bad[x]) sp[y] = vadd(sp[y], b->p[x]), sv[y] = vadd(sv[y], b->v[x]), cnt[y]++;
        }
        for (int i = 0; i < n; i++)
            if (bad[i] && cnt[i] > 0) {
                b->p[i] = vdivs(sp[i], (float)cnt[i]);
                b->v[i] = vdivs(sv[i], (float)cnt[i]);
                bad[i] = 0;
                nbad--;
            }
    }
    for (int i = 0; i < n; i++)
        if (bad[i]) b->p[i] = med, b->v[i] = V(0, 0, 0);
    free(sp), free(sv), free(cnt), free(bad);
    b->aabb = aabb_empty();
    for (int i = 0; i < n; i++) b->aabb.mn = vmin_(b->aabb.mn, b->p[i]), b->aabb.mx = vmax_(b->aabb.mx, b->p[i]);
    b->max_speed = 0;
    for (int i = 0; i < n; i++) b->max_speed = fmax_(b->max_speed, vlen(b->v[i]));
    return reset;
}

/* World::update_sleep (world.cpp:4113-4157) for bodies without sheets or rest damping */
static void update_sleep(const OrcWorld* w, body_t* b, float frame_time) {
    if (!w->sleeping || !b->prm.can_sleep) {
        b->sleep_timer = 0;
        return;
    }
    const float rest = fmax_(w->sleep_speed, b->prm.sleep_speed);
    if (b->max_speed < rest) {
        b->sleep_timer += frame_time;
        if (b->sleep_timer > w->sleep_time) {
            b->sleeping = 1; /* fall_asleep (softbody.h:773-779) */
            for (int i = 0; i < b->n_nodes; i++) b->v[i] = V(0, 0, 0);
        }
    } else {
        b->sleep_timer = 0;
    }
}

/* World::step_substeps (world.cpp:368-585) for bodies that do not touch each other: each awake body is an island of its
 * own (build_islands, world.cpp:636-762), stepped for the whole frame (simulate_island, world.cpp:3211-4020) */
void orc_step_substeps(OrcWorld* w, int n) {
    const float dt = w->dt;
    const float frame_time = (float)n * dt;
    for (int bi = 0; bi < w->nbodies; bi++) {
        body_t* b = &w->bodies[bi];
        if (!w->sleeping) b->sleeping = 0;
        if (b->sleeping) continue;
        /* the island's static candidates over the body's box grown by its travel (world.cpp:738-753) */
        aabb_t a = b->aabb;
        aabb_expand(&a, fmin_(b->max_speed, 200.0f) * frame_time * 2.0f + 0.5f);
        statics_query(w, &a, &b->box_ids, &b->nbox, &b->cyl_ids, &b->ncyl);
        b->terrain_max = w->has_terrain ? hf_max_height(w, a.mn.x, a.mn.z, a.mx.x, a.mx.z) + 0.0f : -1e30f;
        /* simulate_island's top speed before the first substep (world.cpp:3217-3222) */
        float m2 = 0;
        for (int i = 0; i < b->n_nodes; i++) m2 = fmax_(m2, vdot(b->v[i], b->v[i]));
        b->max_speed = sqrtf(m2);
        b->static_contacts = 0;
        for (int s = 0; s < n; s++) {
            beam_forces(w, b);
            int contacts = 0;
            collide_static(w, b, dt / 1.0f, &contacts);
            aabb_t box = aabb_empty();
            float v2 = 0;
            integrate(b, dt / 1.0f, &box, &v2);
            b->static_contacts += contacts;
            b->aabb = box; /* merge of the node ranges (world.cpp:3905-3916) */
            const float ms = sqrtf(v2);
            if (ms > b->max_speed) b->max_speed = ms;
        }
        /* numerical trouble: repair (world.cpp:3964-3979) */
        const v3 ext = vsub(b->aabb.mx, b->aabb.mn);
        if (!isfinite(b->aabb.mn.x) || !isfinite(b->aabb.mx.y) || fmax_(ext.x, fmax_(ext.y, ext.z)) > 800.0f || b->max_speed > kMaxNodeSpeed * 0.9f) {
            const int fixed = repair_nodes(b);
            if (fixed < 0) {
                for (int i = 0; i < b->n_nodes; i++) {
                    if (!isfinite3(b->p[i])) b->p[i] = V(0, -1000, 0);
                    b->v[i] = V(0, 0, 0);
                    b->inv_mass[i] = 0;
                }
                b->aabb = aabb_empty();
                for (int i = 0; i < b->n_nodes; i++) b->aabb.mn = vmin_(b->aabb.mn, b->p[i]), b->aabb.mx = vmax_(b->aabb.mx, b->p[i]);
                b->sleeping = 1;
                continue;
            }
        }
        update_sleep(w, b, frame_time);
    }
}

int orc_body_nodes(OrcWorld* w, int body) { return w->bodies[body].n_nodes; }
int orc_body_beams(OrcWorld* w, int body) { return w->bodies[body].n_beams; }

void orc_get_nodes(OrcWorld* w, int body, float* pos, float* vel, float* inv_mass, float* mass) {
    const body_t* b = &w->bodies[body];
    for (int i = 0; i < b->n_nodes; i++) {
        memcpy(pos + 3 * i, &b->p[i], 12);
        memcpy(vel + 3 * i, &b->v[i], 12);
        if (inv_mass) inv_mass[i] = b->inv_mass[i];
        if (mass) mass[i] = b->mass[i];
    }
}

void orc_set_nodes(OrcWorld* w, int body, const float* pos, const float* vel) {
    body_t* b = &w->bodies[body];
    for (int i = 0; i < b->n_nodes; i++) {
        memcpy(&b->p[i], pos + 3 * i, 12);
        memcpy(&b->v[i], vel + 3 * i, 12);
    }
}

void orc_get_beams(OrcWorld* w, int body, float* L, float* max_pos, float* max_neg, float* strength, float* stress, uint8_t* flags) {
    const body_t* b = &w->bodies[body];
    for (int j = 0; j < b->n_beams; j++)
        L[j] = b->L[j], max_pos[j] = b->max_pos[j], max_neg[j] = b->max_neg[j], strength[j] = b->strength[j], stress[j] = b->stress[j], flags[j] = b->bflags[j];
}

void orc_get_body(OrcWorld* w, int body, float* out) {
    const body_t* b = &w->bodies[body];
    out[0] = b->aabb.mn.x, out[1] = b->aabb.mn.y, out[2] = b->aabb.mn.z;
    out[3] = b->aabb.mx.x, out[4] = b->aabb.mx.y, out[5] = b->aabb.mx.z;
    out[6] = b->max_speed;
    out[7] = b->sleeping ? 1.0f : 0.0f;
    out[8] = (float)b->static_contacts;
    out[9] = (float)b->broken_beams;
    out[10] = b->sleep_timer;
}

/* the portable exp / pow (orc_math.h), for tests of their accuracy against libm */
float orc_math_exp(float x) { return orc_expf(x); }
float orc_math_pow(float x, float y) { return orc_powf(x, y); }
