// Contacts between bodies: islands, the candidate pairs of nodes and collision triangles, their narrow phase and the
// contact response in the reference's pair order.
//
// Reference: World::build_islands (world.cpp:636-762), World::rebuild_pairs (world.cpp:1851-2308: node-triangle
// pairs only - no capsules, plate mid points or self collision), World::fast_pairs (world.cpp:2314-2520),
// World::near_pairs (world.cpp:2525-2598), World::pair_detect (world.cpp:2807-2858), World::collide_pairs
// (world.cpp:2964-3023) with contact_force<1,3> and hull_push_out<3> (world.cpp:59-120), the wake requests of sleeping
// bodies (world.cpp:2983-2995, 3333-3337).
//
// Layout. Collision triangles of all bodies back to back: int4 (a, b, c as global node indices; flags: bit 0 two-sided,
// bit 1 torn, bits 8.. the body) and their longest rest edge squared. Each frame k_islands labels every body with the
// first body of its island (the reference numbers islands in that order and keeps each island's bodies in body
// order). An island with two or more bodies has contact pairs: the contacts add to its nodes' forces (fnode: gravity
// and beams, k_force) before k_integrate takes the static contacts and integrates.
//
// The pair search runs on the substeps the reference rebuilds on (the frame's first and every rebuild interval after):
// one CTA per island (k_rebuild) sets up the island's search - margins, cell size, partners, the slow bodies' spatial
// hash, the fast bodies' dense grids - and lists its queries (a triangle against a hash or a grid); the queries of all
// islands are counted, placed and written by the whole GPU (bl_pair_search.cuh), the pairs near_pairs keeps in the
// reference's order. Every substep k_detect finds the contacts of all pairs in parallel and k_collide applies them one
// island per CTA, pair after pair: contact_force cancels the force accumulated so far on both sides, so the order
// within an island is the reference's.
#pragma once

#include "bl_kernels.cuh"

namespace blg {

constexpr int kIslMaxBodies = 256;     // bodies of one island with contact pairs (more: DEVERR_ISLAND)
constexpr int kGridCells = 48 * 48 * 48;
constexpr float kFastSpeed = 8.0f;     // world.cpp:1881
constexpr float kTornStretch2 = 2.5f * 2.5f; // softbody.h:154
enum : uint32_t { TF_TWO_SIDED = 1, TF_TORN = 2 };
enum : uint32_t { DEVERR_PAIRS = 4, DEVERR_ISLAND = 8, DEVERR_CONTACT_UNSUPPORTED = 32 };

struct IslSearch;
struct ContactRec;

struct Contacts {
    int4* tri;                 // a, b, c, flags | body << 8
    const float* tri_rest2;
    int* parent;               // per body: union-find
    float* ibox;               // per body: island box (6)
    int* isl_live;             // per root body: the island has an awake body
    int* isl_cnt;              // per root body: its bodies
    int* isl_nodes;            // per root body: its nodes
    int* isl_idx;              // per root body: its rank among the islands with pairs
    int* isl_noff;             // per root body: first node of its scratch
    int* isl_poff;             // per root body: its pairs in `pairs`
    int* isl_pcnt;
    int* isl_contacts;         // per root body: this frame's contacts (stats)
    int* pair_total;           // pairs of all islands (reset before each rebuild)
    int2* pairs;               // (node, triangle), global indices
    float4* hit_a;             // per pair: bary.xyz, pen
    float4* hit_b;             // per pair: normal.xyz, w = 1 when the pair is in contact
    uint32_t* hbits;           // per 32 pairs: bit j set when pair 32 w + j is in contact
    int* hidx;                 // per island's pair range: its contacts' pair indices, in pair order
    ContactRec* crec;          // the contacts' records of the islands that run whole (a substep's, taken in turn)
    int* crec_n;               // records taken this substep (reset by k_detect)
    int crec_cap;
    int whole_max;             // contacts an island runs whole at most (bl_gpu_config.contact_whole_max)
    int max_pairs;
    // rebuild scratch
    int* pt_node;              // hashed nodes of an island, in order
    int* pt_body;
    int4* pt_cell;
    int* bk_start;             // buckets (4 n + 65 per island)
    int* bk_fill;
    int* bk_items;             // hashed nodes by bucket
    int* run_end;
    int* g_start;              // fast grids: each fast body's cells' starts (a pool of cell_cap)
    int* g_fill;
    int* g_items;              // fast grids' nodes, each listed once, in the lowest cell of its travel
    float4* g_rec;             // ... in the same order: position, reach of its travel (|v| x travel)
    int* g_hi;                 // ... the highest cell of its travel (x | y << 8 | z << 16)
    int4* sb_cell;             // slow hash items in bucket order: cell, body
    float4* sb_pos;            // ... position, node (bits)
    IslSearch* isl;            // per island with pairs (isl_idx): what its queries read
    int4* q_group;             // query groups: island (isl_idx), kind | k << 1 | ko << 9, triangles, first query
    int2* q_chunk;             // chunks of kQueryChunk queries of one group: group, first triangle of the chunk
    int* q_count;              // per query (a triangle of a group): its pairs, then their running sum over the island
    int* sc;                   // search counters: [0] queries [1] groups [2] chunks [3] grid cells [4] ptmp
    int2* ptmp;                // the count pass's pairs, query by query (ptmp_cap)
    int* q_tmp;                // per query with pairs: its pairs in ptmp (-1: not kept)
    int ptmp_cap;
    int q_cap, grp_cap, chunk_cap, cell_cap;
    int* counters;             // [0] pair searches [1] contacts [2] pairs of the searches
    int interval;              // rebuild interval in substeps (world.cpp:1887)
    float dt;
    float wake_speed;          // WorldSettings::sleep_speed
};

// ------------------------------------------------------------------------------------------ geometry (reference order)
__device__ __forceinline__ v3 cross(v3 a, v3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
__device__ __forceinline__ float length2(v3 a) { return dot(a, a); }
__device__ __forceinline__ v3 vmin3(v3 a, v3 b) { return {smin(a.x, b.x), smin(a.y, b.y), smin(a.z, b.z)}; }
__device__ __forceinline__ v3 vmax3(v3 a, v3 b) { return {smax(a.x, b.x), smax(a.y, b.y), smax(a.z, b.z)}; }
__device__ __forceinline__ v3 neg(v3 a) { return {-a.x, -a.y, -a.z}; }
__device__ __forceinline__ v3 nd_p(const float4* nd, int i) {
    const float4 p = nd[2 * i];
    return V(p.x, p.y, p.z);
}
__device__ __forceinline__ v3 nd_v(const float4* nd, int i) {
    const float4 v = nd[2 * i + 1];
    return V(v.x, v.y, v.z);
}
__device__ __forceinline__ float max_edge2(v3 a, v3 b, v3 c) { return smax(length2(b - a), smax(length2(c - b), length2(a - c))); }

// world.cpp:23-25 (the int products wrap, as the reference's do)
__device__ __forceinline__ uint32_t cell_hash(int x, int y, int z) {
    return ((uint32_t)x * 73856093u) ^ ((uint32_t)y * 19349663u) ^ ((uint32_t)z * 83492791u);
}

// closest_on_triangle (softbody.h:158-190, Ericson 5.1.5)
__device__ v3 closest_on_triangle(v3 p, v3 a, v3 b, v3 c, v3& bary) {
    const v3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0 && d2 <= 0) {
        bary = V(1, 0, 0);
        return a;
    }
    const v3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0 && d4 <= d3) {
        bary = V(0, 1, 0);
        return b;
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const float v = d1 / (d1 - d3);
        bary = V(1 - v, v, 0);
        return a + ab * v;
    }
    const v3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0 && d5 <= d6) {
        bary = V(0, 0, 1);
        return c;
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const float w = d2 / (d2 - d6);
        bary = V(1 - w, 0, w);
        return a + ac * w;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        bary = V(0, 1 - w, w);
        return b + (c - b) * w;
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    bary = V(1 - v - w, v, w);
    return a + ab * v + ac * w;
}

// near_triangle (world.cpp:1135-1142)
__device__ __forceinline__ bool near_triangle(v3 p, v3 a, v3 b, v3 c, v3 tu, float r, bool two_sided, float depth) {
    const float s = dot(p - a, tu);
    v3 bary;
    if (two_sided) return fabsf(s) <= r && length2(closest_on_triangle(p, a, b, c, bary) - p) <= r * r;
    if (s > r || s < -r - depth) return false;
    const v3 q = p - tu * s;
    return length2(closest_on_triangle(q, a, b, c, bary) - q) <= r * r;
}

__device__ __forceinline__ bool outside(v3 p, v3 mn, v3 mx) { return p.x < mn.x || p.y < mn.y || p.z < mn.z || p.x > mx.x || p.y > mx.y || p.z > mx.z; }

// ------------------------------------------------------------------------------------------ block helpers
// exclusive scan of one int per thread of the block; *total: the block's sum. Every thread of the block calls it.
__device__ int block_scan_excl(int v, int& total, int* s_warp) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < nw ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) s_warp[lane] = t;
    }
    __syncthreads();
    const int before = (w > 0 ? s_warp[w - 1] : 0) + x - v;
    total = s_warp[nw - 1];
    __syncthreads();
    return before;
}

// a[0..n) := its inclusive prefix sums, in place, by the whole block: each thread sums a contiguous run, one block scan
// of the runs' sums, each thread rewrites its run (two block scans' barriers however long the array; the same integers
// as scanning it 1,024 entries at a time)
__device__ void block_scan_incl_inplace(int* a, int n, int* s_warp) {
    const int nt = blockDim.x, per = (n + nt - 1) / nt;
    const int lo = min(n, (int)threadIdx.x * per), hi = min(n, lo + per);
    int sum = 0;
    for (int i = lo; i < hi; i++) sum += a[i];
    int tot;
    int run = block_scan_excl(sum, tot, s_warp);
    for (int i = lo; i < hi; i++) run += a[i], a[i] = run;
}

// ------------------------------------------------------------------------------------------ islands (once a frame)
__device__ __forceinline__ int uf_find(volatile int* parent, int x) {
    while (true) {
        const int p = parent[x];
        if (p == x) return x;
        x = p;
    }
}
__device__ void uf_union(int* parent, int a, int b) {
    while (true) {
        a = uf_find(parent, a), b = uf_find(parent, b);
        if (a == b) return;
        if (a > b) {
            const int t = a;
            a = b, b = t;
        }
        if (atomicCAS(&parent[b], b, a) == b) return; // (the larger root under the smaller: a component's root is its first body)
    }
}

// World::build_islands (world.cpp:636-720) for bodies that can touch: node-triangle contacts only (no capsules or
// collision volumes). One block. Bodies with FEM frames take no contacts here: one that would is flagged
// (DEVERR_CONTACT_UNSUPPORTED) and stays in an island of its own.
__global__ void __launch_bounds__(1024) k_islands(Body* __restrict__ bodies, int nb, float frame_time, int world_sleeping, Contacts C,
                                                  uint32_t* __restrict__ deverr) {
    __shared__ int s_warp[32];
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        Body& B = bodies[i];
        if (!world_sleeping) B.sleeping = 0;
        C.parent[i] = i;
        C.isl_live[i] = 0, C.isl_cnt[i] = 0, C.isl_nodes[i] = 0, C.isl_pcnt[i] = 0, C.isl_contacts[i] = 0;
        const float m = (B.sleeping ? 0.05f : smin(B.max_speed, 200.0f) * frame_time * 2.0f + 0.3f) + (B.hull ? B.hull_depth : 0.0f);
        float* bx = C.ibox + 6 * i;
        bx[0] = B.aabb_mn[0] - m, bx[1] = B.aabb_mn[1] - m, bx[2] = B.aabb_mn[2] - m;
        bx[3] = B.aabb_mx[0] + m, bx[4] = B.aabb_mx[1] + m, bx[5] = B.aabb_mx[2] + m;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const Body& Bi = bodies[i];
        const float* a = C.ibox + 6 * i;
        for (int j = i + 1; j < nb; j++) {
            const float* b = C.ibox + 6 * j;
            if (!(a[0] <= b[3] && a[3] >= b[0] && a[1] <= b[4] && a[4] >= b[1] && a[2] <= b[5] && a[5] >= b[2])) continue;
            const Body& Bj = bodies[j];
            if (Bi.sleeping && Bj.sleeping) continue;
            if (Bi.group != 0 && Bi.group == Bj.group) continue;
            const bool can = (Bi.contacters && Bj.ntris > 0) || (Bj.contacters && Bi.ntris > 0);
            if (!can) continue;
            if (Bi.is_fem || Bj.is_fem) {
                atomicOr(deverr, DEVERR_CONTACT_UNSUPPORTED);
                continue;
            }
            uf_union(C.parent, i, j);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        const int r = uf_find(C.parent, i);
        C.parent[i] = r;
        atomicAdd(&C.isl_cnt[r], 1);
        atomicAdd(&C.isl_nodes[r], bodies[i].nnodes);
        if (!bodies[i].sleeping) atomicOr(&C.isl_live[r], 1);
    }
    __syncthreads();
    // the islands with pairs: their rank and their first node of scratch (in body order)
    int carry_n = 0, carry_i = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        const int i = base + threadIdx.x;
        bool pr = false;
        if (i < nb) {
            Body& B = bodies[i];
            const int r = C.parent[i];
            const bool live = C.isl_live[r] != 0;
            B.island = live ? r : -1;
            B.pairs = live && C.isl_cnt[r] > 1 ? 1 : 0;
            B.body_contacts = 0;
            pr = r == i && B.pairs;
        }
        int tn, ti;
        const int on = block_scan_excl(pr ? C.isl_nodes[i] : 0, tn, s_warp);
        const int oi = block_scan_excl(pr ? 1 : 0, ti, s_warp);
        if (pr) C.isl_noff[i] = carry_n + on, C.isl_idx[i] = carry_i + oi;
        carry_n += tn, carry_i += ti;
    }
}

// ------------------------------------------------------------------------------------------ wake requests (each substep)
// simulate_island's substep start (world.cpp:3333-3337): a sleeping body a moving partner touched wakes; its beams step
// again (SoftBody::wake, softbody.h:996).
__global__ void k_wake(Body* __restrict__ bodies, uint32_t* __restrict__ bmeta) {
    Body& B = bodies[blockIdx.x];
    if (!B.wake_request || B.island < 0) return;
    for (int j = threadIdx.x; j < B.nbeams; j += blockDim.x) bmeta[B.beam0 + j] &= ~kBeamAsleep;
    __syncthreads();
    if (threadIdx.x == 0) B.wake_request = 0, B.sleeping = 0, B.sleep_timer = 0.0f;
}

// ------------------------------------------------------------------------------------------ the pair search
} // namespace blg
#include "bl_pair_search.cuh"
namespace blg {

// ------------------------------------------------------------------------------------------ narrow phase (each substep)
// World::pair_detect for node-triangle pairs (world.cpp:2819-2858): hit_a = (bary, pen), hit_b = (normal, 1) when
// the pair is in contact, hit_b.w = 0 when not
__global__ void __launch_bounds__(256) k_detect(const float4* __restrict__ nd, const int4* __restrict__ info, const Body* __restrict__ bodies, Contacts C) {
    const int total = min(*C.pair_total, C.max_pairs);
    if (blockIdx.x == 0 && threadIdx.x == 0) *C.crec_n = 0; // (k_collide takes its records after this kernel)
    // (a warp takes 32 consecutive pairs: its ballot is their word of hit bits)
    for (int i0 = blockIdx.x * blockDim.x; i0 < total; i0 += gridDim.x * blockDim.x) {
        const int i = i0 + (int)threadIdx.x;
        bool hit = false;
        if (i < total) {
            const int2 pr = C.pairs[i];
            const int4 tr = C.tri[pr.y];
            const Body& bn = bodies[info[pr.x].w];
            const Body& bt = bodies[tr.w >> 8];
            float4 ha = make_float4(0, 0, 0, 0), hb = make_float4(0, 0, 0, 0);
            do {
                if (bn.sleeping && bt.sleeping) break;
                if (tr.w & TF_TORN) break; // (torn since the pairs were found)
                const bool two_sided = (tr.w & TF_TWO_SIDED) != 0;
                const v3 np = nd_p(nd, pr.x);
                const v3 a = nd_p(nd, tr.x), b = nd_p(nd, tr.y), cc = nd_p(nd, tr.z);
                v3 bary;
                const float r = bt.faces_only && !two_sided ? bt.face_skin : bn.crad;
                if (!two_sided) {
                    // a hull triangle: over its face pushed out along the face's normal, from as deep as the hull's depth
                    const v3 fn = normalize(cross(b - a, cc - a));
                    const float s = dot(np - a, fn);
                    if (s >= r || s < -bt.hull_depth) break;
                    const v3 q = np - fn * s;
                    const v3 cq = closest_on_triangle(q, a, b, cc, bary);
                    if (length2(cq - q) <= 1e-6f) {
                        ha = make_float4(bary.x, bary.y, bary.z, r - s), hb = make_float4(fn.x, fn.y, fn.z, 0.0f);
                        hit = true;
                        break;
                    }
                    if (s < 0 || bt.faces_only) break;
                } else {
                    const v3 lo = vmin3(a, vmin3(b, cc)) - V(r, r, r), hi = vmax3(a, vmax3(b, cc)) + V(r, r, r);
                    if (outside(np, lo, hi)) break;
                }
                const v3 cp = closest_on_triangle(np, a, b, cc, bary);
                const v3 d = np - cp;
                const float dist2 = dot(d, d);
                if (dist2 >= r * r) break;
                const float dist = sqrtf(dist2);
                v3 nrm;
                if (dist > 1e-5f) {
                    nrm = divs(d, dist);
                } else {
                    nrm = normalize(cross(b - a, cc - a));
                    const v3 vt = nd_v(nd, tr.x) * bary.x + nd_v(nd, tr.y) * bary.y + nd_v(nd, tr.z) * bary.z;
                    if (dot(nd_v(nd, pr.x) - vt, nrm) > 0) nrm = neg(nrm);
                }
                ha = make_float4(bary.x, bary.y, bary.z, r - dist), hb = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
                hit = true;
            } while (false);
            hb.w = hit ? 1.0f : 0.0f;
            C.hit_a[i] = ha;
            C.hit_b[i] = hb;
        }
        const unsigned bits = __ballot_sync(0xffffffffu, hit);
        if ((threadIdx.x & 31) == 0) C.hbits[i >> 5] = bits;
    }
}

// ------------------------------------------------------------------------------------------ response (each substep)
// World::collide_pairs for node-triangle pairs (world.cpp:2975-3023): each contact cancels the forces accumulated so far
// on its node and its triangle's corners (earlier contacts' included), so an island's contacts run one after another
// in pair order, as the reference's loop (world.cpp:2999) - but only contacts that share a node depend on each other.
// A CTA an island:
//  1. its contacts (its pairs with a hit bit, in pair order) listed by a block scan; their nodes hashed into
//     shared-memory force slots and the forces loaded there;
//  2. each contact's record - its slots, the accumulation weights, relative velocity and normal, and every term of the
//     contact law that does not depend on the forces (the slip direction and speed, the Stribeck exponentials, the
//     restitution and push terms, the soft ground's drag and buoyancy) - formed in parallel;
//  3. each contact's level, one above its nodes' earlier contacts' levels (one thread, in pair order), so the contacts
//     of one level touch distinct nodes; the levels run one after another, a level's contacts at once, each contact
//     with only its force-dependent arithmetic (apply_contact) - every contact sees the forces the serial loop gives
//     it. Up to Contacts::whole_max contacts the island runs whole (its records in global memory, its levels over all
//     of it, formed while the records are); more, 512 at a time (records and levels in shared memory);
//  4. the forces written back. An island with more distinct contact nodes than the slots hold runs the loop on global
//     memory (collide_island_global). Results are the same bits every way.
__device__ void collide_island_global(const float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies, Contacts C,
                                      float4* __restrict__ Fs, int root, int off, int cnt);

constexpr int kCollideThreads = 256;
constexpr int kSlotBits = 13, kSlots = 1 << kSlotBits; // force slots (distinct contact nodes an island)
constexpr int kRecChunk = 512;                          // contact records formed at a time
constexpr int kSlotPad = 8;                             // slot levels past the slots (kSlots: a level that stays 0)
constexpr int kStage = 6144;                            // contacts of an island that runs whole (slots, levels staged)

struct alignas(16) ContactRec {
    int sa, sb[3];        // force slots of the node and the triangle's corners
    float ca, cb[3];      // acc = FA ca - sum FB_q cb_q (the terms the movable sides have)
    float wb[3], m;       // barycentric weights; effective mass
    float nx, ny, nz;     // the normal passed to the law (negated where the node's side is immovable)
    float vx, vy, vz;     // the relative velocity passed to the law
    float pen, fric;
    float Vn, rsub;       // vel . normal; the restitution / push term of R where Vn < 0 (else 0); hull: (target - vr) m / dt
    float sx, sy, sz;     // the slip direction (0 where the slip speed is below 1e-9)
    float sv, stop;       // the slip speed; mass sv / dt
    float e1, gsum;       // 1 - exp(-sv / va); the dynamic friction's g + min(t2 sv, 5)
    float dragf, fb0;     // the soft ground's drag factor and buoyancy (where it is soft under the contact)
    int kind;             // 0 none, 1 contact (node movable), 2 contact (node immovable), 3 hull push-out; | ma << 4 | mb << 5
                          // | soft (drag, buoyancy) << 6 | pen >= soft depth << 7
};

__device__ __forceinline__ int slot_hash(int key) { return (int)(((uint32_t)key * 2654435761u) >> (32 - kSlotBits)); }
__device__ __forceinline__ int slot_find(const int* keys, int key) {
    int h = slot_hash(key);
    while (keys[h] != key) h = (h + 1) & (kSlots - 1);
    return h;
}

// One contact of the chain on the forces in the slots: only the force-dependent arithmetic, the reference's operations
// in its order (contact_force<1, 3> / hull_push_out<3> and primitive_collision, world.cpp:59-120,
// static_world.cpp:8-51, split at their force-independent parts, which the record holds)
__device__ __forceinline__ void apply_contact(const ContactRec& R, float* fx, float* fy, float* fz, const GroundModel& gm) {
    const int kind = R.kind & 15;
    const bool ma = R.kind & 16, mb = R.kind & 32;
    v3 FA = V(fx[R.sa], fy[R.sa], fz[R.sa]);
    v3 FB[3];
    for (int q = 0; q < 3; q++) FB[q] = V(fx[R.sb[q]], fy[R.sb[q]], fz[R.sb[q]]);
    v3 acc = V(0, 0, 0);
    if (ma) acc = acc + FA * R.ca;
    for (int q = 0; q < 3; q++)
        if (mb) acc = acc - FB[q] * R.cb[q];
    const v3 nrm = V(R.nx, R.ny, R.nz);
    if (kind == 3) {
        const float fn = R.rsub - dot(acc, nrm) * R.m;
        if (fn > 0) {
            const v3 f = nrm * fn;
            if (ma) FA = FA + f;
            if (mb)
                for (int q = 0; q < 3; q++) FB[q] = FB[q] - f * R.wb[q];
        }
    } else {
        const v3 f_rel = acc * R.m;
        const v3 F = kind == 1 ? f_rel : neg(f_rel);
        const v3 vel = V(R.vx, R.vy, R.vz);
        // primitive_collision (static_world.cpp:8-51) with its force-independent terms from the record
        v3 out = V(0, 0, 0);
        const float Vn = R.Vn, Fn = dot(F, nrm);
        if (R.kind & 64) {
            out = out + vel * R.dragf;
            float Fb = R.fb0;
            if (Vn >= 0 && Fn < 0 && Fb > -Fn) Fb = -Fn;
            out = out + nrm * Fb;
        }
        if (R.kind & 128) {
            float Rn = -Fn;
            if (Vn < 0) Rn -= R.rsub;
            if (Rn > 0) {
                const v3 slipF = F - nrm * Fn;
                const v3 slip = V(R.sx, R.sy, R.sz);
                const float G = Rn * gm.strength * R.fric;
                if (R.sv < gm.va && G > 0 && length(slipF) <= gm.ms * G)
                    out = out + (nrm * Rn - slip * smin(gm.ms * G * R.e1, R.stop) - slipF);
                else
                    out = out + (nrm * Rn - slip * smin(R.gsum * G, smax(0.0f, R.stop + dot(slipF, slip))));
            }
        }
        if (kind == 2) {
            for (int q = 0; q < 3; q++) FB[q] = FB[q] + out * R.wb[q];
        } else {
            FA = FA + out * 1.0f;
            if (mb)
                for (int q = 0; q < 3; q++) FB[q] = FB[q] - out * R.wb[q];
        }
    }
    fx[R.sa] = FA.x, fy[R.sa] = FA.y, fz[R.sa] = FA.z;
    for (int q = 0; q < 3; q++) fx[R.sb[q]] = FB[q].x, fy[R.sb[q]] = FB[q].y, fz[R.sb[q]] = FB[q].z;
}

// One contact's record (pair i of the island; kind 0 where the law gives it no force): its slots, the accumulation
// weights and every force-independent term of the law, and the wake requests of its sleeping sides. True when it is a
// contact (counted).
__device__ __forceinline__ bool form_record(ContactRec& R, int i, const float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies,
                                            const Contacts& C, const int* keys, const GroundModel& gm, float dt) {
    R.kind = 0;
    const float4 hb4 = C.hit_b[i];
    const float4 ha = C.hit_a[i];
    const int2 pr = C.pairs[i];
    const int4 tr = C.tri[pr.y];
    Body& bn = bodies[info[pr.x].w];
    Body& bt = bodies[tr.w >> 8];
    // movable (world.cpp:2983-2993): a sleeping side is immovable and asks to wake when the other moves
    bool ma = true, mb = true;
    if (bn.sleeping) {
        if (sqrtf(bt.acc_v2) > smax(C.wake_speed, bt.sleep_speed) * 1.0f) bn.wake_request = 1;
        ma = false;
    }
    if (bt.sleeping) {
        if (sqrtf(bn.acc_v2) > smax(C.wake_speed, bn.sleep_speed) * 1.0f) bt.wake_request = 1;
        mb = false;
    }
    const int ia = pr.x, ib[3] = {tr.x, tr.y, tr.z};
    const float wb[3] = {ha.x, ha.y, ha.z};
    const v3 n = V(hb4.x, hb4.y, hb4.z);
    const float pen = ha.w;
    const float4 pa = nd[2 * ia], va4 = nd[2 * ia + 1];
    const v3 Av = V(va4.x, va4.y, va4.z);
    const float Aim = pa.w;
    v3 Bv[3];
    float Bim[3];
    for (int q = 0; q < 3; q++) {
        const float4 pq = nd[2 * ib[q]], vq = nd[2 * ib[q] + 1];
        Bv[q] = V(vq.x, vq.y, vq.z), Bim[q] = pq.w;
    }
    R.sa = slot_find(keys, ia);
    for (int q = 0; q < 3; q++) R.sb[q] = slot_find(keys, ib[q]), R.wb[q] = wb[q], R.cb[q] = wb[q] * Bim[q];
    const int mv = (ma ? 16 : 0) | (mb ? 32 : 0);
    if (!(tr.w & TF_TWO_SIDED) && pen > bn.crad) {
        // hull_push_out<3> (world.cpp:97-118): behind a hull's face
        float W = ma ? Aim : 0.0f;
        if (mb)
            for (int q = 0; q < 3; q++) W += wb[q] * wb[q] * Bim[q];
        if (W <= 1e-12f) return false;
        v3 vb = V(0, 0, 0);
        for (int q = 0; q < 3; q++) vb = vb + Bv[q] * wb[q];
        const float m = 1.0f / W, vr = dot(Av - vb, n), target = smin(0.2f * pen / dt, 2.0f);
        R.ca = Aim, R.m = m, R.nx = n.x, R.ny = n.y, R.nz = n.z;
        R.rsub = (target - vr) * m / dt;
        R.kind = 3 | mv;
    } else {
        // contact_force<1, 3> (world.cpp:59-92), the node's weight 1; a tyre node grips with its own friction
        // (world.cpp:3013)
        const int4 ina = info[ia];
        const float fric = ((uint32_t)ina.x & NF_TYRE) ? __int_as_float(ina.y) : 0.8f * smin(bn.cfric, bt.cfric);
        float W = 0;
        if (ma) W += 1.0f * 1.0f * Aim;
        if (mb)
            for (int q = 0; q < 3; q++) W += wb[q] * wb[q] * Bim[q];
        if (W <= 1e-12f) return false;
        const float m = 1.0f / W;
        v3 va = V(0, 0, 0), vb = V(0, 0, 0);
        va = va + Av * 1.0f;
        for (int q = 0; q < 3; q++) vb = vb + Bv[q] * wb[q];
        const v3 vel = ma ? va - vb : vb - va, nrm = ma ? n : neg(n);
        R.ca = 1.0f * Aim, R.m = m, R.fric = fric, R.pen = pen;
        R.nx = nrm.x, R.ny = nrm.y, R.nz = nrm.z, R.vx = vel.x, R.vy = vel.y, R.vz = vel.z;
        // primitive_collision's force-independent terms (static_world.cpp:8-51; push_max 2, slop 0, no
        // restitution)
        const float Vn = dot(vel, nrm), sgl = gm.soft_depth;
        R.Vn = Vn;
        R.rsub = Vn < 0 ? (0.8f * Vn - smin(0.2f * smax(0.0f, pen - sgl - 0.0f) / dt, 2.0f)) * m / dt : 0.0f;
        v3 slip = vel - nrm * Vn;
        const float sv = length(slip);
        if (sv > 1e-9f) slip = divs(slip, sv);
        else slip = V(0, 0, 0);
        R.sx = slip.x, R.sy = slip.y, R.sz = slip.z, R.sv = sv, R.stop = m * sv / dt;
        R.e1 = 1.0f - bl_expf(-sv / gm.va);
        const float g = gm.mc + (gm.ms - gm.mc) * bl_expf(-bl_powf(sv / gm.vs, gm.alpha));
        R.gsum = g + smin(gm.t2 * sv, 5.0f);
        const bool soft = sgl > 0 && pen >= 0;
        R.dragf = soft ? -gm.fluid_drag * smin(1.0f, pen / sgl + 0.2f) : 0.0f;
        R.fb0 = soft ? gm.fluid_density * smin(pen, sgl) * 9.807f * 0.02f : 0.0f;
        R.kind = (ma ? 1 : 2) | mv | (soft ? 64 : 0) | (pen >= sgl ? 128 : 0);
    }
    atomicAdd(&bn.body_contacts, 1);
    atomicAdd(&bt.body_contacts, 1);
    return true;
}

__global__ void __launch_bounds__(kCollideThreads, 1) k_collide(const float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies,
                                                            int nbodies, Contacts C, float4* __restrict__ Fs) {
    extern __shared__ __align__(16) unsigned char csm[];
    int* keys = reinterpret_cast<int*>(csm);
    float* fx = reinterpret_cast<float*>(keys + kSlots);
    float* fy = fx + kSlots;
    float* fz = fy + kSlots;
    ContactRec* rec = reinterpret_cast<ContactRec*>(fz + kSlots);
    unsigned short* slot_lvl = reinterpret_cast<unsigned short*>(rec + kRecChunk); // per slot: its latest contact's level
    __shared__ int used, overflow, ncontacts, s_depth;
    const int root = blockIdx.x, tid = threadIdx.x;
    if (root >= nbodies) return;
    const int cnt = C.isl_pcnt[root];
    if (cnt <= 0 || bodies[root].island != root || !bodies[root].pairs) return;
    const int off = C.isl_poff[root];
    const float dt = C.dt;
    const GroundModel& gm = c_ground[3]; // SURF_CONCRETE
    for (int h = tid; h < kSlots; h += kCollideThreads) keys[h] = -1, slot_lvl[h] = 0;
    if (tid < kSlotPad) slot_lvl[kSlots + tid] = 0;
    if (tid == 0) used = 0, overflow = 0, ncontacts = 0;
    __shared__ int s_scan[32];
    // 0. the island's contacts (its pairs with a hit), in pair order, into hidx[off ...): a run of pairs a thread
    int nh_all;
    {
        // (the range's words of hit bits, a run of words a thread, the bits outside the range masked)
        const int w0 = off >> 5, nw = ((off + cnt - 1) >> 5) - w0 + 1;
        const int per = (nw + kCollideThreads - 1) / kCollideThreads;
        const int lo = min(nw, tid * per), hi = min(nw, lo + per);
        auto word = [&](int w) {
            uint32_t m = C.hbits[w0 + w];
            const int b0 = (w0 + w) << 5;
            if (b0 < off) m &= ~0u << (off - b0);
            if (b0 + 32 > off + cnt) m &= (off + cnt - b0 >= 32) ? ~0u : ((1u << (off + cnt - b0)) - 1u);
            return m;
        };
        int mine = 0;
        for (int w = lo; w < hi; w++) mine += __popc(word(w));
        int at = off + block_scan_excl(mine, nh_all, s_scan);
        for (int w = lo; w < hi; w++)
            for (uint32_t m = word(w); m; m &= m - 1) C.hidx[at++] = ((w0 + w) << 5) + __ffs(m) - 1;
    }
    __syncthreads();
    // 1. the contacts' nodes into slots (four contacts a thread at a time: their loads overlap)
    for (int j0 = tid; j0 < nh_all; j0 += 4 * kCollideThreads) {
        int nodes4[4][4];
        for (int u = 0; u < 4; u++) {
            const int j = j0 + u * kCollideThreads;
            nodes4[u][0] = -1;
            if (j >= nh_all) continue;
            const int2 pr = C.pairs[C.hidx[off + j]];
            const int4 tr = C.tri[pr.y];
            nodes4[u][0] = pr.x, nodes4[u][1] = tr.x, nodes4[u][2] = tr.y, nodes4[u][3] = tr.z;
        }
        for (int u = 0; u < 4; u++) {
            if (nodes4[u][0] < 0) continue;
            for (int q = 0; q < 4; q++) {
                const int node = nodes4[u][q];
                int h = slot_hash(node);
                for (int probe = 0;; probe++) {
                    if (probe >= kSlots / 2 || overflow) {
                        overflow = 1;
                        break;
                    }
                    const int prev = atomicCAS(&keys[h], -1, node);
                    if (prev == -1) {
                        if (atomicAdd(&used, 1) >= kSlots / 2) overflow = 1; // (kept at most half full: short probes)
                        break;
                    }
                    if (prev == node) break;
                    h = (h + 1) & (kSlots - 1);
                }
            }
        }
    }
    __syncthreads();
    if (overflow) {
        if (tid == 0) collide_island_global(nd, info, bodies, C, Fs, root, off, cnt);
        return;
    }
    for (int h = tid; h < kSlots; h += kCollideThreads)
        if (keys[h] >= 0) {
            const float4 f = Fs[keys[h]];
            fx[h] = f.x, fy[h] = f.y, fz[h] = f.z;
        }
    // The island's contacts at once where they fit (kStage at most, and the substep's record buffer has room): their
    // records in global memory, their slots and levels staged in the record chunk's shared memory - levels over the
    // whole island, with no barrier between chunks. Otherwise kRecChunk at a time, below.
    __shared__ int s_base;
    if (tid == 0) {
        int b = -1;
        if (nh_all > 0 && nh_all <= C.whole_max) {
            b = atomicAdd(C.crec_n, nh_all);
            if (b + nh_all > C.crec_cap) b = -1;
        }
        s_base = b;
    }
    __syncthreads();
    if (s_base >= 0) {
        const int base = s_base;
        ushort4* sq = reinterpret_cast<ushort4*>(rec);                          // per contact: its slots
        unsigned short* lv16 = reinterpret_cast<unsigned short*>(sq + kStage); // per contact: its level
        // 2. each contact's slots
        for (int j = tid; j < nh_all; j += kCollideThreads) {
            const int2 pr = C.pairs[C.hidx[off + j]];
            const int4 tr = C.tri[pr.y];
            sq[j] = make_ushort4((unsigned short)slot_find(keys, pr.x), (unsigned short)slot_find(keys, tr.x), (unsigned short)slot_find(keys, tr.y),
                                 (unsigned short)slot_find(keys, tr.z));
        }
        __syncthreads();
        // 3. the levels (one thread, in pair order; a pair the law gives no force keeps its place, which only orders
        // more) while the other warps form the records
        if (tid == 0) {
            int depth = 0;
            ushort4 h = sq[0];
            for (int j = 0; j < nh_all; j++) {
                const ushort4 hn = sq[min(j + 1, nh_all - 1)]; // (loaded before this contact's levels are stored)
                const int l = max(max((int)slot_lvl[h.x], (int)slot_lvl[h.y]), max((int)slot_lvl[h.z], (int)slot_lvl[h.w])) + 1;
                slot_lvl[h.x] = slot_lvl[h.y] = slot_lvl[h.z] = slot_lvl[h.w] = (unsigned short)l;
                lv16[j] = (unsigned short)l;
                depth = max(depth, l);
                h = hn;
            }
            s_depth = depth;
        } else if (tid >= 32) {
            for (int j = tid - 32; j < nh_all; j += kCollideThreads - 32) {
                ContactRec R;
                if (form_record(R, C.hidx[off + j], nd, info, bodies, C, keys, gm, dt)) atomicAdd(&ncontacts, 1);
                C.crec[base + j] = R;
            }
        }
        __syncthreads();
        // by level: counts, ends (a running sum), places (a level's contacts in any order: they share no node)
        const int depth = s_depth;
        unsigned short* ord = reinterpret_cast<unsigned short*>(rec); // (over the slots, done with)
        int* le = reinterpret_cast<int*>(ord + kStage);
        for (int l = tid; l < depth + 3; l += kCollideThreads) le[l] = 0;
        __syncthreads();
        for (int j = tid; j < nh_all; j += kCollideThreads) atomicAdd(&le[lv16[j]], 1);
        __syncthreads();
        block_scan_incl_inplace(le, depth + 1, s_scan);
        __syncthreads();
        if (tid == 0) le[depth + 1] = le[depth];
        __syncthreads();
        for (int j = tid; j < nh_all; j += kCollideThreads) ord[atomicSub(&le[lv16[j]], 1) - 1] = (unsigned short)j; // (le[L]: level L's start)
        __syncthreads();
        // 4. the chain: one warp, level after level, a lane a contact; the next level's records loaded while one runs
        if (tid < 32) {
            const ContactRec* __restrict__ cr = C.crec + base;
            int s0 = le[1], e0 = le[2];
            bool has = s0 + tid < e0;
            ContactRec cur;
            if (has) cur = cr[ord[s0 + tid]];
            for (int L = 1; L <= depth; L++) {
                const int s1 = le[L + 1], e1 = L < depth ? le[L + 2] : s1;
                const bool hasn = s1 + tid < e1;
                ContactRec nxt;
                if (hasn) nxt = cr[ord[s1 + tid]];
                if (has && (cur.kind & 15)) apply_contact(cur, fx, fy, fz, gm);
                for (int k = s0 + tid + 32; k < e0; k += 32) {
                    const ContactRec R = cr[ord[k]];
                    if (R.kind & 15) apply_contact(R, fx, fy, fz, gm);
                }
                __syncwarp();
                cur = nxt, has = hasn, s0 = s1, e0 = e1;
            }
        }
    } else {
        // the island's contacts in pair order, kRecChunk at a time
        __shared__ int order[kRecChunk], lend[kRecChunk + 3], lv[kRecChunk];
        __shared__ int4 sl[kRecChunk + 1]; // per record: its slots (kSlots x 4: not a contact)
        for (int c0 = 0; c0 < nh_all; c0 += kRecChunk) {
            const int nh = min(kRecChunk, nh_all - c0);
            __syncthreads();
            // 2. the records of these contacts
            for (int r = tid; r < nh; r += kCollideThreads) {
                const int i = C.hidx[off + c0 + r];
                ContactRec& R = rec[r];
                sl[r] = make_int4(kSlots, kSlots, kSlots, kSlots); // (none: the slot whose level stays 0)
                if (form_record(R, i, nd, info, bodies, C, keys, gm, dt)) {
                    sl[r] = make_int4(R.sa, R.sb[0], R.sb[1], R.sb[2]);
                    atomicAdd(&ncontacts, 1);
                }
            }
            __syncthreads();
            // 3. the chain. A contact reads and writes the forces of its four nodes only, so one that shares no node with
            // the contacts between it and an earlier one commutes with them: each contact's level is one above the
            // latest level among its nodes' earlier contacts (one thread, in pair order), the contacts sorted by level,
            // then one warp runs them level after level, a level's contacts at once - every contact sees the forces the
            // serial loop gives it. Where the levels are nearly as many as the contacts, one thread runs the loop.
            for (int l = tid; l < kRecChunk + 3; l += kCollideThreads) lend[l] = 0;
            if (tid == 0) {
                int depth = 0, nk = 0;
                int4 h = sl[0];
                for (int r = 0; r < nh; r++) {
                    const int4 hn = sl[r + 1]; // (loaded before this record's levels are stored; sl[nh] is not used)
                    const int l = max(max((int)slot_lvl[h.x], (int)slot_lvl[h.y]), max((int)slot_lvl[h.z], (int)slot_lvl[h.w])) + 1;
                    const int lk = h.x == kSlots ? 0 : l;
                    slot_lvl[h.x] = slot_lvl[h.y] = slot_lvl[h.z] = slot_lvl[h.w] = (unsigned short)lk;
                    lv[r] = lk;
                    depth = max(depth, lk), nk += lk != 0;
                    h = hn;
                }
                s_depth = 5 * depth > 4 * nk ? -1 : depth;
            }
            __syncthreads();
            const int depth = s_depth;
            if (depth < 0) {
                if (tid == 0)
                    for (int r = 0; r < nh; r++)
                        if (lv[r]) apply_contact(rec[r], fx, fy, fz, gm);
            } else if (depth > 0) {
                // by level: counts, ends (a running sum), places (each level's contacts in any order: they share no node)
                for (int r = tid; r < nh; r += kCollideThreads)
                    if (lv[r]) atomicAdd(&lend[lv[r]], 1);
                __syncthreads();
                block_scan_incl_inplace(lend, depth + 1, s_scan);
                __syncthreads();
                if (tid == 0) lend[depth + 1] = lend[depth];
                __syncthreads();
                for (int r = tid; r < nh; r += kCollideThreads)
                    if (lv[r]) order[atomicSub(&lend[lv[r]], 1) - 1] = r; // (lend[L] becomes level L's start)
                __syncthreads();
                if (tid < 32) {
                    // a lane a contact of the level; the next level's first contacts are looked up before this level runs
                    int s0 = lend[1], e0 = lend[2];
                    int rr = s0 + tid < e0 ? order[s0 + tid] : -1;
                    for (int L = 1; L <= depth; L++) {
                        const int s1 = lend[L + 1], e1 = L < depth ? lend[L + 2] : s1;
                        const int rn = s1 + tid < e1 ? order[s1 + tid] : -1;
                        if (rr >= 0) apply_contact(rec[rr], fx, fy, fz, gm);
                        for (int k = s0 + tid + 32; k < e0; k += 32) apply_contact(rec[order[k]], fx, fy, fz, gm);
                        __syncwarp();
                        s0 = s1, e0 = e1, rr = rn;
                    }
                }
            }
            __syncthreads();
            for (int r = tid; r < nh; r += kCollideThreads) {
                const int4 h = sl[r];
                slot_lvl[h.x] = slot_lvl[h.y] = slot_lvl[h.z] = slot_lvl[h.w] = 0;
            }
        }
    }
    __syncthreads();
    // 4. the forces back
    for (int h = tid; h < kSlots; h += kCollideThreads)
        if (keys[h] >= 0) Fs[keys[h]] = make_float4(fx[h], fy[h], fz[h], 0.0f);
    if (tid == 0) {
        C.isl_contacts[root] += ncontacts;
        if (ncontacts) atomicAdd(&C.counters[1], ncontacts);
    }
}
constexpr size_t kCollideSmem = sizeof(int) * kSlots + 3 * sizeof(float) * kSlots + sizeof(ContactRec) * kRecChunk +
                                sizeof(unsigned short) * (kSlots + kSlotPad);

// The serial loop on global memory (the path of an island with more distinct contact nodes than the slots hold)
__device__ void collide_island_global(const float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies, Contacts C,
                                      float4* __restrict__ Fs, int root, int off, int cnt) {
    const float dt = C.dt;
    const GroundModel& gm = c_ground[3]; // SURF_CONCRETE
    int contacts = 0;
    for (int i = off; i < off + cnt; i++) {
        const float4 hb4 = C.hit_b[i];
        if (hb4.w == 0.0f) continue;
        const float4 ha = C.hit_a[i];
        const int2 pr = C.pairs[i];
        const int4 tr = C.tri[pr.y];
        Body& bn = bodies[info[pr.x].w];
        Body& bt = bodies[tr.w >> 8];
        // movable (world.cpp:2983-2993): a sleeping side is immovable and asks to wake when the other moves
        bool ma = true, mb = true;
        if (bn.sleeping) {
            if (sqrtf(bt.acc_v2) > smax(C.wake_speed, bt.sleep_speed) * 1.0f) bn.wake_request = 1;
            ma = false;
        }
        if (bt.sleeping) {
            if (sqrtf(bn.acc_v2) > smax(C.wake_speed, bn.sleep_speed) * 1.0f) bt.wake_request = 1;
            mb = false;
        }
        const int ia = pr.x, ib[3] = {tr.x, tr.y, tr.z};
        const float wb[3] = {ha.x, ha.y, ha.z};
        const v3 n = V(hb4.x, hb4.y, hb4.z);
        const float pen = ha.w;
        const float4 pa = nd[2 * ia], va4 = nd[2 * ia + 1];
        const v3 Av = V(va4.x, va4.y, va4.z);
        const float Aim = pa.w;
        v3 Bv[3];
        float Bim[3];
        for (int q = 0; q < 3; q++) {
            const float4 p = nd[2 * ib[q]], v = nd[2 * ib[q] + 1];
            Bv[q] = V(v.x, v.y, v.z), Bim[q] = p.w;
        }
        const float4 fa4 = Fs[ia];
        v3 FA = V(fa4.x, fa4.y, fa4.z);
        v3 FB[3];
        for (int q = 0; q < 3; q++) {
            const float4 f = Fs[ib[q]];
            FB[q] = V(f.x, f.y, f.z);
        }
        if (!(tr.w & TF_TWO_SIDED) && pen > bn.crad) {
            // hull_push_out<3> (world.cpp:97-118): behind a hull's face
            float W = ma ? Aim : 0.0f;
            if (mb)
                for (int q = 0; q < 3; q++) W += wb[q] * wb[q] * Bim[q];
            if (W <= 1e-12f) continue;
            v3 vb = V(0, 0, 0), acc = V(0, 0, 0);
            if (ma) acc = acc + FA * Aim;
            for (int q = 0; q < 3; q++) {
                vb = vb + Bv[q] * wb[q];
                if (mb) acc = acc - FB[q] * (wb[q] * Bim[q]);
            }
            const float m = 1.0f / W, vr = dot(Av - vb, n), target = smin(0.2f * pen / dt, 2.0f);
            const float fn = (target - vr) * m / dt - dot(acc, n) * m;
            if (fn > 0) {
                const v3 f = n * fn;
                if (ma) FA = FA + f;
                if (mb)
                    for (int q = 0; q < 3; q++) FB[q] = FB[q] - f * wb[q];
            }
        } else {
            // contact_force<1, 3> (world.cpp:59-92), the node's weight 1; a tyre node grips with its own friction
            // (world.cpp:3013)
            const int4 ina = info[ia];
            const float fric = ((uint32_t)ina.x & NF_TYRE) ? __int_as_float(ina.y) : 0.8f * smin(bn.cfric, bt.cfric);
            float W = 0;
            if (ma) W += 1.0f * 1.0f * Aim;
            if (mb)
                for (int q = 0; q < 3; q++) W += wb[q] * wb[q] * Bim[q];
            if (W <= 1e-12f) continue;
            const float m = 1.0f / W;
            v3 va = V(0, 0, 0), vb = V(0, 0, 0), acc = V(0, 0, 0);
            va = va + Av * 1.0f;
            if (ma) acc = acc + FA * (1.0f * Aim);
            for (int q = 0; q < 3; q++) {
                vb = vb + Bv[q] * wb[q];
                if (mb) acc = acc - FB[q] * (wb[q] * Bim[q]);
            }
            const v3 f_rel = acc * m;
            if (!ma) {
                const v3 f = primitive_collision(neg(f_rel), vb - va, m, neg(n), dt, gm, pen, fric, 2.0f, 0.0f, -1.0f);
                for (int q = 0; q < 3; q++) FB[q] = FB[q] + f * wb[q];
            } else {
                const v3 f = primitive_collision(f_rel, va - vb, m, n, dt, gm, pen, fric, 2.0f, 0.0f, -1.0f);
                FA = FA + f * 1.0f;
                if (mb)
                    for (int q = 0; q < 3; q++) FB[q] = FB[q] - f * wb[q];
            }
        }
        Fs[ia] = make_float4(FA.x, FA.y, FA.z, 0.0f);
        for (int q = 0; q < 3; q++) Fs[ib[q]] = make_float4(FB[q].x, FB[q].y, FB[q].z, 0.0f);
        contacts++;
        bn.body_contacts++;
        bt.body_contacts++;
    }
    C.isl_contacts[root] += contacts;
    if (contacts) atomicAdd(&C.counters[1], contacts);
}

} // namespace blg
