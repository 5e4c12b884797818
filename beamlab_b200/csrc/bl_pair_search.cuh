// The pair search between bodies: World::rebuild_pairs with near_pairs' filter (world.cpp:1851-2308, 2314-2520,
// 2525-2598), node-triangle pairs only, in the reference's pair order. Included by bl_contacts.cuh (the Contacts
// layout, the geometry and the block helpers are there).
//
// Four launches on a search substep:
//  * k_rebuild, one CTA per island with pairs: the island's bodies, top and bulk speeds, margins and cell size, the
//    partners, the slow bodies' spatial hash (buckets of cell_hash & mask, each bucket in node order, kept as records
//    in bucket order) and each fast body's dense grid (its nodes in the lowest cell of their travel, in node order
//    within a cell, kept as records in cell order). It leaves the island's search state in C.isl and lists its
//    queries: groups (a slow body's triangles against the hash; a fast body's grid against one partner's triangles),
//    in the reference's order (slow bodies in body order, then fast bodies in body order and their partners in body
//    order), each triangle of a group one query, split in chunks of kQueryChunk.
//  * k_pair_count, over all islands' chunks at once (every SM busy whatever the islands' sizes): one query a thread,
//    its kept pairs counted into q_count and, up to kLocPairs of them, kept in ptmp.
//  * k_pair_place, one CTA per island: the running sum of its queries' counts (the pairs' places in the island's
//    range), the island's range taken from the pair list.
//  * k_pair_write, over the chunks again: the queries' pairs copied to their places (a query with more pairs than the
//    count pass keeps runs again).
// The pairs of an island are the reference's, in its order; the islands' ranges lie in the order the islands finish.
#pragma once

namespace blg {

constexpr int kQueryChunk = 256;       // queries of one chunk (a CTA of k_pair_count / k_pair_write)
constexpr int kQueryGrid = 148 * 8;    // CTAs of k_pair_count / k_pair_write (they stride over the chunks)
constexpr int kLocPairs = 16;          // a query's pairs the count pass keeps (more: the write pass runs it again)

struct IslBody {
    int id;               // global body index
    float sp;             // max_speed now (the frame's running maximum)
    float extra;          // extra pair margin of a fast body
    float bulk;           // bulk speed of a fast body
    float mn[3], mx[3];   // its bounds now
    float bmn[3], bmx[3]; // its box grown by the reach (Island::boxes)
    // the dense grid of a fast body with partners (World::fast_pairs, world.cpp:2330-2362)
    float g_org[3], g_inv;
    int g_dim[3];
    int g_span[3];        // the most cells a node's travel spans along each axis, less one
    int gs0;              // its cells' starts in g_start
    int gi0;              // its nodes' records in g_items / g_rec / g_hi
};

// What an island's queries read (built in shared memory by k_rebuild, then copied to C.isl)
struct alignas(16) IslSearch {
    IslBody b[kIslMaxBodies];
    uint32_t partner[kIslMaxBodies][kIslMaxBodies / 32];
    int nb, root;
    float rmax, margin, inv_cell, slow_reach, travel, T;
    int mask, bk0, pt0;
    int inst0, ninst;     // its queries in q_count (ninst < 0: the island has no search this time)
};

struct RebuildShared {
    IslSearch s;
    double term0[1024];
    double term1[1024];
    int warp[32];
    int npts, fail;
    int g_base, c_base;   // the island's first group and chunk
};

__device__ __forceinline__ bool same_group(const Body& a, const Body& b) { return a.group != 0 && a.group == b.group; }

__device__ __forceinline__ bool box_hits(const float* mn, const float* mx, v3 qmn, v3 qmx) {
    return qmn.x <= mx[0] && qmx.x >= mn[0] && qmn.y <= mx[1] && qmx.y >= mn[1] && qmn.z <= mx[2] && qmx.z >= mn[2];
}
// near_partner (world.cpp:1955-1962)
__device__ bool near_partner(const IslSearch& S, int k, v3 mn, v3 mx) {
    for (int w = 0; w < kIslMaxBodies / 32; w++) {
        uint32_t bits = S.partner[k][w];
        while (bits) {
            const int o = w * 32 + __ffs(bits) - 1;
            bits &= bits - 1;
            if (box_hits(S.b[o].bmn, S.b[o].bmx, mn, mx)) return true;
        }
    }
    return false;
}
__device__ __forceinline__ bool has_partner(const IslSearch& S, int k) {
    for (int w = 0; w < kIslMaxBodies / 32; w++)
        if (S.partner[k][w]) return true;
    return false;
}
__device__ __forceinline__ bool is_partner(const IslSearch& S, int k, int o) { return (S.partner[k][o >> 5] >> (o & 31)) & 1u; }

// near_pairs' test of one candidate (world.cpp:2536-2583); T: the reach's time
__device__ bool near_keep(const float4* __restrict__ nd, const Body& bn, const Body& bt, int node, int4 t, float T) {
    if (t.w & TF_TORN) return false;
    const bool two_sided = (t.w & TF_TWO_SIDED) != 0;
    const v3 xp = nd_p(nd, node), xv = nd_v(nd, node);
    const v3 ap = nd_p(nd, t.x), bp = nd_p(nd, t.y), cp = nd_p(nd, t.z);
    const v3 av = nd_v(nd, t.x), bv = nd_v(nd, t.y), cv = nd_v(nd, t.z);
    v3 bary;
    const v3 q = closest_on_triangle(xp, ap, bp, cp, bary);
    const float r0 = bn.crad + (two_sided ? 0.0f : bt.hull_depth);
    const v3 da = xv - av, db = xv - bv, dc = xv - cv;
    const float vrel = sqrtf(smax(length2(da), smax(length2(db), length2(dc))));
    const float reach = r0 + 1.25f * vrel * T + 0.02f;
    if (length2(xp - q) >= reach * reach) return false;
    const v3 nn = cross(bp - ap, cp - ap);
    const float nl = length(nn);
    if (nl > 1e-12f) {
        const v3 n0 = divs(nn, nl);
        const float s0 = dot(n0, xp - ap);
        if (two_sided || s0 > bn.crad) {
            const float sg = s0 >= 0 ? 1.0f : -1.0f;
            const float close = smax(0.0f, smax(-sg * dot(n0, da), smax(-sg * dot(n0, db), -sg * dot(n0, dc))));
            if (fabsf(s0) - 1.25f * close * T - 0.02f >= bn.crad) return false;
        }
    }
    return true;
}

__device__ __forceinline__ int cell_of(float v, float inv_cell) { return (int)floorf(v * inv_cell); }

// The fast body's grid cell of p (World::fast_pairs' cell_index, world.cpp:2341-2346), per axis
__device__ __forceinline__ int3 grid_cell(const IslBody& G, v3 p) {
    const int x = min(max((int)((p.x - G.g_org[0]) * G.g_inv), 0), G.g_dim[0] - 1);
    const int y = min(max((int)((p.y - G.g_org[1]) * G.g_inv), 0), G.g_dim[1] - 1);
    const int z = min(max((int)((p.z - G.g_org[2]) * G.g_inv), 0), G.g_dim[2] - 1);
    return make_int3(x, y, z);
}
// the cells a node of the fast body is listed in: those within its own travel (world.cpp:2350-2362), as a box of
// cells; m: the travel's reach |v| x travel
__device__ __forceinline__ void node_cells(const IslBody& G, float travel, v3 p, v3 v, float& m, int3& lo, int3& hi) {
    m = length(v) * travel;
    const v3 vm = V(m, m, m);
    lo = grid_cell(G, p - vm);
    hi = grid_cell(G, p + vm);
}

// One triangle of island body kt against the slow bodies' hash (world.cpp:2037-2083), near_pairs' filter applied:
// counts the pairs, and writes the first `cap` of them from `out` when it is given. The hash's records sit in bucket order (cell and
// body; position and node), a run of one body's records ends at run_end.
__device__ int slow_query(const IslSearch& S, const Contacts& C, const Body* __restrict__ bodies, const float4* __restrict__ nd, int kt, int tg,
                          int2* out, int cap) {
    const Body& o = bodies[S.b[kt].id];
    const int4 tr = C.tri[tg];
    if (tr.w & TF_TORN) return 0;
    const bool two_sided = (tr.w & TF_TWO_SIDED) != 0;
    const float depth = two_sided ? 0.0f : o.hull_depth;
    const float extra = S.b[kt].extra;
    const float rq = S.rmax + S.margin + extra + depth;
    const v3 a = nd_p(nd, tr.x), bb = nd_p(nd, tr.y), c = nd_p(nd, tr.z);
    const v3 tmn = vmin3(a, vmin3(bb, c)), tmx = vmax3(a, vmax3(bb, c));
    const v3 vr = V(rq, rq, rq);
    if (!near_partner(S, kt, tmn - vr, tmx + vr)) return 0;
    const v3 tn = cross(bb - a, c - a);
    const float tn2 = dot(tn, tn);
    const v3 tu = tn2 > 1e-20f ? tn * (1.0f / sqrtf(tn2)) : V(0, 0, 0);
    const float ic = S.inv_cell;
    const int x0 = cell_of(tmn.x - rq, ic), x1 = cell_of(tmx.x + rq, ic);
    const int y0 = cell_of(tmn.y - rq, ic), y1 = cell_of(tmx.y + rq, ic);
    const int z0 = cell_of(tmn.z - rq, ic), z1 = cell_of(tmx.z + rq, ic);
    if ((long long)(x1 - x0 + 1) * (y1 - y0 + 1) * (z1 - z0 + 1) > 512) return 0; // degenerate/exploded
    const int bt = S.b[kt].id, bk0 = S.bk0, pt0 = S.pt0;
    const float T = S.T;
    int n = 0;
    for (int z = z0; z <= z1; z++)
        for (int y = y0; y <= y1; y++)
            for (int x = x0; x <= x1; x++) {
                const int bk = (int)(cell_hash(x, y, z) & (uint32_t)S.mask);
                const int k1 = C.bk_start[bk0 + bk + 1];
                for (int k = C.bk_start[bk0 + bk]; k < k1; k++) {
                    const int4 pc = C.sb_cell[pt0 + k];
                    if (pc.w == bt) { // own nodes: skip the whole run
                        k = C.run_end[pt0 + k] - 1;
                        continue;
                    }
                    if (pc.x != x || pc.y != y || pc.z != z) continue; // hash collision
                    const float4 pp = C.sb_pos[pt0 + k];
                    const v3 p = V(pp.x, pp.y, pp.z);
                    if (p.x < tmn.x - rq || p.y < tmn.y - rq || p.z < tmn.z - rq || p.x > tmx.x + rq || p.y > tmx.y + rq || p.z > tmx.z + rq) continue;
                    const Body& b = bodies[pc.w];
                    if (same_group(b, o)) continue;
                    if (b.sleeping && o.sleeping) continue;
                    const float r = b.crad + S.margin + extra;
                    const float rb = r + depth;
                    if (p.x < tmn.x - rb || p.y < tmn.y - rb || p.z < tmn.z - rb || p.x > tmx.x + rb || p.y > tmx.y + rb || p.z > tmx.z + rb) continue;
                    if (!near_triangle(p, a, bb, c, tu, r, two_sided, depth)) continue;
                    const int node = __float_as_int(pp.w);
                    if (!near_keep(nd, b, o, node, tr, T)) continue;
                    if (out && n < cap) out[n] = make_int2(node, tg);
                    n++;
                }
            }
    return n;
}

// One triangle of partner `ko` against fast body `kf`'s grid (world.cpp:2394-2475), near_pairs' filter applied; the
// pairs come out in node order (the reference sorts and deduplicates the cells' lists; here a node listed in several
// cells of the scan is taken in the first of them, and the triangle's pairs are sorted after).
__device__ int fast_query(const IslSearch& S, const Contacts& C, const Body* __restrict__ bodies, const float4* __restrict__ nd, int kf, int ko,
                          int tg, int2* out, int cap) {
    const IslBody& G = S.b[kf];
    const Body& F = bodies[G.id];
    const Body& o = bodies[S.b[ko].id];
    const int4 tr = C.tri[tg];
    if (tr.w & TF_TORN) return 0;
    const bool o_fast = S.b[ko].extra > 0;
    const float fast_extra_o = o_fast ? S.b[ko].extra : 0.0f; // (its bulk x interval x dt)
    const float r = F.crad + S.slow_reach + S.travel * (G.sp + (o_fast ? S.b[ko].sp : 0.0f)) + fast_extra_o;
    const v3 fmn = V(G.mn[0] - r, G.mn[1] - r, G.mn[2] - r), fmx = V(G.mx[0] + r, G.mx[1] + r, G.mx[2] + r);
    const v3 a = nd_p(nd, tr.x), bb = nd_p(nd, tr.y), c = nd_p(nd, tr.z);
    const v3 tmn = vmin3(a, vmin3(bb, c)), tmx = vmax3(a, vmax3(bb, c));
    if (tmx.x < fmn.x || tmx.y < fmn.y || tmx.z < fmn.z || tmn.x > fmx.x || tmn.y > fmx.y || tmn.z > fmx.z) return 0;
    const float r00 = F.crad + (o_fast ? 0.01f : S.slow_reach);
    const float rt = o_fast ? r00 + S.travel * sqrtf(smax(length2(nd_v(nd, tr.x)), smax(length2(nd_v(nd, tr.y)), length2(nd_v(nd, tr.z))))) : r00;
    const bool two_sided = (tr.w & TF_TWO_SIDED) != 0;
    const float depth = two_sided ? 0.0f : o.hull_depth;
    const v3 tn = cross(bb - a, c - a);
    const float tn2 = dot(tn, tn);
    const v3 tu = tn2 > 1e-20f ? tn * (1.0f / sqrtf(tn2)) : V(0, 0, 0);
    const float rr = rt + depth;
    const v3 mn = tmn - V(rr, rr, rr), mx = tmx + V(rr, rr, rr);
    const int x0 = max(0, (int)floorf((mn.x - G.g_org[0]) * G.g_inv)), x1 = min(G.g_dim[0] - 1, (int)((mx.x - G.g_org[0]) * G.g_inv));
    const int y0 = max(0, (int)floorf((mn.y - G.g_org[1]) * G.g_inv)), y1 = min(G.g_dim[1] - 1, (int)((mx.y - G.g_org[1]) * G.g_inv));
    const int z0 = max(0, (int)floorf((mn.z - G.g_org[2]) * G.g_inv)), z1 = min(G.g_dim[2] - 1, (int)((mx.z - G.g_org[2]) * G.g_inv));
    if (x0 > x1 || y0 > y1 || z0 > z1) return 0;
    // The reference lists a node in every cell of its travel and scans the cells of the box: a node is found when its
    // cells' box meets the scan's box. Here each node is listed once, in its lowest cell: the scan starts g_span
    // cells lower and keeps the nodes whose box reaches the scan's box - each found once, as after the reference's
    // sort and deduplication.
    const int gs0 = G.gs0, gi0 = G.gi0;
    const float T = S.T;
    int n = 0;
    for (int z = max(0, z0 - G.g_span[2]); z <= z1; z++)
        for (int y = max(0, y0 - G.g_span[1]); y <= y1; y++) {
            // (a row of cells is one run of records)
            const int row = (z * G.g_dim[1] + y) * G.g_dim[0];
            const int k0 = C.g_start[gs0 + row + max(0, x0 - G.g_span[0])], k1 = C.g_start[gs0 + row + x1 + 1];
            for (int k = k0; k < k1; k++) {
                const int hi = C.g_hi[gi0 + k];
                if ((hi & 255) < x0 || ((hi >> 8) & 255) < y0 || (hi >> 16) < z0) continue;
                const float4 rec = C.g_rec[gi0 + k];
                const v3 p = V(rec.x, rec.y, rec.z);
                const float rn = rt + rec.w, rb = rn + depth;
                if (p.x < tmn.x - rb || p.y < tmn.y - rb || p.z < tmn.z - rb || p.x > tmx.x + rb || p.y > tmx.y + rb || p.z > tmx.z + rb) continue;
                if (!near_triangle(p, a, bb, c, tu, rn, two_sided, depth)) continue;
                const int ni = C.g_items[gi0 + k];
                if (!near_keep(nd, F, o, ni, tr, T)) continue;
                if (out && n < cap) out[n] = make_int2(ni, tg);
                n++;
            }
        }
    if (out && n <= cap)
        for (int i = 1; i < n; i++) { // (by node: the order of the reference's sorted scan)
            const int2 v = out[i];
            int j = i - 1;
            while (j >= 0 && out[j].x > v.x) out[j + 1] = out[j], j--;
            out[j + 1] = v;
        }
    return n;
}

// acc += s_t[0] + s_t[1] + ... one after another, as the reference's loop adds them
__device__ __forceinline__ void serial_add(double& acc, const double* s_t, int n) {
    for (int i = 0; i < n; i++) acc += s_t[i];
}

// World::rebuild_pairs' set-up for one island with pairs (its first body = blockIdx.x); s0: the frame's first substep
// (the bodies' bounds are the frame's, their top speeds are measured now: world.cpp:3216-3222).
__global__ void __launch_bounds__(1024) k_rebuild(Body* __restrict__ bodies, int nbodies, const float4* __restrict__ nd, const int4* __restrict__ info,
                                                  Contacts C, int s0, uint32_t* __restrict__ deverr) {
    const int root = blockIdx.x;
    if (root >= nbodies) return;
    {
        const Body& R = bodies[root];
        if (!R.pairs || R.island != root) return;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RebuildShared& RS = *reinterpret_cast<RebuildShared*>(smem_raw);
    IslSearch& S = RS.s;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int slot = C.isl_idx[root];
    if (tid == 0) S.nb = 0, RS.fail = 0;
    for (int w = tid; w < kIslMaxBodies * (kIslMaxBodies / 32); w += nt) (&S.partner[0][0])[w] = 0u;
    __syncthreads();
    // ---- the island's bodies in body order
    if (tid == 0) {
        int n = 0;
        for (int i = root; i < nbodies; i++)
            if (C.parent[i] == root) {
                if (n < kIslMaxBodies) S.b[n].id = i;
                n++;
            }
        if (n > kIslMaxBodies) atomicOr(deverr, DEVERR_ISLAND), n = 0;
        S.nb = n;
        if (n == 0) C.isl[slot].ninst = -1, C.isl_poff[root] = 0, C.isl_pcnt[root] = 0;
    }
    __syncthreads();
    const int nb = S.nb;
    if (nb == 0) return;
    // ---- top speeds (measured over the nodes on the frame's first substep, world.cpp:3217-3222), bounds now
    if (s0)
        for (int k = 0; k < nb; k++) {
            Body& B = bodies[S.b[k].id];
            if (B.sleeping) continue;
            float m2 = 0.0f;
            for (int i = tid; i < B.nnodes; i += nt) m2 = smax(m2, length2(nd_v(nd, B.node0 + i)));
            for (int o = 16; o > 0; o >>= 1) m2 = fmaxf(m2, __shfl_xor_sync(0xffffffffu, m2, o));
            if ((tid & 31) == 0 && m2 > 0.0f) atomic_max_f(&B.acc_v2, m2);
        }
    __syncthreads();
    for (int k = tid; k < nb; k += nt) {
        const Body& B = bodies[S.b[k].id];
        S.b[k].sp = sqrtf(B.acc_v2);
        const bool acc = !s0 && B.acc_mn[0] <= B.acc_mx[0]; // (stepped in the last substep: its bounds then)
        for (int c = 0; c < 3; c++) S.b[k].mn[c] = acc ? B.acc_mn[c] : B.aabb_mn[c], S.b[k].mx[c] = acc ? B.acc_mx[c] : B.aabb_mx[c];
        S.b[k].extra = 0.0f, S.b[k].bulk = 0.0f;
        S.b[k].g_dim[0] = S.b[k].g_dim[1] = S.b[k].g_dim[2] = 0;
    }
    // ---- torn triangles (world.cpp:1870-1878)
    for (int k = 0; k < nb; k++) {
        const Body& B = bodies[S.b[k].id];
        if (B.sleeping) continue;
        for (int t = tid; t < B.ntris; t += nt) {
            const int tg = B.tri0 + t;
            int4 tr = C.tri[tg];
            const float r2 = C.tri_rest2[tg];
            if (!(tr.w & TF_TORN) && r2 > 0 && max_edge2(nd_p(nd, tr.x), nd_p(nd, tr.y), nd_p(nd, tr.z)) > kTornStretch2 * r2) {
                tr.w |= TF_TORN;
                C.tri[tg] = tr;
            }
        }
    }
    __syncthreads();
    const float dt = C.dt;
    const int interval = C.interval;
    if (tid == 0) {
        float rmax = 0.0f, slow = 0.0f;
        for (int k = 0; k < nb; k++) {
            const Body& B = bodies[S.b[k].id];
            rmax = smax(rmax, B.crad);
            if (S.b[k].sp <= kFastSpeed) slow = smax(slow, S.b[k].sp);
        }
        const float speed = slow + 0.5f;
        S.rmax = rmax;
        S.margin = 2.0f * speed * (float)interval * dt + 0.02f;
        S.slow_reach = 2.0f * speed * (float)interval * dt + 0.01f;
        S.travel = 1.25f * (float)interval * dt;
        S.T = (float)max(interval, 1) * dt;
        S.root = root;
    }
    __syncthreads();
    // ---- bulk speeds of the fast bodies: mass-weighted RMS in node order, in double (world.cpp:1891-1902)
    for (int k = 0; k < nb; k++) {
        const Body& B = bodies[S.b[k].id];
        if (B.sleeping || !(S.b[k].sp > kFastSpeed)) continue;
        double mv2 = 0.0, m = 0.0;
        for (int c0 = 0; c0 < B.nnodes; c0 += nt) {
            const int i = c0 + tid;
            if (i < B.nnodes) {
                const float4 v = nd[2 * (B.node0 + i) + 1];
                RS.term0[tid] = (double)v.w * length2(V(v.x, v.y, v.z));
                RS.term1[tid] = (double)v.w;
            }
            __syncthreads();
            if (tid == 0) {
                const int n = min(nt, B.nnodes - c0);
                for (int j = 0; j < n; j++) mv2 += RS.term0[j], m += RS.term1[j]; // (two running sums, each in node order)
            }
            __syncthreads();
        }
        if (tid == 0) {
            const float bulk = clampf(m > 0 ? 1.25f * (float)sqrt(mv2 / m) : S.b[k].sp, kFastSpeed, 400.0f);
            S.b[k].bulk = bulk;
            S.b[k].extra = bulk * (float)interval * dt;
        }
        __syncthreads();
    }
    // ---- cell size: the mean longest edge of every 7th triangle, in double (world.cpp:1914-1926)
    {
        double tri_size = 0.0;
        int samples = 0;
        for (int k = 0; k < nb; k++) {
            const Body& B = bodies[S.b[k].id];
            const int ns = (B.ntris + 6) / 7;
            for (int c0 = 0; c0 < ns; c0 += nt) {
                const int q = c0 + tid;
                if (q < ns) {
                    const int4 tr = C.tri[B.tri0 + 7 * q];
                    RS.term0[tid] = (double)sqrtf(max_edge2(nd_p(nd, tr.x), nd_p(nd, tr.y), nd_p(nd, tr.z)));
                }
                __syncthreads();
                if (tid == 0) serial_add(tri_size, RS.term0, min(nt, ns - c0));
                __syncthreads();
            }
            samples += ns;
        }
        if (tid == 0) {
            const float mean = samples ? (float)(tri_size / samples) : 1.0f;
            S.inv_cell = 1.0f / clampf(mean + 2.0f * (S.rmax + S.margin), 0.25f, 1.0f);
        }
    }
    __syncthreads();
    // ---- partners: bodies whose boxes, grown by the reach, overlap (world.cpp:1933-1954)
    const float reach = S.rmax + S.margin;
    for (int k = tid; k < nb; k += nt) {
        const Body& B = bodies[S.b[k].id];
        const float g = reach + S.b[k].extra + (B.hull ? B.hull_depth : 0.0f);
        for (int c = 0; c < 3; c++) S.b[k].bmn[c] = S.b[k].mn[c] - g, S.b[k].bmx[c] = S.b[k].mx[c] + g;
    }
    __syncthreads();
    for (int q = tid; q < nb * nb; q += nt) {
        const int a = q / nb, b = q % nb;
        if (b <= a) continue;
        const Body& A = bodies[S.b[a].id];
        const Body& Bb = bodies[S.b[b].id];
        if (same_group(A, Bb) || (A.sleeping && Bb.sleeping)) continue;
        if (!(S.b[a].bmn[0] <= S.b[b].bmx[0] && S.b[a].bmx[0] >= S.b[b].bmn[0] && S.b[a].bmn[1] <= S.b[b].bmx[1] && S.b[a].bmx[1] >= S.b[b].bmn[1] &&
              S.b[a].bmn[2] <= S.b[b].bmx[2] && S.b[a].bmx[2] >= S.b[b].bmn[2]))
            continue;
        atomicOr(&S.partner[a][b >> 5], 1u << (b & 31));
        atomicOr(&S.partner[b][a >> 5], 1u << (a & 31));
    }
    __syncthreads();
    // ---- the spatial hash of the slow bodies' contacter nodes (world.cpp:1966-1978), in body and node order
    const int pt0 = C.isl_noff[root];
    const int bk0 = 4 * pt0 + 65 * slot;
    {
        int base = 0;
        for (int k = 0; k < nb; k++) {
            const Body& B = bodies[S.b[k].id];
            if (!has_partner(S, k) || S.b[k].extra > 0) continue;
            for (int c0 = 0; c0 < B.nnodes; c0 += nt) {
                const int i = c0 + tid;
                bool take = false;
                int4 cell = make_int4(0, 0, 0, 0);
                if (i < B.nnodes && ((uint32_t)info[B.node0 + i].x & NF_CONTACTER)) {
                    const v3 p = nd_p(nd, B.node0 + i);
                    if (near_partner(S, k, p, p)) {
                        take = true;
                        cell = make_int4(cell_of(p.x, S.inv_cell), cell_of(p.y, S.inv_cell), cell_of(p.z, S.inv_cell), 0);
                    }
                }
                int tot;
                const int at = block_scan_excl(take ? 1 : 0, tot, RS.warp);
                if (take) {
                    C.pt_node[pt0 + base + at] = B.node0 + i;
                    C.pt_body[pt0 + base + at] = S.b[k].id;
                    C.pt_cell[pt0 + base + at] = cell;
                }
                base += tot;
            }
        }
        if (tid == 0) {
            int nbk = 64;
            while (nbk < 2 * base) nbk <<= 1;
            RS.npts = base, S.mask = nbk - 1, S.bk0 = bk0, S.pt0 = pt0;
        }
        __syncthreads();
    }
    const int npts = RS.npts, nbk = S.mask + 1;
    int any_tris = 0;
    for (int k = 0; k < nb; k++) any_tris |= bodies[S.b[k].id].ntris > 0;
    const bool slow_search = npts > 0 && any_tris;
    if (slow_search) {
        // buckets: counts, starts, items (each bucket in node order), then the records in bucket order and the runs
        // of one body's records
        for (int q = tid; q <= nbk; q += nt) C.bk_start[bk0 + q] = 0;
        __syncthreads();
        for (int q = tid; q < npts; q += nt) {
            const int4 c = C.pt_cell[pt0 + q];
            atomicAdd(&C.bk_start[bk0 + (int)(cell_hash(c.x, c.y, c.z) & (uint32_t)S.mask) + 1], 1);
        }
        __syncthreads();
        block_scan_incl_inplace(C.bk_start + bk0, nbk + 1, RS.warp);
        __syncthreads();
        for (int q = tid; q < nbk; q += nt) C.bk_fill[bk0 + q] = C.bk_start[bk0 + q];
        __syncthreads();
        for (int q = tid; q < npts; q += nt) {
            const int4 c = C.pt_cell[pt0 + q];
            const int at = atomicAdd(&C.bk_fill[bk0 + (int)(cell_hash(c.x, c.y, c.z) & (uint32_t)S.mask)], 1);
            C.bk_items[pt0 + at] = q;
        }
        __syncthreads();
        for (int q = tid; q < nbk; q += nt) {
            const int k0 = C.bk_start[bk0 + q], k1 = C.bk_start[bk0 + q + 1];
            for (int i = k0 + 1; i < k1; i++) {
                const int v = C.bk_items[pt0 + i];
                int j = i - 1;
                while (j >= k0 && C.bk_items[pt0 + j] > v) C.bk_items[pt0 + j + 1] = C.bk_items[pt0 + j], j--;
                C.bk_items[pt0 + j + 1] = v;
            }
        }
        __syncthreads();
        for (int i = tid; i < npts; i += nt) {
            const int pi = C.bk_items[pt0 + i];
            const int4 c = C.pt_cell[pt0 + pi];
            const int node = C.pt_node[pt0 + pi];
            const v3 p = nd_p(nd, node);
            C.sb_cell[pt0 + i] = make_int4(c.x, c.y, c.z, C.pt_body[pt0 + pi]);
            C.sb_pos[pt0 + i] = make_float4(p.x, p.y, p.z, __int_as_float(node));
        }
        __syncthreads();
        for (int q = tid; q < nbk; q += nt) {
            const int k0 = C.bk_start[bk0 + q], k1 = C.bk_start[bk0 + q + 1];
            for (int i = k1; i-- > k0;) {
                const bool same = i + 1 < k1 && C.sb_cell[pt0 + i + 1].w == C.sb_cell[pt0 + i].w;
                C.run_end[pt0 + i] = same ? C.run_end[pt0 + i + 1] : i + 1;
            }
        }
        __syncthreads();
    }
    // ---- the fast bodies' dense grids (world.cpp:2330-2362), each in cells of its own: every contacter node in the
    // lowest cell of its travel (counts, starts, items ascending within a cell), then its records in cell order
    {
        int noff = 0; // (the body's nodes' place in the island's scratch)
        for (int kf = 0; kf < nb; kf++) {
            const Body& F = bodies[S.b[kf].id];
            const int my_off = noff;
            noff += F.nnodes;
            if (!(S.b[kf].extra > 0) || !has_partner(S, kf)) continue; // (without partners it has no pairs)
            IslBody& G = S.b[kf];
            if (tid == 0) {
                float rmx = 0.0f;
                for (int ko = 0; ko < nb; ko++)
                    if (is_partner(S, kf, ko)) {
                        const float fe = S.b[ko].extra > 0 ? S.b[ko].bulk * (float)interval * dt : 0.0f;
                        rmx = smax(rmx, F.crad + S.slow_reach + fe);
                    }
                const float ex = G.mx[0] - G.mn[0] + 2e-3f, ey = G.mx[1] - G.mn[1] + 2e-3f, ez = G.mx[2] - G.mn[2] + 2e-3f;
                float cellsz = clampf(2.0f * rmx, 0.15f, 2.0f);
                cellsz = smax(cellsz, smax(ex, smax(ey, ez)) / 48.0f);
                G.g_inv = 1.0f / cellsz;
                G.g_org[0] = G.mn[0] - 1e-3f, G.g_org[1] = G.mn[1] - 1e-3f, G.g_org[2] = G.mn[2] - 1e-3f;
                G.g_dim[0] = max(1, min(48, (int)(ex * G.g_inv) + 1));
                G.g_dim[1] = max(1, min(48, (int)(ey * G.g_inv) + 1));
                G.g_dim[2] = max(1, min(48, (int)(ez * G.g_inv) + 1));
                G.g_span[0] = G.g_span[1] = G.g_span[2] = 0;
                const int ncell = G.g_dim[0] * G.g_dim[1] * G.g_dim[2];
                const int gs = atomicAdd(C.sc + 3, ncell + 1);
                if (gs + ncell + 1 > C.cell_cap) {
                    atomicOr(deverr, DEVERR_PAIRS);
                    RS.fail = 1;
                    G.gs0 = -1;
                } else {
                    G.gs0 = gs;
                }
                G.gi0 = pt0 + my_off;
            }
            __syncthreads();
            if (G.gs0 < 0) continue;
            const int ncell = G.g_dim[0] * G.g_dim[1] * G.g_dim[2], gs0 = G.gs0, gi0 = G.gi0;
            for (int q = tid; q <= ncell; q += nt) C.g_start[gs0 + q] = 0;
            __syncthreads();
            for (int i = tid; i < F.nnodes; i += nt) {
                if (!((uint32_t)info[F.node0 + i].x & NF_CONTACTER)) continue;
                float m;
                int3 lo, hi;
                node_cells(G, S.travel, nd_p(nd, F.node0 + i), nd_v(nd, F.node0 + i), m, lo, hi);
                atomicAdd(&C.g_start[gs0 + (lo.z * G.g_dim[1] + lo.y) * G.g_dim[0] + lo.x + 1], 1);
                if (hi.x - lo.x > G.g_span[0]) atomicMax(&G.g_span[0], hi.x - lo.x);
                if (hi.y - lo.y > G.g_span[1]) atomicMax(&G.g_span[1], hi.y - lo.y);
                if (hi.z - lo.z > G.g_span[2]) atomicMax(&G.g_span[2], hi.z - lo.z);
            }
            __syncthreads();
            block_scan_incl_inplace(C.g_start + gs0, ncell + 1, RS.warp);
            __syncthreads();
            for (int q = tid; q < ncell; q += nt) C.g_fill[gs0 + q] = C.g_start[gs0 + q];
            __syncthreads();
            for (int i = tid; i < F.nnodes; i += nt) {
                if (!((uint32_t)info[F.node0 + i].x & NF_CONTACTER)) continue;
                float m;
                int3 lo, hi;
                node_cells(G, S.travel, nd_p(nd, F.node0 + i), nd_v(nd, F.node0 + i), m, lo, hi);
                const int at = atomicAdd(&C.g_fill[gs0 + (lo.z * G.g_dim[1] + lo.y) * G.g_dim[0] + lo.x], 1);
                C.g_items[gi0 + at] = F.node0 + i;
            }
            __syncthreads();
            for (int q = tid; q < ncell; q += nt) {
                const int k0 = C.g_start[gs0 + q], k1 = C.g_start[gs0 + q + 1];
                for (int i = k0 + 1; i < k1; i++) {
                    const int v = C.g_items[gi0 + i];
                    int j = i - 1;
                    while (j >= k0 && C.g_items[gi0 + j] > v) C.g_items[gi0 + j + 1] = C.g_items[gi0 + j], j--;
                    C.g_items[gi0 + j + 1] = v;
                }
            }
            __syncthreads();
            const int cnt = C.g_start[gs0 + ncell];
            for (int i = tid; i < cnt; i += nt) {
                const int node = C.g_items[gi0 + i];
                const v3 p = nd_p(nd, node);
                float m;
                int3 lo, hi;
                node_cells(G, S.travel, p, nd_v(nd, node), m, lo, hi);
                C.g_rec[gi0 + i] = make_float4(p.x, p.y, p.z, m);
                C.g_hi[gi0 + i] = hi.x | hi.y << 8 | hi.z << 16;
            }
            __syncthreads();
        }
    }
    // ---- the island's queries, in the reference's order: the slow search (bodies with partners, triangles in order),
    // then the fast pairs (fast bodies with partners; their partners in body order)
    if (tid == 0) {
        const bool fail = RS.fail != 0;
        for (int pass = 0; pass < 2; pass++) {
            int ng = 0, nq = 0, nch = 0, g = RS.g_base, c = RS.c_base, q = S.inst0;
            auto add = [&](int kind, int k, int ko, int ntris) {
                if (ntris <= 0) return;
                if (pass == 1) {
                    C.q_group[g] = make_int4(slot, kind | k << 1 | ko << 9, ntris, q);
                    for (int t = 0; t < ntris; t += kQueryChunk) C.q_chunk[c++] = make_int2(g, t);
                    g++, q += ntris;
                }
                ng++, nq += ntris, nch += (ntris + kQueryChunk - 1) / kQueryChunk;
            };
            if (!fail) {
                if (slow_search)
                    for (int kt = 0; kt < nb; kt++)
                        if (has_partner(S, kt)) add(0, kt, 0, bodies[S.b[kt].id].ntris);
                for (int kf = 0; kf < nb; kf++) {
                    if (!(S.b[kf].extra > 0) || !has_partner(S, kf)) continue;
                    for (int ko = 0; ko < nb; ko++)
                        if (is_partner(S, kf, ko)) add(1, kf, ko, bodies[S.b[ko].id].ntris);
                }
            }
            if (pass == 1) break;
            S.inst0 = 0, S.ninst = fail ? -1 : 0, RS.g_base = 0, RS.c_base = 0;
            if (ng > 0) {
                const int q0 = atomicAdd(C.sc + 0, nq), g0 = atomicAdd(C.sc + 1, ng), c0 = atomicAdd(C.sc + 2, nch);
                if (q0 + nq > C.q_cap || g0 + ng > C.grp_cap || c0 + nch > C.chunk_cap) {
                    atomicOr(deverr, DEVERR_PAIRS);
                    for (int e = c0; e < min(c0 + nch, C.chunk_cap); e++) C.q_chunk[e] = make_int2(-1, 0); // (its chunks: empty)
                    S.ninst = -1;
                    break;
                }
                S.inst0 = q0, S.ninst = nq, RS.g_base = g0, RS.c_base = c0;
            } else {
                break;
            }
        }
        if (S.ninst < 0) C.isl_poff[root] = 0, C.isl_pcnt[root] = 0;
    }
    __syncthreads();
    {
        const int4* src = reinterpret_cast<const int4*>(&S);
        int4* dst = reinterpret_cast<int4*>(C.isl + slot);
        for (int i = tid; i < (int)(sizeof(IslSearch) / sizeof(int4)); i += nt) dst[i] = src[i];
    }
}

// one query: triangle t of group g (kind 0: island body k's triangles against the slow hash; kind 1: partner ko's
// triangles against fast body k's grid); out: where its pairs go (the first cap of them), or null to count them
__device__ __forceinline__ int run_query(const IslSearch& S, const Contacts& C, const Body* __restrict__ bodies, const float4* __restrict__ nd, int4 g,
                                         int t, int2* out, int cap) {
    const int kind = g.y & 1, k = (g.y >> 1) & 255, ko = g.y >> 9;
    const int tg = bodies[S.b[kind ? ko : k].id].tri0 + t;
    return kind ? fast_query(S, C, bodies, nd, k, ko, tg, out, cap) : slow_query(S, C, bodies, nd, k, tg, out, cap);
}

// every island's queries, kQueryChunk to a CTA: their pairs counted; a query's pairs, up to kLocPairs of them, kept in
// ptmp (q_tmp: where; -1: the query runs again to write them)
__global__ void __launch_bounds__(kQueryChunk) k_pair_count(const Body* __restrict__ bodies, const float4* __restrict__ nd, Contacts C) {
    const int nch = min(C.sc[2], C.chunk_cap);
    for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const int2 cg = C.q_chunk[ch];
        if (cg.x < 0) continue;
        const int4 g = C.q_group[cg.x];
        const int t = cg.y + (int)threadIdx.x;
        if (t >= g.z) continue;
        int2 loc[kLocPairs];
        const int n = run_query(C.isl[g.x], C, bodies, nd, g, t, loc, kLocPairs);
        C.q_count[g.w + t] = n;
        if (n > 0) {
            int at = -1;
            if (n <= kLocPairs) {
                at = atomicAdd(C.sc + 4, n);
                if (at + n <= C.ptmp_cap)
                    for (int k = 0; k < n; k++) C.ptmp[at + k] = loc[k];
                else
                    at = -1;
            }
            C.q_tmp[g.w + t] = at;
        }
    }
}

// one CTA per island with pairs: its queries' counts become their running sum, its range comes from the pair list
__global__ void __launch_bounds__(1024) k_pair_place(const Body* __restrict__ bodies, int nbodies, Contacts C, uint32_t* __restrict__ deverr) {
    const int root = blockIdx.x;
    if (root >= nbodies) return;
    {
        const Body& R = bodies[root];
        if (!R.pairs || R.island != root) return;
    }
    __shared__ int s_warp[32];
    const IslSearch& S = C.isl[C.isl_idx[root]];
    const int inst0 = S.inst0, ninst = S.ninst;
    if (ninst < 0) return;
    block_scan_incl_inplace(C.q_count + inst0, ninst, s_warp);
    __syncthreads();
    if (threadIdx.x == 0) {
        const int total = ninst > 0 ? C.q_count[inst0 + ninst - 1] : 0;
        int off = atomicAdd(C.pair_total, total);
        if (off + total > C.max_pairs) {
            atomicOr(deverr, DEVERR_PAIRS);
            off = -1;
        }
        C.isl_poff[root] = off < 0 ? 0 : off;
        C.isl_pcnt[root] = off < 0 ? 0 : total;
        if (off >= 0) atomicAdd(&C.counters[2], total), atomicAdd(&C.counters[0], 1);
    }
}

// the queries' pairs at their places: copied from ptmp, or the query run again where they were not kept
__global__ void __launch_bounds__(kQueryChunk) k_pair_write(const Body* __restrict__ bodies, const float4* __restrict__ nd, Contacts C) {
    const int nch = min(C.sc[2], C.chunk_cap);
    for (int ch = blockIdx.x; ch < nch; ch += gridDim.x) {
        const int2 cg = C.q_chunk[ch];
        if (cg.x < 0) continue;
        const int4 g = C.q_group[cg.x];
        const int t = cg.y + (int)threadIdx.x;
        if (t >= g.z) continue;
        const IslSearch& S = C.isl[g.x];
        const int q = g.w + t;
        const int start = q > S.inst0 ? C.q_count[q - 1] : 0;
        if (C.q_count[q] == start) continue;
        const int root = S.root;
        if (C.isl_pcnt[root] == 0) continue; // (the pair list was full)
        int2* dst = C.pairs + C.isl_poff[root] + start;
        const int at = C.q_tmp[q];
        if (at >= 0)
            for (int k = 0, n = C.q_count[q] - start; k < n; k++) dst[k] = C.ptmp[at + k];
        else
            run_query(S, C, bodies, nd, g, t, dst, 0x7fffffff);
    }
}

} // namespace blg
