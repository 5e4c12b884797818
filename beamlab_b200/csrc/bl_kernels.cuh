// Kernels of the explicit substep. Per frame (World::step_substeps, world.cpp:368-585):
//
//   k_frame_begin     one thread per body: static candidates over the box grown by its travel, terrain height bound
//   n x { k_beams     one thread per beam: spring-damper, plastic yield, break -> the beam's force scalar (fsc)
//         k_force     one thread per node: gravity + its beams' forces in beam order (each made again from the scalar
//                     and the two positions) -> the node's force
//         (contacts between bodies add to the force: bl_contacts.cuh)
//         k_integrate } one thread per node: static contact, integration, bounds / top speed / contacts per body
//   k_frame_finish    one block: each body's bounds, top speed, repair of runaway nodes, sleep
//   k_sleep_apply     one block per body: a body that fell asleep stops (velocities zero, beams parked)
//
// Determinism: k_force sums a node's forces in the order the reference's serial loop adds them (gravity, then each
// beam in index order: f[a] += fv, f[b] -= fv; softbody.cpp:330-470), from a per-node list of incident beams sorted
// by beam index, so no atomics touch a force; fv = (p_a - p_b) * scalar rounds exactly as the reference's product.
#pragma once

#include "bl_device.cuh"

#include <type_traits>

namespace blg {

// ------------------------------------------------------------------------------------------ statics queries
// Heightfield::sample (static_world.cpp:189-205)
__device__ __forceinline__ bool hf_sample(const Statics& st, float x, float z, float& out_h, v3& n) {
    const float lx = (x - st.ox) / st.cell, lz = (z - st.oz) / st.cell;
    if (!(lx >= 0 && lz >= 0 && lx < st.hnx - 1 && lz < st.hnz - 1)) return false;
    const int ix = (int)lx, iz = (int)lz;
    const float fx = lx - ix, fz = lz - iz;
    const float* row0 = st.h + (size_t)iz * st.hnx;
    const float* row1 = row0 + st.hnx;
    const float h00 = row0[ix], h10 = row0[ix + 1], h01 = row1[ix], h11 = row1[ix + 1];
    if (smin(smin(h00, h10), smin(h01, h11)) < -1e29f) return false;
    if (fx > fz) {
        out_h = h00 + (h10 - h00) * fx + (h11 - h10) * fz;
        n = normalize(V(-(h10 - h00) / st.cell, 1.0f, -(h11 - h10) / st.cell));
    } else {
        out_h = h00 + (h11 - h01) * fx + (h01 - h00) * fz;
        n = normalize(V(-(h11 - h01) / st.cell, 1.0f, -(h01 - h00) / st.cell));
    }
    return true;
}

// Heightfield::surface_at (static_world.cpp:213-218)
__device__ __forceinline__ int hf_surface_at(const Statics& st, float x, float z) {
    int ix = (int)lroundf((x - st.ox) / st.cell), iz = (int)lroundf((z - st.oz) / st.cell);
    ix = max(0, min(st.hnx - 1, ix));
    iz = max(0, min(st.hnz - 1, iz));
    return st.surf[(size_t)iz * st.hnx + ix];
}

// Heightfield::max_height (static_world.cpp:220-231)
__device__ float hf_max_height(const Statics& st, float x0, float z0, float x1, float z1) {
    const int kBlock = 16;
    int bx0 = (int)floorf((x0 - st.ox) / st.cell) / kBlock, bx1 = (int)floorf((x1 - st.ox) / st.cell) / kBlock;
    int bz0 = (int)floorf((z0 - st.oz) / st.cell) / kBlock, bz1 = (int)floorf((z1 - st.oz) / st.cell) / kBlock;
    bx0 = max(0, bx0);
    bz0 = max(0, bz0);
    bx1 = min(st.bx - 1, bx1);
    bz1 = min(st.bz - 1, bz1);
    float m = -1e30f;
    for (int bz = bz0; bz <= bz1; bz++)
        for (int bx = bx0; bx <= bx1; bx++) m = smax(m, st.block_max[(size_t)bz * st.bx + bx]);
    return m;
}

struct Contact {
    v3 normal;
    float depth;
    int surface;
    float max_force;
};

// StaticWorld::collide_point (static_world.cpp:364-474), boxes without hull planes
__device__ bool collide_point(const Statics& st, v3 p, float r, const int* box_ids, int nbox, const int* cyl_ids, int ncyl, bool test_terrain,
                              Contact& out) {
    bool hit = false;
    out.depth = 0;
    out.max_force = 0;
    out.surface = 0;
    out.normal = V(0, 0, 0);
    if (test_terrain && st.has_terrain) {
        float th;
        v3 n;
        if (hf_sample(st, p.x, p.z, th, n)) {
            const float d = (th - p.y) * n.y + r;
            if (d > 0) {
                out.depth = d;
                out.normal = n;
                out.surface = hf_surface_at(st, p.x, p.z);
                hit = true;
            }
        }
    }
    for (int k = 0; k < nbox; k++) {
        const Box& b = st.boxes[box_ids[k]];
        if (p.x < b.mnx - r || p.x > b.mxx + r || p.y < b.mny - r || p.y > b.mxy + r || p.z < b.mnz - r || p.z > b.mxz + r) continue;
        const v3 c0 = V(b.r[0], b.r[1], b.r[2]), c1 = V(b.r[3], b.r[4], b.r[5]), c2 = V(b.r[6], b.r[7], b.r[8]);
        const v3 rel = p - V(b.cx, b.cy, b.cz);
        const v3 l = V(dot(rel, c0), dot(rel, c1), dot(rel, c2));
        const v3 q = V(clampf(l.x, -b.hx, b.hx), clampf(l.y, -b.hy, b.hy), clampf(l.z, -b.hz, b.hz));
        const v3 d = l - q;
        const float dist2 = dot(d, d);
        float depth;
        v3 nl;
        if (dist2 > 1e-12f) {
            if (dist2 >= r * r) continue;
            const float dist = sqrtf(dist2);
            depth = r - dist;
            nl = divs(d, dist);
        } else {
            const v3 pen = V(b.hx, b.hy, b.hz) - vabs(l);
            if (pen.x <= pen.y && pen.x <= pen.z) depth = pen.x, nl = V(signf(l.x), 0, 0);
            else if (pen.y <= pen.z) depth = pen.y, nl = V(0, signf(l.y), 0);
            else depth = pen.z, nl = V(0, 0, signf(l.z));
            depth += r;
        }
        if (depth > out.depth) {
            out.depth = depth;
            out.normal = c0 * nl.x + c1 * nl.y + c2 * nl.z;
            out.surface = b.surface;
            out.max_force = b.max_force;
            hit = true;
        }
    }
    for (int k = 0; k < ncyl; k++) {
        const Cyl& c = st.cyls[cyl_ids[k]];
        const v3 rel = p - V(c.bx, c.by, c.bz);
        if (rel.y < -r || rel.y > c.height + r) continue;
        if (fabsf(rel.x) >= c.radius + r || fabsf(rel.z) >= c.radius + r) continue;
        const float dxz = sqrtf(rel.x * rel.x + rel.z * rel.z);
        const float side = c.radius + r - dxz;
        const float top = c.height + r - rel.y;
        if (side <= 0) continue;
        float depth;
        v3 n;
        if (top < side && rel.y > c.height * 0.5f) depth = top, n = V(0, 1, 0);
        else depth = side, n = dxz > 1e-6f ? V(rel.x / dxz, 0, rel.z / dxz) : V(1, 0, 0);
        if (depth > out.depth) {
            out.depth = depth;
            out.normal = n;
            out.surface = c.surface;
            hit = true;
        }
    }
    return hit;
}

// primitive_collision (static_world.cpp:8-51)
__device__ v3 primitive_collision(v3 F, v3 vel, float mass, v3 normal, float dt, const GroundModel& gm, float pen, float friction_coef, float push_max,
                                  float slop, float restitution) {
    v3 out = V(0, 0, 0);
    const float Vn = dot(vel, normal);
    const float Fn = dot(F, normal);
    const float sgl = gm.soft_depth;
    if (sgl > 0 && pen >= 0) {
        out = out + vel * (-gm.fluid_drag * smin(1.0f, pen / sgl + 0.2f));
        float Fb = gm.fluid_density * smin(pen, sgl) * 9.807f * 0.02f;
        if (Vn >= 0 && Fn < 0 && Fb > -Fn) Fb = -Fn;
        out = out + normal * Fb;
    }
    if (pen >= sgl) {
        float R = -Fn;
        const float take = restitution >= 0 ? 1.0f + smin(restitution, 0.95f) : 0.8f;
        if (Vn < 0) R -= (take * Vn - smin(0.2f * smax(0.0f, pen - sgl - slop) / dt, push_max)) * mass / dt;
        if (R > 0) {
            const v3 slipF = F - normal * Fn;
            v3 slip = vel - normal * Vn;
            const float sv = length(slip);
            if (sv > 1e-9f) slip = divs(slip, sv);
            else slip = V(0, 0, 0);
            const float G = R * gm.strength * friction_coef;
            const float stop = mass * sv / dt;
            if (sv < gm.va && G > 0 && length(slipF) <= gm.ms * G) {
                out = out + (normal * R - slip * smin(gm.ms * G * (1.0f - bl_expf(-sv / gm.va)), stop) - slipF);
            } else {
                const float g = gm.mc + (gm.ms - gm.mc) * bl_expf(-bl_powf(sv / gm.vs, gm.alpha));
                out = out + (normal * R - slip * smin((g + smin(gm.t2 * sv, 5.0f)) * G, smax(0.0f, stop + dot(slipF, slip))));
            }
        }
    }
    return out;
}

// AABB::overlaps (math.h:307-309) of a box's bounds with (mn, mx)
__device__ __forceinline__ bool box_overlaps(const Box& b, const float* mn, const float* mx) {
    return b.mnx <= mx[0] && b.mxx >= mn[0] && b.mny <= mx[1] && b.mxy >= mn[1] && b.mnz <= mx[2] && b.mxz >= mn[2];
}

// ------------------------------------------------------------------------------------------ per frame
// The frame's start for each awake body: its static candidates (StaticWorld::query over its box grown by its travel,
// world.cpp:738-753; static_world.cpp:340-362) and the terrain's height bound there. Sleeping bodies are skipped,
// as build_islands drops their islands (world.cpp:703-713).
__global__ void k_frame_begin(Body* __restrict__ bodies, int nbodies, Statics st, float frame_time, int world_sleeping, uint32_t* __restrict__ deverr) {
    const int bi = blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= nbodies) return;
    Body& B = bodies[bi];
    if (!world_sleeping) B.sleeping = 0;
    if (B.sleeping && B.island < 0) return; // (an island asleep as a whole is not stepped; a sleeping body beside a
                                            // moving one is, and may be woken by it)
    const float m = smin(B.max_speed, 200.0f) * frame_time * 2.0f + 0.5f;
    const float mn[3] = {B.aabb_mn[0] - m, B.aabb_mn[1] - m, B.aabb_mn[2] - m};
    const float mx[3] = {B.aabb_mx[0] + m, B.aabb_mx[1] + m, B.aabb_mx[2] + m};
    int n = 0;
    bool over = false;
    for (int k = 0; k < st.nbig; k++) {
        const int i = st.big[k];
        if (box_overlaps(st.boxes[i], mn, mx)) {
            if (n < kMaxCand) B.box_ids[n] = i;
            n++;
        }
    }
    if (st.gx > 0) {
        int x0 = (int)((mn[0] - st.gox) / st.grid_cell), x1 = (int)((mx[0] - st.gox) / st.grid_cell);
        int z0 = (int)((mn[2] - st.goz) / st.grid_cell), z1 = (int)((mx[2] - st.goz) / st.grid_cell);
        x0 = max(0, x0), z0 = max(0, z0), x1 = min(st.gx - 1, x1), z1 = min(st.gz - 1, z1);
        if (mx[0] >= st.gox && mx[2] >= st.goz)
            for (int z = z0; z <= z1; z++)
                for (int x = x0; x <= x1; x++)
                    for (int q = st.cell_ptr[z * st.gx + x]; q < st.cell_ptr[z * st.gx + x + 1]; q++) {
                        const int i = st.cell_items[q];
                        if (!box_overlaps(st.boxes[i], mn, mx)) continue;
                        bool dup = false;
                        for (int k = 0; k < min(n, kMaxCand); k++)
                            if (B.box_ids[k] == i) {
                                dup = true;
                                break;
                            }
                        if (dup) continue;
                        if (n < kMaxCand) B.box_ids[n] = i;
                        n++;
                    }
    }
    if (n > kMaxCand) over = true, n = kMaxCand;
    B.nbox = n;
    int nc = 0;
    for (int i = 0; i < st.ncyls; i++) {
        const Cyl& c = st.cyls[i];
        if (mx[0] >= c.bx - c.radius && mn[0] <= c.bx + c.radius && mx[2] >= c.bz - c.radius && mn[2] <= c.bz + c.radius && mx[1] >= c.by &&
            mn[1] <= c.by + c.height) {
            if (nc < kMaxCand) B.cyl_ids[nc] = i;
            nc++;
        }
    }
    if (nc > kMaxCand) over = true, nc = kMaxCand;
    B.ncyl = nc;
    if (over) atomicOr(deverr, DEVERR_CANDIDATES);
    B.terrain_max = st.has_terrain ? hf_max_height(st, mn[0], mn[2], mx[0], mx[2]) + 0.0f : -1e30f;
    B.acc_v2 = 0.0f;
    B.acc_contacts = 0;
    if (B.sleeping) B.max_speed = 0.0f; // (simulate_island's top speed of a sleeping body, world.cpp:3217-3222)
}

// ------------------------------------------------------------------------------------------ per substep
// SoftBody::compute_beam_forces, one beam (softbody.cpp:412-470), from its loaded state: meta, s0 = (L, max_pos,
// max_neg, strength), c = (k, d), its ends' states. Nothing is written: the caller stores what BeamOut says. The
// beam's force on its end a is dis * sc (dis = p_a - p_b), on b its negative; sc = kNoPush when the beam does not push.
struct BeamOut {
    float sc;          // force scalar (kNoPush: none)
    float slen;        // Beam::stress (stored when wr_stress)
    float4 s;          // L, max_pos, max_neg, strength after the substep (stored when changed)
    uint32_t meta;     // the meta word after the substep (stored when broke)
    bool wr_stress, changed, broke;
};

__device__ __forceinline__ BeamOut beam_eval(int j, uint32_t meta, float4 s0, float2 c, float4 pa, float4 va, float4 pb, float4 vb,
                                             const float4* __restrict__ bcold) {
    BeamOut o;
    o.sc = kNoPush, o.slen = 0.0f, o.s = s0, o.meta = meta, o.wr_stress = false, o.changed = false, o.broke = false;
    if (meta & kBeamAsleep) return o;
    const uint32_t type = meta & 0xffu;
    uint32_t flags = (meta >> 8) & 0xffu;
    if (!(flags & (BF_BROKEN | BF_SHOCK))) {
        const v3 dis = V(pa.x - pb.x, pa.y - pb.y, pa.z - pb.z);
        const float len2 = dot(dis, dis);
        if (!(len2 < 1e-12f)) { // (a NaN length goes on, as in the reference)
            float4 s = s0; // L, max_pos, max_neg, strength
            const float inv_len = 1.0f / sqrtf(len2);
            const float len = len2 * inv_len;
            const float diff = len - s.x;
            const v3 dv = V(va.x - vb.x, va.y - vb.y, va.z - vb.z);
            float k = c.x, d = c.y;
            const bool brk = (meta & BB_BREAK) != 0;
            bool broke = false, changed = false;
            if (type == BT_ROPE) {
                if (diff < 0) k = 0, d *= 0.1f;
            } else if (type == BT_SUPPORT) {
                if (diff > 0) {
                    k = 0;
                    d *= 0.1f;
                    if (brk && diff > s.x * bcold[j].z) broke = true;
                }
            }
            if (!broke) {
                float slen = -k * diff - d * dot(dv, dis) * inv_len;
                if ((meta & BB_DEFORM) && !(flags & BF_NO_DEFORM) && k != 0) {
                    if (slen > s.y && diff < 0) {
                        const float4 cold = bcold[j]; // plastic, L0, support_limit
                        const float yield_len = s.y / k;
                        const float def = diff + yield_len * (1.0f - cold.x);
                        const float Lold = s.x;
                        s.x = smax(smin(0.1f, 0.3f * cold.y), s.x + def);
                        slen = slen - (slen - s.y) * 0.5f;
                        if (s.x < Lold) s.y *= Lold / s.x;
                        changed = true;
                    } else if (slen < s.z && diff > 0) {
                        const float4 cold = bcold[j];
                        const float yield_len = s.z / k;
                        const float def = diff + yield_len * (1.0f - cold.x);
                        const float Lold = s.x;
                        s.x = s.x + def;
                        slen = slen - (slen - s.z) * 0.5f;
                        if (Lold > 0 && s.x > Lold) s.z *= s.x / Lold;
                        if (!(meta & BB_DUCTILE)) s.w -= def * k;
                        changed = true;
                    }
                }
                o.s = s, o.changed = changed;
                if (brk && fabsf(slen) > s.w && !(flags & BF_NO_BREAK)) {
                    broke = true;
                } else {
                    o.wr_stress = true, o.slen = slen;
                    o.sc = slen * inv_len; // (the force on a is dis * sc: the node's sum makes dis again from the same positions)
                }
            }
            if (broke) {
                flags |= BF_BROKEN;
                o.meta = (meta & ~(0xffu << 8)) | (flags << 8);
                o.broke = true;
            }
        }
    }
    return o;
}

// beam_eval with its results stored at once (k_beams: the next kernel reads the scalar from fsc)
__device__ __forceinline__ void beam_step(int j, uint32_t meta, float4 s0, float2 c, float4 pa, float4 va, float4 pb, float4 vb, float4* __restrict__ bst,
                                          uint32_t* __restrict__ bmeta, const float4* __restrict__ bcold, float* __restrict__ stress,
                                          const int* __restrict__ bbody, float* __restrict__ fsc, Body* __restrict__ bodies) {
    if (meta & kBeamAsleep) return;
    const BeamOut o = beam_eval(j, meta, s0, c, pa, va, pb, vb, bcold);
    if (o.changed) bst[j] = o.s;
    if (o.wr_stress) stress[j] = o.slen;
    if (o.broke) {
        bmeta[j] = o.meta;
        atomicAdd(&bodies[bbody[j]].broken_beams, 1);
    }
    fsc[j] = o.sc;
}

// ------------------------------------------------------------------------------------------ shocks
// SoftBody::compute_shock_forces (softbody.cpp:472-566), a thread a shock: its model's rates for the beam's length and
// rate (type 1 bounded, 2 progressive with soft bump stops, 3 split damping), the break test, the beam's stress, and
// the scalar its ends add after their beams' (k_force: ssc, in the order of the shocks)
struct ShockDev {
    const bl_shock* sh;      // the shocks, each body's in its order (beam: the global beam)
    const int* ptr;          // per node + 1: its shocks in sinc
    const int2* inc;         // (shock | bit 31 where the node is the beam's b end, the other end)
    float* ssc;              // per shock: its scalar (kNoPush: none this substep)
};
__global__ void k_shocks(ShockDev S, int nshocks, const int2* __restrict__ ab, const float4* __restrict__ bst, uint32_t* __restrict__ bmeta,
                         float* __restrict__ stress, const int* __restrict__ bbody, const float4* __restrict__ nd, Body* __restrict__ bodies) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nshocks) return;
    S.ssc[q] = kNoPush;
    const bl_shock s = S.sh[q];
    const int j = (int)s.beam;
    const uint32_t meta = bmeta[j];
    if ((meta & kBeamAsleep) || (((meta >> 8) & 0xffu) & BF_BROKEN)) return;
    const int2 e = ab[j];
    const float4 pa = nd[2 * e.x], va = nd[2 * e.x + 1], pb = nd[2 * e.y], vb = nd[2 * e.y + 1];
    const v3 dis = V(pa.x - pb.x, pa.y - pb.y, pa.z - pb.z);
    const float len2 = dot(dis, dis);
    if (len2 < 1e-12f) return;
    const float inv_len = 1.0f / sqrtf(len2);
    const float len = len2 * inv_len;
    const float4 b4 = bst[j];
    const float L = b4.x;
    const float diff = len - L;
    const float v = dot(V(va.x - vb.x, va.y - vb.y, va.z - vb.z), dis) * inv_len;
    float k, d;
    const float lb = s.long_bound * L, sb = s.short_bound * L;
    auto sqr = [](float x) { return x * x; };
    if (s.type == 1) {
        k = s.spring, d = s.damp;
        float r = 0;
        if (diff > lb) r = diff - lb;
        else if (diff < -sb) r = -diff - sb;
        if (r != 0) {
            r = smin(r, 1.0f);
            k += (s.bound_spring - k) * r;
            d += (s.bound_damp - d) * r;
        }
    } else if (s.type == 2) {
        auto prog = [&](bool out, float& kk, float& dd) {
            if (out) {
                kk = s.spring_out, dd = s.damp_out;
                const float fr = s.long_bound != 0 ? smin(sqr(diff / (s.long_bound * L)), 1.0f) : 1.0f;
                kk += s.prog_spring_out * kk * fr;
                dd += s.prog_damp_out * dd * fr;
            } else {
                kk = s.spring_in, dd = s.damp_in;
                const float fr = s.short_bound != 0 ? smin(sqr(diff / (s.short_bound * L)), 1.0f) : 1.0f;
                kk += s.prog_spring_in * kk * fr;
                dd += s.prog_damp_in * dd * fr;
            }
        };
        prog(v > 0, k, d);
        if (s.soft_bump) {
            const float Lp = 0.8f * L, lpre = s.long_bound * Lp, spre = -s.short_bound * Lp;
            if (diff > lpre) {
                prog(true, k, d);
                const float f2 = s.long_bound != 0 ? smin(sqr((diff - lpre) * 5.0f / (s.long_bound * L)), 1.0f) : 1.0f;
                k += (k + 100) * s.prog_spring_out * f2;
                d += (d + 100) * s.prog_damp_out * f2;
                if (v < 0) k = s.spring_in, d = s.damp_in;
            } else if (diff < spre) {
                prog(false, k, d);
                const float f2 = s.short_bound != 0 ? smin(sqr((diff - spre) * 5.0f / (s.short_bound * L)), 1.0f) : 1.0f;
                k += (k + 100) * s.prog_spring_out * f2;
                d += (d + 100) * s.prog_damp_out * f2;
                if (v > 0) k = s.spring_out, d = s.damp_out;
            }
            if (diff > lb || diff < -sb) {
                k = smax(k, s.bound_spring);
                d = smax(d, s.bound_damp);
            }
        } else if (diff > lb || diff < -sb) {
            k = s.bound_spring, d = s.bound_damp;
        }
    } else {
        k = s.spring_in, d = s.damp_in;
        if (diff > lb) {
            const float r = smin(diff - lb, 1.0f);
            k += (s.bound_spring - k) * r;
            d += (s.bound_damp - d) * r;
        } else if (diff < -sb) {
            const float r = smin(-diff - sb, 1.0f);
            k += (s.bound_spring - k) * r;
            d += (s.bound_damp - d) * r;
        } else if (v > 0) {
            const float w = clampf(fabsf(v), 0.15f, 20.0f);
            k = s.spring_out;
            d = (s.damp_out * s.damp_out_slow * smin(w, s.split_out) + s.damp_out * s.damp_out_fast * smax(0.0f, w - s.split_out)) / w;
        } else if (v < 0) {
            const float w = clampf(fabsf(v), 0.15f, 20.0f);
            k = s.spring_in;
            d = (s.damp_in * s.damp_in_slow * smin(w, s.split_in) + s.damp_in * s.damp_in_fast * smax(0.0f, w - s.split_in)) / w;
        }
    }
    const float slen = -k * diff - d * v;
    if ((meta & BB_BREAK) && fabsf(slen) > b4.w && !(((meta >> 8) & 0xffu) & BF_NO_BREAK)) {
        bmeta[j] = meta | ((uint32_t)BF_BROKEN << 8);
        atomicAdd(&bodies[bbody[j]].broken_beams, 1);
        return;
    }
    stress[j] = slen;
    S.ssc[q] = slen * inv_len;
}

// Two beams a thread (j and j + blockDim.x of the block's pair of tiles): both beams' loads are issued before either
// computes. Thread t < nbodies of the grid also resets body t's bounds accumulator for this substep's k_integrate.
__global__ void __launch_bounds__(256) k_beams(const int2* __restrict__ ab, const float2* __restrict__ kd, float4* __restrict__ bst,
                                               uint32_t* __restrict__ bmeta, const float4* __restrict__ bcold, float* __restrict__ stress,
                                               const int* __restrict__ bbody, float* __restrict__ fsc, const float4* __restrict__ nd,
                                               Body* __restrict__ bodies, int nbeams, int nbodies) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nbodies) {
        Body& B = bodies[t];
        B.acc_mn[0] = B.acc_mn[1] = B.acc_mn[2] = 1e30f;
        B.acc_mx[0] = B.acc_mx[1] = B.acc_mx[2] = -1e30f;
    }
    const int j0 = 2 * blockIdx.x * blockDim.x + threadIdx.x, j1 = j0 + blockDim.x;
    const bool h0 = j0 < nbeams, h1 = j1 < nbeams;
    const uint32_t m0 = h0 ? bmeta[j0] : kBeamAsleep, m1 = h1 ? bmeta[j1] : kBeamAsleep;
    const int2 e0 = h0 ? ab[j0] : make_int2(0, 0), e1 = h1 ? ab[j1] : make_int2(0, 0);
    const float4 s0 = h0 ? bst[j0] : make_float4(0, 0, 0, 0), s1 = h1 ? bst[j1] : make_float4(0, 0, 0, 0);
    const float2 c0 = h0 ? kd[j0] : make_float2(0, 0), c1 = h1 ? kd[j1] : make_float2(0, 0);
    float4 pa0 = make_float4(0, 0, 0, 0), va0 = pa0, pb0 = pa0, vb0 = pa0, pa1 = pa0, va1 = pa0, pb1 = pa0, vb1 = pa0;
    if (h0) pa0 = nd[2 * e0.x], va0 = nd[2 * e0.x + 1], pb0 = nd[2 * e0.y], vb0 = nd[2 * e0.y + 1];
    if (h1) pa1 = nd[2 * e1.x], va1 = nd[2 * e1.x + 1], pb1 = nd[2 * e1.y], vb1 = nd[2 * e1.y + 1];
    if (h0) beam_step(j0, m0, s0, c0, pa0, va0, pb0, vb0, bst, bmeta, bcold, stress, bbody, fsc, bodies);
    if (h1) beam_step(j1, m1, s1, c1, pa1, va1, pb1, vb1, bst, bmeta, bcold, stress, bbody, fsc, bodies);
}

// ------------------------------------------------------------------------------------------ bulk copies (TMA)
// cp.async.bulk global -> shared completing on an mbarrier: the beam arrays stream into shared memory tile after tile
// while the block computes earlier tiles. Every wait is bounded in time (the context's bulk_wait_s, 1 s by default): a
// copy that never lands raises DEVERR_TIMEOUT and the block lets the copies still in flight land (bounded by kWaitNs)
// and stops instead of waiting for ever.
constexpr unsigned long long kWaitNs = 1000000000ull; // 1 s
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// bytes and both addresses multiples of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// the generic proxy's reads of a buffer ordered before the async proxy's next writes into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// waits for the phase of `parity` to complete; false after limit_ns (limit 0: false at once, the run-out path's test)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, unsigned long long limit_ns = kWaitNs) {
    const uint32_t a = smem_u32(bar);
    uint32_t done = 0;
    unsigned long long t0 = 0;
    if (limit_ns == 0) return false;
    for (int it = 0;; it++) {
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (done) return true;
        if (it == 0) t0 = global_ns();
        else if (global_ns() - t0 > limit_ns) return false;
    }
}

// A tyre node on no wheel is a patch of its own: a wheel of one node with no hubs (axle0 -1), which gives the same bits
// (its sums are its own need and cap).
struct WheelDev {
    const int4* wheel;       // axle0, axle1 (global nodes; -1: a lone tyre node's), first of its nodes in wnodes, count
    const int* wnodes;       // the wheels' tyre nodes, each wheel's ascending
    const int* wlist;        // ... each wheel's in the builder's order (the turn's parity, the speed's sum)
    const int* wc_ptr;       // per node + 1: its wheel terms in wc, in wheel order
    const int2* wc;          // (wheel, kind | parity << 2): kind 0 the wheel's turn, 1 its arm (- the reaction), 2 its
                             // near axle node (+ the reaction)
    float4* tcon;            // per node: its static contact this substep (normal xyz, depth w), left for k_tyres
    float4* tfric;           // per node: (friction coefficient, surface, -, 1 while it waits for k_tyres)
    float4* wst;             // per wheel: Wheel::speed, avg_speed, last_torque, last_retorque
    const float4* wctl;      // per wheel: the controller's torque and brake, radius, mass
    const int4* warm;        // per wheel: arm, near_attach (global; -1 none), propulsed
    float4* wcf;             // per wheel: this substep's reaction on the arm (xyz; w 1 where it acts)
    float* wper;             // per wheel: this substep's torque share a tyre node (torque / nodes)
    int nreal;               // the builders' wheels (the lone tyre nodes' come after)
    float tyre_grip;         // WorldSettings::tyre_grip
};

// SoftBody::compute_wheel_forces (softbody.cpp:691-767) a warp a wheel, on the substep's starting state: the
// controller's torque (every substep: the first short step's), the brake's stop torque against the average speed and
// the last reaction, the share a tyre node, the tread's speed (summed in the builder's order), the average speed and
// the reaction of the inertia, and the drive's reaction on the arm; the nodes' terms are k_force's.
__device__ void wheel_step(int w, int lane, const float4* __restrict__ nd, const int4* __restrict__ info, const Body* __restrict__ bodies,
                           const WheelDev& wh, float dt) {
    const int4 W = wh.wheel[w];
    if (W.w == 0 || bodies[info[W.x].w].sleeping) return; // (an asleep body's forces are not made)
    const float4 ctl = wh.wctl[w], st = wh.wst[w];
    const int4 A = wh.warm[w];
    float T = ctl.x;
    if (ctl.y > 0) {
        const float stop = -st.y * ctl.z * ctl.w / dt - st.w;
        T += st.x > 0 ? clampf(stop, -ctl.y, 0.0f) : clampf(stop, 0.0f, ctl.y);
    }
    const float4 H0 = nd[2 * W.x], H1 = nd[2 * W.y], U0 = nd[2 * W.x + 1], U1 = nd[2 * W.y + 1];
    const v3 axis = normalize(V(H1.x - H0.x, H1.y - H0.y, H1.z - H0.z));
    const float per = T / (float)W.w;
    float expected = st.x, speed = 0.0f;
    // (a lane a node: each node's term, then the sum in the builder's order by broadcasts)
    for (int c = 0; c < W.w; c += 32) {
        const int j = c + lane;
        float term = 0.0f;
        bool has = false;
        if (j < W.w) {
            const int ni = wh.wlist[W.z + j];
            const float4 hp = (j & 1) ? H1 : H0, hv = (j & 1) ? U1 : U0, P = nd[2 * ni], Vn = nd[2 * ni + 1];
            v3 rad = V(P.x - hp.x, P.y - hp.y, P.z - hp.z);
            const float rl2 = dot(rad, rad);
            if (!(rl2 < 1e-8f)) {
                const float inv = 1.0f / sqrtf(rl2);
                if (A.z == 2) rad = V(-rad.x, -rad.y, -rad.z);
                const v3 dir = V(axis.y * rad.z - axis.z * rad.y, axis.z * rad.x - axis.x * rad.z, axis.x * rad.y - axis.y * rad.x) * inv;
                term = dot(V(Vn.x - hv.x, Vn.y - hv.y, Vn.z - hv.z), dir), has = true;
            }
        }
        for (unsigned m = __ballot_sync(0xffffffffu, has); m; m &= m - 1) speed += __shfl_sync(0xffffffffu, term, __ffs(m) - 1);
    }
    if (lane != 0) return;
    wh.wper[w] = per;
    const float sp = speed / (float)W.w, avg = 0.99f * st.y + 0.1f * sp;
    float lrt = st.w;
    if (ctl.w > 0 && ctl.z > 0) {
        expected += (st.z / ctl.z) / ctl.w * dt;
        lrt = ctl.w * (sp - expected) / dt;
    }
    float4 cf4 = make_float4(0, 0, 0, 0);
    if (A.x >= 0 && A.y >= 0 && fabsf(T) > 0.01f) {
        const float4 Pa = nd[2 * A.x], Pn = nd[2 * A.y];
        const v3 rr = V(Pa.x - Pn.x, Pa.y - Pn.y, Pa.z - Pn.z);
        v3 r = rr - axis * dot(rr, axis);
        const float off = length(rr - r), rl = length(r);
        if (rl > 0.01f && 2 * off < rl) {
            r = divs(r, rl);
            const v3 cf = V(axis.y * r.z - axis.z * r.y, axis.z * r.x - axis.x * r.z, axis.x * r.y - axis.y * r.x) * (0.5f * T / rl) * (1.0f - 2.0f * off / rl);
            cf4 = make_float4(cf.x, cf.y, cf.z, 1.0f);
        }
    }
    wh.wcf[w] = cf4;
    wh.wst[w] = make_float4(sp, avg, T, lrt);
}
__global__ void __launch_bounds__(256) k_wheels(const float4* __restrict__ nd, const int4* __restrict__ info, const Body* __restrict__ bodies,
                                                WheelDev wh, float dt) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w < wh.nreal) wheel_step(w, threadIdx.x & 31, nd, info, bodies, wh, dt); // (w is the warp's: its lanes go together)
}

// k_beams with the beam arrays staged by bulk copies: a persistent block takes every gridDim.x-th tile of kBeamTile
// beams; kBeamStages tiles are in flight while it computes (one thread issues the copies: each tile's a/b ends, k/d,
// state and meta words, 18 KB). The beam arrays are padded to whole tiles (pads asleep). Per beam the same
// beam_step as k_beams. kEnds16: each beam's ends as two 16-bit offsets from its tile's base node (tbase) in one
// 32-bit word - 4 of the 40 bytes a beam reads - for rigs whose every tile spans fewer than 65,536 nodes (16 KB a tile).
constexpr int kBeamTile = 512;
constexpr int kBeamStages = 3;
constexpr int kBeamThreads = 256;
template <bool kEnds16>
struct BeamStage {
    int2 ab[kBeamTile];
    float2 kd[kBeamTile];
    float4 bst[kBeamTile];
    uint32_t meta[kBeamTile];
};
template <>
struct BeamStage<true> {
    uint32_t ab[kBeamTile];
    float2 kd[kBeamTile];
    float4 bst[kBeamTile];
    uint32_t meta[kBeamTile];
};
template <bool kEnds16>
constexpr size_t beam_smem() { return kBeamStages * sizeof(BeamStage<kEnds16>) + kBeamStages * sizeof(uint64_t); }

template <bool kEnds16>
__global__ void __launch_bounds__(kBeamThreads) k_beams_tma(const void* __restrict__ ab_, const int* __restrict__ tbase, const float2* __restrict__ kd,
                                                            float4* __restrict__ bst, uint32_t* __restrict__ bmeta, const float4* __restrict__ bcold,
                                                            float* __restrict__ stress, const int* __restrict__ bbody, float* __restrict__ fsc,
                                                            const float4* __restrict__ nd, Body* __restrict__ bodies, int nbeams, int nbodies, int ntiles,
                                                            uint32_t* __restrict__ deverr, const int4* __restrict__ info, WheelDev wh, float dt,
                                                            unsigned long long wait_ns) {
    using Stage = BeamStage<kEnds16>;
    using AbT = typename std::remove_reference<decltype(Stage::ab[0])>::type;
    const AbT* ab = static_cast<const AbT*>(ab_);
    extern __shared__ __align__(128) unsigned char smem[];
    Stage* stg = reinterpret_cast<Stage*>(smem);
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kBeamStages * sizeof(Stage));
    const int tid = threadIdx.x;
    for (int t = blockIdx.x * kBeamThreads + tid; t < nbodies; t += gridDim.x * kBeamThreads) {
        Body& B = bodies[t]; // (this substep's bounds accumulator, for k_integrate)
        B.acc_mn[0] = B.acc_mn[1] = B.acc_mn[2] = 1e30f;
        B.acc_mx[0] = B.acc_mx[1] = B.acc_mx[2] = -1e30f;
    }
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    if (tid == 0) {
        for (int s = 0; s < kBeamStages; s++) mbar_init(&full[s], 1);
        mbar_init_fence();
    }
    __syncthreads();
    auto issue = [&](int i) { // this block's i-th tile into stage i % kBeamStages
        const int s = i % kBeamStages;
        const size_t j0 = (size_t)(blockIdx.x + (size_t)i * gridDim.x) * kBeamTile;
        mbar_expect_tx(&full[s], (uint32_t)(sizeof(Stage)));
        bulk_g2s(stg[s].ab, ab + j0, sizeof(stg[s].ab), &full[s]);
        bulk_g2s(stg[s].kd, kd + j0, sizeof(stg[s].kd), &full[s]);
        bulk_g2s(stg[s].bst, bst + j0, sizeof(stg[s].bst), &full[s]);
        bulk_g2s(stg[s].meta, bmeta + j0, sizeof(stg[s].meta), &full[s]);
    };
    if (tid == 0)
        for (int i = 0; i < kBeamStages && i < mine; i++) issue(i);
    int issued = min(kBeamStages, mine);
    int base_next = kEnds16 && mine > 0 ? tbase[blockIdx.x] : 0; // (each tile's base node loaded a tile ahead)
    for (int i = 0; i < mine; i++) {
        const int s = i % kBeamStages;
        const int base = base_next;
        if (kEnds16 && i + 1 < mine) base_next = tbase[blockIdx.x + (i + 1) * gridDim.x];
        const bool late = !mbar_wait(&full[s], (uint32_t)(i / kBeamStages) & 1u, wait_ns);
        if (__syncthreads_or(late)) {
            // a copy did not land in time: flag it, let the copies in flight land (bounded), stop
            if (tid == 0) {
                atomicOr(deverr, DEVERR_TIMEOUT);
                for (int k = i; k < issued; k++) mbar_wait(&full[k % kBeamStages], (uint32_t)(k / kBeamStages) & 1u);
            }
            __syncthreads();
            return;
        }
        const Stage& S = stg[s];
        const int jt = (blockIdx.x + i * gridDim.x) * kBeamTile;
        const int q0 = tid, q1 = tid + kBeamThreads;
        const int j0 = jt + q0, j1 = jt + q1;
        const bool h0 = j0 < nbeams, h1 = j1 < nbeams;
        const uint32_t m0 = S.meta[q0], m1 = S.meta[q1];
        int2 e0, e1;
        if constexpr (kEnds16) {
            const uint32_t w0 = S.ab[q0], w1 = S.ab[q1];
            e0 = make_int2(base + (int)(w0 & 0xffffu), base + (int)(w0 >> 16)), e1 = make_int2(base + (int)(w1 & 0xffffu), base + (int)(w1 >> 16));
        } else {
            e0 = S.ab[q0], e1 = S.ab[q1];
        }
        float4 pa0 = make_float4(0, 0, 0, 0), va0 = pa0, pb0 = pa0, vb0 = pa0, pa1 = pa0, va1 = pa0, pb1 = pa0, vb1 = pa0;
        const bool g0 = h0 && !(m0 & kBeamAsleep), g1 = h1 && !(m1 & kBeamAsleep);
        if (g0) pa0 = nd[2 * e0.x], va0 = nd[2 * e0.x + 1], pb0 = nd[2 * e0.y], vb0 = nd[2 * e0.y + 1];
        if (g1) pa1 = nd[2 * e1.x], va1 = nd[2 * e1.x + 1], pb1 = nd[2 * e1.y], vb1 = nd[2 * e1.y + 1];
        if (h0) beam_step(j0, m0, S.bst[q0], S.kd[q0], pa0, va0, pb0, vb0, bst, bmeta, bcold, stress, bbody, fsc, bodies);
        if (h1) beam_step(j1, m1, S.bst[q1], S.kd[q1], pa1, va1, pb1, vb1, bst, bmeta, bcold, stress, bbody, fsc, bodies);
        __syncthreads(); // (every thread is done with stage s)
        if (tid == 0 && issued < mine) {
            fence_proxy_async();
            issue(issued);
        }
        issued = min(issued + 1, mine);
    }
    // then the wheels (k_wheels' work, a warp a wheel: it reads the substep's starting state as the beams do, and only
    // k_force reads what it writes)
    for (int w = blockIdx.x * (kBeamThreads / 32) + (tid >> 5); w < wh.nreal; w += gridDim.x * (kBeamThreads / 32))
        wheel_step(w, tid & 31, nd, info, bodies, wh, dt);
}

// The frame bodies' gather (NodeFem): their nodes' forces go to the frame's implicit step
struct NodeFem {
    const int* fslot;        // node -> frame node (-1: none)
    const int* iperm;        // frame node -> column
    const int* gdiag_ptr;    // column -> its triangles' corners
    const int2* gdiag;
    const uint8_t* ton;
    const float4* tf;
    const float4* tt;
    float4* torque;
    float4* nforce;
    const float4* ext;       // constant node forces (bl_gpu_set_node_force)
    const uint8_t* mon;      // the members' forces of the substep (k_member_eval)
    const float4* mfa;
    const float4* mta;
    const float4* mtb;
};

// the bounds, top speed and static contacts of a warp's nodes into their bodies' accumulators (a warp of one body
// reduces first)
__device__ __forceinline__ void accumulate_bounds(Body* __restrict__ bodies, int body, bool live, v3 p, v3 pmx, float v2, int contact) {
    const int lane = threadIdx.x & 31;
    const int b0 = __shfl_sync(0xffffffffu, body, 0);
    // (one body's warp: reduced, its lanes that are not live - asleep, a frame's, a tyre node its wheel integrates -
    // adding nothing)
    const bool uniform = __all_sync(0xffffffffu, body == b0) && __any_sync(0xffffffffu, live);
    if (!live) p = V(1e30f, 1e30f, 1e30f), pmx = V(-1e30f, -1e30f, -1e30f), v2 = 0.0f, contact = 0;
    if (uniform) {
        float mnx = p.x, mny = p.y, mnz = p.z, mxx = pmx.x, mxy = pmx.y, mxz = pmx.z, vv = v2;
        int cc = contact;
        for (int o = 16; o > 0; o >>= 1) {
            mnx = fminf(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
            mny = fminf(mny, __shfl_xor_sync(0xffffffffu, mny, o));
            mnz = fminf(mnz, __shfl_xor_sync(0xffffffffu, mnz, o));
            mxx = fmaxf(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
            mxy = fmaxf(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
            mxz = fmaxf(mxz, __shfl_xor_sync(0xffffffffu, mxz, o));
            vv = fmaxf(vv, __shfl_xor_sync(0xffffffffu, vv, o));
            cc += __shfl_xor_sync(0xffffffffu, cc, o);
        }
        if (lane == 0) {
            Body& B = bodies[b0];
            atomic_min_f(&B.acc_mn[0], mnx), atomic_min_f(&B.acc_mn[1], mny), atomic_min_f(&B.acc_mn[2], mnz);
            atomic_max_f(&B.acc_mx[0], mxx), atomic_max_f(&B.acc_mx[1], mxy), atomic_max_f(&B.acc_mx[2], mxz);
            atomic_max_f(&B.acc_v2, vv);
            if (cc) atomicAdd(&B.acc_contacts, cc);
        }
    } else if (live) {
        Body& B = bodies[body];
        atomic_min_f(&B.acc_mn[0], p.x), atomic_min_f(&B.acc_mn[1], p.y), atomic_min_f(&B.acc_mn[2], p.z);
        atomic_max_f(&B.acc_mx[0], pmx.x), atomic_max_f(&B.acc_mx[1], pmx.y), atomic_max_f(&B.acc_mx[2], pmx.z);
        atomic_max_f(&B.acc_v2, v2);
        if (contact) atomicAdd(&B.acc_contacts, contact);
    }
}

// A frame node's force: its triangles' corner forces and torques added in the reference's order (gather_forces,
// frame_fem.cpp:2080-2105) after gravity and its beams; kept in nforce for the frame's implicit step.
__device__ __forceinline__ void fem_gather(const NodeFem& nf, int i, v3 f) {
    const int fs = nf.fslot[i];
    if (fs >= 0) {
        const int k = nf.iperm[fs];
        v3 tq = V(0, 0, 0);
        for (int g = nf.gdiag_ptr[k]; g < nf.gdiag_ptr[k + 1]; g++) {
            const int2 e = nf.gdiag[g];
            if (e.x < 0) { // (a member's end a (+fa, ta) or b (-fa, tb): gather_forces, frame_fem.cpp:2092-2096)
                const int ei = -e.x - 1;
                if (!nf.mon[ei]) continue;
                const float4 fa = nf.mfa[ei], tq4 = e.y == 0 ? nf.mta[ei] : nf.mtb[ei];
                if (e.y == 0) f = V(f.x + fa.x, f.y + fa.y, f.z + fa.z);
                else f = V(f.x - fa.x, f.y - fa.y, f.z - fa.z);
                tq = V(tq.x + tq4.x, tq.y + tq4.y, tq.z + tq4.z);
                continue;
            }
            if (!nf.ton[e.x]) continue;
            const float4 tf = nf.tf[3 * e.x + e.y], tt = nf.tt[3 * e.x + e.y];
            f = V(f.x + tf.x, f.y + tf.y, f.z + tf.z);
            tq = V(tq.x + tt.x, tq.y + tt.y, tq.z + tt.z);
        }
        nf.torque[fs] = make_float4(tq.x, tq.y, tq.z, 0.0f);
    }
    nf.nforce[i] = make_float4(f.x, f.y, f.z, 0.0f);
}

// A node's force: clear_forces' gravity (and any constant node force), then its beams in beam order
// (softbody.cpp:376, 466-467); each beam's force made again from the beam's scalar and the two positions, as k_beams
// made it. ell: the nodes' incidences (beam | bit 31 when the node is the beam's b end, the other end). Into fnode
// for World::collide_static and the integration (k_integrate) - the contacts between bodies add to it first.
// Frame bodies (Body::is_fem): the triangles' forces and torques are gathered onto the frame nodes in the reference's
// order (gather_forces, frame_fem.cpp:2080-2105) and the force is kept in nforce for the frame's implicit step.
// ------------------------------------------------------------------------------------------ air drag
// The parts of the bodies with air drag and their mean velocities (SoftBody::part_labels, softbody.cpp:237-259, and
// clear_forces' sums, softbody.cpp:334-378), one thread a body, serially in node order as the reference sums: every
// substep the labels age; they are made again (union of the unbroken beams, parts numbered by their first node) at the
// first call and when beams broke since and they are 8 calls old. Then per part the mass-weighted mean velocity
// (pmv) and the aerodynamic acceleration (pacc), at node0 + part.
struct DragDev {
    int* up;                 // per node: union-find scratch
    int* pid;                // per node: a root's part number (scratch)
    int* part;               // per node: its part
    float4* pmv;             // per part (at node0 + part): mean velocity; w: the part's mass while summing
    float4* pacc;            // per part: the aerodynamic acceleration
};
__global__ void k_drag_parts(Body* __restrict__ bodies, int nbodies, const float4* __restrict__ nd, const int2* __restrict__ ab,
                             const uint32_t* __restrict__ bmeta, DragDev D) {
    const int bi = blockIdx.x * blockDim.x + threadIdx.x;
    if (bi >= nbodies) return;
    Body& B = bodies[bi];
    if (!B.drag || B.sleeping) return;
    const int n0 = B.node0, nn = B.nnodes;
    B.part_age += 1;
    if (B.part_count == 0 || (B.broken_beams != B.part_key && B.part_age >= 8)) {
        int* u = D.up + n0;
        for (int i = 0; i < nn; i++) u[i] = i;
        auto find = [&](int x) {
            while (u[x] != x) x = u[x] = u[u[x]];
            return x;
        };
        for (int j = B.beam0; j < B.beam0 + B.nbeams; j++) {
            if ((bmeta[j] >> 8) & BF_BROKEN) continue;
            const int2 e = ab[j];
            const int rc = find(e.y - n0);
            u[find(e.x - n0)] = rc;
        }
        int* id = D.pid + n0;
        for (int i = 0; i < nn; i++) u[i] = find(i), id[i] = -1;
        int cnt = 0;
        for (int i = 0; i < nn; i++) {
            if (id[u[i]] < 0) id[u[i]] = cnt++;
            D.part[n0 + i] = id[u[i]];
        }
        B.part_count = cnt, B.part_key = B.broken_beams, B.part_age = 0;
    }
    const int np = B.part_count;
    for (int q = 0; q < np; q++) D.pmv[n0 + q] = make_float4(0, 0, 0, 0);
    float M = 0;
    for (int i = 0; i < nn; i++) {
        const float4 v = nd[2 * (n0 + i) + 1];
        float4& pv = D.pmv[n0 + D.part[n0 + i]];
        pv.x = pv.x + v.x * v.w, pv.y = pv.y + v.y * v.w, pv.z = pv.z + v.z * v.w;
        pv.w = pv.w + v.w;
        M = M + v.w;
    }
    for (int q = 0; q < np; q++) {
        const float4 pv = D.pmv[n0 + q];
        const v3 mv = pv.w > 0 ? divs(V(pv.x, pv.y, pv.z), pv.w) : V(0, 0, 0);
        const v3 a = M > 0 ? mv * (-0.5f * 1.225f * B.aero_cda * length(mv) / M) : V(0, 0, 0);
        D.pmv[n0 + q] = make_float4(mv.x, mv.y, mv.z, 0.0f);
        D.pacc[n0 + q] = make_float4(a.x, a.y, a.z, 0.0f);
    }
}

// ------------------------------------------------------------------------------------------ wheels and tyres
// The wheels of node tyres (Wheel, softbody.h:468-498), free rolling: per wheel its hub nodes and its tyre nodes in
// ascending order (the order the tyre patch's sums run in, world.cpp:871-898); per node its wheel and the parity of
// its place in the wheel's list (the hub it turns about); per node the substep's tyre contact.
// kPacked: the incidences as 32-bit words: the beam's index less the warp's base (ell_base, bits 0-14; 0x7fff:
// padding), bit 15 set where this node is the beam's b end, the other end's index less this node's plus 32768 (bits
// 16-31) - half the bytes of the (beam | b-end bit, other end) pairs, for rigs whose warps' beams and neighbours lie
// close enough (bl_world.cu checks every warp)
template <bool kPacked>
__global__ void __launch_bounds__(256, 6) k_force(const float4* __restrict__ nd, const int4* __restrict__ info, const int* __restrict__ ell_ptr,
                                               const void* __restrict__ ell_, const int* __restrict__ ell_base, const float* __restrict__ fsc,
                                               Body* __restrict__ bodies, float gx, float gy, float gz, int nnodes, int first, NodeFem nf,
                                               float4* __restrict__ fnode, DragDev dg, WheelDev wh, ShockDev sk) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int body = -1;
    float v2 = 0.0f;
    bool live = false;
    if (i < nnodes) {
        // (the node's own loads and its warp's incidence range issued before its body's state arrives)
        const int4 inf = info[i];
        const float4 P = nd[2 * i], Vv = nd[2 * i + 1];
        const int w = i >> 5, lane = i & 31;
        const int q0 = ell_ptr[w], width = (ell_ptr[w + 1] - q0) >> 5;
        const int base = kPacked ? ell_base[w] : 0;
        body = inf.w;
        const Body& B = bodies[body];
        if (!B.sleeping) {
            const float m = Vv.w;
            v3 f;
            if (!B.drag) {
                f = V(gx * m, gy * m, gz * m);
            } else { // (clear_forces with drag: (g + the part's aerodynamic acceleration) m, less RoR's drag on v - its mean)
                const int q = B.node0 + dg.part[i];
                const float4 a = dg.pacc[q];
                f = V((gx + a.x) * m, (gy + a.y) * m, (gz + a.z) * m);
                if (!((uint32_t)inf.x & (NF_TYRE | NF_RIM))) {
                    const float4 mv = dg.pmv[q];
                    const v3 vr = V(Vv.x - mv.x, Vv.y - mv.y, Vv.z - mv.z);
                    f = f - vr * (B.air_drag * length(vr));
                }
            }
            if (B.has_ext) {
                const float4 e = nf.ext[i];
                f = V(f.x + e.x, f.y + e.y, f.z + e.z);
            }
            // (four incidences' loads issued together, then added in order: the gathers overlap)
            auto add = [&](bool pad, bool bend, float sc, float4 Po) {
                if (__float_as_uint(sc) == __float_as_uint(kNoPush) || pad) return;
                if (bend) { // (this node is the beam's b: dis = p_a - p_b, the force subtracted)
                    const v3 dis = V(Po.x - P.x, Po.y - P.y, Po.z - P.z);
                    f = V(f.x - dis.x * sc, f.y - dis.y * sc, f.z - dis.z * sc);
                } else {
                    const v3 dis = V(P.x - Po.x, P.y - Po.y, P.z - Po.z);
                    f = V(f.x + dis.x * sc, f.y + dis.y * sc, f.z + dis.z * sc);
                }
            };
            // the warp's incidences, interleaved: entry q of lane l at ell[ell_ptr[w] + 32 q + l] (a warp's load reads 32
            // neighbours), each node's in beam order, padded to the warp's widest node (a multiple of 4)
            for (int q = 0; q < width; q += 4) {
                int beam[4], other[4];
                bool pad[4], bend[4];
                float sc[4];
                float4 Po[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    if (kPacked) {
                        const uint32_t x = static_cast<const uint32_t*>(ell_)[q0 + 32 * (q + u) + lane];
                        pad[u] = (x & 0x7fffu) == 0x7fffu;
                        beam[u] = base + (int)(x & 0x7fffu), bend[u] = (x & 0x8000u) != 0, other[u] = i + (int)(x >> 16) - 32768;
                    } else {
                        const int2 e = static_cast<const int2*>(ell_)[q0 + 32 * (q + u) + lane];
                        pad[u] = e.y == i; // (padding: (0, the node itself))
                        beam[u] = e.x & 0x7fffffff, bend[u] = e.x < 0, other[u] = e.y;
                    }
                }
#pragma unroll
                for (int u = 0; u < 4; u++) sc[u] = pad[u] ? kNoPush : fsc[beam[u]], Po[u] = nd[2 * other[u]];
#pragma unroll
                for (int u = 0; u < 4; u++) add(pad[u], bend[u], sc[u], Po[u]);
            }
            if (B.has_shocks) // (compute_shock_forces after the beams: the node's shocks in their order)
                for (int q = sk.ptr[i]; q < sk.ptr[i + 1]; q++) {
                    const int2 e = sk.inc[q];
                    add(false, e.x < 0, sk.ssc[e.x & 0x7fffffff], nd[2 * e.y]);
                }
            if (B.has_wheels) // (compute_wheel_forces, softbody.cpp:691-767: the wheels' terms on this node in their order)
                for (int q = wh.wc_ptr[i]; q < wh.wc_ptr[i + 1]; q++) {
                    const int2 e = wh.wc[q];
                    if ((e.y & 3) == 0) { // (a tyre node: its share of the torque along its tangent)
                        const int4 W = wh.wheel[e.x];
                        const float4 H0 = nd[2 * W.x], H1 = nd[2 * W.y];
                        const v3 axis = normalize(V(H1.x - H0.x, H1.y - H0.y, H1.z - H0.z));
                        const float4 hub = (e.y >> 2) ? H1 : H0;
                        v3 rad = V(P.x - hub.x, P.y - hub.y, P.z - hub.z);
                        const float rl2 = dot(rad, rad);
                        if (!(rl2 < 1e-8f)) {
                            const float inv = 1.0f / sqrtf(rl2);
                            if (wh.warm[e.x].z == 2) rad = V(-rad.x, -rad.y, -rad.z);
                            const v3 dir = V(axis.y * rad.z - axis.z * rad.y, axis.z * rad.x - axis.x * rad.z, axis.x * rad.y - axis.y * rad.x) * inv;
                            f = f + dir * (wh.wper[e.x] * inv);
                        }
                    } else { // (the arm, the near axle node: the drive's reaction)
                        const float4 cf = wh.wcf[e.x];
                        if (cf.w != 0.0f) f = (e.y & 3) == 1 ? f - V(cf.x, cf.y, cf.z) : f + V(cf.x, cf.y, cf.z);
                    }
                }
            if (B.is_fem) {
                live = true; // (its bounds and speeds after the frame's step: k_fem_integrate; the start's top speed here)
                if (first) v2 = Vv.x * Vv.x + Vv.y * Vv.y + Vv.z * Vv.z;
                fem_gather(nf, i, f);
            } else {
                fnode[i] = make_float4(f.x, f.y, f.z, 0.0f);
            }
        }
    }
    accumulate_bounds(bodies, body, live, V(1e30f, 1e30f, 1e30f), V(-1e30f, -1e30f, -1e30f), v2, 0);
}

// tyre_contact (static_world.cpp:53-83)
struct TyreC {
    v3 normal_force, need, slide;
    float cap;
    bool touching;
};
__device__ TyreC tyre_contact(v3 F, v3 vel, float mass, v3 normal, float dt, const GroundModel& gm, float pen, float friction_coef) {
    TyreC t;
    t.normal_force = V(0, 0, 0), t.need = V(0, 0, 0), t.slide = V(0, 0, 0), t.cap = 0.0f, t.touching = false;
    const float Vn = dot(vel, normal);
    const float Fn = dot(F, normal);
    const float sgl = gm.soft_depth;
    if (sgl > 0 && pen >= 0) {
        t.normal_force = t.normal_force + vel * (-gm.fluid_drag * smin(1.0f, pen / sgl + 0.2f));
        float Fb = gm.fluid_density * smin(pen, sgl) * 9.807f * 0.02f;
        if (Vn >= 0 && Fn < 0 && Fb > -Fn) Fb = -Fn;
        t.normal_force = t.normal_force + normal * Fb;
    }
    if (pen < sgl) return t;
    float R = -Fn;
    if (Vn < 0) R -= (0.8f * Vn - smin(0.2f * (pen - sgl) / dt, 2.0f)) * mass / dt;
    if (R <= 0) return t;
    t.touching = true;
    t.normal_force = t.normal_force + normal * R;
    const v3 slipF = F - normal * Fn;
    const v3 slipV = vel - normal * Vn;
    const float G = R * gm.strength * friction_coef;
    t.need = V(-slipF.x, -slipF.y, -slipF.z) - slipV * (0.5f * mass / dt);
    t.cap = gm.ms * G;
    const float sv = length(slipV);
    const float mu_slide = smax(gm.mc, 0.85f * gm.ms);
    const float g = mu_slide + (gm.ms - mu_slide) * bl_expf(-bl_powf(sv / gm.vs, gm.alpha)) + smin(gm.t2 * sv, 5.0f);
    const float nl = length(t.need);
    const v3 dir = sv > 0.05f ? slipV * (-1.0f / sv) : (nl > 1e-6f ? t.need * (1.0f / nl) : V(0, 0, 0));
    t.slide = dir * (g * G);
    return t;
}

// SoftBody::integrate_nodes for one node (softbody.cpp:769-795): v += f inv_m dt, the 400 m/s clamp, NaN reset,
// p += v dt; v2: its squared speed after
__device__ __forceinline__ void integrate_node(v3& pos, v3& vel, float inv_mass, v3 f, float dt, float& v2) {
    if (inv_mass > 0) {
        vel = vel + f * (inv_mass * dt);
        v2 = dot(vel, vel);
        if (v2 > kMaxNodeSpeed * kMaxNodeSpeed) {
            vel = vel * (kMaxNodeSpeed / sqrtf(v2));
            v2 = kMaxNodeSpeed * kMaxNodeSpeed;
        } else if (!(v2 >= 0.0f)) {
            vel = V(0, 0, 0);
            v2 = 0;
        }
        pos = pos + vel * dt;
    }
}

// World::collide_static's query for one node (world.cpp:804-832): the terrain if the node is within its reach, the
// body's candidate boxes and cylinders within reach of the node (all of them past 16 of either), StaticWorld::
// collide_point's deepest contact
__device__ __forceinline__ bool static_query(const Statics& st, const Body& B, v3 pos, float r, Contact& c) {
    const bool near_terrain = st.has_terrain && pos.y - r <= B.terrain_max + 0.05f;
    const int nbox = B.nbox, ncyl = B.ncyl;
    if (!near_terrain && nbox == 0 && ncyl == 0) return false;
    int bids[16], cids[16];
    const int* bp = B.box_ids;
    const int* cp = B.cyl_ids;
    int nb = nbox, nc = ncyl;
    if (nbox <= 16 && ncyl <= 16) {
        nb = nc = 0;
        const float rr = r + 0.01f;
        for (int k = 0; k < nbox; k++) {
            const Box& a = st.boxes[B.box_ids[k]];
            if (pos.x >= a.mnx - rr && pos.x <= a.mxx + rr && pos.y >= a.mny - rr && pos.y <= a.mxy + rr && pos.z >= a.mnz - rr && pos.z <= a.mxz + rr)
                bids[nb++] = B.box_ids[k];
        }
        for (int k = 0; k < ncyl; k++) {
            const Cyl& cy = st.cyls[B.cyl_ids[k]];
            const float cr = cy.radius + rr;
            if (fabsf(pos.x - cy.bx) <= cr && fabsf(pos.z - cy.bz) <= cr && pos.y >= cy.by - rr && pos.y <= cy.by + cy.height + rr)
                cids[nc++] = B.cyl_ids[k];
        }
        bp = bids;
        cp = cids;
        if (!near_terrain && nb == 0 && nc == 0) return false;
    }
    return collide_point(st, pos, r, bp, nb, cp, nc, near_terrain, c);
}

// World::collide_static for the node (world.cpp:781-870), then SoftBody::integrate_nodes (softbody.cpp:769-795), on
// the force in fnode (gravity, beams, contacts with other bodies). first: the frame's first substep (the top speed
// starts from the velocities before it, world.cpp:3217-3222). Frame bodies' nodes are integrated after their solve.
// A tyre node (NF_TYRE) in contact leaves its contact in wh.tcon / wh.tfric and its force in fnode to its wheel's
// patch (k_tyres), which takes tyre_contact instead of primitive_collision and integrates it.
__global__ void __launch_bounds__(256) k_integrate(float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies, Statics st,
                                                   float dt, int nnodes, int first, float4* __restrict__ fnode, WheelDev wh) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    int body = -1;
    v3 p = V(1e30f, 1e30f, 1e30f), pmx = V(-1e30f, -1e30f, -1e30f);
    float v2 = 0.0f, v2start = 0.0f;
    int contact = 0;
    bool live = false;
    if (i < nnodes) {
        // (the node's own loads issued before its body's state arrives)
        const int4 inf = info[i];
        const float4 P = nd[2 * i], Vv = nd[2 * i + 1], f4 = fnode[i];
        body = inf.w;
        const Body& B = bodies[body];
        if (!B.sleeping && !B.is_fem) {
            live = true;
            const float m = Vv.w;
            v3 f = V(f4.x, f4.y, f4.z);
            if (first) v2start = Vv.x * Vv.x + Vv.y * Vv.y + Vv.z * Vv.z;
            v3 pos = V(P.x, P.y, P.z), vel = V(Vv.x, Vv.y, Vv.z);
            float inv_mass = P.w;
            const uint32_t flags = (uint32_t)inf.x;
            // ---- static contact (World::collide_static)
            if (!(!(flags & NF_GROUND) || inv_mass <= 0)) {
                if (pos.y < st.kill_y) {
                    vel = V(0, 0, 0);
                    inv_mass = 0;
                } else {
                    {
                        Contact c;
                        if (static_query(st, B, pos, __int_as_float(inf.z), c)) {
                            contact = 1;
                            const GroundModel& gm = c_ground[c.surface < kSurfCount ? c.surface : 0];
                            const float fc = __int_as_float(inf.y) * B.fric;
                            if (c.max_force > 0) {
                                v3 fcn = primitive_collision(f, vel, m, c.normal, dt, gm, c.depth, fc, B.push_max, B.slop, -1.0f);
                                const float fl = length(fcn);
                                if (fl > c.max_force) fcn = fcn * (c.max_force / fl);
                                f = f + fcn;
                            } else if (flags & NF_TYRE) { // (its wheel's patch: k_tyres)
                                wh.tcon[i] = make_float4(c.normal.x, c.normal.y, c.normal.z, c.depth);
                                wh.tfric[i] = make_float4(fc * wh.tyre_grip, __int_as_float(c.surface), 0.0f, 1.0f);
                                live = false;
                            } else {
                                f = f + primitive_collision(f, vel, m, c.normal, dt, gm, c.depth, fc, B.push_max, B.slop, B.bounce);
                            }
                        }
                    }
                }
            }
            if (live) {
            // ---- integration (SoftBody::integrate_nodes)
            integrate_node(pos, vel, inv_mass, f, dt, v2);
            nd[2 * i] = make_float4(pos.x, pos.y, pos.z, inv_mass);
            nd[2 * i + 1] = make_float4(vel.x, vel.y, vel.z, m);
            // the bounds skip a non-finite coordinate as the reference's vmin / vmax do (a NaN never compares less)
            p = V(pos.x == pos.x ? pos.x : 1e30f, pos.y == pos.y ? pos.y : 1e30f, pos.z == pos.z ? pos.z : 1e30f);
            pmx = V(pos.x == pos.x ? pos.x : -1e30f, pos.y == pos.y ? pos.y : -1e30f, pos.z == pos.z ? pos.z : -1e30f);
            v2 = smax(v2, v2start);
            } else {
                contact = 0; // (counted with its wheel's patch)
            }
        }
    }
    accumulate_bounds(bodies, body, live, p, pmx, v2, contact);
}

// World::collide_static's tyre contacts and patches (world.cpp:856-898) and the integration of their nodes: a warp a
// wheel, a lane a tyre node (in chunks of 32) - each node in contact gets tyre_contact on its force and its normal
// force; the touching ones' needs and caps summed in ascending node order (every lane adds the same broadcast values
// in the same order); each touching node sticks (its need) if the patch as a whole can hold, else slides; then
// SoftBody::integrate_nodes for them, the warp's bounds, top speed and contacts into the body's accumulators.
__global__ void __launch_bounds__(256) k_tyres(float4* __restrict__ nd, const int4* __restrict__ info, Body* __restrict__ bodies, float dt,
                                               int nwheels, int first, const float4* __restrict__ fnode, WheelDev wh) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= nwheels) return; // (w is the warp's: its lanes leave together)
    const int4 W = wh.wheel[w];
    if (W.w == 0) return;
    const int body = info[wh.wnodes[W.z]].w;
    v3 need = V(0, 0, 0), mn = V(1e30f, 1e30f, 1e30f), mx = V(-1e30f, -1e30f, -1e30f);
    float cap = 0.0f, vv = 0.0f;
    int cnt = 0;
    // pass 1: the contacts and the patch's sums (one chunk's nodes kept in registers for pass 2)
    int i = -1;
    TyreC t = {};
    v3 f = V(0, 0, 0);
    float4 P = make_float4(0, 0, 0, 0), Vv = P;
    bool pend = false;
    for (int c = 0; c < W.w; c += 32) {
        pend = false;
        if (c + lane < W.w) {
            i = wh.wnodes[W.z + c + lane];
            const float4 tf = wh.tfric[i];
            pend = tf.w != 0.0f;
            if (pend) {
                const float4 cn = wh.tcon[i], f4 = fnode[i];
                P = nd[2 * i], Vv = nd[2 * i + 1];
                const int surf = __float_as_int(tf.y);
                const GroundModel& gm = c_ground[surf < kSurfCount ? surf : 0];
                f = V(f4.x, f4.y, f4.z);
                t = tyre_contact(f, V(Vv.x, Vv.y, Vv.z), Vv.w, V(cn.x, cn.y, cn.z), dt, gm, cn.w, tf.x);
                f = f + t.normal_force;
            }
        }
        const bool touch = pend && t.touching;
        for (unsigned m = __ballot_sync(0xffffffffu, touch); m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            need = V(need.x + __shfl_sync(0xffffffffu, t.need.x, l), need.y + __shfl_sync(0xffffffffu, t.need.y, l),
                     need.z + __shfl_sync(0xffffffffu, t.need.z, l));
            cap = cap + __shfl_sync(0xffffffffu, t.cap, l);
        }
    }
    const bool stick = length(need) <= cap;
    // pass 2: the forces applied and the nodes integrated (a wheel of more than 32 nodes: its contacts again)
    for (int c = 0; c < W.w; c += 32) {
        if (W.w > 32) {
            pend = false;
            if (c + lane < W.w) {
                i = wh.wnodes[W.z + c + lane];
                const float4 tf = wh.tfric[i];
                pend = tf.w != 0.0f;
                if (pend) {
                    const float4 cn = wh.tcon[i], f4 = fnode[i];
                P = nd[2 * i], Vv = nd[2 * i + 1];
                    const int surf = __float_as_int(tf.y);
                    const GroundModel& gm = c_ground[surf < kSurfCount ? surf : 0];
                    f = V(f4.x, f4.y, f4.z);
                    t = tyre_contact(f, V(Vv.x, Vv.y, Vv.z), Vv.w, V(cn.x, cn.y, cn.z), dt, gm, cn.w, tf.x);
                    f = f + t.normal_force;
                }
            }
        }
        if (!pend) continue;
        if (t.touching) f = f + (stick ? t.need : t.slide);
        wh.tfric[i].w = 0.0f;
        v3 pos = V(P.x, P.y, P.z), vel = V(Vv.x, Vv.y, Vv.z);
        float v2 = 0.0f;
        const float v2start = first ? Vv.x * Vv.x + Vv.y * Vv.y + Vv.z * Vv.z : 0.0f;
        integrate_node(pos, vel, P.w, f, dt, v2);
        nd[2 * i] = make_float4(pos.x, pos.y, pos.z, P.w);
        nd[2 * i + 1] = make_float4(vel.x, vel.y, vel.z, Vv.w);
        // (the bounds skip a non-finite coordinate as the reference's vmin / vmax do)
        mn = V(fminf(mn.x, pos.x == pos.x ? pos.x : 1e30f), fminf(mn.y, pos.y == pos.y ? pos.y : 1e30f), fminf(mn.z, pos.z == pos.z ? pos.z : 1e30f));
        mx = V(fmaxf(mx.x, pos.x == pos.x ? pos.x : -1e30f), fmaxf(mx.y, pos.y == pos.y ? pos.y : -1e30f), fmaxf(mx.z, pos.z == pos.z ? pos.z : -1e30f));
        vv = fmaxf(vv, smax(v2, v2start));
        cnt++;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = V(fminf(mn.x, __shfl_xor_sync(0xffffffffu, mn.x, o)), fminf(mn.y, __shfl_xor_sync(0xffffffffu, mn.y, o)),
               fminf(mn.z, __shfl_xor_sync(0xffffffffu, mn.z, o)));
        mx = V(fmaxf(mx.x, __shfl_xor_sync(0xffffffffu, mx.x, o)), fmaxf(mx.y, __shfl_xor_sync(0xffffffffu, mx.y, o)),
               fmaxf(mx.z, __shfl_xor_sync(0xffffffffu, mx.z, o)));
        vv = fmaxf(vv, __shfl_xor_sync(0xffffffffu, vv, o));
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    }
    if (lane == 0 && cnt > 0) {
        Body& B = bodies[body];
        atomic_min_f(&B.acc_mn[0], mn.x), atomic_min_f(&B.acc_mn[1], mn.y), atomic_min_f(&B.acc_mn[2], mn.z);
        atomic_max_f(&B.acc_mx[0], mx.x), atomic_max_f(&B.acc_mx[1], mx.y), atomic_max_f(&B.acc_mx[2], mx.z);
        atomic_max_f(&B.acc_v2, vv);
        atomicAdd(&B.acc_contacts, cnt);
    }
}

// World::collide_static for the frame bodies' nodes (world.cpp:781-870 on a body with a frame of members), before the
// frame's implicit step: a node's contact force into its force (nforce, the step's right side); a frame node pressed on
// records its ground contact's normal for the step (FemFrame::contact_n: doubled where it sticks - slower than 5 cm/s
// along the ground and its friction holding what pushes it along), which the assembly holds with kappa = 200 m
__global__ void k_fem_static(float4* __restrict__ nd, float4* __restrict__ nforce, const int* __restrict__ fem_nodes, int n_fem_nodes,
                             const int* __restrict__ fslot, const int4* __restrict__ info, Body* __restrict__ bodies, Statics st, float dt,
                             float4* __restrict__ contact_n) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_fem_nodes) return;
    const int i = fem_nodes[t];
    const int4 inf = info[i];
    Body& B = bodies[inf.w];
    const float4 P = nd[2 * i], Vv = nd[2 * i + 1];
    if (B.sleeping || !((uint32_t)inf.x & NF_GROUND) || P.w <= 0) return;
    const v3 pos = V(P.x, P.y, P.z), vel = V(Vv.x, Vv.y, Vv.z);
    if (pos.y < st.kill_y) { // (fell off the world)
        nd[2 * i] = make_float4(P.x, P.y, P.z, 0.0f);
        nd[2 * i + 1] = make_float4(0.0f, 0.0f, 0.0f, Vv.w);
        return;
    }
    Contact c;
    if (!static_query(st, B, pos, __int_as_float(inf.z), c)) return;
    atomicAdd(&B.acc_contacts, 1);
    const GroundModel& gm = c_ground[c.surface < kSurfCount ? c.surface : 0];
    const float fc = __int_as_float(inf.y) * B.fric;
    const float4 f4 = nforce[i];
    v3 F = V(f4.x, f4.y, f4.z);
    if (c.max_force > 0) {
        v3 fcn = primitive_collision(F, vel, Vv.w, c.normal, dt, gm, c.depth, fc, B.push_max, B.slop, -1.0f);
        const float fl = length(fcn);
        if (fl > c.max_force) fcn = fcn * (c.max_force / fl);
        F = F + fcn;
    } else {
        const v3 fo = primitive_collision(F, vel, Vv.w, c.normal, dt, gm, c.depth, fc, B.push_max, B.slop, B.bounce);
        F = F + fo;
        const int sl = fslot[i];
        if (sl >= 0) {
            const float fn = dot(fo, c.normal);
            const v3 ft = F - c.normal * dot(F, c.normal), vt = vel - c.normal * dot(vel, c.normal);
            if (fn > 0) {
                const v3 cn = c.normal * (dot(vt, vt) < 0.05f * 0.05f && length(ft) < 0.3f * fn ? 2.0f : 1.0f);
                contact_n[sl] = make_float4(cn.x, cn.y, cn.z, 0.0f);
            }
        }
    }
    nforce[i] = make_float4(F.x, F.y, F.z, f4.w);
}

// ------------------------------------------------------------------------------------------ end of frame
// Block-wide bitonic sort of v[0, P) ascending (P a power of two), in place in global memory.
__device__ void block_bitonic_sort(float* v, int P) {
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < P; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const float a = v[i], b = v[l];
                    const bool up = (i & k) == 0;
                    if (up ? (b < a) : (a < b)) v[i] = b, v[l] = a;
                }
            }
            __syncthreads();
        }
}

__device__ __forceinline__ bool finite3(float x, float y, float z) { return isfinite(x) && isfinite(y) && isfinite(z); }

// Scratch of k_frame_finish, sized for the largest body (P = its node count rounded up to a power of two).
struct RepairScratch {
    float* sort;      // 3 * P
    int* bad;         // P
    float4* np;       // P: new positions of the pass
    float4* nv;       // P: new velocities of the pass
    int P;
};

// World::repair_nodes (world.cpp:4022-4111) of one body by the whole block. Returns the nodes reset, -1 when the body
// cannot be repaired (nothing finite, or most of it bad).
__device__ int repair_body(Body& B, float4* __restrict__ nd, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                           const int2* __restrict__ ab, const uint32_t* __restrict__ bmeta, RepairScratch rs) {
    __shared__ int s_cnt, s_nbad;
    __shared__ float s_med[3];
    const int n = B.nnodes, n0 = B.node0, P = rs.P;
    // the median of the finite positions, per axis (std::nth_element's element: the sorted one at m / 2)
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < P; i += blockDim.x) {
        float x = INFINITY, y = INFINITY, z = INFINITY;
        if (i < n) {
            const float4 p = nd[2 * (n0 + i)];
            if (finite3(p.x, p.y, p.z)) x = p.x, y = p.y, z = p.z, atomicAdd(&s_cnt, 1);
        }
        rs.sort[i] = x, rs.sort[P + i] = y, rs.sort[2 * P + i] = z;
    }
    __syncthreads();
    const int m = s_cnt;
    if (m == 0) return -1;
    for (int a = 0; a < 3; a++) block_bitonic_sort(rs.sort + a * P, P);
    if (threadIdx.x == 0) s_med[0] = rs.sort[m / 2], s_med[1] = rs.sort[P + m / 2], s_med[2] = rs.sort[2 * P + m / 2], s_nbad = 0;
    __syncthreads();
    const v3 med = V(s_med[0], s_med[1], s_med[2]);
    const float lim = 0.9f * kMaxNodeSpeed;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float4 p = nd[2 * (n0 + i)], v = nd[2 * (n0 + i) + 1];
        const bool fin = finite3(p.x, p.y, p.z) && finite3(v.x, v.y, v.z);
        const v3 vv = V(v.x, v.y, v.z);
        const bool b = !fin || dot(vv, vv) > lim * lim || length(V(p.x, p.y, p.z) - med) > 300.0f;
        rs.bad[i] = b;
        if (b) atomicAdd(&s_nbad, 1);
    }
    __syncthreads();
    const int nbad0 = s_nbad;
    if (nbad0 == 0) return 0;
    if (nbad0 * 2 > n) return -1;
    // up to 8 passes: each bad node takes the mean of its good neighbours over unbroken beams, in beam order
    for (int pass = 0; pass < 8; pass++) {
        __syncthreads();
        if (s_nbad == 0) break;
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            rs.nv[i].w = 0.0f;
            if (!rs.bad[i]) continue;
            v3 sp = V(0, 0, 0), sv = V(0, 0, 0);
            int cnt = 0;
            for (int q = inc_ptr[n0 + i]; q < inc_ptr[n0 + i + 1]; q++) {
                const int j = inc[q] & 0x7fffffff;
                if ((bmeta[j] >> 8) & BF_BROKEN) continue;
                const int2 e = ab[j];
                const int y = (e.x == n0 + i ? e.y : e.x) - n0;
                if (rs.bad[y]) continue;
                const float4 py = nd[2 * (n0 + y)], vy = nd[2 * (n0 + y) + 1];
                sp = sp + V(py.x, py.y, py.z);
                sv = sv + V(vy.x, vy.y, vy.z);
                cnt++;
            }
            if (cnt > 0) {
                const v3 np = divs(sp, (float)cnt), nv = divs(sv, (float)cnt);
                rs.np[i] = make_float4(np.x, np.y, np.z, 0.0f);
                rs.nv[i] = make_float4(nv.x, nv.y, nv.z, 1.0f);
            }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x)
            if (rs.nv[i].w != 0.0f) {
                const float4 p = nd[2 * (n0 + i)], v = nd[2 * (n0 + i) + 1];
                nd[2 * (n0 + i)] = make_float4(rs.np[i].x, rs.np[i].y, rs.np[i].z, p.w);
                nd[2 * (n0 + i) + 1] = make_float4(rs.nv[i].x, rs.nv[i].y, rs.nv[i].z, v.w);
                rs.bad[i] = 0;
                atomicSub(&s_nbad, 1);
            }
        __syncthreads();
    }
    // isolated leftovers: at the median, at rest; then the bounds and the top speed afresh
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (rs.bad[i]) {
            const float4 p = nd[2 * (n0 + i)], v = nd[2 * (n0 + i) + 1];
            nd[2 * (n0 + i)] = make_float4(med.x, med.y, med.z, p.w);
            nd[2 * (n0 + i) + 1] = make_float4(0.0f, 0.0f, 0.0f, v.w);
        }
    return nbad0;
}

// Block-wide bounds and top speed of a body (SoftBody::compute_aabb, softbody.cpp:271-275; max of |v|)
__device__ void body_bounds(Body& B, const float4* __restrict__ nd) {
    __shared__ float s_mn[3], s_mx[3], s_v;
    if (threadIdx.x == 0) s_mn[0] = s_mn[1] = s_mn[2] = 1e30f, s_mx[0] = s_mx[1] = s_mx[2] = -1e30f, s_v = 0.0f;
    __syncthreads();
    for (int i = threadIdx.x; i < B.nnodes; i += blockDim.x) {
        const float4 p = nd[2 * (B.node0 + i)], v = nd[2 * (B.node0 + i) + 1];
        if (p.x == p.x) atomic_min_f(&s_mn[0], p.x), atomic_max_f(&s_mx[0], p.x);
        if (p.y == p.y) atomic_min_f(&s_mn[1], p.y), atomic_max_f(&s_mx[1], p.y);
        if (p.z == p.z) atomic_min_f(&s_mn[2], p.z), atomic_max_f(&s_mx[2], p.z);
        const float sp = length(V(v.x, v.y, v.z));
        if (sp == sp) atomic_max_f(&s_v, sp);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int c = 0; c < 3; c++) B.aabb_mn[c] = s_mn[c], B.aabb_mx[c] = s_mx[c];
        B.max_speed = s_v;
    }
    __syncthreads();
}

// The end of the frame, one block for all bodies: each stepped body's bounds (the last substep's), top speed and
// static contacts; the repair of the bodies in numerical trouble (world.cpp:3961-3980); World::update_sleep
// (world.cpp:4113-4157; no sheets, no rest damping).
__global__ void __launch_bounds__(1024) k_frame_finish(Body* __restrict__ bodies, int nbodies, float4* __restrict__ nd,
                                                       const int* __restrict__ inc_ptr, const int* __restrict__ inc, const int2* __restrict__ ab,
                                                       const uint32_t* __restrict__ bmeta, RepairScratch rs, float frame_time, int world_sleeping,
                                                       float world_sleep_speed, float sleep_time, uint32_t* __restrict__ deverr) {
    __shared__ int s_any;
    if (threadIdx.x == 0) s_any = 0;
    __syncthreads();
    for (int bi = threadIdx.x; bi < nbodies; bi += blockDim.x) {
        Body& B = bodies[bi];
        B.needs_repair = 0;
        if (B.sleeping) continue;
        for (int c = 0; c < 3; c++) B.aabb_mn[c] = B.acc_mn[c], B.aabb_mx[c] = B.acc_mx[c];
        B.max_speed = sqrtf(B.acc_v2);
        B.static_contacts = B.acc_contacts;
        const float ex = B.aabb_mx[0] - B.aabb_mn[0], ey = B.aabb_mx[1] - B.aabb_mn[1], ez = B.aabb_mx[2] - B.aabb_mn[2];
        if (!isfinite(B.aabb_mn[0]) || !isfinite(B.aabb_mx[1]) || smax(ex, smax(ey, ez)) > 800.0f || B.max_speed > kMaxNodeSpeed * 0.9f) {
            B.needs_repair = 1;
            s_any = 1;
        }
    }
    __syncthreads();
    if (s_any) {
        if (threadIdx.x == 0) atomicOr(deverr, DEVERR_NONFINITE);
        for (int bi = 0; bi < nbodies; bi++) {
            Body& B = bodies[bi];
            if (!B.needs_repair) continue;
            const int fixed = repair_body(B, nd, inc_ptr, inc, ab, bmeta, rs);
            __syncthreads();
            if (fixed < 0) {
                // exploded: frozen where it is (non-finite nodes far below), asleep (world.cpp:3968-3977)
                for (int i = threadIdx.x; i < B.nnodes; i += blockDim.x) {
                    const float4 p = nd[2 * (B.node0 + i)], v = nd[2 * (B.node0 + i) + 1];
                    const bool fin = finite3(p.x, p.y, p.z);
                    nd[2 * (B.node0 + i)] = make_float4(fin ? p.x : 0.0f, fin ? p.y : -1000.0f, fin ? p.z : 0.0f, 0.0f);
                    nd[2 * (B.node0 + i) + 1] = make_float4(0.0f, 0.0f, 0.0f, v.w);
                }
                const float keep = B.max_speed; // (the frame's top speed stays; the bounds are made afresh)
                __syncthreads();
                body_bounds(B, nd);
                if (threadIdx.x == 0) B.max_speed = keep, B.sleeping = 1, B.fell_asleep = 1, B.needs_repair = 2;
            } else if (fixed > 0) {
                __syncthreads();
                body_bounds(B, nd);
                if (threadIdx.x == 0) B.repaired += fixed;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    for (int bi = threadIdx.x; bi < nbodies; bi += blockDim.x) {
        Body& B = bodies[bi];
        if (B.sleeping) continue; // (asleep before this frame, or frozen just now)
        if (!world_sleeping || !B.can_sleep) {
            B.sleep_timer = 0;
            continue;
        }
        const float rest = smax(world_sleep_speed, B.sleep_speed);
        if (B.max_speed < rest) {
            B.sleep_timer += frame_time;
            if (B.sleep_timer > sleep_time) B.sleeping = 1, B.fell_asleep = 1;
        } else {
            B.sleep_timer = 0;
        }
    }
}

// SoftBody::fall_asleep (softbody.h:773-779) for the bodies that just fell asleep: velocities zero; their beams are
// parked (not stepped while the body sleeps)
__global__ void k_sleep_apply(Body* __restrict__ bodies, float4* __restrict__ nd, uint32_t* __restrict__ bmeta) {
    Body& B = bodies[blockIdx.x];
    if (!B.fell_asleep) return;
    for (int i = threadIdx.x; i < B.nnodes; i += blockDim.x) {
        const float4 v = nd[2 * (B.node0 + i) + 1];
        nd[2 * (B.node0 + i) + 1] = make_float4(0.0f, 0.0f, 0.0f, v.w);
    }
    for (int j = threadIdx.x; j < B.nbeams; j += blockDim.x) bmeta[B.beam0 + j] |= kBeamAsleep;
    __syncthreads();
    if (threadIdx.x == 0) B.fell_asleep = 0;
}

} // namespace blg
