// Host side of the B200 soft-body substep: the context behind include/beamlab_gpu.h.
//
// The context keeps a host description of the statics and of the bodies added, and, once committed, the device
// arrays every kernel reads - all bodies back to back, structure of arrays:
//   nodes   nd  2 x float4 a node: (p.xyz, inv_mass), (v.xyz, mass) - the byte layout of the reference's Node and of
//           bl_node, so whole-state transfers are plain copies      info int4 (flags, friction, radius, body)
//           inc_ptr / inc: each node's incident beams in beam order (beam index, bit 31: the node is the beam's b end)
//   beams   ab int2 (a, b)   kd float2 (k, d)   bst float4 (L, max_pos, max_neg, strength)   bmeta u32 (type, flags,
//           the body's deform/break/ductile bits, asleep)   bcold float4 (plastic, L0, support_limit)   stress f32
//           bbody i32   fsc f32: the substep's beam force scalar (scratch between k_beams and k_force)
//   per node: inc2 - the incidences with the other end (k_force), nodef float4 - the substep's force (k_force, the
//           contacts between bodies, k_integrate)
//   bodies  Body records (bl_device.cuh)
// A frame (bl_gpu_step_substeps) is captured once per substep count as a CUDA graph and replayed.
#include "../../include/beamlab_gpu.h"
#include "bl_contacts.cuh"
#include "bl_fem_host.cuh"
#include "bl_fem_kernels.cuh"
#include "bl_fem_pcg.cuh"
#include "bl_mf_plan.cuh"
#include "bl_multifrontal.cuh"
#include "bl_mlp.cuh"
#include "bl_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <new>
#include <vector>

using namespace blg;

namespace {

struct HostBody {
    std::vector<bl_node> nodes;
    std::vector<bl_node_info> info;
    std::vector<bl_beam> beams;
    std::vector<bl_tri> tris;              // collision triangles (their torn flags come back from the device)
    uint32_t beam_bits = 0; // the body's allow_deform / allow_break / ductile as BB_* bits of its beams' meta words
    Body rec;
    std::vector<float4> ext;               // constant node forces (empty: none)
    std::shared_ptr<FemModel> fem;         // its FEM frame (null: none), with its dynamic state q / w between commits
    std::vector<FemSection> sections;
    std::vector<FrameSectionH> fsections;   // its members' sections
    std::vector<float> fq, fw;             // frame nodes' orientation (4) and angular velocity (3)
    float theta = 0.5f, diss = 0.02f;
    int fem_failures = 0, fem_clamps = 0;
    float repass_credit = 8.0f;            // FemFrame::repass_credit_ (refilled for its next step)
    int elastic_step = 0;                  // FemFrame::elastic_step_ of its next step
    struct Wheel {
        uint32_t axle0, axle1;
        std::vector<uint32_t> nodes;      // its tyre nodes in the given order (the parity of a place: the hub it turns about)
        float radius, mass;
        int propulsed, arm, near_attach;  // (arm, near_attach: the body's nodes, -1 none)
        float torque = 0, brake = 0;      // the controller's, every substep (bl_gpu_set_wheel_drive)
        float st[4] = {0, 0, 0, 0};       // speed, avg_speed, last_torque, last_retorque between commits
    };
    std::vector<Wheel> wheels;             // its node wheels (empty: none)
    int wheel0 = 0;                        // its first wheel among the context's (the last commit's)
    std::vector<bl_shock> shocks;          // its shocks in their order (beam: the body's)
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void free_() {
        if (p) cudaFree(p);
        p = nullptr, n = 0;
    }
    cudaError_t alloc(size_t count) {
        free_();
        n = count;
        return cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(count, 1));
    }
};

} // namespace

struct bl_gpu_ctx {
    bl_gpu_config cfg{};
    cudaStream_t stream = nullptr;
    int last_cuda = 0;
    // host description
    std::vector<HostBody> bodies;
    bool bodies_dirty = false; // bodies added since the last commit
    bool committed = false;
    // statics (host)
    int has_terrain = 0, hnx = 0, hnz = 0, hbx = 0, hbz = 0;
    float cell = 1, ox = 0, oz = 0, kill_y = -200.0f;
    std::vector<float> heights, block_max;
    std::vector<uint8_t> surfaces;
    std::vector<Box> boxes;
    std::vector<Cyl> cyls;
    int gx = 0, gz = 0;
    float gox = 0, goz = 0, grid_cell = 16.0f;
    std::vector<int> cell_ptr, cell_items, big;
    bool statics_dirty = true;
    // device
    DevBuf<float4> nd, bst, bcold, nodef;
    DevBuf<float> fsc;
    DevBuf<int2> inc2;                         // per node's incidences, warp-interleaved (k_force)
    DevBuf<int> ell_ptr;
    bool packed_inc = false;                   // the incidences in their 4-byte form (inc4, ell_base) instead
    DevBuf<uint32_t> inc4;
    DevBuf<int> ell_base;
    int beam_tiles = 0;                        // k_beams_tma's tiles (the beam arrays hold beam_tiles * kBeamTile)
    int beam_grid = 0;                         // its persistent grid (0: not sized yet)
    bool ends16 = false;                       // its beams' ends as 16-bit offsets from their tile's base node
    DevBuf<uint32_t> ab16;
    DevBuf<int> tbase;
    DevBuf<int4> info;
    DevBuf<int> inc_ptr, inc, bbody;
    DevBuf<int2> ab;
    DevBuf<float2> kd;
    DevBuf<uint32_t> bmeta;
    DevBuf<float> stress;
    DevBuf<Body> dbodies;
    DevBuf<float> d_heights, d_block_max;
    DevBuf<uint8_t> d_surf;
    DevBuf<Box> d_boxes;
    DevBuf<Cyl> d_cyls;
    DevBuf<int> d_cell_ptr, d_cell_items, d_big;
    DevBuf<uint32_t> deverr;
    DevBuf<float> rs_sort;
    DevBuf<int> rs_bad;
    DevBuf<float4> rs_np, rs_nv;
    int rs_P = 1;
    int N = 0, M = 0, B = 0;
    Statics st{};
    // FEM frames of all bodies back to back (see bl_fem_kernels.cuh)
    int NF = 0, NT = 0, NB = 0, n_fem_nodes = 0;
    bool any_plastic = false;                  // a yielding shell section on a body that deforms (k_tri_eval<true>)
    bool fem_ground = false;                   // a frame body's node collides with the static world (k_fem_static)
    DevBuf<float4> contact_n;                  // per frame node: its ground contact's normal this step
    bool any_plastic_members = false;          // a yielding member section on a body that deforms (k_member_eval<true>,
                                               // the unload re-pass)
    int64_t NU = 0;                            // block updates of a factorization
    bool any_ext = false;
    bool any_drag = false;                     // some body has air drag (k_drag_parts)
    DevBuf<int> dup, dpid, dpart;
    DevBuf<float4> dpmv, dpacc;
    int NW = 0;                                // the wheels of all bodies, and lone tyre nodes (k_tyres: a warp a wheel)
    int NSH = 0;                               // the shocks of all bodies (k_shocks)
    DevBuf<bl_shock> dshock;
    DevBuf<int> sh_ptr;
    DevBuf<int2> sh_inc;
    DevBuf<float> ssc;
    DevBuf<int4> dwheel;
    DevBuf<int> dwnodes;
    DevBuf<int> dwlist, dwc_ptr;
    DevBuf<int2> dwc;
    DevBuf<float4> dwst, dwctl, dwcf;
    DevBuf<int4> dwarm;
    DevBuf<float> dwper;
    int NWR = 0;                               // of those, the builders' wheels (k_wheels)
    DevBuf<float4> dtcon, dtfric;
    std::vector<int> lvl_grp_ptr, lvl_col_ptr; // per level: its update groups / columns
    int64_t fem_launches = 0;                  // kernels of one substep's frame step (with the Cholesky)
    int64_t chol_launches = 0;                 // of those, the factorization's and substitutions'
    // the frames' solve by PCG (bl_fem_pcg.cuh) and the residual check
    DevBuf<double> px, pr, pz, pp, ppf, ppdi, pred, a0d, a0o, b0, res, plast, pxprev;
    DevBuf<int> pstat;
    DevBuf<long long> piters;
    DevBuf<float> guess, gscale;               // the learned per-frame-node dv guess (3) and preconditioner scale (9)
    int pcg_grid = 1;
    std::vector<int> lvl_ns;                   // per level: the slices of kUnit rows its columns' factor is cut in
    cudaStream_t aux = nullptr;                // (captures the bodies of conditional graph nodes)
    // the learned warm start (bl_mlp.cuh): parameters, the step's features, recorded samples, training scratch
    DevBuf<float> mlp_w, mlp_m, mlp_v, feat, prev_dv, smp_x, smp_t, smp_w, gpart, lpart, gsum;
    DevBuf<__nv_bfloat16> mlp_wb;
    DevBuf<int> adj_ptr, adj, scount, sidx;
    int rec_cap = 0;                           // the samples' capacity
    bool rec_on = false;                       // the step records samples
    int adam_t = 0;
    DevBuf<float4> ext, nforce, fq, fw, ftorque, tr0, tf, tt;
    DevBuf<int> fnode, fbody, fperm, fiperm, grp_tgt, grp_ptr, col_comp, comp_fail, rb_ptr, lvl_col, fem_nodes, fslot;
    DevBuf<int> fcol_ptr, frow, fblk_col, gdiag_ptr, goff_ptr, fem_fail, fem_clamp;
    DevBuf<int2> gdiag, gu, rb;
    DevBuf<int4> goff, tn;
    DevBuf<double> xd, diag, ldiag, off, rhs, dinv, tkv, ch2, chd;
    // the FEM members (k_member_eval)
    int NM = 0;
    DevBuf<int2> mn;
    DevBuf<int> mmeta;
    DevBuf<float> mL0;
    DevBuf<float4> mq, mfa, mta, mtb, mtan, mps, mtg;
    DevBuf<uint32_t> mflag;
    DevBuf<float> credit;
    DevBuf<int> elastic, comp_again, comp_size, body_comp, rp;
    DevBuf<long long> repc;
    DevBuf<FemMemSecDev> msec;
    DevBuf<uint8_t> mon;
    DevBuf<double> mkw, mkv;
    // the top chain of the elimination tree as one dense front (bl_fem_kernels.cuh: FrontDev); front_level: its first
    // level (the level count: none)
    FrontDev front{};
    int front_level = 0;
    DevBuf<int> fcol, fchain;
    DevBuf<int4> fblk;
    DevBuf<double> fD, fb;
    // the multifrontal factorization (bl_multifrontal.cuh), fem_dense_front == 2: fronts, their maps, the pool, and per
    // level its task ranges (assembly; per panel, panel and update tasks)
    MfDev mf{};
    DevBuf<MfFrontDev> mf_fr;
    DevBuf<int> mf_idx, mf_cmap, mf_child, mf_brow;
    DevBuf<double> mf_pool, mf_dt;
    DevBuf<int2> mf_tpan;
    DevBuf<int4> mf_tasm, mf_tupd;
    std::vector<int> mf_level_ptr;             // fronts of each level (execution order)
    std::vector<int> mf_tasm_ptr;              // per level: its assembly tasks
    std::vector<std::vector<int>> mf_tpan_ptr, mf_tupd_ptr; // per level, per panel: its tasks
    size_t mf_smem = 0;                        // the solves' dynamic shared memory (the largest front)
    int fem_mode = 0;                          // the factorization in use: fem_dense_front, 3 resolved to 1 or 2
    unsigned long long wait_ns = 1000000000ull; // the beams kernel's bound on a wait for its bulk copies (bulk_wait_s)
    double mf_flops = 0;
    DevBuf<float> finertia, tX, tk, ttan, tb, tX0, th0, tdmg;
    DevBuf<uint8_t> tbroken, ton, ffixed;
    DevBuf<FemSecDev> fsec;
    FemDev fd{};
    // contacts between bodies (bl_contacts.cuh): on when some body has collision triangles
    bool contacts_on = false;
    int interval = 1, NTRI = 0, max_isl = 0;
    DevBuf<int4> dtri, pt_cell;
    DevBuf<float> tri_rest2, ibox;
    DevBuf<int> parent, isl_live, isl_cnt, isl_nodes, isl_idx, isl_noff, isl_poff, isl_pcnt, isl_contacts, pair_total;
    DevBuf<int> pt_node, pt_body, bk_start, bk_fill, bk_items, run_end, g_start, g_fill, g_items, counters;
    DevBuf<int2> pairs;
    DevBuf<float4> hit_a, hit_b;
    // the pair search's records, island states, queries and counters (bl_pair_search.cuh)
    DevBuf<float4> g_rec, sb_pos;
    DevBuf<int4> sb_cell, q_group;
    DevBuf<int> g_hi, q_count, sc;
    DevBuf<int2> q_chunk, ptmp;
    DevBuf<int> q_tmp;
    DevBuf<IslSearch> isl;
    DevBuf<uint32_t> hbits;
    DevBuf<ContactRec> crec;
    DevBuf<int> crec_n;
    DevBuf<int> hidx;
    Contacts ct{};
    // frames captured as graphs, by substep count
    std::map<int, cudaGraphExec_t> graphs;
    struct ProfGraph {
        cudaGraphExec_t exec = nullptr;
        std::vector<cudaEvent_t> events;
    };
    std::map<int, ProfGraph> pgraphs; // frames with a timing event between kernels (bl_gpu_profile_frame)
    int64_t launches = 0, total_substeps = 0;
    int last_substeps = 0;
    // the stream of the last enqueued work: work on another stream first waits for it, so calls stay ordered
    cudaStream_t last_stream = nullptr;
    cudaEvent_t order_event = nullptr;
};

#define BL_CUDA(ctx, call)                                                                                                                   \
    do {                                                                                                                                     \
        cudaError_t e_ = (call);                                                                                                             \
        if (e_ != cudaSuccess) {                                                                                                             \
            (ctx)->last_cuda = (int)e_;                                                                                                      \
            return e_ == cudaErrorMemoryAllocation ? BL_GPU_ENOMEM : BL_GPU_ECUDA;                                                           \
        }                                                                                                                                    \
    } while (0)

using ProfGraph = bl_gpu_ctx::ProfGraph;

static void drop_graphs(bl_gpu_ctx* c) {
    for (auto& kv : c->graphs) cudaGraphExecDestroy(kv.second);
    c->graphs.clear();
    for (auto& kv : c->pgraphs) {
        cudaGraphExecDestroy(kv.second.exec);
        for (cudaEvent_t e : kv.second.events) cudaEventDestroy(e);
    }
    c->pgraphs.clear();
}

static void free_fem(bl_gpu_ctx* c) {
    c->ext.free_(), c->nforce.free_(), c->fq.free_(), c->fw.free_(), c->ftorque.free_(), c->tr0.free_(), c->tf.free_(), c->tt.free_();
    c->fnode.free_(), c->fbody.free_(), c->fperm.free_(), c->fiperm.free_(), c->grp_tgt.free_(), c->grp_ptr.free_();
    c->col_comp.free_(), c->comp_fail.free_(), c->rb_ptr.free_(), c->lvl_col.free_(), c->fem_nodes.free_(), c->fslot.free_();
    c->fcol_ptr.free_(), c->frow.free_(), c->fblk_col.free_(), c->gdiag_ptr.free_(), c->goff_ptr.free_(), c->fem_fail.free_(), c->fem_clamp.free_();
    c->px.free_(), c->pr.free_(), c->pz.free_(), c->pp.free_(), c->ppf.free_(), c->ppdi.free_(), c->pred.free_(), c->a0d.free_(), c->pxprev.free_();
    c->a0o.free_(), c->b0.free_(), c->res.free_(), c->plast.free_(), c->pstat.free_(), c->piters.free_(), c->guess.free_(), c->gscale.free_();
    c->feat.free_(), c->prev_dv.free_(), c->adj_ptr.free_(), c->adj.free_();
    c->gdiag.free_(), c->gu.free_(), c->rb.free_(), c->goff.free_(), c->tn.free_();
    c->fcol.free_(), c->fchain.free_(), c->fblk.free_(), c->fD.free_(), c->fb.free_(), c->front = FrontDev{}, c->front_level = 0;
    c->mf_fr.free_(), c->mf_idx.free_(), c->mf_cmap.free_(), c->mf_child.free_(), c->mf_brow.free_(), c->mf_pool.free_(), c->mf_dt.free_();
    c->mf_tasm.free_(), c->mf_tpan.free_(), c->mf_tupd.free_(), c->mf = MfDev{}, c->mf_level_ptr.clear(), c->mf_flops = 0;
    c->mn.free_(), c->mmeta.free_(), c->mL0.free_(), c->mq.free_(), c->mfa.free_(), c->mta.free_(), c->mtb.free_(), c->mtan.free_();
    c->msec.free_(), c->mon.free_(), c->mkw.free_(), c->mkv.free_(), c->NM = 0;
    c->mps.free_(), c->mtg.free_(), c->mflag.free_(), c->credit.free_(), c->elastic.free_(), c->comp_again.free_(), c->comp_size.free_();
    c->body_comp.free_(), c->rp.free_(), c->repc.free_();
    c->contact_n.free_(), c->fem_ground = false;
    c->xd.free_(), c->diag.free_(), c->ldiag.free_(), c->off.free_(), c->rhs.free_(), c->dinv.free_(), c->tkv.free_(), c->ch2.free_(), c->chd.free_();
    c->finertia.free_(), c->tX.free_(), c->tk.free_(), c->tb.free_(), c->tX0.free_(), c->th0.free_(), c->tdmg.free_(), c->ttan.free_(), c->tbroken.free_(), c->ton.free_(), c->ffixed.free_(), c->fsec.free_();
}

static void free_contacts(bl_gpu_ctx* c) {
    c->dtri.free_(), c->pt_cell.free_(), c->tri_rest2.free_(), c->ibox.free_(), c->parent.free_(), c->isl_live.free_();
    c->isl_cnt.free_(), c->isl_nodes.free_(), c->isl_idx.free_(), c->isl_noff.free_(), c->isl_poff.free_(), c->isl_pcnt.free_();
    c->isl_contacts.free_(), c->pair_total.free_(), c->pt_node.free_(), c->pt_body.free_(), c->bk_start.free_(), c->bk_fill.free_();
    c->bk_items.free_(), c->run_end.free_(), c->g_start.free_(), c->g_fill.free_(), c->g_items.free_(), c->counters.free_();
    c->pairs.free_(), c->hit_a.free_(), c->hit_b.free_();
    c->g_rec.free_(), c->sb_pos.free_(), c->sb_cell.free_(), c->q_group.free_(), c->g_hi.free_(), c->q_count.free_(), c->sc.free_();
    c->q_chunk.free_(), c->ptmp.free_(), c->q_tmp.free_(), c->isl.free_(), c->hbits.free_(), c->hidx.free_(), c->crec.free_(), c->crec_n.free_();
    c->contacts_on = false;
}

static void free_device(bl_gpu_ctx* c) {
    free_fem(c);
    free_contacts(c);
    c->nd.free_(), c->bst.free_(), c->bcold.free_(), c->nodef.free_(), c->fsc.free_(), c->inc2.free_(), c->ell_ptr.free_(), c->info.free_(), c->inc_ptr.free_(), c->inc.free_();
    c->inc4.free_(), c->ell_base.free_(), c->packed_inc = false;
    c->ab16.free_(), c->tbase.free_(), c->ends16 = false;
    c->dup.free_(), c->dpid.free_(), c->dpart.free_(), c->dpmv.free_(), c->dpacc.free_();
    c->dwheel.free_(), c->dwnodes.free_(), c->dtcon.free_(), c->dtfric.free_(), c->NW = 0;
    c->dwlist.free_(), c->dwc_ptr.free_(), c->dwc.free_(), c->dwst.free_(), c->dwctl.free_(), c->dwcf.free_(), c->dwarm.free_(), c->dwper.free_(), c->NWR = 0;
    c->dshock.free_(), c->sh_ptr.free_(), c->sh_inc.free_(), c->ssc.free_(), c->NSH = 0;
    c->bbody.free_(), c->ab.free_(), c->kd.free_(), c->bmeta.free_(), c->stress.free_(), c->dbodies.free_();
    c->rs_sort.free_(), c->rs_bad.free_(), c->rs_np.free_(), c->rs_nv.free_();
}

static void free_statics(bl_gpu_ctx* c) {
    c->d_heights.free_(), c->d_block_max.free_(), c->d_surf.free_(), c->d_boxes.free_(), c->d_cyls.free_();
    c->d_cell_ptr.free_(), c->d_cell_items.free_(), c->d_big.free_();
}

// Ground models (static_world.cpp:85-114): va, ms, mc, t2, vs, alpha, strength, soft_depth, fluid_drag, fluid_density
static const GroundModel kGroundModels[kSurfCount] = {
    {3, 0.80f, 0.55f, 0.005f, 7, 2, 1, 0, 0, 0},          {3, 0.80f, 0.58f, 0.006f, 4, 2, 1, 0, 0, 0},
    {3, 1.20f, 0.75f, 0.010f, 6, 2, 1, 0, 0, 0},          {3, 1.20f, 0.75f, 0.010f, 6, 2, 1, 0, 0, 0},
    {3, 0.85f, 0.60f, 0.006f, 3, 2, 1, 0, 0, 0},          {2, 0.50f, 0.35f, 0.004f, 3, 2, 1, 0.12f, 60, 1500},
    {3, 0.70f, 0.55f, 0.0001f, 9, 2, 1, 0.03f, 20, 1600}, {3, 0.95f, 0.70f, 0.007f, 8, 2, 1, 0, 0, 0},
    {3, 0.90f, 0.60f, 0.005f, 5, 2, 1, 0, 0, 0},          {3, 0.70f, 0.40f, 0.001f, 3, 2, 1, 0, 0, 0},
    {1, 0.30f, 0.20f, 0.0001f, 3, 2, 1, 0, 0, 0},
};

// ------------------------------------------------------------------------------------------ statics (host)
// StaticWorld::build_grid (static_world.cpp:308-338): 16 m cells over the bounds of the boxes and cylinders; a box
// over more than 64 cells goes to the big list; each cell lists its boxes in box order
static void build_grid_host(bl_gpu_ctx* c) {
    c->cell_ptr.clear(), c->cell_items.clear(), c->big.clear();
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    auto add = [&](float x, float y, float z) {
        const float p[3] = {x, y, z};
        for (int k = 0; k < 3; k++) mn[k] = (p[k] < mn[k]) ? p[k] : mn[k], mx[k] = (mx[k] < p[k]) ? p[k] : mx[k];
    };
    for (const Box& b : c->boxes) add(b.mnx, b.mny, b.mnz), add(b.mxx, b.mxy, b.mxz);
    for (const Cyl& y : c->cyls) add(y.bx - y.radius, y.by - 0.0f, y.bz - y.radius), add(y.bx + y.radius, y.by + y.height, y.bz + y.radius);
    if (!(mn[0] <= mx[0])) {
        c->gx = c->gz = 0;
        return;
    }
    c->gox = mn[0], c->goz = mn[2];
    c->gx = std::max(1, (int)std::ceil((mx[0] - mn[0]) / c->grid_cell) + 1);
    c->gz = std::max(1, (int)std::ceil((mx[2] - mn[2]) / c->grid_cell) + 1);
    std::vector<std::vector<int>> cells((size_t)c->gx * c->gz);
    for (int i = 0; i < (int)c->boxes.size(); i++) {
        const Box& a = c->boxes[i];
        const int x0 = (int)((a.mnx - c->gox) / c->grid_cell), x1 = (int)((a.mxx - c->gox) / c->grid_cell);
        const int z0 = (int)((a.mnz - c->goz) / c->grid_cell), z1 = (int)((a.mxz - c->goz) / c->grid_cell);
        if ((x1 - x0 + 1) * (z1 - z0 + 1) > 64) {
            c->big.push_back(i);
            continue;
        }
        for (int z = z0; z <= z1; z++)
            for (int x = x0; x <= x1; x++) cells[(size_t)z * c->gx + x].push_back(i);
    }
    c->cell_ptr.assign(cells.size() + 1, 0);
    for (size_t k = 0; k < cells.size(); k++) {
        c->cell_ptr[k + 1] = c->cell_ptr[k] + (int)cells[k].size();
        c->cell_items.insert(c->cell_items.end(), cells[k].begin(), cells[k].end());
    }
}

template <class T>
static int upload_vec(bl_gpu_ctx* c, DevBuf<T>& d, const std::vector<T>& h) {
    BL_CUDA(c, d.alloc(h.size()));
    if (!h.empty()) BL_CUDA(c, cudaMemcpyAsync(d.p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, c->stream));
    return BL_GPU_OK;
}

static int commit_statics(bl_gpu_ctx* c) {
    free_statics(c);
    int rc;
    if ((rc = upload_vec(c, c->d_heights, c->heights)) || (rc = upload_vec(c, c->d_block_max, c->block_max)) || (rc = upload_vec(c, c->d_surf, c->surfaces)) ||
        (rc = upload_vec(c, c->d_boxes, c->boxes)) || (rc = upload_vec(c, c->d_cyls, c->cyls)) || (rc = upload_vec(c, c->d_cell_ptr, c->cell_ptr)) ||
        (rc = upload_vec(c, c->d_cell_items, c->cell_items)) || (rc = upload_vec(c, c->d_big, c->big)))
        return rc;
    Statics& s = c->st;
    s.has_terrain = c->has_terrain, s.hnx = c->hnx, s.hnz = c->hnz, s.bx = c->hbx, s.bz = c->hbz;
    s.cell = c->cell, s.ox = c->ox, s.oz = c->oz;
    s.h = c->d_heights.p, s.surf = c->d_surf.p, s.block_max = c->d_block_max.p;
    s.kill_y = c->kill_y;
    s.nboxes = (int)c->boxes.size(), s.ncyls = (int)c->cyls.size();
    s.boxes = c->d_boxes.p, s.cyls = c->d_cyls.p;
    s.gx = c->gx, s.gz = c->gz, s.nbig = (int)c->big.size();
    s.gox = c->gox, s.goz = c->goz, s.grid_cell = c->grid_cell;
    s.cell_ptr = c->d_cell_ptr.p, s.cell_items = c->d_cell_items.p, s.big = c->d_big.p;
    c->statics_dirty = false;
    drop_graphs(c);
    return BL_GPU_OK;
}

// ------------------------------------------------------------------------------------------ bodies
// Brings the device's current state of the committed bodies back into the host description (before a re-commit).
static int pull_state(bl_gpu_ctx* c) {
    if (!c->committed) return BL_GPU_OK;
    std::vector<bl_node> nodes(c->N);
    std::vector<float4> bst(c->M);
    std::vector<uint32_t> meta(c->M);
    std::vector<float> stress(c->M);
    std::vector<Body> recs(c->B);
    BL_CUDA(c, cudaMemcpyAsync(nodes.data(), c->nd.p, sizeof(bl_node) * c->N, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaMemcpyAsync(bst.data(), c->bst.p, sizeof(float4) * c->M, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaMemcpyAsync(meta.data(), c->bmeta.p, sizeof(uint32_t) * c->M, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaMemcpyAsync(stress.data(), c->stress.p, sizeof(float) * c->M, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaMemcpyAsync(recs.data(), c->dbodies.p, sizeof(Body) * c->B, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int bi = 0; bi < c->B; bi++) {
        HostBody& hb = c->bodies[bi];
        const Body& r = recs[bi];
        for (int i = 0; i < r.nnodes; i++) hb.nodes[i] = nodes[r.node0 + i];
        for (int j = 0; j < r.nbeams; j++) {
            bl_beam& b = hb.beams[j];
            const float4 s = bst[r.beam0 + j];
            b.L = s.x, b.max_pos = s.y, b.max_neg = s.z, b.strength = s.w;
            b.flags = (uint8_t)((meta[r.beam0 + j] >> 8) & 0xff);
            b.stress = stress[r.beam0 + j];
        }
        hb.rec = r;
        hb.rec.part_count = 0; // (the parts' labels live in arrays made again at the commit: made again at the next call)
    }
    if (c->contacts_on && c->NTRI > 0) {
        std::vector<int4> tri(c->NTRI);
        BL_CUDA(c, cudaMemcpy(tri.data(), c->dtri.p, sizeof(int4) * c->NTRI, cudaMemcpyDeviceToHost));
        for (int bi = 0; bi < c->B; bi++) {
            HostBody& hb = c->bodies[bi];
            for (int t = 0; t < hb.rec.ntris; t++) hb.tris[t].torn = (tri[hb.rec.tri0 + t].w & TF_TORN) ? 1 : 0;
        }
    }
    if (c->NWR > 0) { // (the wheels' speeds and their last torques and reactions)
        std::vector<float4> st(c->NWR);
        BL_CUDA(c, cudaMemcpy(st.data(), c->dwst.p, sizeof(float4) * c->NWR, cudaMemcpyDeviceToHost));
        for (HostBody& hb : c->bodies)
            for (size_t k = 0; k < hb.wheels.size() && !hb.fem; k++) {
                const float4 v = st[hb.wheel0 + k];
                hb.wheels[k].st[0] = v.x, hb.wheels[k].st[1] = v.y, hb.wheels[k].st[2] = v.z, hb.wheels[k].st[3] = v.w;
            }
    }
    // the frames' dynamic state (their positions in double, orientations, spins) and counters
    if (c->NF > 0) {
        std::vector<double> xd(3 * (size_t)c->NF);
        std::vector<float4> q(c->NF), w(c->NF);
        std::vector<int> ff(c->B), fc(c->B);
        BL_CUDA(c, cudaMemcpy(xd.data(), c->xd.p, sizeof(double) * xd.size(), cudaMemcpyDeviceToHost));
        BL_CUDA(c, cudaMemcpy(q.data(), c->fq.p, sizeof(float4) * c->NF, cudaMemcpyDeviceToHost));
        BL_CUDA(c, cudaMemcpy(w.data(), c->fw.p, sizeof(float4) * c->NF, cudaMemcpyDeviceToHost));
        BL_CUDA(c, cudaMemcpy(ff.data(), c->fem_fail.p, sizeof(int) * c->B, cudaMemcpyDeviceToHost));
        BL_CUDA(c, cudaMemcpy(fc.data(), c->fem_clamp.p, sizeof(int) * c->B, cudaMemcpyDeviceToHost));
        int fo = 0;
        for (int bi = 0; bi < c->B; bi++) {
            HostBody& hb = c->bodies[bi];
            hb.fem_failures = ff[bi], hb.fem_clamps = fc[bi];
            if (!hb.fem) continue;
            const int nf = (int)hb.fem->node.size();
            for (int i = 0; i < nf; i++) {
                for (int j = 0; j < 3; j++) hb.fem->xd[3 * i + j] = xd[3 * (size_t)(fo + i) + j];
                hb.fq[4 * i] = q[fo + i].x, hb.fq[4 * i + 1] = q[fo + i].y, hb.fq[4 * i + 2] = q[fo + i].z, hb.fq[4 * i + 3] = q[fo + i].w;
                hb.fw[3 * i] = w[fo + i].x, hb.fw[3 * i + 1] = w[fo + i].y, hb.fw[3 * i + 2] = w[fo + i].z;
            }
            fo += nf;
        }
        if (c->NT > 0) { // (the triangles' plastic state: rest shapes and frames, stiffnesses, their flow)
            std::vector<float> tX(6 * (size_t)c->NT), tk(162 * (size_t)c->NT), tb(54 * (size_t)c->NT), th0(9 * (size_t)c->NT), tdmg(c->NT);
            std::vector<float4> tr0(3 * (size_t)c->NT);
            BL_CUDA(c, cudaMemcpy(tX.data(), c->tX.p, sizeof(float) * tX.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(tk.data(), c->tk.p, sizeof(float) * tk.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(tb.data(), c->tb.p, sizeof(float) * tb.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(th0.data(), c->th0.p, sizeof(float) * th0.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(tdmg.data(), c->tdmg.p, sizeof(float) * tdmg.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(tr0.data(), c->tr0.p, sizeof(float4) * tr0.size(), cudaMemcpyDeviceToHost));
            int to = 0;
            for (int bi = 0; bi < c->B; bi++) {
                HostBody& hb = c->bodies[bi];
                if (!hb.fem) continue;
                FemModel& M = *hb.fem;
                const size_t nt = M.tn.size();
                std::copy(tX.begin() + 6 * to, tX.begin() + 6 * (to + nt), M.tX.begin());
                std::copy(tk.begin() + 162 * to, tk.begin() + 162 * (to + nt), M.tk.begin());
                std::copy(tb.begin() + 54 * to, tb.begin() + 54 * (to + nt), M.tb.begin());
                std::copy(th0.begin() + 9 * to, th0.begin() + 9 * (to + nt), M.th0.begin());
                std::copy(tdmg.begin() + to, tdmg.begin() + to + nt, M.tdmg.begin());
                for (size_t t = 0; t < nt; t++)
                    for (int i = 0; i < 3; i++) {
                        const float4 r = tr0[3 * (to + t) + i];
                        M.tr0[12 * t + 4 * i] = r.x, M.tr0[12 * t + 4 * i + 1] = r.y, M.tr0[12 * t + 4 * i + 2] = r.z, M.tr0[12 * t + 4 * i + 3] = r.w;
                    }
                to += (int)nt;
            }
        }
        if (c->NM > 0 && c->any_plastic_members) { // (the members' plastic state and rest frames, the re-passes' budget)
            std::vector<float4> mq(2 * (size_t)c->NM), mps(4 * (size_t)c->NM);
            std::vector<uint32_t> mflag(c->NM);
            std::vector<float> credit(c->B);
            std::vector<int> elastic(c->B);
            BL_CUDA(c, cudaMemcpy(mq.data(), c->mq.p, sizeof(float4) * mq.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(mps.data(), c->mps.p, sizeof(float4) * mps.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(mflag.data(), c->mflag.p, sizeof(uint32_t) * mflag.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(credit.data(), c->credit.p, sizeof(float) * credit.size(), cudaMemcpyDeviceToHost));
            BL_CUDA(c, cudaMemcpy(elastic.data(), c->elastic.p, sizeof(int) * elastic.size(), cudaMemcpyDeviceToHost));
            size_t mo = 0;
            for (int bi = 0; bi < c->B; bi++) {
                HostBody& hb = c->bodies[bi];
                hb.repass_credit = credit[bi], hb.elastic_step = elastic[bi];
                if (!hb.fem) continue;
                FemModel& M = *hb.fem;
                const size_t E = M.mn.size();
                M.mps.resize(16 * E), M.mflag.resize(E);
                for (size_t e = 0; e < E; e++) {
                    const float4 qa = mq[2 * (mo + e)], qb = mq[2 * (mo + e) + 1];
                    const float q8[8] = {qa.x, qa.y, qa.z, qa.w, qb.x, qb.y, qb.z, qb.w};
                    for (int k = 0; k < 8; k++) M.mq[8 * e + k] = q8[k];
                    for (int k = 0; k < 4; k++) {
                        const float4 v = mps[4 * (mo + e) + k];
                        M.mps[16 * e + 4 * k] = v.x, M.mps[16 * e + 4 * k + 1] = v.y, M.mps[16 * e + 4 * k + 2] = v.z, M.mps[16 * e + 4 * k + 3] = v.w;
                    }
                    M.mflag[e] = mflag[mo + e];
                }
                mo += E;
            }
        }
    }
    return BL_GPU_OK;
}

// The FEM frames of all bodies on the device, back to back, and the factorization's schedule: the columns by
// elimination-tree level (a column's level is one more than its deepest child's), each level's target blocks (a
// column's diagonal block then its off-diagonal ones) with each target's updates in the order of their source columns,
// each row's blocks in the order of their columns for the forward substitution.
// The multifrontal plan over every frame's columns (global pattern col_ptr / row, components col_comp): the fronts,
// their maps and the pool on the device, and each level's task lists (bl_multifrontal.cuh)
static int commit_multifrontal(bl_gpu_ctx* c, const std::vector<int>& col_ptr, const std::vector<int>& row, const std::vector<int>& col_comp) {
    const int NF = (int)col_ptr.size() - 1;
    std::vector<std::vector<int>> fr_cols;
    std::vector<int> fr_top, fr_comp;
    mf_plan_columns(NF, col_ptr, row, col_comp, fr_cols, fr_top, fr_comp);
    const MfPlan P = mf_finish(NF, col_ptr, row, fr_cols, fr_top, fr_comp);
    const int nfr = (int)P.npiv.size(), nlev = (int)P.level_ptr.size() - 1;
    std::vector<MfFrontDev> fr(nfr);
    long long pool = 0;
    int dtn = 0, maxn = 0;
    for (int f = 0; f < nfr; f++) {
        MfFrontDev& d = fr[f];
        d.n = 6 * (P.npiv[f] + P.nrow[f]), d.p = 6 * P.npiv[f];
        d.off = pool, d.idx0 = P.idx_ptr[f], d.child0 = P.child_ptr[f], d.child1 = P.child_ptr[f + 1], d.comp = P.comp[f];
        d.dt0 = dtn;
        pool += (long long)d.n * (d.n + 1);
        dtn += 2 * kMfT * kMfT * ((d.p + kMfT - 1) / kMfT);
        maxn = std::max(maxn, d.n);
    }
    // each off-diagonal block's row: its node's place in the front of its column
    std::vector<int> brow(std::max<size_t>(row.size(), 1), 0);
    for (int f = 0; f < nfr; f++) {
        const int* first = P.idx.data() + P.idx_ptr[f];
        const int* last = P.idx.data() + P.idx_ptr[f + 1];
        for (int l = 0; l < P.npiv[f]; l++) {
            const int k = first[l];
            for (int pb = col_ptr[k]; pb < col_ptr[k + 1]; pb++) brow[pb] = (int)(std::lower_bound(first, last, row[pb]) - first);
        }
    }
    std::vector<int4> tasm, tupd;
    std::vector<int2> tpan;
    c->mf_tasm_ptr.assign(1, 0), c->mf_tpan_ptr.assign(nlev, {}), c->mf_tupd_ptr.assign(nlev, {});
    int64_t launches = 0;
    for (int L = 0; L < nlev; L++) {
        int np = 0;
        for (int f = P.level_ptr[L]; f < P.level_ptr[L + 1]; f++) {
            const int nt = (fr[f].n + kMfT - 1) / kMfT;
            for (int it = 0; it < nt; it++) {
                for (int jt = 0; jt <= it; jt++) tasm.push_back(make_int4(f, it, jt, 0));
                tasm.push_back(make_int4(f, it, -1, 0));
            }
            np = std::max(np, (fr[f].p + kMfT - 1) / kMfT);
        }
        c->mf_tasm_ptr.push_back((int)tasm.size());
        c->mf_tpan_ptr[L].push_back((int)tpan.size()), c->mf_tupd_ptr[L].push_back((int)tupd.size());
        for (int sp = 0; sp < np; sp++) {
            for (int f = P.level_ptr[L]; f < P.level_ptr[L + 1]; f++) {
                if (fr[f].p <= kMfT * sp) continue;
                const int nt = (fr[f].n + kMfT - 1) / kMfT;
                for (int r = sp; r < nt; r++) tpan.push_back(make_int2(f, r));
                tupd.push_back(make_int4(f, 0, -1, 0));
                for (int i = sp + 1; i < nt; i++) tupd.push_back(make_int4(f, i, -2, 0));
                for (int j = sp + 1; j < nt; j++)
                    for (int i = j; i < nt; i++) tupd.push_back(make_int4(f, i, j, 0));
            }
            c->mf_tpan_ptr[L].push_back((int)tpan.size()), c->mf_tupd_ptr[L].push_back((int)tupd.size());
        }
        launches += 1 + 2 * np + 1;
    }
    int rc;
    if ((rc = upload_vec(c, c->mf_fr, fr)) || (rc = upload_vec(c, c->mf_idx, P.idx)) || (rc = upload_vec(c, c->mf_cmap, P.cmap)) ||
        (rc = upload_vec(c, c->mf_child, P.child.empty() ? std::vector<int>(1, 0) : P.child)) || (rc = upload_vec(c, c->mf_brow, brow)) ||
        (rc = upload_vec(c, c->mf_tasm, tasm)) || (rc = upload_vec(c, c->mf_tpan, tpan.empty() ? std::vector<int2>(1) : tpan)) ||
        (rc = upload_vec(c, c->mf_tupd, tupd.empty() ? std::vector<int4>(1) : tupd)))
        return rc;
    BL_CUDA(c, c->mf_pool.alloc((size_t)std::max(pool, 1LL)));
    BL_CUDA(c, c->mf_dt.alloc((size_t)std::max(dtn, 1)));
    c->mf_smem = sizeof(double) * (size_t)maxn;
    if (c->mf_smem > 200 * 1024) return BL_GPU_ELIMIT; // (a front of more than ~4,200 nodes: its backward solve's vector)
    if (c->mf_smem > 40 * 1024) BL_CUDA(c, cudaFuncSetAttribute(k_mf_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c->mf_smem));
    c->mf = MfDev{c->mf_fr.p, c->mf_idx.p, c->mf_cmap.p, c->mf_child.p, c->mf_brow.p, c->mf_pool.p, c->mf_dt.p, c->mf_tasm.p, c->mf_tpan.p, c->mf_tupd.p};
    c->mf_level_ptr = P.level_ptr;
    c->mf_flops = P.flops;
    c->chol_launches = launches;
    return BL_GPU_OK;
}

// fem_dense_front 3 (automatic): the block-column path with its dense top chain while the frames' factorization makes
// at most this many block updates, the multifrontal one above (measured on B200: the 64 x 64 plate's 1.4 M updates
// factor in 2.3 ms a substep by block columns against 3.9 ms multifrontal; the 10k-node shell body's 12.6 M in 7.8 ms
// against 8.0 ms; beyond, the block columns' update lists and levels grow as fast as the fill)
constexpr int64_t kAutoMultifrontal = 8000000;

static int commit_fem(bl_gpu_ctx* c) {
    int NF = 0, NT = 0, NB = 0, NC = 0, NS = 0, nfem_nodes = 0;
    for (const HostBody& hb : c->bodies)
        if (hb.fem) NF += (int)hb.fem->node.size(), NT += (int)hb.fem->tn.size(), NB += (int)hb.fem->row.size(), NC += hb.fem->ncomp,
                    NS += (int)hb.sections.size(), nfem_nodes += hb.rec.nnodes;
    c->NF = NF, c->NT = NT, c->NB = NB, c->n_fem_nodes = nfem_nodes, c->any_plastic = false, c->any_plastic_members = false;
    c->fem_ground = false;
    c->lvl_grp_ptr.clear(), c->lvl_col_ptr.clear();
    std::vector<float4> ext(c->any_ext ? c->N : 0, make_float4(0, 0, 0, 0));
    for (const HostBody& hb : c->bodies)
        if (!hb.ext.empty())
            for (int i = 0; i < hb.rec.nnodes; i++) ext[hb.rec.node0 + i] = hb.ext[i];
    int rc;
    if ((rc = upload_vec(c, c->ext, ext))) return rc;
    if (NF == 0) {
        c->fd = FemDev{};
        return BL_GPU_OK;
    }
    std::vector<int> fnode(NF), fbody(NF), perm(NF), iperm(NF), col_ptr(NF + 1, 0), row(NB), col_comp(NF), gdiag_ptr(NF + 1, 0), goff_ptr(NB + 1, 0);
    std::vector<int> fem_nodes, fslot(c->N, -1), level(NF, 0);
    std::vector<double> xd(3 * (size_t)NF), ch2(NF), chd(NF);
    std::vector<float4> q(NF), w(NF), tr0(3 * (size_t)NT);
    std::vector<float> inertia(NF), tX(6 * (size_t)NT), tk(162 * (size_t)NT), tb(54 * (size_t)NT), tX0(6 * (size_t)NT), th0(9 * (size_t)NT), tdmg(NT);
    std::vector<int4> tn(NT), goff;
    std::vector<int2> gdiag;
    std::vector<uint8_t> tbroken(NT);
    std::vector<FemSecDev> sec;
    std::vector<std::array<int, 3>> gupd; // every update (global): target, pj, pi - in the reference's order
    std::vector<int> upd_col;             // ... and its source column
    int fo = 0, to = 0, bo = 0, co = 0, so = 0, mo = 0, mso = 0;
    std::vector<int2> mnv;                // members: frame nodes, meta, rest length, rest frames; their sections
    std::vector<int> mmeta;
    std::vector<float> mL0;
    std::vector<float4> mqv, mpsv;
    std::vector<uint32_t> mflagv;
    std::vector<FemMemSecDev> msecv;
    std::vector<int> comp_size, body_comp(c->B + 1, 0);
    std::vector<float> credit(c->B, 8.0f);
    std::vector<int> elastic(c->B, 0);
    for (int bi = 0; bi < c->B; bi++) {
        const HostBody& hb = c->bodies[bi];
        if (!hb.fem) continue;
        const FemModel& M = *hb.fem;
        const int nf = (int)M.node.size(), nt = (int)M.tn.size(), nb = (int)M.row.size();
        // (a section yields where the body deforms: eval_tris' s.yield > 0 and eval_forces' s.Np > 0, with allow_deform)
        const int plastic = (hb.beam_bits & BB_DEFORM) ? 1 : 0;
        for (int i = 0; i < hb.rec.nnodes; i++) fem_nodes.push_back(hb.rec.node0 + i), c->fem_ground |= (hb.info[i].flags & BL_NF_GROUND) != 0;
        const float dt = c->cfg.dt;
        const double h2 = (double)hb.theta * dt * dt, hd = (double)hb.diss * dt * dt;
        for (int i = 0; i < nf; i++) {
            fnode[fo + i] = hb.rec.node0 + (int)M.node[i];
            fslot[hb.rec.node0 + M.node[i]] = fo + i;
            fbody[fo + i] = bi;
            perm[fo + i] = fo + M.perm[i];
            iperm[fo + i] = fo + M.iperm[i];
            for (int j = 0; j < 3; j++) xd[3 * (size_t)(fo + i) + j] = M.xd[3 * i + j];
            q[fo + i] = make_float4(hb.fq[4 * i], hb.fq[4 * i + 1], hb.fq[4 * i + 2], hb.fq[4 * i + 3]);
            w[fo + i] = make_float4(hb.fw[3 * i], hb.fw[3 * i + 1], hb.fw[3 * i + 2], 0.0f);
            inertia[fo + i] = M.inertia[i];
            ch2[fo + i] = h2, chd[fo + i] = hd;
        }
        for (int k = 0; k < nf; k++) {
            col_ptr[fo + k + 1] = bo + M.col_ptr[k + 1];
            gdiag_ptr[fo + k + 1] = (int)gdiag.size() + (M.gdiag_ptr[k + 1] - M.gdiag_ptr[0]);
        }
        for (const auto& g : M.gdiag) gdiag.push_back(make_int2(g[0] < 0 ? g[0] - mo : to + g[0], g[1])); // (members: -(member + 1))
        for (int pb = 0; pb < nb; pb++) {
            row[bo + pb] = fo + M.row[pb];
            goff_ptr[bo + pb + 1] = (int)goff.size() + (M.goff_ptr[pb + 1] - M.goff_ptr[0]);
        }
        for (const auto& g : M.goff) goff.push_back(make_int4(g[0] < 0 ? g[0] - mo : to + g[0], g[1], g[2], 0));
        for (size_t e = 0; e < M.mn.size(); e++) {
            mnv.push_back(make_int2(fo + M.mn[e][0], fo + M.mn[e][1]));
            mmeta.push_back(M.mbroken[e] ? -1 : (int)((mso + M.msec[e]) | (M.mend[2 * e] << 16) | (M.mend[2 * e + 1] << 24)));
            mL0.push_back(M.mL0[e]);
            mqv.push_back(make_float4(M.mq[8 * e], M.mq[8 * e + 1], M.mq[8 * e + 2], M.mq[8 * e + 3]));
            mqv.push_back(make_float4(M.mq[8 * e + 4], M.mq[8 * e + 5], M.mq[8 * e + 6], M.mq[8 * e + 7]));
            const bool st = M.mps.size() == 16 * M.mn.size();
            for (int k = 0; k < 4; k++)
                mpsv.push_back(st ? make_float4(M.mps[16 * e + 4 * k], M.mps[16 * e + 4 * k + 1], M.mps[16 * e + 4 * k + 2], M.mps[16 * e + 4 * k + 3])
                                  : make_float4(0, 0, 0, 0));
            mflagv.push_back(M.mflag.size() == M.mn.size() ? M.mflag[e] : 0u);
        }
        credit[bi] = hb.repass_credit, elastic[bi] = hb.elastic_step;
        for (const FrameSectionH& fs : hb.fsections) // (it yields on a body that deforms: eval_forces' s.Np > 0 && allow_deform)
            msecv.push_back(FemMemSecDev{fs.E, fs.G, fs.rho, fs.A, fs.Iy, fs.Iz, fs.J, fs.As_y, fs.As_z, fs.damping, fs.axial, fs.joint_k,
                                         fs.Np, fs.Mp, fs.Tp, fs.hardening, fs.Np > 0 ? plastic : 0}),
                c->any_plastic_members |= fs.Np > 0 && plastic;
        for (int cc = 0; cc < M.ncomp; cc++) {
            for (int k = M.comp_first[cc]; k < M.comp_first[cc + 1]; k++) col_comp[fo + k] = co + cc;
            comp_size.push_back(M.comp_first[cc + 1] - M.comp_first[cc]);
        }
        for (int t = 0; t < nt; t++) {
            tn[to + t] = make_int4(fo + M.tn[t][0], fo + M.tn[t][1], fo + M.tn[t][2], so + M.tsec[t]);
            for (int x = 0; x < 6; x++) tX[6 * (size_t)(to + t) + x] = M.tX[6 * t + x];
            for (int i = 0; i < 3; i++) tr0[3 * (size_t)(to + t) + i] = make_float4(M.tr0[12 * t + 4 * i], M.tr0[12 * t + 4 * i + 1], M.tr0[12 * t + 4 * i + 2], M.tr0[12 * t + 4 * i + 3]);
            for (int x = 0; x < 162; x++) tk[162 * (size_t)(to + t) + x] = M.tk[162 * t + x];
            for (int x = 0; x < 54; x++) tb[54 * (size_t)(to + t) + x] = M.tb[54 * t + x];
            for (int x = 0; x < 6; x++) tX0[6 * (size_t)(to + t) + x] = M.tX0[6 * t + x];
            for (int x = 0; x < 9; x++) th0[9 * (size_t)(to + t) + x] = M.th0[9 * t + x];
            tdmg[to + t] = M.tdmg[t];
            tbroken[to + t] = M.tbroken[t];
        }
        for (const FemSection& fs : hb.sections)
            sec.push_back(FemSecDev{fs.E, fs.nu, fs.rho, fs.t, fs.damping, fs.drill, fs.yield, fs.yield > 0 ? plastic : 0}),
                c->any_plastic |= fs.yield > 0 && plastic;
        for (int k = 0; k < nf; k++)
            for (int u = M.upd_ptr[k]; u < M.upd_ptr[k + 1]; u++) {
                const auto& up = M.upd[u];
                gupd.push_back({up[2] >= 0 ? NF + bo + up[2] : fo + (-up[2] - 1), bo + up[1], bo + up[0]});
                upd_col.push_back(fo + k);
            }
        // levels: a column's level one more than its deepest child's (its parent: the first row below its diagonal)
        for (int k = 0; k < nf; k++) {
            if (M.col_ptr[k + 1] == M.col_ptr[k]) continue;
            int par = M.row[M.col_ptr[k]];
            for (int pb = M.col_ptr[k]; pb < M.col_ptr[k + 1]; pb++) par = std::min(par, M.row[pb]);
            level[fo + par] = std::max(level[fo + par], level[fo + k] + 1);
        }
        fo += nf, to += nt, bo += nb, co += M.ncomp, so += (int)hb.sections.size();
        body_comp[bi + 1] = co;
        mo += (int)M.mn.size(), mso += (int)hb.fsections.size();
    }
    for (int bi = 0; bi < c->B; bi++) body_comp[bi + 1] = std::max(body_comp[bi + 1], body_comp[bi]);
    int nlev = 0;
    for (int k = 0; k < NF; k++) nlev = std::max(nlev, level[k] + 1);
    // per level: its columns, and the updates they make grouped by target (each group in the order of its columns)
    std::vector<int> lvl_col, grp_tgt, grp_ptr(1, 0);
    std::vector<int2> gu, rbv;
    std::vector<int> rb_ptr(NF + 1, 0);
    std::vector<std::vector<int>> bylev(nlev);
    for (int k = 0; k < NF; k++) bylev[level[k]].push_back(k);
    c->NU = 0; // (the pattern's block updates, whether or not their list was built: sum over columns of d (d + 1) / 2)
    for (int k = 0; k < NF; k++) c->NU += (int64_t)(col_ptr[k + 1] - col_ptr[k]) * (col_ptr[k + 1] - col_ptr[k] + 1) / 2;
    if (c->cfg.fem_dense_front == 3) {
        bool lists = c->NU <= kAutoMultifrontal;
        for (const HostBody& hb : c->bodies)
            if (hb.fem && fem_update_count(*hb.fem) > 0 && hb.fem->upd.empty()) lists = false;
        c->fem_mode = lists ? 1 : 2;
    } else {
        c->fem_mode = c->cfg.fem_dense_front;
    }
    std::vector<std::vector<int>> col_upds(NF);
    for (size_t u = 0; u < gupd.size(); u++) col_upds[upd_col[u]].push_back((int)u);
    c->lvl_grp_ptr.assign(1, 0), c->lvl_col_ptr.assign(1, 0);
    std::vector<int> slot_of(NF + NB, -1);
    for (int L = 0; L < nlev; L++) {
        std::vector<int> tg;                     // the level's targets, in order of first appearance
        std::vector<std::vector<int2>> lists;
        for (int k : bylev[L]) {
            lvl_col.push_back(k);
            for (int u : col_upds[k]) {
                const int t = gupd[u][0];
                if (slot_of[t] < 0) slot_of[t] = (int)tg.size(), tg.push_back(t), lists.emplace_back();
                lists[slot_of[t]].push_back(make_int2(gupd[u][1], gupd[u][2]));
            }
        }
        for (size_t x = 0; x < tg.size(); x++) {
            grp_tgt.push_back(tg[x]);
            gu.insert(gu.end(), lists[x].begin(), lists[x].end());
            grp_ptr.push_back((int)gu.size());
            slot_of[tg[x]] = -1;
        }
        c->lvl_grp_ptr.push_back((int)grp_tgt.size());
        c->lvl_col_ptr.push_back((int)lvl_col.size());
    }
    // begin, triangles, assembly, per level a factor kernel, an update + forward kernel and a backward kernel,
    // velocities, integration
    {   // each row's blocks in the order of their columns
        std::vector<std::vector<int2>> rows(NF);
        for (int k = 0; k < NF; k++)
            for (int pb = col_ptr[k]; pb < col_ptr[k + 1]; pb++) rows[row[pb]].push_back(make_int2(pb, k));
        for (int r = 0; r < NF; r++) {
            rb_ptr[r + 1] = rb_ptr[r] + (int)rows[r].size();
            rbv.insert(rbv.end(), rows[r].begin(), rows[r].end());
        }
    }
    std::vector<int> zeros_nf(NF, 0), zeros_b(c->B, 0), zeros_c(NC, 0);
    for (int bi = 0; bi < c->B; bi++) zeros_b[bi] = c->bodies[bi].fem_failures;
    std::vector<int> clamps_b(c->B);
    for (int bi = 0; bi < c->B; bi++) clamps_b[bi] = c->bodies[bi].fem_clamps;
    std::vector<float4> zero4(NF, make_float4(0, 0, 0, 0));
    if ((rc = upload_vec(c, c->fnode, fnode)) || (rc = upload_vec(c, c->fbody, fbody)) || (rc = upload_vec(c, c->fperm, perm)) ||
        (rc = upload_vec(c, c->fiperm, iperm)) || (rc = upload_vec(c, c->xd, xd)) || (rc = upload_vec(c, c->fq, q)) || (rc = upload_vec(c, c->fw, w)) ||
        (rc = upload_vec(c, c->finertia, inertia)) || (rc = upload_vec(c, c->ftorque, zero4)) || (rc = upload_vec(c, c->tn, tn)) ||
        (rc = upload_vec(c, c->tX, tX)) || (rc = upload_vec(c, c->tr0, tr0)) || (rc = upload_vec(c, c->tk, tk)) || (rc = upload_vec(c, c->tb, tb)) ||
        (rc = upload_vec(c, c->tX0, tX0)) || (rc = upload_vec(c, c->th0, th0)) || (rc = upload_vec(c, c->tdmg, tdmg)) || (rc = upload_vec(c, c->tbroken, tbroken)) ||
        (rc = upload_vec(c, c->fsec, sec)) || (rc = upload_vec(c, c->fcol_ptr, col_ptr)) || (rc = upload_vec(c, c->frow, row)) ||
        (rc = upload_vec(c, c->gdiag_ptr, gdiag_ptr)) || (rc = upload_vec(c, c->gdiag, gdiag)) || (rc = upload_vec(c, c->goff_ptr, goff_ptr)) ||
        (rc = upload_vec(c, c->goff, goff)) || (rc = upload_vec(c, c->grp_tgt, grp_tgt)) || (rc = upload_vec(c, c->grp_ptr, grp_ptr)) ||
        (rc = upload_vec(c, c->gu, gu)) || (rc = upload_vec(c, c->col_comp, col_comp)) || (rc = upload_vec(c, c->comp_fail, zeros_c)) || (rc = upload_vec(c, c->rb_ptr, rb_ptr)) ||
        (rc = upload_vec(c, c->rb, rbv)) || (rc = upload_vec(c, c->lvl_col, lvl_col)) || (rc = upload_vec(c, c->ch2, ch2)) ||
        (rc = upload_vec(c, c->chd, chd)) || (rc = upload_vec(c, c->fem_fail, zeros_b)) || (rc = upload_vec(c, c->fem_clamp, clamps_b)) ||
        (rc = upload_vec(c, c->fem_nodes, fem_nodes)) || (rc = upload_vec(c, c->fslot, fslot)))
        return rc;
    {
        std::vector<int> blk_col(std::max(NB, 1), 0);
        for (int k = 0; k < NF; k++)
            for (int pb = col_ptr[k]; pb < col_ptr[k + 1]; pb++) blk_col[pb] = k;
        if ((rc = upload_vec(c, c->fblk_col, blk_col))) return rc;
    }
    BL_CUDA(c, c->nforce.alloc(c->N));
    BL_CUDA(c, c->tf.alloc(3 * (size_t)NT));
    BL_CUDA(c, c->tt.alloc(3 * (size_t)NT));
    BL_CUDA(c, c->ttan.alloc(18 * (size_t)NT));
    BL_CUDA(c, c->tkv.alloc(18 * (size_t)NT));
    BL_CUDA(c, c->ton.alloc(NT));
    BL_CUDA(c, c->diag.alloc(36 * (size_t)NF));
    BL_CUDA(c, c->off.alloc(36 * (size_t)std::max(NB, 1)));
    BL_CUDA(c, c->rhs.alloc(6 * (size_t)NF));
    BL_CUDA(c, c->dinv.alloc(6 * (size_t)NF));
    BL_CUDA(c, c->ffixed.alloc(NF));
    BL_CUDA(c, cudaMemsetAsync(c->ton.p, 0, NT, c->stream));
    FemDev& F = c->fd;
    F.nf = NF, F.ntri = NT, F.nblk = NB;
    F.fnode = c->fnode.p, F.fbody = c->fbody.p, F.perm = c->fperm.p, F.iperm = c->fiperm.p, F.xd = c->xd.p, F.q = c->fq.p, F.w = c->fw.p;
    F.inertia = c->finertia.p, F.torque = c->ftorque.p, F.tn = c->tn.p, F.tX = c->tX.p, F.tr0 = c->tr0.p, F.tk = c->tk.p,
          F.tb = c->tb.p, F.tX0 = c->tX0.p, F.th0 = c->th0.p, F.tdmg = c->tdmg.p, F.tbroken = c->tbroken.p;
    F.tf = c->tf.p, F.tt = c->tt.p, F.ttan = c->ttan.p, F.tkv = c->tkv.p, F.ton = c->ton.p, F.sec = c->fsec.p, F.col_ptr = c->fcol_ptr.p, F.row = c->frow.p;
    F.blk_col = c->fblk_col.p;
    F.gdiag_ptr = c->gdiag_ptr.p, F.gdiag = c->gdiag.p, F.goff_ptr = c->goff_ptr.p, F.goff = c->goff.p, F.diag = c->diag.p, F.off = c->off.p;
    F.rhs = c->rhs.p, F.dinv = c->dinv.p, F.fixed = c->ffixed.p, F.grp_tgt = c->grp_tgt.p, F.grp_ptr = c->grp_ptr.p, F.gu = c->gu.p;
    F.col_comp = c->col_comp.p, F.comp_fail = c->comp_fail.p, F.rb_ptr = c->rb_ptr.p;
    F.rb = c->rb.p, F.lvl_col = c->lvl_col.p, F.ch2 = c->ch2.p, F.chd = c->chd.p, F.body_failures = c->fem_fail.p, F.body_clamps = c->fem_clamp.p;
    F.h = c->cfg.dt, F.step = c->cfg.dt;
    c->lvl_ns.assign(std::max<size_t>(c->lvl_col_ptr.size(), 1) - 1, 1);
    for (size_t L = 0; L + 1 < c->lvl_col_ptr.size(); L++)
        for (int ci = c->lvl_col_ptr[L]; ci < c->lvl_col_ptr[L + 1]; ci++) {
            const int k = lvl_col[ci];
            c->lvl_ns[L] = std::max(c->lvl_ns[L], (6 * (col_ptr[k + 1] - col_ptr[k]) + kUnit - 1) / kUnit);
        }
    BL_CUDA(c, c->ldiag.alloc(36 * (size_t)NF));
    F.ldiag = c->ldiag.p;
    F.contact_n = nullptr;
    if (c->fem_ground) {
        BL_CUDA(c, c->contact_n.alloc(NF));
        F.contact_n = c->contact_n.p;
    }
    {   // the members
        const int E = (int)mnv.size();
        if ((rc = upload_vec(c, c->mn, mnv)) || (rc = upload_vec(c, c->mmeta, mmeta)) || (rc = upload_vec(c, c->mL0, mL0)) ||
            (rc = upload_vec(c, c->mq, mqv)) || (rc = upload_vec(c, c->msec, msecv)))
            return rc;
        BL_CUDA(c, c->mfa.alloc(E));
        BL_CUDA(c, c->mta.alloc(E));
        BL_CUDA(c, c->mtb.alloc(E));
        BL_CUDA(c, c->mtan.alloc(E));
        BL_CUDA(c, c->mon.alloc(E));
        BL_CUDA(c, c->mkw.alloc(144 * (size_t)E));
        BL_CUDA(c, c->mkv.alloc(12 * (size_t)E));
        BL_CUDA(c, cudaMemsetAsync(c->mon.p, 0, std::max(E, 1), c->stream));
        F.nmem = E, F.mn = c->mn.p, F.mmeta = c->mmeta.p, F.mL0 = c->mL0.p, F.mq = c->mq.p, F.msec = c->msec.p;
        F.mfa = c->mfa.p, F.mta = c->mta.p, F.mtb = c->mtb.p, F.mon = c->mon.p, F.mtan = c->mtan.p, F.mkw = c->mkw.p, F.mkv = c->mkv.p;
        c->NM = E;
        if (c->any_plastic_members) { // (the members' plastic state, their tangents, the re-passes' budget)
            std::vector<int> rp(2, 0);
            if ((rc = upload_vec(c, c->mps, mpsv)) || (rc = upload_vec(c, c->mflag, mflagv)) || (rc = upload_vec(c, c->credit, credit)) ||
                (rc = upload_vec(c, c->elastic, elastic)) || (rc = upload_vec(c, c->comp_again, zeros_c)) ||
                (rc = upload_vec(c, c->comp_size, comp_size)) || (rc = upload_vec(c, c->body_comp, body_comp)) || (rc = upload_vec(c, c->rp, rp)) ||
                (rc = upload_vec(c, c->repc, std::vector<long long>(1, 0))))
                return rc;
            BL_CUDA(c, c->mtg.alloc(6 * (size_t)E));
            F.mps = c->mps.p, F.mtg = c->mtg.p, F.mflag = c->mflag.p, F.credit = c->credit.p, F.elastic = c->elastic.p;
            F.comp_again = c->comp_again.p, F.comp_size = c->comp_size.p, F.body_comp = c->body_comp.p, F.rp = c->rp.p, F.nbody = c->B;
            F.repc = c->repc.p;
        }
    }
    {   // the top chain (the levels from front_level up have one column each) as one dense front, when every row of
        // its columns is a chain column and it is long enough to pay
        const int nlev = (int)c->lvl_col_ptr.size() - 1;
        int top = nlev;
        while (top > 0 && c->lvl_col_ptr[top] - c->lvl_col_ptr[top - 1] == 1) top--;
        const int m = c->fem_mode == 1 ? nlev - top : 0;
        std::vector<int> chain(NF, -1), fcol;
        std::vector<int4> fblk;
        bool closed = m >= kFrontMin && 6 * m <= 8192; // (D at most 512 MB, its solve's vector in shared memory)
        for (int x = 0; closed && x < m; x++) fcol.push_back(lvl_col[c->lvl_col_ptr[top + x]]), chain[fcol.back()] = x;
        for (int x = 0; closed && x < m; x++) {
            const int k = fcol[x];
            for (int pb = col_ptr[k]; pb < col_ptr[k + 1]; pb++) {
                if (chain[row[pb]] < 0) closed = false;
                else fblk.push_back(make_int4(pb, chain[row[pb]], x, 0));
            }
        }
        c->front_level = nlev;
        c->front = FrontDev{};
        if (closed) {
            FrontDev& X = c->front;
            X.m = m, X.nt = (6 * m + kFT - 1) / kFT, X.N = kFT * X.nt, X.nblk = (int)fblk.size();
            if ((rc = upload_vec(c, c->fcol, fcol)) || (rc = upload_vec(c, c->fblk, fblk)) || (rc = upload_vec(c, c->fchain, chain))) return rc;
            BL_CUDA(c, c->fD.alloc((size_t)X.N * X.N));
            BL_CUDA(c, c->fb.alloc((size_t)X.N));
            X.col = c->fcol.p, X.blk = c->fblk.p, X.chain = c->fchain.p, X.D = c->fD.p, X.b = c->fb.p;
            if ((size_t)X.N * sizeof(double) > 48 * 1024)
                BL_CUDA(c, cudaFuncSetAttribute(k_front_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(X.N * sizeof(double))));
            c->front_level = top;
        }
        c->chol_launches = 3 * (int64_t)c->front_level;
        if (c->front_level < nlev) c->chol_launches += 1 + c->front.nt + 2 * (c->front.nt - 1) + 2;
        if (c->fem_mode == 2 && (rc = commit_multifrontal(c, col_ptr, row, col_comp))) return rc;
        c->fem_launches = 4 + (c->NT > 0 ? 1 : 0) + (c->NM > 0 ? 1 : 0) + c->chol_launches; // (begin, triangles, members, assembly, velocity, integration)
    }
    // PCG: vectors, block-Jacobi factors, the grid's partial sums (one cooperative launch: as many blocks as fit)
    for (DevBuf<double>* d : {&c->px, &c->pr, &c->pz, &c->pp, &c->ppdi}) BL_CUDA(c, d->alloc(6 * (size_t)NF));
    BL_CUDA(c, c->ppf.alloc(36 * (size_t)NF));
    int per_sm = 0, nsm = 0, dev = c->cfg.device;
    BL_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fem_pcg, 256, 0));
    BL_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    c->pcg_grid = std::max(1, std::min(per_sm * nsm, (NF + 7) / 8));
    BL_CUDA(c, c->pred.alloc(2 * 8 * (size_t)c->pcg_grid * 8)); // (two buffers, 8 sums a warp, 8 warps a block)
    BL_CUDA(c, c->pxprev.alloc(6 * (size_t)NF));
    BL_CUDA(c, cudaMemsetAsync(c->pxprev.p, 0, sizeof(double) * 6 * NF, c->stream));
    BL_CUDA(c, c->pstat.alloc(4));
    BL_CUDA(c, c->piters.alloc(1));
    BL_CUDA(c, c->plast.alloc(1));
    BL_CUDA(c, c->res.alloc(4));
    BL_CUDA(c, cudaMemsetAsync(c->pstat.p, 0, 4 * sizeof(int), c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->piters.p, 0, sizeof(long long), c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->plast.p, 0, sizeof(double), c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->res.p, 0, 4 * sizeof(double), c->stream));
    if (c->cfg.fem_check_residual) {
        BL_CUDA(c, c->a0d.alloc(36 * (size_t)NF));
        BL_CUDA(c, c->a0o.alloc(36 * (size_t)std::max(NB, 1)));
        BL_CUDA(c, c->b0.alloc(6 * (size_t)NF));
    }
    BL_CUDA(c, c->guess.alloc(3 * (size_t)NF));
    BL_CUDA(c, c->gscale.alloc(9 * (size_t)NF));
    {   // each frame node's 1-ring (the frame nodes it shares a triangle with), ascending: the network's neighbourhood
        std::vector<std::vector<int>> nb(NF);
        for (const int4& t : tn) {
            const int v[3] = {t.x, t.y, t.z};
            for (int a = 0; a < 3; a++)
                for (int b2 = 0; b2 < 3; b2++)
                    if (a != b2) nb[v[a]].push_back(v[b2]);
        }
        std::vector<int> aptr(NF + 1, 0), av;
        for (int i = 0; i < NF; i++) {
            std::sort(nb[i].begin(), nb[i].end());
            nb[i].erase(std::unique(nb[i].begin(), nb[i].end()), nb[i].end());
            av.insert(av.end(), nb[i].begin(), nb[i].end());
            aptr[i + 1] = (int)av.size();
        }
        if ((rc = upload_vec(c, c->adj_ptr, aptr)) || (rc = upload_vec(c, c->adj, av))) return rc;
    }
    BL_CUDA(c, c->feat.alloc((size_t)kIn * NF));
    BL_CUDA(c, c->prev_dv.alloc(3 * (size_t)NF));
    BL_CUDA(c, cudaMemsetAsync(c->prev_dv.p, 0, sizeof(float) * 3 * NF, c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->guess.p, 0, sizeof(float) * 3 * NF, c->stream));
    {
        std::vector<float> eye(9 * (size_t)NF, 0.0f);
        for (int i = 0; i < NF; i++) eye[9 * i] = eye[9 * i + 4] = eye[9 * i + 8] = 1.0f;
        BL_CUDA(c, cudaMemcpyAsync(c->gscale.p, eye.data(), sizeof(float) * eye.size(), cudaMemcpyHostToDevice, c->stream));
        BL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    return BL_GPU_OK;
}

// Lays every body out back to back on the device and builds each node's incident-beam list.
// The collision triangles of all bodies back to back and the contacts' scratch (bl_contacts.cuh), when some body has
// triangles and the world collides bodies.
static int commit_contacts(bl_gpu_ctx* c, std::vector<Body>& recs) {
    free_contacts(c);
    int T = 0;
    for (int bi = 0; bi < c->B; bi++) recs[bi].tri0 = T, recs[bi].ntris = (int)c->bodies[bi].tris.size(), T += recs[bi].ntris;
    c->NTRI = T;
    c->contacts_on = T > 0 && c->cfg.inter_body_collisions != 0;
    if (!c->contacts_on) {
        for (Body& r : recs) r.island = -1, r.pairs = 0;
        return BL_GPU_OK;
    }
    std::vector<int4> tri(T);
    std::vector<float> rest2(T);
    for (int bi = 0; bi < c->B; bi++) {
        const HostBody& hb = c->bodies[bi];
        const int n0 = recs[bi].node0;
        for (int t = 0; t < recs[bi].ntris; t++) {
            const bl_tri& x = hb.tris[t];
            const int fl = (x.two_sided ? (int)TF_TWO_SIDED : 0) | (x.torn ? (int)TF_TORN : 0) | (bi << 8);
            tri[recs[bi].tri0 + t] = make_int4(n0 + (int)x.a, n0 + (int)x.b, n0 + (int)x.c, fl);
            rest2[recs[bi].tri0 + t] = x.rest_edge2;
        }
    }
    const int N = c->N, B = c->B;
    c->max_isl = B / 2 + 1; // (an island with pairs holds two bodies or more)
    int rc;
    if ((rc = upload_vec(c, c->dtri, tri)) || (rc = upload_vec(c, c->tri_rest2, rest2))) return rc;
    BL_CUDA(c, c->ibox.alloc(6 * (size_t)B));
    for (DevBuf<int>* d : {&c->parent, &c->isl_live, &c->isl_cnt, &c->isl_nodes, &c->isl_idx, &c->isl_noff, &c->isl_poff, &c->isl_pcnt, &c->isl_contacts})
        BL_CUDA(c, d->alloc(B));
    BL_CUDA(c, c->pair_total.alloc(1));
    BL_CUDA(c, c->counters.alloc(4));
    BL_CUDA(c, cudaFuncSetAttribute(k_collide, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kCollideSmem));
    BL_CUDA(c, c->pairs.alloc(c->cfg.max_pairs));
    BL_CUDA(c, c->hit_a.alloc(c->cfg.max_pairs));
    BL_CUDA(c, c->hit_b.alloc(c->cfg.max_pairs));
    BL_CUDA(c, c->hbits.alloc((size_t)c->cfg.max_pairs / 32 + 1));
    BL_CUDA(c, c->hidx.alloc(c->cfg.max_pairs));
    const int crec_cap = std::max(c->cfg.max_pairs / 4, 65536);
    BL_CUDA(c, c->crec.alloc(crec_cap));
    BL_CUDA(c, c->crec_n.alloc(1));
    BL_CUDA(c, cudaMemsetAsync(c->crec_n.p, 0, sizeof(int), c->stream));
    for (DevBuf<int>* d : {&c->pt_node, &c->pt_body, &c->bk_items, &c->run_end}) BL_CUDA(c, d->alloc(N));
    BL_CUDA(c, c->pt_cell.alloc(N));
    BL_CUDA(c, c->bk_start.alloc(4 * (size_t)N + 65 * (size_t)B + 1));
    BL_CUDA(c, c->bk_fill.alloc(4 * (size_t)N + 65 * (size_t)B + 1));
    // (fast grids: the starts of every fast body's cells from one pool, the fill counters one grid per island)
    const int cell_cap = std::min(B, 512) * (kGridCells + 1);
    BL_CUDA(c, c->g_start.alloc((size_t)cell_cap));
    BL_CUDA(c, c->g_fill.alloc((size_t)c->max_isl * (kGridCells + 1)));
    BL_CUDA(c, c->g_items.alloc(N));
    BL_CUDA(c, c->g_rec.alloc(N));
    BL_CUDA(c, c->g_hi.alloc(N));
    BL_CUDA(c, c->sb_cell.alloc(N));
    BL_CUDA(c, c->sb_pos.alloc(N));
    // queries: a triangle against a hash or a grid; a full list flags DEVERR_PAIRS
    const int q_cap = std::max(8 * std::max(c->NTRI, 1) + 65536, c->cfg.max_pairs), grp_cap = B * std::min(B, kIslMaxBodies) + B, chunk_cap = grp_cap + q_cap / kQueryChunk;
    BL_CUDA(c, c->isl.alloc(c->max_isl));
    BL_CUDA(c, c->q_count.alloc(q_cap));
    BL_CUDA(c, c->q_group.alloc(grp_cap));
    BL_CUDA(c, c->q_chunk.alloc(chunk_cap));
    BL_CUDA(c, c->q_tmp.alloc(q_cap));
    BL_CUDA(c, c->ptmp.alloc(c->cfg.max_pairs));
    BL_CUDA(c, c->sc.alloc(8));
    BL_CUDA(c, cudaMemsetAsync(c->sc.p, 0, 8 * sizeof(int), c->stream));
    BL_CUDA(c, cudaFuncSetAttribute(k_rebuild, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(RebuildShared)));
    // (the pair list starts as valid indices: k_detect reads up to the last search's total)
    BL_CUDA(c, cudaMemsetAsync(c->pairs.p, 0, sizeof(int2) * c->cfg.max_pairs, c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->pair_total.p, 0, sizeof(int), c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->counters.p, 0, 4 * sizeof(int), c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->isl_pcnt.p, 0, sizeof(int) * B, c->stream));
    BL_CUDA(c, cudaMemsetAsync(c->isl_contacts.p, 0, sizeof(int) * B, c->stream));
    const double hz = std::max(1.0f, c->cfg.collision_hz);
    c->interval = std::max(1, (int)std::ceil(1.0 / (hz * (double)c->cfg.dt) - 1e-6)); // (world.cpp:1887)
    Contacts& C = c->ct;
    C.tri = c->dtri.p, C.tri_rest2 = c->tri_rest2.p, C.parent = c->parent.p, C.ibox = c->ibox.p;
    C.isl_live = c->isl_live.p, C.isl_cnt = c->isl_cnt.p, C.isl_nodes = c->isl_nodes.p, C.isl_idx = c->isl_idx.p;
    C.isl_noff = c->isl_noff.p, C.isl_poff = c->isl_poff.p, C.isl_pcnt = c->isl_pcnt.p, C.isl_contacts = c->isl_contacts.p;
    C.pair_total = c->pair_total.p, C.pairs = c->pairs.p, C.hit_a = c->hit_a.p, C.hit_b = c->hit_b.p, C.max_pairs = c->cfg.max_pairs;
    C.pt_node = c->pt_node.p, C.pt_body = c->pt_body.p, C.pt_cell = c->pt_cell.p, C.bk_start = c->bk_start.p, C.bk_fill = c->bk_fill.p;
    C.bk_items = c->bk_items.p, C.run_end = c->run_end.p, C.g_start = c->g_start.p, C.g_fill = c->g_fill.p, C.g_items = c->g_items.p;
    C.g_rec = c->g_rec.p, C.g_hi = c->g_hi.p, C.sb_cell = c->sb_cell.p, C.sb_pos = c->sb_pos.p, C.isl = c->isl.p;
    C.q_group = c->q_group.p, C.q_chunk = c->q_chunk.p, C.q_count = c->q_count.p, C.sc = c->sc.p;
    C.ptmp = c->ptmp.p, C.q_tmp = c->q_tmp.p, C.ptmp_cap = c->cfg.max_pairs;
    C.hbits = c->hbits.p, C.hidx = c->hidx.p, C.crec = c->crec.p, C.crec_n = c->crec_n.p, C.crec_cap = crec_cap;
    C.whole_max = c->cfg.contact_whole_max;
    C.q_cap = q_cap, C.grp_cap = grp_cap, C.chunk_cap = chunk_cap, C.cell_cap = cell_cap;
    C.counters = c->counters.p, C.interval = c->interval, C.dt = c->cfg.dt, C.wake_speed = c->cfg.sleep_speed;
    return BL_GPU_OK;
}

static int commit_bodies(bl_gpu_ctx* c) {
    int rc = pull_state(c);
    if (rc) return rc;
    int N = 0, M = 0, maxn = 1;
    for (HostBody& hb : c->bodies) {
        hb.rec.node0 = N, hb.rec.nnodes = (int)hb.nodes.size(), hb.rec.beam0 = M, hb.rec.nbeams = (int)hb.beams.size();
        N += hb.rec.nnodes, M += hb.rec.nbeams, maxn = std::max(maxn, hb.rec.nnodes);
    }
    const int B = (int)c->bodies.size();
    std::vector<bl_node> nodes(N);
    std::vector<float4> bst(M), bcold(M);
    std::vector<int4> info(N);
    std::vector<int2> ab(M);
    std::vector<float2> kd(M);
    std::vector<uint32_t> meta(M);
    std::vector<float> stress(M);
    std::vector<int> bbody(M), inc_ptr(N + 1, 0), inc(2 * (size_t)M);
    std::vector<Body> recs(B);
    for (int bi = 0; bi < B; bi++) {
        const HostBody& hb = c->bodies[bi];
        const Body& r = hb.rec;
        recs[bi] = r;
        for (int i = 0; i < r.nnodes; i++) {
            const bl_node& n = hb.nodes[i];
            const bl_node_info& f = hb.info[i];
            nodes[r.node0 + i] = n;
            int fr, ra;
            std::memcpy(&fr, &f.friction, 4), std::memcpy(&ra, &f.radius, 4);
            info[r.node0 + i] = make_int4((int)f.flags, fr, ra, bi);
        }
        for (int j = 0; j < r.nbeams; j++) {
            const bl_beam& b = hb.beams[j];
            const int g = r.beam0 + j;
            ab[g] = make_int2(r.node0 + (int)b.a, r.node0 + (int)b.b);
            kd[g] = make_float2(b.k, b.d);
            bst[g] = make_float4(b.L, b.max_pos, b.max_neg, b.strength);
            bcold[g] = make_float4(b.plastic, b.L0, b.support_limit, 0.0f);
            stress[g] = b.stress;
            bbody[g] = bi;
            inc_ptr[ab[g].x + 1]++, inc_ptr[ab[g].y + 1]++;
        }
    }
    // each beam's meta word: type, flags, the body's deform/break/ductile bits, asleep
    for (int bi = 0; bi < B; bi++) {
        const HostBody& hb = c->bodies[bi];
        const Body& r = hb.rec;
        const uint32_t bits = hb.beam_bits;
        for (int j = 0; j < r.nbeams; j++) {
            const bl_beam& b = hb.beams[j];
            meta[r.beam0 + j] = (uint32_t)b.type | ((uint32_t)b.flags << 8) | bits | (r.sleeping ? kBeamAsleep : 0u);
        }
    }
    c->any_ext = false;
    bool any_drag = false;
    for (int bi = 0; bi < B; bi++) {
        recs[bi].is_fem = c->bodies[bi].fem ? 1 : 0;
        recs[bi].has_ext = c->bodies[bi].ext.empty() ? 0 : 1;
        c->any_ext |= recs[bi].has_ext != 0;
        any_drag |= recs[bi].drag != 0;
        recs[bi].has_wheels = c->bodies[bi].wheels.empty() ? 0 : 1;
        recs[bi].has_shocks = c->bodies[bi].shocks.empty() ? 0 : 1;
    }
    free_device(c);
    c->N = N, c->M = M, c->B = B;
    if ((rc = commit_contacts(c, recs))) return rc;
    for (int i = 0; i < N; i++) inc_ptr[i + 1] += inc_ptr[i];
    {
        std::vector<int> fill(inc_ptr.begin(), inc_ptr.end() - 1);
        for (int g = 0; g < M; g++) {
            inc[fill[ab[g].x]++] = g;
            inc[fill[ab[g].y]++] = (int)((uint32_t)g | 0x80000000u);
        }
    }
    // the arrays k_beams_tma streams padded to whole tiles (the pads asleep: never stepped)
    const size_t Mpad = (size_t)(M + kBeamTile - 1) / kBeamTile * kBeamTile;
    ab.resize(Mpad, make_int2(0, 0)), kd.resize(Mpad, make_float2(0, 0)), bst.resize(Mpad, make_float4(0, 0, 0, 0)), meta.resize(Mpad, kBeamAsleep);
    c->beam_tiles = (int)(Mpad / kBeamTile);
    static_assert(sizeof(bl_node) == 2 * sizeof(float4), "bl_node is two float4");
    BL_CUDA(c, c->nd.alloc(2 * (size_t)N));
    if (N) BL_CUDA(c, cudaMemcpyAsync(c->nd.p, nodes.data(), sizeof(bl_node) * N, cudaMemcpyHostToDevice, c->stream));
    if ((rc = upload_vec(c, c->info, info)) || (rc = upload_vec(c, c->inc_ptr, inc_ptr)) ||
        (rc = upload_vec(c, c->inc, inc)) || (rc = upload_vec(c, c->ab, ab)) || (rc = upload_vec(c, c->kd, kd)) || (rc = upload_vec(c, c->bst, bst)) ||
        (rc = upload_vec(c, c->bmeta, meta)) || (rc = upload_vec(c, c->bcold, bcold)) || (rc = upload_vec(c, c->stress, stress)) ||
        (rc = upload_vec(c, c->bbody, bbody)) || (rc = upload_vec(c, c->dbodies, recs)))
        return rc;
    BL_CUDA(c, c->fsc.alloc(M));
    c->any_drag = any_drag;
    if (any_drag) { // (the parts' scratch and means: k_drag_parts)
        BL_CUDA(c, c->dup.alloc(N));
        BL_CUDA(c, c->dpid.alloc(N));
        BL_CUDA(c, c->dpart.alloc(N));
        BL_CUDA(c, c->dpmv.alloc(N));
        BL_CUDA(c, c->dpacc.alloc(N));
    }
    {   // the wheels: per wheel its hubs and its tyre nodes (ascending: the patch's sums run in node order), per node its
        // wheel and the parity of its place in the wheel's list; every other tyre node of a body without a frame a wheel
        // of its own with no hubs (a patch of one node: the same bits as its own stick test)
        std::vector<int4> wh, warm;
        std::vector<int> wn, wl;
        std::vector<int2> nw;
        std::vector<float4> wst, wctl;
        std::vector<std::vector<int2>> wterm; // per node: its wheel terms in wheel order
        for (int bi = 0; bi < B; bi++) {
            HostBody& hb = c->bodies[bi];
            hb.wheel0 = (int)wh.size();
            if (hb.fem) continue;
            const int n0 = recs[bi].node0;
            for (const HostBody::Wheel& w : hb.wheels) {
                if (nw.empty()) nw.assign(N, make_int2(-1, 0)), wterm.resize(N);
                const int first = (int)wn.size(), k = (int)wh.size();
                for (size_t j = 0; j < w.nodes.size(); j++) {
                    wn.push_back(n0 + (int)w.nodes[j]), wl.push_back(n0 + (int)w.nodes[j]);
                    nw[n0 + w.nodes[j]] = make_int2(k, (int)(j & 1));
                    wterm[n0 + w.nodes[j]].push_back(make_int2(k, (int)((j & 1) << 2)));
                }
                if (w.arm >= 0 && w.near_attach >= 0) {
                    wterm[n0 + w.arm].push_back(make_int2(k, 1));
                    wterm[n0 + w.near_attach].push_back(make_int2(k, 2));
                }
                std::sort(wn.begin() + first, wn.end());
                wh.push_back(make_int4(n0 + (int)w.axle0, n0 + (int)w.axle1, first, (int)w.nodes.size()));
                warm.push_back(make_int4(w.arm >= 0 ? n0 + w.arm : -1, w.near_attach >= 0 ? n0 + w.near_attach : -1, w.propulsed, 0));
                wst.push_back(make_float4(w.st[0], w.st[1], w.st[2], w.st[3]));
                wctl.push_back(make_float4(w.torque, w.brake, w.radius, w.mass));
            }
            for (int i = 0; i < recs[bi].nnodes; i++)
                if ((hb.info[i].flags & BL_NF_TYRE) && (nw.empty() || nw[n0 + i].x < 0)) {
                    if (nw.empty()) nw.assign(N, make_int2(-1, 0));
                    nw[n0 + i] = make_int2((int)wh.size(), 0);
                    wh.push_back(make_int4(-1, -1, (int)wn.size(), 1));
                    wn.push_back(n0 + i);
                }
        }
        c->NW = (int)wh.size(), c->NWR = (int)warm.size();
        if (c->NW > 0) {
            std::vector<int> wc_ptr(N + 1, 0);
            std::vector<int2> wc;
            for (int i = 0; i < N && !wterm.empty(); i++) {
                wc.insert(wc.end(), wterm[i].begin(), wterm[i].end());
                wc_ptr[i + 1] = (int)wc.size();
            }
            if ((rc = upload_vec(c, c->dwheel, wh)) || (rc = upload_vec(c, c->dwnodes, wn)) || (rc = upload_vec(c, c->dwlist, wl)) ||
                (rc = upload_vec(c, c->dwc_ptr, wc_ptr)) || (rc = upload_vec(c, c->dwc, wc)) || (rc = upload_vec(c, c->dwst, wst)) ||
                (rc = upload_vec(c, c->dwctl, wctl)) || (rc = upload_vec(c, c->dwarm, warm)))
                return rc;
            BL_CUDA(c, c->dwcf.alloc(std::max(c->NWR, 1)));
            BL_CUDA(c, c->dwper.alloc(std::max(c->NWR, 1)));
            BL_CUDA(c, cudaMemsetAsync(c->dwcf.p, 0, sizeof(float4) * std::max(c->NWR, 1), c->stream));
            BL_CUDA(c, cudaMemsetAsync(c->dwper.p, 0, sizeof(float) * std::max(c->NWR, 1), c->stream));
            BL_CUDA(c, c->dtcon.alloc(N));
            BL_CUDA(c, c->dtfric.alloc(N));
            BL_CUDA(c, cudaMemsetAsync(c->dtfric.p, 0, sizeof(float4) * N, c->stream));
        }
    }
    {   // the shocks of all bodies in their order (each's beam global), and per node its shocks' incidences in that order
        std::vector<bl_shock> sh;
        std::vector<std::vector<int2>> per;
        for (int bi = 0; bi < B; bi++)
            for (const bl_shock& x : c->bodies[bi].shocks) {
                bl_shock g = x;
                g.beam = (uint32_t)(recs[bi].beam0 + (int)x.beam);
                if (per.empty()) per.resize(N);
                const int2 e = ab[g.beam], q = make_int2((int)sh.size(), 0);
                per[e.x].push_back(make_int2(q.x, e.y)), per[e.y].push_back(make_int2((int)((uint32_t)q.x | 0x80000000u), e.x));
                sh.push_back(g);
            }
        c->NSH = (int)sh.size();
        if (c->NSH > 0) {
            std::vector<int> ptr(N + 1, 0);
            std::vector<int2> inc;
            for (int i = 0; i < N; i++) {
                inc.insert(inc.end(), per[i].begin(), per[i].end());
                ptr[i + 1] = (int)inc.size();
            }
            if ((rc = upload_vec(c, c->dshock, sh)) || (rc = upload_vec(c, c->sh_ptr, ptr)) || (rc = upload_vec(c, c->sh_inc, inc))) return rc;
            BL_CUDA(c, c->ssc.alloc(c->NSH));
        }
    }
    c->beam_grid = 0, c->ends16 = false;
    if (c->cfg.beam_kernel == 0 && M > 0) {
        // each tile's beams' ends as 16-bit offsets from its lowest node, where every tile spans fewer than 65,536 nodes
        std::vector<int> tbase(c->beam_tiles, 0);
        std::vector<uint32_t> ab16(Mpad, 0u);
        bool fits = true;
        for (int t = 0; t < c->beam_tiles && fits; t++) {
            const int j0 = t * kBeamTile, j1 = std::min(M, j0 + kBeamTile);
            int lo = INT32_MAX, hi = -1;
            for (int j = j0; j < j1; j++) lo = std::min(lo, std::min(ab[j].x, ab[j].y)), hi = std::max(hi, std::max(ab[j].x, ab[j].y));
            if (j1 <= j0) continue;
            fits = hi - lo < 65536;
            tbase[t] = lo;
            for (int j = j0; j < j1 && fits; j++) ab16[j] = (uint32_t)(ab[j].x - lo) | ((uint32_t)(ab[j].y - lo) << 16);
        }
        if (fits) {
            if ((rc = upload_vec(c, c->ab16, ab16)) || (rc = upload_vec(c, c->tbase, tbase))) return rc;
            c->ends16 = true;
        }
        // k_beams_tma: a persistent grid of as many blocks as fit on the device at once (at most one a tile)
        const size_t smem = c->ends16 ? beam_smem<true>() : beam_smem<false>();
        const void* fn = c->ends16 ? (const void*)k_beams_tma<true> : (const void*)k_beams_tma<false>;
        BL_CUDA(c, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0, sms = 0;
        BL_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBeamThreads, smem));
        BL_CUDA(c, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->cfg.device));
        if (c->cfg.beams_per_sm > 0) per_sm = std::min(per_sm, (int)c->cfg.beams_per_sm);
        if (per_sm > 0) c->beam_grid = std::min(c->beam_tiles, per_sm * sms);
    }
    BL_CUDA(c, c->nodef.alloc(N));
    {   // the incidences with their other ends, per warp of 32 nodes interleaved (entry q of lane l at 32 q + l), each
        // warp's width its widest node's count rounded up to 4, padded with (0, the node itself)
        const int nw = (N + 31) / 32;
        std::vector<int> eptr(nw + 1, 0);
        for (int w = 0; w < nw; w++) {
            int width = 0;
            for (int l = 0; l < 32 && 32 * w + l < N; l++) width = std::max(width, inc_ptr[32 * w + l + 1] - inc_ptr[32 * w + l]);
            width = (width + 3) / 4 * 4;
            eptr[w + 1] = eptr[w] + 32 * width;
        }
        std::vector<int2> ell(eptr[nw]);
        for (int w = 0; w < nw; w++) {
            const int width = (eptr[w + 1] - eptr[w]) / 32;
            for (int l = 0; l < 32; l++) {
                const int i = 32 * w + l;
                for (int q = 0; q < width; q++) {
                    int2 v = make_int2(0, i < N ? i : 0);
                    if (i < N && q < inc_ptr[i + 1] - inc_ptr[i]) {
                        const int e = inc[inc_ptr[i] + q];
                        const int2 e2 = ab[e & 0x7fffffff];
                        v = make_int2(e, e < 0 ? e2.x : e2.y); // (the other end)
                    }
                    ell[eptr[w] + 32 * q + l] = v;
                }
            }
        }
        if ((rc = upload_vec(c, c->ell_ptr, eptr))) return rc;
        // the 4-byte form where every warp's beams lie within 32,767 of its first and every neighbour within 32,767
        // nodes (k_force<true>): half the bytes of the incidence stream
        std::vector<int> base(nw, 0);
        bool packed = c->cfg.beam_kernel == 0;
        for (int w = 0; w < nw && packed; w++) {
            int lo = INT32_MAX;
            for (int q = eptr[w]; q < eptr[w + 1]; q++) {
                const int i = 32 * w + (q - eptr[w]) % 32;
                if (!(i >= N || ell[q].y == i)) lo = std::min(lo, ell[q].x & 0x7fffffff); // (not padding)
            }
            base[w] = lo == INT32_MAX ? 0 : lo;
            for (int q = eptr[w]; q < eptr[w + 1] && packed; q++) {
                const int i = 32 * w + (q - eptr[w]) % 32;
                if (i >= N || ell[q].y == i) continue;
                const int g = ell[q].x & 0x7fffffff;
                if (g - base[w] >= 0x7fff || g < base[w] || std::abs(ell[q].y - i) > 32767) packed = false;
            }
        }
        c->packed_inc = packed;
        if (packed) {
            std::vector<uint32_t> pk(ell.size());
            for (int w = 0; w < nw; w++)
                for (int q = eptr[w]; q < eptr[w + 1]; q++) {
                    const int i = 32 * w + (q - eptr[w]) % 32;
                    const bool pad = i >= N || ell[q].y == i;
                    pk[q] = pad ? (0x7fffu | (32768u << 16))
                                : (uint32_t)((ell[q].x & 0x7fffffff) - base[w]) | (ell[q].x < 0 ? 0x8000u : 0u) |
                                      ((uint32_t)(ell[q].y - i + 32768) << 16);
                }
            if ((rc = upload_vec(c, c->inc4, pk)) || (rc = upload_vec(c, c->ell_base, base))) return rc;
        } else if ((rc = upload_vec(c, c->inc2, ell))) {
            return rc;
        }
    }
    int P = 1;
    while (P < maxn) P <<= 1;
    c->rs_P = P;
    BL_CUDA(c, c->rs_sort.alloc(3 * (size_t)P));
    BL_CUDA(c, c->rs_bad.alloc(P));
    BL_CUDA(c, c->rs_np.alloc(P));
    BL_CUDA(c, c->rs_nv.alloc(P));
    c->N = N, c->M = M, c->B = B;
    if ((rc = commit_fem(c))) return rc;
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->bodies_dirty = false;
    c->committed = true;
    drop_graphs(c);
    return BL_GPU_OK;
}

// Orders work about to be enqueued on s after everything the context enqueued before, on whichever stream.
static int order_on(bl_gpu_ctx* c, cudaStream_t s) {
    if (c->last_stream != s) {
        BL_CUDA(c, cudaEventRecord(c->order_event, c->last_stream));
        BL_CUDA(c, cudaStreamWaitEvent(s, c->order_event, 0));
        c->last_stream = s;
    }
    return BL_GPU_OK;
}

static int ensure_committed(bl_gpu_ctx* c) {
    int rc;
    if (c->statics_dirty && (rc = commit_statics(c))) return rc;
    if (c->bodies_dirty && (rc = commit_bodies(c))) return rc;
    return BL_GPU_OK;
}

// One frame of n substeps on stream s. ev (5n + 4 events, or null): recorded before the first kernel, after the
// frame's start, in each substep after the beams (and triangles), the nodes' forces, the contacts between bodies, the
// integration and the FEM frames' step, and after the frame's end kernels.
static bool rebuild_at(const bl_gpu_ctx* c, int k) { return k % c->interval == 0; } // (s == 0 || s >= next_rebuild)

static int64_t frame_launches(const bl_gpu_ctx* c, int n) {
    int64_t per = 3 + (c->any_drag ? 1 : 0) + (c->NW > 0 ? 1 : 0) + (c->NWR > 0 && c->beam_grid == 0 ? 1 : 0) + (c->NSH > 0 ? 1 : 0);
    if (c->NF > 0) {
        per += c->fem_launches + (c->cfg.fem_check_residual ? 2 : 0) + (c->fem_ground ? 1 : 0);
        // (the unload re-pass: its checks, conditions and account; its passes' kernels, which run only where a check
        // finds an unload, are not counted - launched without a graph they always run)
        if (c->any_plastic_members) per += c->cfg.graphs ? 5 : 3 + 2 * (1 + c->chol_launches);
        if (c->cfg.fem_solver != BL_GPU_FEM_CHOLESKY) per += 1 - c->chol_launches; // (the Cholesky runs on a fallback only)
        const bool learned = c->cfg.fem_solver == BL_GPU_FEM_PCG_LEARNED, rec = c->rec_on;
        per += (learned || rec ? 2 : 0) + (learned ? 1 : 0) + (rec ? 3 : 0);
    }
    int64_t total = per * n + 3;
    if (c->contacts_on) {
        total += 1 + 3 * (int64_t)n; // k_islands; k_wake, k_detect, k_collide a substep
        for (int k = 0; k < n; k++) total += rebuild_at(c, k) ? 4 : 0; // (k_rebuild, k_pair_count, k_pair_place, k_pair_write)
    }
    return total;
}

static MlpDev mlp_dev(const bl_gpu_ctx* c) {
    MlpDev M{};
    M.wb = c->mlp_wb.p, M.w = c->mlp_w.p, M.m = c->mlp_m.p, M.v = c->mlp_v.p;
    M.adj_ptr = c->adj_ptr.p, M.adj = c->adj.p, M.prev_dv = c->prev_dv.p, M.feat = c->feat.p;
    M.sx = c->smp_x.p, M.st = c->smp_t.p, M.sw = c->smp_w.p, M.scount = c->scount.p, M.cap = std::max(c->rec_cap, 1);
    return M;
}

// A condition of the graph being captured on s (its default 1 at every launch of the graph); false when s is not
// capturing.
static bool make_condition(bl_gpu_ctx* c, cudaStream_t s, cudaGraphConditionalHandle* h) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    if (cudaStreamGetCaptureInfo(s, &st, nullptr, &g, nullptr, nullptr) != cudaSuccess || st != cudaStreamCaptureStatusActive) return false;
    return cudaGraphConditionalHandleCreate(h, g, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
}

// body(stream) under an IF node of the graph being captured on s, after everything captured so far (the body is
// captured on the context's aux stream into the node's body graph); without capture, body(s) runs as it is.
template <class Fn>
static void enqueue_if(bl_gpu_ctx* c, cudaStream_t s, cudaGraphConditionalHandle h, bool have, Fn body) {
    if (!have) {
        body(s);
        return;
    }
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd);
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeIf;
    p.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    if (cudaGraphAddNode(&node, g, deps, nd, &p) != cudaSuccess) {
        body(s); // (recorded as an error by the capture's end if the graph is unusable)
        return;
    }
    cudaGraph_t bg = p.conditional.phGraph_out[0];
    cudaStreamBeginCaptureToGraph(c->aux, bg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    body(c->aux);
    cudaGraph_t out = nullptr;
    cudaStreamEndCapture(c->aux, &out);
    cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies);
}

// The frames' PCG solve: one cooperative launch of k_fem_pcg (bl_fem_pcg.cuh)
static void launch_pcg(bl_gpu_ctx* c, cudaStream_t s, cudaGraphConditionalHandle h, bool have, int solver) {
    const bool learned = solver == BL_GPU_FEM_PCG_LEARNED;
    PcgArgs P{};
    P.x = c->px.p, P.r = c->pr.p, P.z = c->pz.p, P.p = c->pp.p, P.pf = c->ppf.p, P.pdi = c->ppdi.p;
    P.guess = learned ? c->guess.p : nullptr;
    P.scale = learned && c->cfg.pcg_learned_scale ? c->gscale.p : nullptr;
    P.xprev = c->pxprev.p;
    P.use_prev = (learned || solver == BL_GPU_FEM_PCG_PREVIOUS) ? 1 : 0;
    P.red = c->pred.p, P.stat = c->pstat.p, P.iters_total = c->piters.p, P.last_res = c->plast.p;
    P.cond = h, P.has_cond = have ? 1 : 0;
    P.max_iters = c->cfg.pcg_max_iters, P.tol = (double)c->cfg.pcg_tol;
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(c->pcg_grid), lc.blockDim = dim3(256), lc.dynamicSmemBytes = 0, lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    lc.attrs = at, lc.numAttrs = 1;
    cudaLaunchKernelEx(&lc, k_fem_pcg, c->fd, P);
}

static int enqueue_frame(bl_gpu_ctx* c, int n, cudaStream_t s, cudaEvent_t* ev = nullptr) {
    int q = 0;
    auto mark = [&]() {
        if (ev) cudaEventRecordWithFlags(ev[q++], s, cudaEventRecordExternal); // (a timing node of the captured graph)
    };
    mark();
    const float dt = c->cfg.dt;
    const float frame_time = (float)n * dt;
    const int tb = 256;
    const int gb = std::max((c->M + 2 * tb - 1) / (2 * tb), (c->B + tb - 1) / tb), gbody = (c->B + tb - 1) / tb;
    // (the node kernels' block sizes: bl_gpu_config.force_block / integrate_block, 256 unless tuned)
    const int fb = c->cfg.force_block > 0 ? c->cfg.force_block : 256, ib = c->cfg.integrate_block > 0 ? c->cfg.integrate_block : 256;
    const int gfn = (c->N + fb - 1) / fb, gin = (c->N + ib - 1) / ib;
    const Contacts& CT = c->ct;
    if (c->contacts_on) k_islands<<<1, 1024, 0, s>>>(c->dbodies.p, c->B, frame_time, c->cfg.sleeping, CT, c->deverr.p);
    k_frame_begin<<<std::max(gbody, 1), tb, 0, s>>>(c->dbodies.p, c->B, c->st, frame_time, c->cfg.sleeping, c->deverr.p);
    mark();
    DragDev dg{c->dup.p, c->dpid.p, c->dpart.p, c->dpmv.p, c->dpacc.p};
    WheelDev wh{c->dwheel.p, c->dwnodes.p, c->dwlist.p, c->dwc_ptr.p, c->dwc.p, c->dtcon.p, c->dtfric.p, c->dwst.p, c->dwctl.p,
                c->dwarm.p, c->dwcf.p, c->dwper.p, c->NWR, c->cfg.tyre_grip};
    ShockDev sk{c->dshock.p, c->sh_ptr.p, c->sh_inc.p, c->ssc.p};
    NodeFem nfm{c->fslot.p, c->fiperm.p, c->gdiag_ptr.p, c->gdiag.p, c->ton.p, c->tf.p, c->tt.p, c->ftorque.p, c->nforce.p, c->ext.p,
                c->mon.p, c->mfa.p, c->mta.p, c->mtb.p};
    const FemDev& F = c->fd;
    for (int k = 0; k < n; k++) {
        if (c->contacts_on) {
            // wake requests, then the pair search on its substeps (on the positions and velocities the substep starts from)
            k_wake<<<c->B, 256, 0, s>>>(c->dbodies.p, c->bmeta.p);
            if (rebuild_at(c, k)) {
                cudaMemsetAsync(c->pair_total.p, 0, sizeof(int), s);
                cudaMemsetAsync(c->sc.p, 0, 8 * sizeof(int), s);
                k_rebuild<<<c->B, 1024, sizeof(RebuildShared), s>>>(c->dbodies.p, c->B, c->nd.p, c->info.p, CT, k == 0 ? 1 : 0, c->deverr.p);
                k_pair_count<<<kQueryGrid, kQueryChunk, 0, s>>>(c->dbodies.p, c->nd.p, CT);
                k_pair_place<<<c->B, 1024, 0, s>>>(c->dbodies.p, c->B, CT, c->deverr.p);
                k_pair_write<<<kQueryGrid, kQueryChunk, 0, s>>>(c->dbodies.p, c->nd.p, CT);
            }
        }
        mark();
        if (c->any_drag) k_drag_parts<<<(c->B + 63) / 64, 64, 0, s>>>(c->dbodies.p, c->B, c->nd.p, c->ab.p, c->bmeta.p, dg);
        if (c->NF > 0) k_fem_begin<<<(c->NF + tb - 1) / tb, tb, 0, s>>>(F, c->nd.p);
        if (c->beam_grid > 0) {
            // (the wheels' step in the same launch, after each block's tiles)
            if (c->ends16)
                k_beams_tma<true><<<c->beam_grid, kBeamThreads, beam_smem<true>(), s>>>(c->ab16.p, c->tbase.p, c->kd.p, c->bst.p, c->bmeta.p, c->bcold.p,
                                                                                       c->stress.p, c->bbody.p, c->fsc.p, c->nd.p, c->dbodies.p, c->M, c->B,
                                                                                       c->beam_tiles, c->deverr.p, c->info.p, wh, dt, c->wait_ns);
            else
                k_beams_tma<false><<<c->beam_grid, kBeamThreads, beam_smem<false>(), s>>>(c->ab.p, nullptr, c->kd.p, c->bst.p, c->bmeta.p, c->bcold.p,
                                                                                         c->stress.p, c->bbody.p, c->fsc.p, c->nd.p, c->dbodies.p, c->M, c->B,
                                                                                         c->beam_tiles, c->deverr.p, c->info.p, wh, dt, c->wait_ns);
        } else {
            k_beams<<<std::max(gb, 1), tb, 0, s>>>(c->ab.p, c->kd.p, c->bst.p, c->bmeta.p, c->bcold.p, c->stress.p, c->bbody.p, c->fsc.p, c->nd.p,
                                                   c->dbodies.p, c->M, c->B);
            if (c->NWR > 0) k_wheels<<<(c->NWR + 7) / 8, 256, 0, s>>>(c->nd.p, c->info.p, c->dbodies.p, wh, dt);
        }
        if (c->NSH > 0)
            k_shocks<<<(c->NSH + 127) / 128, 128, 0, s>>>(sk, c->NSH, c->ab.p, c->bst.p, c->bmeta.p, c->stress.p, c->bbody.p, c->nd.p, c->dbodies.p);
        if (c->NT > 0 && c->any_plastic) k_tri_eval<true><<<(c->NT + 127) / 128, 128, 0, s>>>(F, c->nd.p);
        else if (c->NT > 0) k_tri_eval<false><<<(c->NT + 127) / 128, 128, 0, s>>>(F, c->nd.p);
        if (c->NM > 0 && c->any_plastic_members) k_member_eval<true><<<(c->NM + 127) / 128, 128, 0, s>>>(F, c->nd.p);
        else if (c->NM > 0) k_member_eval<false><<<(c->NM + 127) / 128, 128, 0, s>>>(F, c->nd.p);
        mark();
        if (c->packed_inc)
            k_force<true><<<std::max(gfn, 1), fb, 0, s>>>(c->nd.p, c->info.p, c->ell_ptr.p, c->inc4.p, c->ell_base.p, c->fsc.p, c->dbodies.p,
                                                         c->cfg.gravity[0], c->cfg.gravity[1], c->cfg.gravity[2], c->N, k == 0 ? 1 : 0, nfm, c->nodef.p, dg, wh, sk);
        else
            k_force<false><<<std::max(gfn, 1), fb, 0, s>>>(c->nd.p, c->info.p, c->ell_ptr.p, c->inc2.p, nullptr, c->fsc.p, c->dbodies.p,
                                                          c->cfg.gravity[0], c->cfg.gravity[1], c->cfg.gravity[2], c->N, k == 0 ? 1 : 0, nfm, c->nodef.p, dg, wh, sk);
        mark();
        if (c->contacts_on) {
            // contacts between bodies on the forces so far (World::collide_pairs, before the static contacts)
            k_detect<<<148 * 4, 256, 0, s>>>(c->nd.p, c->info.p, c->dbodies.p, CT);
            k_collide<<<c->B, kCollideThreads, kCollideSmem, s>>>(c->nd.p, c->info.p, c->dbodies.p, c->B, CT, c->nodef.p);
        }
        mark();
        k_integrate<<<std::max(gin, 1), ib, 0, s>>>(c->nd.p, c->info.p, c->dbodies.p, c->st, dt, c->N, k == 0 ? 1 : 0, c->nodef.p, wh);
        if (c->NW > 0) k_tyres<<<(c->NW + 7) / 8, 256, 0, s>>>(c->nd.p, c->info.p, c->dbodies.p, dt, c->NW, k == 0 ? 1 : 0, c->nodef.p, wh);
        mark();
        if (c->NF > 0) {
            // the frames' implicit step: assembly, factorization and substitutions level by level, velocities, integration
            if (c->fem_ground) { // (the frame nodes' static contacts: their forces, the ground's hold in the step)
                cudaMemsetAsync(c->contact_n.p, 0, sizeof(float4) * c->NF, s);
                k_fem_static<<<(c->n_fem_nodes + 127) / 128, 128, 0, s>>>(c->nd.p, c->nforce.p, c->fem_nodes.p, c->n_fem_nodes, c->fslot.p, c->info.p,
                                                                        c->dbodies.p, c->st, dt, c->contact_n.p);
            }
            k_fem_assemble_all<<<(c->NF + c->NB + 127) / 128, 128, 0, s>>>(F, c->nd.p, c->nforce.p);
            if (c->cfg.fem_check_residual) {
                cudaMemcpyAsync(c->a0d.p, c->diag.p, sizeof(double) * 36 * c->NF, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(c->a0o.p, c->off.p, sizeof(double) * 36 * std::max(c->NB, 1), cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(c->b0.p, c->rhs.p, sizeof(double) * 6 * c->NF, cudaMemcpyDeviceToDevice, s);
            }
            const bool learned = c->cfg.fem_solver == BL_GPU_FEM_PCG_LEARNED, rec = c->rec_on;
            const MlpDev MD = mlp_dev(c);
            if (learned || rec) k_mlp_features<<<(c->NF + 127) / 128, 128, 0, s>>>(F, MD, c->nd.p, c->nforce.p);
            if (rec) k_mlp_record_pre<<<(c->NF + 127) / 128, 128, 0, s>>>(F, MD);
            if (learned) k_mlp_infer<<<(c->NF + kLanes - 1) / kLanes, kLanes, 0, s>>>(F, MD, c->guess.p, c->gscale.p);
            auto cholesky = [c, &F](cudaStream_t cs) {
                if (c->fem_mode == 2) {
                    // multifrontal: per level of the front tree its fronts assembled, then panel by panel factored and
                    // updated with the right side carried along (the forward substitution); the backward from the root down
                    const MfDev& M = c->mf;
                    const int nlev = (int)c->mf_level_ptr.size() - 1;
                    for (int L = 0; L < nlev; L++) {
                        k_mf_assemble<<<c->mf_tasm_ptr[L + 1] - c->mf_tasm_ptr[L], 256, 0, cs>>>(F, M, c->mf_tasm_ptr[L]);
                        const std::vector<int>& tp = c->mf_tpan_ptr[L];
                        const std::vector<int>& tu = c->mf_tupd_ptr[L];
                        for (size_t sp = 0; sp + 1 < tp.size(); sp++) {
                            k_mf_panel<<<tp[sp + 1] - tp[sp], 256, 0, cs>>>(M, tp[sp], (int)sp, F.comp_fail);
                            k_mf_update<<<tu[sp + 1] - tu[sp], 256, 0, cs>>>(M, tu[sp], (int)sp);
                        }
                    }
                    for (int L = nlev - 1; L >= 0; L--)
                        k_mf_backward<<<c->mf_level_ptr[L + 1] - c->mf_level_ptr[L], 256, c->mf_smem, cs>>>(F, M, c->mf_level_ptr[L]);
                    return;
                }
                // the levels of the elimination tree two launches each (factor; updates with the forward substitution),
                // then the backward substitution a launch a level from the top down
                const int nlev = (int)c->lvl_col_ptr.size() - 1, top = c->front_level;
                for (int L = 0; L < top; L++) {
                    const int c0 = c->lvl_col_ptr[L], c1 = c->lvl_col_ptr[L + 1], g0 = c->lvl_grp_ptr[L], g1 = c->lvl_grp_ptr[L + 1];
                    k_fem_chol_level<<<dim3(c1 - c0, c->lvl_ns[L]), kUnit, 0, cs>>>(F, c0);
                    k_fem_update_forward_level<<<(g1 - g0 + 3) / 4 + (c1 - c0), kUnit, 0, cs>>>(F, g0, g1, c0);
                }
                if (top < nlev) {
                    // the top chain: its dense front scattered, its right side, then panel by panel the factor with
                    // the forward substitution, then the backward substitution
                    const FrontDev& X = c->front;
                    cudaMemsetAsync(X.D, 0, sizeof(double) * X.N * X.N, cs);
                    const int ns = 36 * (X.m + X.nblk) + X.N - 6 * X.m;
                    k_front_scatter<<<(ns + 255) / 256, 256, 0, cs>>>(F, X);
                    k_front_rhs<<<X.m, kUnit, 0, cs>>>(F, X);
                    for (int p = 0; p < X.nt; p++) {
                        k_front_potrf<<<1, 32, 0, cs>>>(F, X, p);
                        const int t = X.nt - p - 1;
                        if (t > 0) {
                            k_front_trsm<<<t, kFT, 0, cs>>>(X, p);
                            k_front_syrk<<<t * (t + 1) / 2, 256, 0, cs>>>(X, p);
                        }
                    }
                    k_front_solve<<<1, 1024, sizeof(double) * X.N, cs>>>(F, X);
                }
                for (int L = top - 1; L >= 0; L--) {
                    const int c0 = c->lvl_col_ptr[L], c1 = c->lvl_col_ptr[L + 1];
                    k_fem_backward_level<<<c1 - c0, kUnit, 0, cs>>>(F, c0);
                }
            };
            if (c->cfg.fem_solver == BL_GPU_FEM_CHOLESKY) {
                cholesky(s);
            } else {
                // PCG first; the Cholesky under a conditional node that the PCG kernel sets when it missed the tolerance
                cudaGraphConditionalHandle h{};
                const bool have = make_condition(c, s, &h);
                launch_pcg(c, s, h, have, c->cfg.fem_solver);
                enqueue_if(c, s, h, have, cholesky);
                // (the solution, PCG's or the fallback's, is the next solve's guess)
                cudaMemcpyAsync(c->pxprev.p, c->rhs.p, sizeof(double) * 6 * c->NF, cudaMemcpyDeviceToDevice, s);
            }
            if (c->any_plastic_members) {
                // the unload re-pass (frame_fem.cpp:2959-2995): where the step unloads a flowing hinge (bar, twist), its
                // elastic tangent and the step again - assembled and factored again, at most twice; each pass under an
                // IF node its check sets (launched without a graph, the passes run and solve the same system again)
                auto repass = [c, &F, cholesky](cudaStream_t cs) {
                    k_fem_assemble_all<<<(c->NF + c->NB + 127) / 128, 128, 0, cs>>>(F, c->nd.p, c->nforce.p);
                    if (c->cfg.fem_check_residual) {
                        cudaMemcpyAsync(c->a0d.p, c->diag.p, sizeof(double) * 36 * c->NF, cudaMemcpyDeviceToDevice, cs);
                        cudaMemcpyAsync(c->a0o.p, c->off.p, sizeof(double) * 36 * std::max(c->NB, 1), cudaMemcpyDeviceToDevice, cs);
                        cudaMemcpyAsync(c->b0.p, c->rhs.p, sizeof(double) * 6 * c->NF, cudaMemcpyDeviceToDevice, cs);
                    }
                    cholesky(cs);
                };
                for (int pass = 0; pass < 2; pass++) {
                    k_member_unload<<<(c->NM + 127) / 128, 128, 0, s>>>(F, c->nd.p, pass);
                    cudaGraphConditionalHandle h{};
                    const bool have = make_condition(c, s, &h);
                    if (have) k_repass_cond<<<1, 1, 0, s>>>(c->rp.p, pass, h);
                    enqueue_if(c, s, h, have, repass);
                }
                k_repass_account<<<(c->B + 127) / 128, 128, 0, s>>>(F);
            }
            if (c->cfg.fem_check_residual) {
                k_fem_residual<<<(c->NF + 3) / 4, 128, 0, s>>>(F, c->a0d.p, c->a0o.p, c->b0.p, c->res.p);
                k_fem_residual_done<<<1, 1, 0, s>>>(c->res.p);
            }
            if (rec) {
                k_mlp_record_post<<<(c->NF + 127) / 128, 128, 0, s>>>(F, MD);
                k_mlp_record_done<<<1, 1, 0, s>>>(MD, c->NF);
            }
            if (learned || rec) k_mlp_store_dv<<<(c->NF + 127) / 128, 128, 0, s>>>(F, MD);
            k_fem_velocity<<<(c->NF + 127) / 128, 128, 0, s>>>(F, c->nd.p, c->nforce.p);
            k_fem_integrate<<<(c->n_fem_nodes + 255) / 256, 256, 0, s>>>(F, c->nd.p, c->nforce.p, c->fem_nodes.p, c->n_fem_nodes, c->fslot.p, c->info.p,
                                                                       c->dbodies.p, dt);
        }
        mark();
    }
    RepairScratch rs{c->rs_sort.p, c->rs_bad.p, c->rs_np.p, c->rs_nv.p, c->rs_P};
    k_frame_finish<<<1, 1024, 0, s>>>(c->dbodies.p, c->B, c->nd.p, c->inc_ptr.p, c->inc.p, c->ab.p, c->bmeta.p, rs, frame_time, c->cfg.sleeping,
                                      c->cfg.sleep_speed, c->cfg.sleep_time, c->deverr.p);
    mark();
    k_sleep_apply<<<std::max(c->B, 1), 256, 0, s>>>(c->dbodies.p, c->nd.p, c->bmeta.p);
    mark();
    return BL_GPU_OK;
}

// A body's FEM frame of triangle elements made ready (bl_fem_host.cuh): frame nodes in the order FemFrame::add_tri
// makes them, FemFrame::finalize's rest shapes and inertias, analyse's pattern, the elements' stiffnesses.
static int build_fem_model(const bl_node* nodes, const bl_node_info* info, int32_t n_nodes, const bl_fem_desc& fd, std::vector<FemSection>& sections,
                           std::vector<FrameSectionH>& fsections, std::shared_ptr<FemModel>& out, bool want_updates = true) {
    if (fd.n_tris < 0 || fd.n_members < 0 || (fd.n_tris > 0 && (!fd.tris || !fd.sections || fd.n_sections <= 0)) ||
        (fd.n_members > 0 && (!fd.members || !fd.frame_sections || fd.n_frame_sections <= 0)) || fd.n_tris + fd.n_members == 0 || !nodes || !info)
        return BL_GPU_EINVAL;
    sections.clear(), fsections.clear();
    for (int k = 0; k < (fd.n_tris > 0 ? fd.n_sections : 0); k++) {
        const bl_shell_section& ss = fd.sections[k];
        if (!(ss.t > 0) || !(ss.E > 0)) return BL_GPU_EINVAL;
        sections.push_back(FemSection{ss.E, ss.nu, ss.rho, ss.t, ss.yield, ss.damping, ss.drill});
    }
    for (int k = 0; k < (fd.n_members > 0 ? fd.n_frame_sections : 0); k++) {
        const bl_frame_section& fs = fd.frame_sections[k];
        if (!(fs.E > 0) || !(fs.G > 0) || !(fs.A > 0) || fs.Np < 0 || fs.Mp < 0 || fs.Tp < 0) return BL_GPU_EINVAL;
        fsections.push_back(FrameSectionH{fs.E, fs.G, fs.rho, fs.A, fs.Iy, fs.Iz, fs.J, fs.As_y, fs.As_z, fs.damping, fs.axial, fs.joint_k,
                                          fs.Np, fs.Mp, fs.Tp, fs.hardening});
    }
    auto M = std::make_shared<FemModel>();
    std::vector<int> slot(n_nodes, -1);
    auto add_node = [&](uint32_t bn) {
        if (slot[bn] < 0) slot[bn] = (int)M->node.size(), M->node.push_back(bn);
        return slot[bn];
    };
    auto add_tris = [&]() {
        for (int t = 0; t < fd.n_tris; t++) {
            const bl_fem_tri& tr = fd.tris[t];
            if (tr.a >= (uint32_t)n_nodes || tr.b >= (uint32_t)n_nodes || tr.c >= (uint32_t)n_nodes || tr.section >= fd.n_sections) return false;
            const int a = add_node(tr.a), b = add_node(tr.b), cc = add_node(tr.c);
            M->tn.push_back({a, b, cc});
            M->tsec.push_back(tr.section);
            M->tmass.push_back(tr.mass);
        }
        return true;
    };
    if (fd.tris_first && !add_tris()) return BL_GPU_EINVAL;
    std::vector<float> mpm;
    for (int e = 0; e < fd.n_members; e++) { // (the add_element calls, in the order the caller made them)
        const bl_fem_member& mb = fd.members[e];
        if (mb.a >= (uint32_t)n_nodes || mb.b >= (uint32_t)n_nodes || mb.section >= fd.n_frame_sections || mb.end_a > BL_FJ_ELASTIC ||
            mb.end_b > BL_FJ_ELASTIC)
            return BL_GPU_EINVAL;
        const int a = add_node(mb.a), b = add_node(mb.b);
        M->mn.push_back({a, b});
        M->msec.push_back(mb.section);
        M->mend.push_back(mb.end_a), M->mend.push_back(mb.end_b);
        M->mmass.push_back(mb.mass);
        const FrameSectionH& fs = fsections[mb.section];
        mpm.push_back(fs.rho * fs.A); // (FrameSection::mass_per_m)
    }
    if (!fd.tris_first && !add_tris()) return BL_GPU_EINVAL;
    // (a frame of triangles on the ground: its plates' mid points take contacts too - collide_static_mids - not on this
    // path; a frame of members takes its nodes' static contacts)
    for (uint32_t bn : M->node)
        if ((info[bn].flags & BL_NF_GROUND) && !M->tn.empty()) return BL_GPU_EUNSUPPORTED;
    for (int i = 0; i < n_nodes; i++)
        if (info[i].flags & BL_NF_TYRE) return BL_GPU_EUNSUPPORTED; // (tyre nodes on a frame body)
    std::vector<float> px(n_nodes), py(n_nodes), pz(n_nodes), ms(n_nodes);
    for (int i = 0; i < n_nodes; i++) px[i] = nodes[i].p[0], py[i] = nodes[i].p[1], pz[i] = nodes[i].p[2], ms[i] = nodes[i].mass;
    fem_finalize(*M, px.data(), py.data(), pz.data(), ms.data(), mpm);
    bool again = false;
    for (size_t t = 0; t < M->tn.size(); t++) // (the caller's mass, else its section's over its area: tri_mass, frame_fem.h:373)
        if (!(M->tmass[t] > 0)) M->tmass[t] = sections[M->tsec[t]].rho * sections[M->tsec[t]].t * M->tarea0[t], again = true;
    if (again) fem_finalize(*M, px.data(), py.data(), pz.data(), ms.data(), mpm); // (the inertias from those masses)
    fem_analyse(*M, want_updates);
    M->tk.assign(162 * M->tn.size(), 0.0f), M->tb.assign(54 * M->tn.size(), 0.0f);
    for (size_t t = 0; t < M->tn.size(); t++) {
        if (M->tbroken[t]) continue;
        float X[3][2];
        for (int i = 0; i < 3; i++) X[i][0] = M->tX[6 * t + 2 * i], X[i][1] = M->tX[6 * t + 2 * i + 1];
        const FemSection& fs = sections[M->tsec[t]];
        tri_local_k(X, TriSec{fs.E, fs.nu, fs.t, fs.drill}, &M->tk[162 * t], &M->tb[54 * t]);
    }
    out = M;
    return BL_GPU_OK;
}

// ------------------------------------------------------------------------------------------ C ABI
extern "C" {

void bl_gpu_default_config(bl_gpu_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->gravity[0] = 0, cfg->gravity[1] = -9.81f, cfg->gravity[2] = 0;
    cfg->dt = 0.0005f;
    cfg->sleeping = 1;
    cfg->sleep_speed = 0.06f;
    cfg->sleep_time = 1.0f;
    cfg->device = 0;
    cfg->deterministic = 1;
    cfg->collision_hz = 120.0f;
    cfg->inter_body_collisions = 1;
    cfg->max_pairs = 1 << 21;
    cfg->fem_solver = BL_GPU_FEM_CHOLESKY;
    cfg->pcg_max_iters = 200;
    cfg->pcg_tol = 1e-6f;
    cfg->fem_check_residual = 0;
    cfg->pcg_learned_scale = 0;
    cfg->graphs = 1;
    cfg->beam_kernel = 0;
    cfg->fem_dense_front = 3;
    cfg->force_block = 0;
    cfg->integrate_block = 0;
    cfg->beams_per_sm = 0;
    cfg->tyre_grip = 1.0f;
    cfg->bulk_wait_s = 1.0f;
    cfg->contact_whole_max = kStage;
}

int bl_gpu_abi_version(void) { return BL_GPU_ABI_VERSION; }

const char* bl_gpu_error_string(int code) {
    switch (code) {
    case BL_GPU_OK: return "ok";
    case BL_GPU_EINVAL: return "invalid argument";
    case BL_GPU_ENOMEM: return "out of memory";
    case BL_GPU_ECUDA: return "CUDA error";
    case BL_GPU_EUNSUPPORTED: return "unsupported feature";
    case BL_GPU_ELIMIT: return "capacity exceeded";
    case BL_GPU_ENODEVICE: return "no sm_100 CUDA device";
    case BL_GPU_ESTATE: return "invalid state";
    default: return "unknown error";
    }
}

int bl_gpu_create(const bl_gpu_config* cfg, bl_gpu_ctx** out) {
    if (!out) return BL_GPU_EINVAL;
    *out = nullptr;
    bl_gpu_config c0;
    bl_gpu_default_config(&c0);
    if (cfg) c0 = *cfg;
    if (!(c0.dt > 0) || c0.deterministic != 1 || c0.max_pairs < 1 || c0.fem_solver < 0 || c0.fem_solver > 3 || c0.pcg_max_iters < 0 ||
        !(c0.pcg_tol > 0) || c0.beam_kernel < 0 || c0.beam_kernel > 1 || c0.fem_dense_front < 0 || c0.fem_dense_front > 3 ||
        !(c0.force_block == 0 || c0.force_block == 64 || c0.force_block == 128 || c0.force_block == 256) ||
        !(c0.integrate_block == 0 || c0.integrate_block == 64 || c0.integrate_block == 128 || c0.integrate_block == 256) ||
        c0.beams_per_sm < 0 || c0.beams_per_sm > 16 || !(c0.tyre_grip >= 0) || !(c0.bulk_wait_s >= 0 && c0.bulk_wait_s <= 10) ||
        c0.contact_whole_max < 0 || c0.contact_whole_max > kStage)
        return BL_GPU_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || c0.device < 0 || c0.device >= ndev) return BL_GPU_ENODEVICE;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, c0.device) != cudaSuccess || prop.major != 10) return BL_GPU_ENODEVICE;
    bl_gpu_ctx* c = new (std::nothrow) bl_gpu_ctx();
    if (!c) return BL_GPU_ENOMEM;
    c->cfg = c0;
    c->wait_ns = (unsigned long long)((double)c0.bulk_wait_s * 1e9);
    auto fail = [&](cudaError_t e) {
        c->last_cuda = (int)e;
        delete c;
        return e == cudaErrorMemoryAllocation ? BL_GPU_ENOMEM : BL_GPU_ECUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(c0.device)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaStreamCreateWithFlags(&c->aux, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
    if ((e = cudaEventCreateWithFlags(&c->order_event, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
    c->last_stream = c->stream;
    if ((e = cudaMemcpyToSymbol(c_ground, kGroundModels, sizeof(kGroundModels))) != cudaSuccess) return fail(e);
    if ((e = c->deverr.alloc(1)) != cudaSuccess) return fail(e);
    for (DevBuf<float>* d : {&c->mlp_w, &c->mlp_m, &c->mlp_v, &c->gsum})
        if ((e = d->alloc(kParams)) != cudaSuccess) return fail(e);
    if ((e = c->mlp_wb.alloc(kParams)) != cudaSuccess) return fail(e);
    if ((e = c->scount.alloc(1)) != cudaSuccess) return fail(e);
    if ((e = cudaMemset(c->scount.p, 0, sizeof(int))) != cudaSuccess) return fail(e);
    if (bl_gpu_mlp_init(c, 1) != BL_GPU_OK) {
        const int rc0 = c->last_cuda;
        delete c;
        return rc0 == cudaErrorMemoryAllocation ? BL_GPU_ENOMEM : BL_GPU_ECUDA;
    }
    if ((e = cudaMemset(c->deverr.p, 0, sizeof(uint32_t))) != cudaSuccess) return fail(e);
    *out = c;
    return BL_GPU_OK;
}

int bl_gpu_destroy(bl_gpu_ctx* c) {
    if (!c) return BL_GPU_EINVAL;
    cudaSetDevice(c->cfg.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    free_device(c);
    free_statics(c);
    c->deverr.free_();
    if (c->order_event) cudaEventDestroy(c->order_event);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->aux) cudaStreamDestroy(c->aux);
    delete c;
    return BL_GPU_OK;
}

int bl_gpu_set_terrain(bl_gpu_ctx* c, int32_t nx, int32_t nz, float cell, float origin_x, float origin_z, const float* heights, const uint8_t* surfaces) {
    if (!c || !heights || nx < 2 || nz < 2 || !(cell > 0)) return BL_GPU_EINVAL;
    c->hnx = nx, c->hnz = nz, c->cell = cell, c->ox = origin_x, c->oz = origin_z;
    c->heights.assign(heights, heights + (size_t)nx * nz);
    if (surfaces) c->surfaces.assign(surfaces, surfaces + (size_t)nx * nz);
    else c->surfaces.assign((size_t)nx * nz, 0);
    // Heightfield::update_bounds (static_world.cpp:163-184): maxima over 16 x 16 cells, a vertex in every block it borders
    const int kBlock = 16;
    c->hbx = (nx - 1 + kBlock - 1) / kBlock, c->hbz = (nz - 1 + kBlock - 1) / kBlock;
    c->block_max.assign((size_t)c->hbx * c->hbz, -1e30f);
    for (int z = 0; z < nz; z++)
        for (int x = 0; x < nx; x++) {
            const float v = heights[(size_t)z * nx + x];
            const int bx0 = std::max(0, (x - 1) / kBlock), bx1 = std::min(c->hbx - 1, x / kBlock);
            const int bz0 = std::max(0, (z - 1) / kBlock), bz1 = std::min(c->hbz - 1, z / kBlock);
            for (int bz = bz0; bz <= bz1; bz++)
                for (int bx = bx0; bx <= bx1; bx++) {
                    float& m = c->block_max[(size_t)bz * c->hbx + bx];
                    m = (m < v) ? v : m;
                }
        }
    c->has_terrain = 1;
    c->statics_dirty = true;
    return BL_GPU_OK;
}

int bl_gpu_add_box(bl_gpu_ctx* c, const float center[3], const float half[3], const float q[4], int32_t surface, float max_force) {
    if (!c || !center || !half || !q || surface < 0 || surface > 255) return BL_GPU_EINVAL;
    Box b{};
    b.cx = center[0], b.cy = center[1], b.cz = center[2];
    b.hx = half[0], b.hy = half[1], b.hz = half[2];
    // to_mat3 (math.h:166-174)
    const float x = q[0], y = q[1], z = q[2], w = q[3];
    const float xx = x * x, yy = y * y, zz = z * z, xy = x * y, xz = x * z, yz = y * z, wx = w * x, wy = w * y, wz = w * z;
    const float r[9] = {1 - 2 * (yy + zz), 2 * (xy + wz), 2 * (xz - wy), 2 * (xy - wz), 1 - 2 * (xx + zz), 2 * (yz + wx),
                        2 * (xz + wy),     2 * (yz - wx), 1 - 2 * (xx + yy)};
    std::memcpy(b.r, r, sizeof(r));
    // StaticBox::update_aabb (static_world.cpp:242-246): e = |c0| hx + |c1| hy + |c2| hz
    float e[3];
    for (int k = 0; k < 3; k++) e[k] = std::fabs(r[k]) * b.hx + std::fabs(r[3 + k]) * b.hy + std::fabs(r[6 + k]) * b.hz;
    b.mnx = b.cx - e[0], b.mny = b.cy - e[1], b.mnz = b.cz - e[2];
    b.mxx = b.cx + e[0], b.mxy = b.cy + e[1], b.mxz = b.cz + e[2];
    b.surface = surface;
    b.max_force = max_force;
    c->boxes.push_back(b);
    c->statics_dirty = true;
    return BL_GPU_OK;
}

int bl_gpu_add_cylinder(bl_gpu_ctx* c, const float base[3], float radius, float height, int32_t surface) {
    if (!c || !base || surface < 0 || surface > 255) return BL_GPU_EINVAL;
    c->cyls.push_back(Cyl{base[0], base[1], base[2], radius, height, surface});
    c->statics_dirty = true;
    return BL_GPU_OK;
}

int bl_gpu_build_grid(bl_gpu_ctx* c) {
    if (!c) return BL_GPU_EINVAL;
    build_grid_host(c);
    c->statics_dirty = true;
    return BL_GPU_OK;
}

int bl_gpu_set_kill_y(bl_gpu_ctx* c, float y) {
    if (!c) return BL_GPU_EINVAL;
    c->kill_y = y;
    c->statics_dirty = true;
    return BL_GPU_OK;
}

int bl_gpu_add_body(bl_gpu_ctx* c, const bl_body_desc* d, int32_t* body_id) {
    if (!c || !d || d->n_nodes < 0 || d->n_beams < 0 || (d->n_nodes > 0 && (!d->nodes || !d->info)) || (d->n_beams > 0 && !d->beams)) return BL_GPU_EINVAL;
    if ((int64_t)d->n_beams * 2 + 2 * (int64_t)c->M > 0x7fffffffLL) return BL_GPU_ELIMIT;
    for (int j = 0; j < d->n_beams; j++) {
        const bl_beam& b = d->beams[j];
        if (b.a >= (uint32_t)d->n_nodes || b.b >= (uint32_t)d->n_nodes || b.type > BL_BT_SUPPORT) return BL_GPU_EINVAL;
    }
    if (d->n_tris < 0 || (d->n_tris > 0 && !d->tris)) return BL_GPU_EINVAL;
    for (int t = 0; t < d->n_tris; t++)
        if (d->tris[t].a >= (uint32_t)d->n_nodes || d->tris[t].b >= (uint32_t)d->n_nodes || d->tris[t].c >= (uint32_t)d->n_nodes) return BL_GPU_EINVAL;
    if (d->self_collision) return BL_GPU_EUNSUPPORTED;                               // (a body's nodes against its own triangles)
    const bool has_frame = d->fem && (d->fem->n_tris > 0 || d->fem->n_members > 0);
    if (d->n_tris > 0 && has_frame) return BL_GPU_EUNSUPPORTED; // (contacts of frame nodes)
    if (has_frame && d->n_beams > 0) {
        // a beam on a frame node is a spring of the frame's implicit step in the reference (its links, frame_fem.cpp:
        // 576-590, 2774-2825): not on this path
        std::vector<uint8_t> on_frame(d->n_nodes, 0);
        for (int t = 0; d->fem->tris && t < d->fem->n_tris; t++) {
            const bl_fem_tri& ft = d->fem->tris[t];
            if (ft.a < (uint32_t)d->n_nodes) on_frame[ft.a] = 1;
            if (ft.b < (uint32_t)d->n_nodes) on_frame[ft.b] = 1;
            if (ft.c < (uint32_t)d->n_nodes) on_frame[ft.c] = 1;
        }
        for (int e = 0; d->fem->members && e < d->fem->n_members; e++) {
            const bl_fem_member& mb = d->fem->members[e];
            if (mb.a < (uint32_t)d->n_nodes) on_frame[mb.a] = 1;
            if (mb.b < (uint32_t)d->n_nodes) on_frame[mb.b] = 1;
        }
        for (int j = 0; j < d->n_beams; j++)
            if (on_frame[d->beams[j].a] || on_frame[d->beams[j].b]) return BL_GPU_EUNSUPPORTED;
    }
    if (has_frame && d->allow_deform && d->allow_break) { // (yielding: its tears, bisections and splits are topology events)
        for (int k = 0; d->fem->n_tris > 0 && d->fem->sections && k < d->fem->n_sections; k++)
            if (d->fem->sections[k].yield > 0) return BL_GPU_EUNSUPPORTED;
        for (int k = 0; d->fem->n_members > 0 && d->fem->frame_sections && k < d->fem->n_frame_sections; k++)
            if (d->fem->frame_sections[k].Np > 0) return BL_GPU_EUNSUPPORTED;
    }
    if (c->bodies.size() >= (size_t)(1 << 23)) return BL_GPU_ELIMIT;               // (a triangle keeps its body in 23 bits)
    HostBody hb;
    hb.nodes.assign(d->nodes, d->nodes + d->n_nodes);
    hb.info.assign(d->info, d->info + d->n_nodes);
    hb.beams.assign(d->beams, d->beams + d->n_beams);
    if (d->n_tris > 0) hb.tris.assign(d->tris, d->tris + d->n_tris);
    Body& r = hb.rec;
    std::memset(&r, 0, sizeof(r));
    r.crad = d->collision_radius, r.cfric = d->contact_friction, r.hull_depth = d->hull_depth, r.face_skin = d->face_skin;
    r.faces_only = d->faces_only ? 1 : 0, r.group = d->collision_group, r.island = -1;
    if (!(d->air_drag >= 0) || !(d->aero_cda >= 0)) return BL_GPU_EINVAL;
    r.air_drag = d->air_drag, r.aero_cda = d->aero_cda, r.drag = (d->air_drag > 0 || d->aero_cda > 0) ? 1 : 0;
    if (r.drag && d->fem && (d->fem->n_tris > 0 || d->fem->n_members > 0)) return BL_GPU_EUNSUPPORTED; // (a frame's parts)
    if (d->n_wheels < 0 || (d->n_wheels > 0 && !d->wheels)) return BL_GPU_EINVAL;
    if (d->n_wheels > 0) {
        if (has_frame) return BL_GPU_EUNSUPPORTED; // (tyre nodes of a frame body: its implicit step's)
        std::vector<uint8_t> on_wheel(d->n_nodes, 0);
        for (int k = 0; k < d->n_wheels; k++) {
            const bl_wheel& w = d->wheels[k];
            if (w.axle0 >= (uint32_t)d->n_nodes || w.axle1 >= (uint32_t)d->n_nodes || w.n_nodes < 0 || (w.n_nodes > 0 && !w.nodes) ||
                w.propulsed < 0 || w.propulsed > 2 || w.arm < -1 || w.arm >= d->n_nodes || w.near_attach < -1 || w.near_attach >= d->n_nodes)
                return BL_GPU_EINVAL;
            HostBody::Wheel hw{w.axle0, w.axle1, {}, w.radius, w.mass, w.propulsed, w.arm, w.near_attach};
            for (int j = 0; j < w.n_nodes; j++) {
                // (a node on one wheel once: the reference adds a wheel's turn per place and shares a node's patch with its
                // last wheel only)
                if (w.nodes[j] >= (uint32_t)d->n_nodes) return BL_GPU_EINVAL;
                if (on_wheel[w.nodes[j]]++) return BL_GPU_EUNSUPPORTED;
                hw.nodes.push_back(w.nodes[j]);
            }
            hb.wheels.push_back(std::move(hw));
        }
        if (hb.wheels.size() > 32767) return BL_GPU_ELIMIT; // (SoftBody::node_wheel: 16-bit)
    }
    if (d->n_shocks < 0 || (d->n_shocks > 0 && !d->shocks)) return BL_GPU_EINVAL;
    {   // every BL_BF_SHOCK beam has its one shock, every shock a BL_BF_SHOCK beam
        std::vector<uint8_t> seen(d->n_beams, 0);
        for (int q = 0; q < d->n_shocks; q++) {
            const uint32_t j = d->shocks[q].beam;
            if (j >= (uint32_t)d->n_beams || !(d->beams[j].flags & BL_BF_SHOCK) || seen[j]++) return BL_GPU_EINVAL;
        }
        for (int j = 0; j < d->n_beams; j++)
            if ((d->beams[j].flags & BL_BF_SHOCK) && !seen[j]) return BL_GPU_EINVAL;
        if (d->n_shocks > 0 && has_frame) return BL_GPU_EUNSUPPORTED; // (shocks on frame nodes: the implicit step's springs)
        hb.shocks.assign(d->shocks, d->shocks + d->n_shocks);
    }
    for (const bl_tri& t : hb.tris) r.hull |= t.two_sided ? 0 : 1;
    for (int i = 0; i < d->n_nodes; i++) r.contacters |= (d->info[i].flags & BL_NF_CONTACTER) ? 1 : 0;
    r.fric = d->ground_friction;
    r.bounce = d->bounce, r.push_max = d->contact_push_max, r.slop = d->contact_slop;
    r.terrain_max = -1e30f;
    r.sleeping = d->sleeping ? 1 : 0;
    r.can_sleep = d->can_sleep ? 1 : 0;
    r.sleep_speed = d->sleep_speed;
    r.max_speed = d->max_speed;
    // SoftBody::compute_aabb (softbody.cpp:271-275)
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    for (const bl_node& n : hb.nodes)
        for (int k = 0; k < 3; k++) mn[k] = (n.p[k] < mn[k]) ? n.p[k] : mn[k], mx[k] = (mx[k] < n.p[k]) ? n.p[k] : mx[k];
    for (int k = 0; k < 3; k++) r.aabb_mn[k] = mn[k], r.aabb_mx[k] = mx[k];
    hb.beam_bits = (d->allow_deform ? BB_DEFORM : 0u) | (d->allow_break ? BB_BREAK : 0u) | (d->ductile ? BB_DUCTILE : 0u);
    if (d->fem && (d->fem->n_tris > 0 || d->fem->n_members > 0)) {
        std::shared_ptr<FemModel> M;
        const int mode = c->cfg.fem_dense_front;
        const int rc = build_fem_model(d->nodes, d->info, d->n_nodes, *d->fem, hb.sections, hb.fsections, M, mode == 0 || mode == 1);
        if (!rc && mode == 3 && fem_update_count(*M) <= kAutoMultifrontal) fem_update_list(*M); // (the block-column path may be chosen)
        if (rc) return rc;
        hb.fq.assign(4 * M->node.size(), 0.0f);
        for (size_t i = 0; i < M->node.size(); i++) hb.fq[4 * i + 3] = 1.0f;
        hb.fw.assign(3 * M->node.size(), 0.0f);
        // (solve_begin's clamps, frame_fem.cpp:2525-2526)
        hb.diss = std::min(std::max(d->fem->dissipation, 0.0f), 1.0f);
        hb.theta = std::min(std::max(d->fem->theta, 0.25f + 0.5f * hb.diss), 1.0f);
        hb.fem = M;
    }
    c->bodies.push_back(std::move(hb));
    c->bodies_dirty = true;
    if (body_id) *body_id = (int32_t)c->bodies.size() - 1;
    return BL_GPU_OK;
}

int bl_gpu_step_substeps(bl_gpu_ctx* c, int32_t n, void* stream) {
    if (!c || n < 0) return BL_GPU_EINVAL;
    if (n == 0) return BL_GPU_OK;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    c->last_substeps = n;
    c->total_substeps += n;
    if (c->B == 0) return BL_GPU_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    if (!c->cfg.graphs) {
        // the plain path: every kernel of the frame launched on s, no capture (a PCG fallback always factors)
        if ((rc = order_on(c, s))) return rc;
        enqueue_frame(c, n, s);
        BL_CUDA(c, cudaGetLastError());
        c->launches += frame_launches(c, n);
        return BL_GPU_OK;
    }
    auto it = c->graphs.find(n);
    if (it == c->graphs.end()) {
        // capture the frame once on the context's stream, replay it from then on
        cudaGraph_t g = nullptr;
        BL_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_frame(c, n, c->stream);
        BL_CUDA(c, cudaStreamEndCapture(c->stream, &g));
        cudaGraphExec_t ex = nullptr;
        cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        BL_CUDA(c, e);
        it = c->graphs.emplace(n, ex).first;
    }
    if ((rc = order_on(c, s))) return rc;
    BL_CUDA(c, cudaGraphLaunch(it->second, s));
    c->launches += frame_launches(c, n);
    return BL_GPU_OK;
}

int bl_gpu_synchronize(bl_gpu_ctx* c) {
    if (!c) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    BL_CUDA(c, cudaDeviceSynchronize());
    return BL_GPU_OK;
}

static int check_body(bl_gpu_ctx* c, int32_t body) {
    if (!c || body < 0 || body >= (int32_t)c->bodies.size()) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    return ensure_committed(c);
}

int bl_gpu_download_nodes(bl_gpu_ctx* c, int32_t body, bl_node* out) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if (!out) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaDeviceSynchronize());
    const Body& r = c->bodies[body].rec;
    if (r.nnodes) BL_CUDA(c, cudaMemcpyAsync(out, c->nd.p + 2 * (size_t)r.node0, sizeof(bl_node) * r.nnodes, cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    return BL_GPU_OK;
}

int bl_gpu_upload_nodes(bl_gpu_ctx* c, int32_t body, const bl_node* nodes) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if (!nodes) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaDeviceSynchronize());
    const Body& r = c->bodies[body].rec;
    if (r.nnodes) BL_CUDA(c, cudaMemcpyAsync(c->nd.p + 2 * (size_t)r.node0, nodes, sizeof(bl_node) * r.nnodes, cudaMemcpyHostToDevice, c->stream));
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    return BL_GPU_OK;
}

int bl_gpu_download_beams(bl_gpu_ctx* c, int32_t body, bl_beam* out) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if (!out) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaDeviceSynchronize());
    const HostBody& hb = c->bodies[body];
    const Body& r = hb.rec;
    std::vector<float4> bst(r.nbeams);
    std::vector<uint32_t> meta(r.nbeams);
    std::vector<float> stress(r.nbeams);
    if (r.nbeams > 0) {
        BL_CUDA(c, cudaMemcpyAsync(bst.data(), c->bst.p + r.beam0, sizeof(float4) * r.nbeams, cudaMemcpyDeviceToHost, c->stream));
        BL_CUDA(c, cudaMemcpyAsync(meta.data(), c->bmeta.p + r.beam0, sizeof(uint32_t) * r.nbeams, cudaMemcpyDeviceToHost, c->stream));
        BL_CUDA(c, cudaMemcpyAsync(stress.data(), c->stress.p + r.beam0, sizeof(float) * r.nbeams, cudaMemcpyDeviceToHost, c->stream));
        BL_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    for (int j = 0; j < r.nbeams; j++) {
        bl_beam b = hb.beams[j];
        b.L = bst[j].x, b.max_pos = bst[j].y, b.max_neg = bst[j].z, b.strength = bst[j].w;
        b.flags = (uint8_t)((meta[j] >> 8) & 0xff);
        b.stress = stress[j];
        out[j] = b;
    }
    return BL_GPU_OK;
}

int bl_gpu_body_state(bl_gpu_ctx* c, int32_t body, bl_body_state* out) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if (!out) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaDeviceSynchronize());
    Body r;
    BL_CUDA(c, cudaMemcpyAsync(&r, c->dbodies.p + body, sizeof(Body), cudaMemcpyDeviceToHost, c->stream));
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 3; k++) out->aabb_min[k] = r.aabb_mn[k], out->aabb_max[k] = r.aabb_mx[k];
    out->max_speed = r.max_speed;
    out->sleeping = r.sleeping;
    out->static_contacts = r.static_contacts;
    out->broken_beams = r.broken_beams;
    out->sleep_timer = r.sleep_timer;
    out->repaired_nodes = r.repaired;
    out->body_contacts = r.body_contacts;
    out->wake_request = r.wake_request;
    out->fem_failures = out->fem_clamps = 0;
    if (c->NF > 0) {
        BL_CUDA(c, cudaMemcpy(&out->fem_failures, c->fem_fail.p + body, sizeof(int), cudaMemcpyDeviceToHost));
        BL_CUDA(c, cudaMemcpy(&out->fem_clamps, c->fem_clamp.p + body, sizeof(int), cudaMemcpyDeviceToHost));
    }
    return BL_GPU_OK;
}

int bl_gpu_stats(bl_gpu_ctx* c, bl_world_stats* out) {
    if (!c || !out) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    BL_CUDA(c, cudaDeviceSynchronize());
    std::memset(out, 0, sizeof(*out));
    std::vector<Body> recs(c->B);
    if (c->B) BL_CUDA(c, cudaMemcpy(recs.data(), c->dbodies.p, sizeof(Body) * c->B, cudaMemcpyDeviceToHost));
    for (const Body& r : recs) {
        if (r.sleeping) out->sleeping_bodies++;
        else out->active_bodies++, out->active_nodes += r.nnodes, out->active_beams += r.nbeams;
    }
    BL_CUDA(c, cudaMemcpy(&out->device_errors, c->deverr.p, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    out->substeps = c->last_substeps;
    out->total_substeps = c->total_substeps;
    out->kernel_launches = c->launches;
    if (c->NF > 0 && c->cfg.fem_solver != BL_GPU_FEM_CHOLESKY) { // (the factorization's kernels ran on the fallbacks)
        int st[4];
        BL_CUDA(c, cudaMemcpy(st, c->pstat.p, sizeof(st), cudaMemcpyDeviceToHost));
        out->kernel_launches += (int64_t)st[1] * c->chol_launches;
    }
    if (c->contacts_on) {
        int cnt[4];
        BL_CUDA(c, cudaMemcpy(cnt, c->counters.p, sizeof(cnt), cudaMemcpyDeviceToHost));
        int total = 0;
        BL_CUDA(c, cudaMemcpy(&total, c->pair_total.p, sizeof(int), cudaMemcpyDeviceToHost));
        out->pair_searches = cnt[0], out->contacts = cnt[1], out->pairs = total;
        for (int i = 0; i < (int)recs.size(); i++) out->islands += (recs[i].pairs && recs[i].island == i) ? 1 : 0;
    }
    return BL_GPU_OK;
}

// ---- the learned warm start's network (bl_mlp.cuh)
static int mlp_upload(bl_gpu_ctx* c, const float* w) {
    BL_CUDA(c, cudaMemcpy(c->mlp_w.p, w, sizeof(float) * kParams, cudaMemcpyHostToDevice));
    BL_CUDA(c, cudaMemset(c->mlp_m.p, 0, sizeof(float) * kParams));
    BL_CUDA(c, cudaMemset(c->mlp_v.p, 0, sizeof(float) * kParams));
    k_mlp_sync_bf16<<<(kParams + 255) / 256, 256, 0, c->stream>>>(mlp_dev(c));
    BL_CUDA(c, cudaGetLastError());
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    c->adam_t = 0;
    return BL_GPU_OK;
}

int bl_gpu_mlp_init(bl_gpu_ctx* c, uint64_t seed) {
    if (!c) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    // uniform in +-sqrt(6 / fan_in) (He), biases zero; the last layer 10x smaller (the guess starts near sl(dv) = 0)
    std::vector<float> w(kParams, 0.0f);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 1;
    auto uni = [&]() {
        x ^= x << 13, x ^= x >> 7, x ^= x << 17;
        return (float)((x >> 11) * (1.0 / 9007199254740992.0));
    };
    auto fill = [&](int off, int nout, int nin, float gain) {
        const float a = gain * std::sqrt(6.0f / (float)nin);
        for (int q = 0; q < nout * nin; q++) w[off + q] = (2.0f * uni() - 1.0f) * a;
    };
    fill(kOffW1, kHid, kIn, 1.0f), fill(kOffW2, kHid, kHid, 1.0f), fill(kOffW3, kHid, kHid, 1.0f), fill(kOffW4, kOut, kHid, 0.1f);
    return mlp_upload(c, w.data());
}

int bl_gpu_mlp_set_weights(bl_gpu_ctx* c, const float* w, int32_t n) {
    if (!c || !w || n != kParams) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    return mlp_upload(c, w);
}

int bl_gpu_mlp_get_weights(bl_gpu_ctx* c, float* w, int32_t n) {
    if (!c || !w || n != kParams) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    BL_CUDA(c, cudaDeviceSynchronize());
    BL_CUDA(c, cudaMemcpy(w, c->mlp_w.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
    return BL_GPU_OK;
}

int bl_gpu_mlp_record(bl_gpu_ctx* c, int32_t capacity) {
    if (!c || capacity < 0) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    BL_CUDA(c, cudaDeviceSynchronize());
    if (capacity == 0) {
        c->rec_on = false;
    } else {
        BL_CUDA(c, c->smp_x.alloc((size_t)kIn * capacity));
        BL_CUDA(c, c->smp_t.alloc((size_t)kOut * capacity));
        BL_CUDA(c, c->smp_w.alloc((size_t)kOut * capacity));
        BL_CUDA(c, cudaMemset(c->scount.p, 0, sizeof(int)));
        c->rec_cap = capacity, c->rec_on = true;
    }
    drop_graphs(c); // (the frames are captured again with or without the recording kernels)
    return BL_GPU_OK;
}

int bl_gpu_mlp_samples(bl_gpu_ctx* c, int32_t* n) {
    if (!c || !n) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    BL_CUDA(c, cudaDeviceSynchronize());
    int k = 0;
    BL_CUDA(c, cudaMemcpy(&k, c->scount.p, sizeof(int), cudaMemcpyDeviceToHost));
    *n = std::min(k, c->rec_cap);
    return BL_GPU_OK;
}

// one pass of k_mlp_grad over n samples (x, t, w on the device; idx: the samples, or null) and, with lr > 0, Adam
static int mlp_batch(bl_gpu_ctx* c, const float* x, const float* t, const float* w, const int* idx, int n, float lr, float* gsum, double* acc) {
    const int nblk = (n + kLanes - 1) / kLanes;
    if (c->gpart.n < (size_t)nblk * kParams) BL_CUDA(c, c->gpart.alloc((size_t)nblk * kParams));
    if (c->lpart.n < (size_t)nblk) BL_CUDA(c, c->lpart.alloc(nblk));
    const MlpDev M = mlp_dev(c);
    k_mlp_grad<<<nblk, kLanes, 0, c->stream>>>(M, x, t, w, idx, n, c->gpart.p, c->lpart.p);
    if (lr > 0) c->adam_t++;
    k_mlp_adam<<<(kParams + 255) / 256, 256, 0, c->stream>>>(M, c->gpart.p, nblk, gsum, lr, 0.9f, 0.999f, 1e-8f, std::max(c->adam_t, 1));
    if (acc) k_loss_acc<<<1, 32, 0, c->stream>>>(c->lpart.p, nblk, acc);
    BL_CUDA(c, cudaGetLastError());
    return BL_GPU_OK;
}

int bl_gpu_mlp_train(bl_gpu_ctx* c, int32_t epochs, int32_t batch, float lr, uint64_t seed, float* loss) {
    if (!c || epochs < 0 || batch < 1 || !(lr > 0)) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    BL_CUDA(c, cudaDeviceSynchronize());
    int n = 0;
    int rc = bl_gpu_mlp_samples(c, &n);
    if (rc) return rc;
    if (n == 0) return BL_GPU_ESTATE;
    BL_CUDA(c, c->sidx.alloc(n));
    DevBuf<double> acc;
    BL_CUDA(c, acc.alloc(1));
    std::vector<int> order(n);
    uint64_t x = seed * 0x9E3779B97F4A7C15ull + 7;
    auto next = [&]() {
        x ^= x << 13, x ^= x >> 7, x ^= x << 17;
        return x;
    };
    for (int e = 0; e < epochs; e++) {
        for (int i = 0; i < n; i++) order[i] = i;
        for (int i = n - 1; i > 0; i--) std::swap(order[i], order[(int)(next() % (uint64_t)(i + 1))]);
        BL_CUDA(c, cudaMemcpyAsync(c->sidx.p, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c->stream));
        BL_CUDA(c, cudaMemsetAsync(acc.p, 0, sizeof(double), c->stream));
        for (int b0 = 0; b0 < n; b0 += batch)
            if ((rc = mlp_batch(c, c->smp_x.p, c->smp_t.p, c->smp_w.p, c->sidx.p + b0, std::min(batch, n - b0), lr, nullptr, acc.p))) {
                acc.free_();
                return rc;
            }
        BL_CUDA(c, cudaStreamSynchronize(c->stream)); // (the next epoch's order overwrites sidx)
    }
    double a = 0;
    BL_CUDA(c, cudaMemcpy(&a, acc.p, sizeof(double), cudaMemcpyDeviceToHost));
    acc.free_();
    if (loss) *loss = (float)(a / n);
    return BL_GPU_OK;
}

int bl_gpu_mlp_forward(bl_gpu_ctx* c, const float* x, int32_t n, float* y) {
    if (!c || n < 0 || (n > 0 && (!x || !y))) return BL_GPU_EINVAL;
    if (n == 0) return BL_GPU_OK;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    DevBuf<float> dx, dy;
    BL_CUDA(c, dx.alloc((size_t)kIn * n));
    BL_CUDA(c, dy.alloc((size_t)kOut * n));
    BL_CUDA(c, cudaMemcpy(dx.p, x, sizeof(float) * kIn * n, cudaMemcpyHostToDevice));
    k_mlp_forward_batch<<<(n + kLanes - 1) / kLanes, kLanes, 0, c->stream>>>(mlp_dev(c), dx.p, n, dy.p);
    BL_CUDA(c, cudaGetLastError());
    BL_CUDA(c, cudaStreamSynchronize(c->stream));
    BL_CUDA(c, cudaMemcpy(y, dy.p, sizeof(float) * kOut * n, cudaMemcpyDeviceToHost));
    dx.free_(), dy.free_();
    return BL_GPU_OK;
}

int bl_gpu_mlp_gradient(bl_gpu_ctx* c, const float* x, const float* t, const float* w, int32_t n, float* grad, float* loss) {
    if (!c || n < 1 || !x || !t || !w || !grad) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    DevBuf<float> dx, dt, dw;
    DevBuf<double> acc;
    BL_CUDA(c, dx.alloc((size_t)kIn * n));
    BL_CUDA(c, dt.alloc((size_t)kOut * n));
    BL_CUDA(c, dw.alloc((size_t)kOut * n));
    BL_CUDA(c, acc.alloc(1));
    BL_CUDA(c, cudaMemcpy(dx.p, x, sizeof(float) * kIn * n, cudaMemcpyHostToDevice));
    BL_CUDA(c, cudaMemcpy(dt.p, t, sizeof(float) * kOut * n, cudaMemcpyHostToDevice));
    BL_CUDA(c, cudaMemcpy(dw.p, w, sizeof(float) * kOut * n, cudaMemcpyHostToDevice));
    BL_CUDA(c, cudaMemset(acc.p, 0, sizeof(double)));
    int rc = mlp_batch(c, dx.p, dt.p, dw.p, nullptr, n, 0.0f, c->gsum.p, acc.p);
    if (!rc) {
        BL_CUDA(c, cudaStreamSynchronize(c->stream));
        BL_CUDA(c, cudaMemcpy(grad, c->gsum.p, sizeof(float) * kParams, cudaMemcpyDeviceToHost));
        double a = 0;
        BL_CUDA(c, cudaMemcpy(&a, acc.p, sizeof(double), cudaMemcpyDeviceToHost));
        if (loss) *loss = (float)(a / n);
    }
    dx.free_(), dt.free_(), dw.free_(), acc.free_();
    return rc;
}

int bl_gpu_fem_stats(bl_gpu_ctx* c, bl_fem_stats* out) {
    if (!c || !out) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    std::memset(out, 0, sizeof(*out));
    if (c->NF == 0) return BL_GPU_OK;
    BL_CUDA(c, cudaDeviceSynchronize());
    int st[4];
    long long it = 0;
    double res[4], last = 0;
    BL_CUDA(c, cudaMemcpy(st, c->pstat.p, sizeof(st), cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(&it, c->piters.p, sizeof(it), cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(res, c->res.p, sizeof(res), cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(&last, c->plast.p, sizeof(last), cudaMemcpyDeviceToHost));
    out->pcg_solves = st[0], out->pcg_fallbacks = st[1], out->last_iterations = st[2], out->pcg_iterations = it;
    out->last_pcg_residual = last, out->max_residual = res[0], out->last_residual = res[3];
    out->columns = c->NF, out->blocks = c->NB, out->updates = c->NU, out->levels = (int64_t)c->lvl_col_ptr.size() - 1;
    out->fronts = c->fem_mode == 2 ? (int64_t)c->mf_fr.n : 0;
    out->factor_flops = c->fem_mode == 2 ? c->mf_flops : 432.0 * (double)c->NU;
    if (c->fem_mode == 2) out->levels = (int64_t)c->mf_level_ptr.size() - 1;
    if (c->any_plastic_members) {
        long long rp = 0;
        BL_CUDA(c, cudaMemcpy(&rp, c->repc.p, sizeof(rp), cudaMemcpyDeviceToHost));
        out->repasses = rp;
    }
    return BL_GPU_OK;
}

int bl_gpu_download_pairs(bl_gpu_ctx* c, int32_t* pairs, int32_t capacity, int32_t* n_pairs) {
    if (!c || !n_pairs || capacity < 0 || (capacity > 0 && !pairs)) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    *n_pairs = 0;
    if (!c->contacts_on) return BL_GPU_OK;
    BL_CUDA(c, cudaDeviceSynchronize());
    std::vector<int> poff(c->B), pcnt(c->B);
    std::vector<Body> recs(c->B);
    BL_CUDA(c, cudaMemcpy(poff.data(), c->isl_poff.p, sizeof(int) * c->B, cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(pcnt.data(), c->isl_pcnt.p, sizeof(int) * c->B, cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(recs.data(), c->dbodies.p, sizeof(Body) * c->B, cudaMemcpyDeviceToHost));
    std::vector<int4> tri(c->NTRI), nodeinfo(c->N);
    BL_CUDA(c, cudaMemcpy(tri.data(), c->dtri.p, sizeof(int4) * c->NTRI, cudaMemcpyDeviceToHost));
    BL_CUDA(c, cudaMemcpy(nodeinfo.data(), c->info.p, sizeof(int4) * c->N, cudaMemcpyDeviceToHost));
    std::vector<int2> pr;
    int w = 0;
    for (int r = 0; r < c->B; r++) { // (islands in the order of their first body)
        if (pcnt[r] <= 0) continue;
        pr.resize(pcnt[r]);
        BL_CUDA(c, cudaMemcpy(pr.data(), c->pairs.p + poff[r], sizeof(int2) * pcnt[r], cudaMemcpyDeviceToHost));
        for (const int2& p : pr) {
            if (w < capacity) {
                const int bn = nodeinfo[p.x].w, bt = tri[p.y].w >> 8;
                pairs[4 * w] = bn, pairs[4 * w + 1] = p.x - recs[bn].node0, pairs[4 * w + 2] = bt, pairs[4 * w + 3] = p.y - recs[bt].tri0;
            }
            w++;
        }
    }
    *n_pairs = w;
    return BL_GPU_OK;
}

int bl_gpu_device_nodes(bl_gpu_ctx* c, void** nodes, int32_t* total) {
    if (!c) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    if (nodes) *nodes = c->nd.p;
    if (total) *total = c->N;
    return BL_GPU_OK;
}

static int all_nodes_copy(bl_gpu_ctx* c, bl_node* host, int32_t n, void* stream, bool to_device) {
    if (!c || !host) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    if (n != c->N) return BL_GPU_EINVAL;
    if (n == 0) return BL_GPU_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    if ((rc = order_on(c, s))) return rc;
    if (to_device) BL_CUDA(c, cudaMemcpyAsync(c->nd.p, host, sizeof(bl_node) * (size_t)n, cudaMemcpyHostToDevice, s));
    else BL_CUDA(c, cudaMemcpyAsync(host, c->nd.p, sizeof(bl_node) * (size_t)n, cudaMemcpyDeviceToHost, s));
    return BL_GPU_OK;
}

int bl_gpu_upload_all_nodes(bl_gpu_ctx* c, const bl_node* nodes, int32_t n, void* stream) {
    return all_nodes_copy(c, const_cast<bl_node*>(nodes), n, stream, true);
}

int bl_gpu_download_all_nodes(bl_gpu_ctx* c, bl_node* out, int32_t n, void* stream) { return all_nodes_copy(c, out, n, stream, false); }

int bl_gpu_profile_frame(bl_gpu_ctx* c, int32_t n, void* stream, bl_frame_profile* out) {
    if (!c || !out || n <= 0) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    int rc = ensure_committed(c);
    if (rc) return rc;
    std::memset(out, 0, sizeof(*out));
    out->substeps = n;
    if (c->B == 0) return BL_GPU_OK;
    cudaStream_t s = stream ? (cudaStream_t)stream : c->stream;
    auto it = c->pgraphs.find(n);
    if (it == c->pgraphs.end()) {
        ProfGraph pg;
        pg.events.resize(6 * (size_t)n + 4);
        for (cudaEvent_t& e : pg.events) BL_CUDA(c, cudaEventCreate(&e));
        cudaGraph_t g = nullptr;
        BL_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_frame(c, n, c->stream, pg.events.data());
        BL_CUDA(c, cudaStreamEndCapture(c->stream, &g));
        cudaError_t e = cudaGraphInstantiate(&pg.exec, g, 0);
        cudaGraphDestroy(g);
        BL_CUDA(c, e);
        it = c->pgraphs.emplace(n, pg).first;
    }
    const ProfGraph& pg = it->second;
    if ((rc = order_on(c, s))) return rc;
    BL_CUDA(c, cudaGraphLaunch(pg.exec, s));
    BL_CUDA(c, cudaStreamSynchronize(s));
    c->launches += frame_launches(c, n);
    c->total_substeps += n;
    c->last_substeps = n;
    cudaError_t terr = cudaSuccess;
    auto el = [&](int a, int b) {
        float ms = 0;
        const cudaError_t e = cudaEventElapsedTime(&ms, pg.events[a], pg.events[b]);
        if (e != cudaSuccess) terr = e;
        return ms;
    };
    out->begin_ms = el(0, 1);
    for (int k = 0; k < n; k++) {
        const int b = 1 + 6 * k;
        out->search_ms += el(b, b + 1);
        out->beams_ms += el(b + 1, b + 2), out->force_ms += el(b + 2, b + 3), out->contacts_ms += el(b + 3, b + 4);
        out->integrate_ms += el(b + 4, b + 5), out->fem_ms += el(b + 5, b + 6);
    }
    out->nodes_ms = out->force_ms + out->contacts_ms + out->integrate_ms + out->fem_ms;
    out->finish_ms = el(1 + 6 * n, 3 + 6 * n);
    out->frame_ms = el(0, 3 + 6 * n);
    BL_CUDA(c, terr);
    return BL_GPU_OK;
}

int bl_gpu_set_node_force(bl_gpu_ctx* c, int32_t body, int32_t node, const float force[3]) {
    if (!c || body < 0 || body >= (int32_t)c->bodies.size() || !force) return BL_GPU_EINVAL;
    HostBody& hb = c->bodies[body];
    if (node < 0 || node >= (int32_t)hb.nodes.size()) return BL_GPU_EINVAL;
    BL_CUDA(c, cudaSetDevice(c->cfg.device));
    const bool had = !hb.ext.empty();
    if (!had) hb.ext.assign(hb.nodes.size(), make_float4(0, 0, 0, 0));
    hb.ext[node] = make_float4(force[0], force[1], force[2], 0.0f);
    if (!had || !c->committed) { // (the body's first: its flag and the array are laid out again)
        int rc = pull_state(c);
        if (rc) return rc;
        c->bodies_dirty = true;
        return BL_GPU_OK;
    }
    if (c->bodies_dirty) return BL_GPU_OK;
    BL_CUDA(c, cudaDeviceSynchronize());
    BL_CUDA(c, cudaMemcpy(c->ext.p + hb.rec.node0 + node, &hb.ext[node], sizeof(float4), cudaMemcpyHostToDevice));
    return BL_GPU_OK;
}

int bl_gpu_download_fem(bl_gpu_ctx* c, int32_t body, int32_t* n, int32_t* node, double* xd, float* q, float* w) {
    int rc = check_body(c, body);
    if (rc) return rc;
    BL_CUDA(c, cudaDeviceSynchronize());
    const HostBody& hb = c->bodies[body];
    if (n) *n = hb.fem ? (int32_t)hb.fem->node.size() : 0;
    if (!hb.fem) return BL_GPU_OK;
    int fo = 0;
    for (int bi = 0; bi < body; bi++)
        if (c->bodies[bi].fem) fo += (int)c->bodies[bi].fem->node.size();
    const int nf = (int)hb.fem->node.size();
    if (node)
        for (int i = 0; i < nf; i++) node[i] = (int32_t)hb.fem->node[i];
    if (xd) BL_CUDA(c, cudaMemcpy(xd, c->xd.p + 3 * (size_t)fo, sizeof(double) * 3 * nf, cudaMemcpyDeviceToHost));
    if (q || w) {
        std::vector<float4> tmp(nf);
        if (q) {
            BL_CUDA(c, cudaMemcpy(tmp.data(), c->fq.p + fo, sizeof(float4) * nf, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nf; i++) q[4 * i] = tmp[i].x, q[4 * i + 1] = tmp[i].y, q[4 * i + 2] = tmp[i].z, q[4 * i + 3] = tmp[i].w;
        }
        if (w) {
            BL_CUDA(c, cudaMemcpy(tmp.data(), c->fw.p + fo, sizeof(float4) * nf, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nf; i++) w[3 * i] = tmp[i].x, w[3 * i + 1] = tmp[i].y, w[3 * i + 2] = tmp[i].z;
        }
    }
    return BL_GPU_OK;
}

int bl_gpu_set_wheel_drive(bl_gpu_ctx* c, int32_t body, int32_t wheel, float torque, float brake) {
    int rc = check_body(c, body);
    if (rc) return rc;
    HostBody& hb = c->bodies[body];
    if (wheel < 0 || wheel >= (int)hb.wheels.size() || !std::isfinite(torque) || !(brake >= 0) || !std::isfinite(brake)) return BL_GPU_EINVAL;
    hb.wheels[wheel].torque = torque, hb.wheels[wheel].brake = brake;
    if (c->committed && !c->bodies_dirty && c->NWR > 0) {
        const float tb[2] = {torque, brake};
        BL_CUDA(c, cudaSetDevice(c->cfg.device));
        BL_CUDA(c, cudaMemcpy(c->dwctl.p + hb.wheel0 + wheel, tb, sizeof(tb), cudaMemcpyHostToDevice));
    }
    return BL_GPU_OK;
}

int bl_gpu_download_wheels(bl_gpu_ctx* c, int32_t body, int32_t* n, float* speed, float* avg_speed) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if ((rc = ensure_committed(c))) return rc;
    const HostBody& hb = c->bodies[body];
    const int nw = (int)hb.wheels.size();
    if (n) *n = nw;
    if (nw == 0 || (!speed && !avg_speed)) return BL_GPU_OK;
    std::vector<float4> st(nw);
    BL_CUDA(c, cudaDeviceSynchronize());
    BL_CUDA(c, cudaMemcpy(st.data(), c->dwst.p + hb.wheel0, sizeof(float4) * nw, cudaMemcpyDeviceToHost));
    for (int k = 0; k < nw; k++) {
        if (speed) speed[k] = st[k].x;
        if (avg_speed) avg_speed[k] = st[k].y;
    }
    return BL_GPU_OK;
}

int bl_gpu_wheel_speed(bl_gpu_ctx* c, int32_t body, float* wheel_speed, float* wheel_spin) {
    if (!wheel_speed || !wheel_spin) return BL_GPU_EINVAL;
    int32_t n = 0;
    int rc = bl_gpu_download_wheels(c, body, &n, nullptr, nullptr);
    if (rc) return rc;
    std::vector<float> sp(n), av(n);
    if (n > 0 && (rc = bl_gpu_download_wheels(c, body, &n, sp.data(), av.data()))) return rc;
    // (compute_wheel_forces' sums over the forward-propelled wheels in their order)
    const HostBody& hb = c->bodies[body];
    float speed_sum = 0, spin_sum = 0;
    int nprop = 0;
    for (int k = 0; k < n; k++)
        if (hb.wheels[k].propulsed == 1 && !hb.wheels[k].nodes.empty())
            speed_sum += sp[k], spin_sum += sp[k] / std::max(0.05f, hb.wheels[k].radius), nprop++;
    *wheel_speed = nprop > 0 ? speed_sum / nprop : 0.0f;
    *wheel_spin = nprop > 0 ? spin_sum / nprop : 0.0f;
    return BL_GPU_OK;
}

int bl_gpu_download_fem_tris(bl_gpu_ctx* c, int32_t body, int32_t* n, float* rest, float* frames, float* plastic_stretch) {
    int rc = check_body(c, body);
    if (rc) return rc;
    if ((rc = ensure_committed(c))) return rc;
    BL_CUDA(c, cudaDeviceSynchronize());
    const HostBody& hb = c->bodies[body];
    const int nt = hb.fem ? (int)hb.fem->tn.size() : 0;
    if (n) *n = nt;
    if (nt == 0) return BL_GPU_OK;
    size_t to = 0;
    for (int bi = 0; bi < body; bi++)
        if (c->bodies[bi].fem) to += c->bodies[bi].fem->tn.size();
    if (rest) BL_CUDA(c, cudaMemcpy(rest, c->tX.p + 6 * to, sizeof(float) * 6 * nt, cudaMemcpyDeviceToHost));
    if (frames) BL_CUDA(c, cudaMemcpy(frames, c->tr0.p + 3 * to, sizeof(float4) * 3 * nt, cudaMemcpyDeviceToHost));
    if (plastic_stretch) BL_CUDA(c, cudaMemcpy(plastic_stretch, c->tdmg.p + to, sizeof(float) * nt, cudaMemcpyDeviceToHost));
    return BL_GPU_OK;
}

int bl_gpu_body_range(bl_gpu_ctx* c, int32_t body, int32_t* first_node, int32_t* n_nodes, int32_t* first_beam, int32_t* n_beams) {
    int rc = check_body(c, body);
    if (rc) return rc;
    const Body& r = c->bodies[body].rec;
    if (first_node) *first_node = r.node0;
    if (n_nodes) *n_nodes = r.nnodes;
    if (first_beam) *first_beam = r.beam0;
    if (n_beams) *n_beams = r.nbeams;
    return BL_GPU_OK;
}

int bl_fem_pattern(const bl_node* nodes, const bl_node_info* info, int32_t n_nodes, const bl_fem_desc* fem, int32_t sizes[4], int32_t* perm,
                   int32_t* col_ptr, int32_t* row, int32_t* upd, float* rest, float* inertia) {
    if (!fem || !sizes || n_nodes < 0) return BL_GPU_EINVAL;
    std::vector<FemSection> secs;
    std::vector<FrameSectionH> fsecs;
    std::shared_ptr<FemModel> M;
    const int rc = build_fem_model(nodes, info, n_nodes, *fem, secs, fsecs, M);
    if (rc) return rc;
    const int nf = (int)M->node.size();
    sizes[0] = nf, sizes[1] = (int32_t)M->row.size(), sizes[2] = (int32_t)M->upd.size(), sizes[3] = M->ncomp;
    if (perm) std::copy(M->perm.begin(), M->perm.end(), perm);
    if (col_ptr) std::copy(M->col_ptr.begin(), M->col_ptr.end(), col_ptr);
    if (row) std::copy(M->row.begin(), M->row.end(), row);
    if (upd)
        for (size_t u = 0; u < M->upd.size(); u++) upd[3 * u] = M->upd[u][0], upd[3 * u + 1] = M->upd[u][1], upd[3 * u + 2] = M->upd[u][2];
    if (rest) std::copy(M->tX.begin(), M->tX.end(), rest);
    if (inertia) std::copy(M->inertia.begin(), M->inertia.end(), inertia);
    return BL_GPU_OK;
}

int bl_gpu_last_cuda_error(bl_gpu_ctx* c) { return c ? c->last_cuda : 0; }

} // extern "C"
