// Kernels of the implicit FEM shell step (FemFrame, src/phys/frame_fem.cpp) for bodies of triangle elements.
//
// Per substep, for every frame:
//   k_fem_begin        frame nodes: double positions re-synced where something else moved a node (frame_fem.cpp:1866-1872)
//   k_tri_eval         triangles: co-rotated frame, deformation, -K d, K v, membrane tension's geometric stiffness
//                      (tri_kinematics + eval_tris, frame_fem.cpp:1584-1621, 1661-1831; elastic sections)
//   (k_force)          the frame bodies' node forces, their triangles' forces and torques gathered in the reference's
//                      order (gather_forces, frame_fem.cpp:2080-2105)
//   k_fem_assemble_all columns and blocks: the blocks of (M + (theta h^2 + beta h) K + theta h^2 Kg) and the right side
//                      h f - (theta_d h^2 + beta h) K v (gather_part, frame_fem.cpp:916-1086)
//   k_fem_chol_level / k_fem_update_forward_level: the right-looking block Cholesky level by level of the elimination
//                      tree: the level's columns factored (chol6, right_solve_lt), then their updates T -= P Q^T, one
//                      warp per target block (frame_fem.cpp:2193-2220, 2887-2919), with the level's L y = r
//   k_fem_backward_level: L^T x = y by levels, from the top down (frame_fem.cpp:2944-2954)
//   k_fem_velocity     columns: the new velocities to forces m dv / step, spins advanced, safety clamps
//                      (frame_fem.cpp:2998-3025)
//   k_fem_integrate    the frame bodies' nodes: SoftBody::integrate_nodes, then FemFrame::sync_positions
//                      (softbody.cpp:769-795, frame_fem.cpp:3407-3422)
// The factorization's sums per block are the reference's (same 6 x 6 loops, same order of updates); the element
// kernels call the GPU's atan2 / sin / cos, which differ from libm's in the last bit, so the step matches the reference
// within a tolerance, not bitwise.
#pragma once

#include "bl_device.cuh"

namespace blg {

struct FemSecDev {
    float E, nu, rho, t, damping, drill;
    float yield;             // ShellSection::yield (Pa)
    int plastic;             // yield > 0 on a body that deforms (SoftBody::allow_deform): the triangle flows
};

// All frames of the context, back to back (frame nodes, triangles, columns, blocks in one index space each)
struct FemDev {
    int nf, ntri, nblk;
    const int* fnode;        // frame node -> global body node
    const int* fbody;        // frame node -> body
    const int* perm;         // column -> frame node
    const int* iperm;        // frame node -> column
    double* xd;              // 3 / frame node
    float4* q;               // orientation (x y z w)
    float4* w;               // angular velocity
    const float* inertia;
    float4* torque;
    const int4* tn;          // triangle: frame nodes, section
    float* tX;               // 6 / triangle: the rest shape (flows with a yielding membrane)
    float4* tr0;             // 3 / triangle: the rest frames (the bending's plastic rotations baked in)
    float* tk;               // 162 / triangle (built again where the membrane flowed)
    float* tb;               // 54 / triangle: the bending's curvatures from the corners' rotations (tri_b_)
    const float* tX0;        // 6 / triangle: the authored rest shape
    float* th0;              // 9 / triangle: the corners' plastic rest rotations (FrameTri::th0)
    float* tdmg;             // per triangle: the plastic stretch reached (FrameTri::dmg)
    const uint8_t* tbroken;
    float4* tf;              // 3 / triangle: corner forces
    float4* tt;              // 3 / triangle: corner torques
    float* ttan;             // 18 / triangle: e1 e2 e3, g[3][3]
    double* tkv;             // 18 / triangle
    uint8_t* ton;
    const FemSecDev* sec;
    const int* col_ptr;
    const int* row;
    const int* blk_col;      // block -> its column
    const int* gdiag_ptr;
    const int2* gdiag;       // (triangle, corner)
    const int* goff_ptr;
    const int4* goff;        // (triangle, row corner, column corner)
    double* diag;            // 36 / column: the assembled diagonal blocks (updated in place as the factor proceeds)
    double* ldiag;           // 36 / column: the factored diagonal blocks
    double* off;             // 36 / block
    double* rhs;             // 6 / column
    double* dinv;            // 6 / column
    uint8_t* fixed;          // / column
    const int* grp_tgt;      // per level, per target its columns update: the target (column k: k; block p: nf + p)
    const int* grp_ptr;      // ... and its updates in gu
    const int2* gu;          // (pj, pi) of each update, in the order of its source column
    const int* col_comp;     // column -> component
    int* comp_fail;
    const int* rb_ptr;       // / column: the blocks in its row, in the order of their columns
    const int2* rb;          // (block, column)
    const int* lvl_col;      // columns grouped by level
    const double* ch2;       // / column: theta h^2
    const double* chd;       // / column: theta_d h^2 (numerical dissipation)
    int* body_failures;      // / body
    int* body_clamps;        // / body
    float h, step;
    const float4* contact_n; // per frame node: its ground contact's normal this step, doubled where it sticks (null: none)
    // members (k_member_eval)
    int nmem;
    const int2* mn;          // frame nodes a, b
    const int* mmeta;        // section | joint at a << 16 | joint at b << 24; -1: broken at rest
    const float* mL0;
    float4* mq;              // 2 / member: its rest frame in a's and in b's frame (the plastic rotations baked in)
    const struct FemMemSecDev* msec;
    float4* mfa;             // force on a (on b: its negative)
    float4* mta;             // torque on a
    float4* mtb;             // torque on b
    uint8_t* mon;            // evaluated this substep (FemFrame::Tangent::on)
    float4* mtan;            // the tangent's axis e1 and N / L (its geometric stiffness)
    double* mkw;             // 144 / member: the world blocks aa, bb, ba, ab (FemFrame::mem_kw_)
    double* mkv;             // 12 / member: K v (FemFrame::mem_kv_)
    // the members' plasticity (FrameElement's plastic state, FemFrame::Tangent) and the unload re-pass
    float4* mps;             // 4 / member: (up, tp, bt, dmg_a), (pa, pb), (ba, bb), (dmg_b, -, -, -)
    float4* mtg;             // 6 / member: the tangent - (e1, L), (e2, ka), (e3, kt), (cy0 cy1 cy2 cz0), (cz1 cz2 N T),
                             // (ma, mb)
    uint32_t* mflag;         // / member: yield (bits 0-3), unload (8-11), elastic_hold (16-23)
    float* credit;           // / body: FemFrame::repass_credit_
    int* elastic;            // / body: FemFrame::elastic_step_
    int* comp_again;         // / component: bit p - pass p's check found a hinge the step unloads
    const int* comp_size;    // / component: its columns
    const int* body_comp;    // / body + 1: its components' range
    int* rp;                 // [0], [1]: a re-pass after pass 0, pass 1
    long long* repc;         // the re-passes run
    int nbody;
};

// ------------------------------------------------------------------------------------------ quaternions (math.h:105-215)
struct q4 {
    float x, y, z, w;
};
__device__ __forceinline__ q4 qmul(q4 a, q4 b) {
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
            a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
__device__ __forceinline__ q4 qconj(q4 q) { return {-q.x, -q.y, -q.z, q.w}; }
__device__ __forceinline__ q4 qnormalize(q4 q) {
    const float l = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (!(l > 1e-12f)) return {0, 0, 0, 1};
    const float i = 1.0f / l;
    return {q.x * i, q.y * i, q.z * i, q.w * i};
}
__device__ __forceinline__ q4 qfrom_mat3(v3 c0, v3 c1, v3 c2) {
    const float m00 = c0.x, m11 = c1.y, m22 = c2.z;
    const float tr = m00 + m11 + m22;
    q4 q{0, 0, 0, 1};
    if (tr > 0) {
        const float s = sqrtf(tr + 1.0f) * 2;
        q.w = 0.25f * s, q.x = (c1.z - c2.y) / s, q.y = (c2.x - c0.z) / s, q.z = (c0.y - c1.x) / s;
    } else if (m00 > m11 && m00 > m22) {
        const float s = sqrtf(1.0f + m00 - m11 - m22) * 2;
        q.w = (c1.z - c2.y) / s, q.x = 0.25f * s, q.y = (c1.x + c0.y) / s, q.z = (c2.x + c0.z) / s;
    } else if (m11 > m22) {
        const float s = sqrtf(1.0f + m11 - m00 - m22) * 2;
        q.w = (c2.x - c0.z) / s, q.x = (c1.x + c0.y) / s, q.y = 0.25f * s, q.z = (c2.y + c1.z) / s;
    } else {
        const float s = sqrtf(1.0f + m22 - m00 - m11) * 2;
        q.w = (c0.y - c1.x) / s, q.x = (c2.x + c0.z) / s, q.y = (c2.y + c1.z) / s, q.z = 0.25f * s;
    }
    return qnormalize(q);
}
__device__ __forceinline__ v3 quat_log(q4 qin) {
    const q4 q = qin.w < 0 ? q4{qin.x * -1.0f, qin.y * -1.0f, qin.z * -1.0f, qin.w * -1.0f} : qin;
    const v3 v = V(q.x, q.y, q.z);
    const float s = length(v);
    if (s < 1e-8f) return v * 2.0f;
    const float angle = 2.0f * atan2f(s, q.w);
    return v * (angle / s);
}
__device__ __forceinline__ q4 quat_exp(v3 rv) {
    const float a = length(rv);
    if (a < 1e-8f) return qnormalize(q4{rv.x * 0.5f, rv.y * 0.5f, rv.z * 0.5f, 1.0f});
    const v3 ax = normalize(divs(rv, a));
    const float hh = a * 0.5f, s = sinf(hh);
    return {ax.x * s, ax.y * s, ax.z * s, cosf(hh)};
}

__device__ __forceinline__ double dmax0(double x) { return (0.0 < x) ? x : 0.0; }

// ------------------------------------------------------------------------------------------ per frame node
__global__ void k_fem_begin(FemDev F, const float4* __restrict__ nd) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.nf) return;
    const float4 p = nd[2 * F.fnode[i]];
    double* x = F.xd + 3 * (size_t)i;
    if ((float)x[0] != p.x || (float)x[1] != p.y || (float)x[2] != p.z) x[0] = p.x, x[1] = p.y, x[2] = p.z;
}

// ------------------------------------------------------------------------------------------ per triangle
// the element built again where its membrane flowed (tri_build_k, frame_fem.cpp:1625-1647): out of line, its 18 x 18
// doubles in local memory only for the triangles that flow
__device__ __noinline__ void tri_rebuild_k(FemDev F, int ti, const FemSecDev& s, const float X[3][2]) {
    tri_local_k(X, TriSec{s.E, s.nu, s.t, s.drill}, F.tk + 162 * (size_t)ti, F.tb + 54 * (size_t)ti);
}

__device__ __forceinline__ double von_mises(const double m[3]) {
    const double v = m[0] * m[0] - m[0] * m[1] + m[1] * m[1] + 3 * m[2] * m[2];
    return sqrt((0.0 < v) ? v : 0.0);
}

// A yielding shell section (the flow eval_tris applies on a body that does not break, frame_fem.cpp:1690-1741), in
// three steps of this file's own:
//  membrane_return: where the membrane's von Mises stress exceeds the yield stress, the stress is returned radially to
//    the yield surface: the fraction r = 1 - yield / sigma_eq of the in-plane displacements becomes permanent - the rest
//    shape moves by it (then recentred on its centroid) and the element is built again - and the plastic stretch
//    reached (the largest principal stretch of the rest shape against the authored one) is kept in dmg;
//  bending_return: the same on the largest von Mises moment of the three sample points against the plate's plastic
//    moment yield t^2 / 4: the corners' plastic rotations take the fraction r of their bending rotations;
//  bake_rotations: a corner's plastic rotation past 0.02 rad goes into its rest frame.
// X, th0, d, b3 / c3 / A2 and sig are the caller's and are updated.
__device__ __forceinline__ float principal_stretch(const float* X0, const float X[3][2]) {
    // F maps the authored edges (from corner 0) to the current rest edges; the stretch is sqrt of C = F^T F's larger
    // eigenvalue, less one (0 where the authored shape is degenerate)
    const double e0[2][2] = {{(double)X0[2] - X0[0], (double)X0[4] - X0[0]}, {(double)X0[3] - X0[1], (double)X0[5] - X0[1]}};
    const double e[2][2] = {{(double)X[1][0] - X[0][0], (double)X[2][0] - X[0][0]}, {(double)X[1][1] - X[0][1], (double)X[2][1] - X[0][1]}};
    const double det = e0[0][0] * e0[1][1] - e0[0][1] * e0[1][0];
    if (!(fabs(det) > 1e-12)) return 0.0f;
    const double inv[2][2] = {{e0[1][1] / det, -e0[0][1] / det}, {-e0[1][0] / det, e0[0][0] / det}};
    double Fm[2][2];
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) Fm[i][j] = e[i][0] * inv[0][j] + e[i][1] * inv[1][j];
    const double c00 = Fm[0][0] * Fm[0][0] + Fm[1][0] * Fm[1][0], c11 = Fm[0][1] * Fm[0][1] + Fm[1][1] * Fm[1][1];
    const double c01 = Fm[0][0] * Fm[0][1] + Fm[1][0] * Fm[1][1];
    const double lmax = 0.5 * (c00 + c11 + sqrt((c00 - c11) * (c00 - c11) + 4 * c01 * c01));
    return (float)(sqrt(lmax) - 1.0);
}

template <class Membrane>
__device__ __forceinline__ bool membrane_return(FemDev F, int ti, const FemSecDev& s, float X[3][2], double d[18], double b3[3], double c3[3],
                                                double& A2, const double sig[3], float& dmg, Membrane membrane) {
    const double seq = von_mises(sig);
    if (!(seq > s.yield)) return false;
    const double r = 1.0 - s.yield / seq;
    for (int i = 0; i < 3; i++)
        for (int a = 0; a < 2; a++) X[i][a] += (float)(r * d[6 * i + a]), d[6 * i + a] *= 1 - r;
    const float mx = (X[0][0] + X[1][0] + X[2][0]) / 3.0f, my = (X[0][1] + X[1][1] + X[2][1]) / 3.0f;
    for (int i = 0; i < 3; i++) X[i][0] -= mx, X[i][1] -= my;
    dmg = smax(dmg, principal_stretch(F.tX0 + 6 * (size_t)ti, X));
    tri_rebuild_k(F, ti, s, X);
    tri_grad(X, b3, c3, A2);
    membrane();
    return true;
}

__device__ __forceinline__ void bending_return(FemDev F, int ti, const FemSecDev& s, v3 th0[3], double d[18], float& dmg) {
    const float* Bc = F.tb + 54 * (size_t)ti;
    const double D = s.E * s.t * s.t * s.t / (12.0f * (1.0f - s.nu * s.nu)), nu = s.nu, Mp = 0.25 * s.yield * (double)s.t * s.t;
    double worst = 0;
    for (int pt = 0; pt < 3; pt++) {
        const float* Bp = Bc + 18 * pt;
        double k[3];
        for (int row = 0; row < 3; row++) {
            k[row] = 0;
            for (int i = 0; i < 3; i++) k[row] += Bp[6 * row + 2 * i] * d[6 * i + 3] + Bp[6 * row + 2 * i + 1] * d[6 * i + 4];
        }
        const double m[3] = {D * (k[0] + nu * k[1]), D * (nu * k[0] + k[1]), D * 0.5 * (1 - nu) * k[2]};
        const double vm = von_mises(m);
        worst = (worst < vm) ? vm : worst;
    }
    if (!(worst > Mp)) return;
    const double r = 1.0 - Mp / worst;
    for (int i = 0; i < 3; i++) {
        th0[i].x += (float)(r * d[6 * i + 3]), th0[i].y += (float)(r * d[6 * i + 4]);
        d[6 * i + 3] *= 1 - r, d[6 * i + 4] *= 1 - r;
    }
    dmg = smax(dmg, 1e-5f);
}

__device__ __forceinline__ void bake_rotations(FemDev F, int ti, v3 th0[3]) {
    for (int i = 0; i < 3; i++) {
        if (!(dot(th0[i], th0[i]) > 0.02f * 0.02f)) continue;
        const float4 rf = F.tr0[3 * ti + i];
        const q4 r0 = qnormalize(qmul(q4{rf.x, rf.y, rf.z, rf.w}, quat_exp(V(-th0[i].x, -th0[i].y, -th0[i].z))));
        F.tr0[3 * ti + i] = make_float4(r0.x, r0.y, r0.z, r0.w);
        th0[i] = V(0, 0, 0);
    }
}

template <class Membrane>
__device__ void tri_plastic_flow(FemDev F, int ti, const FemSecDev& s, float X[3][2], v3 th0[3], double d[18], double b3[3], double c3[3],
                                 double& A2, const double sig[3], Membrane membrane) {
    float dmg = F.tdmg[ti];
    const bool rest_moved = membrane_return(F, ti, s, X, d, b3, c3, A2, sig, dmg, membrane);
    bending_return(F, ti, s, th0, d, dmg);
    bake_rotations(F, ti, th0);
    if (rest_moved)
        for (int i = 0; i < 3; i++) F.tX[6 * ti + 2 * i] = X[i][0], F.tX[6 * ti + 2 * i + 1] = X[i][1];
    for (int i = 0; i < 3; i++) F.th0[9 * ti + 3 * i] = th0[i].x, F.th0[9 * ti + 3 * i + 1] = th0[i].y, F.th0[9 * ti + 3 * i + 2] = th0[i].z;
    F.tdmg[ti] = dmg;
}

// kPlastic: the variant for contexts with a yielding section (its flow's registers and the element's rebuild kept out
// of the elastic one)
template <bool kPlastic>
__global__ void __launch_bounds__(128) k_tri_eval(FemDev F, const float4* __restrict__ nd) {
    const int ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= F.ntri) return;
    F.ton[ti] = 0;
    if (F.tbroken[ti]) return;
    const int4 tn = F.tn[ti];
    const int fnv[3] = {tn.x, tn.y, tn.z};
    const FemSecDev s = F.sec[tn.w];
    float X[3][2];
    for (int i = 0; i < 3; i++) X[i][0] = F.tX[6 * ti + 2 * i], X[i][1] = F.tX[6 * ti + 2 * i + 1];
    v3 th0[3];
    for (int i = 0; i < 3; i++) th0[i] = kPlastic ? V(F.th0[9 * ti + 3 * i], F.th0[9 * ti + 3 * i + 1], F.th0[9 * ti + 3 * i + 2]) : V(0, 0, 0);
    // ---- the co-rotated frame (tri_kinematics, frame_fem.cpp:1584-1621, defines the same one): the plane's normal n
    // from the corners, a first in-plane axis t1 along the edge 0 -> 1, then the in-plane rotation that best aligns the
    // rest shape with the current corners about their centroid. That rotation is the least-squares one: its cosine and
    // sine are the normalised sums of the dot and cross products of rest and current corner vectors, so no angle is
    // formed. The local displacements are the corners' coordinates on the aligned axes less the rest shape; the
    // corners' rotations are their frames' rotations relative to the element's, as rotation vectors.
    double x[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) x[i][j] = F.xd[3 * (size_t)fnv[i] + j];
    double r[3][3], u01[3], u02[3], n[3];
    for (int j = 0; j < 3; j++) {
        const double cj = (x[0][j] + x[1][j] + x[2][j]) / 3.0;
        for (int i = 0; i < 3; i++) r[i][j] = x[i][j] - cj;
        u01[j] = x[1][j] - x[0][j], u02[j] = x[2][j] - x[0][j];
    }
    n[0] = u01[1] * u02[2] - u01[2] * u02[1], n[1] = u01[2] * u02[0] - u01[0] * u02[2], n[2] = u01[0] * u02[1] - u01[1] * u02[0];
    const double nl = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]), al = sqrt(u01[0] * u01[0] + u01[1] * u01[1] + u01[2] * u01[2]);
    if (!(nl > 1e-12) || !(al > 1e-9) || !isfinite(nl)) return;
    double t1[3], t2[3];
    for (int j = 0; j < 3; j++) n[j] /= nl, t1[j] = u01[j] / al;
    t2[0] = n[1] * t1[2] - n[2] * t1[1], t2[1] = n[2] * t1[0] - n[0] * t1[2], t2[2] = n[0] * t1[1] - n[1] * t1[0];
    double dotsum = 0, crosssum = 0;
    for (int i = 0; i < 3; i++) {
        const double px = r[i][0] * t1[0] + r[i][1] * t1[1] + r[i][2] * t1[2], py = r[i][0] * t2[0] + r[i][1] * t2[1] + r[i][2] * t2[2];
        dotsum += X[i][0] * px + X[i][1] * py, crosssum += X[i][0] * py - X[i][1] * px;
    }
    const double rot = sqrt(dotsum * dotsum + crosssum * crosssum);
    const double cp = rot > 0 ? dotsum / rot : 1.0, sp = rot > 0 ? crosssum / rot : 0.0;
    double e1d[3], e2d[3];
    for (int j = 0; j < 3; j++) e1d[j] = cp * t1[j] + sp * t2[j], e2d[j] = cp * t2[j] - sp * t1[j];
    const v3 e1 = V((float)e1d[0], (float)e1d[1], (float)e1d[2]), e2 = V((float)e2d[0], (float)e2d[1], (float)e2d[2]);
    const v3 e3 = V((float)n[0], (float)n[1], (float)n[2]);
    const q4 Ec = qconj(qfrom_mat3(e1, e2, e3));
    double d[18];
    for (int i = 0; i < 3; i++) {
        d[6 * i] = r[i][0] * e1d[0] + r[i][1] * e1d[1] + r[i][2] * e1d[2] - X[i][0];
        d[6 * i + 1] = r[i][0] * e2d[0] + r[i][1] * e2d[1] + r[i][2] * e2d[2] - X[i][1];
        d[6 * i + 2] = 0;
        const float4 qf = F.q[fnv[i]], rf = F.tr0[3 * ti + i];
        const q4 corner = qnormalize(qmul(q4{qf.x, qf.y, qf.z, qf.w}, q4{rf.x, rf.y, rf.z, rf.w})); // (the corner's frame)
        const v3 th = quat_log(qmul(Ec, corner)) - th0[i];
        d[6 * i + 3] = th.x, d[6 * i + 4] = th.y, d[6 * i + 5] = th.z;
    }
    // ---- eval_tris (frame_fem.cpp:1661-1831)
    double b3[3], c3[3], A2;
    tri_grad(X, b3, c3, A2);
    if (!(A2 > 0)) return;
    const double nu = s.nu, Dm = (double)s.E / (1 - nu * nu);
    double sig[3];
    // the constant membrane strain (du/dx, dv/dy, du/dy + dv/dx from the area coordinates' gradients) and its
    // plane-stress stress
    auto membrane = [&]() {
        double ux = 0, vy = 0, shear = 0;
        for (int i = 0; i < 3; i++) {
            const double gx = b3[i] / A2, gy = c3[i] / A2, u = d[6 * i], v = d[6 * i + 1];
            ux += gx * u, vy += gy * v, shear += gy * u + gx * v;
        }
        sig[0] = Dm * (ux + nu * vy), sig[1] = Dm * (nu * ux + vy), sig[2] = Dm * 0.5 * (1 - nu) * shear;
    };
    membrane();
    if (kPlastic && s.plastic) tri_plastic_flow(F, ti, s, X, th0, d, b3, c3, A2, sig, membrane);
    const float* Km = F.tk + 162 * (size_t)ti;
    const float* Kp = Km + 81;
    double vl[18];
    {
        const double E[3][3] = {{e1.x, e2.x, e3.x}, {e1.y, e2.y, e3.y}, {e1.z, e2.z, e3.z}};
        for (int i = 0; i < 3; i++) {
            const float4 vv = nd[2 * F.fnode[fnv[i]] + 1], om = F.w[fnv[i]];
            for (int a2 = 0; a2 < 3; a2++) {
                vl[6 * i + a2] = E[0][a2] * vv.x + E[1][a2] * vv.y + E[2][a2] * vv.z;
                vl[6 * i + 3 + a2] = E[0][a2] * om.x + E[1][a2] * om.y + E[2][a2] * om.z;
            }
        }
    }
    const int kMem[3] = {0, 1, 5}, kPlate[3] = {2, 3, 4};
    double f[18], fl[18];
    {
        double dm[9], dp[9], vm[9], vp[9];
        for (int a = 0; a < 9; a++) {
            const int ci = 6 * (a / 3);
            dm[a] = d[ci + kMem[a % 3]], dp[a] = d[ci + kPlate[a % 3]];
            vm[a] = vl[ci + kMem[a % 3]], vp[a] = vl[ci + kPlate[a % 3]];
        }
        double fm[9] = {}, fp[9] = {}, um[9] = {}, up[9] = {};
        for (int cc = 0; cc < 9; cc++)
            for (int a = 0; a < 9; a++) {
                const double km = (double)Km[cc * 9 + a], kp = (double)Kp[cc * 9 + a];
                fm[a] += km * dm[cc], um[a] += km * vm[cc];
                fp[a] += kp * dp[cc], up[a] += kp * vp[cc];
            }
        for (int a = 0; a < 9; a++) {
            const int ci = 6 * (a / 3);
            f[ci + kMem[a % 3]] = fm[a], fl[ci + kMem[a % 3]] = um[a];
            f[ci + kPlate[a % 3]] = fp[a], fl[ci + kPlate[a % 3]] = up[a];
        }
    }
    for (int i = 0; i < 3; i++) {
        const v3 fo = e1 * (float)f[6 * i] + e2 * (float)f[6 * i + 1] + e3 * (float)f[6 * i + 2];
        const v3 to = e1 * (float)f[6 * i + 3] + e2 * (float)f[6 * i + 4] + e3 * (float)f[6 * i + 5];
        F.tf[3 * ti + i] = make_float4(-fo.x, -fo.y, -fo.z, 0.0f);
        F.tt[3 * ti + i] = make_float4(-to.x, -to.y, -to.z, 0.0f);
    }
    float* tg = F.ttan + 18 * (size_t)ti;
    tg[0] = e1.x, tg[1] = e1.y, tg[2] = e1.z, tg[3] = e2.x, tg[4] = e2.y, tg[5] = e2.z, tg[6] = e3.x, tg[7] = e3.y, tg[8] = e3.z;
    {
        const double sx = sig[0] * s.t, sy = sig[1] * s.t, sxy = sig[2] * s.t;
        const double tr = 0.5 * (sx + sy), df = sqrt(0.25 * (sx - sy) * (sx - sy) + sxy * sxy);
        const double l1 = dmax0(tr + df), l2 = dmax0(tr - df);
        double vx = sxy, vy = l1 - sx;
        if (fabs(vx) + fabs(vy) < 1e-12 * (fabs(sx) + fabs(sy) + 1)) vx = sx >= sy ? 1 : 0, vy = sx >= sy ? 0 : 1;
        const double vln = sqrt(vx * vx + vy * vy);
        vx /= vln, vy /= vln;
        const double S00 = l1 * vx * vx + l2 * vy * vy, S01 = (l1 - l2) * vx * vy, S11 = l1 * vy * vy + l2 * vx * vx;
        const double A = 0.5 * A2;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const double gi0 = b3[i] / A2, gi1 = c3[i] / A2, gj0 = b3[j] / A2, gj1 = c3[j] / A2;
                tg[9 + 3 * i + j] = (float)(A * (gi0 * (S00 * gj0 + S01 * gj1) + gi1 * (S01 * gj0 + S11 * gj1)));
            }
    }
    {
        const double E[3][3] = {{e1.x, e2.x, e3.x}, {e1.y, e2.y, e3.y}, {e1.z, e2.z, e3.z}};
        double* kv = F.tkv + 18 * (size_t)ti;
        for (int i = 0; i < 3; i++)
            for (int pp = 0; pp < 3; pp++) {
                kv[6 * i + pp] = E[pp][0] * fl[6 * i] + E[pp][1] * fl[6 * i + 1] + E[pp][2] * fl[6 * i + 2];
                kv[6 * i + 3 + pp] = E[pp][0] * fl[6 * i + 3] + E[pp][1] * fl[6 * i + 4] + E[pp][2] * fl[6 * i + 5];
            }
    }
    F.ton[ti] = 1;
}

// ------------------------------------------------------------------------------------------ members (frame beams)
// FemFrame::eval_forces for elastic members (frame_fem.cpp:1896-2070 with no plastic limits: Np = Mp = Tp = 0, no
// joint damping, no break force): the co-rotated frame (kinematics, frame_fem.cpp:1384-1406), the joints' end
// stiffnesses (stiffness, frame_fem.cpp:1408-1476), the axial force, torque and end moments, the nodal forces
// -B^T g, the tangent and its world blocks with K v (member_world_k / element_matrix, frame_fem.cpp:1834-1850,
// 2157-2186), a thread a member, float where the reference is float and double where it is double.
constexpr float kPi = 3.14159265358979323846f;

struct FemMemSecDev { // FrameSection (frame_fem.h:90-112)
    float E, G, rho, A, Iy, Iz, J, As_y, As_z, damping, axial, joint_k;
    float Np, Mp, Tp, hardening;
    int plastic;             // Np > 0 on a body that deforms: the member yields (eval_forces' plastic)
};
enum : int { FJ_RIGID = 0, FJ_BALL = 1, FJ_HINGE_V = 2, FJ_HINGE_H = 3, FJ_SWIVEL = 4, FJ_ELASTIC = 5 };

__device__ __forceinline__ v3 cross3(v3 a, v3 b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
__device__ __forceinline__ v3 qrotate(q4 q, v3 p) { // quat::rotate (math.h:150-154)
    const v3 u = V(q.x, q.y, q.z);
    const v3 t = cross3(u, p) * 2.0f;
    return p + t * q.w + cross3(u, t);
}
__device__ __forceinline__ q4 qscale(q4 q, float s) { return {q.x * s, q.y * s, q.z * s, q.w * s}; }
__device__ __forceinline__ q4 qadd(q4 a, q4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
// quat::axis_angle (math.h:136-140)
__device__ __forceinline__ q4 qaxis_angle(v3 axis, float angle) {
    const float h = angle * 0.5f, s = sinf(h);
    const v3 a = normalize(axis);
    return {a.x * s, a.y * s, a.z * s, cosf(h)};
}
// quat_from_to (math.h:203-212): the minimal rotation taking unit a to unit b
__device__ __forceinline__ q4 qfrom_to(v3 a, v3 b) {
    const float d = dot(a, b);
    if (d < -0.999999f) {
        const v3 t = fabsf(a.x) < 0.7f ? V(1, 0, 0) : V(0, 1, 0); // (any_perpendicular, math.h:82-85)
        return qaxis_angle(normalize(cross3(a, t)), 3.14159265358979323846f);
    }
    const v3 c = cross3(a, b);
    return qnormalize(q4{c.x, c.y, c.z, 1.0f + d});
}
// slerp (math.h:227-232)
__device__ __forceinline__ q4 qslerp(q4 a, q4 b, float t) {
    float d = a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
    if (d < 0) b = qscale(b, -1.0f), d = -d;
    if (d > 0.9995f) return qnormalize(qadd(a, qscale(qadd(b, qscale(a, -1.0f)), t)));
    const float th = acosf(d), s = sinf(th);
    return qadd(qscale(a, sinf((1 - t) * th) / s), qscale(b, sinf(t * th) / s));
}

// A member end's joint (FemFrame's joint kinds, frame_fem.cpp:1420-1431): what it frees - the twist, the rotation about
// the member's y, about its z - and, for an elastic joint, its compliance (rad per N m).
struct JointEnd {
    bool free_twist, free_y, free_z;
    double flex;
};
__device__ __forceinline__ JointEnd joint_end(int kind, float joint_k) {
    JointEnd j{kind == FJ_BALL || kind == FJ_SWIVEL, kind == FJ_BALL || kind == FJ_HINGE_H, kind == FJ_BALL || kind == FJ_HINGE_V, 0.0};
    if (kind == FJ_ELASTIC && joint_k > 0) j.flex = 1.0 / (double)joint_k;
    return j;
}

// One bending plane's end stiffness [aa, ab, bb]: (M_a, M_b) = K (theta_a, theta_b). Built from the Timoshenko member's
// flexibility, F = L / (6 EI) [2 -1; -1 2] + 1 / (G As L) [1 1; 1 1] (the second term its shear, none without a
// shear area), with each held end's joint compliance added on its diagonal, then inverted. A released end carries no
// moment: only the other end's entry is left, the inverse of its own diagonal flexibility (its joint's included);
// with both released the plane carries nothing. (The same stiffness as stiffness / ends2, frame_fem.cpp:1414-1476.)
__device__ __forceinline__ void end_pair(float out[3], float E, float I, float G, float As, float L, bool free_a, bool free_b, double flex_a,
                                         double flex_b) {
    out[0] = out[1] = out[2] = 0.0f;
    if (!free_a && !free_b && flex_a == 0 && flex_b == 0) {
        // both ends held rigidly: the inverse in closed form, the Timoshenko element's end-moment stiffness
        // EI / (L (1 + phi)) [4 + phi, 2 - phi; 2 - phi, 4 + phi] with phi = 12 EI / (G As L^2), in float as the
        // section's stiffness is stored
        const float phi = As > 0 ? 12.0f * E * I / (G * As * L * L) : 0.0f;
        const float k0 = E * I / (L * (1.0f + phi));
        out[0] = out[2] = (4.0f + phi) * k0;
        out[1] = (2.0f - phi) * k0;
        return;
    }
    const double EI = (double)E * I;
    if (!(EI > 0) || (free_a && free_b)) return;
    const double bend = L / (6.0 * EI), shear = As > 0 ? 1.0 / ((double)G * As * L) : 0.0;
    const double faa = 2 * bend + shear + flex_a, fbb = 2 * bend + shear + flex_b, fab = -bend + shear;
    if (free_a) {
        out[2] = (float)(1.0 / fbb);
    } else if (free_b) {
        out[0] = (float)(1.0 / faa);
    } else {
        const double det = faa * fbb - fab * fab;
        if (!(det > 0)) return;
        out[0] = (float)(fbb / det), out[1] = (float)(-fab / det), out[2] = (float)(faa / det);
    }
}

// FemFrame::condense (frame_fem.cpp:1414-1418), for the tangent of a flowing hinge: the end turns freely, so the
// plane's pair keeps only the other end's condensed stiffness (its Schur complement)
__device__ __forceinline__ void condense(float c[3], bool pin_a, bool pin_b) {
    if (pin_a && pin_b) c[0] = c[1] = c[2] = 0;
    else if (pin_a) c[2] = c[0] > 0 ? c[2] - c[1] * c[1] / c[0] : 0, c[0] = c[1] = 0;
    else if (pin_b) c[0] = c[2] > 0 ? c[0] - c[1] * c[1] / c[2] : 0, c[1] = c[2] = 0;
}

// The member's tangent in world axes (member_world_k / element_matrix, frame_fem.cpp:1834-1850, 2157-2186, of the
// effective tangent FemFrame::effective gives, frame_fem.cpp:2147-2155: the flowing parts its yield bits less its
// unload bits name - hinges condensed, axial and twist at 1 %), as K = B^T D B: B maps the 12 end dofs
// [u_a, phi_a, u_b, phi_b] to the six deformations - elongation e1.(u_b - u_a), twist e1.(phi_b - phi_a), each end's
// rotation about e2 against the chord e2.phi + e3.(u_b - u_a) / L and about e3 e3.phi - e2.(u_b - u_a) / L - and D is
// ka, kt and the two planes' end pairs. Stored as its four 6 x 6 world blocks with K v at the ends' velocities.
__device__ void member_world_k(const FemDev& F, const float4* __restrict__ nd, int ei, int2 ab, v3 e1, v3 e2, v3 e3, float L, float ka, float kt,
                               const float cy_in[3], const float cz_in[3], uint32_t y) {
    float cy[3] = {cy_in[0], cy_in[1], cy_in[2]}, cz[3] = {cz_in[0], cz_in[1], cz_in[2]};
    if (y & 3) condense(cy, y & 1, y & 2), condense(cz, y & 1, y & 2);
    if (y & 4) ka *= 0.01f;
    if (y & 8) kt *= 0.01f;
    const double iL = 1.0 / L;
    const double a1[3] = {e1.x, e1.y, e1.z}, a2[3] = {e2.x, e2.y, e2.z}, a3[3] = {e3.x, e3.y, e3.z};
    double B[6][12];
    for (int r = 0; r < 6; r++)
        for (int q = 0; q < 12; q++) B[r][q] = 0;
    for (int j = 0; j < 3; j++) {
        const double g = a3[j] * iL, h = a2[j] * iL;
        B[0][j] = -a1[j], B[0][6 + j] = a1[j];
        B[1][3 + j] = -a1[j], B[1][9 + j] = a1[j];
        B[2][j] = -g, B[2][6 + j] = g, B[2][3 + j] = a2[j];
        B[3][j] = -g, B[3][6 + j] = g, B[3][9 + j] = a2[j];
        B[4][j] = h, B[4][6 + j] = -h, B[4][3 + j] = a3[j];
        B[5][j] = h, B[5][6 + j] = -h, B[5][9 + j] = a3[j];
    }
    double DB[6][12];
    for (int q = 0; q < 12; q++) {
        DB[0][q] = (double)ka * B[0][q], DB[1][q] = (double)kt * B[1][q];
        DB[2][q] = (double)cy[0] * B[2][q] + (double)cy[1] * B[3][q], DB[3][q] = (double)cy[1] * B[2][q] + (double)cy[2] * B[3][q];
        DB[4][q] = (double)cz[0] * B[4][q] + (double)cz[1] * B[5][q], DB[5][q] = (double)cz[1] * B[4][q] + (double)cz[2] * B[5][q];
    }
    double K[12][12];
    for (int r = 0; r < 12; r++)
        for (int q = r; q < 12; q++) {
            double v = 0;
            for (int k = 0; k < 6; k++) v += B[k][r] * DB[k][q];
            K[r][q] = K[q][r] = v;
        }
    double* W = F.mkw + 144 * (size_t)ei;
    for (int r = 0; r < 6; r++)
        for (int q = 0; q < 6; q++)
            W[r * 6 + q] = K[r][q], W[36 + r * 6 + q] = K[6 + r][6 + q], W[72 + r * 6 + q] = K[6 + r][q], W[108 + r * 6 + q] = K[r][6 + q];
    const float4 va = nd[2 * F.fnode[ab.x] + 1], vb = nd[2 * F.fnode[ab.y] + 1], wa = F.w[ab.x], wb = F.w[ab.y];
    const double u[12] = {va.x, va.y, va.z, wa.x, wa.y, wa.z, vb.x, vb.y, vb.z, wb.x, wb.y, wb.z};
    double* kv = F.mkv + 12 * (size_t)ei;
    for (int r = 0; r < 12; r++) {
        double s2 = 0;
        for (int q = 0; q < 12; q++) s2 += K[r][q] * u[q];
        kv[r] = s2;
    }
}

template <bool kPlastic>
__global__ void __launch_bounds__(128) k_member_eval(FemDev F, const float4* __restrict__ nd) {
    const int ei = blockIdx.x * blockDim.x + threadIdx.x;
    if (ei >= F.nmem) return;
    F.mon[ei] = 0;
    const int meta = F.mmeta[ei];
    if (meta < 0) return; // (broken: no length at rest)
    const int2 ab = F.mn[ei];
    const int endA = (meta >> 16) & 0xff, endB = (meta >> 24) & 0x7f;
    const FemMemSecDev s = F.msec[meta & 0xffff];
    const float L0 = F.mL0[ei];
    // ---- kinematics
    const double* xa = F.xd + 3 * (size_t)ab.x;
    const double* xb = F.xd + 3 * (size_t)ab.y;
    const double dx = xb[0] - xa[0], dy = xb[1] - xa[1], dz = xb[2] - xa[2];
    const double Ld = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(Ld > 1e-6) || !isfinite(Ld)) return;
    const float L = (float)Ld;
    const double dL = Ld - (double)L0;
    const v3 e1 = V((float)(dx / Ld), (float)(dy / Ld), (float)(dz / Ld));
    const float4 qa4 = F.q[ab.x], qb4 = F.q[ab.y], ra4 = F.mq[2 * ei], rb4 = F.mq[2 * ei + 1];
    const q4 Ea = qnormalize(qmul(q4{qa4.x, qa4.y, qa4.z, qa4.w}, q4{ra4.x, ra4.y, ra4.z, ra4.w}));
    const q4 Eb = qnormalize(qmul(q4{qb4.x, qb4.y, qb4.z, qb4.w}, q4{rb4.x, rb4.y, rb4.z, rb4.w}));
    const bool fta = endA == FJ_BALL || endA == FJ_SWIVEL, ftb = endB == FJ_BALL || endB == FJ_SWIVEL;
    const float tw8 = fta == ftb ? 0.5f : fta ? 1.0f : 0.0f; // (twist_weight, frame_fem.cpp:1372-1375)
    const q4 Em = tw8 <= 0.0f ? Ea : tw8 >= 1.0f ? Eb : qslerp(Ea, Eb, tw8);
    const q4 E = qnormalize(qmul(qfrom_to(normalize(qrotate(Em, V(1, 0, 0))), e1), Em));
    const q4 Ec = qconj(E);
    const v3 ra = quat_log(qmul(Ec, Ea)), rb = quat_log(qmul(Ec, Eb));
    const v3 e2 = qrotate(E, V(0, 1, 0)), e3 = qrotate(E, V(0, 0, 1));
    // ---- the section's stiffness with the joints: axial, twist (a freed twist carries none; elastic joints add their
    // compliances in series) and the two bending planes' end pairs
    const JointEnd ja = joint_end(endA, s.joint_k), jb = joint_end(endB, s.joint_k);
    const float ka = s.axial * s.E * s.A / L0;
    const float kt = (ja.free_twist || jb.free_twist) ? 0.0f
                     : (ja.flex + jb.flex > 0) ? (float)(1.0 / ((double)L0 / ((double)s.G * s.J) + ja.flex + jb.flex))
                                               : s.G * s.J / L0;
    float cy[3], cz[3];
    end_pair(cy, s.E, s.Iy, s.G, s.As_z, L0, ja.free_y, jb.free_y, ja.flex, jb.flex);
    end_pair(cz, s.E, s.Iz, s.G, s.As_y, L0, ja.free_z, jb.free_z, ja.flex, jb.flex);
    // ---- the section's forces: axial yield at Np (compression at the lower of Np and the Euler load of 0.7 L), the
    // twist's at Tp, radial-return hinges at the ends against the hardened plastic moment, twice (eval_forces,
    // frame_fem.cpp:1915-1982); an elastic section's plastic parts stay 0
    const bool plastic = kPlastic && s.plastic;
    float up = 0, tp = 0, bt = 0, dmga = 0, dmgb = 0, pax = 0, pay = 0, pbx = 0, pby = 0, bax = 0, bay = 0, bbx = 0, bby = 0;
    uint32_t fl = 0;
    if (kPlastic) {
        const float4 s0 = F.mps[4 * ei], s1 = F.mps[4 * ei + 1], s2 = F.mps[4 * ei + 2], s3 = F.mps[4 * ei + 3];
        up = s0.x, tp = s0.y, bt = s0.z, dmga = s0.w, pax = s1.x, pay = s1.y, pbx = s1.z, pby = s1.w;
        bax = s2.x, bay = s2.y, bbx = s2.z, bby = s2.w, dmgb = s3.x;
        fl = F.mflag[ei];
    }
    const float delta = (float)dL;
    float N = ka * (delta - up);
    float flow_ax = 0, flow_t = 0, flow_a = 0, flow_b = 0;
    if (plastic) {
        const float Nt = s.Np, Le = 0.7f * L0;
        const float Nc = smin(s.Np, kPi * kPi * s.E * smin(s.Iy, s.Iz) / (Le * Le));
        if (N > Nt || N < -Nc) {
            const float lim = N > 0 ? Nt : -Nc;
            const float dup = (N - lim) / ka;
            up += dup;
            flow_ax = fabsf(dup) / L0;
            N = lim;
        }
    }
    const float twist = rb.x - ra.x;
    float T = kt * (twist - tp);
    if (plastic && s.Tp > 0 && kt > 0 && fabsf(T) > s.Tp) {
        const float lim = T > 0 ? s.Tp : -s.Tp;
        const float dtp = (T - lim) / kt;
        tp += dtp;
        flow_t = fabsf(dtp);
        T = lim;
    }
    float Max, May, Mbx, Mby;
    auto moments = [&]() {
        const float dax = ra.y - pax, day = ra.z - pay, dbx = rb.y - pbx, dby = rb.z - pby;
        Max = cy[0] * dax + cy[1] * dbx, May = cz[0] * day + cz[1] * dby;
        Mbx = cy[1] * dax + cy[2] * dbx, Mby = cz[1] * day + cz[2] * dby;
    };
    moments();
    if (plastic && s.Mp > 0) {
        auto yield_end = [&](float Mx, float My, float cyy, float czz, float& px, float& py, float bx, float by, float& dmg, float& flow) {
            const float Mp = s.Mp * (1.0f + s.hardening * smin(1.0f, dmg));
            const float l = sqrtf(Mx * Mx + My * My);
            if (l <= Mp) return false;
            const float r = 1.0f - Mp / l;
            const float dpx = cyy > 0 ? Mx * r / cyy : 0.0f, dpy = czz > 0 ? My * r / czz : 0.0f;
            px = px + dpx, py = py + dpy;
            flow += sqrtf(dpx * dpx + dpy * dpy);
            const float qx = px + bx, qy = py + by;
            dmg = smax(dmg, sqrtf(qx * qx + qy * qy));
            return true;
        };
        for (int it = 0; it < 2; it++) {
            if (yield_end(Max, May, cy[0], cz[0], pax, pay, bax, bay, dmga, flow_a)) moments();
            if (yield_end(Mbx, Mby, cy[2], cz[2], pbx, pby, bbx, bby, dmgb, flow_b)) moments();
        }
    }
    const float Sy = Max + Mbx, Sz = May + Mby;
    const v3 fav = e1 * N + e3 * (Sy / L) - e2 * (Sz / L);
    const v3 tav = e1 * T - e2 * Max - e3 * May;
    const v3 tbv = e1 * (-T) - e2 * Mbx - e3 * Mby;
    F.mfa[ei] = make_float4(fav.x, fav.y, fav.z, 0.0f);
    F.mta[ei] = make_float4(tav.x, tav.y, tav.z, 0.0f);
    F.mtb[ei] = make_float4(tbv.x, tbv.y, tbv.z, 0.0f);
    uint32_t y = 0;
    if (kPlastic) {
        // the plastic rotations into the rest frames past 0.02 rad, the twist half into each end (frame_fem.cpp:
        // 2045-2054)
        const float kBake = 0.02f;
        if (pax * pax + pay * pay > kBake * kBake) {
            const float4 q = F.mq[2 * ei];
            const q4 n = qnormalize(qmul(q4{q.x, q.y, q.z, q.w}, quat_exp(V(0, -pax, -pay))));
            F.mq[2 * ei] = make_float4(n.x, n.y, n.z, n.w);
            bax = bax + pax, bay = bay + pay, pax = pay = 0;
        }
        if (pbx * pbx + pby * pby > kBake * kBake) {
            const float4 q = F.mq[2 * ei + 1];
            const q4 n = qnormalize(qmul(q4{q.x, q.y, q.z, q.w}, quat_exp(V(0, -pbx, -pby))));
            F.mq[2 * ei + 1] = make_float4(n.x, n.y, n.z, n.w);
            bbx = bbx + pbx, bby = bby + pby, pbx = pby = 0;
        }
        if (fabsf(tp) > kBake) {
            const float4 qa = F.mq[2 * ei], qb = F.mq[2 * ei + 1];
            const q4 na = qnormalize(qmul(q4{qa.x, qa.y, qa.z, qa.w}, quat_exp(V(0.5f * tp, 0, 0))));
            const q4 nb = qnormalize(qmul(q4{qb.x, qb.y, qb.z, qb.w}, quat_exp(V(-0.5f * tp, 0, 0))));
            F.mq[2 * ei] = make_float4(na.x, na.y, na.z, na.w), F.mq[2 * ei + 1] = make_float4(nb.x, nb.y, nb.z, nb.w);
            bt += tp, tp = 0;
        }
        F.mps[4 * ei] = make_float4(up, tp, bt, dmga);
        F.mps[4 * ei + 1] = make_float4(pax, pay, pbx, pby);
        F.mps[4 * ei + 2] = make_float4(bax, bay, bbx, bby);
        F.mps[4 * ei + 3] = make_float4(dmgb, 0.0f, 0.0f, 0.0f);
        // the tangent: elastic, the parts flowing this step plastic unless the step unloads them (frame_fem.cpp:
        // 2056-2069): held elastic 16 steps after an unload, and while the re-passes' budget is spent
        const float kFlow = 1e-4f;
        const uint32_t yl = (flow_a > kFlow ? 1u : 0u) | (flow_b > kFlow ? 2u : 0u) | (flow_ax > 0.1f * kFlow ? 4u : 0u) | (flow_t > kFlow ? 8u : 0u);
        uint32_t hold = (fl >> 16) & 0xff, unload = 0;
        if (hold > 0) hold--, unload = yl;
        if (F.elastic[F.fbody[ab.x]]) unload = yl;
        F.mflag[ei] = yl | (unload << 8) | (hold << 16);
        F.mtg[6 * ei] = make_float4(e1.x, e1.y, e1.z, L);
        F.mtg[6 * ei + 1] = make_float4(e2.x, e2.y, e2.z, ka);
        F.mtg[6 * ei + 2] = make_float4(e3.x, e3.y, e3.z, kt);
        F.mtg[6 * ei + 3] = make_float4(cy[0], cy[1], cy[2], cz[0]);
        F.mtg[6 * ei + 4] = make_float4(cz[1], cz[2], N, T);
        F.mtg[6 * ei + 5] = make_float4(Max, May, Mbx, Mby);
        y = yl & ~unload;
    }
    F.mon[ei] = 1;
    F.mtan[ei] = make_float4(e1.x, e1.y, e1.z, N > 0 ? N / L : 0.0f);
    member_world_k(F, nd, ei, ab, e1, e2, e3, L, ka, kt, cy, cz, y);
}

// The unload check after pass `pass`'s solve (frame_fem.cpp:2959-2989): a flowing part of a member whose end rates
// from the solution run against its moment (force, torque) gets its elastic tangent (held 16 steps), its world blocks
// again; its component is marked for another pass. Pass 1's check runs only where pass 1 ran.
__global__ void k_member_unload(FemDev F, const float4* __restrict__ nd, int pass) {
    const int ei = blockIdx.x * blockDim.x + threadIdx.x;
    if (ei >= F.nmem || (pass > 0 && F.rp[pass - 1] == 0) || !F.mon[ei]) return;
    const uint32_t fl = F.mflag[ei];
    const uint32_t yl = fl & 0xf, unload = (fl >> 8) & 0xf, y = yl & ~unload;
    if (!y) return;
    const int2 ab = F.mn[ei];
    auto vel = [&](int fn, v3& v, v3& om) {
        const int col = F.iperm[fn];
        if (F.fixed[col]) {
            v = om = V(0, 0, 0);
            return;
        }
        const double* x = F.rhs + 6 * (size_t)col;
        const float4 nv = nd[2 * F.fnode[fn] + 1], w = F.w[fn];
        v = V(nv.x + (float)x[0], nv.y + (float)x[1], nv.z + (float)x[2]);
        om = V(w.x + (float)x[3], w.y + (float)x[4], w.z + (float)x[5]);
    };
    v3 va, wa, vb, wb;
    vel(ab.x, va, wa), vel(ab.y, vb, wb);
    const float4 t0 = F.mtg[6 * ei], t1 = F.mtg[6 * ei + 1], t2 = F.mtg[6 * ei + 2], t4 = F.mtg[6 * ei + 4], t5 = F.mtg[6 * ei + 5];
    const v3 e1 = V(t0.x, t0.y, t0.z), e2 = V(t1.x, t1.y, t1.z), e3 = V(t2.x, t2.y, t2.z);
    const float iL = 1.0f / t0.w;
    const v3 dv = vb - va;
    const float rax = dot(e3, dv) * iL + dot(e2, wa), ray = -dot(e2, dv) * iL + dot(e3, wa);
    const float rbx = dot(e3, dv) * iL + dot(e2, wb), rby = -dot(e2, dv) * iL + dot(e3, wb);
    uint32_t u = 0;
    if ((y & 1) && rax * t5.x + ray * t5.y < 0) u |= 1;
    if ((y & 2) && rbx * t5.z + rby * t5.w < 0) u |= 2;
    if ((y & 4) && dot(e1, dv) * t4.z < 0) u |= 4;
    if ((y & 8) && dot(e1, wb - wa) * t4.w < 0) u |= 8;
    if (!u) return;
    const uint32_t un = unload | u;
    F.mflag[ei] = yl | (un << 8) | (16u << 16);
    const float4 t3 = F.mtg[6 * ei + 3];
    const float cy[3] = {t3.x, t3.y, t3.z}, cz[3] = {t3.w, t4.x, t4.y};
    member_world_k(F, nd, ei, ab, e1, e2, e3, t0.w, t1.w, t2.w, cy, cz, yl & ~un);
    atomicOr(&F.comp_again[F.col_comp[F.iperm[ab.x]]], 1 << pass);
    F.rp[pass] = 1;
}

// the condition of the IF node of pass + 1's re-pass: set where pass `pass`'s check found an unload
__global__ void k_repass_cond(const int* __restrict__ rp, int pass, cudaGraphConditionalHandle h) {
    cudaGraphSetConditional(h, rp[pass] ? 1u : 0u);
}

// The re-passes' budget (FemFrame::begin_forces, frame_fem.cpp:1863-1864, and solve's accounting, frame_fem.cpp:2591,
// 2990): a body's re-passes of components of 60 columns or more spent from its credit, then its credit for the next
// step refilled by a quarter (at most 8); with less than one left its next step's tangents stay elastic.
__global__ void k_repass_account(FemDev F) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b == 0) *F.repc += F.rp[0] + F.rp[1], F.rp[0] = F.rp[1] = 0;
    if (b >= F.nbody) return;
    float cr = F.credit[b];
    for (int cc = F.body_comp[b]; cc < F.body_comp[b + 1]; cc++) {
        const int bits = F.comp_again[cc];
        if (bits && F.comp_size[cc] >= 60) cr -= (float)__popc(bits);
        F.comp_again[cc] = 0;
    }
    cr = smin(8.0f, cr + 0.25f);
    F.credit[b] = cr;
    F.elastic[b] = cr < 1.0f ? 1 : 0;
}

// gather_part's member block (frame_fem.cpp:927-941): block blk (0 aa, 1 bb, 2 ba, 3 ab) times c, with the geometric
// stiffness of its tension (sign gs)
__device__ __forceinline__ void member_block_add(const FemDev& F, int ei, int blk, double h2, double gs, double* D) {
    const int meta = F.mmeta[ei];
    const double c = h2 + (double)F.msec[meta & 0xffff].damping * F.h;
    const double* B = F.mkw + 144 * (size_t)ei + 36 * blk;
    for (int x = 0; x < 36; x++) D[x] += c * B[x];
    const float4 t = F.mtan[ei];
    const double gg = h2 * t.w;
    if (gg != 0) {
        double P[9];
        const double ee[3] = {t.x, t.y, t.z};
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) P[r * 3 + q] = gg * ((r == q ? 1.0 : 0.0) - ee[r] * ee[q]);
        for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) D[r * 6 + q] += gs * P[r * 3 + q];
    }
}

// ------------------------------------------------------------------------------------------ assembly
// A triangle's block of corners (i, j) in the world's axes times c, with its tension's geometric stiffness
// (gather_part's tri_block, frame_fem.cpp:961-1003)
__device__ void tri_block_add(const FemDev& F, int t, int i, int j, double h2, double* D) {
    const FemSecDev s = F.sec[F.tn[t].w];
    const double c = h2 + (double)s.damping * F.h;
    const float* tg = F.ttan + 18 * (size_t)t;
    const double E[3][3] = {{tg[0], tg[3], tg[6]}, {tg[1], tg[4], tg[7]}, {tg[2], tg[5], tg[8]}};
    const float* Km = F.tk + 162 * (size_t)t;
    const float* Kp = Km + 81;
#define BL_M(s2, t2) ((double)Km[(3 * i + (s2)) * 9 + 3 * j + (t2)])
#define BL_P(s2, t2) ((double)Kp[(3 * i + (s2)) * 9 + 3 * j + (t2)])
    for (int ra = 0; ra < 2; ra++)
        for (int cb = 0; cb < 2; cb++) {
            double T[3][3];
            for (int pp = 0; pp < 3; pp++) {
                const double E0 = E[pp][0], E1 = E[pp][1], E2 = E[pp][2];
                if (ra == 0 && cb == 0) {
                    T[pp][0] = E0 * BL_M(0, 0) + E1 * BL_M(1, 0);
                    T[pp][1] = E0 * BL_M(0, 1) + E1 * BL_M(1, 1);
                    T[pp][2] = E2 * BL_P(0, 0);
                } else if (ra == 0) {
                    T[pp][0] = E2 * BL_P(0, 1);
                    T[pp][1] = E2 * BL_P(0, 2);
                    T[pp][2] = E0 * BL_M(0, 2) + E1 * BL_M(1, 2);
                } else if (cb == 0) {
                    T[pp][0] = E2 * BL_M(2, 0);
                    T[pp][1] = E2 * BL_M(2, 1);
                    T[pp][2] = E0 * BL_P(1, 0) + E1 * BL_P(2, 0);
                } else {
                    T[pp][0] = E0 * BL_P(1, 1) + E1 * BL_P(2, 1);
                    T[pp][1] = E0 * BL_P(1, 2) + E1 * BL_P(2, 2);
                    T[pp][2] = E2 * BL_M(2, 2);
                }
            }
            for (int pp = 0; pp < 3; pp++)
                for (int qq = 0; qq < 3; qq++) D[(3 * ra + pp) * 6 + 3 * cb + qq] += c * (T[pp][0] * E[qq][0] + T[pp][1] * E[qq][1] + T[pp][2] * E[qq][2]);
        }
#undef BL_M
#undef BL_P
    const double gg = h2 * tg[9 + 3 * i + j];
    if (gg != 0)
        for (int pp = 0; pp < 3; pp++) D[pp * 7] += gg;
}

// One column's diagonal block and right side; nforce: the nodes' forces of the substep
__device__ __forceinline__ void assemble_column(const FemDev& F, const float4* __restrict__ nd, const float4* __restrict__ nforce, int k) {
    const int i = F.perm[k];
    const int bn = F.fnode[i];
    const float4 P = nd[2 * bn], Vv = nd[2 * bn + 1];
    const double h2 = F.ch2[k], hd = F.chd[k];
    double D[36];
    double* R = F.rhs + 6 * (size_t)k;
    for (int x = 0; x < 36; x++) D[x] = 0.0;
    if (k == 0 || F.col_comp[k] != F.col_comp[k - 1]) F.comp_fail[F.col_comp[k]] = 0;
    const bool fixed = P.w <= 0;
    F.fixed[k] = fixed;
    if (fixed) {
        for (int j = 0; j < 6; j++) D[j * 7] = 1.0, R[j] = 0.0;
    } else {
        D[0] = D[7] = D[14] = Vv.w;
        D[21] = D[28] = D[35] = F.inertia[i];
        double rd[6] = {0, 0, 0, 0, 0, 0};
        for (int qq = F.gdiag_ptr[k]; qq < F.gdiag_ptr[k + 1]; qq++) {
            const int2 g = F.gdiag[qq];
            if (g.x < 0) { // (a member's end: -(member + 1), end)
                const int ei = -g.x - 1;
                if (!F.mon[ei]) continue;
                member_block_add(F, ei, g.y, h2, 1.0, D);
                const double cr = hd + (double)F.msec[F.mmeta[ei] & 0xffff].damping * F.h;
                if (cr != 0) {
                    const double* kv = F.mkv + 12 * (size_t)ei + 6 * g.y;
                    for (int j = 0; j < 6; j++) rd[j] -= cr * kv[j];
                }
                continue;
            }
            if (!F.ton[g.x]) continue;
            tri_block_add(F, g.x, g.y, g.y, h2, D);
            const double cr = hd + (double)F.sec[F.tn[g.x].w].damping * F.h;
            if (cr != 0) {
                const double* kv = F.tkv + 18 * (size_t)g.x + 6 * g.y;
                for (int j = 0; j < 6; j++) rd[j] -= cr * kv[j];
            }
        }
        const float4 f = nforce[bn], m = F.torque[i];
        const double h = F.h;
        R[0] = h * (double)f.x, R[1] = h * (double)f.y, R[2] = h * (double)f.z;
        R[3] = h * (double)m.x, R[4] = h * (double)m.y, R[5] = h * (double)m.z;
        if (F.contact_n) {
            // a ground contact: kappa n n^T towards the normal velocity change it asked for, kappa = 200 m; sticking,
            // along the ground too towards stopping its sliding (gather_part, frame_fem.cpp:1043-1064)
            const float4 c4 = F.contact_n[i];
            v3 cn = V(c4.x, c4.y, c4.z);
            const float l2 = dot(cn, cn);
            if (l2 > 0) {
                const bool stick = l2 > 2.0f;
                if (stick) cn = cn * 0.5f;
                const double kap = 200.0 * Vv.w, want = F.step * (double)dot(V(f.x, f.y, f.z), cn) / Vv.w;
                const double nn[3] = {cn.x, cn.y, cn.z};
                for (int p = 0; p < 3; p++) {
                    for (int q2 = 0; q2 < 3; q2++) D[p * 6 + q2] += kap * nn[p] * nn[q2];
                    R[p] += kap * want * nn[p];
                }
                if (stick) {
                    const v3 vel = V(Vv.x, Vv.y, Vv.z);
                    const v3 vt = vel - cn * dot(vel, cn);
                    const double wt[3] = {-vt.x, -vt.y, -vt.z};
                    for (int p = 0; p < 3; p++) {
                        for (int q2 = 0; q2 < 3; q2++) D[p * 6 + q2] += kap * ((p == q2 ? 1.0 : 0.0) - nn[p] * nn[q2]);
                        R[p] += kap * wt[p];
                    }
                }
            }
        }
        for (int j = 0; j < 6; j++) R[j] += rd[j];
    }
    double* Dg = F.diag + 36 * (size_t)k;
    for (int x = 0; x < 36; x++) Dg[x] = D[x];
}

// The off-diagonal blocks, a thread each (pb: the block; its column from blk_col): zero where a corner is fixed, else
// the sum of its triangles' blocks in their order
__device__ __forceinline__ void assemble_off(const FemDev& F, const float4* __restrict__ nd, int pb) {
    const int k = F.blk_col[pb];
    const double h2 = F.ch2[k];
    double O[36];
    for (int x = 0; x < 36; x++) O[x] = 0.0;
    const bool fixed = nd[2 * F.fnode[F.perm[k]]].w <= 0;
    const int rnode = F.fnode[F.perm[F.row[pb]]];
    if (!fixed && F.goff_ptr[pb] != F.goff_ptr[pb + 1] && !(nd[2 * rnode].w <= 0))
        for (int qq = F.goff_ptr[pb]; qq < F.goff_ptr[pb + 1]; qq++) {
            const int4 g = F.goff[qq];
            if (g.x < 0) { // (a member's block: -(member + 1), 2 ba / 3 ab)
                if (F.mon[-g.x - 1]) member_block_add(F, -g.x - 1, g.y, h2, -1.0, O);
            } else if (F.ton[g.x]) {
                tri_block_add(F, g.x, g.y, g.z, h2, O);
            }
        }
    double* Og = F.off + 36 * (size_t)pb;
    for (int x = 0; x < 36; x++) Og[x] = O[x];
}

// The columns' diagonal blocks and right sides (threads [0, nf)) and the off-diagonal blocks (threads [nf, nf + nblk))
__global__ void __launch_bounds__(128) k_fem_assemble_all(FemDev F, const float4* __restrict__ nd, const float4* __restrict__ nforce) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < F.nf) assemble_column(F, nd, nforce, t);
    else if (t < F.nf + F.nblk) assemble_off(F, nd, t - F.nf);
}

// ------------------------------------------------------------------------------------------ factorization
// The Cholesky factor of one 6 x 6 block (what chol6, frame_fem.cpp:2193-2209, computes), by one thread, right-looking:
// each pivot's square root, its column scaled by the pivot's inverse, then the trailing lower triangle less that
// column's outer product. A (row-major) gets L in its lower triangle and zeros above; dinv the pivots' inverses. False
// at a pivot that is not positive (the block is not positive definite).
__device__ bool chol6_dev(double* A, double* dinv) {
    for (int k = 0; k < 6; k++) {
        const double piv = A[7 * k];
        if (!(piv > 0)) return false;
        const double d = sqrt(piv), id = 1.0 / d;
        A[7 * k] = d, dinv[k] = id;
        for (int i = k + 1; i < 6; i++) A[6 * i + k] *= id, A[6 * k + i] = 0;
        for (int j = k + 1; j < 6; j++)
            for (int i = j; i < 6; i++) A[6 * i + j] -= A[6 * i + k] * A[6 * j + k];
    }
    return true;
}

// The factorization's and substitutions' column work is done by units of 128 threads (4 warps) with a shared buffer
// sm of 72 doubles and a barrier of their own (bar: a named barrier id, or 0 for a unit that is the whole block). A
// unit takes one column (one slice of its rows, for the factor); the results do not depend on how units are launched.
constexpr int kUnit = 128;
__device__ __forceinline__ void unit_sync(int bar) {
    if (bar == 0) __syncthreads();
    else asm volatile("bar.sync %0, 128;" ::"r"(bar) : "memory");
}

// A column's factor, slice `slice` of `nslice` of its rows: the diagonal block (and its inverse diagonal) staged in
// sm by the first warp, chol6 there by its first thread - every slice's unit factors it alike, and slice 0's stores
// the factor in ldiag (the assembled diag stays as it is: another slice may still be reading it) - then the unit's
// rows of the column's off-diagonal blocks against it, X := X L^-T (right_solve_lt, frame_fem.cpp:2211-2220), a row a
// thread. The operations and their order are chol6's and right_solve_lt's.
__device__ __forceinline__ void chol_unit(const FemDev& F, int ci, int slice, int nslice, int ut, int bar, double* sm) {
    const int k = F.lvl_col[ci];
    unit_sync(bar); // (sm free)
    if (ut < 32) {
        const double* A = F.diag + 36 * (size_t)k;
        sm[ut] = A[ut];
        if (ut < 4) sm[32 + ut] = A[32 + ut];
        if (ut < 6) sm[36 + ut] = F.dinv[6 * (size_t)k + ut];
        __syncwarp();
        if (ut == 0) sm[42] = chol6_dev(sm, sm + 36) ? 1.0 : 0.0;
    }
    unit_sync(bar);
    const bool ok = sm[42] != 0.0;
    if (slice == 0) {
        if (ut < 36) F.ldiag[36 * (size_t)k + ut] = sm[ut];
        if (ut < 6) F.dinv[6 * (size_t)k + ut] = sm[36 + ut];
        if (ut == 0 && !ok) atomicExch(&F.comp_fail[F.col_comp[k]], 1);
    }
    if (!ok) return;
    double L[21], di[6];
    for (int j = 0, x = 0; j < 6; j++) {
        di[j] = sm[36 + j];
        for (int m = 0; m <= j; m++) L[x++] = sm[j * 6 + m];
    }
    const int nrows = 6 * (F.col_ptr[k + 1] - F.col_ptr[k]);
    for (int rr = slice * kUnit + ut; rr < nrows; rr += nslice * kUnit) {
        double* xrow = F.off + 36 * (size_t)(F.col_ptr[k] + rr / 6) + 6 * (rr % 6);
        double x[6];
        for (int j = 0; j < 6; j++) x[j] = xrow[j];
        for (int j = 0, b = 0; j < 6; j++) {
            double s = x[j];
            for (int m = 0; m < j; m++) s -= L[b + m] * x[m];
            x[j] = s * di[j];
            b += j + 1;
        }
        for (int j = 0; j < 6; j++) xrow[j] = x[j];
    }
}

// The level's columns' updates (the right-looking step of frame_fem.cpp:2910-2914), one warp per target block: the
// updates this level's columns make to it, in the order of those columns, T -= P Q^T each (sub_abt's sums,
// frame_fem.cpp:2276-2288). A target meets every level's updates in the order of the levels. pq: 72 doubles.
__device__ __forceinline__ void update_group(const FemDev& F, int gi, int lane, double* pq) {
    const int tgt = F.grp_tgt[gi];
    double* T = tgt < F.nf ? F.diag + 36 * (size_t)tgt : F.off + 36 * (size_t)(tgt - F.nf);
    const int e0 = lane, e1 = lane + 32; // (lane e, and e + 32 for e < 4, own entry e = 6 r + c)
    double acc0 = T[e0], acc1 = lane < 4 ? T[e1] : 0.0;
    for (int u = F.grp_ptr[gi]; u < F.grp_ptr[gi + 1]; u++) {
        const int2 pp = F.gu[u];
        const double* Pm = F.off + 36 * (size_t)pp.x; // P = L(pj)
        const double* Qm = F.off + 36 * (size_t)pp.y; // Q = L(pi)
        __syncwarp();
        for (int x = lane; x < 72; x += 32) pq[x] = x < 36 ? Pm[x] : Qm[x - 36];
        __syncwarp();
        {
            const int r = e0 / 6, cc = e0 % 6;
            double s = 0;
            for (int m = 0; m < 6; m++) s += pq[r * 6 + m] * pq[36 + cc * 6 + m];
            acc0 -= s;
        }
        if (lane < 4) {
            const int r = e1 / 6, cc = e1 % 6;
            double s = 0;
            for (int m = 0; m < 6; m++) s += pq[r * 6 + m] * pq[36 + cc * 6 + m];
            acc1 -= s;
        }
    }
    T[e0] = acc0;
    if (lane < 4) T[e1] = acc1;
}

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// A unit's six partial sums s[] (one set a thread) to their total in thread 0's s[]: each warp's by a butterfly,
// then the four warps' in order (sm[48..71])
__device__ __forceinline__ void unit_sum6(double* s, int ut, int bar, double* sm) {
    for (int j = 0; j < 6; j++) s[j] = warp_sum(s[j]);
    if ((ut & 31) == 0)
        for (int j = 0; j < 6; j++) sm[48 + 6 * (ut >> 5) + j] = s[j];
    unit_sync(bar);
    if (ut == 0)
        for (int j = 0; j < 6; j++) s[j] = ((sm[48 + j] + sm[54 + j]) + sm[60 + j]) + sm[66 + j];
}

// L y = r for a column: the blocks in its row (from the columns before it) spread over the unit and summed, then
// forward6 (frame_fem.cpp:2304-2310, 2944-2948) by the unit's first thread on the factored diagonal block, its
// inverse diagonal and r, staged in sm while the row is summed.
__device__ __forceinline__ void forward_unit(const FemDev& F, int ci, int ut, int bar, double* sm) {
    const int k = F.lvl_col[ci];
    unit_sync(bar); // (sm free)
    if (ut < 36) sm[ut] = F.ldiag[36 * (size_t)k + ut];
    if (ut < 6) sm[36 + ut] = F.dinv[6 * (size_t)k + ut], sm[42 + ut] = F.rhs[6 * (size_t)k + ut];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int q = F.rb_ptr[k] + ut; q < F.rb_ptr[k + 1]; q += kUnit) {
        const int2 bc = F.rb[q];
        const double* L = F.off + 36 * (size_t)bc.x;
        const double* yk = F.rhs + 6 * (size_t)bc.y;
        for (int ii = 0; ii < 6; ii++) {
            double t = 0;
            for (int j = 0; j < 6; j++) t += L[ii * 6 + j] * yk[j];
            s[ii] += t;
        }
    }
    unit_sum6(s, ut, bar, sm);
    if (ut != 0) return;
    double y[6];
    for (int j = 0; j < 6; j++) y[j] = sm[42 + j] - s[j];
    for (int j = 0; j < 6; j++) {
        double t = y[j];
        for (int m = 0; m < j; m++) t -= sm[j * 6 + m] * y[m];
        y[j] = t * sm[36 + j];
    }
    for (int j = 0; j < 6; j++) F.rhs[6 * (size_t)k + j] = y[j];
}

// L^T x = y for a column (the levels from the top down): its blocks' L^T x_row over the unit, summed, then backward6
// (frame_fem.cpp:2296-2303, 2311-2317, 2949-2954) by the unit's first thread, staged as forward's.
__device__ __forceinline__ void backward_unit(const FemDev& F, int ci, int ut, int bar, double* sm) {
    const int k = F.lvl_col[ci];
    unit_sync(bar); // (sm free)
    if (ut < 36) sm[ut] = F.ldiag[36 * (size_t)k + ut];
    if (ut < 6) sm[36 + ut] = F.dinv[6 * (size_t)k + ut], sm[42 + ut] = F.rhs[6 * (size_t)k + ut];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int pb = F.col_ptr[k] + ut; pb < F.col_ptr[k + 1]; pb += kUnit) {
        const double* L = F.off + 36 * (size_t)pb;
        const double* xr = F.rhs + 6 * (size_t)F.row[pb];
        for (int j = 0; j < 6; j++) {
            double t = 0;
            for (int ii = 0; ii < 6; ii++) t += L[ii * 6 + j] * xr[ii];
            s[j] += t;
        }
    }
    unit_sum6(s, ut, bar, sm);
    if (ut != 0) return;
    double x[6];
    for (int j = 0; j < 6; j++) x[j] = sm[42 + j] - s[j];
    for (int j = 5; j >= 0; j--) {
        double t = x[j];
        for (int m = j + 1; m < 6; m++) t -= sm[m * 6 + j] * x[m];
        x[j] = t * sm[36 + j];
    }
    for (int j = 0; j < 6; j++) F.rhs[6 * (size_t)k + j] = x[j];
}

// A level's columns' factors: block (x, y) takes the level's column c0 + x, slice y of gridDim.y of its rows
__global__ void __launch_bounds__(kUnit) k_fem_chol_level(FemDev F, int c0) {
    __shared__ double sm[72];
    chol_unit(F, c0 + blockIdx.x, blockIdx.y, gridDim.y, threadIdx.x, 0, sm);
}

// A level's updates and its forward substitution in one launch (independent: the updates write blocks of later
// columns, the substitution reads this level's and earlier columns' factors): blocks [0, ceil((g1 - g0) / 4)) take
// the update targets (a warp each), the rest a column each.
__global__ void __launch_bounds__(kUnit) k_fem_update_forward_level(FemDev F, int g0, int g1, int c0) {
    __shared__ double sm[4][72];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nub = (g1 - g0 + 3) / 4;
    if ((int)blockIdx.x < nub) {
        const int gi = g0 + blockIdx.x * 4 + wib;
        if (gi < g1) update_group(F, gi, lane, sm[wib]);
    } else {
        forward_unit(F, c0 + blockIdx.x - nub, threadIdx.x, 0, sm[0]);
    }
}

__global__ void __launch_bounds__(kUnit) k_fem_backward_level(FemDev F, int c0) {
    __shared__ double sm[72];
    backward_unit(F, c0 + blockIdx.x, threadIdx.x, 0, sm);
}

// ------------------------------------------------------------------------------------------ the top chain as one dense front
// The top of the elimination tree is a chain of single columns (160 of the 64 x 64 plate's 267 levels): every row of a
// chain column's factor is a later chain column (a column's rows are its ancestors in the tree). After the levels
// below have made their updates, the chain's blocks form one dense lower triangle D (6 m x 6 m, padded with an
// identity to whole 32 x 32 tiles), factored by a blocked right-looking Cholesky - per 32-column panel a tile
// factorization (one warp), the panel's triangular solves and the trailing rank-32 updates - and solved densely; the
// levels below then run their backward substitutions on the chain's solution. The sums run in another order than the
// block schedule's (the step is a tolerance match with the reference either way: its element kernels call the GPU's
// transcendentals).
constexpr int kFT = 32;       // tile
constexpr int kFrontMin = 8;  // the shortest chain made a dense front (columns)

struct FrontDev {
    int m, N, nt;            // chain columns, D's size (6 m rounded up to tiles), tiles a side
    const int* col;          // chain column c -> its column
    const int4* blk;         // the chain's off-diagonal blocks: (block, row's chain index, column's chain index, 0)
    int nblk;
    const int* chain;        // column -> its chain index, or -1
    double* D;               // N x N, row-major: the chain's blocks (lower triangle), then the factor
    double* b;               // N: the chain's right side, then its forward substitution's result
};

// D's lower triangle from the chain's diagonal and off-diagonal blocks; the padding's diagonal 1 (D zero before)
__global__ void k_front_scatter(FemDev F, FrontDev X) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int nd = 36 * X.m, no = 36 * X.nblk;
    if (t < nd) {
        const int c = t / 36, e = t % 36, i = e / 6, j = e % 6;
        if (j <= i) X.D[(size_t)(6 * c + i) * X.N + 6 * c + j] = F.diag[36 * (size_t)X.col[c] + e];
    } else if (t < nd + no) {
        const int q = t - nd, e = q % 36;
        const int4 bl = X.blk[q / 36];
        X.D[(size_t)(6 * bl.y + e / 6) * X.N + 6 * bl.z + e % 6] = F.off[36 * (size_t)bl.x + e];
    } else if (t < nd + no + X.N - 6 * X.m) {
        const int r = 6 * X.m + (t - nd - no);
        X.D[(size_t)r * X.N + r] = 1.0;
    }
}

// The diagonal tile p: Cholesky in place by one warp, lane i holding row i in registers (column j's entries shared
// through shared memory each step); a non-positive pivot fails the chain's component
__global__ void __launch_bounds__(32) k_front_potrf(FemDev F, FrontDev X, int p) {
    __shared__ double col[kFT];
    const int lane = threadIdx.x;
    double* T = X.D + (size_t)(kFT * p) * X.N + kFT * p;
    double a[kFT];
#pragma unroll
    for (int l = 0; l < kFT; l++) a[l] = T[(size_t)lane * X.N + l];
    bool ok = true;
#pragma unroll
    for (int j = 0; j < kFT; j++) {
        const double s = __shfl_sync(0xffffffffu, a[j], j);
        ok = ok && s > 0;
        const double id = rsqrt(s), d = s * id;
        a[j] = lane == j ? d : (lane > j ? a[j] * id : a[j]);
        col[lane] = a[j];
        __syncwarp();
#pragma unroll
        for (int l = j + 1; l < kFT; l++)
            if (l <= lane) a[l] -= a[j] * col[l];
        __syncwarp();
    }
#pragma unroll
    for (int l = 0; l < kFT; l++) T[(size_t)lane * X.N + l] = l <= lane ? a[l] : 0.0;
    if (!ok && lane == 0) atomicExch(&F.comp_fail[F.col_comp[X.col[0]]], 1);
    // the forward substitution's tile: y_p = L_pp^-1 b_p (b_p already less the earlier panels' parts)
    double y = X.b[kFT * p + lane];
#pragma unroll
    for (int j = 0; j < kFT; j++) {
        if (lane == j) y /= a[j];
        const double yj = __shfl_sync(0xffffffffu, y, j);
        if (lane > j) y -= a[j] * yj;
    }
    X.b[kFT * p + lane] = y;
}

// The panel below tile p: L_ip = A_ip L_pp^-T for the tiles i > p (a block each; thread r: row r of the tile)
__global__ void __launch_bounds__(kFT) k_front_trsm(FrontDev X, int p) {
    __shared__ double L[kFT][kFT + 1];
    __shared__ double id[kFT];
    const int r = threadIdx.x, i = p + 1 + blockIdx.x;
    const double* P = X.D + (size_t)(kFT * p) * X.N + kFT * p;
    for (int q = 0; q < kFT; q++) L[q][r] = P[(size_t)q * X.N + r];
    __syncwarp();
    id[r] = 1.0 / L[r][r];
    __syncwarp();
    double* row = X.D + (size_t)(kFT * i + r) * X.N + kFT * p;
    double x[kFT];
#pragma unroll
    for (int j = 0; j < kFT; j++) x[j] = row[j];
#pragma unroll
    for (int j = 0; j < kFT; j++) {
        double s = x[j];
#pragma unroll
        for (int l = 0; l < j; l++) s -= x[l] * L[j][l];
        x[j] = s * id[j];
    }
#pragma unroll
    for (int j = 0; j < kFT; j++) row[j] = x[j];
    // the forward substitution: b_i -= L_ip y_p
    double sy = 0;
#pragma unroll
    for (int j = 0; j < kFT; j++) sy += x[j] * X.b[kFT * p + j];
    X.b[kFT * i + r] -= sy;
}

// The trailing update of panel p: A_ij -= L_ip L_jp^T for p < j <= i (a block a tile, 256 threads of 2 x 2 entries)
__global__ void __launch_bounds__(256) k_front_syrk(FrontDev X, int p) {
    __shared__ double Li[kFT][kFT + 1], Lj[kFT][kFT + 1];
    // (blockIdx.x -> (i, j): i = p + 1 + a, j = p + 1 + b, b <= a, row a of the triangle holding a + 1 tiles)
    const int q = blockIdx.x;
    int a = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
    while ((a + 1) * (a + 2) / 2 <= q) a++;
    while (a * (a + 1) / 2 > q) a--;
    const int bb = q - a * (a + 1) / 2;
    const int i = p + 1 + a, j = p + 1 + bb;
    const int t = threadIdx.x;
    for (int e = t; e < kFT * kFT; e += 256) {
        const int rr = e / kFT, cc = e % kFT;
        Li[rr][cc] = X.D[(size_t)(kFT * i + rr) * X.N + kFT * p + cc];
        Lj[rr][cc] = X.D[(size_t)(kFT * j + rr) * X.N + kFT * p + cc];
    }
    __syncthreads();
    const int r0 = 2 * (t / 16), c0 = 2 * (t % 16);
    double acc[2][2] = {{0, 0}, {0, 0}};
#pragma unroll 8
    for (int k = 0; k < kFT; k++) {
        const double x0 = Li[r0][k], x1 = Li[r0 + 1][k], y0 = Lj[c0][k], y1 = Lj[c0 + 1][k];
        acc[0][0] += x0 * y0, acc[0][1] += x0 * y1, acc[1][0] += x1 * y0, acc[1][1] += x1 * y1;
    }
    double* T = X.D + (size_t)(kFT * i + r0) * X.N + kFT * j + c0;
    T[0] -= acc[0][0], T[1] -= acc[0][1], T[X.N] -= acc[1][0], T[X.N + 1] -= acc[1][1];
}

// The chain's right side: each chain column's r less its row's blocks from the columns below the chain times their y
// (forward_unit's sum without the chain's own columns), a unit a chain column
__global__ void __launch_bounds__(kUnit) k_front_rhs(FemDev F, FrontDev X) {
    __shared__ double sm[72];
    const int c = blockIdx.x, ut = threadIdx.x, k = X.col[c];
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int q = F.rb_ptr[k] + ut; q < F.rb_ptr[k + 1]; q += kUnit) {
        const int2 bc = F.rb[q];
        if (X.chain[bc.y] >= 0) continue;
        const double* L = F.off + 36 * (size_t)bc.x;
        const double* yk = F.rhs + 6 * (size_t)bc.y;
        for (int ii = 0; ii < 6; ii++) {
            double t = 0;
            for (int j = 0; j < 6; j++) t += L[ii * 6 + j] * yk[j];
            s[ii] += t;
        }
    }
    unit_sum6(s, ut, 0, sm);
    if (ut == 0)
        for (int j = 0; j < 6; j++) X.b[6 * c + j] = F.rhs[6 * (size_t)k + j] - s[j];
    if (c == 0)
        for (int r = 6 * X.m + ut; r < X.N; r += kUnit) X.b[r] = 0.0; // (the padding's)
}

// L^T x = y over the dense factor (y: the forward substitution's result, left in b by the factorization's kernels),
// by one block: per tile from the last, its 32 x 32 diagonal staged in shared memory (with the inverses of its
// diagonal) and solved by one warp (lane t: row t), then the earlier rows updated by the block; x into the chain
// columns' rhs
__global__ void __launch_bounds__(1024) k_front_solve(FemDev F, FrontDev X) {
    extern __shared__ double v[]; // N
    __shared__ double Tt[kFT][kFT + 1];
    __shared__ double inv[kFT];
    const int t = threadIdx.x, n6 = 6 * X.m, lane = t & 31;
    for (int r = t; r < X.N; r += blockDim.x) v[r] = X.b[r];
    for (int p = X.nt - 1; p >= 0; p--) {
        const int r0 = kFT * p;
        __syncthreads();
        Tt[t / kFT][t % kFT] = X.D[(size_t)(r0 + t / kFT) * X.N + r0 + t % kFT]; // (1024 threads: the whole tile)
        __syncthreads();
        if (t < kFT) inv[t] = 1.0 / Tt[t][t];
        __syncthreads();
        if (t < 32) {
            double x = v[r0 + lane];
#pragma unroll
            for (int j = kFT - 1; j >= 0; j--) {
                if (lane == j) x *= inv[j];
                const double xj = __shfl_sync(0xffffffffu, x, j);
                if (lane < j) x -= Tt[j][lane] * xj;
            }
            v[r0 + lane] = x;
        }
        __syncthreads();
        for (int r = t; r < r0; r += blockDim.x) {
            double s = 0;
#pragma unroll
            for (int j = 0; j < kFT; j++) s += X.D[(size_t)(r0 + j) * X.N + r] * v[r0 + j];
            v[r] -= s;
        }
    }
    __syncthreads();
    for (int r = t; r < n6; r += blockDim.x) F.rhs[6 * (size_t)X.col[r / 6] + r % 6] = v[r];
}

// ------------------------------------------------------------------------------------------ after the solve
__global__ void k_fem_velocity(FemDev F, const float4* __restrict__ nd, float4* __restrict__ nforce) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= F.nf) return;
    const int i = F.perm[k];
    F.torque[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f); // (used by this step: torques from outside add up until the next)
    if (F.comp_fail[F.col_comp[k]]) {
        if (k == 0 || F.col_comp[k] != F.col_comp[k - 1]) atomicAdd(&F.body_failures[F.fbody[i]], 1);
        return; // (a failed factorization: the elements' forces stay in the node forces, an explicit step this once)
    }
    if (F.fixed[k]) {
        F.w[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        return;
    }
    const double* x = F.rhs + 6 * (size_t)k;
    const int bn = F.fnode[i];
    const float mass = nd[2 * bn + 1].w;
    v3 dv = V((float)x[0], (float)x[1], (float)x[2]);
    const v3 dw = V((float)x[3], (float)x[4], (float)x[5]);
    if (!isfinite(dv.x + dv.y + dv.z + dw.x + dw.y + dw.z)) {
        atomicAdd(&F.body_failures[F.fbody[i]], 1);
        return;
    }
    const float kMaxDv = 40.0f, kMaxW = 3000.0f;
    {
        const float l = length(dv);
        if (l > kMaxDv) dv = dv * (kMaxDv / l), atomicAdd(&F.body_clamps[F.fbody[i]], 1);
    }
    const v3 fv = dv * (mass / F.step);
    nforce[bn] = make_float4(fv.x, fv.y, fv.z, 0.0f);
    const float4 w0 = F.w[i];
    v3 wn = V(w0.x, w0.y, w0.z) + dw;
    {
        const float l = length(wn);
        if (l > kMaxW) wn = wn * (kMaxW / l), atomicAdd(&F.body_clamps[F.fbody[i]], 1);
    }
    F.w[i] = make_float4(wn.x, wn.y, wn.z, 0.0f);
}

// The frame bodies' nodes: SoftBody::integrate_nodes with the forces the solve left (softbody.cpp:769-795), the body's
// bounds and top speed; then a frame node's FemFrame::sync_positions (frame_fem.cpp:3407-3422): its double position
// advanced by h v, its orientation turned by w h, its float position taken from the double one unless something moved
// it. fem_nodes: the frame bodies' nodes (global node indices), fslot: a node's frame node (-1: none).
__global__ void __launch_bounds__(256) k_fem_integrate(FemDev F, float4* __restrict__ nd, const float4* __restrict__ nforce,
                                                       const int* __restrict__ fem_nodes, int n_fem_nodes, const int* __restrict__ fslot,
                                                       const int4* __restrict__ info, Body* __restrict__ bodies, float dt) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_fem_nodes) return;
    const int i = fem_nodes[t];
    Body& B = bodies[info[i].w];
    if (B.sleeping) return;
    float4 P = nd[2 * i], Vv = nd[2 * i + 1];
    v3 pos = V(P.x, P.y, P.z), vel = V(Vv.x, Vv.y, Vv.z);
    float v2 = 0.0f;
    if (P.w > 0) {
        const float4 f4 = nforce[i];
        vel = vel + V(f4.x, f4.y, f4.z) * (P.w * dt);
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
    const int fs = fslot[i];
    if (fs >= 0) {
        double* x = F.xd + 3 * (size_t)fs;
        const double h = F.h;
        x[0] += h * vel.x, x[1] += h * vel.y, x[2] += h * vel.z;
        const float4 w4 = F.w[fs];
        const v3 w = V(w4.x, w4.y, w4.z);
        if (dot(w, w) > 0) {
            const float4 q0 = F.q[fs];
            const q4 qn = qnormalize(qmul(quat_exp(w * F.h), q4{q0.x, q0.y, q0.z, q0.w}));
            F.q[fs] = make_float4(qn.x, qn.y, qn.z, qn.w);
        }
        const double tol = 1e-4 * (1.0 + fabs((double)pos.x) + fabs((double)pos.y) + fabs((double)pos.z));
        if (P.w > 0 && fabs(x[0] - pos.x) <= tol && fabs(x[1] - pos.y) <= tol && fabs(x[2] - pos.z) <= tol)
            pos = V((float)x[0], (float)x[1], (float)x[2]);
        else
            x[0] = pos.x, x[1] = pos.y, x[2] = pos.z;
    }
    nd[2 * i] = make_float4(pos.x, pos.y, pos.z, P.w);
    nd[2 * i + 1] = make_float4(vel.x, vel.y, vel.z, Vv.w);
    if (pos.x == pos.x) atomic_min_f(&B.acc_mn[0], pos.x), atomic_max_f(&B.acc_mx[0], pos.x);
    if (pos.y == pos.y) atomic_min_f(&B.acc_mn[1], pos.y), atomic_max_f(&B.acc_mx[1], pos.y);
    if (pos.z == pos.z) atomic_min_f(&B.acc_mn[2], pos.z), atomic_max_f(&B.acc_mx[2], pos.z);
    atomic_max_f(&B.acc_v2, v2);
}

} // namespace blg
