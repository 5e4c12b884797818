// Host side of the FEM shell step: a body's triangle elements made ready for the GPU.
//
// fem_setup restates, for triangle elements (no members, mounts or springs), what the reference does once a frame is
// built (FemFrame::finalize, frame_fem.cpp:224-429; FemFrame::analyse, frame_fem.cpp:544-860;
// FemFrame::gather_lists, frame_fem.cpp:863-901; tri_local_k / tri_build_k, frame_fem.cpp:1524-1648), with the same
// integer results - frame node numbering, components, the exact minimum-degree elimination order, the factor's column
// patterns and update list, the assembly's gather lists - and the rest shapes, rest frames, inertias and element
// stiffnesses in the reference's float / double arithmetic. It then derives the GPU's schedule: the elimination tree's
// levels, each target block's updates in source-column order, each row's blocks for the forward substitution.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

namespace blg {

struct FemSection { // ShellSection (frame_fem.h:114-150): the elastic step's fields
    float E, nu, rho, t, yield, damping, drill;
    float D() const { return E * t * t * t / (12.0f * (1.0f - nu * nu)); }
};

struct HF3 {
    float x, y, z;
};
struct HQ {
    float x, y, z, w;
};
static inline HF3 h3(float x, float y, float z) { return {x, y, z}; }
static inline HF3 hsub(HF3 a, HF3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline HF3 hadd(HF3 a, HF3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline HF3 hmul(HF3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
static inline float hdot(HF3 a, HF3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline HF3 hcross(HF3 a, HF3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
static inline float hlen(HF3 a) { return std::sqrt(hdot(a, a)); }
static inline HF3 hnormalize(HF3 a) {
    const float l = hlen(a);
    return l > 1e-12f ? hmul(a, 1.0f / l) : h3(0, 0, 0);
}
static inline HQ hqmul(HQ a, HQ b) { // quat::operator* (math.h:142-147)
    return {a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x, a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w,
            a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z};
}
static inline HQ hqconj(HQ q) { return {-q.x, -q.y, -q.z, q.w}; }
static inline HQ hqnormalize(HQ q) { // math.h:160-163
    const float l = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (!(l > 1e-12f)) return {0, 0, 0, 1};
    const float i = 1.0f / l;
    return {q.x * i, q.y * i, q.z * i, q.w * i};
}
// from_mat3 (math.h:175-201) of the matrix with columns c0, c1, c2
static inline HQ hfrom_mat3(HF3 c0, HF3 c1, HF3 c2) {
    const float m00 = c0.x, m11 = c1.y, m22 = c2.z;
    const float tr = m00 + m11 + m22;
    HQ q{0, 0, 0, 1};
    if (tr > 0) {
        const float s = std::sqrt(tr + 1.0f) * 2;
        q.w = 0.25f * s, q.x = (c1.z - c2.y) / s, q.y = (c2.x - c0.z) / s, q.z = (c0.y - c1.x) / s;
    } else if (m00 > m11 && m00 > m22) {
        const float s = std::sqrt(1.0f + m00 - m11 - m22) * 2;
        q.w = (c1.z - c2.y) / s, q.x = 0.25f * s, q.y = (c1.x + c0.y) / s, q.z = (c2.x + c0.z) / s;
    } else if (m11 > m22) {
        const float s = std::sqrt(1.0f + m11 - m00 - m22) * 2;
        q.w = (c2.x - c0.z) / s, q.x = (c1.x + c0.y) / s, q.y = 0.25f * s, q.z = (c2.y + c1.z) / s;
    } else {
        const float s = std::sqrt(1.0f + m22 - m00 - m11) * 2;
        q.w = (c0.y - c1.x) / s, q.x = (c2.x + c0.z) / s, q.y = (c2.y + c1.z) / s, q.z = 0.25f * s;
    }
    return hqnormalize(q);
}

// The element's stiffness (below) is built on the host once per triangle and on the GPU again where a triangle's
// membrane flows (k_tri_eval): one source for both, compiled for each, so that both give the same bits.
#define BL_HD __host__ __device__

// The DKT bending's curvature-displacement matrix at area coordinates (xi, eta) (frame_fem.cpp:1482-1509)
BL_HD inline void dkt_b(const double x[3], const double y[3], double xi, double eta, double B[3][9]) {
    const double x23 = x[1] - x[2], x31 = x[2] - x[0], x12 = x[0] - x[1];
    const double y23 = y[1] - y[2], y31 = y[2] - y[0], y12 = y[0] - y[1];
    double P[7], q[7], r[7], t[7];
    const double xs[3] = {x23, x31, x12}, ys[3] = {y23, y31, y12};
    for (int k = 4; k <= 6; k++) {
        const double xij = xs[k - 4], yij = ys[k - 4], l2 = xij * xij + yij * yij;
        P[k] = -6 * xij / l2, q[k] = 3 * xij * yij / l2, t[k] = -6 * yij / l2, r[k] = 3 * yij * yij / l2;
    }
    const double a = 1 - 2 * xi, bb = 1 - 2 * eta;
    const double Hx_xi[9] = {P[6] * a + (P[5] - P[6]) * eta, q[6] * a - (q[5] + q[6]) * eta, -4 + 6 * (xi + eta) + r[6] * a - eta * (r[5] + r[6]),
                             -P[6] * a + eta * (P[4] + P[6]), q[6] * a - eta * (q[6] - q[4]), -2 + 6 * xi + r[6] * a + eta * (r[4] - r[6]),
                             -eta * (P[5] + P[4]), eta * (q[4] - q[5]), -eta * (r[5] - r[4])};
    const double Hy_xi[9] = {t[6] * a + eta * (t[5] - t[6]), 1 + r[6] * a - eta * (r[5] + r[6]), -q[6] * a + eta * (q[5] + q[6]),
                             -t[6] * a + eta * (t[4] + t[6]), -1 + r[6] * a + eta * (r[4] - r[6]), -q[6] * a - eta * (q[4] - q[6]),
                             -eta * (t[4] + t[5]), eta * (r[4] - r[5]), -eta * (q[4] - q[5])};
    const double Hx_eta[9] = {-P[5] * bb - xi * (P[6] - P[5]), q[5] * bb - xi * (q[5] + q[6]), -4 + 6 * (xi + eta) + r[5] * bb - xi * (r[5] + r[6]),
                              xi * (P[4] + P[6]), xi * (q[4] - q[6]), -xi * (r[6] - r[4]),
                              P[5] * bb - xi * (P[4] + P[5]), q[5] * bb + xi * (q[4] - q[5]), -2 + 6 * eta + r[5] * bb + xi * (r[4] - r[5])};
    const double Hy_eta[9] = {-t[5] * bb - xi * (t[6] - t[5]), 1 + r[5] * bb - xi * (r[5] + r[6]), -q[5] * bb + xi * (q[5] + q[6]),
                              xi * (t[4] + t[6]), xi * (r[4] - r[6]), -xi * (q[4] - q[6]),
                              t[5] * bb - xi * (t[4] + t[5]), -1 + r[5] * bb + xi * (r[4] - r[5]), -q[5] * bb - xi * (q[4] - q[5])};
    const double A2 = x31 * y12 - x12 * y31, iA = 1.0 / A2;
    for (int j = 0; j < 9; j++) {
        B[0][j] = (y31 * Hx_xi[j] + y12 * Hx_eta[j]) * iA;
        B[1][j] = (-x31 * Hy_xi[j] - x12 * Hy_eta[j]) * iA;
        B[2][j] = (-x31 * Hx_xi[j] - x12 * Hx_eta[j] + y31 * Hy_xi[j] + y12 * Hy_eta[j]) * iA;
    }
}

// the membrane's shape gradients (frame_fem.cpp:1513-1520)
BL_HD inline void tri_grad(const float X[3][2], double b[3], double c[3], double& A2) {
    for (int i = 0; i < 3; i++) {
        const int j = (i + 1) % 3, k = (i + 2) % 3;
        b[i] = (double)X[j][1] - X[k][1];
        c[i] = (double)X[k][0] - X[j][0];
    }
    A2 = ((double)X[1][0] - X[0][0]) * ((double)X[2][1] - X[0][1]) - ((double)X[2][0] - X[0][0]) * ((double)X[1][1] - X[0][1]);
}

// The element's stiffness in its own axes, 18 dofs [u v w theta_x theta_y theta_z] per corner: CST membrane, DKT
// bending at three points, the drilling spring (frame_fem.cpp:1524-1574); packed as the reference's tri_k_: the
// membrane's 9 x 9 then the plate's; and the bending's curvatures at the three points from the corners' rotations
// alone, tri_b_ (tri_build_k, frame_fem.cpp:1625-1647). s: the section's E, nu, t, drill and its D() (float).
struct TriSec {
    float E, nu, t, drill;
    BL_HD float D() const { return E * t * t * t / (12.0f * (1.0f - nu * nu)); }
};
BL_HD inline void tri_local_k(const float X[3][2], const TriSec& s, float P[162], float Bc[54]) {
    const double kGauss[3][2] = {{1.0 / 6, 1.0 / 6}, {2.0 / 3, 1.0 / 6}, {1.0 / 6, 2.0 / 3}};
    const int kMem[3] = {0, 1, 5}, kPlate[3] = {2, 3, 4};
    double K[18][18];
    for (int i = 0; i < 18; i++)
        for (int j = 0; j < 18; j++) K[i][j] = 0;
    double b[3], c[3], A2;
    tri_grad(X, b, c, A2);
    if (A2 > 0) {
        const double A = 0.5 * A2, nu = s.nu;
        const double Dm = (double)s.E * s.t / (1 - nu * nu);
        double Bm[3][6];
        for (int i = 0; i < 3; i++) {
            Bm[0][2 * i] = b[i] / A2, Bm[1][2 * i] = 0, Bm[2][2 * i] = c[i] / A2;
            Bm[0][2 * i + 1] = 0, Bm[1][2 * i + 1] = c[i] / A2, Bm[2][2 * i + 1] = b[i] / A2;
        }
        const double D3[3][3] = {{1, nu, 0}, {nu, 1, 0}, {0, 0, 0.5 * (1 - nu)}};
        for (int p = 0; p < 6; p++)
            for (int q = 0; q < 6; q++) {
                double v = 0;
                for (int r = 0; r < 3; r++)
                    for (int t = 0; t < 3; t++) v += Bm[r][p] * D3[r][t] * Bm[t][q];
                K[6 * (p / 2) + p % 2][6 * (q / 2) + q % 2] += A * Dm * v;
            }
        const double x[3] = {X[0][0], X[1][0], X[2][0]}, y[3] = {X[0][1], X[1][1], X[2][1]};
        const double Db = s.D();
        for (const auto& g : kGauss) {
            double B[3][9];
            dkt_b(x, y, g[0], g[1], B);
            for (int p = 0; p < 9; p++)
                for (int q = 0; q < 9; q++) {
                    double v = 0;
                    for (int r = 0; r < 3; r++)
                        for (int t = 0; t < 3; t++) v += B[r][p] * D3[r][t] * B[t][q];
                    K[6 * (p / 3) + 2 + p % 3][6 * (q / 3) + 2 + q % 3] += A2 / 6.0 * Db * v;
                }
        }
        const double G = (double)s.E / (2 * (1 + nu)), kd = (double)s.drill * G * s.t * A;
        double gu[3], gv[3];
        for (int i = 0; i < 3; i++) gu[i] = -c[i] / (2 * A2), gv[i] = b[i] / (2 * A2);
        for (int i = 0; i < 3; i++) {
            K[6 * i + 5][6 * i + 5] += kd;
            for (int j = 0; j < 3; j++) {
                K[6 * i + 5][6 * j] -= kd * gu[j], K[6 * j][6 * i + 5] -= kd * gu[j];
                K[6 * i + 5][6 * j + 1] -= kd * gv[j], K[6 * j + 1][6 * i + 5] -= kd * gv[j];
                K[6 * i][6 * j] += 3 * kd * gu[i] * gu[j], K[6 * i][6 * j + 1] += 3 * kd * gu[i] * gv[j];
                K[6 * i + 1][6 * j] += 3 * kd * gv[i] * gu[j], K[6 * i + 1][6 * j + 1] += 3 * kd * gv[i] * gv[j];
            }
        }
    }
    for (int a = 0; a < 9; a++)
        for (int cc = 0; cc < 9; cc++) {
            const int im = 6 * (a / 3) + kMem[a % 3], jm = 6 * (cc / 3) + kMem[cc % 3];
            const int ip = 6 * (a / 3) + kPlate[a % 3], jp = 6 * (cc / 3) + kPlate[cc % 3];
            P[a * 9 + cc] = (float)K[im < jm ? im : jm][im < jm ? jm : im];
            P[81 + a * 9 + cc] = (float)K[ip < jp ? ip : jp][ip < jp ? jp : ip];
        }
    const double x[3] = {X[0][0], X[1][0], X[2][0]}, y[3] = {X[0][1], X[1][1], X[2][1]};
    for (int g = 0; g < 3; g++) {
        double B[3][9];
        dkt_b(x, y, kGauss[g][0], kGauss[g][1], B);
        for (int r = 0; r < 3; r++)
            for (int i = 0; i < 3; i++) Bc[g * 18 + r * 6 + 2 * i] = (float)B[r][3 * i + 1], Bc[g * 18 + r * 6 + 2 * i + 1] = (float)B[r][3 * i + 2];
    }
}

struct FrameSectionH { // FrameSection (frame_fem.h:90-112): the member step's fields
    float E, G, rho, A, Iy, Iz, J, As_y, As_z, damping, axial, joint_k;
    float Np, Mp, Tp, hardening;
};

// One body's frame of members and triangle elements, as built and analysed
struct FemModel {
    // frame nodes (in the order add_element and add_tri made them: each member's a, b, then each triangle's corners)
    std::vector<uint32_t> node;      // body node of each frame node
    std::vector<double> xd;          // 3 per frame node
    std::vector<float> inertia;
    // members (FemFrame::elems)
    std::vector<std::array<int, 2>> mn;  // frame nodes a, b
    std::vector<uint16_t> msec;
    std::vector<uint8_t> mend;       // 2 per member: the joints at a, b
    std::vector<float> mL0, mmass;   // rest length; the mass it put on its nodes
    std::vector<float> mq;           // 8 per member: its rest frame in its end nodes' frames, qa then qb (x y z w)
    std::vector<float> mps;          // 16 per member: its plastic state (up tp bt dmg_a, pa pb, ba bb, dmg_b - - -)
    std::vector<uint32_t> mflag;     // per member: its tangent's yield and unload bits and its elastic hold
    std::vector<uint8_t> mbroken;
    std::vector<int> mblock;         // its off-diagonal block (-1: its ends share a column)
    std::vector<uint8_t> mswap;      // the block's row is its a end
    // triangles
    std::vector<std::array<int, 3>> tn;  // frame nodes
    std::vector<uint16_t> tsec;
    std::vector<float> tX;           // 6 per triangle: the rest shape
    std::vector<float> tr0;          // 12 per triangle: the rest frames (quaternion x y z w per corner)
    std::vector<float> tmass, tarea0;
    std::vector<uint8_t> tbroken;
    std::vector<float> tk;           // 162 per triangle
    std::vector<float> tb;           // 54 per triangle: the bending's curvatures from the corners' rotations (tri_b_)
    std::vector<float> tX0;          // 6 per triangle: the authored rest shape (the plastic stretch is against it)
    std::vector<float> th0;          // 9 per triangle: the corners' plastic rest rotations not yet baked into tr0
    std::vector<float> tdmg;         // per triangle: the plastic stretch reached (FrameTri::dmg)
    // the pattern
    int ncomp = 0;
    std::vector<int> comp_first;     // per component: its first column (and a last entry: n)
    std::vector<int> perm, iperm, col_ptr, row;
    std::vector<int> upd_ptr;        // per column
    std::vector<std::array<int, 3>> upd; // (pi, pj, target)
    std::vector<std::array<int, 3>> tri_block;
    std::vector<std::array<uint8_t, 3>> tri_swap;
    // gather lists, members first (gather_lists, frame_fem.cpp:863-901): per column its members' ends (-(member + 1),
    // end 0 a / 1 b) and its triangles' corners (tri, corner); per off-diagonal block (-(member + 1), 2: block (b, a)
    // / 3: block (a, b), 0) and (tri, i, j)
    std::vector<int> gdiag_ptr, goff_ptr;
    std::vector<std::array<int, 2>> gdiag;
    std::vector<std::array<int, 3>> goff;
};

// FemFrame::finalize (frame_fem.cpp:224-260) and the node inertias (node_inertia, frame_fem.cpp:3075-3086): p, mass - the
// body's node positions and masses; mpm - each member's section's mass per metre (FrameSection::mass_per_m)
static void fem_finalize(FemModel& M, const float* px, const float* py, const float* pz, const float* mass, const std::vector<float>& mpm) {
    const size_t n = M.node.size();
    M.xd.resize(n * 3);
    for (size_t i = 0; i < n; i++) M.xd[3 * i] = px[M.node[i]], M.xd[3 * i + 1] = py[M.node[i]], M.xd[3 * i + 2] = pz[M.node[i]];
    const size_t E = M.mn.size();
    M.mL0.assign(E, 0.0f), M.mq.assign(8 * E, 0.0f), M.mbroken.assign(E, 0);
    for (size_t e = 0; e < E; e++) {
        const int a = M.mn[e][0], b = M.mn[e][1];
        const HF3 xa = h3(px[M.node[a]], py[M.node[a]], pz[M.node[a]]), xb = h3(px[M.node[b]], py[M.node[b]], pz[M.node[b]]);
        const HF3 d = hsub(xb, xa);
        const float L0 = hlen(d);
        M.mL0[e] = L0;
        if (L0 < 1e-5f || a == b) {
            M.mbroken[e] = 1;
            continue;
        }
        // the rest frame: x along the member, y towards the world's up (a vertical member: towards x)
        const HF3 e1 = hmul(d, 1.0f / L0);
        const HF3 ref = std::fabs(e1.y) < 0.9f ? h3(0, 1, 0) : h3(1, 0, 0);
        const HF3 e2 = hnormalize(hsub(ref, hmul(e1, hdot(e1, ref)))), e3 = hcross(e1, e2);
        const HQ E0 = hfrom_mat3(e1, e2, e3);
        const HQ r = hqnormalize(hqmul(hqconj(HQ{0, 0, 0, 1}), E0)); // (both ends' rest orientation: the identity)
        for (int h = 0; h < 2; h++) M.mq[8 * e + 4 * h] = r.x, M.mq[8 * e + 4 * h + 1] = r.y, M.mq[8 * e + 4 * h + 2] = r.z, M.mq[8 * e + 4 * h + 3] = r.w;
        if (M.mmass[e] <= 0) M.mmass[e] = mpm[e] * L0;
    }
    const size_t T = M.tn.size();
    M.tX.assign(T * 6, 0.0f), M.tr0.assign(T * 12, 0.0f), M.tarea0.assign(T, 0.0f), M.tbroken.assign(T, 0);
    for (size_t t = 0; t < T; t++) {
        const int* fn = M.tn[t].data();
        const HF3 x0 = h3(px[M.node[fn[0]]], py[M.node[fn[0]]], pz[M.node[fn[0]]]);
        const HF3 x1 = h3(px[M.node[fn[1]]], py[M.node[fn[1]]], pz[M.node[fn[1]]]);
        const HF3 x2 = h3(px[M.node[fn[2]]], py[M.node[fn[2]]], pz[M.node[fn[2]]]);
        const HF3 nn = hcross(hsub(x1, x0), hsub(x2, x0));
        const float a2 = hlen(nn);
        if (!(a2 > 1e-8f) || fn[0] == fn[1] || fn[1] == fn[2] || fn[0] == fn[2]) {
            M.tbroken[t] = 1;
            continue;
        }
        const float ia2 = 1.0f / a2;
        const HF3 e3 = hmul(nn, ia2), e1 = hnormalize(hsub(x1, x0)), e2 = hcross(e3, e1);
        const HF3 c = hmul(hadd(hadd(x0, x1), x2), 1.0f / 3.0f);
        const HF3 xs[3] = {x0, x1, x2};
        for (int i = 0; i < 3; i++) M.tX[6 * t + 2 * i] = hdot(hsub(xs[i], c), e1), M.tX[6 * t + 2 * i + 1] = hdot(hsub(xs[i], c), e2);
        M.tarea0[t] = 0.5f * a2;
        const HQ E0 = hfrom_mat3(e1, e2, e3);
        for (int i = 0; i < 3; i++) {
            const HQ r = hqnormalize(hqmul(hqconj(HQ{0, 0, 0, 1}), E0)); // (the node's rest orientation: the identity)
            M.tr0[12 * t + 4 * i] = r.x, M.tr0[12 * t + 4 * i + 1] = r.y, M.tr0[12 * t + 4 * i + 2] = r.z, M.tr0[12 * t + 4 * i + 3] = r.w;
        }
    }
    M.tX0 = M.tX, M.th0.assign(T * 9, 0.0f), M.tdmg.assign(T, 0.0f);
    M.inertia.assign(n, 0.0f);
    std::vector<float> I(n, 0.0f);
    // (the members' halves first, each node's sum in member order: the lumped m L^2 / 78 an end, m = mass_per_m L0)
    for (size_t e = 0; e < E; e++) {
        if (M.mbroken[e]) continue;
        const float add = mpm[e] * M.mL0[e] * M.mL0[e] * M.mL0[e] / 78.0f;
        I[M.mn[e][0]] += add;
        if (M.mn[e][1] != M.mn[e][0]) I[M.mn[e][1]] += add;
    }
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        const int* fn = M.tn[t].data();
        const float add = M.tmass[t] * M.tarea0[t] / 108.0f;
        // (the reference loops the nodes, each over all triangles in order: each node's sum in triangle order)
        for (int i = 0; i < 3; i++)
            if (!(i > 0 && fn[i] == fn[0]) && !(i > 1 && fn[i] == fn[1])) I[fn[i]] += add;
    }
    for (size_t i = 0; i < n; i++) {
        const float mn = mass[M.node[i]];
        M.inertia[i] = std::max(I[i], std::max(1e-6f, mn * 1e-4f));
    }
}

// FemFrame::analyse + gather_lists (frame_fem.cpp:544-901) for members and triangle elements
static void fem_analyse(FemModel& M) {
    const int n = (int)M.node.size();
    const size_t T = M.tn.size();
    std::vector<int> up(n);
    for (int i = 0; i < n; i++) up[i] = i;
    auto find = [&](int x) {
        while (up[x] != x) x = up[x] = up[up[x]];
        return x;
    };
    const size_t E = M.mn.size();
    for (size_t e = 0; e < E; e++) up[find(M.mn[e][0])] = find(M.mn[e][1]);
    for (size_t t = 0; t < T; t++)
        if (!M.tbroken[t]) up[find(M.tn[t][0])] = find(M.tn[t][1]), up[find(M.tn[t][1])] = find(M.tn[t][2]);
    std::vector<std::pair<int, int>> edge;
    for (size_t e = 0; e < E; e++)
        if (M.mn[e][0] != M.mn[e][1]) edge.push_back({M.mn[e][0], M.mn[e][1]});
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        const int a = M.tn[t][0], b = M.tn[t][1], c = M.tn[t][2];
        if (a != b) edge.push_back({a, b});
        if (b != c) edge.push_back({b, c});
        if (c != a) edge.push_back({c, a});
    }
    std::vector<int> comp_of(n, -1), roots;
    for (int i = 0; i < n; i++) {
        const int r = find(i);
        if (comp_of[r] < 0) comp_of[r] = (int)roots.size(), roots.push_back(r);
        comp_of[i] = comp_of[r];
    }
    const int nc = (int)roots.size();
    // each node's neighbours once
    std::vector<std::vector<int>> adj(n);
    for (const auto& e : edge) adj[e.first].push_back(e.second), adj[e.second].push_back(e.first);
    std::vector<std::vector<int>> comp_nodes(nc);
    for (int i = 0; i < n; i++) comp_nodes[comp_of[i]].push_back(i);
    M.ncomp = nc;
    M.perm.assign(n, 0), M.iperm.assign(n, 0);
    M.comp_first.assign(nc + 1, 0);
    // exact minimum degree over the elimination graph as bit rows: the node taken is the first of least degree in the
    // component's order; its elimination joins its neighbours to each other
    std::vector<int> cols_ptr(n + 1, 0), cols_buf, loc(n, -1), deg;
    std::vector<uint64_t> bits, bucket;
    int k = 0;
    for (int c = 0; c < nc; c++) {
        M.comp_first[c] = k;
        const std::vector<int>& cn = comp_nodes[c];
        const int m = (int)cn.size(), W = (m + 63) / 64;
        for (int x = 0; x < m; x++) loc[cn[x]] = x;
        bits.assign((size_t)m * W, 0ull);
        bucket.assign((size_t)(m + 1) * W, 0ull);
        deg.assign(m, 0);
        int mind = m;
        for (int x = 0; x < m; x++) {
            uint64_t* rx = &bits[(size_t)x * W];
            for (int y0 : adj[cn[x]]) {
                const int y = loc[y0];
                rx[y >> 6] |= 1ull << (y & 63);
            }
            int d = 0;
            for (int q = 0; q < W; q++) d += __builtin_popcountll(rx[q]);
            deg[x] = d;
            bucket[(size_t)d * W + (x >> 6)] |= 1ull << (x & 63);
            mind = std::min(mind, d);
        }
        for (int step = 0; step < m; step++, k++) {
            int v = -1;
            while (v < 0) {
                const uint64_t* bd = &bucket[(size_t)mind * W];
                for (int w = 0; w < W; w++)
                    if (bd[w]) {
                        v = (w << 6) + __builtin_ctzll(bd[w]);
                        break;
                    }
                if (v < 0) mind++;
            }
            bucket[(size_t)deg[v] * W + (v >> 6)] &= ~(1ull << (v & 63));
            M.perm[k] = cn[v];
            M.iperm[cn[v]] = k;
            uint64_t* rv = &bits[(size_t)v * W];
            for (int w = 0; w < W; w++)
                for (uint64_t bb = rv[w]; bb; bb &= bb - 1) {
                    const int y = (w << 6) + __builtin_ctzll(bb);
                    cols_buf.push_back(cn[y]);
                    uint64_t* ry = &bits[(size_t)y * W];
                    for (int q = 0; q < W; q++) ry[q] |= rv[q];
                    ry[y >> 6] &= ~(1ull << (y & 63));
                    ry[v >> 6] &= ~(1ull << (v & 63));
                    int d = 0;
                    for (int q = 0; q < W; q++) d += __builtin_popcountll(ry[q]);
                    bucket[(size_t)deg[y] * W + (y >> 6)] &= ~(1ull << (y & 63));
                    bucket[(size_t)d * W + (y >> 6)] |= 1ull << (y & 63);
                    deg[y] = d;
                    mind = std::min(mind, d);
                }
            for (int w = 0; w < W; w++) rv[w] = 0;
            cols_ptr[k + 1] = (int)cols_buf.size();
        }
    }
    M.comp_first[nc] = k;
    // the columns' rows (sorted) and the right-looking update list with its targets
    M.col_ptr.assign(n + 1, 0);
    M.row.resize(cols_buf.size());
    for (int kk = 0; kk < n; kk++) {
        const int a0 = cols_ptr[kk], a1 = cols_ptr[kk + 1];
        for (int q = a0; q < a1; q++) M.row[q] = M.iperm[cols_buf[q]];
        std::sort(M.row.begin() + a0, M.row.begin() + a1);
        M.col_ptr[kk + 1] = a1;
    }
    auto find_block = [&](int col, int r) {
        const int* a = M.row.data() + M.col_ptr[col];
        const int* e = M.row.data() + M.col_ptr[col + 1];
        const int* it = std::lower_bound(a, e, r);
        return it != e && *it == r ? (int)(it - M.row.data()) : -1;
    };
    M.upd_ptr.assign(n + 1, 0);
    M.upd.clear();
    for (int kk = 0; kk < n; kk++) {
        for (int pi = M.col_ptr[kk]; pi < M.col_ptr[kk + 1]; pi++) {
            const int c = M.row[pi], qe = M.col_ptr[c + 1];
            int q = M.col_ptr[c];
            for (int pj = pi; pj < M.col_ptr[kk + 1]; pj++) {
                int target;
                if (pi == pj) {
                    target = -(c + 1);
                } else {
                    const int rr = M.row[pj];
                    while (q < qe && M.row[q] < rr) q++;
                    target = q < qe && M.row[q] == rr ? q : -1;
                }
                M.upd.push_back({pi, pj, target});
            }
        }
        M.upd_ptr[kk + 1] = (int)M.upd.size();
    }
    M.mblock.assign(E, -1);
    M.mswap.assign(E, 0);
    for (size_t e = 0; e < E; e++) {
        const int ka = M.iperm[M.mn[e][0]], kb = M.iperm[M.mn[e][1]];
        if (ka == kb) continue;
        M.mblock[e] = find_block(std::min(ka, kb), std::max(ka, kb));
        M.mswap[e] = ka > kb;
    }
    M.tri_block.assign(T, {-1, -1, -1});
    M.tri_swap.assign(T, {0, 0, 0});
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        for (int e = 0; e < 3; e++) {
            const int ki = M.iperm[M.tn[t][e]], kj = M.iperm[M.tn[t][(e + 1) % 3]];
            if (ki == kj) continue;
            M.tri_block[t][e] = find_block(std::min(ki, kj), std::max(ki, kj));
            M.tri_swap[t][e] = ki > kj;
        }
    }
    // gather lists in the triangles' order (gather_lists, frame_fem.cpp:863-901)
    M.gdiag_ptr.assign(n + 1, 0);
    M.goff_ptr.assign(M.row.size() + 1, 0);
    for (size_t e = 0; e < E; e++) {
        M.gdiag_ptr[M.iperm[M.mn[e][0]] + 1]++, M.gdiag_ptr[M.iperm[M.mn[e][1]] + 1]++;
        if (M.mblock[e] >= 0) M.goff_ptr[M.mblock[e] + 1]++;
    }
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        for (int c = 0; c < 3; c++) M.gdiag_ptr[M.iperm[M.tn[t][c]] + 1]++;
        for (int e = 0; e < 3; e++)
            if (M.tri_block[t][e] >= 0) M.goff_ptr[M.tri_block[t][e] + 1]++;
    }
    for (size_t q = 1; q < M.gdiag_ptr.size(); q++) M.gdiag_ptr[q] += M.gdiag_ptr[q - 1];
    for (size_t q = 1; q < M.goff_ptr.size(); q++) M.goff_ptr[q] += M.goff_ptr[q - 1];
    M.gdiag.assign(M.gdiag_ptr.back(), {0, 0});
    M.goff.assign(M.goff_ptr.back(), {0, 0, 0});
    std::vector<int> fd(M.gdiag_ptr.begin(), M.gdiag_ptr.end() - 1), fo(M.goff_ptr.begin(), M.goff_ptr.end() - 1);
    for (size_t e = 0; e < E; e++) {
        M.gdiag[fd[M.iperm[M.mn[e][0]]]++] = {-(int)e - 1, 0};
        M.gdiag[fd[M.iperm[M.mn[e][1]]]++] = {-(int)e - 1, 1};
        if (M.mblock[e] >= 0) M.goff[fo[M.mblock[e]]++] = {-(int)e - 1, M.mswap[e] ? 3 : 2, 0}; // (the row node's: b, or a)
    }
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        for (int c = 0; c < 3; c++) M.gdiag[fd[M.iperm[M.tn[t][c]]]++] = {(int)t, c};
        for (int e = 0; e < 3; e++)
            if (M.tri_block[t][e] >= 0) { // (the block's row is the later corner in the order)
                const int i = e, j = (e + 1) % 3;
                M.goff[fo[M.tri_block[t][e]]++] = {(int)t, M.tri_swap[t][e] ? i : j, M.tri_swap[t][e] ? j : i};
            }
    }
}

} // namespace blg
