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
#include <functional>
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

// ------------------------------------------------------------------------------------------ the shell element
// A flat triangle in its own axes (x, y in its plane): corners X[i], 6 dofs each (u, v, w, theta_x, theta_y,
// theta_z). Membrane: the constant-strain triangle. Bending: the discrete Kirchhoff triangle (DKT; Batoz, Bathe & Ho,
// Int. J. Numer. Meth. Eng. 15, 1980), sampled at three points. Drilling: a penalty tying each corner's theta_z to the
// element's in-plane rotation. Restated here from those definitions (the reference's tri_local_k,
// frame_fem.cpp:1524-1574, builds the same element).

// The triangle's linear geometry: twice its signed area and the area coordinates' gradients, dL_i/dx = b_i / A2,
// dL_i/dy = c_i / A2, where (b_i, c_i) is the edge opposite corner i (from corner i+1 to corner i+2) turned by -90
// degrees.
struct TriGeom {
    double b[3], c[3], A2;
};
template <class XY>
BL_HD inline TriGeom tri_geom(const XY& X) {
    TriGeom g;
    for (int i = 0; i < 3; i++) {
        const int j = i == 2 ? 0 : i + 1, k = j == 2 ? 0 : j + 1;
        const double ex = (double)X[k][0] - X[j][0], ey = (double)X[k][1] - X[j][1];
        g.b[i] = -ey, g.c[i] = ex;
    }
    g.A2 = ((double)X[1][0] - X[0][0]) * ((double)X[2][1] - X[0][1]) - ((double)X[2][0] - X[0][0]) * ((double)X[1][1] - X[0][1]);
    return g;
}
// (the form the element kernels use)
BL_HD inline void tri_grad(const float X[3][2], double b[3], double c[3], double& A2) {
    const TriGeom g = tri_geom(X);
    for (int i = 0; i < 3; i++) b[i] = g.b[i], c[i] = g.c[i];
    A2 = g.A2;
}

// The DKT curvatures (kappa_x, kappa_y, 2 kappa_xy) at area coordinates (L1, L2) = (xi, eta) from the 9 bending dofs
// (w, theta_x, theta_y per corner). The normal's rotation beta = (theta_y, -theta_x) is interpolated quadratically
// over the six-node triangle; at each edge's midpoint its tangential part is what a cubic w along the edge gives
// (beta_s = -dw/ds: -3 (w_j - w_i) / (2 l) - (beta_s,i + beta_s,j) / 4) and its normal part the corners' mean; the
// curvatures are beta's derivatives: kappa_x = dbeta_x/dx, kappa_y = dbeta_y/dy, 2 kappa_xy = dbeta_x/dy + dbeta_y/dx.
BL_HD inline void dkt_b(const double x[3], const double y[3], double xi, double eta, double B[3][9]) {
    const double xy[3][2] = {{x[0], y[0]}, {x[1], y[1]}, {x[2], y[2]}};
    const TriGeom g = tri_geom(xy);
    const double L[3] = {1 - xi - eta, xi, eta};
    // beta at the six nodes (corners 0-2, then the midpoints of edges 01, 12, 20) as rows over the 9 dofs
    double bx[6][9], by[6][9];
    for (int a = 0; a < 6; a++)
        for (int d = 0; d < 9; d++) bx[a][d] = by[a][d] = 0;
    for (int i = 0; i < 3; i++) bx[i][3 * i + 2] = 1, by[i][3 * i + 1] = -1;
    for (int e = 0; e < 3; e++) {
        const int i = e, j = e == 2 ? 0 : e + 1;
        const double ex = x[j] - x[i], ey = y[j] - y[i], l = sqrt(ex * ex + ey * ey);
        const double sx = ex / l, sy = ey / l, nx = sy, ny = -sx;
        for (int d = 0; d < 9; d++) {
            double bs = -0.25 * ((bx[i][d] + bx[j][d]) * sx + (by[i][d] + by[j][d]) * sy);
            const double bn = 0.5 * ((bx[i][d] + bx[j][d]) * nx + (by[i][d] + by[j][d]) * ny);
            if (d == 3 * i) bs += 1.5 / l;
            if (d == 3 * j) bs -= 1.5 / l;
            bx[3 + e][d] = bs * sx + bn * nx, by[3 + e][d] = bs * sy + bn * ny;
        }
    }
    // the quadratic shape functions' gradients: corner L(2L - 1), midpoint 4 L_i L_j
    double nxd[6], nyd[6];
    for (int i = 0; i < 3; i++) nxd[i] = (4 * L[i] - 1) * g.b[i] / g.A2, nyd[i] = (4 * L[i] - 1) * g.c[i] / g.A2;
    for (int e = 0; e < 3; e++) {
        const int i = e, j = e == 2 ? 0 : e + 1;
        nxd[3 + e] = 4 * (L[i] * g.b[j] + L[j] * g.b[i]) / g.A2, nyd[3 + e] = 4 * (L[i] * g.c[j] + L[j] * g.c[i]) / g.A2;
    }
    for (int d = 0; d < 9; d++) {
        double kx = 0, ky = 0, kxy = 0;
        for (int a = 0; a < 6; a++) kx += nxd[a] * bx[a][d], ky += nyd[a] * by[a][d], kxy += nyd[a] * bx[a][d] + nxd[a] * by[a][d];
        B[0][d] = kx, B[1][d] = ky, B[2][d] = kxy;
    }
}

// The element's stiffness in its own axes, stored as the membrane's 9 x 9 (dofs u, v, theta_z per corner) then the
// plate's 9 x 9 (w, theta_x, theta_y per corner) - P[162] - and the bending's curvatures from the corners' rotations
// alone at the three sample points (kappa rows x (theta_x, theta_y) per corner) - Bc[54]. s: the section's E, nu, t,
// drill and its plate rigidity D() (float, as the section's).
struct TriSec {
    float E, nu, t, drill;
    BL_HD float D() const { return E * t * t * t / (12.0f * (1.0f - nu * nu)); }
};
BL_HD inline void tri_local_k(const float X[3][2], const TriSec& s, float P[162], float Bc[54]) {
    // the three sample points (area coordinates L1, L2) of the bending, each weighted by a third of the area
    const double pts[3][2] = {{1.0 / 6, 1.0 / 6}, {2.0 / 3, 1.0 / 6}, {1.0 / 6, 2.0 / 3}};
    double Km[9][9], Kp[9][9]; // membrane (u, v, theta_z) and plate (w, theta_x, theta_y), corner-major
    for (int r = 0; r < 9; r++)
        for (int q = 0; q < 9; q++) Km[r][q] = Kp[r][q] = 0;
    const TriGeom g = tri_geom(X);
    const double x[3] = {X[0][0], X[1][0], X[2][0]}, y[3] = {X[0][1], X[1][1], X[2][1]};
    if (g.A2 > 0) {
        const double nu = s.nu, A = 0.5 * g.A2, half = 0.5 * (1 - nu);
        // membrane: A t Bm^T Dm Bm pair by pair, Bm of corner i = [b_i 0; 0 c_i; c_i b_i] / A2
        const double km = A * ((double)s.E * s.t / (1 - nu * nu)) / (g.A2 * g.A2);
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) {
                const double bi = g.b[i], ci = g.c[i], bj = g.b[j], cj = g.c[j];
                Km[3 * i][3 * j] += km * (bi * bj + half * ci * cj);
                Km[3 * i][3 * j + 1] += km * (nu * bi * cj + half * ci * bj);
                Km[3 * i + 1][3 * j] += km * (nu * ci * bj + half * bi * cj);
                Km[3 * i + 1][3 * j + 1] += km * (ci * cj + half * bi * bj);
            }
        // bending: sum over the points of (A / 3) D B^T [1 nu 0; nu 1 0; 0 0 (1 - nu) / 2] B
        const double kb = A / 3.0 * (double)s.D();
        for (const auto& pt : pts) {
            double B[3][9];
            dkt_b(x, y, pt[0], pt[1], B);
            for (int q = 0; q < 9; q++) {
                const double m0 = B[0][q] + nu * B[1][q], m1 = nu * B[0][q] + B[1][q], m2 = half * B[2][q]; // (D B)_q / D
                for (int r = 0; r < 9; r++) Kp[r][q] += kb * (B[0][r] * m0 + B[1][r] * m1 + B[2][r] * m2);
            }
        }
        // drilling: (kd / 2) sum_i (theta_z,i - omega)^2, omega = (dv/dx - du/dy) / 2 the element's in-plane rotation;
        // with go omega's gradient over u / v, each corner adds kd r r^T, r = e(theta_z,i) - go
        const double kd = (double)s.drill * ((double)s.E / (2 * (1 + nu))) * s.t * A;
        double go[9];
        for (int j = 0; j < 3; j++) go[3 * j] = -g.c[j] / (2 * g.A2), go[3 * j + 1] = g.b[j] / (2 * g.A2), go[3 * j + 2] = 0;
        for (int i = 0; i < 3; i++) {
            double r[9];
            for (int q = 0; q < 9; q++) r[q] = -go[q];
            r[3 * i + 2] += 1;
            for (int a = 0; a < 9; a++)
                for (int q = 0; q < 9; q++) Km[a][q] += kd * r[a] * r[q];
        }
    }
    // (both stored exactly symmetric: each pair from the upper triangle)
    for (int r = 0; r < 9; r++)
        for (int q = 0; q < 9; q++) {
            const int lo = r < q ? r : q, hi = r < q ? q : r;
            P[r * 9 + q] = (float)Km[lo][hi], P[81 + r * 9 + q] = (float)Kp[lo][hi];
        }
    for (int p = 0; p < 3; p++) {
        double B[3][9];
        dkt_b(x, y, pts[p][0], pts[p][1], B);
        for (int k = 0; k < 3; k++)
            for (int i = 0; i < 3; i++) Bc[18 * p + 6 * k + 2 * i] = (float)B[k][3 * i + 1], Bc[18 * p + 6 * k + 2 * i + 1] = (float)B[k][3 * i + 2];
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

// ------------------------------------------------------------------------------------------ the symbolic phase
// What FemFrame::analyse + gather_lists (frame_fem.cpp:544-901) compute for members and triangle elements, by a
// design of this file's own. The results that must match the reference bit for bit are fixed by rules, not by the
// reference's data structures:
//  * components: frame nodes joined by members and unbroken triangles, numbered in order of their lowest node;
//  * the elimination order, component after component: exact minimum degree on the elimination graph (a node's degree
//    counts its neighbours once the nodes before it are eliminated, each elimination joining its neighbours into a
//    clique), the ties going to the lowest frame node;
//  * the factor's pattern: column k's rows are its node's neighbours at its elimination, in elimination positions,
//    ascending;
//  * the update list: for each column k, each pair of its rows (i <= j, by position) in order - the product of blocks
//    i and j of column k subtracts from block (row j, column row i), or from that column's diagonal when i == j.
// Here the elimination graph is never formed: the ordering runs on the quotient graph, in which every eliminated
// node becomes an element standing for the clique of its neighbours and absorbs the elements next to it, so that a
// node's neighbourhood is its remaining node neighbours plus the nodes of its elements, and every degree is counted
// exactly (no approximate degrees, no supervariables: either could change a tie). The least (degree, node) is kept
// in a binary heap whose stale entries are skipped when they surface.

struct FemComponents {
    int count = 0;
    std::vector<int> of;                 // per frame node
    std::vector<std::vector<int>> nodes; // per component, its nodes ascending
};

// each frame node's distinct neighbours (CSR, ascending) from the members and the unbroken triangles' edges
static void fem_graph(const FemModel& M, std::vector<int>& ptr, std::vector<int>& nbr) {
    const int n = (int)M.node.size();
    std::vector<std::vector<int>> adj(n);
    auto join = [&](int a, int b) {
        if (a == b) return;
        adj[a].push_back(b), adj[b].push_back(a);
    };
    for (const auto& m : M.mn) join(m[0], m[1]);
    for (size_t t = 0; t < M.tn.size(); t++)
        if (!M.tbroken[t])
            for (int e = 0; e < 3; e++) join(M.tn[t][e], M.tn[t][(e + 1) % 3]);
    ptr.assign(n + 1, 0);
    nbr.clear();
    for (int i = 0; i < n; i++) {
        std::sort(adj[i].begin(), adj[i].end());
        adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
        nbr.insert(nbr.end(), adj[i].begin(), adj[i].end());
        ptr[i + 1] = (int)nbr.size();
    }
}

// connected components by breadth-first search from each not yet labelled node in ascending order: component c is
// the one whose lowest node is the c-th lowest such node
static FemComponents fem_components(int n, const std::vector<int>& ptr, const std::vector<int>& nbr) {
    FemComponents C;
    C.of.assign(n, -1);
    std::vector<int> queue;
    for (int s = 0; s < n; s++) {
        if (C.of[s] >= 0) continue;
        const int c = C.count++;
        queue.assign(1, s);
        C.of[s] = c;
        for (size_t h = 0; h < queue.size(); h++)
            for (int q = ptr[queue[h]]; q < ptr[queue[h] + 1]; q++)
                if (C.of[nbr[q]] < 0) C.of[nbr[q]] = c, queue.push_back(nbr[q]);
        std::sort(queue.begin(), queue.end());
        C.nodes.push_back(queue);
    }
    return C;
}

// Exact minimum degree on the quotient graph of one component. Appends the component's nodes to order (in elimination
// order) and, per eliminated node, its neighbours at elimination (frame node ids) to reach / reach_ptr.
struct QuotientGraph {
    std::vector<std::vector<int>> var_adj;  // per node: node neighbours not yet covered by an element
    std::vector<std::vector<int>> elem_adj; // per node: adjacent elements (an element is named by its eliminated node)
    std::vector<std::vector<int>> members;  // per element: the nodes of its clique
    std::vector<uint8_t> eliminated, absorbed;
    std::vector<int> degree, mark;
    int stamp = 0;

    explicit QuotientGraph(int n) : var_adj(n), elem_adj(n), members(n), eliminated(n, 0), absorbed(n, 0), degree(n, 0), mark(n, 0) {}

    int next_stamp() {
        if (++stamp == 0x7fffffff) std::fill(mark.begin(), mark.end(), 0), stamp = 1;
        return stamp;
    }
    // |neighbourhood of y| - |fresh| where the nodes of element `fresh` (marked with `inside`) are counted by the caller
    int outside_count(int y, int fresh, int inside) {
        const int seen = next_stamp();
        int d = 0;
        for (int z : var_adj[y])
            if (mark[z] != inside && mark[z] != seen) mark[z] = seen, d++;
        for (int e : elem_adj[y]) {
            if (e == fresh) continue;
            for (int z : members[e])
                if (z != y && mark[z] != inside && mark[z] != seen) mark[z] = seen, d++;
        }
        return d;
    }
};

static void fem_min_degree(const std::vector<int>& comp, const std::vector<int>& ptr, const std::vector<int>& nbr, QuotientGraph& G,
                           std::vector<int>& order, std::vector<int>& reach, std::vector<int>& reach_ptr) {
    typedef std::pair<int, int> Key; // (degree, node): the heap's least is the next pivot
    std::vector<Key> heap;
    auto push = [&](int d, int y) {
        heap.push_back({d, y});
        std::push_heap(heap.begin(), heap.end(), std::greater<Key>());
    };
    for (int x : comp) {
        G.var_adj[x].assign(nbr.begin() + ptr[x], nbr.begin() + ptr[x + 1]);
        G.degree[x] = ptr[x + 1] - ptr[x];
        push(G.degree[x], x);
    }
    std::vector<int> clique;
    for (size_t step = 0; step < comp.size(); step++) {
        int p = -1;
        while (p < 0) {
            std::pop_heap(heap.begin(), heap.end(), std::greater<Key>());
            const Key k = heap.back();
            heap.pop_back();
            if (!G.eliminated[k.second] && G.degree[k.second] == k.first) p = k.second;
        }
        G.eliminated[p] = 1;
        order.push_back(p);
        // p's neighbourhood: its node neighbours and the nodes of its elements, which p's element absorbs
        const int in = G.next_stamp();
        G.mark[p] = in;
        clique.clear();
        for (int z : G.var_adj[p])
            if (G.mark[z] != in) G.mark[z] = in, clique.push_back(z);
        for (int e : G.elem_adj[p]) {
            for (int z : G.members[e])
                if (G.mark[z] != in) G.mark[z] = in, clique.push_back(z);
            G.absorbed[e] = 1;
            std::vector<int>().swap(G.members[e]);
        }
        std::vector<int>().swap(G.var_adj[p]);
        std::vector<int>().swap(G.elem_adj[p]);
        reach.insert(reach.end(), clique.begin(), clique.end());
        reach_ptr.push_back((int)reach.size());
        G.members[p] = clique;
        // each neighbour: its node neighbours inside the clique are now covered by p's element (p itself goes too),
        // its absorbed elements are replaced by p's; then its exact degree
        for (int y : clique) {
            std::vector<int>& va = G.var_adj[y];
            size_t w = 0;
            for (int z : va)
                if (G.mark[z] != in) va[w++] = z;
            va.resize(w);
            std::vector<int>& ea = G.elem_adj[y];
            w = 0;
            for (int e : ea)
                if (!G.absorbed[e]) ea[w++] = e;
            ea.resize(w);
            ea.push_back(p);
        }
        const int base = (int)clique.size() - 1; // (each neighbour sees the rest of the clique)
        for (int y : clique) {
            const int d = base + G.outside_count(y, p, in);
            if (d != G.degree[y]) G.degree[y] = d, push(d, y);
        }
    }
}

// The pattern's block updates, whether or not their list is built: sum over the columns of d (d + 1) / 2
static int64_t fem_update_count(const FemModel& M) {
    int64_t u = 0;
    for (size_t k = 0; k + 1 < M.col_ptr.size(); k++) u += (int64_t)(M.col_ptr[k + 1] - M.col_ptr[k]) * (M.col_ptr[k + 1] - M.col_ptr[k] + 1) / 2;
    return u;
}

// The update list of the column-by-column factorization: each source column k: the rows of column c = row[i]
// scattered into a position table once, then every later row j of column k looked up in it
static void fem_update_list(FemModel& M) {
    const int n = (int)M.node.size();
    M.upd.clear();
    M.upd_ptr.assign(n + 1, 0);
    std::vector<int> pos(n, -1);
    for (int k = 0; k < n; k++) {
        const int a0 = M.col_ptr[k], a1 = M.col_ptr[k + 1];
        for (int i = a0; i < a1; i++) {
            const int c = M.row[i];
            for (int q = M.col_ptr[c]; q < M.col_ptr[c + 1]; q++) pos[M.row[q]] = q;
            M.upd.push_back({i, i, -(c + 1)});
            for (int j = i + 1; j < a1; j++) M.upd.push_back({i, j, pos[M.row[j]]});
            for (int q = M.col_ptr[c]; q < M.col_ptr[c + 1]; q++) pos[M.row[q]] = -1;
        }
        M.upd_ptr[k + 1] = (int)M.upd.size();
    }
}

// FemModel's ordering, pattern, block maps and gather lists; the update list too where want_updates
static void fem_analyse(FemModel& M, bool want_updates = true) {
    const int n = (int)M.node.size();
    const size_t T = M.tn.size(), E = M.mn.size();
    std::vector<int> gptr, gnbr;
    fem_graph(M, gptr, gnbr);
    const FemComponents C = fem_components(n, gptr, gnbr);
    M.ncomp = C.count;
    M.comp_first.assign(C.count + 1, 0);
    std::vector<int> order, reach, reach_ptr(1, 0);
    order.reserve(n);
    QuotientGraph G(n);
    for (int c = 0; c < C.count; c++) {
        M.comp_first[c] = (int)order.size();
        fem_min_degree(C.nodes[c], gptr, gnbr, G, order, reach, reach_ptr);
    }
    M.comp_first[C.count] = n;
    M.perm = order;
    M.iperm.assign(n, 0);
    for (int k = 0; k < n; k++) M.iperm[order[k]] = k;
    // the pattern: column k's rows are the elimination positions of its node's neighbours at elimination, ascending
    M.col_ptr.assign(reach_ptr.begin(), reach_ptr.end());
    M.row.resize(reach.size());
    for (size_t q = 0; q < reach.size(); q++) M.row[q] = M.iperm[reach[q]];
    for (int k = 0; k < n; k++) std::sort(M.row.begin() + M.col_ptr[k], M.row.begin() + M.col_ptr[k + 1]);
    // the off-diagonal block (row r, column k < r): its index in row, or -1 where the pattern has none
    auto block_at = [&](int k, int r) {
        const auto first = M.row.begin() + M.col_ptr[k], last = M.row.begin() + M.col_ptr[k + 1];
        const auto range = std::equal_range(first, last, r);
        return range.first == range.second ? -1 : (int)(range.first - M.row.begin());
    };
    M.upd.clear();
    M.upd_ptr.assign(n + 1, 0);
    if (want_updates) fem_update_list(M);
    // each member's and each triangle edge's block (the block's row is the end eliminated later)
    M.mblock.assign(E, -1), M.mswap.assign(E, 0);
    for (size_t e = 0; e < E; e++) {
        const int ka = M.iperm[M.mn[e][0]], kb = M.iperm[M.mn[e][1]];
        if (ka != kb) M.mblock[e] = block_at(std::min(ka, kb), std::max(ka, kb)), M.mswap[e] = ka > kb;
    }
    M.tri_block.assign(T, {-1, -1, -1});
    M.tri_swap.assign(T, {0, 0, 0});
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        for (int e = 0; e < 3; e++) {
            const int ki = M.iperm[M.tn[t][e]], kj = M.iperm[M.tn[t][(e + 1) % 3]];
            if (ki != kj) M.tri_block[t][e] = block_at(std::min(ki, kj), std::max(ki, kj)), M.tri_swap[t][e] = ki > kj;
        }
    }
    // gather lists: each column's entries (members' ends, then triangles' corners) and each block's (members, then
    // triangle edges), each in element order - built as lists and flattened
    std::vector<std::vector<std::array<int, 2>>> dl(n);
    std::vector<std::vector<std::array<int, 3>>> ol(M.row.size());
    for (size_t e = 0; e < E; e++) {
        const int tag = -(int)e - 1;
        dl[M.iperm[M.mn[e][0]]].push_back({tag, 0});
        dl[M.iperm[M.mn[e][1]]].push_back({tag, 1});
        if (M.mblock[e] >= 0) ol[M.mblock[e]].push_back({tag, M.mswap[e] ? 3 : 2, 0}); // (3: the row node is the a end)
    }
    for (size_t t = 0; t < T; t++) {
        if (M.tbroken[t]) continue;
        for (int c = 0; c < 3; c++) dl[M.iperm[M.tn[t][c]]].push_back({(int)t, c});
        for (int e = 0; e < 3; e++) {
            if (M.tri_block[t][e] < 0) continue;
            const int i = e, j = (e + 1) % 3; // (the entry: the block's row corner, then its column corner)
            ol[M.tri_block[t][e]].push_back(M.tri_swap[t][e] ? std::array<int, 3>{(int)t, i, j} : std::array<int, 3>{(int)t, j, i});
        }
    }
    M.gdiag_ptr.assign(1, 0), M.goff_ptr.assign(1, 0);
    M.gdiag.clear(), M.goff.clear();
    for (const auto& l : dl) M.gdiag.insert(M.gdiag.end(), l.begin(), l.end()), M.gdiag_ptr.push_back((int)M.gdiag.size());
    for (const auto& l : ol) M.goff.insert(M.goff.end(), l.begin(), l.end()), M.goff_ptr.push_back((int)M.goff.size());
}

} // namespace blg
