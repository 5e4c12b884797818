// The implicit FEM step solved by preconditioned conjugate gradients, and the solve's residual.
//
// (A dv = rhs: the system k_fem_assemble_all leaves in diag / off / rhs - M + (theta h^2 + beta h) K + theta h^2 Kg over
// the frame's 6-DOF nodes, frame_fem.cpp:916-1086 - in the factor's column order.) The reference solves it by the
// block Cholesky (frame_fem.cpp:2887-2954), which this library runs as the default and as the arbiter of its error.
// k_fem_pcg solves the same system by CG with a block-Jacobi preconditioner (each column's 6 x 6 diagonal block, its translational 3 x 3
// part optionally scaled by a learned S: z = T D^-1 T^T r with T = diag(S, I), symmetric positive definite for any
// invertible S) from an initial guess: zero, or the best combination (in the energy norm: the Galerkin projection onto
// their span) of the last substep's solution and, with the learned warm start, the network's per-node dv. The
// projection makes a guess safe: its error in the A-norm is never larger than that of a zero start, however rough the
// network's prediction. One cooperative launch per solve: a warp per
// column for A p (the column's lower blocks transposed plus its row's blocks, fill blocks skipped), grid-wide sums in
// a fixed order (the result does not depend on timing), until |r| <= tol |rhs| or the iteration budget is spent. On
// success it writes dv where the Cholesky would have left it and clears the graph's condition, so the factorization
// (captured under a conditional node) does not run; otherwise rhs stays and the Cholesky solves it: the fallback.
#pragma once

#include <cooperative_groups.h>

#include "bl_fem_kernels.cuh"

namespace blg {

namespace cgr = cooperative_groups;

struct PcgArgs {
    double* x;               // 6 / column
    double* r;
    double* z;
    double* p;
    double* pf;              // 36 / column: Cholesky factor of the column's diagonal block
    double* pdi;             // 6 / column: its inverse diagonal
    const float* guess;      // 3 / frame node: the network's translational dv (null: none)
    double* xprev;           // 6 / column: the last substep's solution (kept here after every solve)
    int use_prev;            // the last solution joins the initial guess
    const float* scale;      // 9 / frame node: the preconditioner's translational scale S (null: identity)
    double* red;             // 2 x 8 / warp of the grid: partial sums (two buffers used in turn: a block may still read
                             // one reduction's partials while another block writes the next's)
    int* stat;               // [0] solves [1] fallbacks [2] iterations of the last solve [3] solves with a failed block factor
    long long* iters_total;
    double* last_res;        // relative residual of the last solve
    cudaGraphConditionalHandle cond; // set to 1 when the Cholesky must run
    int has_cond;
    int max_iters;
    double tol;
};

// y = (A x)_k for column k by one warp (lane 0 gets the result): its diagonal block, its lower blocks transposed
// (A_{k,row} = A_{row,k}^T) and its row's blocks (A_{k,col}); blocks no element touches (the factor's fill) are zero
__device__ __forceinline__ void spmv_col(const FemDev& F, const double* __restrict__ Ad, const double* __restrict__ Ao, int k,
                                         const double* __restrict__ x, int lane, double* y) {
    double s[6] = {0, 0, 0, 0, 0, 0};
    for (int pb = F.col_ptr[k] + lane; pb < F.col_ptr[k + 1]; pb += 32) {
        if (F.goff_ptr[pb] == F.goff_ptr[pb + 1]) continue;
        const double* B = Ao + 36 * (size_t)pb;
        const double* xr = x + 6 * (size_t)F.row[pb];
        for (int j = 0; j < 6; j++) {
            double t = 0;
            for (int i = 0; i < 6; i++) t += B[i * 6 + j] * xr[i];
            s[j] += t;
        }
    }
    for (int q = F.rb_ptr[k] + lane; q < F.rb_ptr[k + 1]; q += 32) {
        const int2 bc = F.rb[q];
        if (F.goff_ptr[bc.x] == F.goff_ptr[bc.x + 1]) continue;
        const double* B = Ao + 36 * (size_t)bc.x;
        const double* xc = x + 6 * (size_t)bc.y;
        for (int i = 0; i < 6; i++) {
            double t = 0;
            for (int j = 0; j < 6; j++) t += B[i * 6 + j] * xc[j];
            s[i] += t;
        }
    }
    for (int j = 0; j < 6; j++) s[j] = warp_sum(s[j]);
    if (lane == 0) {
        const double* D = Ad + 36 * (size_t)k;
        const double* xk = x + 6 * (size_t)k;
        for (int i = 0; i < 6; i++) {
            double t = 0;
            for (int j = 0; j < 6; j++) t += D[i * 6 + j] * xk[j];
            y[i] = t + s[i];
        }
    }
}

// z = T D^-1 T^T r for column k (one thread), D^-1 through the block's Cholesky factor
__device__ __forceinline__ void precond(const PcgArgs& P, const FemDev& F, int k, const double* r, double* z) {
    const double* L = P.pf + 36 * (size_t)k;
    const double* di = P.pdi + 6 * (size_t)k;
    double u[6];
    for (int j = 0; j < 6; j++) u[j] = r[j];
    const float* S = P.scale ? P.scale + 9 * (size_t)F.perm[k] : nullptr;
    if (S) { // T^T r: S^T on the translational part
        const double a = u[0], b = u[1], c = u[2];
        u[0] = S[0] * a + S[3] * b + S[6] * c, u[1] = S[1] * a + S[4] * b + S[7] * c, u[2] = S[2] * a + S[5] * b + S[8] * c;
    }
    for (int j = 0; j < 6; j++) {
        double t = u[j];
        for (int m = 0; m < j; m++) t -= L[j * 6 + m] * u[m];
        u[j] = t * di[j];
    }
    for (int j = 5; j >= 0; j--) {
        double t = u[j];
        for (int m = j + 1; m < 6; m++) t -= L[m * 6 + j] * u[m];
        u[j] = t * di[j];
    }
    if (S) {
        const double a = u[0], b = u[1], c = u[2];
        u[0] = S[0] * a + S[1] * b + S[2] * c, u[1] = S[3] * a + S[4] * b + S[5] * c, u[2] = S[6] * a + S[7] * b + S[8] * c;
    }
    for (int j = 0; j < 6; j++) z[j] = u[j];
}

// the grid's partial sums (buffer `buf`, 8 a warp) added in a fixed order by warp 0 of each block into s_tot: every
// block gets the same totals, so every block takes the same branches and meets the same grid syncs
__device__ __forceinline__ void grid_totals(const PcgArgs& P, int buf, int nw, int nv, double* s_tot) {
    const double* red = P.red + (size_t)buf * 8 * nw;
    if (threadIdx.x < 32) {
        double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int w = threadIdx.x; w < nw; w += 32)
            for (int c = 0; c < nv; c++) t[c] += red[8 * (size_t)w + c];
        for (int c = 0; c < nv; c++) t[c] = warp_sum(t[c]);
        if (threadIdx.x == 0)
            for (int c = 0; c < nv; c++) s_tot[c] = t[c];
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_fem_pcg(FemDev F, PcgArgs P) {
    cgr::grid_group grid = cgr::this_grid();
    __shared__ double s_tot[8];
    const int lane = threadIdx.x & 31;
    const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
    const int nf = F.nf;
    double* red0 = P.red;                  // (the loop's first reduction)
    double* red1 = P.red + 8 * (size_t)nw; // (the set-up's and the loop's second)
    const bool guess = P.guess || P.use_prev;
    // ---- the preconditioner's factors; the guess's basis: u1 = the network's dv (in x), u2 = the last solution (in p)
    double nbad = 0;
    for (int k = gw; k < nf; k += nw) {
        if (lane != 0) continue;
        double* L = P.pf + 36 * (size_t)k;
        const double* D = F.diag + 36 * (size_t)k;
        for (int x = 0; x < 36; x++) L[x] = D[x];
        if (!chol6_dev(L, P.pdi + 6 * (size_t)k)) nbad += 1;
        const int i = F.perm[k];
        const bool fx = F.fixed[k] != 0;
        for (int j = 0; j < 6; j++) {
            P.x[6 * (size_t)k + j] = (P.guess && !fx && j < 3) ? (double)P.guess[3 * i + j] : 0.0;
            P.p[6 * (size_t)k + j] = (P.use_prev && !fx) ? P.xprev[6 * (size_t)k + j] : 0.0;
        }
    }
    double a1 = 0, a2 = 0;
    if (guess) {
        // Galerkin: x0 = a1 u1 + a2 u2 with [u.A u][a] = [u.b]; A u1 into z, A u2 into r
        grid.sync();
        double pr[6] = {0, 0, 0, 0, 0, 0};
        for (int k = gw; k < nf; k += nw) {
            double au1[6], au2[6];
            spmv_col(F, F.diag, F.off, k, P.x, lane, au1);
            spmv_col(F, F.diag, F.off, k, P.p, lane, au2);
            if (lane != 0) continue;
            const double* b = F.rhs + 6 * (size_t)k;
            const double* u1 = P.x + 6 * (size_t)k;
            const double* u2 = P.p + 6 * (size_t)k;
            for (int j = 0; j < 6; j++) {
                P.z[6 * (size_t)k + j] = au1[j], P.r[6 * (size_t)k + j] = au2[j];
                pr[0] += u1[j] * au1[j], pr[1] += u1[j] * au2[j], pr[2] += u2[j] * au2[j], pr[3] += u1[j] * b[j], pr[4] += u2[j] * b[j];
            }
        }
        if (lane == 0)
            for (int c = 0; c < 5; c++) red0[8 * (size_t)gw + c] = pr[c];
        grid.sync();
        grid_totals(P, 0, nw, 5, s_tot);
        const double g11 = s_tot[0], g12 = s_tot[1], g22 = s_tot[2], c1 = s_tot[3], c2 = s_tot[4];
        const double det = g11 * g22 - g12 * g12;
        if (g11 > 0 && g22 > 0 && det > 1e-12 * g11 * g22) {
            a1 = (c1 * g22 - c2 * g12) / det, a2 = (g11 * c2 - g12 * c1) / det;
        } else if (g11 > 0 && (!(g22 > 0) || c1 * c1 / g11 >= c2 * c2 / g22)) {
            a1 = c1 / g11;
        } else if (g22 > 0) {
            a2 = c2 / g22;
        }
        if (!(a1 == a1) || !(a2 == a2)) a1 = a2 = 0; // (NaN: from zero)
    }
    grid.sync();
    // ---- x0, r = b - A x0, z = P r, p = z
    double pr[4] = {0, 0, 0, 0}; // (lane 0: b.b, r.z, r.r)
    for (int k = gw; k < nf; k += nw) {
        if (lane != 0) continue;
        const double* b = F.rhs + 6 * (size_t)k;
        double r[6], z[6];
        for (int j = 0; j < 6; j++) {
            const size_t q = 6 * (size_t)k + j;
            if (guess) {
                r[j] = b[j] - a1 * P.z[q] - a2 * P.r[q];
                P.x[q] = a1 * P.x[q] + a2 * P.p[q];
            } else {
                r[j] = b[j];
                P.x[q] = 0.0;
            }
        }
        precond(P, F, k, r, z);
        for (int j = 0; j < 6; j++) {
            P.r[6 * (size_t)k + j] = r[j], P.z[6 * (size_t)k + j] = z[j], P.p[6 * (size_t)k + j] = z[j];
            pr[0] += b[j] * b[j], pr[1] += r[j] * z[j], pr[2] += r[j] * r[j];
        }
    }
    if (lane == 0) {
        for (int c = 0; c < 3; c++) red1[8 * (size_t)gw + c] = pr[c];
        red1[8 * (size_t)gw + 3] = nbad;
    }
    grid.sync();
    grid_totals(P, 1, nw, 4, s_tot);
    const double bb = s_tot[0];
    double rz = s_tot[1], rr = s_tot[2];
    const double lim = P.tol * P.tol * bb;
    const bool bad = s_tot[3] > 0 || !(rr == rr); // (a diagonal block not positive definite, a NaN: the Cholesky decides)
    int it = 0;
    bool ok = !bad && rr <= lim;
    while (!ok && !bad && it < P.max_iters) {
        it++;
        // q = A p (in z's place after use: kept in r's partner buffer q := z), p.q
        double pq = 0;
        for (int k = gw; k < nf; k += nw) {
            double q[6];
            spmv_col(F, F.diag, F.off, k, P.p, lane, q);
            if (lane != 0) continue;
            const double* pk = P.p + 6 * (size_t)k;
            for (int j = 0; j < 6; j++) P.z[6 * (size_t)k + j] = q[j], pq += pk[j] * q[j];
        }
        if (lane == 0) red0[8 * (size_t)gw] = pq;
        grid.sync();
        grid_totals(P, 0, nw, 1, s_tot);
        const double alpha = rz / s_tot[0];
        double rzn = 0, rrn = 0;
        for (int k = gw; k < nf; k += nw) {
            if (lane != 0) continue;
            double* xk = P.x + 6 * (size_t)k;
            double* rk = P.r + 6 * (size_t)k;
            double* zk = P.z + 6 * (size_t)k;
            const double* pk = P.p + 6 * (size_t)k;
            double r[6], z[6];
            for (int j = 0; j < 6; j++) xk[j] += alpha * pk[j], r[j] = rk[j] - alpha * zk[j], rk[j] = r[j];
            precond(P, F, k, r, z);
            for (int j = 0; j < 6; j++) zk[j] = z[j], rzn += r[j] * z[j], rrn += r[j] * r[j];
        }
        if (lane == 0) red1[8 * (size_t)gw] = rzn, red1[8 * (size_t)gw + 1] = rrn;
        grid.sync();
        grid_totals(P, 1, nw, 2, s_tot);
        rr = s_tot[1];
        if (!(rr == rr)) break; // (NaN: the Cholesky decides)
        if (rr <= lim) {
            ok = true;
            break;
        }
        const double beta = s_tot[0] / rz;
        rz = s_tot[0];
        for (int k = gw; k < nf; k += nw) {
            if (lane != 0) continue;
            double* pk = P.p + 6 * (size_t)k;
            const double* zk = P.z + 6 * (size_t)k;
            for (int j = 0; j < 6; j++) pk[j] = zk[j] + beta * pk[j];
        }
        grid.sync();
    }
    if (ok)
        for (int k = gw; k < nf; k += nw)
            if (lane == 0)
                for (int j = 0; j < 6; j++) F.rhs[6 * (size_t)k + j] = P.x[6 * (size_t)k + j];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.stat[0]++;
        if (!ok) P.stat[1]++;
        if (bad) P.stat[3]++;
        P.stat[2] = it;
        *P.iters_total += it;
        *P.last_res = bb > 0 ? sqrt(rr / bb) : 0.0;
        if (P.has_cond) cudaGraphSetConditional(P.cond, ok ? 0u : 1u);
    }
}

// The relative residual |A x - b| / |b| of the system as assembled (copies Ad, Ao, b made before the factorization)
// for the solution x the step took (rhs): a check of the solve, kept as its maximum in res[0] (res[1], res[2]: the
// sums of this solve). One warp a column; the sums by atomics (a diagnostic: their order may vary).
__global__ void __launch_bounds__(128) k_fem_residual(FemDev F, const double* __restrict__ Ad, const double* __restrict__ Ao,
                                                      const double* __restrict__ b, double* __restrict__ res) {
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (k >= F.nf) return;
    double ax[6];
    spmv_col(F, Ad, Ao, k, F.rhs, lane, ax);
    if (lane != 0) return;
    double rr = 0, bb = 0;
    for (int j = 0; j < 6; j++) {
        const double d = ax[j] - b[6 * (size_t)k + j];
        rr += d * d, bb += b[6 * (size_t)k + j] * b[6 * (size_t)k + j];
    }
    atomicAdd(&res[1], rr);
    atomicAdd(&res[2], bb);
}

__global__ void k_fem_residual_done(double* res) {
    const double r = res[2] > 0 ? sqrt(res[1] / res[2]) : 0.0;
    if (r > res[0] || !(r == r)) res[0] = r;
    res[3] = r;
    res[1] = res[2] = 0.0;
}

} // namespace blg
