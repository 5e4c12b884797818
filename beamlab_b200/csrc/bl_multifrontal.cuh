// The multifrontal factorization and solves of the frames' implicit step (the plan: bl_mf_plan.cuh).
//
// Each front is a dense lower triangle, column-major (leading dimension: its size n in degrees of freedom), in the
// pool; its first p degrees of freedom are its pivots. Per level of the front tree, leaves first:
//   k_mf_assemble  a CTA per (front, 32-wide tile column): the tile column zeroed, the assembled system's blocks of its
//                  pivot columns (diag, off) scattered in, then each child's Schur complement added in the children's
//                  order (extend-add; a CTA owns its columns, so nothing races and the sums' order is fixed);
//   per 32-wide panel s of the pivots, two launches:
//   k_mf_panel     a warp per (front, row tile r >= s): the panel's diagonal tile factored in shared memory (every warp
//                  alike; the warp of r == s keeps it in the side buffer dt and writes the tile's trailing Schur
//                  complement, where the panel ends inside the tile, back to the front), then its row tile solved
//                  against it, X := X L^-T, and, past a partial panel, the rest of the row tile updated;
//   k_mf_update    a CTA per trailing tile (i >= j > s): A_ij -= L_is L_js^T; and a CTA per front copying the panel's
//                  diagonal tile back from dt (no warp of the panel launch reads the front's diagonal tile any more).
// Then, per level again, leaves first, k_mf_forward (a CTA per front: the front's right side from rhs and the
// children's update vectors, L y = b through its pivots panel by panel, its update vector for its parent), and from the
// root down k_mf_backward (a CTA per front: the pivots' right side less L21^T x of its rows, then L^T x = z). rhs holds
// the solution in column order, as the block-column path leaves it.
// A pivot that is not positive marks the front's component failed (the reference's chol6 failing, frame_fem.cpp:
// 2900-2909: that component's step falls back to its explicit forces); the factorization goes on with a unit pivot
// so that nothing but that component's numbers are touched.
#pragma once

#include "bl_fem_kernels.cuh"

namespace blg {

constexpr int kMfT = 32; // tile and panel width

struct MfFrontDev {
    long long off;   // its dense triangle in the pool (doubles)
    int n, p;        // degrees of freedom: all, pivots
    int idx0;        // its nodes (global columns: pivots, then rows) in idx; its rows' places in its parent's list at
                     // cmap[idx0 + p / 6]
    int child0, child1;
    int comp;
    int u0;          // its update vector (n - p doubles) in u
    int dt0;         // its diagonal tiles (a panel each, 32 x 32) in dt
};

struct MfDev {
    const MfFrontDev* fr;
    const int* idx;
    const int* cmap;
    const int* child;
    double* pool;
    double* u;
    double* dt;
    const int2* tcol; // assembly: (front, tile column)
    const int2* tpan; // panel: (front, row tile)
    const int4* tupd; // update: (front, i, j); i == j == -1: the diagonal tile copied back
};

// the node list's position of global column r in [lo, hi) (present by construction)
__device__ __forceinline__ int mf_find(const int* idx, int lo, int hi, int r) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (idx[mid] < r) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) k_mf_assemble(FemDev F, MfDev M, int t0) {
    const int2 task = M.tcol[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, c0 = kMfT * task.y, c1 = min(c0 + kMfT, n), npiv = fr.p / 6, nnode = n / 6;
    double* A = M.pool + fr.off;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rows = n - c0;
    for (int e = tid; e < (c1 - c0) * rows; e += blockDim.x) A[(size_t)(c0 + e / rows) * n + c0 + e % rows] = 0.0;
    __syncthreads();
    // the assembled blocks of the pivot columns in [c0, c1): a warp a degree-of-freedom column, a lane a row entry
    for (int c = c0 + warp; c < c1; c += 8) {
        const int l = c / 6, j = c % 6;
        if (l >= npiv) continue;
        const int k = M.idx[fr.idx0 + l];
        double* col = A + (size_t)c * n;
        if (lane < 6) col[6 * l + lane] = F.diag[36 * (size_t)k + 6 * lane + j];
        const int b0 = F.col_ptr[k], nb = F.col_ptr[k + 1] - b0;
        for (int e = lane; e < 6 * nb; e += 32) {
            const int pb = b0 + e / 6, i = e % 6;
            const int lr = mf_find(M.idx, fr.idx0, fr.idx0 + nnode, F.row[pb]) - fr.idx0;
            col[6 * lr + i] = F.off[36 * (size_t)pb + 6 * i + j];
        }
    }
    // the children's Schur complements, child after child
    const int cn0 = c0 / 6, cn1 = (c1 - 1) / 6; // this tile column's nodes
    for (int q = fr.child0; q < fr.child1; q++) {
        __syncthreads();
        const MfFrontDev cf = M.fr[M.child[q]];
        const int pc = cf.p, nc = cf.n, nr = (nc - pc) / 6;
        const int* cm = M.cmap + cf.idx0 + pc / 6;
        const double* Cm = M.pool + cf.off;
        // the child's row nodes that land in this tile column (cm ascends): [a, b)
        int lo = 0, hi = nr;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cm[mid] < cn0) lo = mid + 1;
            else hi = mid;
        }
        const int a = lo;
        hi = nr;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cm[mid] <= cn1) lo = mid + 1;
            else hi = mid;
        }
        const int b = lo;
        for (int cc = 6 * a + warp; cc < 6 * b; cc += 8) {
            const int C = 6 * cm[cc / 6] + cc % 6;
            if (C < c0 || C >= c1) continue;
            const double* src = Cm + (size_t)(pc + cc) * nc + pc;
            double* dst = A + (size_t)C * n;
            for (int rr = cc + lane; rr < nc - pc; rr += 32) dst[6 * cm[rr / 6] + rr % 6] += src[rr];
        }
    }
}

// The panel's diagonal tile [c0, c0 + 32)^2 of a front, rows/columns past n as zeros, factored in D over its first w
// columns by one warp (right-looking; lane = row). full: also the tile's trailing part (the Schur complement of the
// columns past w); otherwise only the first w columns are formed. Returns false at a pivot that is not positive.
__device__ __forceinline__ bool mf_factor_tile(double (*D)[kMfT + 1], double* dinv, int w, int ncols, bool full) {
    const int lane = threadIdx.x & 31;
    bool ok = true;
    const int jend = full ? ncols : w;
    for (int k = 0; k < w; k++) {
        __syncwarp();
        double dk = D[k][k];
        if (!(dk > 0)) ok = false, dk = 1.0;
        const double d = sqrt(dk), id = 1.0 / d;
        __syncwarp();
        if (lane == k) D[k][k] = d, dinv[k] = id;
        if (lane > k) D[lane][k] *= id;
        __syncwarp();
        if (lane > k)
            for (int j = k + 1; j <= lane && j < jend; j++) D[lane][j] -= D[lane][k] * D[j][k];
    }
    __syncwarp();
    return ok;
}

__global__ void __launch_bounds__(32) k_mf_panel(MfDev M, int t0, int s, int* comp_fail) {
    __shared__ double D[kMfT][kMfT + 1], R[kMfT][kMfT + 1], dinv[kMfT];
    const int2 task = M.tpan[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, c0 = kMfT * s, w = min(kMfT, fr.p - c0), ncols = min(kMfT, n - c0), lane = threadIdx.x;
    double* A = M.pool + fr.off;
    const bool diag = task.y == s;
    const int jload = diag ? ncols : w; // (a row tile's warp reads only the panel's columns of the diagonal tile)
    for (int j = 0; j < kMfT; j++) D[lane][j] = (j < jload && lane < ncols) ? A[(size_t)(c0 + j) * n + c0 + lane] : 0.0;
    __syncwarp();
    const bool ok = mf_factor_tile(D, dinv, w, ncols, diag);
    if (diag) {
        double* T = M.dt + fr.dt0 + (size_t)s * kMfT * kMfT; // (column-major, its first w columns)
        for (int j = 0; j < w; j++) T[j * kMfT + lane] = D[lane][j];
        for (int j = w; j < ncols; j++) // (the trailing Schur complement, lower part)
            if (lane >= j && lane < ncols) A[(size_t)(c0 + j) * n + c0 + lane] = D[lane][j];
        if (!ok && lane == 0) atomicExch(&comp_fail[fr.comp], 1);
        return;
    }
    const int r0 = kMfT * task.y, nr = min(kMfT, n - r0);
    for (int j = 0; j < ncols; j++) R[lane][j] = lane < nr ? A[(size_t)(c0 + j) * n + r0 + lane] : 0.0;
    __syncwarp();
    if (lane < nr) {
        for (int j = 0; j < w; j++) {
            double t = R[lane][j];
            for (int m = 0; m < j; m++) t -= R[lane][m] * D[j][m];
            R[lane][j] = t * dinv[j];
        }
        for (int j = w; j < ncols; j++) {
            double t = R[lane][j];
            for (int m = 0; m < w; m++) t -= R[lane][m] * D[j][m];
            R[lane][j] = t;
        }
        for (int j = 0; j < ncols; j++) A[(size_t)(c0 + j) * n + r0 + lane] = R[lane][j];
    }
}

__global__ void __launch_bounds__(256) k_mf_update(MfDev M, int t0, int s) {
    __shared__ double Li[kMfT][kMfT + 1], Lj[kMfT][kMfT + 1]; // [m][row]
    const int4 task = M.tupd[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, c0 = kMfT * s, w = min(kMfT, fr.p - c0), tid = threadIdx.x;
    double* A = M.pool + fr.off;
    if (task.y < 0) { // the panel's diagonal tile back into the front
        const double* T = M.dt + fr.dt0 + (size_t)s * kMfT * kMfT;
        const int ncols = min(kMfT, n - c0);
        for (int e = tid; e < w * kMfT; e += blockDim.x) {
            const int j = e / kMfT, i = e % kMfT;
            if (i >= j && i < ncols) A[(size_t)(c0 + j) * n + c0 + i] = T[j * kMfT + i];
        }
        return;
    }
    const int i0 = kMfT * task.y, j0 = kMfT * task.z;
    for (int e = tid; e < kMfT * kMfT; e += blockDim.x) {
        const int m = e / kMfT, r = e % kMfT;
        Li[m][r] = (m < w && i0 + r < n) ? A[(size_t)(c0 + m) * n + i0 + r] : 0.0;
        Lj[m][r] = (m < w && j0 + r < n) ? A[(size_t)(c0 + m) * n + j0 + r] : 0.0;
    }
    __syncthreads();
    const int r = tid & 31, g = tid >> 5; // (row r, columns 4 g .. 4 g + 3)
    double acc[4] = {0, 0, 0, 0};
    for (int m = 0; m < w; m++) {
        const double li = Li[m][r];
        for (int c = 0; c < 4; c++) acc[c] += li * Lj[m][4 * g + c];
    }
    if (i0 + r < n)
        for (int c = 0; c < 4; c++) {
            const int col = j0 + 4 * g + c;
            if (col < n && (task.y != task.z || 4 * g + c <= r)) A[(size_t)col * n + i0 + r] -= acc[c];
        }
}

// L y = b through a front's pivots; its update vector (its rows' part of b less L21 y) for its parent
__global__ void __launch_bounds__(256) k_mf_forward(FemDev F, MfDev M, int f0) {
    extern __shared__ double wsh[];
    __shared__ double T[kMfT][kMfT + 1];
    const MfFrontDev fr = M.fr[f0 + blockIdx.x];
    const int n = fr.n, p = fr.p, tid = threadIdx.x;
    const int* idx = M.idx + fr.idx0;
    const double* A = M.pool + fr.off;
    for (int e = tid; e < n; e += blockDim.x) wsh[e] = e < p ? F.rhs[6 * (size_t)idx[e / 6] + e % 6] : 0.0;
    for (int q = fr.child0; q < fr.child1; q++) {
        __syncthreads();
        const MfFrontDev cf = M.fr[M.child[q]];
        const int* cm = M.cmap + cf.idx0 + cf.p / 6;
        const double* uc = M.u + cf.u0;
        for (int e = tid; e < cf.n - cf.p; e += blockDim.x) wsh[6 * cm[e / 6] + e % 6] += uc[e];
    }
    for (int s = 0; kMfT * s < p; s++) {
        const int c0 = kMfT * s, w = min(kMfT, p - c0), nt = min(kMfT, n - c0);
        __syncthreads();
        if (tid < 32) {
            for (int j = 0; j < w; j++) T[tid][j] = tid < nt ? A[(size_t)(c0 + j) * n + c0 + tid] : 0.0;
            __syncwarp();
            for (int j = 0; j < w; j++) {
                const double yj = wsh[c0 + j] / T[j][j];
                __syncwarp();
                if (tid == j) wsh[c0 + j] = yj;
                else if (tid > j && tid < nt) wsh[c0 + tid] -= T[tid][j] * yj;
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = c0 + kMfT + tid; e < n; e += blockDim.x) {
            double t = 0;
            for (int j = 0; j < w; j++) t += A[(size_t)(c0 + j) * n + e] * wsh[c0 + j];
            wsh[e] -= t;
        }
    }
    __syncthreads();
    for (int e = tid; e < n; e += blockDim.x) {
        if (e < p) F.rhs[6 * (size_t)idx[e / 6] + e % 6] = wsh[e];
        else M.u[fr.u0 + e - p] = wsh[e];
    }
}

// L^T x = z through a front's pivots, its rows' x known (its ancestors')
__global__ void __launch_bounds__(256) k_mf_backward(FemDev F, MfDev M, int f0) {
    extern __shared__ double xsh[];
    __shared__ double T[kMfT][kMfT + 1];
    const MfFrontDev fr = M.fr[f0 + blockIdx.x];
    const int n = fr.n, p = fr.p, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int* idx = M.idx + fr.idx0;
    const double* A = M.pool + fr.off;
    for (int e = tid; e < n; e += blockDim.x) xsh[e] = F.rhs[6 * (size_t)idx[e / 6] + e % 6];
    __syncthreads();
    // z = y - L21^T x_rows: a warp a pivot column
    for (int j = warp; j < p; j += 8) {
        double t = 0;
        for (int e = p + lane; e < n; e += 32) t += A[(size_t)j * n + e] * xsh[e];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) xsh[j] -= t;
    }
    for (int s = (p - 1) / kMfT; s >= 0; s--) {
        const int c0 = kMfT * s, w = min(kMfT, p - c0), b1 = min(c0 + kMfT, p);
        __syncthreads();
        // the pivot rows below the panel: z_j -= sum_{e in [c0 + 32, p)} L_ej x_e
        for (int j = c0 + warp; j < b1; j += 8) {
            double t = 0;
            for (int e = b1 + lane; e < p; e += 32) t += A[(size_t)j * n + e] * xsh[e];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) xsh[j] -= t;
        }
        __syncthreads();
        if (tid < 32) {
            for (int j = 0; j < w; j++) T[tid][j] = tid < w ? A[(size_t)(c0 + j) * n + c0 + tid] : 0.0;
            __syncwarp();
            for (int j = w - 1; j >= 0; j--) {
                double t = (tid > j && tid < w) ? T[tid][j] * xsh[c0 + tid] : 0.0;
                for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
                if (tid == 0) xsh[c0 + j] = (xsh[c0 + j] - t) / T[j][j];
                __syncwarp();
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < p; e += blockDim.x) F.rhs[6 * (size_t)idx[e / 6] + e % 6] = xsh[e];
}

} // namespace blg
