// The multifrontal factorization and solves of the frames' implicit step (the plan: bl_mf_plan.cuh).
//
// Each front is dense and column-major in the pool: n x (n + 1) doubles, leading dimension n (its size in degrees of
// freedom); its first p degrees of freedom are its pivots, its last column the right side b. Only the lower triangle of
// the first n columns is used. Factoring the pivots with b carried along as one more column gives, in b, the forward
// substitution's y on the pivots and the update vector of the rows (b_rows - L21 y) for the parent, as the Schur
// complement of the rows is left in the trailing triangle: no separate forward pass.
// Per level of the front tree, leaves first:
//   k_mf_assemble  a CTA per 32 x 32 tile of a front's lower triangle (and per 32-row tile of b): zeroed, the assembled
//                  system's blocks of the pivot columns (diag, off; each off block's row in the front precomputed)
//                  written in, then each child's Schur complement (and update vector) added in the children's order -
//                  extend-add; a CTA owns its tile, so nothing races and the sums' order is fixed;
//   per 32-wide panel s of the pivots, two launches:
//   k_mf_panel     a CTA per (front, row tile r >= s): the panel's diagonal tile factored and its triangle inverted in
//                  shared memory by the whole block (every CTA alike); the CTA of r == s keeps both in the side buffer dt,
//                  writes the tile's trailing Schur complement where the panel ends inside the tile, and solves the
//                  panel's part of b (y_s = L_ss^-1 b_s); a row tile's CTA forms X = A_rs L_ss^-T by all its warps and,
//                  past a partial panel, updates the rest of its tile;
//   k_mf_update    a CTA per trailing tile (i >= j > s): A_ij -= L_is L_js^T; per row tile i > s of b: b_i -= L_is y_s;
//                  and per front the panel's diagonal tile copied back from dt (no CTA of the panel launch reads the
//                  front's diagonal tile any more).
// Then from the root down, k_mf_backward (a CTA per front): z = y - L21^T x of its rows (its ancestors' solution), then
// panel by panel from the last, z_s -= L_(below,s)^T x_below and x_s = L_ss^-T z_s with the stored inverse. rhs gets
// the solution in column order, as the block-column path leaves it.
// A pivot that is not positive marks the front's component failed (the reference's chol6 failing, frame_fem.cpp:
// 2900-2909: that component's step falls back to its explicit forces); the factorization goes on with a unit pivot
// so that nothing but that component's numbers are touched.
#pragma once

#include "bl_fem_kernels.cuh"

namespace blg {

constexpr int kMfT = 32; // tile and panel width

struct MfFrontDev {
    long long off;   // its dense block in the pool (doubles): n x (n + 1), column-major
    int n, p;        // degrees of freedom: all, pivots
    int idx0;        // its nodes (global columns: pivots, then rows) in idx; its rows' places in its parent's list at
                     // cmap[idx0 + p / 6]
    int child0, child1;
    int comp;
    int dt0;         // its diagonal tiles and their inverses (a panel each: 2 x 32 x 32) in dt
};

struct MfDev {
    const MfFrontDev* fr;
    const int* idx;
    const int* cmap;
    const int* child;
    const int* brow;  // per off-diagonal block of the pattern: its row's node in the front of its column
    double* pool;
    double* dt;
    const int4* tasm; // assembly: (front, row tile, column tile; -1: b)
    const int2* tpan; // panel: (front, row tile)
    const int4* tupd; // update: (front, i, j); (-1, -1): the diagonal tile copied back; (i, -2): b's row tile i
};

// the range [lo, hi) of nodes q of a child's rows (cm ascending) whose places in the parent lie in [a, b]
__device__ __forceinline__ void mf_range(const int* cm, int nr, int a, int b, int& lo, int& hi) {
    int l = 0, h = nr;
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (cm[mid] < a) l = mid + 1;
        else h = mid;
    }
    lo = l, h = nr;
    while (l < h) {
        const int mid = (l + h) >> 1;
        if (cm[mid] <= b) l = mid + 1;
        else h = mid;
    }
    hi = l;
}

__global__ void __launch_bounds__(256) k_mf_assemble(FemDev F, MfDev M, int t0) {
    const int4 task = M.tasm[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, npiv = fr.p / 6, tid = threadIdx.x;
    const bool rhs = task.z < 0;
    const int r0 = kMfT * task.y, r1 = min(r0 + kMfT, n);
    const int c0 = rhs ? n : kMfT * task.z, c1 = rhs ? n + 1 : min(c0 + kMfT, n);
    double* A = M.pool + fr.off;
    const int nr = r1 - r0, nc = c1 - c0;
    for (int e = tid; e < nr * nc; e += blockDim.x) A[(size_t)(c0 + e / nr) * n + r0 + e % nr] = 0.0;
    __syncthreads();
    if (rhs) {
        for (int r = r0 + tid; r < r1 && r < fr.p; r += blockDim.x) A[(size_t)n * n + r] = F.rhs[6 * (size_t)M.idx[fr.idx0 + r / 6] + r % 6];
    } else {
        // the assembled blocks of the pivot columns in [c0, c1) whose rows fall in [r0, r1): a thread a column entry
        for (int c = c0; c < c1; c++) {
            const int l = c / 6, j = c % 6;
            if (l >= npiv) break;
            const int k = M.idx[fr.idx0 + l];
            double* col = A + (size_t)c * n;
            const int b0 = F.col_ptr[k], nb = F.col_ptr[k + 1] - b0;
            for (int e = tid; e < 6 * (nb + 1); e += blockDim.x) {
                const int q = e / 6, i = e % 6;
                const int r = q == 0 ? 6 * l + i : 6 * M.brow[b0 + q - 1] + i;
                if (r < r0 || r >= r1) continue;
                col[r] = q == 0 ? F.diag[36 * (size_t)k + 6 * i + j] : F.off[36 * (size_t)(b0 + q - 1) + 6 * i + j];
            }
        }
    }
    // the children's Schur complements (and update vectors), child after child
    for (int q = fr.child0; q < fr.child1; q++) {
        __syncthreads();
        const MfFrontDev cf = M.fr[M.child[q]];
        const int pc = cf.p, ncd = cf.n, cnr = (ncd - pc) / 6;
        const int* cm = M.cmap + cf.idx0 + pc / 6;
        const double* Cm = M.pool + cf.off;
        int ra, rb;
        mf_range(cm, cnr, r0 / 6, (r1 - 1) / 6, ra, rb);
        if (ra >= rb) continue;
        if (rhs) {
            for (int rr = 6 * ra + tid; rr < 6 * rb; rr += blockDim.x) {
                const int R = 6 * cm[rr / 6] + rr % 6;
                if (R >= r0 && R < r1) A[(size_t)n * n + R] += Cm[(size_t)ncd * ncd + pc + rr];
            }
            continue;
        }
        int ca, cb;
        mf_range(cm, cnr, c0 / 6, (c1 - 1) / 6, ca, cb);
        const int nrr = 6 * (rb - ra), ncc = 6 * (cb - ca);
        for (int e = tid; e < nrr * ncc; e += blockDim.x) {
            const int cc = 6 * ca + e / nrr, rr = 6 * ra + e % nrr;
            if (rr < cc) continue;
            const int C = 6 * cm[cc / 6] + cc % 6, R = 6 * cm[rr / 6] + rr % 6;
            if (C < c0 || C >= c1 || R < r0 || R >= r1) continue;
            A[(size_t)C * n + R] += Cm[(size_t)(pc + cc) * ncd + pc + rr];
        }
    }
}

// The panel's diagonal tile (rows/columns past n as zeros) in D, factored over its first w columns by the whole block,
// right-looking, with the inverse of its w x w triangle built in the same sweep (Y starts as the identity; at column k
// its row k is scaled by the pivot's inverse and the rows below lose D_rk times it). full: also the tile's trailing
// part (the Schur complement of the columns past w). Two barriers a column; a thread a few entries of each update.
// (Measured against one warp owning a column each: that took 40 % longer, its lanes' loops uneven.) Returns false at a
// pivot that is not positive.
__device__ __forceinline__ bool mf_factor_tile(double (*D)[kMfT + 1], double (*Y)[kMfT + 1], int w, int ncols, bool full, int* bad) {
    const int tid = threadIdx.x, nth = blockDim.x;
    for (int e = tid; e < kMfT * kMfT; e += nth) {
        const int i = e & (kMfT - 1), j = e / kMfT;
        Y[i][j] = (i == j && i < w) ? 1.0 : 0.0;
    }
    if (tid == 0) *bad = 0;
    __syncthreads();
    const int jend = full ? ncols : w;
    for (int k = 0; k < w; k++) {
        double dk = D[k][k];
        if (!(dk > 0)) dk = 1.0;
        const double id = 1.0 / sqrt(dk);
        // the trailing lower triangle and the inverse's rows below k, from column k and row k of Y scaled on the fly
        for (int e = tid; e < kMfT * kMfT; e += nth) {
            const int i = e & (kMfT - 1), j = e / kMfT;
            if (j > k && j <= i && j < jend) D[i][j] -= (D[i][k] * id) * (D[j][k] * id);
            if (i > k && i < w && j <= k) Y[i][j] -= (D[i][k] * id) * (Y[k][j] * id);
        }
        __syncthreads();
        if (tid < kMfT) {
            if (tid > k) D[tid][k] *= id;
            else if (tid == k) {
                if (!(D[k][k] > 0)) *bad = 1;
                D[k][k] = 1.0 / id;
            }
        } else if (tid < 2 * kMfT && tid - kMfT <= k) {
            Y[k][tid - kMfT] *= id;
        }
        __syncthreads();
    }
    return *bad == 0;
}

__global__ void __launch_bounds__(256) k_mf_panel(MfDev M, int t0, int s, int* comp_fail) {
    __shared__ double D[kMfT][kMfT + 1], Li[kMfT][kMfT + 1], R[kMfT][kMfT + 1];
    __shared__ int bad;
    const int2 task = M.tpan[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, c0 = kMfT * s, w = min(kMfT, fr.p - c0), ncols = min(kMfT, n - c0), tid = threadIdx.x;
    double* A = M.pool + fr.off;
    const bool diag = task.y == s;
    const int jload = diag ? ncols : w; // (a row tile's CTA reads only the panel's columns of the diagonal tile)
    for (int e = tid; e < kMfT * kMfT; e += blockDim.x) {
        const int j = e / kMfT, i = e % kMfT;
        D[i][j] = (j < jload && i < ncols) ? A[(size_t)(c0 + j) * n + c0 + i] : 0.0;
    }
    __syncthreads();
    const bool ok = mf_factor_tile(D, Li, w, ncols, diag, &bad);
    if (diag) {
        double* T = M.dt + fr.dt0 + (size_t)s * 2 * kMfT * kMfT; // (L then L^-1, column-major)
        for (int e = tid; e < kMfT * kMfT; e += blockDim.x) {
            const int j = e / kMfT, i = e % kMfT;
            T[e] = D[i][j], T[kMfT * kMfT + e] = Li[i][j];
            if (j >= w && j < ncols && i >= j && i < ncols) A[(size_t)(c0 + j) * n + c0 + i] = D[i][j]; // (trailing Schur complement)
        }
        // b's panel rows: y_s = L^-1 b_s, then the tile's rows past w (past a partial panel): b_i -= L_i y_s
        double* b = A + (size_t)n * n + c0;
        __shared__ double y[kMfT];
        if (tid < kMfT) {
            double t = 0;
            if (tid < w)
                for (int m = 0; m <= tid; m++) t += Li[tid][m] * b[m];
            y[tid] = t;
        }
        __syncthreads();
        if (tid < w) b[tid] = y[tid];
        else if (tid < ncols) {
            double t = b[tid];
            for (int m = 0; m < w; m++) t -= D[tid][m] * y[m];
            b[tid] = t;
        }
        if (!ok && tid == 0) atomicExch(&comp_fail[fr.comp], 1);
        return;
    }
    const int r0 = kMfT * task.y, nr = min(kMfT, n - r0);
    for (int e = tid; e < kMfT * kMfT; e += blockDim.x) {
        const int j = e / kMfT, i = e % kMfT;
        R[i][j] = (j < ncols && i < nr) ? A[(size_t)(c0 + j) * n + r0 + i] : 0.0;
    }
    __syncthreads();
    // X = A_rs[:, :w] L^-T: X_ij = sum_{m <= j} A_im Li_jm; a thread four entries of one column
    const int i = tid & 31, jg = tid >> 5;
    double x[4];
    for (int c = 0; c < 4; c++) {
        const int j = 4 * jg + c;
        double t = 0;
        if (j < w)
            for (int m = 0; m <= j; m++) t += R[i][m] * Li[j][m];
        x[c] = t;
    }
    __syncthreads();
    for (int c = 0; c < 4; c++)
        if (4 * jg + c < w) R[i][4 * jg + c] = x[c];
    __syncthreads();
    // past a partial panel: the rest of the tile's columns less X L21_tile^T
    for (int c = 0; c < 4; c++) {
        const int j = 4 * jg + c;
        if (j < w || j >= ncols) continue;
        double t = R[i][j];
        for (int m = 0; m < w; m++) t -= R[i][m] * D[j][m];
        x[c] = t;
    }
    __syncthreads();
    for (int c = 0; c < 4; c++) {
        const int j = 4 * jg + c;
        if (j >= w && j < ncols) R[i][j] = x[c];
    }
    __syncthreads();
    for (int e = tid; e < kMfT * kMfT; e += blockDim.x) {
        const int j = e / kMfT, ii = e % kMfT;
        if (j < ncols && ii < nr) A[(size_t)(c0 + j) * n + r0 + ii] = R[ii][j];
    }
}

__global__ void __launch_bounds__(256) k_mf_update(MfDev M, int t0, int s) {
    __shared__ double Li[kMfT][kMfT + 1], Lj[kMfT][kMfT + 1]; // [m][row]
    const int4 task = M.tupd[t0 + blockIdx.x];
    const MfFrontDev fr = M.fr[task.x];
    const int n = fr.n, c0 = kMfT * s, w = min(kMfT, fr.p - c0), tid = threadIdx.x;
    double* A = M.pool + fr.off;
    if (task.z == -1) { // the panel's diagonal tile back into the front
        const double* T = M.dt + fr.dt0 + (size_t)s * 2 * kMfT * kMfT;
        const int ncols = min(kMfT, n - c0);
        for (int e = tid; e < w * kMfT; e += blockDim.x) {
            const int j = e / kMfT, i = e % kMfT;
            if (i >= j && i < ncols) A[(size_t)(c0 + j) * n + c0 + i] = T[e];
        }
        return;
    }
    const int i0 = kMfT * task.y;
    if (task.z == -2) { // b's row tile: b_i -= L_is y_s
        const double* b = A + (size_t)n * n;
        if (tid < kMfT && i0 + tid < n) {
            double t = 0;
            for (int m = 0; m < w; m++) t += A[(size_t)(c0 + m) * n + i0 + tid] * b[c0 + m];
            A[(size_t)n * n + i0 + tid] -= t;
        }
        return;
    }
    const int j0 = kMfT * task.z;
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

// L^T x = y through a front's pivots, its rows' x known (its ancestors'); y from the front's b column
__global__ void __launch_bounds__(256) k_mf_backward(FemDev F, MfDev M, int f0) {
    extern __shared__ double xsh[];
    __shared__ double Lt[kMfT][kMfT + 1];
    const MfFrontDev fr = M.fr[f0 + blockIdx.x];
    const int n = fr.n, p = fr.p, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int* idx = M.idx + fr.idx0;
    const double* A = M.pool + fr.off;
    for (int e = tid; e < n; e += blockDim.x) xsh[e] = e < p ? A[(size_t)n * n + e] : F.rhs[6 * (size_t)idx[e / 6] + e % 6];
    __syncthreads();
    // z = y - L21^T x_rows: a warp a pivot column
    for (int j = warp; j < p; j += 8) {
        double t = 0;
        for (int e = p + lane; e < n; e += 32) t += A[(size_t)j * n + e] * xsh[e];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) xsh[j] -= t;
    }
    for (int s = (p - 1) / kMfT; s >= 0; s--) {
        const int c0 = kMfT * s, w = min(kMfT, p - c0), b1 = c0 + w;
        __syncthreads();
        // the pivot rows below the panel: z_j -= sum_{e in [b1, p)} L_ej x_e, a warp a column
        for (int j = c0 + warp; j < b1; j += 8) {
            double t = 0;
            for (int e = b1 + lane; e < p; e += 32) t += A[(size_t)j * n + e] * xsh[e];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (lane == 0) xsh[j] -= t;
        }
        const double* Ti = M.dt + fr.dt0 + (size_t)s * 2 * kMfT * kMfT + kMfT * kMfT; // (L^-1, column-major)
        for (int e = tid; e < kMfT * kMfT; e += blockDim.x) Lt[e % kMfT][e / kMfT] = Ti[e];
        __syncthreads();
        // x_s = L^-T z_s: x_j = sum_{i >= j} Linv_ij z_i
        double t = 0;
        if (tid < w)
            for (int i = tid; i < w; i++) t += Lt[i][tid] * xsh[c0 + i];
        __syncthreads();
        if (tid < w) xsh[c0 + tid] = t;
    }
    __syncthreads();
    for (int e = tid; e < p; e += blockDim.x) F.rhs[6 * (size_t)idx[e / 6] + e % 6] = xsh[e];
}

} // namespace blg
