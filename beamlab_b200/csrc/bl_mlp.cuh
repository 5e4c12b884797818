// The learned warm start of the FEM step's PCG solve: a per-node MLP 36 -> 64 -> 64 -> 64 -> 12 (ReLU), BF16 weights
// with FP32 accumulation, its inference in the step, the recording of training samples from the Cholesky's solves,
// and its training (forward, backward, Adam) on the GPU. No counterpart in the reference.
//
// Features of a frame node i (column k = iperm[i]), with sl(x) = sign(x) log(1 + |x| / s0), s0 = 1 mm/s:
//   0-2   sl(h F_i / m_i)             the explicit step's velocity change (F: the node's force before the solve)
//   3-5   sl(dv_i of the last solve)
//   6-8   sl(v_i)
//   9-11  the mean of features 0-2 over the node's 1-ring (the frame nodes it shares a triangle with)
//   12-14 the mean of features 3-5 over the 1-ring
//   15-32 the edges to the first six 1-ring nodes (in frame-node order), (x_j - x_i) / their mean length; zeros after
//   33-35 log(D_aa / m_i): the translational diagonal of the node's 6 x 6 diagonal block of A over its mass
// Outputs: y 0-2 -> the guess dv = isl(y) (the inverse of sl); y 3-11 -> S = I + 0.25 tanh(y) entrywise (3 x 3, row
// major): the preconditioner's translational scale (bl_fem_pcg.cuh).
// Training targets (recorded from the Cholesky's solutions): sl(dv) for y 0-2; for the diagonal of S the ratio of the
// solution to the block-Jacobi estimate u = (D^-1 rhs)_a, clamped to [0.76, 1.24] (weight 0.1 where |u_a| > 1e-9 m/s),
// zero for its off-diagonal entries (weight 0.01).
//
// Parameters, one float vector: W1 (64 x 36, row = output), b1 (64), W2 (64 x 64), b2, W3 (64 x 64), b3, W4 (12 x 64), b4.
// The forward's four layers run on the tensor cores (mma.sync m16n8k16, BF16 inputs and weights, FP32 accumulation,
// FP32 bias and ReLU; each layer's input rounded to BF16); the backward (data and weight gradients) runs in FP32 on the
// BF16-rounded activations the forward used.
#pragma once

#include <cuda_bf16.h>

#include "bl_fem_kernels.cuh"

namespace blg {

constexpr int kIn = 36, kHid = 64, kOut = 12;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kHid * kIn, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid, kOffW3 = kOffB2 + kHid;
constexpr int kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid, kOffB4 = kOffW4 + kOut * kHid, kParams = kOffB4 + kOut;
constexpr float kS0 = 1e-3f;
constexpr int kLanes = 32;   // samples a block (one warp)
constexpr int kLd = 33;      // shared-memory row stride (a feature's 32 samples, padded against bank conflicts)

struct MlpDev {
    const __nv_bfloat16* wb; // the parameters in BF16 (what the forward reads)
    float* w;                // FP32 master copy (what Adam updates)
    float* m;                // Adam moments
    float* v;
    // the step's side
    const int* adj_ptr;      // per frame node: its 1-ring (frame nodes sharing a triangle), ascending
    const int* adj;
    float* prev_dv;          // 3 / frame node: dv of the last solve
    float* feat;             // kIn / frame node: this substep's features
    // recorded samples (a ring of cap samples)
    float* sx;               // kIn / sample
    float* st;               // kOut / sample: targets
    float* sw;               // kOut / sample: weights
    int* scount;             // samples recorded so far
    int cap;
};

__device__ __forceinline__ float slog(float x) { return x < 0 ? -log1pf(-x / kS0) : log1pf(x / kS0); }
__device__ __forceinline__ float islog(float y) { return y < 0 ? -kS0 * expm1f(-y) : kS0 * expm1f(y); }

// ------------------------------------------------------------------------------------------ the network (one sample a lane)
constexpr int kKIn = 48;         // the first layer's inputs padded to whole k-steps of 16 (36 features + 12 zeros)
constexpr int kPadIn = 64 + 8;   // the staged activations' row stride in BF16 (144 B: rows fall in distinct banks)
constexpr int kOutPad = 16;      // the last layer's outputs padded to two n-tiles of 8

struct MlpTc {
    __nv_bfloat16 act[kLanes * kPadIn];   // the current layer's input
    __nv_bfloat16 w[kHid * kPadIn];       // the current layer's weights, nout x nin
};

// activations in shared memory, [feature][kLd]: lane s holds its sample in column s; the backward's deltas share
// their storage with the forward's tensor-core staging (live one after the other)
struct MlpSmem {
    float a0[kIn * kLd];
    float a1[kHid * kLd];
    float a2[kHid * kLd];
    float a3[kHid * kLd];
    float y[kOut * kLd];
    union {
        struct {
            float d0[kHid * kLd];
            float d1[kHid * kLd];
        };
        MlpTc tc;
    };
};

// ------------------------------------------------------------------------------------------ the layers on the tensor cores
// One warp runs a layer's 32 samples x nout outputs as mma.sync m16n8k16 tiles (BF16 operands, FP32 accumulation):
// A = the layer's input, 32 samples x nin, BF16, row-major in shared memory (row stride kPadIn); B = the weights,
// nout x nin row-major (the "col" operand as it is), BF16 in shared memory. The inputs are rounded to BF16 as they are
// staged (the activations the next layer reads are the BF16 values); the accumulators, bias and ReLU stay FP32.
__device__ __forceinline__ void mma_bf16(float c[4], const uint32_t a[4], const uint32_t b[2]) {
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, {%0, %1, %2, %3};"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ uint32_t lds32(const __nv_bfloat16* p) { return *reinterpret_cast<const uint32_t*>(p); }

// out[o * kLd + s] = (relu)(b_o + sum_i W[o][i] act[s][i]) for the 32 samples; the layer's weights (nout x nin from
// global, zero rows past nout) staged first. nin: a multiple of 16; nout_t: n-tiles of 8.
__device__ __forceinline__ void dense_tc(const __nv_bfloat16* __restrict__ W, const __nv_bfloat16* __restrict__ b, int nin, int nin_real, int nout,
                                         int nout_t, MlpTc& T, float* out, bool relu) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int e = lane; e < nout_t * 8 * nin; e += 32) {
        const int o = e / nin, i = e % nin;
        T.w[o * kPadIn + i] = (o < nout && i < nin_real) ? W[(size_t)o * nin_real + i] : __float2bfloat16(0.0f);
    }
    __syncwarp();
    for (int mt = 0; mt < 2; mt++) {
        for (int nt = 0; nt < nout_t; nt++) {
            float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            for (int k0 = 0; k0 < nin; k0 += 16) {
                const __nv_bfloat16* a_lo = T.act + (16 * mt + g) * kPadIn + k0 + 2 * t;
                const __nv_bfloat16* a_hi = a_lo + 8 * kPadIn;
                const uint32_t a[4] = {lds32(a_lo), lds32(a_hi), lds32(a_lo + 8), lds32(a_hi + 8)};
                const __nv_bfloat16* wp = T.w + (8 * nt + g) * kPadIn + k0 + 2 * t;
                const uint32_t bb[2] = {lds32(wp), lds32(wp + 8)};
                mma_bf16(c, a, bb);
            }
            // c0, c1: sample 16 mt + g, outputs 8 nt + 2 t, + 1; c2, c3: sample + 8
            for (int q = 0; q < 4; q++) {
                const int smp = 16 * mt + g + (q >= 2 ? 8 : 0), o = 8 * nt + 2 * t + (q & 1);
                if (o < nout) {
                    const float v = c[q] + __bfloat162float(b[o]);
                    out[o * kLd + smp] = relu ? fmaxf(v, 0.0f) : v;
                }
            }
        }
    }
    __syncwarp();
}

// the next layer's input: `in` ([feature][kLd], FP32) as BF16 rows, padded with zeros to nin_pad
__device__ __forceinline__ void stage_act(const float* in, int nin, int nin_pad, MlpTc& T) {
    const int lane = threadIdx.x & 31;
    __syncwarp();
    for (int e = lane; e < kLanes * nin_pad; e += 32) {
        const int smp = e / nin_pad, i = e % nin_pad;
        T.act[smp * kPadIn + i] = __float2bfloat16(i < nin ? in[i * kLd + smp] : 0.0f);
    }
    __syncwarp();
}

// The forward of the warp's 32 samples (S.a0 holds their features): a1..a3 and y in S, the BF16-rounded inputs of
// each layer written back into a0..a3 (what the backward's weight gradients multiply)
__device__ void mlp_forward(const MlpDev& M, MlpSmem& S, MlpTc& T) {
    const int lane = threadIdx.x & 31;
    float* acts[4] = {S.a0, S.a1, S.a2, S.a3};
    const int nins[4] = {kIn, kHid, kHid, kHid};
    for (int l = 0; l < 4; l++) {
        const int nin = nins[l], nin_pad = l == 0 ? kKIn : kHid;
        stage_act(acts[l], nin, nin_pad, T);
        for (int e = lane; e < kLanes * nin; e += 32) { // (the layer's input as the tensor cores read it)
            const int smp = e / nin, i = e % nin;
            acts[l][i * kLd + smp] = __bfloat162float(T.act[smp * kPadIn + i]);
        }
        const int offw[4] = {kOffW1, kOffW2, kOffW3, kOffW4}, offb[4] = {kOffB1, kOffB2, kOffB3, kOffB4};
        const int nout = l == 3 ? kOut : kHid;
        dense_tc(M.wb + offw[l], M.wb + offb[l], nin_pad, nin, nout, l == 3 ? kOutPad / 8 : kHid / 8, T, l == 3 ? S.y : acts[l + 1], l < 3);
    }
    __syncwarp();
}

// ------------------------------------------------------------------------------------------ the step's side
// The features of every frame node (after the assembly: diag holds A's diagonal blocks, nforce the nodes' forces)
__global__ void k_mlp_features(FemDev F, MlpDev M, const float4* __restrict__ nd, const float4* __restrict__ nforce) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.nf) return;
    float* x = M.feat + (size_t)kIn * i;
    auto explicit_dv = [&](int j, float* e) {
        const int bn = F.fnode[j];
        const float4 f = nforce[bn];
        const float m = nd[2 * bn + 1].w;
        const float s = m > 0 ? F.h / m : 0.0f;
        e[0] = slog(f.x * s), e[1] = slog(f.y * s), e[2] = slog(f.z * s);
    };
    float e[3];
    explicit_dv(i, e);
    const int bn = F.fnode[i];
    const float4 P = nd[2 * bn], Vv = nd[2 * bn + 1];
    for (int a = 0; a < 3; a++) x[a] = e[a], x[3 + a] = slog(M.prev_dv[3 * i + a]);
    x[6] = slog(Vv.x), x[7] = slog(Vv.y), x[8] = slog(Vv.z);
    float me[3] = {0, 0, 0}, mp[3] = {0, 0, 0};
    const int j0 = M.adj_ptr[i], j1 = M.adj_ptr[i + 1];
    float mean_len = 0;
    for (int q = j0; q < j1; q++) {
        const int j = M.adj[q];
        float ej[3];
        explicit_dv(j, ej);
        for (int a = 0; a < 3; a++) me[a] += ej[a], mp[a] += slog(M.prev_dv[3 * j + a]);
        const float4 Pj = nd[2 * F.fnode[j]];
        mean_len += sqrtf((Pj.x - P.x) * (Pj.x - P.x) + (Pj.y - P.y) * (Pj.y - P.y) + (Pj.z - P.z) * (Pj.z - P.z));
    }
    const int nn = j1 - j0;
    const float inv = nn > 0 ? 1.0f / (float)nn : 0.0f;
    for (int a = 0; a < 3; a++) x[9 + a] = me[a] * inv, x[12 + a] = mp[a] * inv;
    mean_len = nn > 0 ? mean_len * inv : 1.0f;
    const float il = mean_len > 0 ? 1.0f / mean_len : 0.0f;
    for (int q = 0; q < 6; q++) {
        if (q < nn) {
            const float4 Pj = nd[2 * F.fnode[M.adj[j0 + q]]];
            x[15 + 3 * q] = (Pj.x - P.x) * il, x[16 + 3 * q] = (Pj.y - P.y) * il, x[17 + 3 * q] = (Pj.z - P.z) * il;
        } else {
            x[15 + 3 * q] = x[16 + 3 * q] = x[17 + 3 * q] = 0.0f;
        }
    }
    const int k = F.iperm[i];
    const double* D = F.diag + 36 * (size_t)k;
    const float m = Vv.w;
    for (int a = 0; a < 3; a++) x[33 + a] = (m > 0 && !(P.w <= 0)) ? logf(fmaxf((float)(D[a * 7] / (double)m), 1e-6f)) : 0.0f;
}

// The network on every frame node's features: the PCG's guess and scale
__global__ void __launch_bounds__(kLanes) k_mlp_infer(FemDev F, MlpDev M, float* __restrict__ guess, float* __restrict__ gscale) {
    __shared__ __align__(16) MlpSmem S;
    MlpTc& T = S.tc;
    const int s = threadIdx.x;
    const int i = blockIdx.x * kLanes + s;
    const bool on = i < F.nf;
    for (int f = 0; f < kIn; f++) S.a0[f * kLd + s] = on ? M.feat[(size_t)kIn * i + f] : 0.0f;
    mlp_forward(M, S, T);
    if (!on) return;
    for (int a = 0; a < 3; a++) guess[3 * i + a] = islog(S.y[a * kLd + s]);
    for (int q = 0; q < 9; q++) gscale[9 * i + q] = ((q % 4) == 0 ? 1.0f : 0.0f) + 0.25f * tanhf(S.y[(3 + q) * kLd + s]);
}

// Recording, before the solve: each frame node's features and the block-Jacobi estimate u = (D^-1 rhs)_a (kept in
// the targets' slots 3-5 until k_mlp_record_post)
__global__ void k_mlp_record_pre(FemDev F, MlpDev M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.nf) return;
    const size_t slot = (size_t)((*M.scount + i) % M.cap);
    for (int f = 0; f < kIn; f++) M.sx[kIn * slot + f] = M.feat[(size_t)kIn * i + f];
    const int k = F.iperm[i];
    double L[36], di[6], u[6];
    for (int x = 0; x < 36; x++) L[x] = F.diag[36 * (size_t)k + x];
    for (int j = 0; j < 6; j++) u[j] = F.rhs[6 * (size_t)k + j];
    if (chol6_dev(L, di)) {
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
    } else {
        for (int j = 0; j < 6; j++) u[j] = 0.0;
    }
    for (int a = 0; a < 3; a++) M.st[kOut * slot + 3 + a] = (float)u[a];
}

// Recording, after the solve: the targets from the solution dv (in rhs) and u
__global__ void k_mlp_record_post(FemDev F, MlpDev M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.nf) return;
    const size_t slot = (size_t)((*M.scount + i) % M.cap);
    const int k = F.iperm[i];
    const bool fixed = F.fixed[k] != 0;
    float* t = M.st + kOut * slot;
    float* w = M.sw + kOut * slot;
    float u[3];
    for (int a = 0; a < 3; a++) u[a] = t[3 + a];
    for (int a = 0; a < 3; a++) {
        const float dv = (float)F.rhs[6 * (size_t)k + a];
        t[a] = slog(dv), w[a] = fixed ? 0.0f : 1.0f;
    }
    for (int q = 0; q < 9; q++) {
        const int r = q / 3, c = q % 3;
        if (r == c) {
            const float dv = (float)F.rhs[6 * (size_t)k + r];
            const bool ok = !fixed && fabsf(u[r]) > 1e-9f;
            const float ratio = ok ? fminf(fmaxf(dv / u[r], 0.76f), 1.24f) : 1.0f;
            t[3 + q] = atanhf((ratio - 1.0f) / 0.25f);
            w[3 + q] = ok ? 0.1f : 0.0f;
        } else {
            t[3 + q] = 0.0f, w[3 + q] = fixed ? 0.0f : 0.01f;
        }
    }
}

__global__ void k_mlp_record_done(MlpDev M, int nf) { *M.scount += nf; }

// After the solve: each frame node's dv for the next substep's features
__global__ void k_mlp_store_dv(FemDev F, MlpDev M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= F.nf) return;
    const int k = F.iperm[i];
    const bool fixed = F.fixed[k] != 0;
    for (int a = 0; a < 3; a++) M.prev_dv[3 * i + a] = fixed ? 0.0f : (float)F.rhs[6 * (size_t)k + a];
}

// ------------------------------------------------------------------------------------------ training
// The loss L = sum_s sum_o w_so (y_so - t_so)^2 / (2 n) over a batch of n samples (idx: the samples, null: x, t, w in
// order) and its gradient: a block of 32 samples does the forward, the backward, and its share of the gradient summed
// over its samples in order (gpart: kParams a block; lpart: the block's loss). Deterministic.
__global__ void __launch_bounds__(kLanes) k_mlp_grad(MlpDev M, const float* __restrict__ x, const float* __restrict__ t, const float* __restrict__ w,
                                                     const int* __restrict__ idx, int n, float* __restrict__ gpart, float* __restrict__ lpart) {
    __shared__ __align__(16) MlpSmem S;
    MlpTc& T = S.tc;
    const int s = threadIdx.x;
    const int q = blockIdx.x * kLanes + s;
    const bool on = q < n;
    const size_t smp = on ? (size_t)(idx ? idx[q] : q) : 0;
    for (int f = 0; f < kIn; f++) S.a0[f * kLd + s] = on ? x[kIn * smp + f] : 0.0f;
    mlp_forward(M, S, T);
    // d4 = w (y - t) / n into y's place; the sample's loss
    float loss = 0.0f;
    const float inv_n = 1.0f / (float)n;
    for (int o = 0; o < kOut; o++) {
        const float wo = on ? w[kOut * smp + o] : 0.0f;
        const float e = on ? S.y[o * kLd + s] - t[kOut * smp + o] : 0.0f;
        loss += 0.5f * wo * e * e;
        S.y[o * kLd + s] = wo * e * inv_n;
    }
    // d3 = W4^T d4 (.) [a3 > 0] -> d0;  d2 = W3^T d3 (.) [a2 > 0] -> d1;  d1 = W2^T d2 (.) [a1 > 0] -> d0 (after W2's gradient)
    auto back = [&](const __nv_bfloat16* W, int nin, int nout, const float* dout, const float* act, float* din) {
        for (int i2 = 0; i2 < nin; i2++) {
            float acc = 0.0f;
            for (int o = 0; o < nout; o++) acc += __bfloat162float(W[(size_t)o * nin + i2]) * dout[o * kLd + s];
            din[i2 * kLd + s] = act[i2 * kLd + s] > 0.0f ? acc : 0.0f;
        }
    };
    // the block's gradient of one layer: dW[o][i] = sum_s d[o][s] a[i][s], db[o] = sum_s d[o][s]
    auto layer_grad = [&](float* g, int off_w, int off_b, int nin, int nout, const float* d, const float* a) {
        __syncthreads();
        for (int e = s; e < nout * nin; e += kLanes) {
            const int o = e / nin, i2 = e % nin;
            float acc = 0.0f;
            for (int r = 0; r < kLanes; r++) acc += d[o * kLd + r] * a[i2 * kLd + r];
            g[off_w + e] = acc;
        }
        for (int o = s; o < nout; o += kLanes) {
            float acc = 0.0f;
            for (int r = 0; r < kLanes; r++) acc += d[o * kLd + r];
            g[off_b + o] = acc;
        }
        __syncthreads();
    };
    float* g = gpart + (size_t)blockIdx.x * kParams;
    layer_grad(g, kOffW4, kOffB4, kHid, kOut, S.y, S.a3);
    back(M.wb + kOffW4, kHid, kOut, S.y, S.a3, S.d0);
    layer_grad(g, kOffW3, kOffB3, kHid, kHid, S.d0, S.a2);
    back(M.wb + kOffW3, kHid, kHid, S.d0, S.a2, S.d1);
    layer_grad(g, kOffW2, kOffB2, kHid, kHid, S.d1, S.a1);
    back(M.wb + kOffW2, kHid, kHid, S.d1, S.a1, S.d0);
    layer_grad(g, kOffW1, kOffB1, kIn, kHid, S.d0, S.a0);
    // the block's loss, in lane order
    S.d1[s] = loss;
    __syncthreads();
    if (s == 0) {
        float l = 0.0f;
        for (int r = 0; r < kLanes; r++) l += S.d1[r];
        lpart[blockIdx.x] = l;
    }
}

// The blocks' gradients summed in block order (into gsum), and, with lr > 0, one Adam step (t: its count from 1) of
// the FP32 parameters and their BF16 copy
__global__ void k_mlp_adam(MlpDev M, const float* __restrict__ gpart, int nblocks, float* __restrict__ gsum, float lr, float b1, float b2, float eps,
                           int t) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float g = 0.0f;
    for (int b = 0; b < nblocks; b++) g += gpart[(size_t)b * kParams + p];
    if (gsum) gsum[p] = g;
    if (!(lr > 0)) return;
    const float m = b1 * M.m[p] + (1.0f - b1) * g;
    const float v = b2 * M.v[p] + (1.0f - b2) * g * g;
    M.m[p] = m, M.v[p] = v;
    const float mh = m / (1.0f - powf(b1, (float)t)), vh = v / (1.0f - powf(b2, (float)t));
    const float wn = M.w[p] - lr * mh / (sqrtf(vh) + eps);
    M.w[p] = wn;
    ((__nv_bfloat16*)M.wb)[p] = __float2bfloat16(wn);
}

// acc += the blocks' losses, in block order
__global__ void k_loss_acc(const float* __restrict__ lpart, int nblocks, double* acc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0;
        for (int b = 0; b < nblocks; b++) s += lpart[b];
        *acc += s;
    }
}

__global__ void k_mlp_sync_bf16(MlpDev M) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) ((__nv_bfloat16*)M.wb)[p] = __float2bfloat16(M.w[p]);
}

// The network's outputs for n samples (tests)
__global__ void __launch_bounds__(kLanes) k_mlp_forward_batch(MlpDev M, const float* __restrict__ x, int n, float* __restrict__ y) {
    __shared__ __align__(16) MlpSmem S;
    MlpTc& T = S.tc;
    const int s = threadIdx.x;
    const int q = blockIdx.x * kLanes + s;
    const bool on = q < n;
    for (int f = 0; f < kIn; f++) S.a0[f * kLd + s] = on ? x[(size_t)kIn * q + f] : 0.0f;
    mlp_forward(M, S, T);
    if (on)
        for (int o = 0; o < kOut; o++) y[(size_t)kOut * q + o] = S.y[o * kLd + s];
}

} // namespace blg
