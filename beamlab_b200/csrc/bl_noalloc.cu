// bl_gpu_substep_noalloc: one explicit substep of one body over buffers the caller owns, allocating nothing.
//
// Who needs it: a caller whose GPU memory belongs to another allocator - a game engine's or a framework's pool that
// hands out every buffer, or a frame loop in which allocation is forbidden (a real-time budget, a region of CUDA
// stream capture) - cannot let the library cudaMalloc. The context API (bl_gpu_create / bl_gpu_add_body) allocates
// its device arrays; this entry point takes the body's device buffers from the caller instead and keeps its one piece
// of scratch, the per-beam force between the two kernels, in a fixed array compiled into the library.
//
// The scratch: g_noalloc_fv, BL_GPU_NOALLOC_MAX_BEAMS float4 (16 MiB), a file-scope __device__ array that every GPU
// which loads the library holds until the process exits. In host code its name stands for a host-side shadow, not a
// device address, so the kernel gets the address that cudaGetSymbolAddress returns in the calling thread's current
// CUDA context. The address belongs to the context (a caller's own cuCtxCreate context, or a primary context made
// again after cudaDeviceReset, has its own copy of the array), so it is looked up again on every call whose stream is
// not being captured and kept per context for the calls made during a capture; the first call in a context should
// come before any stream capture begins. Every call shares the array; a call writes each slot before it reads it, so
// nothing needs clearing, but two calls whose kernels overlap on the GPU race on it.
#include "../../include/beamlab_gpu.h"
#include "bl_math.cuh"

#include <cuda_runtime.h>

#include <mutex>

namespace {

static __device__ __align__(256) float4 g_noalloc_fv[BL_GPU_NOALLOC_MAX_BEAMS];

struct f3 {
    float x, y, z;
};
__device__ __forceinline__ f3 sub3(f3 a, f3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float smin_(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax_(float a, float b) { return (a < b) ? b : a; }

// SoftBody::compute_beam_forces (softbody.cpp:412-470) on bl_beam records, one beam a thread; the beam's force goes
// to the scratch (w = 1: it pushes this substep), its state is updated in place.
__global__ void k_noalloc_beams(const bl_node* __restrict__ nodes, bl_beam* __restrict__ beams, int n_beams, int deform, int brk, int ductile,
                                float4* __restrict__ fv) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n_beams) return;
    bl_beam b = beams[j];
    float4 out = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (!(b.flags & (BL_BF_BROKEN | BL_BF_SHOCK))) {
        const bl_node& na = nodes[b.a];
        const bl_node& nb = nodes[b.b];
        const f3 dis = sub3({na.p[0], na.p[1], na.p[2]}, {nb.p[0], nb.p[1], nb.p[2]});
        const float len2 = dot3(dis, dis);
        if (!(len2 < 1e-12f)) {
            const float inv_len = 1.0f / sqrtf(len2);
            const float len = len2 * inv_len;
            const float diff = len - b.L;
            const f3 dv = sub3({na.v[0], na.v[1], na.v[2]}, {nb.v[0], nb.v[1], nb.v[2]});
            float k = b.k, d = b.d;
            bool broke = false, changed = false;
            if (b.type == BL_BT_ROPE) {
                if (diff < 0) k = 0, d *= 0.1f;
            } else if (b.type == BL_BT_SUPPORT) {
                if (diff > 0) {
                    k = 0;
                    d *= 0.1f;
                    if (brk && diff > b.L * b.support_limit) broke = true;
                }
            }
            if (!broke) {
                float slen = -k * diff - d * dot3(dv, dis) * inv_len;
                if (deform && !(b.flags & BL_BF_NO_DEFORM) && k != 0) {
                    if (slen > b.max_pos && diff < 0) {
                        const float yield_len = b.max_pos / k;
                        const float def = diff + yield_len * (1.0f - b.plastic);
                        const float Lold = b.L;
                        b.L = smax_(smin_(0.1f, 0.3f * b.L0), b.L + def);
                        slen = slen - (slen - b.max_pos) * 0.5f;
                        if (b.L < Lold) b.max_pos *= Lold / b.L;
                        changed = true;
                    } else if (slen < b.max_neg && diff > 0) {
                        const float yield_len = b.max_neg / k;
                        const float def = diff + yield_len * (1.0f - b.plastic);
                        const float Lold = b.L;
                        b.L = b.L + def;
                        slen = slen - (slen - b.max_neg) * 0.5f;
                        if (Lold > 0 && b.L > Lold) b.max_neg *= b.L / Lold;
                        if (!ductile) b.strength -= def * k;
                        changed = true;
                    }
                }
                if (brk && fabsf(slen) > b.strength && !(b.flags & BL_BF_NO_BREAK)) {
                    broke = true;
                } else {
                    b.stress = slen;
                    changed = true;
                    const float sc = slen * inv_len;
                    out = make_float4(dis.x * sc, dis.y * sc, dis.z * sc, 1.0f);
                }
            }
            if (broke) b.flags |= BL_BF_BROKEN, changed = true;
            if (changed) beams[j] = b;
        }
    }
    fv[j] = out;
}

// clear_forces' gravity, the node's beams in beam order (softbody.cpp:376, 466-467), SoftBody::integrate_nodes
// (softbody.cpp:769-795)
__global__ void k_noalloc_nodes(bl_node* __restrict__ nodes, int n_nodes, const int* __restrict__ inc_ptr, const int* __restrict__ inc,
                                const float4* __restrict__ fv, float gx, float gy, float gz, float dt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    bl_node x = nodes[i];
    const float m = x.mass;
    float fx = gx * m, fy = gy * m, fz = gz * m;
    for (int q = inc_ptr[i]; q < inc_ptr[i + 1]; q++) {
        const int e = inc[q];
        const float4 b = fv[e & 0x7fffffff];
        if (b.w != 0.0f) {
            if (e < 0) fx = fx - b.x, fy = fy - b.y, fz = fz - b.z;
            else fx = fx + b.x, fy = fy + b.y, fz = fz + b.z;
        }
    }
    if (x.inv_mass > 0) {
        const float s = x.inv_mass * dt;
        float vx = x.v[0] + fx * s, vy = x.v[1] + fy * s, vz = x.v[2] + fz * s;
        const float v2 = vx * vx + vy * vy + vz * vz;
        if (v2 > 400.0f * 400.0f) {
            const float c = 400.0f / sqrtf(v2);
            vx *= c, vy *= c, vz *= c;
        } else if (!(v2 >= 0.0f)) {
            vx = vy = vz = 0.0f;
        }
        x.v[0] = vx, x.v[1] = vy, x.v[2] = vz;
        x.p[0] = x.p[0] + vx * dt, x.p[1] = x.p[1] + vy * dt, x.p[2] = x.p[2] + vz * dt;
        nodes[i] = x;
    }
}

// The scratch's address per CUDA context, for the calls made while their stream is being captured (a capture forbids
// nothing here, but a context's first lookup may load the library's module). cuCtxGetCurrent is reached through the
// runtime's driver entry point, so the library does not link libcuda itself.
typedef int (*ctx_get_current_fn)(void** ctx);
struct ScratchSlot {
    void* ctx;
    float4* fv;
};
std::mutex g_setup_mutex;
ScratchSlot g_slots[64] = {};
int g_next_slot = 0;
ctx_get_current_fn g_ctx_get_current = nullptr;

int current_context(void** ctx) {
    if (!g_ctx_get_current) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn)
            return BL_GPU_ECUDA;
        g_ctx_get_current = (ctx_get_current_fn)fn;
    }
    *ctx = nullptr;
    return (g_ctx_get_current(ctx) == 0 && *ctx) ? BL_GPU_OK : BL_GPU_ECUDA;
}

// The scratch's address in the current context: looked up afresh unless the stream is capturing, then remembered.
int scratch_address(cudaStream_t s, float4** out) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    // a runtime call first, so that the thread has a current context (the device's primary one if it had none)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool capturing = cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
    void* ctx = nullptr;
    if (current_context(&ctx) != BL_GPU_OK) return BL_GPU_ECUDA;
    int slot = -1;
    for (int i = 0; i < 64; i++)
        if (g_slots[i].ctx == ctx) slot = i;
    if (capturing && slot >= 0) {
        *out = g_slots[slot].fv;
        return BL_GPU_OK;
    }
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_fv) != cudaSuccess || !p) return BL_GPU_ECUDA;
    if (slot < 0) slot = g_next_slot, g_next_slot = (g_next_slot + 1) % 64;
    g_slots[slot] = {ctx, (float4*)p};
    *out = (float4*)p;
    return BL_GPU_OK;
}

} // namespace

extern "C" int bl_gpu_substep_noalloc(bl_node* nodes, int32_t n_nodes, bl_beam* beams, int32_t n_beams, const int32_t* inc_ptr, const int32_t* inc,
                                      const float gravity[3], float dt, int32_t allow_deform, int32_t allow_break, int32_t ductile, void* stream) {
    if (n_nodes < 0 || n_beams < 0 || !gravity || !(dt > 0) || (n_nodes > 0 && (!nodes || !inc_ptr)) || (n_beams > 0 && (!beams || !inc)))
        return BL_GPU_EINVAL;
    if (n_beams > BL_GPU_NOALLOC_MAX_BEAMS) return BL_GPU_ELIMIT;
    cudaStream_t s = (cudaStream_t)stream;
    float4* fv = nullptr;
    if (scratch_address(s, &fv) != BL_GPU_OK) return BL_GPU_ECUDA;
    if (n_nodes == 0) return BL_GPU_OK;
    // each launch's own status (cudaLaunchKernel returns it), not an earlier error left pending by other code
    if (n_beams > 0) {
        const bl_node* cn = nodes;
        void* args[] = {(void*)&cn, (void*)&beams, (void*)&n_beams, (void*)&allow_deform, (void*)&allow_break, (void*)&ductile, (void*)&fv};
        if (cudaLaunchKernel((const void*)k_noalloc_beams, dim3((n_beams + 255) / 256), dim3(256), args, 0, s) != cudaSuccess) return BL_GPU_ECUDA;
    }
    const float4* cfv = fv;
    float gx = gravity[0], gy = gravity[1], gz = gravity[2];
    void* args[] = {(void*)&nodes, (void*)&n_nodes, (void*)&inc_ptr, (void*)&inc, (void*)&cfv, (void*)&gx, (void*)&gy, (void*)&gz, (void*)&dt};
    if (cudaLaunchKernel((const void*)k_noalloc_nodes, dim3((n_nodes + 255) / 256), dim3(256), args, 0, s) != cudaSuccess) return BL_GPU_ECUDA;
    return BL_GPU_OK;
}
