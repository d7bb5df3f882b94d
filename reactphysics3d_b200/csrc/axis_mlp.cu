// Training and inference kernels of the learned separating-axis MLP.
//
// Training is plain fp32 CUDA-core arithmetic on bf16-rounded weights
// (fp32 master copy, Adam state in fp32):
//   mlp_forward_backward: one sample per thread; forward pass, softmax
//       cross-entropy, and the backward pass down to the hidden layers;
//       writes the activations and their gradients to scratch rows
//   mlp_weight_grads:     one parameter per thread; reduces activation x
//       gradient products over the batch in a fixed order (deterministic)
//   mlp_adam:             bias-corrected Adam on the fp32 masters
//   mlp_pack:             bf16 mma.m16n8k16 B fragments for inference
// Inference (mlp_predict and the fused SAT kernels) runs the packed weights
// on the bf16 tensor cores (axis_mlp.cuh).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <mutex>

#include "axis_mlp.cuh"
#include "mlp_launch.h"

namespace rp3dg {

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// One sample per thread.  Scratch rows (per sample): h1[64], h2[64], dh1[64],
// dh2[64], dz[16].  loss_sum accumulates the batch's summed cross-entropy.
__global__ void __launch_bounds__(128) mlp_forward_backward(const float* __restrict__ params, const float* __restrict__ x,
                                                            const uint8_t* __restrict__ y, uint32_t n,
                                                            float* __restrict__ scratch, float* loss_sum) {
    __shared__ float w1[MLP_IN * MLP_H], w2[MLP_H * MLP_H], w3[MLP_H * MLP_OUT];
    __shared__ float b1[MLP_H], b2[MLP_H], b3[MLP_OUT];
    __shared__ float red[128];
    for (int k = threadIdx.x; k < MLP_IN * MLP_H; k += blockDim.x) w1[k] = bf16r(params[MLP_OFF_W1 + k]);
    for (int k = threadIdx.x; k < MLP_H * MLP_H; k += blockDim.x) w2[k] = bf16r(params[MLP_OFF_W2 + k]);
    for (int k = threadIdx.x; k < MLP_H * MLP_OUT; k += blockDim.x) w3[k] = bf16r(params[MLP_OFF_W3 + k]);
    for (int k = threadIdx.x; k < MLP_H; k += blockDim.x) { b1[k] = params[MLP_OFF_B1 + k]; b2[k] = params[MLP_OFF_B2 + k]; }
    for (int k = threadIdx.x; k < MLP_OUT; k += blockDim.x) b3[k] = params[MLP_OFF_B3 + k];
    __syncthreads();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float sample_loss = 0.0f;
    if (i < n) {
        float* row = scratch + size_t(i) * MLP_SCRATCH_ROW;
        float* h1 = row;
        float* h2 = row + 64;
        float* dh1 = row + 128;
        float* dh2 = row + 192;
        float* dz = row + 256;
        float xi[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; k++) xi[k] = x[size_t(i) * MLP_IN + k];
        for (int j = 0; j < MLP_H; j++) {
            float s = b1[j];
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) s += xi[k] * w1[k * MLP_H + j];
            h1[j] = s > 0.0f ? s : 0.0f;
        }
        for (int j = 0; j < MLP_H; j++) {
            float s = b2[j];
            for (int k = 0; k < MLP_H; k++) s += h1[k] * w2[k * MLP_H + j];
            h2[j] = s > 0.0f ? s : 0.0f;
        }
        float z[MLP_OUT];
        float zmax = -FLT_MAX;
#pragma unroll
        for (int j = 0; j < MLP_OUT; j++) {
            float s = b3[j];
            for (int k = 0; k < MLP_H; k++) s += h2[k] * w3[k * MLP_OUT + j];
            z[j] = s;
            zmax = fmaxf(zmax, s);
        }
        float se = 0.0f;
#pragma unroll
        for (int j = 0; j < MLP_OUT; j++) { z[j] = expf(z[j] - zmax); se += z[j]; }
        const uint32_t yi = y[i] < MLP_OUT ? y[i] : MLP_NO_PROPOSAL;
        const float inv_n = 1.0f / float(n);
#pragma unroll
        for (int j = 0; j < MLP_OUT; j++) {
            const float p = z[j] / se;
            if (uint32_t(j) == yi) sample_loss = -logf(fmaxf(p, 1e-30f));
            dz[j] = (p - (uint32_t(j) == yi ? 1.0f : 0.0f)) * inv_n;
        }
        for (int k = 0; k < MLP_H; k++) {
            float s = 0.0f;
#pragma unroll
            for (int j = 0; j < MLP_OUT; j++) s += dz[j] * w3[k * MLP_OUT + j];
            dh2[k] = h2[k] > 0.0f ? s : 0.0f;
        }
        for (int k = 0; k < MLP_H; k++) {
            float s = 0.0f;
            for (int j = 0; j < MLP_H; j++) s += dh2[j] * w2[k * MLP_H + j];
            dh1[k] = h1[k] > 0.0f ? s : 0.0f;
        }
    }
    red[threadIdx.x] = sample_loss;
    __syncthreads();
    for (int s = 64; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0 && loss_sum) atomicAdd(loss_sum, red[0]);
}

// One parameter per thread: gradient = sum over samples of (input activation
// x output gradient), summed in sample order.
__global__ void __launch_bounds__(128) mlp_weight_grads(const float* __restrict__ x, const float* __restrict__ scratch,
                                                        uint32_t n, float* __restrict__ grads) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= uint32_t(MLP_NPARAMS)) return;
    float s = 0.0f;
    if (p < uint32_t(MLP_OFF_B1)) {  // w1[k][j] = sum x[k] * dh1[j]
        const uint32_t k = p / MLP_H, j = p % MLP_H;
        for (uint32_t i = 0; i < n; i++) s += x[size_t(i) * MLP_IN + k] * scratch[size_t(i) * MLP_SCRATCH_ROW + 128 + j];
    } else if (p < uint32_t(MLP_OFF_W2)) {
        const uint32_t j = p - MLP_OFF_B1;
        for (uint32_t i = 0; i < n; i++) s += scratch[size_t(i) * MLP_SCRATCH_ROW + 128 + j];
    } else if (p < uint32_t(MLP_OFF_B2)) {  // w2[k][j] = sum h1[k] * dh2[j]
        const uint32_t q = p - MLP_OFF_W2, k = q / MLP_H, j = q % MLP_H;
        for (uint32_t i = 0; i < n; i++) s += scratch[size_t(i) * MLP_SCRATCH_ROW + k] * scratch[size_t(i) * MLP_SCRATCH_ROW + 192 + j];
    } else if (p < uint32_t(MLP_OFF_W3)) {
        const uint32_t j = p - MLP_OFF_B2;
        for (uint32_t i = 0; i < n; i++) s += scratch[size_t(i) * MLP_SCRATCH_ROW + 192 + j];
    } else if (p < uint32_t(MLP_OFF_B3)) {  // w3[k][j] = sum h2[k] * dz[j]
        const uint32_t q = p - MLP_OFF_W3, k = q / MLP_OUT, j = q % MLP_OUT;
        for (uint32_t i = 0; i < n; i++) s += scratch[size_t(i) * MLP_SCRATCH_ROW + 64 + k] * scratch[size_t(i) * MLP_SCRATCH_ROW + 256 + j];
    } else {
        const uint32_t j = p - MLP_OFF_B3;
        for (uint32_t i = 0; i < n; i++) s += scratch[size_t(i) * MLP_SCRATCH_ROW + 256 + j];
    }
    grads[p] = s;
}

__global__ void mlp_adam(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ m,
                         float* __restrict__ v, float lr, float beta1, float beta2, float eps, float bc1, float bc2) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= uint32_t(MLP_NPARAMS)) return;
    const float g = grads[p];
    const float mi = beta1 * m[p] + (1.0f - beta1) * g;
    const float vi = beta2 * v[p] + (1.0f - beta2) * g * g;
    m[p] = mi;
    v[p] = vi;
    params[p] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// bf16 B fragments of the three layers (layout in axis_mlp.cuh).
__global__ void mlp_pack(const float* __restrict__ params, MlpPacked* __restrict__ out) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    auto frag = [&](int off, int K, int N, int ks, int nt, int lane) {
        const int g = lane >> 2, t = lane & 3, col = 8 * nt + g;
        auto w = [&](int k) { return k < K ? params[off + k * N + col] : 0.0f; };
        const int k0 = 16 * ks + 2 * t;
        uint2 r;
        r.x = pack_bf16x2(w(k0), w(k0 + 1));
        r.y = pack_bf16x2(w(k0 + 8), w(k0 + 9));
        return r;
    };
    if (e < uint32_t(MLP_FRAG_L1)) {
        const int lane = e & 31, blk = e >> 5, nt = blk % (MLP_H / 8), ks = blk / (MLP_H / 8);
        out->l1[e] = frag(MLP_OFF_W1, MLP_IN, MLP_H, ks, nt, lane);
    } else if (e < uint32_t(MLP_FRAG_L1 + MLP_FRAG_L2)) {
        const uint32_t q = e - MLP_FRAG_L1;
        const int lane = q & 31, blk = q >> 5, nt = blk % (MLP_H / 8), ks = blk / (MLP_H / 8);
        out->l2[q] = frag(MLP_OFF_W2, MLP_H, MLP_H, ks, nt, lane);
    } else if (e < uint32_t(MLP_FRAG_L1 + MLP_FRAG_L2 + MLP_FRAG_L3)) {
        const uint32_t q = e - MLP_FRAG_L1 - MLP_FRAG_L2;
        const int lane = q & 31, blk = q >> 5, nt = blk % (MLP_OUT / 8), ks = blk / (MLP_OUT / 8);
        out->l3[q] = frag(MLP_OFF_W3, MLP_H, MLP_OUT, ks, nt, lane);
    }
    if (e < uint32_t(MLP_H)) { out->b1[e] = params[MLP_OFF_B1 + e]; out->b2[e] = params[MLP_OFF_B2 + e]; }
    if (e < uint32_t(MLP_OUT)) out->b3[e] = params[MLP_OFF_B3 + e];
}

// Tensor-core inference over feature rows: one warp per 32 rows.
__global__ void __launch_bounds__(128) mlp_predict(const MlpPacked* __restrict__ w, const float* __restrict__ x,
                                                   uint32_t n, uint8_t* __restrict__ cls) {
    __shared__ float tile[4][32][MLP_KPAD];
    __shared__ uint32_t out[4][32];
    __shared__ MlpPacked s_w;
    {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(w);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&s_w);
        for (uint32_t k = threadIdx.x; k < sizeof(MlpPacked) / 4; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t nwarps = gridDim.x * 4;
    for (uint32_t t0 = (blockIdx.x * 4 + warp) * 32u; t0 < n; t0 += nwarps * 32u) {
        const uint32_t i = t0 + lane;
#pragma unroll
        for (int k = 0; k < MLP_KPAD; k++) tile[warp][lane][k] = (i < n && k < MLP_IN) ? x[size_t(i) * MLP_IN + k] : 0.0f;
        __syncwarp();
        const uint32_t c = mlp_infer_tile(tile[warp], s_w, lane, out[warp]);
        if (i < n) cls[i] = uint8_t(c);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// features and labels of pair batches
// ---------------------------------------------------------------------------
RD bool shape_poly(const rp3dg_shape* shapes, int32_t idx, const BoxTables* bt, const uint32_t* mesh_words,
                   BoxPoly& b, MeshPoly& m) {
    const float4 prm = reinterpret_cast<const float4*>(shapes + idx)[0];
    const int4 kk = reinterpret_cast<const int4*>(shapes + idx)[1];
    if (kk.x == RP3DG_SHAPE_BOX) {
        b.he = V(prm.x, prm.y, prm.z);
        b.t = bt;
        return true;
    }
    m.h = reinterpret_cast<const MeshHdr*>(mesh_words) + kk.y;
    m.w = mesh_words;
    return false;
}

__global__ void axis_features_kernel(const MlpPairArgs a, float* __restrict__ feat) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    float f[MLP_IN];
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) {
        for (int k = 0; k < MLP_IN; k++) feat[size_t(i) * MLP_IN + k] = 0.0f;
        return;
    }
    const float4 p1 = a.pos1[i], q1 = a.rot1[i], p2 = a.pos2[i], q2 = a.rot2[i];
    const xform t1 = X(V(p1.x, p1.y, p1.z), Q(q1.x, q1.y, q1.z, q1.w));
    const xform t2 = X(V(p2.x, p2.y, p2.z), Q(q2.x, q2.y, q2.z, q2.w));
    BoxPoly b1, b2;
    MeshPoly m1, m2;
    const bool isb1 = shape_poly(a.shapes, i1, a.box, a.mesh_words, b1, m1);
    const bool isb2 = shape_poly(a.shapes, i2, a.box, a.mesh_words, b2, m2);
    if (isb1 && isb2) axis_features(t1, t2, b1, b2, false, f);
    else if (!isb1 && isb2) axis_features(t1, t2, m1, b2, true, f);
    else if (isb1 && !isb2) axis_features(t1, t2, b1, m2, false, f);
    else axis_features(t1, t2, m1, m2, true, f);
    for (int k = 0; k < MLP_IN; k++) feat[size_t(i) * MLP_IN + k] = f[k];
}

__global__ void axis_labels_kernel(const MlpPairArgs a, const uint8_t* __restrict__ colliding,
                                   const rp3dg_lastframe* __restrict__ cache, uint8_t* __restrict__ labels) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const int32_t i1 = a.shape1[i], i2 = a.shape2[i];
    if (uint32_t(i1) >= a.nb_shapes || uint32_t(i2) >= a.nb_shapes) { labels[i] = MLP_NO_PROPOSAL; return; }
    const int k1 = reinterpret_cast<const int4*>(a.shapes + i1)[1].x;
    const int k2 = reinterpret_cast<const int4*>(a.shapes + i2)[1].x;
    const uint4 c = reinterpret_cast<const uint4*>(cache)[i];
    LastFrame lf;
    lf.flags = c.w & 0xffu;
    lf.sat_face = (c.w >> 8) & 0xffu;
    lf.sat_e1 = (c.w >> 16) & 0xffu;
    lf.sat_e2 = (c.w >> 24) & 0xffu;
    labels[i] = uint8_t(axis_label(colliding[i] != 0, lf, k1 == RP3DG_SHAPE_BOX, k2 == RP3DG_SHAPE_BOX, a.box));
}

// Box topology for this translation unit (uploaded with the narrow-phase copy).
__constant__ BoxTables c_mlp_box_tables;

void upload_mlp_box_tables(const BoxTables& t, cudaStream_t s) {
    cudaMemcpyToSymbolAsync(c_mlp_box_tables, &t, sizeof(BoxTables), 0, cudaMemcpyHostToDevice, s);
}

cudaError_t launch_axis_features(const MlpPairArgs& a, float* feat, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    MlpPairArgs b = a;
    void* box = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&box, c_mlp_box_tables);
    if (e != cudaSuccess) return e;
    b.box = static_cast<const BoxTables*>(box);
    axis_features_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(b, feat);
    return cudaGetLastError();
}

cudaError_t launch_axis_labels(const MlpPairArgs& a, const uint8_t* colliding, const rp3dg_lastframe* cache,
                               uint8_t* labels, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    MlpPairArgs b = a;
    void* box = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&box, c_mlp_box_tables);
    if (e != cudaSuccess) return e;
    b.box = static_cast<const BoxTables*>(box);
    axis_labels_kernel<<<(a.n + 127) / 128, 128, 0, s>>>(b, colliding, cache, labels);
    return cudaGetLastError();
}

cudaError_t launch_mlp_grads(const float* params, const float* x, const uint8_t* y, uint32_t n, float* scratch,
                             float* grads, float* loss_sum, cudaStream_t s) {
    if (n == 0) return cudaErrorInvalidValue;
    mlp_forward_backward<<<(n + 127) / 128, 128, 0, s>>>(params, x, y, n, scratch, loss_sum);
    mlp_weight_grads<<<(MLP_NPARAMS + 127) / 128, 128, 0, s>>>(x, scratch, n, grads);
    return cudaGetLastError();
}

cudaError_t launch_mlp_adam(float* params, const float* grads, float* m, float* v, float lr, int step, cudaStream_t s) {
    const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.0f - powf(beta1, float(step)), bc2 = 1.0f - powf(beta2, float(step));
    mlp_adam<<<(MLP_NPARAMS + 127) / 128, 128, 0, s>>>(params, grads, m, v, lr, beta1, beta2, eps, bc1, bc2);
    return cudaGetLastError();
}

cudaError_t launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t s) {
    const int total = MLP_FRAG_L1 + MLP_FRAG_L2 + MLP_FRAG_L3;
    mlp_pack<<<(total + 127) / 128, 128, 0, s>>>(params, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Allocation-free gradients (rp3dg_axis_mlp_grads_noalloc).
//
// Some callers cannot allocate device memory while they run: an engine whose
// host application hands out a fixed GPU memory budget at start-up and
// forbids later cudaMalloc calls (allocations can stall every stream of the
// device and can fail once the budget is in use).  rp3dg_axis_mlp_grads grows
// its training scratch with cudaMalloc whenever a larger batch comes in; this
// variant uses a fixed array in the library's device image instead.  Every
// GPU that loads the library holds the array (4.4 MB) until the process exits.
// All calls share it and it keeps the previous call's contents: the loss word
// is cleared on every call, the rows are fully rewritten for the samples in
// use, and calls that overlap on the GPU (two streams, two threads) race.
// ---------------------------------------------------------------------------
static __device__ __align__(256) float g_mlp_noalloc_scratch[MLP_NOALLOC_MAX_SAMPLES * MLP_SCRATCH_ROW + 64];

namespace {
constexpr int NOALLOC_MAX_DEVICES = 64;
float* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_noalloc_mutex;
}  // namespace

// Device address of the scratch array on the current device, looked up once
// per device (the host-side name of the array is not a device address).  The
// address belongs to the device's current context: a process that resets the
// device (cudaDeviceReset) while the library is loaded gets a new module
// image, so the cached address is dropped whenever a call fails and the next
// call looks it up again; callers that reset a device must not have a call of
// this entry point in flight on it.
static void noalloc_forget() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    g_noalloc_ptr[dev] = nullptr;
}

static cudaError_t noalloc_scratch(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_mlp_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

cudaError_t launch_mlp_grads_noalloc(const float* params, const float* x, const uint8_t* y, uint32_t n, float* grads,
                                     float* loss_host, cudaStream_t s) {
    if (n == 0 || n > MLP_NOALLOC_MAX_SAMPLES) return cudaErrorInvalidValue;
    float* scratch = nullptr;
    cudaError_t e = noalloc_scratch(&scratch);
    if (e != cudaSuccess) return e;
    float* loss_word = scratch + size_t(MLP_NOALLOC_MAX_SAMPLES) * MLP_SCRATCH_ROW;
    e = cudaMemsetAsync(loss_word, 0, sizeof(float), s);
    if (e != cudaSuccess) { noalloc_forget(); return e; }
    mlp_forward_backward<<<(n + 127) / 128, 128, 0, s>>>(params, x, y, n, scratch, loss_word);
    mlp_weight_grads<<<(MLP_NPARAMS + 127) / 128, 128, 0, s>>>(x, scratch, n, grads);
    e = cudaGetLastError();
    if (e != cudaSuccess) { noalloc_forget(); return e; }
    if (!loss_host) return e;
    float sum = 0.0f;
    e = cudaMemcpyAsync(&sum, loss_word, sizeof(float), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) *loss_host = sum / float(n);
    else noalloc_forget();
    return e;
}

cudaError_t launch_mlp_predict(const MlpPacked* w, const float* x, uint32_t n, uint8_t* cls, int num_sms, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const uint32_t blocks_needed = (n + 127) / 128;
    const uint32_t cap = uint32_t(num_sms) * 8u;
    mlp_predict<<<blocks_needed < cap ? blocks_needed : cap, 128, 0, s>>>(w, x, n, cls);
    return cudaGetLastError();
}

}  // namespace rp3dg
