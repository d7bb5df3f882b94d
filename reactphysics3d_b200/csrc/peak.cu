// FP32 throughput microkernel: the denominator of the narrow phase's FP32
// roofline, measured on the device the library runs on (no clock or power
// setting is touched; the GPU runs at whatever clock it has).
//
// Every thread runs CHAINS independent dependency chains; a step of a chain
// is one multiply and one add (or one fused multiply-add) with explicit
// round-to-nearest intrinsics, so the compiler can neither contract nor drop
// them.  The narrow-phase kernels are compiled without FMA contraction (their
// results must equal the reference's, which has none), so the multiply + add
// rate is the peak their arithmetic can reach; the FMA rate (two operations
// per instruction) is measured beside it for context.
#include <cuda_runtime.h>

#include "../../include/rp3dg.h"

namespace {

constexpr int PEAK_BLOCK = 256;
constexpr int CHAINS = 8;

template <bool FMA>
__global__ void __launch_bounds__(PEAK_BLOCK) fp32_peak_kernel(int iters, float a, float b, float* sink) {
    float x[CHAINS];
#pragma unroll
    for (int k = 0; k < CHAINS; k++) x[k] = float(threadIdx.x + k);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < CHAINS; k++) {
            if (FMA) x[k] = __fmaf_rn(x[k], a, b);
            else x[k] = __fadd_rn(__fmul_rn(x[k], a), b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < CHAINS; k++) s = __fadd_rn(s, x[k]);
    // a store the compiler cannot prove dead (the value never equals -1 for
    // the inputs the host passes), so every chain must be computed
    if (s == -1.0f) sink[blockIdx.x * PEAK_BLOCK + threadIdx.x] = s;
}

}  // namespace

extern "C" int rp3dg_measure_fp32_peak(int device, int fused, double* ops_per_second) {
    if (!ops_per_second) return RP3DG_EINVAL;
    *ops_per_second = 0.0;
    int nsm = 0;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return RP3DG_ECUDA;
    // 8 resident CTAs of 256 threads per SM: 64 warps, the SM's limit
    const int blocks = nsm * 8;
    const int iters = 8192;
    float* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    e = cudaMalloc(&sink, size_t(blocks) * PEAK_BLOCK * sizeof(float));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    double best = 0.0;
    for (int rep = 0; rep < 6 && e == cudaSuccess; rep++) {
        e = cudaEventRecord(t0, s);
        if (fused) fp32_peak_kernel<true><<<blocks, PEAK_BLOCK, 0, s>>>(iters, 0.999f, 0.001f, sink);
        else fp32_peak_kernel<false><<<blocks, PEAK_BLOCK, 0, s>>>(iters, 0.999f, 0.001f, sink);
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventRecord(t1, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(t1);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
        // the first launch is a warm-up
        if (e == cudaSuccess && rep > 0 && ms > 0.0f) {
            const double ops = double(blocks) * PEAK_BLOCK * double(iters) * CHAINS * 2.0;
            const double r = ops / (double(ms) * 1e-3);
            if (r > best) best = r;
        }
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (s) cudaStreamDestroy(s);
    cudaFree(sink);
    if (e != cudaSuccess) return RP3DG_ECUDA;
    *ops_per_second = best;
    return 0;
}
