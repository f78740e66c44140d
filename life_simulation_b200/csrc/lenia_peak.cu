// life_simulation_b200/csrc/lenia_peak.cu -- the FP32 fused multiply-add
// peak of the device as a measured number (the denominator of the direct
// path's FLOP/s roofline): every thread runs 8 independent FMA chains for a
// fixed number of iterations, grid = 8 CTAs of 256 threads per SM, timed by
// CUDA events; scalar FFMA and packed FFMA2 (two FMAs per instruction) are
// timed separately. No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/lenia_b200.h"
#include "abi_guard.h"

namespace lenia {
namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

// Written only if a chain's result is negative (never, for these inputs), so
// the work cannot be removed.
__device__ float g_peak_sink;

// a_c = a_c * b + c per chain.
__global__ void __launch_bounds__(256) fma_peak_kernel(float b, float c) {
    float a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = float(threadIdx.x + k) * 1e-3f;
#pragma unroll 4
    for (int i = 0; i < kIters; ++i)
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = fmaf(a[k], b, c);
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k];
    if (s < 0.0f) g_peak_sink = s;
}

__global__ void __launch_bounds__(256) fma2_peak_kernel(float b, float c) {
    float2 a[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) a[k] = make_float2(float(threadIdx.x + k) * 1e-3f, float(k) * 1e-3f);
    const float2 bb = make_float2(b, b), cc = make_float2(c, c);
#pragma unroll 4
    for (int i = 0; i < kIters; ++i)
#pragma unroll
        for (int k = 0; k < kChains; ++k) a[k] = __ffma2_rn(a[k], bb, cc);
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += a[k].x + a[k].y;
    if (s < 0.0f) g_peak_sink = s;
}

}  // namespace
}  // namespace lenia

// Best of `reps` timed launches of each kernel after one warm-up; FLOP = 2 per
// FMA. out_ffma / out_ffma2 in TFLOP/s.
extern "C" int lenia_fp32_peak(int reps, double* out_ffma, double* out_ffma2, void* stream) {
    if (!out_ffma || !out_ffma2 || reps < 1) return LENIA_ERR_INVALID_ARG;
    return lenia::abi_guard(nullptr, [&]() -> int {
        using namespace lenia;
        int dev = 0, sms = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            return LENIA_ERR_NO_DEVICE;
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int blocks = 8 * sms;
        cudaEvent_t e0, e1;
        if (cudaEventCreate(&e0) != cudaSuccess) return LENIA_ERR_CUDA;
        if (cudaEventCreate(&e1) != cudaSuccess) {
            cudaEventDestroy(e0);
            return LENIA_ERR_CUDA;
        }
        const double flops = 2.0 * double(blocks) * 256.0 * kIters * kChains;
        double best[2] = {0.0, 0.0};
        cudaError_t err = cudaSuccess;
        for (int which = 0; which < 2 && err == cudaSuccess; ++which) {
            for (int r = 0; r <= reps && err == cudaSuccess; ++r) {
                cudaEventRecord(e0, s);
                if (which == 0)
                    fma_peak_kernel<<<blocks, 256, 0, s>>>(0.999f, 1e-4f);
                else
                    fma2_peak_kernel<<<blocks, 256, 0, s>>>(0.999f, 1e-4f);
                cudaEventRecord(e1, s);
                err = cudaEventSynchronize(e1);
                float ms = 0.0f;
                if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
                const double f = which == 0 ? 1.0 : 2.0;  // FFMA2: two FMAs per chain step
                if (err == cudaSuccess && r > 0 && ms > 0.0f) best[which] = std::max(best[which], f * flops / (ms * 1e-3) / 1e12);
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (err != cudaSuccess) return LENIA_ERR_CUDA;
        *out_ffma = best[0];
        *out_ffma2 = best[1];
        return LENIA_OK;
    });
}
