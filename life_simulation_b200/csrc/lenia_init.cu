// life_simulation_b200/csrc/lenia_init.cu -- field initialisers: the
// value-noise soup (leniaInit, Shaders/Field/Lenia.metal:29-61) and the
// organism stamps (leniaStampInit, Shaders/Field/Lenia.metal:242-303). One
// thread per pixel; they run once per reset and are not on the timed path.
#include <cuda_runtime.h>

#include <cstdint>

#include "lenia_device.cuh"
#include "lenia_kernels.h"

namespace lenia {

namespace {

// leniaValueNoise (Lenia.metal:32-41): smoothstep-interpolated lattice hash.
__device__ float value_noise(float px, float py, uint32_t tag, uint32_t seed) {
    const float ix = floorf(px) + 512.0f, iy = floorf(py) + 512.0f;
    float fx = px - floorf(px), fy = py - floorf(py);
    fx = __fmul_rn(__fmul_rn(fx, fx), __fsub_rn(3.0f, __fmul_rn(2.0f, fx)));
    fy = __fmul_rn(__fmul_rn(fy, fy), __fsub_rn(3.0f, __fmul_rn(2.0f, fy)));
    const float a = rand01(uint32_t(ix), uint32_t(iy), tag, seed);
    const float b = rand01(uint32_t(ix + 1.0f), uint32_t(iy), tag, seed);
    const float c = rand01(uint32_t(ix), uint32_t(iy + 1.0f), tag, seed);
    const float d = rand01(uint32_t(ix + 1.0f), uint32_t(iy + 1.0f), tag, seed);
    const float ab = __fadd_rn(a, __fmul_rn(__fsub_rn(b, a), fx));
    const float cd = __fadd_rn(c, __fmul_rn(__fsub_rn(d, c), fx));
    return __fadd_rn(ab, __fmul_rn(__fsub_rn(cd, ab), fy));
}

__global__ void init_noise_kernel(float* __restrict__ A, InitParams p) {
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= p.width || gy >= p.height) return;
    const float scale = fmaxf(p.init_scale, 2.0f);
    const float px = __fdiv_rn(float(gx), scale), py = __fdiv_rn(float(gy), scale);
    // Separate roundings (no contraction) so the soup matches the reference
    // arithmetic bit for bit.
    float v = __fadd_rn(__fadd_rn(__fmul_rn(0.55f, value_noise(px, py, 11u, p.seed)),
                                  __fmul_rn(0.30f, value_noise(__fmul_rn(px, 2.13f),
                                                               __fmul_rn(py, 2.13f), 23u, p.seed))),
                        __fmul_rn(0.15f, value_noise(__fmul_rn(px, 4.31f), __fmul_rn(py, 4.31f),
                                                     37u, p.seed)));
    v = __fdiv_rn(__fsub_rn(v, __fsub_rn(1.0f, p.init_coverage)), fmaxf(p.init_coverage, 1e-3f));
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    A[size_t(gy) * p.width + gx] = __fmul_rn(v, 0.9f);
}

__global__ void init_stamp_kernel(float* __restrict__ A, uint32_t w, uint32_t h,
                                  const float* __restrict__ org, uint32_t ow, uint32_t oh,
                                  uint32_t count, uint32_t rotate, uint32_t seed) {
    const uint32_t gx = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t gy = blockIdx.y * blockDim.y + threadIdx.y;
    if (gx >= w || gy >= h) return;
    const float ocx = __fmul_rn(float(ow), 0.5f), ocy = __fmul_rn(float(oh), 0.5f);
    const uint32_t n = count < 32u ? count : 32u;
    float a = 0.0f;
    for (uint32_t i = 0; i < n; ++i) {
        const float cx = __fmul_rn(rand01(i, 0u, 907u, seed), float(w));
        const float cy = __fmul_rn(rand01(0u, i, 911u, seed), float(h));
        uint32_t variant = 0u;
        if (rotate != 0u) {
            const uint32_t v = uint32_t(__fmul_rn(rand01(i, 1u, 919u, seed), 8.0f));
            variant = v < 7u ? v : 7u;
        }
        float dx = __fsub_rn(__fadd_rn(float(gx), 0.5f), cx);
        float dy = __fsub_rn(__fadd_rn(float(gy), 0.5f), cy);
        dx = __fsub_rn(dx, __fmul_rn(float(w), roundf(__fdiv_rn(dx, float(w)))));
        dy = __fsub_rn(dy, __fmul_rn(float(h), roundf(__fdiv_rn(dy, float(h)))));
        if (variant & 4u) dx = -dx;
        const uint32_t rot = variant & 3u;
        float lx = dx, ly = dy;
        if (rot == 1u) { lx = dy; ly = -dx; }
        else if (rot == 2u) { lx = -dx; ly = -dy; }
        else if (rot == 3u) { lx = -dy; ly = dx; }
        const int ix = int(floorf(__fadd_rn(lx, ocx)));
        const int iy = int(floorf(__fadd_rn(ly, ocy)));
        if (ix >= 0 && ix < int(ow) && iy >= 0 && iy < int(oh)) a = fmaxf(a, __ldg(org + size_t(iy) * ow + ix));
    }
    A[size_t(gy) * w + gx] = fminf(fmaxf(a, 0.0f), 1.0f);
}

}  // namespace

cudaError_t launch_init_noise(float* A, const InitParams& p, cudaStream_t s) {
    dim3 block(32, 8), grid((p.width + 31) / 32, (p.height + 7) / 8);
    init_noise_kernel<<<grid, block, 0, s>>>(A, p);
    return cudaGetLastError();
}

cudaError_t launch_init_stamp(float* A, uint32_t w, uint32_t h, const float* org, uint32_t ow,
                              uint32_t oh, uint32_t count, uint32_t rotate, uint32_t seed,
                              cudaStream_t s) {
    dim3 block(32, 8), grid((w + 31) / 32, (h + 7) / 8);
    init_stamp_kernel<<<grid, block, 0, s>>>(A, w, h, org, ow, oh, count, rotate, seed);
    return cudaGetLastError();
}

}  // namespace lenia
