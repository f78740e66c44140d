// life_simulation_b200/csrc/colormap.cuh -- the cosine palette of the colour
// layer (Shaders/Render/ColorMap.metal:24-35), shared by the colour map and
// the batched form's activity statistic.
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "lenia_kernels.h"

namespace lenia {

// Channel `ch` of a one-channel field texel read as (A, 0, 0, 1).
__device__ __forceinline__ float channel_of(float r, uint32_t ch) { return ch == 0u ? r : ch >= 3u ? 1.0f : 0.0f; }

// The palette of a channel value v as the four halves of an RGBA16F texel:
// t = clamp(v * inputScale + inputBias, 0, 1), rgb = max(a + b cos(2 pi
// (c t + d)), 0) * exposure, alpha = t. Every step but the cosine rounds
// separately (no fused multiply-adds), as the reference's arithmetic.
__device__ __forceinline__ void palette_rgba16f(const ColorMapParams& p, float v, __half (&out)[4]) {
    float t = __fadd_rn(__fmul_rn(v, p.input_scale), p.input_bias);
    t = fminf(fmaxf(t, 0.0f), 1.0f);
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float phase = __fmul_rn(6.28318530718f, __fadd_rn(__fmul_rn(p.c[i], t), p.d[i]));
        out[i] = __float2half_rn(__fmul_rn(fmaxf(__fadd_rn(p.a[i], __fmul_rn(p.b[i], cosf(phase))), 0.0f), p.exposure));
    }
    out[3] = __float2half_rn(t);
}

}  // namespace lenia
