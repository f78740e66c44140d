// life_simulation_b200/csrc/lenia_device.cuh -- device helpers shared by
// every Lenia kernel: the PCG hash (bit-exact with the reference), and the
// growth map + Euler step + noise + blob injection + clip epilogue.
#pragma once
#include <cstdint>

#include "lenia_types.h"

namespace lenia {

// pcg_hash, Shaders/Common/Random.metal:5-9 (integer, bit-exact).
__host__ __device__ __forceinline__ uint32_t pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

// rand01, Shaders/Common/Random.metal:16-19: top 24 bits / 2^24, exact in f32.
__host__ __device__ __forceinline__ float rand01(uint32_t px, uint32_t py, uint32_t tag,
                                                 uint32_t seed) {
    uint32_t h = pcg_hash(px ^ pcg_hash(py ^ pcg_hash(tag ^ seed)));
    return float(h >> 8) * (1.0f / 16777216.0f);
}

// The per-pixel mu shift of muJitter (Lenia.metal:89-93 and :176-180).
__device__ __forceinline__ float mu_jitter_shift(const StepParams& p, uint32_t gx, uint32_t gy) {
    if (p.mu_jitter > 0.0f) {
        float j = rand01(gx, gy, 401u + p.audio_frame % 613u, p.seed) - 0.5f;
        return j * p.mu_jitter * 0.05f;
    }
    return 0.0f;
}

// bell(u; mu, sigma) = exp(-0.5 t^2), t = (u - mu) / sigma (Lenia.metal:156-159).
__device__ __forceinline__ float bell(float u, float mu, float sigma) {
    float t = (u - mu) / sigma;
    return expf(-0.5f * t * t);
}

// The same bell with a precomputed 1/sigma and one hardware base-2
// exponential: exp(-0.5 t^2) = 2^(-0.5 log2(e) t^2). ex2.approx.ftz has a
// relative error below 2^-22 (negligible against the FP32 FFT's rounding),
// and it replaces an IEEE division and the full-range expf sequence; used on
// the spectral path, where the growth map is a large share of the row pass.
// 2^x by the SFU's approximate base-2 exponential (relative error < 2^-22,
// subnormal results flushed to zero).
__device__ __forceinline__ float ex2_fast(float x) {
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// One kernel's growth terms at a pixel pair of the spectral row passes:
// bell(u) = exp(-(u - mu)^2 / (2 sigma^2)) = 2^-((u*sc - mu*sc)^2) with
// sc = sqrt(log2(e) / 2) / sigma, and the term h * (2 bell - 1) (growth mode
// 0) or h * bell (mode 1) as g1 * bell + g0 -- in packed FP32x2 pairs (one
// FFMA2, one FMUL2, two SFU exponentials, one FFMA2 per pair). With mu
// jitter the pair's centres come per pixel (mu + shift).
struct GrowthPair {
    float mu, sc;
    float2 SC, MSC, G1, G0;
    __device__ __forceinline__ GrowthPair(float mu_, float inv_sigma, float h, bool asym) : mu(mu_) {
        sc = inv_sigma * 0.84932180028801904272f;
        SC = make_float2(sc, sc);
        MSC = make_float2(-mu * sc, -mu * sc);
        const float g1 = asym ? h : 2.0f * h, g0 = asym ? 0.0f : -h;
        G1 = make_float2(g1, g1);
        G0 = make_float2(g0, g0);
    }
    // u: the potentials of pixels (x0, gy), (x0 + 1, gy).
    __device__ __forceinline__ float2 term(float2 u, const StepParams& p, bool jitter, uint32_t x0,
                                           uint32_t gy) const;
};

__device__ __forceinline__ float bell_fast(float u, float mu, float inv_sigma) {
    const float t = (u - mu) * inv_sigma;
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(-0.72134752044448170368f * t * t));
    return r;
}

// Running growth sums over kernels in the reference's order
// (Lenia.metal:188-195): sum_k h_k*bell_k and sum_k h_k*(2*bell_k - 1).
struct GrowthAcc {
    float weighted = 0.0f;
    float std_sum = 0.0f;
    __device__ __forceinline__ void add(float h, float b) {
        weighted += h * b;
        std_sum += h * (2.0f * b - 1.0f);
    }
};

// Euler step, noise stir, blob injection and clip (Lenia.metal:197-231,
// identical to leniaStep's :95-127 for one kernel of weight 1).
__device__ __forceinline__ float growth_finish(const StepParams& p, float A, const GrowthAcc& acc,
                                               uint32_t gx, uint32_t gy) {
    float A2;
    if (p.growth_mode == 1u) {
        float target = (p.sum_weights > 1e-6f) ? (acc.weighted / p.sum_weights) : A;
        A2 = A + p.dt * (target - A);
    } else {
        A2 = A + p.dt * acc.std_sum;
    }
    if (p.noise_amount > 0.0f) {
        float n = rand01(gx, gy, 503u, p.seed) - 0.5f;
        A2 += n * p.noise_amount * 0.03f;
    }
    if (p.inject_amount > 0.0f) {
        float uvx = (float(gx) + 0.5f) / float(p.width);
        float uvy = (float(gy) + 0.5f) / float(p.height);
        float aspect = float(p.width) / float(p.height);
        uint32_t cycle = p.frame_index / 12u;
        float blobR = float(p.radius) * 0.9f / float(p.height);
        for (uint32_t i = 0; i < p.inject_count; ++i) {
            float cx = rand01(i, cycle, 811u, p.seed);
            float cy = rand01(cycle, i, 823u, p.seed);
            float dx = uvx - cx, dy = uvy - cy;
            dx = dx - roundf(dx);
            dy = dy - roundf(dy);
            dx *= aspect;
            float r2 = (dx * dx + dy * dy) / (blobR * blobR);
            float bump = expf(-r2 * 0.5f);
            float a = fminf(fmaxf(bump * p.inject_amount, 0.0f), 1.0f);
            A2 = A2 + (0.6f - A2) * a;
        }
    }
    return fminf(fmaxf(A2, 0.0f), 1.0f);
}

// Out-of-line copies for kernels whose code size matters (the spectral row
// pass): noise, injection and mu jitter are rare, and inlining them grows
// the kernel past the instruction cache. Same arithmetic as above.
static __device__ __noinline__ float growth_finish_call(const StepParams& p, float A, float weighted, float std_sum,
                                                 uint32_t gx, uint32_t gy) {
    GrowthAcc acc;
    acc.weighted = weighted;
    acc.std_sum = std_sum;
    return growth_finish(p, A, acc, gx, gy);
}
static __device__ __noinline__ float mu_jitter_shift_call(const StepParams& p, uint32_t gx, uint32_t gy) {
    return mu_jitter_shift(p, gx, gy);
}

__device__ __forceinline__ float2 GrowthPair::term(float2 u, const StepParams& p, bool jitter, uint32_t x0,
                                                   uint32_t gy) const {
    float2 d;  // (u - mu) * sc for both pixels
    if (jitter) {
        const float m0 = mu + mu_jitter_shift_call(p, x0, gy);
        const float m1 = mu + mu_jitter_shift_call(p, x0 + 1u, gy);
        d = make_float2((u.x - m0) * sc, (u.y - m1) * sc);
    } else {
        d = __ffma2_rn(u, SC, MSC);
    }
    const float2 q = __fmul2_rn(d, d);
    const float2 b = make_float2(ex2_fast(-q.x), ex2_fast(-q.y));
    return __ffma2_rn(b, G1, G0);
}
// growth_finish with the common case (no noise, no injection) inline.
__device__ __forceinline__ float growth_finish_lean(const StepParams& p, float A, float weighted, float std_sum,
                                                    uint32_t gx, uint32_t gy) {
    if (p.noise_amount > 0.0f || p.inject_amount > 0.0f) return growth_finish_call(p, A, weighted, std_sum, gx, gy);
    float A2;
    if (p.growth_mode == 1u) {
        const float target = (p.sum_weights > 1e-6f) ? (weighted / p.sum_weights) : A;
        A2 = A + p.dt * (target - A);
    } else {
        A2 = A + p.dt * std_sum;
    }
    return fminf(fmaxf(A2, 0.0f), 1.0f);
}

}  // namespace lenia
