// life_simulation_b200/csrc/lenia_types.h -- parameter blocks shared by the
// host module and the CUDA kernels (plain structs, passed by value at launch).
#pragma once
#include <cstdint>

namespace lenia {

constexpr int kMaxKernels = 4;   // Lenia.cpp:225-230 caps "kernels" at 4
constexpr int kMaxRadius = 32;   // direct path radius limit of this library
constexpr int kMaxBetas = 8;     // kernel shells per kernel

// Everything one substep's growth epilogue needs. It merges the reference's
// LeniaParams (Lenia.metal:10-27) and LeniaMultiParams (Lenia.metal:138-154);
// the direct single-kernel path is the K=1, weight=1 case of the multi form.
struct StepParams {
    float dt;
    float mu[kMaxKernels];
    float sigma[kMaxKernels];
    float weight[kMaxKernels];
    float sum_weights;        // sum_k weight[k] accumulated in kernel order
    uint32_t num_kernels;
    uint32_t growth_mode;     // 0 standard 2*bell-1, 1 asymptotic bell-A
    float noise_amount;
    float mu_jitter;
    float inject_amount;
    uint32_t inject_count;
    uint32_t radius;          // integer radius (blob size of the injection)
    uint32_t seed;            // substep seed pcgHash(seed ^ (frame*197 + s))
    uint32_t width;
    uint32_t height;
    uint32_t frame_index;     // ctx.frameIndex (injection cycle)
    uint32_t audio_frame;     // AudioUniforms.frameIndex (muJitter tag)
};

// leniaInit's inputs (Lenia.metal:43-61).
struct InitParams {
    float init_coverage;
    float init_scale;
    uint32_t seed;
    uint32_t width;
    uint32_t height;
};

}  // namespace lenia
