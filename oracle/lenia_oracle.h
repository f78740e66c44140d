/* oracle/lenia_oracle.h -- CPU oracle for the Lenia field update.
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's Lenia
 * hot path, used by tests/, the smoke check and bench.py's CPU-baseline leg to
 * check the CUDA kernels. It is never linked into or called by the product.
 *
 * Every arithmetic kernel exists in an FP32 build (suffix _f32), whose
 * operation order and float rounding follow the reference's Metal source
 * term by term (so it reproduces the CPU-compiled reference bit for bit), and
 * an FP64 build (suffix _f64) of the same source, which is the accuracy
 * oracle. Integer work (the PCG hash and seed derivation) is shared.
 * Constants keep their float values in both builds.
 */
#ifndef LENIA_ORACLE_H
#define LENIA_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Mirrors LeniaParams, Shaders/Field/Lenia.metal:10-27 (scalar-packed). */
typedef struct lo_params {
    float dt, growth_mu, growth_sigma, noise_amount, mu_jitter;
    float init_coverage, init_scale, inject_amount;
    uint32_t inject_count, radius, kernel_size, seed, width, height, frame_index, growth_mode;
} lo_params;

/* Mirrors LeniaMultiParams, Shaders/Field/Lenia.metal:138-154. */
typedef struct lo_multi_params {
    float dt;
    float k_mu[4], k_sigma[4], k_weight[4];
    uint32_t num_kernels, growth_mode;
    float noise_amount, mu_jitter, inject_amount;
    uint32_t inject_count, radius, seed, width, height, frame_index;
} lo_multi_params;

/* Kernel radial profiles. */
enum { LO_CORE_GAUSS_SHELL = 0, LO_CORE_EXP = 1 };

/* ---- integer (bit-exact) ---- */
uint32_t lo_pcg_hash(uint32_t v);
uint32_t lo_derive_seed(uint32_t global_seed, uint32_t purpose_tag);
float lo_rand01(uint32_t px, uint32_t py, uint32_t tag, uint32_t seed);

/* ---- kernel construction (float weights, double normalisation sum) ---- */
void lo_build_direct_lut(uint32_t radius, float shell_mu, float shell_sigma, int core, float* out);
void lo_build_ring_image(uint32_t w, uint32_t h, float radius_k, float shell_sigma,
                         const float* betas, uint32_t nbetas, int core, float* out);

/* ---- inits (FP32, as the reference) ---- */
void lo_init_noise(const lo_params* p, float* out);
void lo_init_stamp(uint32_t w, uint32_t h, const float* org, uint32_t ow, uint32_t oh,
                   uint32_t stamp_count, uint32_t stamp_rotate, uint32_t seed, float* out);

/* ---- one direct step (leniaStep) ---- */
void lo_step_direct_f32(const float* src, float* dst, const float* lut, const lo_params* p,
                        uint32_t audio_frame);
void lo_step_direct_f64(const double* src, double* dst, const float* lut, const lo_params* p,
                        uint32_t audio_frame);

/* ---- growth over precomputed potentials (leniaGrowthMulti) ---- */
void lo_growth_multi_f32(const float* src, float* dst, const float* const* pot,
                         const lo_multi_params* p, uint32_t audio_frame);
void lo_growth_multi_f64(const double* src, double* dst, const double* const* pot,
                         const lo_multi_params* p, uint32_t audio_frame);

/* ---- potentials by direct circular convolution, FP64 ----
 * pot[y*w+x] = sum over taps of kimg[tap] * src[(y+dy) mod h][(x+dx) mod w],
 * kimg in the wrap-centred layout of the ring image (tap (0,0) at index 0). */
void lo_conv_direct_f64(const double* src, const float* kimg, uint32_t w, uint32_t h,
                        double* pot);

/* ---- the reference's FFT path in FP32 (radix-2 Stockham, per-stage) ----
 * In-place 2D complex transform of (re, im), w and h powers of two, in the
 * reference's stage order (all X stages, then all Y stages). */
void lo_fft2d_ref_f32(float* re, float* im, uint32_t w, uint32_t h, int dir);
/* Full FFT substep: potentials for nk kernels from their spectra
 * (kre/kim: nk planes), then leniaGrowthMulti. */
void lo_step_fft_ref_f32(const float* src, float* dst, const float* kre, const float* kim,
                         const lo_multi_params* p, uint32_t audio_frame);

#ifdef __cplusplus
}
#endif
#endif
