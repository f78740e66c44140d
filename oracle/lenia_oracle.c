/* oracle/lenia_oracle.c -- CPU oracle for the Lenia field update.
 *
 * TEST INFRASTRUCTURE ONLY (see lenia_oracle.h): the oracle the CUDA path is
 * compared against, never part of the product. Reference citations are
 * file:line within daitomanabe/life-simulation.
 */
#include "lenia_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- integer */

/* pcg_hash, Shaders/Common/Random.metal:5-9 == LifeCore/Math/Random.h:34-38 */
uint32_t lo_pcg_hash(uint32_t v) {
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

/* deriveSeed, LifeCore/Math/Random.h:42-44 */
uint32_t lo_derive_seed(uint32_t global_seed, uint32_t purpose_tag) {
    return lo_pcg_hash(global_seed ^ lo_pcg_hash(purpose_tag));
}

/* rand01, Shaders/Common/Random.metal:16-19: top 24 hash bits / 2^24 */
float lo_rand01(uint32_t px, uint32_t py, uint32_t tag, uint32_t seed) {
    uint32_t h = lo_pcg_hash(px ^ lo_pcg_hash(py ^ lo_pcg_hash(tag ^ seed)));
    return (float)(h >> 8) * (1.0f / 16777216.0f);
}

/* ------------------------------------------------------ precision bodies */

#define R_T float
#define SUF _f32
#include "lenia_oracle_body.h"
#undef R_T
#undef SUF

#define R_T double
#define SUF _f64
#include "lenia_oracle_body.h"
#undef R_T
#undef SUF

/* --------------------------------------------------- kernel construction */

/* Chan's exponential core exp(4 - 1/(r(1-r))) on r in (0,1), zero outside.
 * Not in the reference; evaluated in FP64. */
static double lo_exp_core(double r) {
    if (!(r > 0.0 && r < 1.0)) return 0.0;
    return exp(4.0 - 1.0 / (r * (1.0 - r)));
}

/* buildKernelTexture, Modules/FieldModules/Lenia.cpp:410-446: direct LUT of
 * (2R+1)^2 weights, r = |d|/R, Gaussian shell bell(r; shellMu, shellSigma)
 * on 0 < r <= 1, float arithmetic, double sum, scaled by float(1/sum).
 * LO_CORE_EXP replaces the shell by the exponential core (FP64, then
 * normalised in FP64 and rounded once). */
void lo_build_direct_lut(uint32_t radius, float shell_mu, float shell_sigma, int core, float* out) {
    const uint32_t R = radius, size = 2 * radius + 1;
    double sum = 0.0;
    if (core == LO_CORE_EXP) {
        double* tmp = (double*)malloc(sizeof(double) * size * size);
        for (uint32_t y = 0; y < size; ++y)
            for (uint32_t x = 0; x < size; ++x) {
                double dx = (double)((int)x - (int)R), dy = (double)((int)y - (int)R);
                double r = R ? sqrt(dx * dx + dy * dy) / (double)R : 0.0;
                double w = lo_exp_core(r);
                tmp[y * size + x] = w;
                sum += w;
            }
        for (uint32_t i = 0; i < size * size; ++i) out[i] = sum > 0.0 ? (float)(tmp[i] / sum) : 0.0f;
        free(tmp);
        return;
    }
    for (uint32_t y = 0; y < size; ++y)
        for (uint32_t x = 0; x < size; ++x) {
            float dx = (float)((int)x - (int)R);
            float dy = (float)((int)y - (int)R);
            float r = sqrtf(dx * dx + dy * dy) / (float)R;
            float w = 0.0f;
            if (r <= 1.0f && r > 0.0f) {
                float t = (r - shell_mu) / shell_sigma;
                w = expf(-0.5f * t * t);
            }
            out[y * size + x] = w;
            sum += w;
        }
    if (sum > 0.0) {
        float inv = (float)(1.0 / sum);
        for (uint32_t i = 0; i < size * size; ++i) out[i] *= inv;
    }
}

/* buildRingKernelImage, Modules/FieldModules/Lenia.cpp:95-125: a w x h image
 * with the kernel centred at (0,0), toroidally wrapped; B = nbetas shells,
 * u = (r/Rk)*B, i = min(floor(u), B-1), w = betas[i]*bell(u-i; 0.5,
 * shellSigma*B) on 0 < r <= Rk; float arithmetic, double sum, float(1/sum)
 * scale. LO_CORE_EXP: w = betas[i]*exp_core(u - i), FP64 then rounded. */
void lo_build_ring_image(uint32_t w, uint32_t h, float radius_k, float shell_sigma,
                         const float* betas, uint32_t nbetas, int core, float* out) {
    memset(out, 0, sizeof(float) * (size_t)w * h);
    if (nbetas == 0 || radius_k <= 0.0f) return;
    const uint32_t B = nbetas;
    const float Bf = (float)B;
    double sum = 0.0;
    if (core == LO_CORE_EXP) {
        double* tmp = (double*)calloc((size_t)w * h, sizeof(double));
        for (uint32_t y = 0; y < h; ++y) {
            int dy = (int)y;
            if (dy > (int)(h / 2)) dy -= (int)h;
            for (uint32_t x = 0; x < w; ++x) {
                int dx = (int)x;
                if (dx > (int)(w / 2)) dx -= (int)w;
                double r = sqrt((double)dx * dx + (double)dy * dy);
                double v = 0.0;
                if (r > 0.0 && r <= (double)radius_k) {
                    double u = (r / (double)radius_k) * (double)B;
                    uint32_t i = (uint32_t)u;
                    if (i > B - 1) i = B - 1;
                    v = (double)betas[i] * lo_exp_core(u - (double)i);
                }
                tmp[(size_t)y * w + x] = v;
                sum += v;
            }
        }
        for (size_t i = 0; i < (size_t)w * h; ++i) out[i] = sum > 0.0 ? (float)(tmp[i] / sum) : 0.0f;
        free(tmp);
        return;
    }
    for (uint32_t y = 0; y < h; ++y) {
        int dy = (int)y;
        if (dy > (int)(h / 2)) dy -= (int)h;
        for (uint32_t x = 0; x < w; ++x) {
            int dx = (int)x;
            if (dx > (int)(w / 2)) dx -= (int)w;
            float r = sqrtf((float)dx * (float)dx + (float)dy * (float)dy);
            float v = 0.0f;
            if (r > 0.0f && r <= radius_k) {
                float u = (r / radius_k) * Bf;
                uint32_t i = (uint32_t)u;
                if (i > B - 1) i = B - 1;
                float t = (u - (float)i - 0.5f) / (shell_sigma * Bf);
                v = betas[i] * expf(-0.5f * t * t);
            }
            out[(size_t)y * w + x] = v;
            sum += v;
        }
    }
    if (sum > 0.0) {
        float inv = (float)(1.0 / sum);
        for (size_t i = 0; i < (size_t)w * h; ++i) out[i] *= inv;
    }
}

/* ------------------------------------------------------------------ inits */

/* leniaValueNoise, Shaders/Field/Lenia.metal:32-41 */
static float lo_value_noise(float px, float py, uint32_t tag, uint32_t seed) {
    float ix = floorf(px) + 512.0f, iy = floorf(py) + 512.0f;
    float fx = px - floorf(px), fy = py - floorf(py);
    fx = fx * fx * (3.0f - 2.0f * fx);
    fy = fy * fy * (3.0f - 2.0f * fy);
    float a = lo_rand01((uint32_t)ix, (uint32_t)iy, tag, seed);
    float b = lo_rand01((uint32_t)(ix + 1.0f), (uint32_t)(iy + 0.0f), tag, seed);
    float c = lo_rand01((uint32_t)(ix + 0.0f), (uint32_t)(iy + 1.0f), tag, seed);
    float d = lo_rand01((uint32_t)(ix + 1.0f), (uint32_t)(iy + 1.0f), tag, seed);
    float ab = a + (b - a) * fx, cd = c + (d - c) * fx;
    return ab + (cd - ab) * fy;
}

/* leniaInit, Shaders/Field/Lenia.metal:43-61: 3-octave value noise soup. */
void lo_init_noise(const lo_params* p, float* out) {
    const uint32_t W = p->width, H = p->height;
    const float scale = p->init_scale > 2.0f ? p->init_scale : 2.0f;  /* max(initScale, 2) */
    const float cov = p->init_coverage > 1e-3f ? p->init_coverage : 1e-3f;
#pragma omp parallel for schedule(static)
    for (long gy = 0; gy < (long)H; ++gy)
        for (uint32_t gx = 0; gx < W; ++gx) {
            float px = (float)gx / scale, py = (float)gy / scale;
            float v = 0.55f * lo_value_noise(px, py, 11u, p->seed) +
                      0.30f * lo_value_noise(px * 2.13f, py * 2.13f, 23u, p->seed) +
                      0.15f * lo_value_noise(px * 4.31f, py * 4.31f, 37u, p->seed);
            v = (v - (1.0f - p->init_coverage)) / cov;
            v = v < 0.0f ? 0.0f : v;
            v = 1.0f < v ? 1.0f : v;
            v *= 0.9f;
            out[(size_t)gy * W + gx] = v;
        }
}

/* leniaStampInit, Shaders/Field/Lenia.metal:258-303: up to 32 organism
 * stamps at hashed centres, 8 dihedral orientations, nearest sampling, max. */
void lo_init_stamp(uint32_t w, uint32_t h, const float* org, uint32_t ow, uint32_t oh,
                   uint32_t stamp_count, uint32_t stamp_rotate, uint32_t seed, float* out) {
    const float ocx = (float)ow * 0.5f, ocy = (float)oh * 0.5f;
    const uint32_t count = stamp_count < 32u ? stamp_count : 32u;
#pragma omp parallel for schedule(static)
    for (long gy = 0; gy < (long)h; ++gy)
        for (uint32_t gx = 0; gx < w; ++gx) {
            float A = 0.0f;
            for (uint32_t i = 0; i < count; ++i) {
                float cx = lo_rand01(i, 0u, 907u, seed) * (float)w;
                float cy = lo_rand01(0u, i, 911u, seed) * (float)h;
                uint32_t variant = 0u;
                if (stamp_rotate != 0u) {
                    uint32_t v = (uint32_t)(lo_rand01(i, 1u, 919u, seed) * 8.0f);
                    variant = v < 7u ? v : 7u;
                }
                float dx = (float)gx + 0.5f - cx;
                float dy = (float)gy + 0.5f - cy;
                dx -= (float)w * roundf(dx / (float)w);
                dy -= (float)h * roundf(dy / (float)h);
                if (variant & 4u) dx = -dx;
                uint32_t rot = variant & 3u;
                float lx_f = dx, ly_f = dy;
                if (rot == 1u) { lx_f = dy; ly_f = -dx; }
                else if (rot == 2u) { lx_f = -dx; ly_f = -dy; }
                else if (rot == 3u) { lx_f = -dy; ly_f = dx; }
                lx_f += ocx;
                ly_f += ocy;
                int lx = (int)floorf(lx_f), ly = (int)floorf(ly_f);
                if (lx >= 0 && lx < (int)ow && ly >= 0 && ly < (int)oh) {
                    float v = org[(size_t)ly * ow + lx];
                    A = (A < v) ? v : A;  /* max(A, v) */
                }
            }
            A = A < 0.0f ? 0.0f : A;
            A = 1.0f < A ? 1.0f : A;
            out[(size_t)gy * w + gx] = A;
        }
}

/* ------------------------------------------------ FP64 direct convolution */

void lo_conv_direct_f64(const double* src, const float* kimg, uint32_t w, uint32_t h,
                        double* pot) {
    /* Gather the nonzero taps once: offsets (dx, dy) in (-w/2, w/2] x (-h/2, h/2]. */
    size_t n = 0;
    for (size_t i = 0; i < (size_t)w * h; ++i) n += kimg[i] != 0.0f;
    int* tx = (int*)malloc(sizeof(int) * (n + 1));
    int* ty = (int*)malloc(sizeof(int) * (n + 1));
    double* tw = (double*)malloc(sizeof(double) * (n + 1));
    size_t t = 0;
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            float v = kimg[(size_t)y * w + x];
            if (v == 0.0f) continue;
            tx[t] = (int)x;
            ty[t] = (int)y;
            tw[t] = (double)v;
            ++t;
        }
    /* Circular convolution pot[n] = sum_d K[d] * A[n - d]. */
#pragma omp parallel for schedule(static)
    for (long gy = 0; gy < (long)h; ++gy)
        for (uint32_t gx = 0; gx < w; ++gx) {
            double acc = 0.0;
            for (size_t k = 0; k < n; ++k) {
                uint32_t qx = (gx + w - (uint32_t)tx[k]) % w;
                uint32_t qy = ((uint32_t)gy + h - (uint32_t)ty[k]) % h;
                acc += tw[k] * src[(size_t)qy * w + qx];
            }
            pot[(size_t)gy * w + gx] = acc;
        }
    free(tx);
    free(ty);
    free(tw);
}

/* ------------------------------------- the reference's radix-2 FFT (FP32) */

/* One fftStageX/Y pass, Shaders/Common/FFT.metal:65-121, for every row
 * (axis 0) or column (axis 1): radix-2 Stockham autosort with per-thread
 * cos/sin twiddles, optional 1/N scale on the inverse's last stage. */
static void lo_fft_stage_f32(const float* sre, const float* sim, float* dre, float* dim,
                             uint32_t w, uint32_t h, int axis, uint32_t N, uint32_t Ns, int dir,
                             int normalize) {
    const uint32_t halfN = N / 2u;
    const uint32_t lines = axis == 0 ? h : w;
#pragma omp parallel for schedule(static)
    for (long l = 0; l < (long)lines; ++l) {
        for (uint32_t j = 0; j < halfN; ++j) {
            float angle = -(float)dir * 6.28318530718f * (float)(j % Ns) / (float)(Ns * 2u);
            float twx = cosf(angle), twy = sinf(angle);
            size_t i0, i1, o0, o1;
            uint32_t idxD = (j / Ns) * Ns * 2u + (j % Ns);
            if (axis == 0) {
                i0 = (size_t)l * w + j;
                i1 = (size_t)l * w + j + halfN;
                o0 = (size_t)l * w + idxD;
                o1 = (size_t)l * w + idxD + Ns;
            } else {
                i0 = (size_t)j * w + l;
                i1 = (size_t)(j + halfN) * w + l;
                o0 = (size_t)idxD * w + l;
                o1 = (size_t)(idxD + Ns) * w + l;
            }
            float v0x = sre[i0], v0y = sim[i0];
            float ax = sre[i1], ay = sim[i1];
            float v1x = ax * twx - ay * twy; /* fftComplexMul, FFT.metal:59-61 */
            float v1y = ax * twy + ay * twx;
            float o0x = v0x + v1x, o0y = v0y + v1y;
            float o1x = v0x - v1x, o1y = v0y - v1y;
            if (normalize) {
                float inv = 1.0f / (float)N;
                o0x *= inv; o0y *= inv; o1x *= inv; o1y *= inv;
            }
            dre[o0] = o0x; dim[o0] = o0y;
            dre[o1] = o1x; dim[o1] = o1y;
        }
    }
}

static uint32_t lo_log2u(uint32_t v) {
    uint32_t r = 0;
    while (v > 1u) { v >>= 1; ++r; }
    return r;
}

/* encodeFFT2D, Modules/FieldModules/Lenia.cpp:57-85: all log2(w) X stages
 * then all log2(h) Y stages, ping-ponging; the inverse (dir < 0) scales on
 * the last stage of each axis. */
void lo_fft2d_ref_f32(float* re, float* im, uint32_t w, uint32_t h, int dir) {
    const size_t n = (size_t)w * h;
    float* bre = (float*)malloc(sizeof(float) * n);
    float* bim = (float*)malloc(sizeof(float) * n);
    float *cre = re, *cim = im, *nre = bre, *nim = bim;
    uint32_t sx = lo_log2u(w), sy = lo_log2u(h);
    for (uint32_t s = 0; s < sx; ++s) {
        lo_fft_stage_f32(cre, cim, nre, nim, w, h, 0, w, 1u << s, dir, dir < 0 && s + 1 == sx);
        float* t = cre; cre = nre; nre = t;
        t = cim; cim = nim; nim = t;
    }
    for (uint32_t s = 0; s < sy; ++s) {
        lo_fft_stage_f32(cre, cim, nre, nim, w, h, 1, h, 1u << s, dir, dir < 0 && s + 1 == sy);
        float* t = cre; cre = nre; nre = t;
        t = cim; cim = nim; nim = t;
    }
    if (cre != re) {
        memcpy(re, cre, sizeof(float) * n);
        memcpy(im, cim, sizeof(float) * n);
    }
    free(bre);
    free(bim);
}

/* One FFT-path substep, Modules/FieldModules/Lenia.cpp:576-643:
 * realToComplex, forward FFT2D of the state, then per kernel
 * complexMulScale (normalize=0, FFT.metal:131-142), inverse FFT2D,
 * complexToReal, and finally leniaGrowthMulti. */
void lo_step_fft_ref_f32(const float* src, float* dst, const float* kre, const float* kim,
                         const lo_multi_params* p, uint32_t audio_frame) {
    const uint32_t w = p->width, h = p->height;
    const size_t n = (size_t)w * h;
    float* sre = (float*)malloc(sizeof(float) * n);
    float* sim = (float*)calloc(n, sizeof(float));
    float* pre = (float*)malloc(sizeof(float) * n);
    float* pim = (float*)malloc(sizeof(float) * n);
    float* pots = (float*)calloc(4 * n, sizeof(float));
    memcpy(sre, src, sizeof(float) * n);
    lo_fft2d_ref_f32(sre, sim, w, h, +1);
    const uint32_t nk = p->num_kernels < 4u ? p->num_kernels : 4u;
    for (uint32_t k = 0; k < nk; ++k) {
        const float* br = kre + k * n;
        const float* bi = kim + k * n;
        for (size_t i = 0; i < n; ++i) {
            float ax = sre[i], ay = sim[i];
            pre[i] = ax * br[i] - ay * bi[i];
            pim[i] = ax * bi[i] + ay * br[i];
        }
        lo_fft2d_ref_f32(pre, pim, w, h, -1);
        memcpy(pots + k * n, pre, sizeof(float) * n);
    }
    const float* pp[4] = {pots, pots + n, pots + 2 * n, pots + 3 * n};
    lo_growth_multi_f32(src, dst, pp, p, audio_frame);
    free(sre);
    free(sim);
    free(pre);
    free(pim);
    free(pots);
}
