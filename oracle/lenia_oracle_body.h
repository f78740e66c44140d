/* oracle/lenia_oracle_body.h -- precision-generic part of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY. Included twice by lenia_oracle.c, with
 * R_T = float / SUF = _f32 and R_T = double / SUF = _f64. Each expression
 * keeps the reference's evaluation order (C evaluates left to right exactly
 * like MSL for these binary operators), and constants keep their float value
 * (RF(x) casts a float literal to R_T), so the FP32 build reproduces the
 * reference's rounding and the FP64 build only adds precision.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUF)
#define RF(x) ((R_T)(x))

static inline R_T FN(lo_exp)(R_T x) { return sizeof(R_T) == 4 ? (R_T)expf((float)x) : (R_T)exp((double)x); }
static inline R_T FN(lo_round)(R_T x) { return sizeof(R_T) == 4 ? (R_T)roundf((float)x) : (R_T)round((double)x); }
static inline R_T FN(lo_clamp)(R_T v, R_T lo, R_T hi) {
    /* clamp(v, lo, hi) = min(max(v, lo), hi) */
    R_T m = (v < lo) ? lo : v;
    return (hi < m) ? hi : m;
}
static inline R_T FN(lo_mix)(R_T a, R_T b, R_T t) { return a + (b - a) * t; }

/* Shared epilogue of leniaStep (Lenia.metal:101-127) and leniaGrowthMulti
 * (Lenia.metal:209-231): noise stir, blob injection, clamp to [0,1]. */
static inline R_T FN(lo_noise_inject)(R_T A2, uint32_t gx, uint32_t gy, float noise_amount,
                                      float inject_amount, uint32_t inject_count,
                                      uint32_t radius, uint32_t seed, uint32_t width,
                                      uint32_t height, uint32_t frame_index) {
    if (noise_amount > 0.0f) {
        R_T n = (R_T)lo_rand01(gx, gy, 503u, seed) - RF(0.5f);
        A2 += n * (R_T)noise_amount * RF(0.03f);
    }
    if (inject_amount > 0.0f) {
        R_T uvx = ((R_T)(float)gx + RF(0.5f)) / (R_T)(float)width;
        R_T uvy = ((R_T)(float)gy + RF(0.5f)) / (R_T)(float)height;
        R_T aspect = (R_T)(float)width / (R_T)(float)height;
        uint32_t cycle = frame_index / 12u;
        R_T blobR = (R_T)(float)radius * RF(0.9f) / (R_T)(float)height;
        for (uint32_t i = 0; i < inject_count; ++i) {
            R_T cx = (R_T)lo_rand01(i, cycle, 811u, seed);
            R_T cy = (R_T)lo_rand01(cycle, i, 823u, seed);
            R_T dx = uvx - cx, dy = uvy - cy;
            dx = dx - FN(lo_round)(dx);
            dy = dy - FN(lo_round)(dy);
            dx *= aspect;
            R_T r2 = (dx * dx + dy * dy) / (blobR * blobR);
            R_T bump = FN(lo_exp)(-r2 * RF(0.5f));
            A2 = FN(lo_mix)(A2, RF(0.6f), FN(lo_clamp)(bump * (R_T)inject_amount, RF(0.0f), RF(1.0f)));
        }
    }
    return FN(lo_clamp)(A2, RF(0.0f), RF(1.0f));
}

/* leniaStep, Shaders/Field/Lenia.metal:63-128: direct toroidal convolution
 * over the (2R+1)^2 LUT (zero weights skipped, dy outer, dx inner), growth
 * (mode 0 standard, mode 1 asymptotic), muJitter, noise, inject, clamp. */
void FN(lo_step_direct)(const R_T* src, R_T* dst, const float* lut, const lo_params* p,
                        uint32_t audio_frame) {
    const int R = (int)p->radius;
    const int W = (int)p->width, H = (int)p->height;
    const int ks = 2 * R + 1;
#pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; ++gy) {
        for (int gx = 0; gx < W; ++gx) {
            R_T u = RF(0.0f);
            for (int dy = -R; dy <= R; ++dy) {
                for (int dx = -R; dx <= R; ++dx) {
                    float w = lut[(dy + R) * ks + (dx + R)];
                    if (w == 0.0f) continue;
                    int qx = (gx + dx) % W, qy = (gy + dy) % H; /* wrapCoord, CommonTypes.metal:39-45 */
                    if (qx < 0) qx += W;
                    if (qy < 0) qy += H;
                    u += (R_T)w * src[(size_t)qy * W + qx];
                }
            }
            R_T A = src[(size_t)gy * W + gx];
            R_T mu = (R_T)p->growth_mu;
            if (p->mu_jitter > 0.0f) {
                R_T j = (R_T)lo_rand01((uint32_t)gx, (uint32_t)gy, 401u + audio_frame % 613u, p->seed) - RF(0.5f);
                mu += j * (R_T)p->mu_jitter * RF(0.05f);
            }
            R_T t = (u - mu) / (R_T)p->growth_sigma;
            R_T bell = FN(lo_exp)(RF(-0.5f) * t * t);
            R_T A2 = (p->growth_mode == 1u) ? A + (R_T)p->dt * (bell - A)
                                            : A + (R_T)p->dt * (RF(2.0f) * bell - RF(1.0f));
            dst[(size_t)gy * W + gx] = FN(lo_noise_inject)(
                A2, (uint32_t)gx, (uint32_t)gy, p->noise_amount, p->inject_amount, p->inject_count,
                p->radius, p->seed, p->width, p->height, p->frame_index);
        }
    }
}

/* leniaBell, Lenia.metal:156-159 */
static inline R_T FN(lo_bell)(R_T u, R_T mu, R_T sigma) {
    R_T t = (u - mu) / sigma;
    return FN(lo_exp)(RF(-0.5f) * t * t);
}

/* leniaGrowthMulti, Shaders/Field/Lenia.metal:161-232. */
void FN(lo_growth_multi)(const R_T* src, R_T* dst, const R_T* const* pot,
                         const lo_multi_params* p, uint32_t audio_frame) {
    const int W = (int)p->width, H = (int)p->height;
#pragma omp parallel for schedule(static)
    for (int gy = 0; gy < H; ++gy) {
        for (int gx = 0; gx < W; ++gx) {
            size_t i = (size_t)gy * W + gx;
            R_T A = src[i];
            R_T muJ = RF(0.0f);
            if (p->mu_jitter > 0.0f) {
                R_T j = (R_T)lo_rand01((uint32_t)gx, (uint32_t)gy, 401u + audio_frame % 613u, p->seed) - RF(0.5f);
                muJ = j * (R_T)p->mu_jitter * RF(0.05f);
            }
            R_T bell[4] = {RF(0.0f), RF(0.0f), RF(0.0f), RF(0.0f)};
            for (uint32_t k = 0; k < 4; ++k)
                if (p->num_kernels > k)
                    bell[k] = FN(lo_bell)(pot[k][i], (R_T)p->k_mu[k] + muJ, (R_T)p->k_sigma[k]);
            R_T sumWeighted = RF(0.0f), sumWeights = RF(0.0f), sumStd = RF(0.0f);
            for (uint32_t k = 0; k < p->num_kernels && k < 4u; ++k) {
                sumWeighted += (R_T)p->k_weight[k] * bell[k];
                sumWeights += (R_T)p->k_weight[k];
                sumStd += (R_T)p->k_weight[k] * (RF(2.0f) * bell[k] - RF(1.0f));
            }
            R_T A2;
            if (p->growth_mode == 1u) {
                R_T target = (sumWeights > RF(1e-6f)) ? (sumWeighted / sumWeights) : A;
                A2 = A + (R_T)p->dt * (target - A);
            } else {
                A2 = A + (R_T)p->dt * sumStd;
            }
            dst[i] = FN(lo_noise_inject)(A2, (uint32_t)gx, (uint32_t)gy, p->noise_amount,
                                         p->inject_amount, p->inject_count, p->radius, p->seed,
                                         p->width, p->height, p->frame_index);
        }
    }
}

#undef FN
#undef RF
#undef CAT
#undef CAT2
