/* include/lenia_b200.h -- C ABI of the B200 Lenia field update.
 *
 * A drop-in for the reference's Lenia module step (daitomanabe/life-simulation,
 * Modules/FieldModules/Lenia.{h,cpp} behind the module plugin interface
 * LifeCore/Sim/SimulationModule.h). Every entry point takes and returns plain
 * C types; device memory is owned by the context (the reference's
 * ResourcePool role, LifeCore/Metal/ResourcePool.h:1-6) and the caller sees
 * device pointers only through lenia_field_device_ptr().
 *
 * All functions return a status: LENIA_OK (0); LENIA_WARN_FALLBACK (> 0) when
 * the reference would have printed a "[life] ..." warning and fallen back
 * (Lenia.cpp:226-228, :245-251, :259-269, :285-298, :306-312) -- the call
 * succeeded and lenia_last_message() says what was substituted; or a negative
 * LENIA_ERR_* code, after which the context is unchanged (or, for
 * LENIA_ERR_CUDA, should be destroyed).
 *
 * Threading: a context is used from one host thread at a time (the
 * reference's encode runs on the caller thread, LifeCore/Metal/
 * CommandGraph.mm:69-88). Work is queued on the CUDA stream passed to
 * lenia_encode()/lenia_step() (NULL = the context's own stream).
 */
#ifndef LENIA_B200_H
#define LENIA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LENIA_B200_ABI_VERSION 1

enum {
    LENIA_OK = 0,
    LENIA_WARN_FALLBACK = 1,
    LENIA_ERR_INVALID_ARG = -1,
    LENIA_ERR_UNSUPPORTED = -2,
    LENIA_ERR_CUDA = -3,
    LENIA_ERR_TIMEOUT = -4,
    LENIA_ERR_STATE = -5,
    LENIA_ERR_NO_DEVICE = -6,
    LENIA_ERR_PARSE = -7,
};

/* Convolution paths. DIRECT and FFT are the reference's convMode values
 * "direct" and "fft" (Lenia.cpp:213-214); DIRECT_MULTI ("directMulti") is
 * this library's direct convolution over all "kernels" (the FFT path's math
 * without the FFT), used to cross-check the two paths. */
enum { LENIA_CONV_DIRECT = 0, LENIA_CONV_FFT = 1, LENIA_CONV_DIRECT_MULTI = 2 };
/* Kernel radial profile. GAUSS_SHELL is the reference's (Lenia.cpp:410-446,
 * :95-125); EXP is exp(4 - 1/(r(1-r))) (Chan's exponential core). */
enum { LENIA_CORE_GAUSS_SHELL = 0, LENIA_CORE_EXP = 1 };
enum { LENIA_INIT_NOISE = 0, LENIA_INIT_STAMP = 1 };

/* One entry of the scene "kernels" array (KernelDef, Lenia.h:99-105). */
typedef struct lenia_kernel_def {
    float radius_scale; /* R_k = radius * radius_scale */
    float mu;
    float sigma;
    float weight;       /* h_k */
    uint32_t num_betas; /* 1..8 ring peaks */
    float betas[8];
} lenia_kernel_def;

/* Setup-time parameters: the module's scene "params" block
 * (Lenia.h:29-36, parsed at Lenia.cpp:208-357). */
typedef struct lenia_config {
    uint32_t sim_width;       /* 0 = scene width  (simWidth)  */
    uint32_t sim_height;      /* 0 = scene height (simHeight) */
    uint32_t conv_mode;       /* LENIA_CONV_* (convMode) */
    uint32_t fft_any_size;    /* 0: the reference's power-of-two rule for FFT
                                 (falls back to direct); 1: any even width and
                                 a height whose factors are 2, 3, 5 */
    uint32_t has_radius;      /* 0: radius defaults to 13 or the organism's R */
    uint32_t radius;          /* radius (px) */
    uint32_t num_kernels;     /* 0..4 entries of `kernels` (more: truncated) */
    lenia_kernel_def kernels[4];
    uint32_t kernel_core;     /* LENIA_CORE_* (kernelCore) */
    float kernel_shell_mu;    /* kernelShellMu (0.5) */
    float kernel_shell_sigma; /* kernelShellSigma (0.15) */
    float init_coverage;      /* initCoverage (0.4) */
    float init_scale;         /* initScale (24) */
    uint32_t init_mode;       /* LENIA_INIT_* (initMode) */
    /* Organism (initMode "stamp" / useOrganismParams, Lenia.cpp:271-321).
     * organism_cells: row-major org_height x org_width values in [0,1], or
     * NULL when no organism is given; the pointer is read during
     * lenia_create only. */
    const float* organism_cells;
    uint32_t org_width, org_height;
    float org_R, org_T, org_mu, org_sigma;
    uint32_t stamp_count;          /* stampCount (6, max 32) */
    uint32_t stamp_rotate;         /* stampRotate (1) */
    uint32_t use_organism_params;  /* useOrganismParams (1) */
    /* fftPrecision: arithmetic of the spectral path's column DFT stages.
     * LENIA_FFT_FP32 (default): FP32 on the CUDA cores. LENIA_FFT_BF16X3 /
     * LENIA_FFT_FP16X3: on the tensor cores with split-precision BF16 / FP16
     * hi/lo operands and FP32 accumulation, for column lengths 256 and 4096
     * (other sizes fall back to FP32 with a warning). No counterpart in the
     * reference. */
    uint32_t fft_precision;
} lenia_config;
enum { LENIA_FFT_FP32 = 0, LENIA_FFT_BF16X3 = 1, LENIA_FFT_FP16X3 = 2 };

/* Per-frame values the reference reads through param(ctx, key, fallback)
 * (Lenia.cpp:456-464) plus the frame's indices. */
typedef struct lenia_frame_params {
    float dt;
    float growth_mu;
    float growth_sigma;
    float noise_amount;
    float mu_jitter;
    float inject_amount;
    uint32_t inject_count;
    uint32_t growth_mode;     /* 0 standard, 1 asymptotic */
    uint32_t frame_index;     /* SimulationContext::frameIndex */
    uint32_t audio_frame;     /* AudioUniforms::frameIndex */
} lenia_frame_params;

/* What setup resolved (after the reference's fallbacks). */
typedef struct lenia_info {
    uint32_t sim_width, sim_height;
    uint32_t conv_mode;       /* path actually used */
    uint32_t radius;          /* integer radius after rounding */
    uint32_t num_kernels;     /* kernels convolved per substep */
    uint32_t use_stamp_init;
    uint64_t device_bytes;    /* device memory held by the context */
    uint32_t fft_radix_row[8], fft_radix_col[8]; /* FFT plans (0-terminated) */
    uint32_t fft_precision;   /* LENIA_FFT_* of the column DFT stages in use */
    uint32_t direct_tma;      /* 1: the direct path loads interior halo tiles by TMA */
    uint32_t direct_split;    /* direct path: thread groups sharing a tile's kernel rows (1, 2, 4, 8) */
    uint32_t direct_outputs_per_thread; /* direct path: 8, or 16 on large tiles where faster */
    uint32_t direct_taps;     /* direct path: nonzero kernel taps summed over its kernels */
    uint32_t direct_rows_per_thread; /* direct path: output rows per thread, 1 or 2 (large tiles where faster) */
    uint32_t tc_engine;       /* column DFT stages on the tensor cores: 0 none, 1 mma.sync tiles (radix 16),
                                 2 tcgen05 GEMMs (radix 64, 4096-row fields), 3 the same pipelined over
                                 two operand slots */
} lenia_info;

typedef struct lenia_ctx lenia_ctx;

/* Fills `cfg` with the reference's defaults (Lenia.h:77-105). */
void lenia_config_defaults(lenia_config* cfg);

/* configure + setup (SimulationModule::configure, SimulationModule.h:112-115;
 * LeniaModule::setup, Lenia.cpp:208-408) on the current CUDA device.
 * scene_w/scene_h: SimulationContext::width/height. */
int lenia_create(const lenia_config* cfg, uint32_t scene_w, uint32_t scene_h, lenia_ctx** out);

/* Same, from the module's scene JSON "params" object, text as in the
 * reference presets (Presets/lenia_*.json). Numeric and boolean leaves become
 * per-frame base values (Scene::applyBaseParams, LifeCore/Params/Scene.cpp:
 * 96-113). An "organism" path is read relative to the working directory or
 * `base_dir` (may be NULL), as LeniaModule::setup does (Lenia.cpp:151-204). */
int lenia_create_json(const char* params_json, uint32_t scene_w, uint32_t scene_h,
                      const char* base_dir, lenia_ctx** out);

int lenia_destroy(lenia_ctx* ctx);

/* The host half of lenia_create_json without touching a device: what setup
 * would resolve for these params (sizes, path after the reference's
 * fallbacks, radius, kernel count); out->device_bytes is 0. Warnings are
 * returned by lenia_last_message(NULL). Useful to validate a preset. */
int lenia_inspect_json(const char* params_json, uint32_t scene_w, uint32_t scene_h,
                       const char* base_dir, lenia_info* out);

/* LeniaModule::reset (Lenia.cpp:448-451): seed = deriveSeed(seed, "LEN1");
 * the next encode re-initialises the field. */
int lenia_reset(lenia_ctx* ctx, uint32_t seed);

/* Base value of a per-frame parameter, by the key param() uses ("dt",
 * "growthMu", ...): ParameterBus::setBase for "<instance>.<key>"
 * (LifeCore/Params/ParameterBus.h:98-99). */
int lenia_set_param(lenia_ctx* ctx, const char* key, float value);
/* Manual override layer (ParameterBus::setOverride / clearOverride,
 * ParameterBus.h:111-113): wins over base and mappings. */
int lenia_set_override(lenia_ctx* ctx, const char* key, float value);
int lenia_clear_override(lenia_ctx* ctx, const char* key);
/* The frame parameters encode would use now (param(ctx, key, fallback) for
 * every key, Lenia.cpp:456-464), with the given frame indices. */
int lenia_resolve_frame_params(lenia_ctx* ctx, uint32_t frame_index, uint32_t audio_frame,
                               lenia_frame_params* out);

/* One frame: LeniaModule::updateCPU + encode (Lenia.cpp:453-644). Runs the
 * init pass if needed, then max(1, substeps) substeps with substep seeds
 * pcgHash(seed ^ (frame_index*197 + s)). Parameters come from the base and
 * override values above. Asynchronous on `stream` (NULL: context stream). */
int lenia_encode(lenia_ctx* ctx, uint32_t frame_index, uint32_t substeps,
                 uint32_t audio_frame, void* stream);

/* Same as lenia_encode with explicit per-frame parameters (bypasses the
 * parameter table). */
int lenia_step(lenia_ctx* ctx, const lenia_frame_params* fp, uint32_t substeps, void* stream);

/* Waits for the context's queued work; LENIA_ERR_CUDA if any failed
 * (CommandGraph::lastFrameHadError, CommandGraph.h:89-94). */
int lenia_sync(lenia_ctx* ctx);

/* The state field (outputField / namedOutput("field"), Lenia.h:63-71):
 * sim_height x sim_width floats, row-major. upload replaces it and marks
 * the init as done (like SimulationModule::loadState, SimulationModule.h:
 * 60-78); download waits for queued work. */
int lenia_field_size(lenia_ctx* ctx, uint32_t* width, uint32_t* height);
int lenia_upload(lenia_ctx* ctx, const float* host, size_t count);
int lenia_download(lenia_ctx* ctx, float* host, size_t count);
/* Device-to-device forms, ordered on `stream`. */
int lenia_upload_device(lenia_ctx* ctx, const float* dev, size_t count, void* stream);
int lenia_download_device(lenia_ctx* ctx, float* dev, size_t count, void* stream);
/* Current device buffer of the field; valid until the next encode/step.
 * Treat as read-only: write through lenia_upload_device. */
int lenia_field_device_ptr(lenia_ctx* ctx, const float** dev);

int lenia_get_info(lenia_ctx* ctx, lenia_info* out);

/* The context's own CUDA stream (used when NULL is passed as `stream`). */
int lenia_get_stream(lenia_ctx* ctx, void** stream);

/* Per-pass GPU timing (the reference's per-pass counter samples,
 * LifeCore/Metal/GPUTimer.h:1-40, CommandGraph.mm:108-122). With profiling
 * on, every kernel launch is bracketed by CUDA events on its stream;
 * lenia_profile_read waits for them and returns the accumulated device time
 * and launch count per phase since profiling was enabled or last read.
 * The launch counter runs whether or not profiling is on. */
enum {
    LENIA_PHASE_INIT = 0,       /* noise or stamp init */
    LENIA_PHASE_DIRECT = 1,     /* fused direct convolution + growth */
    LENIA_PHASE_ROW_FFT = 2,    /* row pass A -> row spectrum */
    LENIA_PHASE_COLUMN = 3,     /* column FFT, spectrum products, inverse */
    LENIA_PHASE_ROW_GROWTH = 4, /* inverse row pass + growth (+ next row FFT) */
    LENIA_PHASE_COLORMAP = 5,   /* field -> RGBA16F colour layer */
    LENIA_PHASE_COUNT = 8
};
typedef struct lenia_profile_data {
    uint64_t launches;                  /* kernels launched since the last read */
    uint32_t count[LENIA_PHASE_COUNT];  /* timed launches per phase */
    double ms[LENIA_PHASE_COUNT];       /* device milliseconds per phase */
} lenia_profile_data;
int lenia_profile(lenia_ctx* ctx, int enable);
int lenia_profile_read(lenia_ctx* ctx, lenia_profile_data* out);
/* Launch shapes of the spectral passes (extension; the reference has no
 * counterpart): columns per CTA of the column pass (8, 4, 2, or
 * 4 | LENIA_COLS_HALF_THREADS) and rows per
 * CTA of the inverse row pass (4, 2 or 1, | LENIA_ROWS_PIPELINED for the
 * software-pipelined variant), as the setup autotuner picked them; 0, 0 on
 * the direct path and on the runtime-plan spectral path. lenia_set_tuning
 * replaces them until the next setup (reproducible timings, or a choice
 * made under the caller's own conditions); a shape the field size cannot
 * launch, or a context without these passes, is LENIA_ERR_INVALID_ARG. */
#define LENIA_ROWS_PIPELINED 0x100
/* Columns per CTA 4 | LENIA_COLS_HALF_THREADS: the column pass with half the
 * threads per CTA, each thread taking two last-pass items. */
#define LENIA_COLS_HALF_THREADS 0x40
int lenia_get_tuning(lenia_ctx* ctx, int* cols_per_cta, int* rows_per_cta);
int lenia_set_tuning(lenia_ctx* ctx, int cols_per_cta, int rows_per_cta);
/* ---- Colour map (the module's output layer) ----
 * The field as an RGBA16F image through the module's cosine palette
 * (Shaders/Render/ColorMap.metal: t = clamp(v * input_scale + input_bias,
 * 0, 1), rgb = max(a + b cos(2 pi (c t + d)), 0) * exposure, alpha = t; v
 * the channel `channel` of the field read as (A, 0, 0, 1)). The palette is
 * the reference Lenia module's (ColorMapPass defaults with d = (0.60, 0.45,
 * 0.30), channel 0, Lenia.cpp:349-354) updated by the params' "colorMap"
 * block (ColorMapPass.cpp:70-101). */
typedef struct lenia_colormap {
    float a[3], b[3], c[3], d[3];
    float input_scale, input_bias, exposure;
    uint32_t channel;
} lenia_colormap;
int lenia_get_colormap(lenia_ctx* ctx, lenia_colormap* out);
int lenia_set_colormap(lenia_ctx* ctx, const lenia_colormap* cm);
/* The palette a params JSON object gives (host only, no device). */
int lenia_colormap_from_json(const char* params_json, lenia_colormap* out);
/* The current field's colour layer into `dst` (device, width x height
 * pixels of 4 halves, RGBA): colorMapField when the size is the field's,
 * else colorMapFieldScaled (bilinear, wrapping, at output pixel centres) --
 * the module's output at the scene resolution (Lenia.cpp:646-652).
 * Asynchronous on `stream` after the queued steps. */
int lenia_render_rgba16f(lenia_ctx* ctx, void* dst, uint32_t width, uint32_t height, void* stream);
/* lenia_step followed by lenia_render_rgba16f of the new field, with the
 * colour pass fused into the last substep where it can be (extension; the
 * reference encodes the step and then colorMapField, Lenia.cpp:562-652):
 * when width x height is the sim size, the context is on the compile-time-
 * plan spectral path and dst is 16-byte aligned, the last substep's row
 * pass writes the texels from the values it has just computed, saving the
 * colour pass's re-read of the field and its launch. Otherwise the two run
 * in turn. The texels are the same either way. */
int lenia_step_render(lenia_ctx* ctx, const lenia_frame_params* fp, uint32_t substeps, void* dst, uint32_t width,
                      uint32_t height, void* stream);

/* ---- Many worlds at once (batched sweep) ----
 * Replaces the reference's one-world-at-a-time variant loop
 * (Apps/LifePresetLab/main.cpp:718-795, a SceneRunner per variant): n
 * independent worlds of any sizes and parameters, each a single-ring Lenia
 * (the direct module's kernel, Lenia.cpp:410-446), stepped together. A
 * substep of the whole batch is either one persistent launch over a work
 * list of every world's column groups, direct tiles and row groups (where
 * every spectral world's size has a persistent body: heights 64, 128, 216,
 * 256, 512, 1024 and widths 128, 256, 384, 512, 1024), or one direct launch
 * over every direct world plus one column and one row launch per field size
 * with spectral worlds; creation times both and keeps the faster
 * (lenia_batch_launch_form). lenia_batch_step replays k substeps as one
 * captured CUDA graph. The path of
 * each world is chosen at creation: LENIA_BATCH_AUTO times the direct and
 * spectral passes on the batch's own buffers and gives each world the
 * cheaper one. Each world evolves exactly as it would alone. */
typedef struct lenia_world {
    uint32_t width, height;
    uint32_t radius;          /* kernel radius (px) */
    float mu, sigma, dt;      /* growth centre, width, time step */
    uint32_t growth_mode;     /* 0 standard, 1 asymptotic */
    uint32_t kernel_core;     /* LENIA_CORE_* */
    float shell_mu, shell_sigma; /* Gaussian shell (reference defaults 0.5, 0.15) */
    uint32_t seed;            /* reset seed: deriveSeed(seed, "LEN1") for the substep seeds */
} lenia_world;
enum { LENIA_BATCH_AUTO = 0, LENIA_BATCH_DIRECT = 1, LENIA_BATCH_FFT = 2 };
typedef struct lenia_batch lenia_batch;
int lenia_batch_create(const lenia_world* worlds, uint32_t n, uint32_t policy, lenia_batch** out);
int lenia_batch_destroy(lenia_batch* b);
/* Field of one world, height x width floats (host memory). */
int lenia_batch_upload(lenia_batch* b, uint32_t world, const float* host);
int lenia_batch_download(lenia_batch* b, uint32_t world, float* host);
/* `steps` substeps of every world (frame indices advance by one per substep,
 * seeds as the single-world module's). Asynchronous on `stream`. */
int lenia_batch_step(lenia_batch* b, uint32_t steps, void* stream);
/* Activity of every world: mean and variance of its field (n doubles each). */
int lenia_batch_stats(lenia_batch* b, double* mean, double* var);
/* LENIA_CONV_DIRECT or LENIA_CONV_FFT: the path the batch gave a world. */
int lenia_batch_world_path(lenia_batch* b, uint32_t world, uint32_t* path);
/* The reference Lenia module's noise init (leniaInit, Lenia.metal:43-61) of
 * one world on the device, from reset seed `seed` (deriveSeed(seed, "LEN1"),
 * Lenia.cpp:448-451) with initCoverage / initScale. */
int lenia_batch_init_noise(lenia_batch* b, uint32_t world, uint32_t seed, float init_coverage, float init_scale);
/* Activity of every world as the sweep runner measures it
 * (Apps/LifePresetLab/main.cpp:61-82): mean and standard deviation of the
 * luma 0.2126 R + 0.7152 G + 0.0722 B of the world's RGBA16F colour layer
 * through palette `cm` (n doubles each). */
int lenia_batch_activity(lenia_batch* b, const lenia_colormap* cm, double* mean_luma, double* stddev_luma);
/* Waits for the batch's work. LENIA_ERR_CUDA also when, in the persistent
 * form, a row group's bounded wait for its world's column groups ran out
 * (a device fault elsewhere; those rows were left unwritten). */
int lenia_batch_sync(lenia_batch* b);
const char* lenia_batch_last_message(lenia_batch* b);
/* Launch form of a substep (extension; the reference runs one variant at a
 * time): LENIA_BATCH_FORM_PERSISTENT (one launch) or
 * LENIA_BATCH_FORM_PER_SIZE, as chosen at creation (LENIA_BATCH_PERSISTENT=0/1
 * in the environment forces it). lenia_batch_set_launch_form switches it
 * (LENIA_ERR_UNSUPPORTED when some spectral size has no persistent body);
 * both forms give the same fields. */
enum { LENIA_BATCH_FORM_PER_SIZE = 0, LENIA_BATCH_FORM_PERSISTENT = 1 };
int lenia_batch_launch_form(lenia_batch* b, uint32_t* form);
int lenia_batch_set_launch_form(lenia_batch* b, uint32_t form);

/* ---- One spectral substep without device allocation ----
 * No counterpart in the reference (its module always owns its textures).
 *
 * For callers that cannot allocate device memory at the point where they
 * step the field: a real-time frame callback, where cudaMalloc/cudaFree can
 * synchronise the whole device and stall the frame, or a host application
 * that reserves the GPU's memory up front and hands out only its own
 * buffers. The caller owns the field buffers; everything else the step needs
 * (row spectrum, per-kernel potentials, kernel spectra, FFT twiddle tables)
 * lives in one static device array of LENIA_NOALLOC_SCRATCH_BYTES (8 MiB),
 * which every GPU that loads this library holds until the process exits.
 * No call allocates or frees device memory.
 *
 * field_in, field_out: distinct, 16-byte aligned device buffers of height x
 *   width floats.
 * cfg: kernels, num_kernels (0: one kernel from fp's growth mu/sigma; more
 *   than 4: the first 4, as the module's setup truncates), radius,
 *   kernel_shell_sigma, kernel_core; its other fields are unused. A zero
 *   sigma (a kernel's, or fp->growth_sigma when num_kernels is 0) is
 *   LENIA_ERR_INVALID_ARG.
 * fp: the per-frame values; seed: the substep seed (the module uses
 *   pcgHash(deriveSeed(reset_seed) ^ (frame_index*197 + substep))).
 * Sizes: even width, width/2 and height with prime factors 2, 3, 5 only, and
 *   4*W*H*(1 + K) + 4*K*(W/2+1)*(H/2+1) bytes plus small tables must fit in
 *   the array (e.g. 512x512 with 4 kernels); larger fields return
 *   LENIA_ERR_UNSUPPORTED and lenia_noalloc_last_message() says why.
 * The first call on a device, and the first call after the field size or the
 * kernel shapes change, builds the kernel spectra on the host and copies
 * them into the array synchronously on `stream`; other calls only queue
 * kernels on `stream`. All calls share the one array and each call fully
 * rewrites the parts it reads, so nothing needs clearing, but calls that
 * overlap on the GPU (other streams or host threads) race on it. A
 * cudaDeviceReset discards the array with the context; calls after one are
 * not supported (the tables are rebuilt only if the array's device address
 * changed). Host-side failures, an allocation of the host tables included,
 * return a status; no C++ exception leaves the call. */
#define LENIA_NOALLOC_SCRATCH_BYTES (8u * 1024u * 1024u)
int lenia_fft_step_noalloc(const float* field_in, float* field_out, uint32_t width, uint32_t height,
                           const lenia_config* cfg, const lenia_frame_params* fp, uint32_t seed,
                           void* stream);
/* Message of the calling thread's last failed lenia_fft_step_noalloc. */
const char* lenia_noalloc_last_message(void);

/* ---- Gradient of a rollout (adjoint of the spectral step) ----
 * No counterpart in the reference (it only steps forward). A batch of worlds
 * of one size shares one set of kernels and growth parameters; each world has
 * its own initial field. lenia_adjoint_forward runs T spectral steps of the
 * reference's multi-kernel update (Lenia.metal:188-231 without noise, mu
 * jitter or injection) from A_0 to A_T and keeps A every `checkpoint_every`
 * steps; lenia_adjoint_backward takes dL/dA_T and returns dL/dA_0 and dL/d of
 * every scalar parameter, recomputing each segment between checkpoints
 * (checkpointed backpropagation through time). The backward of a step is
 * hand-written: clip mask (subgradient 1 strictly inside (0, 1), 0 on or
 * outside), growth derivative, and the adjoint convolution as spectrum
 * products between forward and inverse FFTs.
 *
 * Kernels are built in FP64 ring by ring (buildRingKernelImage's formula,
 * Lenia.cpp:95-125): K_k = sum_i beta_i R_i / sum_i beta_i sum(R_i).
 * Sizes: the compile-time FFT sizes of the spectral path (height and width/2
 * in 64, 128, 192(width only), 256, 512, 960(width only), 1024(height),
 * 1080(height), 2048, 4096(height); e.g. 512x512, 1920x1080). */
typedef struct lenia_adjoint_config {
    uint32_t width, height;
    uint32_t batch;             /* worlds */
    uint32_t radius;            /* R (px); kernel k has radius R * radius_scale */
    uint32_t kernel_core;       /* LENIA_CORE_* */
    float shell_sigma;          /* Gaussian shell width (LENIA_CORE_GAUSS_SHELL) */
    uint32_t growth_mode;       /* 0 standard, 1 asymptotic */
    float dt;
    uint32_t num_kernels;       /* 1..4 */
    lenia_kernel_def kernels[4];
    uint32_t steps;             /* T >= 1 */
    uint32_t checkpoint_every;  /* 1..T */
} lenia_adjoint_config;
typedef struct lenia_adjoint lenia_adjoint;
/* Parameter gradient layout (doubles): kernel k at k * 11 + {0: mu,
 * 1: sigma, 2: weight, 3..10: betas[0..7]}, then dt at index 44. */
#define LENIA_ADJOINT_PARAMS_PER_KERNEL 11
#define LENIA_ADJOINT_NUM_PARAMS 45
int lenia_adjoint_create(const lenia_adjoint_config* cfg, lenia_adjoint** out);
int lenia_adjoint_destroy(lenia_adjoint* a);
/* New parameter values (same num_kernels and num_betas per kernel; radius
 * scales and the core stay). Takes effect for the next forward. */
int lenia_adjoint_set_params(lenia_adjoint* a, const lenia_kernel_def* kernels, uint32_t num_kernels,
                             float dt);
/* a0: batch x height x width floats (device); a_final receives A_T (device).
 * Asynchronous on `stream` (NULL: the context's stream). */
int lenia_adjoint_forward(lenia_adjoint* a, const float* a0, float* a_final, void* stream);
/* After lenia_adjoint_forward (same parameters): g_final = dL/dA_T (device,
 * batch x height x width); g_initial receives dL/dA_0 (device, may alias
 * g_final); grad_params, if not NULL, receives LENIA_ADJOINT_NUM_PARAMS
 * doubles (device), summed over the batch. Asynchronous on `stream`. */
int lenia_adjoint_backward(lenia_adjoint* a, const float* g_final, float* g_initial, double* grad_params,
                           void* stream);
/* Device memory held, and launches issued since creation. */
int lenia_adjoint_stats(lenia_adjoint* a, uint64_t* device_bytes, uint64_t* launches);
const char* lenia_adjoint_last_message(lenia_adjoint* a);


/* ---- State files (.npy) ----
 * NumPy .npy v1.0, float32, C order (LifeCore/IO/NpyWriter.h:15-31): the
 * reference's state exchange format. Reading requires the caller's shape:
 * the payload is sized from it, never from the file, and a bad magic, a
 * truncated header or payload, another dtype, a Fortran-order array or a
 * different shape is an error (LENIA_ERR_PARSE; nothing is written to `out`
 * beyond a complete read). Host only. lenia_last_message(NULL) says why a
 * call on this thread failed. */
int lenia_npy_write_f32(const char* path, const float* data, size_t count, const uint32_t* shape, uint32_t ndim);
int lenia_npy_read_f32(const char* path, const uint32_t* shape, uint32_t ndim, float* out, size_t count);
/* The field as (sim_height, sim_width) float32 (SimulationModule::dumpState /
 * loadState, LifeCore/Sim/SimulationModule.h:48-78). Loading replaces the
 * field and counts as the init (the next encode does not re-initialise). */
int lenia_save_state(lenia_ctx* ctx, const char* path);
int lenia_load_state(lenia_ctx* ctx, const char* path);

/* ---- Parameter bus and scenes ----
 * The reference's ParameterBus (LifeCore/Params/ParameterBus.{h,cpp}) and
 * scene loader (LifeCore/Params/Scene.cpp): a table of "<module>.<param>"
 * values that a context reads its per-frame parameters from. Final value:
 * the override if set, else ((set ?: base) + sum of adds) * product of muls,
 * where the set/add/mul terms come from the mappings evaluated by the last
 * lenia_bus_update. A context has its own bus unless one is attached; a
 * scene's modules share one (SceneRunner, LifeCore/Sim/SceneRunner.cpp). The
 * bus is host-side only (no device work). */
typedef struct lenia_bus lenia_bus;
enum { LENIA_MAP_ADD = 0, LENIA_MAP_SET = 1, LENIA_MAP_MUL = 2 };
/* One mapping (AudioMappingSpec, ParameterBus.h:44-99). source: an input
 * name (see lenia_bus_set_feature) or a time source
 * "time.<sin|tri|ramp|noise>:<period s>[@<phase 0..1>]". in_max > in_min
 * normalises the source to 0..1 first; then v * scale + offset, smoothed
 * with time constant `smoothing` s (0: none), contributed to `target` in
 * `mode` (LENIA_MAP_*). */
typedef struct lenia_mapping {
    const char* source;
    const char* target;
    float in_min, in_max;
    float scale, offset;
    float smoothing;
    uint32_t mode;
} lenia_mapping;
typedef struct lenia_scene_info {
    uint32_t seed, width, height;   /* "seed", "resolution" (1234, 1920x1080) */
    uint32_t num_modules, num_mappings;
} lenia_scene_info;
int lenia_bus_create(uint32_t seed, lenia_bus** out);
int lenia_bus_destroy(lenia_bus* bus);
/* Scene::parse + applyBaseParams (Scene.cpp:24-113): the scene's seed,
 * every module's numeric/boolean params as "<name>.<key>" bases, and the
 * mappings of "audioMappings", "musicMappings" and "automation". A malformed
 * time source fails the load (LENIA_ERR_PARSE), as in the reference. */
int lenia_bus_load_scene(lenia_bus* bus, const char* scene_json, lenia_scene_info* info);
int lenia_bus_add_mapping(lenia_bus* bus, const lenia_mapping* mapping);
int lenia_bus_set_base(lenia_bus* bus, const char* key, float value);
int lenia_bus_set_override(lenia_bus* bus, const char* key, float value);
int lenia_bus_clear_override(lenia_bus* bus, const char* key);
/* This frame's input values, by the reference's source names: audio
 * channels kick/snare/hihat/perc/beat (".raw", ".smoothed", ".peak",
 * ".trigger", ".hold"; the bare name is ".smoothed"), rms, low, mid, high,
 * centroid, flux, time; "lane.<name>"; "section.energy", "section.progress",
 * "section.changed"; events as "event:<type>.active" (1 while it runs),
 * ".started", ".ended", ".progress" and its own curves "event:<type>.<curve>"
 * (which have no value while the event does not run). Unset names read 0.
 * Values persist until changed or cleared. */
int lenia_bus_set_feature(lenia_bus* bus, const char* name, float value);
/* The current section's role and index ("section.is:<role>", "section.n:<k>"). */
int lenia_bus_set_section(lenia_bus* bus, const char* role, int32_t index);
int lenia_bus_clear_features(lenia_bus* bus);
/* ParameterBus::update (ParameterBus.cpp:267-343): evaluates every mapping
 * and advances the bus clock (the time sources' input) by dt seconds. */
int lenia_bus_update(lenia_bus* bus, float dt);
/* param(ctx, key, fallback) for a full key ("lenia0.growthMu"). */
int lenia_bus_value(lenia_bus* bus, const char* key, float fallback, float* out);
const char* lenia_bus_last_message(lenia_bus* bus);
/* The Lenia module of a scene document: the module named `module_name` (NULL:
 * the first of type "Lenia"), set up from its params at the scene's
 * resolution, its instance name the module's name. With `bus` (loaded from
 * the same scene by lenia_bus_load_scene) the context reads that bus, which
 * must outlive it; with NULL it gets its own bus loaded from the scene. */
int lenia_create_scene_module(const char* scene_json, const char* module_name, lenia_bus* bus,
                              const char* base_dir, lenia_ctx** out);
/* Reads per-frame parameters from `bus` from now on (NULL: the context's own
 * bus again). The bus must outlive the attachment. */
int lenia_attach_bus(lenia_ctx* ctx, lenia_bus* bus);

/* ---- Device characterisation ----
 * The FP32 fused multiply-add peak of the current device, measured: 8
 * independent FMA chains per thread, 8 CTAs of 256 threads per SM, best of
 * `reps` timed launches (CUDA events on `stream`) of a scalar-FFMA kernel and
 * of a packed-FFMA2 kernel, in TFLOP/s (2 FLOP per FMA). The denominator of
 * the direct path's FLOP/s roofline. No counterpart in the reference. */
int lenia_fp32_peak(int reps, double* tflops_ffma, double* tflops_ffma2, void* stream);

/* Message of the last warning or error on this context ("" if none). */
const char* lenia_last_message(lenia_ctx* ctx);
const char* lenia_status_string(int status);

#ifdef __cplusplus
}
#endif
#endif /* LENIA_B200_H */
