// life_simulation_b200/csrc/lenia_module.h -- host-side mirror of the
// reference's Lenia module (Modules/FieldModules/Lenia.h:50-196) on the
// module lifecycle of LifeCore/Sim/SimulationModule.h:39-128
// (configure -> setup -> reset -> per frame updateCPU + encode -> outputField),
// driving the CUDA kernels of this library instead of Metal passes.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/lenia_b200.h"
#include "json_lite.h"
#include "lenia_kernels.h"
#include "lenia_types.h"
#include "param_bus.h"

namespace lenia {

struct KernelDef {  // Lenia.h:99-105
    float radius_scale = 1.0f;
    float mu = 0.15f;
    float sigma = 0.017f;
    float weight = 1.0f;
    std::vector<float> betas{1.0f};
};

struct OrganismData {  // Lenia.cpp:137-145
    float R = 13.0f, T = 10.0f, mu = 0.15f, sigma = 0.015f;
    uint32_t width = 0, height = 0;
    std::vector<float> cells;
};

// Everything setup() reads, after parsing (C struct or JSON).
// The Lenia module's palette: ColorMapParams defaults
// (LifeCore/Render/ColorMapPass.h:13-23) with Lenia's phases, channel and
// scale (Lenia.cpp:349-354), then the params' "colorMap" block.
ColorMapParams lenia_default_colormap();
// ColorMapPass::configure's "colorMap" block (LifeCore/Render/ColorMapPass.cpp:
// 70-101): "palette": "mono", "a"/"b"/"c"/"d" (3 numbers), "inputScale",
// "inputBias", "exposure", "channel".
void colormap_from_json(const Json& params, ColorMapParams& cm);

struct ModuleConfig {
    ColorMapParams colormap = lenia_default_colormap();
    uint32_t sim_width = 0, sim_height = 0;
    uint32_t conv_mode = LENIA_CONV_DIRECT;
    bool fft_any_size = false;
    uint32_t fft_precision = LENIA_FFT_FP32;  // fftPrecision (extension)
    bool has_radius = false;
    uint32_t radius = 13;
    bool has_kernels = false;
    std::vector<KernelDef> kernels;
    uint32_t kernel_core = LENIA_CORE_GAUSS_SHELL;
    float shell_mu = 0.5f, shell_sigma = 0.15f;
    float init_coverage = 0.4f, init_scale = 24.0f;
    bool want_stamp = false;
    bool has_organism_path = false;  // "organism" named (loaded or not)
    bool organism_loaded = false;
    OrganismData organism;
    std::string organism_error;
    uint32_t stamp_count = 6;
    bool stamp_rotate = true;
    bool use_organism_params = true;
    std::vector<std::string> warnings;  // produced while parsing
};

class LeniaModule {
public:
    LeniaModule();
    ~LeniaModule();
    LeniaModule(const LeniaModule&) = delete;
    LeniaModule& operator=(const LeniaModule&) = delete;

    // SimulationModule::configure (SimulationModule.h:112-115).
    void configure(std::string instance, ModuleConfig cfg) {
        instance_ = std::move(instance);
        cfg_ = std::move(cfg);
        colormap_ = cfg_.colormap;
    }
    // LeniaModule::setup (Lenia.cpp:208-408). Returns LENIA_OK,
    // LENIA_WARN_FALLBACK, or an error.
    int setup(uint32_t scene_w, uint32_t scene_h);
    // The host half of setup (sizes, paths, fallbacks, radius) without any
    // device work; setup() calls it first.
    int resolve(uint32_t scene_w, uint32_t scene_h);
    // LeniaModule::reset (Lenia.cpp:448-451).
    void reset(uint32_t seed);
    // LeniaModule::updateCPU (Lenia.cpp:453): only the frame index of the
    // audio state reaches the kernels (AudioUniforms::frameIndex).
    void updateCPU(uint32_t audio_frame) { audio_frame_ = audio_frame; }
    // LeniaModule::encode (Lenia.cpp:455-644) with per-frame values read
    // from `params` (param(ctx, key, fallback)).
    int encode(uint32_t frame_index, uint32_t substeps, const ParameterBus& params,
               cudaStream_t stream);
    // encode with explicit per-frame values.
    int step(const lenia_frame_params& fp, uint32_t substeps, cudaStream_t stream);
    // step, then the colour layer of the new field into a dst_w x dst_h
    // RGBA16F buffer. At the sim size on the compile-time-plan spectral path
    // the last substep's row pass writes it (no separate colour pass); other
    // sizes and paths run render() after the step. Same texels either way.
    int stepRender(const lenia_frame_params& fp, uint32_t substeps, void* rgba16f, uint32_t dst_w, uint32_t dst_h,
                   cudaStream_t stream);
    // Per-frame values as encode would read them (Lenia.cpp:456-464).
    lenia_frame_params resolveFrameParams(const ParameterBus& params, uint32_t frame_index,
                                          uint32_t audio_frame) const;

    // outputField (Lenia.h:63): the current state buffer on the device.
    const float* outputField() const { return field_[cur_]; }
    float* mutableField() { return field_[cur_]; }
    void fieldWritten() {
        needs_field_init_ = false;
        spectrum_valid_ = false;
    }
    uint32_t width() const { return w_; }
    uint32_t height() const { return h_; }
    void info(lenia_info* out) const;
    const std::string& message() const { return message_; }
    const std::string& instance() const { return instance_; }
    const ColorMapParams& colormap() const { return colormap_; }
    void setColormap(const ColorMapParams& cm) { colormap_ = cm; }
    // The colour map of the current field into a dst_w x dst_h RGBA16F
    // device buffer (the module's outputField, Lenia.cpp:646-652).
    int render(void* rgba16f, uint32_t dst_w, uint32_t dst_h, cudaStream_t stream);
    void setMessage(std::string m) { message_ = std::move(m); }
    cudaStream_t stream() const { return stream_; }

    // Launch shapes of the compile-time-plan spectral passes (columns and
    // rows per CTA; 0, 0 when the context does not use them).
    void tuning(int* cols, int* rows) const;
    int setTuning(int cols, int rows);

    // Per-launch event timing (GPUTimer's role, LifeCore/Metal/GPUTimer.h).
    void setProfiling(bool on);
    // Device-side failures recorded by the kernels (read after a sync):
    // LENIA_OK, or an error with its message.
    int checkDeviceFlags();
    bool directTma() const { return direct_tma_.on; }
    int readProfile(lenia_profile_data* out);

private:
    // Launches `fn` as one kernel of `phase`, counted and, when profiling,
    // bracketed by CUDA events on stream `s`.
    template <typename F>
    cudaError_t launch(int phase, cudaStream_t s, F&& fn);
    cudaEvent_t takeEvent();
    int fail(int code, const std::string& what);
    int cudaFail(cudaError_t e, const char* where);
    int buildDirectTables();
    int buildSpectralTables(const std::vector<KernelDef>& eff);
    int autotuneSpectral();
    // The tensor-core column pass: kTcgen05, or mma.sync at `choice` columns per CTA.
    cudaError_t launchColumnTc(int choice, const float2* S, float2* U, cudaStream_t s);
    int stepImpl(const lenia_frame_params& fp, uint32_t substeps, cudaStream_t stream, void* rgba16f);
    int initField(const lenia_frame_params& fp, cudaStream_t s);
    int initKernels(const lenia_frame_params& fp);
    void fillStepParams(const lenia_frame_params& fp, uint32_t seed, StepParams& p) const;
    void release();

    std::string instance_ = "lenia0";
    ColorMapParams colormap_ = lenia_default_colormap();
    ModuleConfig cfg_;
    std::string message_;
    std::vector<std::string> warnings_;

    // Resolved at setup.
    uint32_t w_ = 0, h_ = 0;
    bool use_fft_ = false, direct_multi_ = false, use_stamp_ = false;
    uint32_t radius_ = 13;
    float fallback_mu_ = 0.15f, fallback_sigma_ = 0.017f, fallback_dt_ = 0.1f;
    std::vector<KernelDef> kernels_;
    std::vector<float> direct_lut_;  // reference LUT, direct mode

    // Runtime state.
    uint32_t seed_ = 0;
    uint32_t audio_frame_ = 0;
    bool needs_field_init_ = true;
    bool needs_kernel_init_ = true;
    bool spectrum_valid_ = false;
    int cur_ = 0;
    int device_ = 0;
    cudaStream_t stream_ = nullptr;

    // Multi-kernel growth parameters fixed at init (Lenia.cpp:503-545).
    uint32_t num_k_ = 1;
    float k_mu_[kMaxKernels] = {0.15f, 0.15f, 0.15f, 0.15f};
    float k_sigma_[kMaxKernels] = {0.017f, 0.017f, 0.017f, 0.017f};
    float k_weight_[kMaxKernels] = {1.0f, 0.0f, 0.0f, 0.0f};

    // Device resources.
    float* field_[2] = {nullptr, nullptr};
    DirectTma direct_tma_;          // halo-tile tensor maps of field_[0], field_[1]
    int* d_tma_err_ = nullptr;      // halo loads (direct) or MMA waits (tcgen05 column pass) that ran out
    float* d_weights_ = nullptr;
    uint32_t* d_spans_ = nullptr;
    float* d_org_ = nullptr;
    float2* d_S_ = nullptr;
    float2* d_U_ = nullptr;
    float* d_khat_ = nullptr;
    float2* d_tw_row_ = nullptr;
    float2* d_tw_col_ = nullptr;
    float2* d_tw_r2c_ = nullptr;
    uint64_t device_bytes_ = 0;
    DirectGeometry dgeo_{};
    int direct_tile_ = kDirectTile64x16;
    int direct_nk_ = 1;
    int direct_split_ = 1;  // kernel-row thread groups per tile (small fields)
    int direct_ox_ = 8;     // outputs per thread (16: large tiles, when faster)
    int direct_oy_ = 1;     // output rows per thread (2: large tiles, when faster)
    uint32_t direct_taps_ = 0;  // nonzero taps over the direct path's kernels
    FftGeometry fgeo_{};
    bool fast_col_ = false, fast_row_ = false;  // compile-time-plan passes
    int col_batch_ = 2, row_batch_ = 2;         // autotuned per size
    uint32_t tc_precision_ = LENIA_FFT_FP32;    // column DFT stages on the tensor cores
    int tc_batch_ = 2;
    FastTables fast_{};
    float2* d_fast_tw_[4] = {nullptr, nullptr, nullptr, nullptr};

    // Launch accounting and profiling.
    uint64_t launches_ = 0;
    bool profiling_ = false;
    struct TimedLaunch {
        int phase;
        cudaEvent_t start, stop;
    };
    std::vector<TimedLaunch> timed_;
    std::vector<cudaEvent_t> event_pool_;
};

// Parsing of the scene "params" object (Lenia.cpp:208-357) and of the C
// struct into ModuleConfig.
int config_from_json(const Json& params, const std::string& base_dir, ModuleConfig& out,
                     std::string& error);
int config_from_struct(const lenia_config& c, ModuleConfig& out, std::string& error);

// Host-side kernel construction shared with the batched form.
void build_direct_lut(uint32_t radius, float shell_mu, float shell_sigma, uint32_t core,
                      std::vector<float>& out);
void build_ring_image(uint32_t w, uint32_t h, float radius_k, float shell_sigma,
                      const std::vector<float>& betas, uint32_t core, std::vector<float>& out);
bool fft_plan(int n, FftPlan& plan);
void fill_twiddles(int n, std::vector<float2>& tw);
// Real even spectrum of a wrap-centred kernel image, divided by (w*h):
// out[kx * (h/2+1) + ky], kx <= w/2, ky <= h/2 (FP64, rounded once).
void kernel_spectrum(const std::vector<float>& img, uint32_t w, uint32_t h,
                     std::vector<float>& out);
// The same spectrum unnormalised and unrounded, of an FP64 image.
void even_spectrum_f64(const std::vector<double>& img, uint32_t w, uint32_t h, std::vector<double>& out);
// The rings of a kernel separately, FP64, peak 1 each, unnormalised
// (buildRingKernelImage's terms, Lenia.cpp:95-125).
void ring_shells_f64(uint32_t w, uint32_t h, double radius_k, double shell_sigma, uint32_t nshell,
                     uint32_t core, std::vector<std::vector<double>>& rings);
uint32_t pcg_hash_host(uint32_t v);
uint32_t derive_seed(uint32_t global_seed, uint32_t tag);

}  // namespace lenia
