// life_simulation_b200/csrc/lenia_module.cpp -- host logic of the Lenia
// module: parameter parsing and fallbacks (Lenia.cpp:208-357), kernel
// construction (Lenia.cpp:95-125, :410-446), seeds (Lenia.cpp:448-451,
// :564), the encode loop (Lenia.cpp:455-644), and the device resources the
// kernels need (the ResourcePool role of LifeCore/Metal/ResourcePool.h).
#include "lenia_module.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace lenia {

// ------------------------------------------------------------- utilities

uint32_t pcg_hash_host(uint32_t v) {  // LifeCore/Math/Random.h:34-38
    uint32_t state = v * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

uint32_t derive_seed(uint32_t global_seed, uint32_t tag) {  // Random.h:42-44
    return pcg_hash_host(global_seed ^ pcg_hash_host(tag));
}

static bool is_pow2(uint32_t v) { return v != 0 && (v & (v - 1u)) == 0; }

// -------------------------------------------------- kernel construction

static double exp_core(double r) {
    if (!(r > 0.0 && r < 1.0)) return 0.0;
    return std::exp(4.0 - 1.0 / (r * (1.0 - r)));
}

// buildKernelTexture, Lenia.cpp:410-446 (Gaussian shell: float arithmetic,
// double sum, float(1/sum) scale, exactly as the reference). The
// exponential core is evaluated and normalised in FP64 and rounded once.
void build_direct_lut(uint32_t R, float shell_mu, float shell_sigma, uint32_t core,
                      std::vector<float>& out) {
    const uint32_t size = 2 * R + 1;
    out.assign(size_t(size) * size, 0.0f);
    double sum = 0.0;
    if (core == LENIA_CORE_EXP) {
        std::vector<double> tmp(out.size(), 0.0);
        for (uint32_t y = 0; y < size; ++y)
            for (uint32_t x = 0; x < size; ++x) {
                double dx = double(int(x) - int(R)), dy = double(int(y) - int(R));
                double r = R ? std::sqrt(dx * dx + dy * dy) / double(R) : 0.0;
                tmp[size_t(y) * size + x] = exp_core(r);
                sum += tmp[size_t(y) * size + x];
            }
        for (size_t i = 0; i < out.size(); ++i) out[i] = sum > 0.0 ? float(tmp[i] / sum) : 0.0f;
        return;
    }
    for (uint32_t y = 0; y < size; ++y)
        for (uint32_t x = 0; x < size; ++x) {
            float dx = float(int(x) - int(R));
            float dy = float(int(y) - int(R));
            float r = std::sqrt(dx * dx + dy * dy) / float(R);
            float w = 0.0f;
            if (r <= 1.0f && r > 0.0f) {
                float t = (r - shell_mu) / shell_sigma;
                w = std::exp(-0.5f * t * t);
            }
            out[size_t(y) * size + x] = w;
            sum += w;
        }
    if (sum > 0.0) {
        float inv = float(1.0 / sum);
        for (auto& w : out) w *= inv;
    }
}

// buildRingKernelImage, Lenia.cpp:95-125: w x h image, kernel centred at
// (0,0) and wrapped; B shells; float arithmetic with a double sum for the
// Gaussian shell, FP64 for the exponential core.
void build_ring_image(uint32_t w, uint32_t h, float radius_k, float shell_sigma,
                      const std::vector<float>& betas, uint32_t core, std::vector<float>& out) {
    out.assign(size_t(w) * h, 0.0f);
    if (betas.empty() || radius_k <= 0.0f) return;
    const uint32_t B = uint32_t(betas.size());
    const float Bf = float(B);
    double sum = 0.0;
    if (core == LENIA_CORE_EXP) {
        std::vector<double> tmp(out.size(), 0.0);
        for (uint32_t y = 0; y < h; ++y) {
            int dy = int(y);
            if (dy > int(h / 2)) dy -= int(h);
            for (uint32_t x = 0; x < w; ++x) {
                int dx = int(x);
                if (dx > int(w / 2)) dx -= int(w);
                double r = std::sqrt(double(dx) * dx + double(dy) * dy);
                double v = 0.0;
                if (r > 0.0 && r <= double(radius_k)) {
                    double u = (r / double(radius_k)) * double(B);
                    uint32_t i = std::min<uint32_t>(uint32_t(u), B - 1);
                    v = double(betas[i]) * exp_core(u - double(i));
                }
                tmp[size_t(y) * w + x] = v;
                sum += v;
            }
        }
        for (size_t i = 0; i < out.size(); ++i) out[i] = sum > 0.0 ? float(tmp[i] / sum) : 0.0f;
        return;
    }
    for (uint32_t y = 0; y < h; ++y) {
        int dy = int(y);
        if (dy > int(h / 2)) dy -= int(h);
        for (uint32_t x = 0; x < w; ++x) {
            int dx = int(x);
            if (dx > int(w / 2)) dx -= int(w);
            float r = std::sqrt(float(dx) * float(dx) + float(dy) * float(dy));
            float v = 0.0f;
            if (r > 0.0f && r <= radius_k) {
                float u = (r / radius_k) * Bf;
                uint32_t i = std::min<uint32_t>(uint32_t(u), B - 1);
                float t = (u - float(i) - 0.5f) / (shell_sigma * Bf);
                v = betas[i] * std::exp(-0.5f * t * t);
            }
            out[size_t(y) * w + x] = v;
            sum += v;
        }
    }
    if (sum > 0.0) {
        float inv = float(1.0 / sum);
        for (auto& v : out) v *= inv;
    }
}

// Ring by ring in FP64: the terms of buildRingKernelImage (Lenia.cpp:95-125)
// with peak 1 each, unnormalised (the kernel is sum_i beta_i R_i over
// sum_i beta_i sum(R_i)). The gradient form needs the rings separately.
void ring_shells_f64(uint32_t w, uint32_t h, double radius_k, double shell_sigma, uint32_t nshell,
                     uint32_t core, std::vector<std::vector<double>>& rings) {
    rings.assign(nshell, std::vector<double>(size_t(w) * h, 0.0));
    if (nshell == 0 || radius_k <= 0.0) return;
    for (uint32_t y = 0; y < h; ++y) {
        int dy = int(y);
        if (dy > int(h / 2)) dy -= int(h);
        for (uint32_t x = 0; x < w; ++x) {
            int dx = int(x);
            if (dx > int(w / 2)) dx -= int(w);
            const double r = std::sqrt(double(dx) * dx + double(dy) * dy);
            if (!(r > 0.0 && r <= radius_k)) continue;
            const double u = r / radius_k * double(nshell);
            const uint32_t i = std::min<uint32_t>(uint32_t(u), nshell - 1);
            double v;
            if (core == LENIA_CORE_EXP) {
                v = exp_core(u - double(i));
            } else {
                const double t = (u - double(i) - 0.5) / (shell_sigma * double(nshell));
                v = std::exp(-0.5 * t * t);
            }
            rings[i][size_t(y) * w + x] = v;
        }
    }
}

// The kernel image is real and even in x and y separately (it depends on
// dx^2 + dy^2 over offsets that are symmetric on the torus), so its DFT is
// real: K^(kx, ky) = sum K[y][x] cos(2 pi kx x / w) cos(2 pi ky y / h),
// evaluated in FP64 over the nonzero taps, separably.
template <typename T>
static void even_spectrum(const std::vector<T>& img, uint32_t w, uint32_t h, std::vector<double>& out) {
    const uint32_t M1 = w / 2 + 1, Hh = h / 2 + 1;
    std::vector<double> cw(w), ch(h);
    for (uint32_t m = 0; m < w; ++m) cw[m] = std::cos(2.0 * M_PI * double(m) / double(w));
    for (uint32_t m = 0; m < h; ++m) ch[m] = std::cos(2.0 * M_PI * double(m) / double(h));
    std::vector<uint32_t> rows;
    std::vector<std::vector<std::pair<uint32_t, double>>> taps;
    for (uint32_t y = 0; y < h; ++y) {
        std::vector<std::pair<uint32_t, double>> t;
        for (uint32_t x = 0; x < w; ++x)
            if (img[size_t(y) * w + x] != T(0)) t.emplace_back(x, double(img[size_t(y) * w + x]));
        if (!t.empty()) {
            rows.push_back(y);
            taps.push_back(std::move(t));
        }
    }
    std::vector<double> rowsum(rows.size() * M1, 0.0);
    for (size_t i = 0; i < rows.size(); ++i)
        for (uint32_t kx = 0; kx < M1; ++kx) {
            double s = 0.0;
            for (const auto& t : taps[i]) s += t.second * cw[(uint64_t(kx) * t.first) % w];
            rowsum[i * M1 + kx] = s;
        }
    out.assign(size_t(M1) * Hh, 0.0);
    for (uint32_t kx = 0; kx < M1; ++kx)
        for (uint32_t ky = 0; ky < Hh; ++ky) {
            double s = 0.0;
            for (size_t i = 0; i < rows.size(); ++i) s += rowsum[i * M1 + kx] * ch[(uint64_t(ky) * rows[i]) % h];
            out[size_t(kx) * Hh + ky] = s;
        }
}

void even_spectrum_f64(const std::vector<double>& img, uint32_t w, uint32_t h, std::vector<double>& out) {
    even_spectrum(img, w, h, out);
}

// Divided by w*h (the inverse transforms of the spectral path are
// unnormalised) and rounded once.
void kernel_spectrum(const std::vector<float>& img, uint32_t w, uint32_t h,
                     std::vector<float>& out) {
    std::vector<double> d;
    even_spectrum(img, w, h, d);
    const double norm = 1.0 / (double(w) * double(h));
    out.resize(d.size());
    for (size_t i = 0; i < d.size(); ++i) out[i] = float(d[i] * norm);
}

bool fft_plan(int n, FftPlan& plan) {
    plan.n = n;
    plan.npass = 0;
    if (n < 1) return false;
    int m = n;
    auto push = [&](int r) {
        if (plan.npass >= kMaxPasses) return false;
        plan.radix[plan.npass++] = r;
        return true;
    };
    while (m % 16 == 0) { if (!push(16)) return false; m /= 16; }
    if (m % 8 == 0) { if (!push(8)) return false; m /= 8; }
    if (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
    if (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
    while (m % 5 == 0) { if (!push(5)) return false; m /= 5; }
    while (m % 3 == 0) { if (!push(3)) return false; m /= 3; }
    return m == 1;
}

void fill_twiddles(int n, std::vector<float2>& tw) {
    tw.resize(size_t(n));
    for (int t = 0; t < n; ++t) {
        const double a = 2.0 * M_PI * double(t) / double(n);
        tw[size_t(t)] = make_float2(float(std::cos(a)), float(-std::sin(a)));
    }
}

// ------------------------------------------------------------- parsing

static bool load_organism_file(const std::string& path, OrganismData& out, std::string& err) {
    // loadOrganismJSON, Lenia.cpp:151-204.
    std::ifstream f(path);
    if (!f) {
        err = "cannot open organism file: " + path;
        return false;
    }
    std::stringstream ss;
    ss << f.rdbuf();
    std::string perr;
    Json j = Json::parse(ss.str(), &perr);
    if (!perr.empty()) {
        err = "organism JSON parse error: " + perr;
        return false;
    }
    const Json* cells = j.find("cells");
    if (!cells || !cells->is_array() || cells->size() == 0) {
        err = "organism JSON missing non-empty \"cells\" array";
        return false;
    }
    const auto& rows = cells->items();
    if (!rows[0].is_array() || rows[0].size() == 0) {
        err = "organism JSON \"cells\" rows must be non-empty arrays";
        return false;
    }
    const size_t cols = rows[0].size();
    out.cells.clear();
    out.cells.reserve(rows.size() * cols);
    for (size_t r = 0; r < rows.size(); ++r) {
        if (!rows[r].is_array() || rows[r].size() != cols) {
            err = "organism JSON \"cells\" row " + std::to_string(r) + " length mismatch (expected " +
                  std::to_string(cols) + " columns)";
            return false;
        }
        for (size_t c = 0; c < cols; ++c) {
            const Json& v = rows[r].items()[c];
            float fv = v.is_number() ? float(v.as_number()) : 0.0f;
            if (!v.is_number() || fv < 0.0f || fv > 1.0f) {
                err = "organism JSON cell value out of [0,1] at row " + std::to_string(r) + " col " +
                      std::to_string(c);
                return false;
            }
            out.cells.push_back(fv);
        }
    }
    out.R = j.value_float("R", 13.0f);
    out.T = j.value_float("T", 10.0f);
    out.mu = j.value_float("mu", 0.15f);
    out.sigma = j.value_float("sigma", 0.015f);
    out.width = uint32_t(cols);
    out.height = uint32_t(rows.size());
    return true;
}

ColorMapParams lenia_default_colormap() {
    ColorMapParams cm{};
    for (int i = 0; i < 3; ++i) {
        cm.a[i] = 0.5f;
        cm.b[i] = 0.5f;
        cm.c[i] = 1.0f;
    }
    cm.d[0] = 0.60f;
    cm.d[1] = 0.45f;
    cm.d[2] = 0.30f;
    cm.input_scale = 1.0f;
    cm.input_bias = 0.0f;
    cm.exposure = 1.0f;
    cm.channel = 0;
    return cm;
}

void colormap_from_json(const Json& params, ColorMapParams& cm) {
    const Json* j = params.find("colorMap");
    if (!j || !j->is_object()) return;
    if (j->value_string("palette", "") == "mono") {  // black (t = 0) to white (t = 1)
        for (int i = 0; i < 3; ++i) cm.a[i] = cm.b[i] = cm.c[i] = cm.d[i] = 0.5f;
    }
    const auto vec3 = [&](const char* key, float* v) {
        const Json* a = j->find(key);
        if (a && a->is_array() && a->size() >= 3)
            for (int i = 0; i < 3; ++i) v[i] = float(a->items()[size_t(i)].as_number());
    };
    vec3("a", cm.a);
    vec3("b", cm.b);
    vec3("c", cm.c);
    vec3("d", cm.d);
    cm.input_scale = j->value_float("inputScale", cm.input_scale);
    cm.input_bias = j->value_float("inputBias", cm.input_bias);
    cm.exposure = j->value_float("exposure", cm.exposure);
    cm.channel = j->value_u32("channel", cm.channel);
}

int config_from_json(const Json& p, const std::string& base_dir, ModuleConfig& c,
                     std::string& error) {
    if (!p.is_object()) {
        error = "params must be a JSON object";
        return LENIA_ERR_PARSE;
    }
    c = ModuleConfig();
    c.sim_width = p.value_u32("simWidth", 0u);
    c.sim_height = p.value_u32("simHeight", 0u);
    const std::string conv = p.value_string("convMode", "direct");
    c.conv_mode = conv == "fft" ? LENIA_CONV_FFT
                  : conv == "directMulti" ? LENIA_CONV_DIRECT_MULTI
                                          : LENIA_CONV_DIRECT;
    c.fft_any_size = p.value_bool("fftAnySize", false);
    colormap_from_json(p, c.colormap);
    const std::string prec = p.value_string("fftPrecision", "fp32");
    if (prec == "bf16x3") {
        c.fft_precision = LENIA_FFT_BF16X3;
    } else if (prec == "fp16x3") {
        c.fft_precision = LENIA_FFT_FP16X3;
    } else if (prec != "fp32") {
        c.warnings.push_back("\"fftPrecision\" must be \"fp32\", \"bf16x3\" or \"fp16x3\" (got \"" + prec +
                             "\"); using \"fp32\"");
    }
    if (p.contains("radius")) {
        c.has_radius = true;
        c.radius = p.value_u32("radius", 13u);
    }
    const Json* kj = p.find("kernels");
    if (kj && kj->is_array() && kj->size() > 0) {
        c.has_kernels = true;
        for (const Json& k : kj->items()) {
            if (c.kernels.size() >= 4) {
                c.warnings.push_back("\"kernels\" has more than 4 entries; truncating to 4");
                break;
            }
            KernelDef kd;
            kd.radius_scale = k.value_float("radiusScale", 1.0f);
            kd.mu = k.value_float("mu", 0.15f);
            kd.sigma = k.value_float("sigma", 0.017f);
            kd.weight = k.value_float("weight", 1.0f);
            kd.betas.clear();
            const Json* b = k.find("betas");
            if (b && b->is_array())
                for (const Json& v : b->items()) kd.betas.push_back(v.is_number() ? float(v.as_number()) : 0.0f);
            if (kd.betas.empty()) kd.betas.push_back(1.0f);
            if (kd.betas.size() > size_t(kMaxBetas)) {
                error = "a kernel has more than 8 betas";
                return LENIA_ERR_UNSUPPORTED;
            }
            c.kernels.push_back(std::move(kd));
        }
    }
    c.kernel_core = p.value_string("kernelCore", "gaussShell") == "exp" ? LENIA_CORE_EXP
                                                                       : LENIA_CORE_GAUSS_SHELL;
    c.shell_mu = p.value_float("kernelShellMu", 0.5f);
    c.shell_sigma = p.value_float("kernelShellSigma", 0.15f);
    c.init_coverage = p.value_float("initCoverage", 0.4f);
    c.init_scale = p.value_float("initScale", 24.0f);
    c.want_stamp = p.value_string("initMode", "noise") == "stamp";
    const std::string org = p.value_string("organism", "");
    c.use_organism_params = p.value_bool("useOrganismParams", true);
    c.stamp_count = std::min<uint32_t>(32u, p.value_u32("stampCount", 6u));
    c.stamp_rotate = p.value_bool("stampRotate", true);
    if (!org.empty()) {
        c.has_organism_path = true;
        std::string err;
        c.organism_loaded = load_organism_file(org, c.organism, err);
        if (!c.organism_loaded && !base_dir.empty() && org[0] != '/') {
            std::string err2;
            c.organism_loaded = load_organism_file(base_dir + "/" + org, c.organism, err2);
        }
        if (!c.organism_loaded) c.organism_error = "failed to load organism \"" + org + "\": " + err;
    }
    return LENIA_OK;
}

int config_from_struct(const lenia_config& s, ModuleConfig& c, std::string& error) {
    c = ModuleConfig();
    c.sim_width = s.sim_width;
    c.sim_height = s.sim_height;
    if (s.conv_mode > LENIA_CONV_DIRECT_MULTI) {
        error = "conv_mode out of range";
        return LENIA_ERR_INVALID_ARG;
    }
    c.conv_mode = s.conv_mode;
    c.fft_any_size = s.fft_any_size != 0;
    if (s.fft_precision > LENIA_FFT_FP16X3) {
        error = "fft_precision out of range";
        return LENIA_ERR_INVALID_ARG;
    }
    c.fft_precision = s.fft_precision;
    c.has_radius = s.has_radius != 0;
    c.radius = s.radius;
    uint32_t nk = s.num_kernels;
    if (nk > 4) {
        c.warnings.push_back("\"kernels\" has more than 4 entries; truncating to 4");
        nk = 4;
    }
    c.has_kernels = s.num_kernels > 0;
    for (uint32_t i = 0; i < nk; ++i) {
        const lenia_kernel_def& k = s.kernels[i];
        if (k.num_betas > uint32_t(kMaxBetas)) {
            error = "a kernel has more than 8 betas";
            return LENIA_ERR_UNSUPPORTED;
        }
        KernelDef kd;
        kd.radius_scale = k.radius_scale;
        kd.mu = k.mu;
        kd.sigma = k.sigma;
        kd.weight = k.weight;
        kd.betas.assign(k.betas, k.betas + k.num_betas);
        if (kd.betas.empty()) kd.betas.push_back(1.0f);
        c.kernels.push_back(std::move(kd));
    }
    if (s.kernel_core > LENIA_CORE_EXP) {
        error = "kernel_core out of range";
        return LENIA_ERR_INVALID_ARG;
    }
    c.kernel_core = s.kernel_core;
    c.shell_mu = s.kernel_shell_mu;
    c.shell_sigma = s.kernel_shell_sigma;
    c.init_coverage = s.init_coverage;
    c.init_scale = s.init_scale;
    c.want_stamp = s.init_mode == LENIA_INIT_STAMP;
    c.use_organism_params = s.use_organism_params != 0;
    c.stamp_count = std::min<uint32_t>(32u, s.stamp_count);
    c.stamp_rotate = s.stamp_rotate != 0;
    if (s.organism_cells) {
        c.has_organism_path = true;
        if (s.org_width == 0 || s.org_height == 0) {
            c.organism_error = "organism has zero size";
        } else {
            c.organism.cells.assign(s.organism_cells,
                                    s.organism_cells + size_t(s.org_width) * s.org_height);
            c.organism.width = s.org_width;
            c.organism.height = s.org_height;
            c.organism.R = s.org_R;
            c.organism.T = s.org_T;
            c.organism.mu = s.org_mu;
            c.organism.sigma = s.org_sigma;
            c.organism_loaded = true;
            for (size_t i = 0; i < c.organism.cells.size(); ++i) {
                float v = c.organism.cells[i];
                if (!(v >= 0.0f && v <= 1.0f)) {
                    c.organism_loaded = false;
                    c.organism_error = "organism cell value out of [0,1] at index " + std::to_string(i);
                    break;
                }
            }
        }
    }
    return LENIA_OK;
}

// --------------------------------------------------------------- module

LeniaModule::LeniaModule() = default;
LeniaModule::~LeniaModule() { release(); }

void LeniaModule::release() {
    if (stream_) {
        cudaStreamSynchronize(stream_);
    }
    auto rel = [](auto*& p) {
        if (p) cudaFree(p);
        p = nullptr;
    };
    rel(field_[0]);
    rel(field_[1]);
    rel(d_tma_err_);
    direct_tma_ = DirectTma();
    rel(d_weights_);
    rel(d_spans_);
    rel(d_org_);
    rel(d_S_);
    rel(d_U_);
    rel(d_khat_);
    rel(d_tw_row_);
    rel(d_tw_col_);
    rel(d_tw_r2c_);
    for (auto& t : d_fast_tw_) rel(t);
    fast_col_ = fast_row_ = false;
    fast_ = FastTables();
    d_weights_ = nullptr;
    d_spans_ = nullptr;
    d_org_ = nullptr;
    d_S_ = d_U_ = nullptr;
    d_khat_ = nullptr;
    d_tw_row_ = d_tw_col_ = d_tw_r2c_ = nullptr;
    for (const TimedLaunch& t : timed_) {
        event_pool_.push_back(t.start);
        event_pool_.push_back(t.stop);
    }
    timed_.clear();
    for (cudaEvent_t e : event_pool_)
        if (e) cudaEventDestroy(e);
    event_pool_.clear();
    if (stream_) cudaStreamDestroy(stream_);
    stream_ = nullptr;
    device_bytes_ = 0;
}

int LeniaModule::fail(int code, const std::string& what) {
    message_ = what;
    return code;
}

int LeniaModule::cudaFail(cudaError_t e, const char* where) {
    return fail(LENIA_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

template <typename T>
static cudaError_t dev_alloc(T** p, size_t count, uint64_t& total) {
    total += uint64_t(count) * sizeof(T);
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

static bool fft_size_supported(uint32_t w, uint32_t h, FftPlan& row, FftPlan& col) {
    if (w < 2 || (w & 1u) || h < 1) return false;
    return fft_plan(int(w / 2), row) && fft_plan(int(h), col);
}

int LeniaModule::resolve(uint32_t scene_w, uint32_t scene_h) {
    message_.clear();
    warnings_ = cfg_.warnings;
    std::vector<std::string>& warn = warnings_;
    w_ = cfg_.sim_width ? cfg_.sim_width : scene_w;
    h_ = cfg_.sim_height ? cfg_.sim_height : scene_h;
    if (w_ == 0 || h_ == 0) return fail(LENIA_ERR_INVALID_ARG, "field size is zero");
    if (uint64_t(w_) * h_ > (uint64_t(1) << 31)) return fail(LENIA_ERR_UNSUPPORTED, "field too large");

    // Lenia.cpp:213-251 (convMode, power-of-two rule for the FFT path).
    use_fft_ = cfg_.conv_mode == LENIA_CONV_FFT;
    direct_multi_ = cfg_.conv_mode == LENIA_CONV_DIRECT_MULTI;
    FftPlan prow{}, pcol{};
    if (use_fft_) {
        if (!cfg_.fft_any_size && !(is_pow2(w_) && is_pow2(h_))) {
            warn.push_back("convMode=\"fft\" requires simWidth/simHeight to be powers of two (got " +
                           std::to_string(w_) + "x" + std::to_string(h_) +
                           "); falling back to convMode=\"direct\"");
            use_fft_ = false;
        } else if (!fft_size_supported(w_, h_, prow, pcol)) {
            warn.push_back("convMode=\"fft\": " + std::to_string(w_) + "x" + std::to_string(h_) +
                           " needs an even width and sizes with factors 2, 3, 5 only; falling back "
                           "to convMode=\"direct\"");
            use_fft_ = false;
        }
    }
    // fftPrecision (extension): tensor-core column stages where the column
    // plan is all radix 16 and the compile-time-plan passes run.
    tc_precision_ = LENIA_FFT_FP32;
    if (cfg_.fft_precision != LENIA_FFT_FP32) {
        FastPlan cf, ri;
        const bool ok = use_fft_ && w_ % 2 == 0 && (w_ / 2) % kSpectralBlock == 0 && tc_col_plan(int(h_)) &&
                        fast_col_plan(int(h_), cf) && fast_row_plan(int(w_ / 2), ri);
        if (ok) {
            tc_precision_ = cfg_.fft_precision;
        } else {
            warn.push_back("\"fftPrecision\" on the tensor cores needs convMode=\"fft\" with simHeight 256 or 4096 "
                           "(got " + std::to_string(w_) + "x" + std::to_string(h_) + "); using \"fp32\"");
        }
    }
    const bool multi = use_fft_ || direct_multi_;
    // Lenia.cpp:253-269: "kernels" without the FFT path keeps kernels[0].
    float radius_scale_override = 1.0f;
    fallback_mu_ = 0.15f;
    fallback_sigma_ = 0.017f;
    fallback_dt_ = 0.1f;
    if (cfg_.has_kernels && !multi) {
        warn.push_back("\"kernels\" requires convMode=\"fft\"; continuing in direct mode using kernels[0] only");
        radius_scale_override = cfg_.kernels[0].radius_scale;
        fallback_mu_ = cfg_.kernels[0].mu;
        fallback_sigma_ = cfg_.kernels[0].sigma;
    }
    kernels_ = multi ? cfg_.kernels : std::vector<KernelDef>();

    // Lenia.cpp:271-321: organism / stamp init.
    bool want_stamp = cfg_.want_stamp;
    bool want_org_params = cfg_.use_organism_params;
    if (cfg_.has_organism_path && want_org_params && cfg_.has_kernels) {
        warn.push_back("\"useOrganismParams\" cannot be combined with \"kernels\"; ignoring organism parameter overrides");
        want_org_params = false;
    }
    if (want_stamp && !cfg_.has_organism_path) {
        warn.push_back("initMode=\"stamp\" requires an \"organism\" path; falling back to noise init");
        want_stamp = false;
    }
    uint32_t org_radius_default = 13u;
    if (cfg_.has_organism_path && !cfg_.organism_loaded) {
        warn.push_back(cfg_.organism_error + "; falling back to noise init");
        want_stamp = false;
    }
    if (cfg_.organism_loaded && want_org_params) {
        org_radius_default = uint32_t(std::round(cfg_.organism.R));
        fallback_mu_ = cfg_.organism.mu;
        fallback_sigma_ = cfg_.organism.sigma;
        if (cfg_.organism.T > 1e-6f) fallback_dt_ = 1.0f / cfg_.organism.T;
    }
    use_stamp_ = want_stamp && cfg_.organism_loaded;
    radius_ = uint32_t(std::round(float(cfg_.has_radius ? cfg_.radius : org_radius_default) *
                                  radius_scale_override));
    fgeo_.row = prow;
    fgeo_.col = pcol;
    num_k_ = multi ? uint32_t(std::max<size_t>(1, std::min<size_t>(4, kernels_.size()))) : 1u;
    // The direct path's radius limit (buildDirectTables), here as well so
    // that the host-only inspection reports what setup would.
    if (!use_fft_ && !direct_multi_ && radius_ > uint32_t(kMaxRadius))
        return fail(LENIA_ERR_UNSUPPORTED,
                    "direct convolution supports radius <= 32 (got " + std::to_string(radius_) + ")");
    if (!use_fft_ && direct_multi_) {
        for (size_t k = 0; k < std::max<size_t>(1, std::min<size_t>(4, kernels_.size())); ++k) {
            const float scale = kernels_.empty() ? 1.0f : kernels_[k].radius_scale;
            if (!(float(radius_) * scale <= float(kMaxRadius)))
                return fail(LENIA_ERR_UNSUPPORTED, "direct convolution supports kernel radius <= 32");
        }
    }
    if (!warn.empty()) {
        std::string m;
        for (const auto& w : warn) m += (m.empty() ? "" : "\n") + ("[life] " + instance_ + ": " + w);
        message_ = m;
        return LENIA_WARN_FALLBACK;
    }
    return LENIA_OK;
}

int LeniaModule::setup(uint32_t scene_w, uint32_t scene_h) {
    release();
    const int resolved = resolve(scene_w, scene_h);
    if (resolved < 0) return resolved;
    const std::string warn_msg = message_;
    if (cudaGetDevice(&device_) != cudaSuccess) return fail(LENIA_ERR_NO_DEVICE, "no CUDA device");
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking)) != cudaSuccess)
        return cudaFail(e, "cudaStreamCreate");
    const size_t npx = size_t(w_) * h_;
    for (float*& f : field_) {
        if ((e = dev_alloc(&f, npx, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc field");
        cudaMemsetAsync(f, 0, npx * sizeof(float), stream_);
    }
    if (use_stamp_) {
        const size_t n = cfg_.organism.cells.size();
        if ((e = dev_alloc(&d_org_, n, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc organism");
        cudaMemcpy(d_org_, cfg_.organism.cells.data(), n * sizeof(float), cudaMemcpyHostToDevice);
    }

    int rc = LENIA_OK;
    if (use_fft_) {
        std::vector<KernelDef> eff = kernels_;
        if (eff.empty()) eff.push_back(KernelDef());  // implicit kernel: betas [1], scale 1
        rc = buildSpectralTables(eff);
    } else {
        rc = buildDirectTables();
    }
    if (rc < 0) return rc;
    cudaStreamSynchronize(stream_);
    if ((e = cudaGetLastError()) != cudaSuccess) return cudaFail(e, "setup");
    needs_field_init_ = true;
    needs_kernel_init_ = true;
    spectrum_valid_ = false;
    cur_ = 0;
    message_ = warn_msg;
    return resolved;
}

// Direct LUTs in the padded per-row layout of lenia_direct.cu, plus the
// per-row chunk spans over the nonzero taps.
int LeniaModule::buildDirectTables() {
    std::vector<std::vector<float>> luts;  // each (2r+1)^2 for the common halo r
    int r = 0;
    if (!direct_multi_) {
        if (radius_ > uint32_t(kMaxRadius))
            return fail(LENIA_ERR_UNSUPPORTED, "direct convolution supports radius <= 32 (got " +
                                                   std::to_string(radius_) + ")");
        build_direct_lut(radius_, cfg_.shell_mu, cfg_.shell_sigma, cfg_.kernel_core, direct_lut_);
        r = int(radius_);
        luts.push_back(direct_lut_);
    } else {
        std::vector<KernelDef> eff = kernels_;
        if (eff.empty()) eff.push_back(KernelDef());
        if (eff.size() > 4) eff.resize(4);
        std::vector<std::vector<float>> imgs;
        for (const auto& k : eff) {
            const float rk = float(radius_) * k.radius_scale;
            if (!(rk <= float(kMaxRadius)))
                return fail(LENIA_ERR_UNSUPPORTED, "direct convolution supports kernel radius <= 32");
            r = std::max(r, int(std::ceil(rk)));
            std::vector<float> img;
            build_ring_image(w_, h_, rk, cfg_.shell_sigma, k.betas, cfg_.kernel_core, img);
            imgs.push_back(std::move(img));
        }
        // Cut each image to the (2r+1)^2 window; every torus offset is
        // taken once (dx in (-w/2, w/2], dy in (-h/2, h/2]).
        const int ks = 2 * r + 1;
        for (const auto& img : imgs) {
            std::vector<float> lut(size_t(ks) * ks, 0.0f);
            for (int dy = -r; dy <= r; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const bool xin = (w_ % 2 == 0) ? (dx > -int(w_ / 2) && dx <= int(w_ / 2))
                                                   : (dx >= -int(w_ / 2) && dx <= int(w_ / 2));
                    const bool yin = (h_ % 2 == 0) ? (dy > -int(h_ / 2) && dy <= int(h_ / 2))
                                                   : (dy >= -int(h_ / 2) && dy <= int(h_ / 2));
                    if (!xin || !yin) continue;
                    const uint32_t x = uint32_t((dx % int(w_) + int(w_)) % int(w_));
                    const uint32_t y = uint32_t((dy % int(h_) + int(h_)) % int(h_));
                    lut[size_t(dy + r) * ks + (dx + r)] = img[size_t(y) * w_ + x];
                }
            luts.push_back(std::move(lut));
        }
    }
    direct_nk_ = int(luts.size());
    num_k_ = uint32_t(direct_nk_);
    direct_taps_ = 0;
    for (const auto& lut : luts)
        for (float v : lut) direct_taps_ += v != 0.0f ? 1u : 0u;
    dgeo_.r = r;
    dgeo_.ksize = 2 * r + 1;
    dgeo_.xp = (r + 3) / 4 * 4;
    dgeo_.wp = 2 * dgeo_.xp + 8;
    const int ks = dgeo_.ksize;
    std::vector<float> wts(size_t(direct_nk_) * ks * dgeo_.wp, 0.0f);
    std::vector<uint32_t> spans(size_t(direct_nk_) * ks, 0u);
    for (int k = 0; k < direct_nk_; ++k)
        for (int dy = 0; dy < ks; ++dy) {
            int lo = 1 << 30, hi = -(1 << 30);
            for (int dx = -r; dx <= r; ++dx) {
                const float v = luts[size_t(k)][size_t(dy) * ks + (dx + r)];
                wts[(size_t(k) * ks + dy) * dgeo_.wp + (dx + dgeo_.xp)] = v;
                if (v != 0.0f) {
                    lo = std::min(lo, dx);
                    hi = std::max(hi, dx);
                }
            }
            uint32_t packed = 0;
            if (lo <= hi) {
                // Chunks on the 8-tap grid that starts at dx = -xp (every row
                // on one grid, so the two-rows-per-thread kernel can walk the
                // union of two rows' spans; the extra taps weigh zero).
                const int start = -dgeo_.xp + (lo + dgeo_.xp) / 8 * 8;
                const int count = (hi - start + 1 + 7) / 8;
                packed = uint32_t(start + 128) | (uint32_t(count) << 16);
            } else {
                packed = uint32_t(128);
            }
            spans[size_t(k) * ks + dy] = packed;
        }
    cudaError_t e;
    if ((e = dev_alloc(&d_weights_, wts.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc weights");
    if ((e = dev_alloc(&d_spans_, spans.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc spans");
    cudaMemcpy(d_weights_, wts.data(), wts.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_spans_, spans.data(), spans.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
    // Tile shape: the largest tile that still gives >= 2 CTAs per SM.
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
    const auto tiles = [&](int tw, int th) { return ((w_ + tw - 1) / tw) * ((h_ + th - 1) / th); };
    if (tiles(64, 32) >= 2 * sms) direct_tile_ = kDirectTile64x32;
    else if (tiles(64, 16) >= 2 * sms) direct_tile_ = kDirectTile64x16;
    else direct_tile_ = kDirectTile32x16;
    if (direct_smem_bytes(direct_tile_, direct_nk_, dgeo_) > 220 * 1024) direct_tile_ = kDirectTile32x16;
    // A field too small to give ~16 warps per SM at one thread per 8 outputs
    // (64 threads per 32x16 tile) splits each tile's kernel rows over up to 8
    // thread groups. A size rule, not a timing, so a configuration always
    // sums in the same order (the same bits run to run).
    direct_split_ = 1;
    if (direct_tile_ == kDirectTile32x16) {
        const int warps = tiles(32, 16) * 2;
        while (direct_split_ < 8 && 2 * direct_split_ <= dgeo_.ksize && warps * direct_split_ < 16 * sms)
            direct_split_ *= 2;
        while (direct_split_ > 1 && direct_smem_bytes(direct_tile_, direct_nk_, dgeo_) +
                                            direct_split_smem_bytes(direct_split_, direct_nk_) > 220 * 1024)
            direct_split_ /= 2;
    }
    // Outputs per thread on large tiles: 8 or 16 along x (64x32 tiles) times 1
    // or 2 rows (64x32 and 64x16 tiles, no split), whichever runs fastest here
    // (a few steps each on the context's own buffers; the same bits in every
    // variant). LENIA_DIRECT_OX ("8" / "16") and LENIA_DIRECT_OY ("1" / "2")
    // at setup force either.
    direct_ox_ = 8;
    direct_oy_ = 1;
    const char* ox_env = std::getenv("LENIA_DIRECT_OX");
    const char* oy_env = std::getenv("LENIA_DIRECT_OY");
    const int ox_forced = ox_env ? std::atoi(ox_env) : 0;
    const int oy_forced = oy_env ? std::atoi(oy_env) : 0;
    struct Shape {
        int ox, oy;
    };
    std::vector<Shape> shapes;
    const bool big = direct_tile_ == kDirectTile64x32 || direct_tile_ == kDirectTile64x16;
    for (int ox : {8, 16})
        for (int oy : {1, 2}) {
            if (ox == 16 && direct_tile_ != kDirectTile64x32) continue;
            if (oy == 2 && (!big || direct_split_ != 1)) continue;
            if ((ox_forced == 8 || ox_forced == 16) && ox != ox_forced) continue;
            if ((oy_forced == 1 || oy_forced == 2) && oy != oy_forced) continue;
            shapes.push_back({ox, oy});
        }
    if (shapes.size() == 1) {
        direct_ox_ = shapes[0].ox;
        direct_oy_ = shapes[0].oy;
    } else if (shapes.size() > 1) {
        StepParams p{};
        p.width = w_;
        p.height = h_;
        p.num_kernels = uint32_t(direct_nk_);
        for (int k = 0; k < 4; ++k) p.sigma[k] = 1.0f;
        cudaEvent_t a = takeEvent(), b = takeEvent();
        std::vector<float> best(shapes.size(), 1e30f);
        // Six rounds over the candidates, the first untimed (clocks ramp up
        // from idle at setup); the minimum of the other five per candidate.
        for (int rep = 0; rep < 6; ++rep)
            for (size_t v = 0; v < shapes.size(); ++v) {
                cudaEventRecord(a, stream_);
                for (int i = 0; i < 3; ++i)
                    launch_direct_step(direct_tile_, direct_nk_, field_[0], field_[1], d_weights_, d_spans_, dgeo_, p,
                                       stream_, nullptr, 0, direct_split_, shapes[v].ox, shapes[v].oy);
                cudaEventRecord(b, stream_);
                cudaEventSynchronize(b);
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess && rep > 0) best[v] = std::min(best[v], ms);
            }
        event_pool_.push_back(a);
        event_pool_.push_back(b);
        if ((e = cudaGetLastError()) != cudaSuccess) return cudaFail(e, "direct shape choice");
        size_t pick = 0;
        for (size_t v = 1; v < shapes.size(); ++v)
            if (best[v] < best[pick]) pick = v;
        direct_ox_ = shapes[pick].ox;
        direct_oy_ = shapes[pick].oy;
    }
    // Halo tiles by TMA where the size allows it (interior tiles only).
    // LENIA_DIRECT_TMA in the environment at setup: 0 keeps element loads,
    // 1 uses TMA wherever the size allows; unset, the faster one here.
    const char* tma_env = std::getenv("LENIA_DIRECT_TMA");
    const bool tma_off = tma_env && tma_env[0] == '0' && tma_env[1] == '\0';
    const bool tma_forced = tma_env && tma_env[0] == '1' && tma_env[1] == '\0';
    if (!tma_off && direct_tma_encode(direct_tile_, dgeo_, field_, int(w_), int(h_), direct_tma_)) {
        if ((e = dev_alloc(&d_tma_err_, 1, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc flags");
        cudaMemset(d_tma_err_, 0, sizeof(int));
        direct_tma_.err = d_tma_err_;
    }
    if (direct_tma_.on && !tma_forced) {
        // One bulk copy per CTA wins on small fields and loses to the
        // element loads of many CTAs on large ones: keep whichever is faster
        // here (a few steps each on the context's own buffers).
        StepParams p{};
        p.width = w_;
        p.height = h_;
        p.num_kernels = uint32_t(direct_nk_);
        for (int k = 0; k < 4; ++k) p.sigma[k] = 1.0f;
        cudaEvent_t a = takeEvent(), b = takeEvent();
        float best[2] = {1e30f, 1e30f};
        for (int rep = 0; rep < 3; ++rep)
            for (int v = 0; v < 2; ++v) {
                cudaEventRecord(a, stream_);
                for (int i = 0; i < 3; ++i)
                    launch_direct_step(direct_tile_, direct_nk_, field_[0], field_[1], d_weights_, d_spans_, dgeo_, p,
                                       stream_, v ? &direct_tma_ : nullptr, 0, direct_split_, direct_ox_,
                                       direct_oy_);
                cudaEventRecord(b, stream_);
                cudaEventSynchronize(b);
                float ms = 0.0f;
                if (cudaEventElapsedTime(&ms, a, b) == cudaSuccess && rep > 0) best[v] = std::min(best[v], ms);
            }
        event_pool_.push_back(a);
        event_pool_.push_back(b);
        cudaMemsetAsync(field_[1], 0, sizeof(float) * w_ * h_, stream_);
        if ((e = cudaGetLastError()) != cudaSuccess) return cudaFail(e, "direct staging choice");
        if (!(best[1] < best[0])) direct_tma_.on = false;
    }
    return LENIA_OK;
}

cudaError_t LeniaModule::launchColumnTc(int choice, const float2* S, float2* U, cudaStream_t s) {
    if (choice == kTcgen05 || choice == kTcgen05Pipelined)
        return launch_col_tc05(fgeo_, int(tc_precision_), choice == kTcgen05Pipelined, S, U, d_tma_err_, s);
    return launch_col_tc(fgeo_, fast_, int(tc_precision_), choice, S, U, s);
}

int LeniaModule::checkDeviceFlags() {
    if (!d_tma_err_) return LENIA_OK;
    int n = 0;
    const cudaError_t e = cudaMemcpy(&n, d_tma_err_, sizeof n, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cudaFail(e, "read device flags");
    if (n != 0) {
        cudaMemset(d_tma_err_, 0, sizeof(int));
        if (use_fft_)
            return fail(LENIA_ERR_CUDA, "tensor-core column pass: " + std::to_string(n) +
                                            " CTA(s) stopped after a wait for an MMA ran out; their columns were "
                                            "not written");
        return fail(LENIA_ERR_CUDA, "direct path: " + std::to_string(n) +
                                        " halo tile load(s) did not arrive in time; those tiles were not written");
    }
    return LENIA_OK;
}

int LeniaModule::buildSpectralTables(const std::vector<KernelDef>& eff) {
    const uint32_t nk = uint32_t(std::min<size_t>(4, eff.size()));
    const int M = int(w_ / 2), H = int(h_), Hh = H / 2 + 1;
    fgeo_.W = int(w_);
    fgeo_.H = H;
    fgeo_.M = M;
    fgeo_.nk = int(nk);
    // Rows per CTA in the row passes: 4 (32 B column segments) if two CTAs
    // still fit on an SM, else fewer.
    const auto row_smem = [&](int rb) {
        return sizeof(float2) * (size_t(2 * M + 1) + 2 * size_t(rb) * M) + sizeof(float) * size_t(rb) * w_;
    };
    const auto col_smem = [&](int cb) { return sizeof(float2) * (size_t(H) + 3 * size_t(cb) * H); };
    int rb = 4;
    while (rb > 1 && row_smem(rb) > 110 * 1024) rb /= 2;
    if (row_smem(rb) > 220 * 1024) return fail(LENIA_ERR_UNSUPPORTED, "field width too large for the FFT path");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_);
    int cb = std::max(1, std::min(8, M / (2 * sms)));
    while (cb > 1 && col_smem(cb) > 110 * 1024) --cb;
    if (col_smem(cb) > 220 * 1024) return fail(LENIA_ERR_UNSUPPORTED, "field height too large for the FFT path");
    fgeo_.rows_per_cta = rb;
    fgeo_.cols_per_cta = cb;

    std::vector<float2> tr, tc, t2;
    fill_twiddles(M, tr);
    fill_twiddles(H, tc);
    fill_twiddles(int(w_), t2);
    t2.resize(size_t(M) + 1);  // exp(-2 pi i k / W), k <= M
    std::vector<float> khat(size_t(nk) * (M + 1) * Hh);
    for (uint32_t k = 0; k < nk; ++k) {
        std::vector<float> img, spec;
        const float rk = float(radius_) * eff[k].radius_scale;  // Lenia.cpp:519
        build_ring_image(w_, h_, rk, cfg_.shell_sigma, eff[k].betas, cfg_.kernel_core, img);
        kernel_spectrum(img, w_, h_, spec);
        std::copy(spec.begin(), spec.end(), khat.begin() + size_t(k) * (M + 1) * Hh);
    }
    cudaError_t e;
    const size_t spec = size_t(M) * H;
    if ((e = dev_alloc(&d_S_, spec, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc spectrum");
    if ((e = dev_alloc(&d_U_, spec * nk, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc potentials");
    if ((e = dev_alloc(&d_khat_, khat.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc khat");
    if ((e = dev_alloc(&d_tw_row_, tr.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc twiddles");
    if ((e = dev_alloc(&d_tw_col_, tc.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc twiddles");
    if ((e = dev_alloc(&d_tw_r2c_, t2.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc twiddles");
    cudaMemcpy(d_khat_, khat.data(), khat.size() * sizeof(float), cudaMemcpyHostToDevice);
    cudaMemcpy(d_tw_row_, tr.data(), tr.size() * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(d_tw_col_, tc.data(), tc.size() * sizeof(float2), cudaMemcpyHostToDevice);
    cudaMemcpy(d_tw_r2c_, t2.data(), t2.size() * sizeof(float2), cudaMemcpyHostToDevice);
    fgeo_.tw_row = d_tw_row_;
    fgeo_.tw_col = d_tw_col_;
    fgeo_.tw_r2c = d_tw_r2c_;
    fgeo_.khat = d_khat_;
    num_k_ = nk;

    // Compile-time-plan passes where this size has one; per-pass twiddle
    // tables for the plan and its reverse.
    // The fast passes share the blocked spectral layout, so they are used
    // together or not at all.
    FastPlan cf, ri;
    const bool fast = fast_col_plan(H, cf) && fast_row_plan(M, ri) && M % kSpectralBlock == 0;
    fast_col_ = fast_row_ = fast;
    auto upload_plan = [&](const FastPlan& pl, float2*& dst) -> int {
        std::vector<float2> tw;
        fast_plan_twiddles(pl, tw);
        if (tw.empty()) tw.push_back(make_float2(1.0f, 0.0f));
        if ((e = dev_alloc(&dst, tw.size(), device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc twiddles");
        cudaMemcpy(dst, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
        return LENIA_OK;
    };
    auto reversed = [](const FastPlan& pl) {
        FastPlan r = pl;
        for (int i = 0; i < pl.np; ++i) r.radix[i] = pl.radix[pl.np - 1 - i];
        return r;
    };
    if (fast_col_) {
        if (upload_plan(cf, d_fast_tw_[0]) < 0 || upload_plan(reversed(cf), d_fast_tw_[1]) < 0) return LENIA_ERR_CUDA;
        fast_.col_twf = d_fast_tw_[0];
        fast_.col_twi = d_fast_tw_[1];
    }
    if (fast_row_) {
        if (upload_plan(ri, d_fast_tw_[2]) < 0 || upload_plan(reversed(ri), d_fast_tw_[3]) < 0) return LENIA_ERR_CUDA;
        fast_.row_twi = d_fast_tw_[2];
        fast_.row_twf = d_fast_tw_[3];
    }
    if (tc_precision_ != LENIA_FFT_FP32 && tc05_col_plan(int(h_)) && !d_tma_err_) {
        // The tcgen05 column pass counts CTAs whose MMA wait ran out here.
        cudaError_t e;
        if ((e = dev_alloc(&d_tma_err_, 1, device_bytes_)) != cudaSuccess) return cudaFail(e, "cudaMalloc flags");
        cudaMemset(d_tma_err_, 0, sizeof(int));
    }
    return autotuneSpectral();
}

// Picks columns (rows) per CTA of the compile-time-plan passes by timing
// each candidate on this context's own buffers (contents irrelevant).
int LeniaModule::autotuneSpectral() {
    if (!fast_col_ && !fast_row_) return LENIA_OK;
    cudaEvent_t a = takeEvent(), b = takeEvent();
    StepParams p{};
    p.num_kernels = uint32_t(fgeo_.nk);
    p.width = w_;
    p.height = h_;
    p.sigma[0] = p.sigma[1] = p.sigma[2] = p.sigma[3] = 1.0f;
    auto time_it = [&](auto&& fn) {
        float best = 1e30f;
        for (int rep = 0; rep < 4; ++rep) {
            cudaEventRecord(a, stream_);
            if (fn() != cudaSuccess) return 1e30f;
            cudaEventRecord(b, stream_);
            cudaEventSynchronize(b);
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, a, b);
            if (rep > 0) best = std::min(best, ms);
        }
        return best;
    };
    // A candidate must beat the current choice by 3 % to replace it (the
    // timings run with warm caches; larger batches coalesce better cold).
    // LENIA_AUTOTUNE_LOG=1 prints every candidate's time to stderr.
    const char* log_env = std::getenv("LENIA_AUTOTUNE_LOG");
    const bool log = log_env && *log_env && *log_env != '0';
    float best_col = 1e30f, best_row = 1e30f;
    for (int c : kColCandidates) {
        if (!fast_shapes_supported(int(h_), int(w_ / 2), c, 4)) continue;
        const float t = time_it([&] { return launch_col_fast(fgeo_, fast_, c, d_S_, d_U_, stream_); });
        if (log)
            std::fprintf(stderr, "lenia autotune %ux%u column cols/CTA %d%s: %.4f ms\n", w_, h_, c & 0xF,
                         (c & kHalfThreads) ? " half threads" : "", t);
        if (t < 0.97f * best_col) { best_col = t; col_batch_ = c; }
    }
    // Row candidates are timed as they run in a step: three column + row
    // pairs back to back (the row pass follows the column pass it reads).
    for (int c : kRowCandidates) {
        if (!fast_shapes_supported(int(h_), int(w_ / 2), col_batch_, c)) continue;
        const float t = time_it([&] {
            cudaError_t e = cudaSuccess;
            for (int i = 0; i < 3 && e == cudaSuccess; ++i) {
                e = launch_col_fast(fgeo_, fast_, col_batch_, d_S_, d_U_, stream_);
                if (e == cudaSuccess)
                    e = launch_row_fast(fgeo_, fast_, c, d_U_, field_[0], field_[1], d_S_, p, fgeo_.nk, stream_);
            }
            return e;
        });
        if (log)
            std::fprintf(stderr, "lenia autotune %ux%u 3 steps with rows/CTA %d%s: %.4f ms\n", w_, h_, c & 7,
                         (c & kRowPipelined) ? " pipelined" : "", t);
        if (t < 0.97f * best_row) { best_row = t; row_batch_ = c; }
    }
    if (tc_precision_ != LENIA_FFT_FP32) {
        // Candidates: the tcgen05 pass (4096-row fields) and the mma.sync
        // pass at each columns-per-CTA count. LENIA_TC_ENGINE=tcgen05 or
        // =mma at setup keeps only that engine's candidates.
        const char* eng = std::getenv("LENIA_TC_ENGINE");
        const std::string e = eng ? eng : "";
        std::vector<int> cands;
        if (tc05_col_plan(int(h_))) {
            if (e.empty() || e == "tcgen05" || e == "tcgen05_pipelined") cands.push_back(kTcgen05Pipelined);
            if (e.empty() || e == "tcgen05" || e == "tcgen05_serial") cands.push_back(kTcgen05);
        }
        if (cands.empty() || e.empty() || e == "mma")
            for (int c : {8, 4, 2, 1}) cands.push_back(c);
        float best_tc = 1e30f;
        for (int c : cands) {
            const float t = time_it([&] { return launchColumnTc(c, d_S_, d_U_, stream_); });
            if (t < 0.97f * best_tc) { best_tc = t; tc_batch_ = c; }
        }
        if (best_tc >= 1e29f) tc_precision_ = LENIA_FFT_FP32;
        cudaGetLastError();
    }
    if (best_col >= 1e29f || best_row >= 1e29f) fast_col_ = fast_row_ = false;
    cudaGetLastError();
    event_pool_.push_back(a);
    event_pool_.push_back(b);
    cudaMemsetAsync(field_[0], 0, sizeof(float) * w_ * h_, stream_);
    cudaMemsetAsync(field_[1], 0, sizeof(float) * w_ * h_, stream_);
    return LENIA_OK;
}

void LeniaModule::tuning(int* cols, int* rows) const {
    const bool on = fast_col_ && fast_row_;
    *cols = on ? col_batch_ : 0;
    *rows = on ? row_batch_ : 0;
}

int LeniaModule::setTuning(int cols, int rows) {
    if (!(fast_col_ && fast_row_))
        return fail(LENIA_ERR_INVALID_ARG, "launch shapes apply to the compile-time-plan spectral passes only");
    if (!fast_shapes_supported(int(h_), int(w_ / 2), cols, rows))
        return fail(LENIA_ERR_INVALID_ARG, "unsupported launch shape: " + std::to_string(cols) + " columns, " +
                                               std::to_string(rows) + " rows per CTA for " + std::to_string(w_) +
                                               "x" + std::to_string(h_));
    col_batch_ = cols;
    row_batch_ = rows;
    return LENIA_OK;
}

cudaEvent_t LeniaModule::takeEvent() {
    if (!event_pool_.empty()) {
        cudaEvent_t e = event_pool_.back();
        event_pool_.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

template <typename F>
cudaError_t LeniaModule::launch(int phase, cudaStream_t s, F&& fn) {
    TimedLaunch t{phase, nullptr, nullptr};
    if (profiling_) {
        t.start = takeEvent();
        t.stop = takeEvent();
        cudaEventRecord(t.start, s);
    }
    const cudaError_t e = fn();
    ++launches_;
    if (profiling_) {
        cudaEventRecord(t.stop, s);
        timed_.push_back(t);
    }
    return e;
}

void LeniaModule::setProfiling(bool on) {
    lenia_profile_data scratch;
    readProfile(&scratch);  // drop what was recorded so far
    profiling_ = on;
    launches_ = 0;
}

int LeniaModule::readProfile(lenia_profile_data* out) {
    std::memset(out, 0, sizeof(*out));
    out->launches = launches_;
    launches_ = 0;
    for (const TimedLaunch& t : timed_) {
        float ms = 0.0f;
        if (cudaEventSynchronize(t.stop) == cudaSuccess && cudaEventElapsedTime(&ms, t.start, t.stop) == cudaSuccess &&
            t.phase >= 0 && t.phase < LENIA_PHASE_COUNT) {
            out->ms[t.phase] += double(ms);
            out->count[t.phase] += 1;
        }
        event_pool_.push_back(t.start);
        event_pool_.push_back(t.stop);
    }
    timed_.clear();
    return LENIA_OK;
}

void LeniaModule::reset(uint32_t seed) {
    seed_ = derive_seed(seed, 0x4C454E31u);  // "LEN1", Lenia.cpp:449
    needs_field_init_ = true;
    needs_kernel_init_ = true;
}

// param(ctx, key, fallback) reads "<instance>.<key>" from the bus
// (SimulationModule.h:120-123, Lenia.cpp:456-464).
lenia_frame_params LeniaModule::resolveFrameParams(const ParameterBus& bus, uint32_t frame_index,
                                                   uint32_t audio_frame) const {
    const auto param = [&](const char* key, float fallback) { return bus.value(instance_ + "." + key, fallback); };
    lenia_frame_params fp{};
    fp.dt = param("dt", fallback_dt_);
    fp.growth_mu = param("growthMu", fallback_mu_);
    fp.growth_sigma = param("growthSigma", fallback_sigma_);
    fp.noise_amount = param("noiseAmount", 0.0f);
    fp.mu_jitter = param("muJitter", 0.0f);
    fp.inject_amount = param("injectAmount", 0.0f);
    fp.inject_count = uint32_t(param("injectCount", 3.0f) + 0.5f);
    fp.growth_mode = uint32_t(param("growthMode", 1.0f) + 0.5f);
    fp.frame_index = frame_index;
    fp.audio_frame = audio_frame;
    return fp;
}

int LeniaModule::encode(uint32_t frame_index, uint32_t substeps, const ParameterBus& params,
                        cudaStream_t stream) {
    return step(resolveFrameParams(params, frame_index, audio_frame_), substeps, stream);
}

int LeniaModule::render(void* rgba16f, uint32_t dst_w, uint32_t dst_h, cudaStream_t s) {
    if (!rgba16f || dst_w == 0 || dst_h == 0) return fail(LENIA_ERR_INVALID_ARG, "render: null buffer or empty size");
    if (!field_[0]) return fail(LENIA_ERR_STATE, "render: module not set up");
    const cudaError_t e = launch(LENIA_PHASE_COLORMAP, s, [&] {
        return launch_colormap(field_[cur_], int(w_), int(h_), colormap_, rgba16f, int(dst_w), int(dst_h), s);
    });
    if (e != cudaSuccess) return cudaFail(e, "colour map");
    return LENIA_OK;
}

int LeniaModule::initField(const lenia_frame_params&, cudaStream_t s) {
    cudaError_t e;
    if (use_stamp_) {
        e = launch(LENIA_PHASE_INIT, s, [&] {
            return launch_init_stamp(field_[cur_], w_, h_, d_org_, cfg_.organism.width, cfg_.organism.height,
                                     cfg_.stamp_count, cfg_.stamp_rotate ? 1u : 0u, seed_, s);
        });
    } else {
        InitParams ip{cfg_.init_coverage, cfg_.init_scale, seed_, w_, h_};
        e = launch(LENIA_PHASE_INIT, s, [&] { return launch_init_noise(field_[cur_], ip, s); });
    }
    if (e != cudaSuccess) return cudaFail(e, "init launch");
    return LENIA_OK;
}

// Lenia.cpp:497-545: per-kernel growth parameters are fixed when the
// field is (re)initialised; without "kernels" one implicit kernel takes the
// frame's growthMu/growthSigma.
int LeniaModule::initKernels(const lenia_frame_params& fp) {
    if (!(use_fft_ || direct_multi_)) return LENIA_OK;
    std::vector<KernelDef> eff = kernels_;
    if (eff.empty()) {
        KernelDef kd;
        kd.mu = fp.growth_mu;
        kd.sigma = fp.growth_sigma;
        eff.push_back(kd);
    }
    num_k_ = uint32_t(std::min<size_t>(4, eff.size()));
    for (uint32_t k = 0; k < 4; ++k) {
        if (k < num_k_) {
            k_mu_[k] = eff[k].mu;
            k_sigma_[k] = eff[k].sigma;
            k_weight_[k] = eff[k].weight;
        } else {
            k_mu_[k] = 0.15f;
            k_sigma_[k] = 0.017f;
            k_weight_[k] = 0.0f;
        }
    }
    return LENIA_OK;
}

void LeniaModule::fillStepParams(const lenia_frame_params& fp, uint32_t seed, StepParams& p) const {
    std::memset(&p, 0, sizeof(p));
    p.dt = fp.dt;
    if (use_fft_ || direct_multi_) {
        p.num_kernels = num_k_;
        float sw = 0.0f;
        for (uint32_t k = 0; k < 4; ++k) {
            p.mu[k] = k_mu_[k];
            p.sigma[k] = k_sigma_[k];
            p.weight[k] = k_weight_[k];
            if (k < num_k_) sw += k_weight_[k];
        }
        p.sum_weights = sw;
    } else {
        p.num_kernels = 1;
        p.mu[0] = fp.growth_mu;
        p.sigma[0] = fp.growth_sigma;
        p.weight[0] = 1.0f;
        p.sum_weights = 1.0f;
    }
    p.growth_mode = fp.growth_mode;
    p.noise_amount = fp.noise_amount;
    p.mu_jitter = fp.mu_jitter;
    p.inject_amount = fp.inject_amount;
    p.inject_count = fp.inject_count;
    p.radius = radius_;
    p.seed = seed;
    p.width = w_;
    p.height = h_;
    p.frame_index = fp.frame_index;
    p.audio_frame = fp.audio_frame;
}

int LeniaModule::step(const lenia_frame_params& fp, uint32_t substeps, cudaStream_t stream) {
    return stepImpl(fp, substeps, stream, nullptr);
}

int LeniaModule::stepRender(const lenia_frame_params& fp, uint32_t substeps, void* rgba16f, uint32_t dst_w,
                            uint32_t dst_h, cudaStream_t stream) {
    if (!rgba16f || dst_w == 0 || dst_h == 0) return fail(LENIA_ERR_INVALID_ARG, "render: null buffer or empty size");
    if (!field_[0]) return fail(LENIA_ERR_STATE, "module is not set up");
    const bool fused = use_fft_ && fast_row_ && dst_w == w_ && dst_h == h_ &&
                       (reinterpret_cast<uintptr_t>(rgba16f) & 15u) == 0;
    const int rc = stepImpl(fp, substeps, stream, fused ? rgba16f : nullptr);
    if (rc < 0 || fused) return rc;
    return render(rgba16f, dst_w, dst_h, stream ? stream : stream_);
}

// `rgba16f` (or null): the last substep's row pass also writes the colour
// layer of its result at the sim size.
int LeniaModule::stepImpl(const lenia_frame_params& fp, uint32_t substeps, cudaStream_t stream, void* rgba16f) {
    if (!field_[0]) return fail(LENIA_ERR_STATE, "module is not set up");
    cudaStream_t s = stream ? stream : stream_;
    int rc;
    if (needs_field_init_) {
        if ((rc = initField(fp, s)) < 0) return rc;
        needs_field_init_ = false;
        spectrum_valid_ = false;
    }
    if (needs_kernel_init_) {
        if ((rc = initKernels(fp)) < 0) return rc;
        needs_kernel_init_ = false;
    }
    const uint32_t n = std::max(1u, substeps);
    StepParams p;
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t seed = pcg_hash_host(seed_ ^ (fp.frame_index * 197u + i));  // Lenia.cpp:564
        fillStepParams(fp, seed, p);
        float* src = field_[cur_];
        float* dst = field_[cur_ ^ 1];
        cudaError_t e;
        if (use_fft_) {
            if (!spectrum_valid_) {
                e = launch(LENIA_PHASE_ROW_FFT, s, [&] {
                    return fast_row_ ? launch_row_fast(fgeo_, fast_, row_batch_, nullptr, src, nullptr, d_S_, p, 0, s)
                                     : launch_row_r2c(fgeo_, src, d_S_, s);
                });
                if (e != cudaSuccess) return cudaFail(e, "row pass");
            }
            e = launch(LENIA_PHASE_COLUMN, s, [&] {
                if (tc_precision_ != LENIA_FFT_FP32) return launchColumnTc(tc_batch_, d_S_, d_U_, s);
                return fast_col_ ? launch_col_fast(fgeo_, fast_, col_batch_, d_S_, d_U_, s)
                                 : launch_col_conv(fgeo_, d_S_, d_U_, s);
            });
            if (e != cudaSuccess) return cudaFail(e, "column pass");
            void* out_rgba = i + 1 == n ? rgba16f : nullptr;
            e = launch(LENIA_PHASE_ROW_GROWTH, s, [&] {
                return fast_row_ ? launch_row_fast(fgeo_, fast_, row_batch_, d_U_, src, dst, d_S_, p, fgeo_.nk, s,
                                                   out_rgba, &colormap_)
                                 : launch_row_c2r_growth(fgeo_, d_U_, src, dst, d_S_, p, s);
            });
            if (e != cudaSuccess) return cudaFail(e, "growth pass");
            spectrum_valid_ = true;
        } else {
            e = launch(LENIA_PHASE_DIRECT, s, [&] {
                return launch_direct_step(direct_tile_, direct_nk_, src, dst, d_weights_, d_spans_, dgeo_, p, s,
                                          &direct_tma_, cur_, direct_split_, direct_ox_, direct_oy_);
            });
            if (e != cudaSuccess) return cudaFail(e, "direct step");
        }
        cur_ ^= 1;
    }
    return LENIA_OK;
}

void LeniaModule::info(lenia_info* o) const {
    std::memset(o, 0, sizeof(*o));
    o->sim_width = w_;
    o->sim_height = h_;
    o->conv_mode = use_fft_ ? LENIA_CONV_FFT : direct_multi_ ? LENIA_CONV_DIRECT_MULTI : LENIA_CONV_DIRECT;
    o->radius = radius_;
    o->num_kernels = num_k_;
    o->use_stamp_init = use_stamp_ ? 1u : 0u;
    o->device_bytes = device_bytes_;
    o->fft_precision = tc_precision_;
    o->tc_engine = tc_precision_ == LENIA_FFT_FP32 ? 0u
                   : tc_batch_ == kTcgen05          ? 2u
                   : tc_batch_ == kTcgen05Pipelined ? 3u
                                                    : 1u;
    o->direct_tma = (!use_fft_ && direct_tma_.on) ? 1u : 0u;
    o->direct_split = use_fft_ ? 0u : uint32_t(direct_split_);
    o->direct_outputs_per_thread = use_fft_ ? 0u : uint32_t(direct_ox_);
    o->direct_rows_per_thread = use_fft_ ? 0u : uint32_t(direct_oy_);
    o->direct_taps = use_fft_ ? 0u : direct_taps_;
    if (use_fft_) {
        for (int i = 0; i < fgeo_.row.npass && i < 8; ++i) o->fft_radix_row[i] = uint32_t(fgeo_.row.radix[i]);
        for (int i = 0; i < fgeo_.col.npass && i < 8; ++i) o->fft_radix_col[i] = uint32_t(fgeo_.col.radix[i]);
    }
}

}  // namespace lenia
