// life_simulation_b200/csrc/lenia_noalloc.cu -- one spectral-path substep
// that allocates no device memory (lenia_fft_step_noalloc in
// include/lenia_b200.h).
//
// Who needs it: callers that cannot allocate device memory at the point they
// step the field -- a real-time frame callback, where cudaMalloc/cudaFree can
// synchronise the whole device and stall the frame, or a host application that
// reserves the GPU's memory up front and only hands out its own buffers. They
// pass the field in and out as their own device buffers; everything else the
// step needs (row spectrum, per-kernel potentials, kernel spectra, twiddle
// tables) lives in one fixed-size static device array below, which every GPU
// that loads this library holds until the process exits.
//
// The array's host-side name is not a device address: the device address is
// fetched with cudaGetSymbolAddress (with the device current) on every call --
// it is cheap -- and the kernels receive that pointer. If it differs from the
// address the tables were uploaded to (the context was torn down and the
// module reloaded, e.g. after cudaDeviceReset), the tables are rebuilt.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/lenia_b200.h"
#include "abi_guard.h"
#include "lenia_kernels.h"
#include "lenia_module.h"

namespace {

// The scratch every no-allocation call shares (LENIA_NOALLOC_SCRATCH_BYTES).
__device__ __align__(256) unsigned char g_noalloc_scratch[LENIA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

// Launch shape of the compile-time-plan passes (columns / rows per CTA).
constexpr int kColsPerCta = 4;
constexpr int kRowsPerCta = 2;

struct DeviceScratch {
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch the tables were put in
    std::string key;                // field size + kernel shapes the tables hold
};

std::mutex g_mu;
DeviceScratch g_dev[kMaxDevices];
thread_local std::string g_noalloc_error;

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

int fail(int code, std::string msg) {
    g_noalloc_error = std::move(msg);
    return code;
}

}  // namespace

extern "C" const char* lenia_noalloc_last_message(void) { return g_noalloc_error.c_str(); }

namespace {

int step_noalloc(const float* field_in, float* field_out, uint32_t width, uint32_t height, const lenia_config* cfg,
                 const lenia_frame_params* fp, uint32_t seed, void* stream) {
    using namespace lenia;
    if (!field_in || !field_out || !cfg || !fp)
        return fail(LENIA_ERR_INVALID_ARG, "null argument");
    if (field_in == field_out) return fail(LENIA_ERR_INVALID_ARG, "field_in and field_out must differ");
    // The row pass stages the field with 16-byte asynchronous copies.
    if ((reinterpret_cast<uintptr_t>(field_in) | reinterpret_cast<uintptr_t>(field_out)) & 15u)
        return fail(LENIA_ERR_INVALID_ARG, "field_in and field_out must be 16-byte aligned");
    FftPlan prow{}, pcol{};
    if (width < 2 || (width & 1u) || height < 1 || !fft_plan(int(width / 2), prow) || !fft_plan(int(height), pcol))
        return fail(LENIA_ERR_UNSUPPORTED,
                    "field size needs an even width and sizes with factors 2, 3, 5 only");
    // More than 4 kernels are truncated to the first 4, as the module's setup
    // does (Lenia.cpp:225-230).
    const uint32_t num_kernels = std::min<uint32_t>(cfg->num_kernels, 4u);

    // Kernels: the config's, or one implicit kernel (Lenia.cpp:503-512).
    struct K {
        float scale, mu, sigma, weight;
        std::vector<float> betas;
    };
    std::vector<K> ks;
    for (uint32_t i = 0; i < num_kernels; ++i) {
        const lenia_kernel_def& d = cfg->kernels[i];
        if (d.num_betas > 8) return fail(LENIA_ERR_UNSUPPORTED, "a kernel has more than 8 betas");
        if (!(d.sigma != 0.0f)) return fail(LENIA_ERR_INVALID_ARG, "a kernel's sigma must be nonzero");
        K k{d.radius_scale, d.mu, d.sigma, d.weight, std::vector<float>(d.betas, d.betas + d.num_betas)};
        if (k.betas.empty()) k.betas.push_back(1.0f);
        ks.push_back(std::move(k));
    }
    if (ks.empty()) {
        if (!(fp->growth_sigma != 0.0f)) return fail(LENIA_ERR_INVALID_ARG, "growth_sigma must be nonzero");
        ks.push_back(K{1.0f, fp->growth_mu, fp->growth_sigma, 1.0f, {1.0f}});
    }
    const int nk = int(ks.size());
    const uint32_t radius = cfg->radius;

    const int M = int(width / 2), H = int(height), Hh = H / 2 + 1;
    FastPlan cf, ri;
    // Compile-time-plan kernels at 4 columns and 2 rows per CTA where the
    // catalogue has the size and that launch shape fits; else the
    // runtime-plan kernels.
    const bool fast = fast_col_plan(H, cf) && fast_row_plan(M, ri) && M % kSpectralBlock == 0 &&
                      fast_shapes_supported(H, M, kColsPerCta, kRowsPerCta);

    // Scratch layout (256-byte aligned regions).
    const size_t spec = size_t(M) * H * sizeof(float2);
    std::vector<float2> tw_row, tw_col, tw_r2c, f_cf, f_ci, f_ri, f_rf;
    fill_twiddles(M, tw_row);
    fill_twiddles(H, tw_col);
    fill_twiddles(int(width), tw_r2c);
    tw_r2c.resize(size_t(M) + 1);
    if (fast) {
        FastPlan rcf = cf, rri = ri;
        for (int i = 0; i < cf.np; ++i) rcf.radix[i] = cf.radix[cf.np - 1 - i];
        for (int i = 0; i < ri.np; ++i) rri.radix[i] = ri.radix[ri.np - 1 - i];
        fast_plan_twiddles(cf, f_cf);
        fast_plan_twiddles(rcf, f_ci);
        fast_plan_twiddles(ri, f_ri);
        fast_plan_twiddles(rri, f_rf);
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align256(off + std::max<size_t>(bytes, 1));
        return o;
    };
    const size_t o_S = take(spec);
    const size_t o_U = take(spec * nk);
    const size_t o_kh = take(size_t(nk) * (M + 1) * Hh * sizeof(float));
    const size_t o_twr = take(tw_row.size() * sizeof(float2));
    const size_t o_twc = take(tw_col.size() * sizeof(float2));
    const size_t o_tw2 = take(tw_r2c.size() * sizeof(float2));
    const size_t o_fcf = take(f_cf.size() * sizeof(float2));
    const size_t o_fci = take(f_ci.size() * sizeof(float2));
    const size_t o_fri = take(f_ri.size() * sizeof(float2));
    const size_t o_frf = take(f_rf.size() * sizeof(float2));
    if (off > size_t(LENIA_NOALLOC_SCRATCH_BYTES))
        return fail(LENIA_ERR_UNSUPPORTED,
                    "field too large for the no-allocation scratch (" + std::to_string(off) + " bytes needed, " +
                        std::to_string(LENIA_NOALLOC_SCRATCH_BYTES) + " available)");

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return fail(LENIA_ERR_NO_DEVICE, "no CUDA device");
    const cudaStream_t s = static_cast<cudaStream_t>(stream);

    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch& d = g_dev[dev];
    {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return fail(LENIA_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        if (p != d.base) d.key.clear();  // a new module instance: its array holds no tables yet
        d.base = static_cast<unsigned char*>(p);
    }

    // Tables depend on the field size and the kernel shapes only; rebuild and
    // copy them in (synchronously on `stream`) when those change.
    std::string key = std::to_string(width) + "x" + std::to_string(height) + "|" + std::to_string(radius) + "|" +
                      std::to_string(cfg->kernel_core) + "|";
    {
        char buf[64];
        std::snprintf(buf, sizeof buf, "%a|", double(cfg->kernel_shell_sigma));
        key += buf;
        for (const K& k : ks) {
            std::snprintf(buf, sizeof buf, "%a:", double(k.scale));
            key += buf;
            for (float b : k.betas) {
                std::snprintf(buf, sizeof buf, "%a,", double(b));
                key += buf;
            }
            key += ";";
        }
    }
    unsigned char* base = d.base;
    if (d.key != key) {
        std::vector<float> khat(size_t(nk) * (M + 1) * Hh), img, sp;
        for (int k = 0; k < nk; ++k) {
            build_ring_image(width, height, float(radius) * ks[k].scale, cfg->kernel_shell_sigma, ks[k].betas,
                             cfg->kernel_core, img);
            kernel_spectrum(img, width, height, sp);
            std::copy(sp.begin(), sp.end(), khat.begin() + size_t(k) * (M + 1) * Hh);
        }
        auto put = [&](size_t o, const void* src, size_t bytes) {
            return bytes ? cudaMemcpyAsync(base + o, src, bytes, cudaMemcpyHostToDevice, s) : cudaSuccess;
        };
        cudaError_t e = put(o_kh, khat.data(), khat.size() * sizeof(float));
        if (e == cudaSuccess) e = put(o_twr, tw_row.data(), tw_row.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_twc, tw_col.data(), tw_col.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_tw2, tw_r2c.data(), tw_r2c.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_fcf, f_cf.data(), f_cf.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_fci, f_ci.data(), f_ci.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_fri, f_ri.data(), f_ri.size() * sizeof(float2));
        if (e == cudaSuccess) e = put(o_frf, f_rf.data(), f_rf.size() * sizeof(float2));
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // host tables go out of scope
        if (e != cudaSuccess) {
            d.key.clear();
            return fail(LENIA_ERR_CUDA, std::string("table upload: ") + cudaGetErrorString(e));
        }
        d.key = key;
    }

    FftGeometry g{};
    g.W = int(width);
    g.H = H;
    g.M = M;
    g.row = prow;
    g.col = pcol;
    g.tw_row = reinterpret_cast<const float2*>(base + o_twr);
    g.tw_col = reinterpret_cast<const float2*>(base + o_twc);
    g.tw_r2c = reinterpret_cast<const float2*>(base + o_tw2);
    g.khat = reinterpret_cast<const float*>(base + o_kh);
    g.nk = nk;
    // Runtime-plan batch sizes as the module chooses them (shared-memory fit).
    int rb = 4;
    while (rb > 1 && sizeof(float2) * (size_t(2 * M + 1) + 2 * size_t(rb) * M) + sizeof(float) * size_t(rb) * width >
                         110 * 1024)
        rb /= 2;
    g.rows_per_cta = rb;
    g.cols_per_cta = 1;
    FastTables t{};
    t.col_twf = reinterpret_cast<const float2*>(base + o_fcf);
    t.col_twi = reinterpret_cast<const float2*>(base + o_fci);
    t.row_twi = reinterpret_cast<const float2*>(base + o_fri);
    t.row_twf = reinterpret_cast<const float2*>(base + o_frf);
    float2* S = reinterpret_cast<float2*>(base + o_S);
    float2* U = reinterpret_cast<float2*>(base + o_U);

    StepParams p;
    std::memset(&p, 0, sizeof p);
    p.dt = fp->dt;
    p.num_kernels = uint32_t(nk);
    float sw = 0.0f;
    for (int k = 0; k < 4; ++k) {
        p.mu[k] = k < nk ? ks[k].mu : 0.15f;
        p.sigma[k] = k < nk ? ks[k].sigma : 0.017f;
        p.weight[k] = k < nk ? ks[k].weight : 0.0f;
        if (k < nk) sw += ks[k].weight;
    }
    p.sum_weights = sw;
    p.growth_mode = fp->growth_mode;
    p.noise_amount = fp->noise_amount;
    p.mu_jitter = fp->mu_jitter;
    p.inject_amount = fp->inject_amount;
    p.inject_count = fp->inject_count;
    p.radius = radius;
    p.seed = seed;
    p.width = width;
    p.height = height;
    p.frame_index = fp->frame_index;
    p.audio_frame = fp->audio_frame;

    cudaError_t e;
    if (fast) {
        e = launch_row_fast(g, t, kRowsPerCta, nullptr, field_in, nullptr, S, p, 0, s);
        if (e == cudaSuccess) e = launch_col_fast(g, t, kColsPerCta, S, U, s);
        if (e == cudaSuccess) e = launch_row_fast(g, t, kRowsPerCta, U, field_in, field_out, nullptr, p, nk, s);
    } else {
        e = launch_row_r2c(g, field_in, S, s);
        if (e == cudaSuccess) e = launch_col_conv(g, S, U, s);
        if (e == cudaSuccess) e = launch_row_c2r_growth(g, U, field_in, field_out, nullptr, p, s);
    }
    if (e != cudaSuccess) return fail(LENIA_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    g_noalloc_error.clear();
    return LENIA_OK;
}

}  // namespace

// No C++ exception leaves the C ABI: a failed host allocation (the kernel
// spectra are built in host vectors) or any other exception becomes a status.
extern "C" int lenia_fft_step_noalloc(const float* field_in, float* field_out, uint32_t width,
                                      uint32_t height, const lenia_config* cfg,
                                      const lenia_frame_params* fp, uint32_t seed, void* stream) {
    return lenia::abi_guard(&g_noalloc_error,
                            [&] { return step_noalloc(field_in, field_out, width, height, cfg, fp, seed, stream); });
}
