// life_simulation_b200/csrc/lenia_batch.cu -- many independent Lenia worlds
// of uneven sizes and parameters stepped together (the batched sweep form;
// the reference sweeps variants one SceneRunner at a time,
// Apps/LifePresetLab/main.cpp:718-795).
//
// Two launch forms of a substep, whichever the autotuner measures faster:
//   * persistent (lenia_batch_persistent.cu): ONE launch over a device work
//     list of every world's column groups, direct tiles and row groups; row
//     groups wait on per-world counters for their world's column groups, and
//     the last CTA advances every world's substep seed and frame index;
//   * per size: one direct launch over a flat tile list of every direct
//     world, and for each field size with spectral worlds one column-pass and
//     one row-pass launch over a world table (blockIdx.y = world), then a tiny
//     kernel advances the seeds and frame indices.
// Either way a CUDA graph captured once replays any number of substeps.
// Worlds never interact; a world's result is the same as stepping it alone
// through a single-world context.
//
// Path choice (the autotuner): at creation the direct kernel's cost per
// pixel-tap and each size's spectral-step cost per pixel are measured on the
// batch's own buffers; each world takes the cheaper path for its radius.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/lenia_b200.h"
#include "abi_guard.h"
#include "colormap.cuh"
#include "lenia_device.cuh"
#include "lenia_kernels.h"
#include "lenia_module.h"

namespace lenia {
namespace {

// After a substep: every world's frame index + 1 and its next substep seed
// pcgHash(seed ^ (frame * 197)) (Modules/FieldModules/Lenia.cpp:564), written
// into both parity tables' copies of its parameters (loc[2*i], loc[2*i+1]).
__global__ void advance_kernel(StepParams* const* loc, int n, const uint32_t* base_seed, uint32_t* frame) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t f = frame[i] + 1u;
    frame[i] = f;
    const uint32_t seed = pcg_hash(base_seed[i] ^ (f * 197u));
    for (int k = 0; k < 2; ++k) {
        StepParams* p = loc[2 * i + k];
        p->frame_index = f;
        p->audio_frame = f;
        p->seed = seed;
    }
}

// Per-world sum and sum of squares of the current field (FP64 accumulation).
__global__ void stats_kernel(const float* const* fields, const int* npx, double* out, int n) {
    const int w = blockIdx.y;
    if (w >= n) return;
    const float* f = fields[w];
    const int count = npx[w];
    double s = 0.0, s2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const double v = double(f[i]);
        s += v;
        s2 += v * v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 2 * w, s);
        atomicAdd(out + 2 * w + 1, s2);
    }
}

// Per-world luma statistics of the colour layer (Apps/LifePresetLab/
// main.cpp:61-82): each pixel's RGBA16F palette texel, luma 0.2126 R +
// 0.7152 G + 0.0722 B of the halves in double; sum and sum of squares.
__global__ void activity_kernel(const float* const* fields, const int* npx, ColorMapParams cm, double* out, int n) {
    const int w = blockIdx.y;
    if (w >= n) return;
    const float* f = fields[w];
    const int count = npx[w];
    double s = 0.0, s2 = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        __half px[4];
        palette_rgba16f(cm, channel_of(f[i], cm.channel), px);
        const double l = 0.2126 * double(__half2float(px[0])) + 0.7152 * double(__half2float(px[1])) +
                         0.0722 * double(__half2float(px[2]));
        s += l;
        s2 += l * l;
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, o);
        s2 += __shfl_down_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(out + 2 * w, s);
        atomicAdd(out + 2 * w + 1, s2);
    }
}

uint32_t nnz_taps(const std::vector<float>& lut) {
    uint32_t n = 0;
    for (float v : lut) n += v != 0.0f;
    return n;
}

}  // namespace

struct BatchContext {
    std::vector<lenia_world> worlds;
    std::vector<int> path;        // LENIA_CONV_DIRECT or LENIA_CONV_FFT per world
    std::vector<size_t> field_off;  // offset of the world's two fields (floats)
    float* fields = nullptr;      // all worlds, [field0 | field1] per world
    int cur = 0;                  // which half holds the current state
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string message;

    // Direct worlds.
    float* d_wts = nullptr;
    uint32_t* d_spans = nullptr;
    DirectWorld* d_dtab[2] = {nullptr, nullptr};
    int3* d_tiles = nullptr;
    int ntiles = 0, max_r = 0;
    std::vector<int> direct_ids;

    // Spectral worlds, per size class.
    struct SizeClass {
        int W, H, M;
        std::vector<int> ids;
        float2* S = nullptr;   // per world M*H
        float2* U = nullptr;   // per world M*H (one kernel)
        float* khat = nullptr; // per world (M+1)*(H/2+1)
        float2* tw_r2c = nullptr;
        float2* tw[4] = {nullptr, nullptr, nullptr, nullptr};
        FastTables t{};
        SpectralWorld* d_stab[2] = {nullptr, nullptr};  // steady state
        SpectralWorld* d_r2c[2] = {nullptr, nullptr};   // row spectrum of the current state
        int col_batch = 4, row_batch = 2;
    };
    std::vector<SizeClass> classes;

    // Where each world's parameters live in the two parity tables, and the
    // device-side seed/frame state.
    StepParams** d_param_loc = nullptr;  // [2 * n]
    uint32_t* d_base_seed = nullptr;
    uint32_t* d_frame = nullptr;
    bool spectra_valid = false;

    // Stats.
    const float** d_field_ptrs[2] = {nullptr, nullptr};
    int* d_npx = nullptr;
    double* d_stats = nullptr;

    // The persistent form (lenia_batch_persistent.cu): one launch per
    // substep over a work list per parity; usable when every spectral world's
    // size has a persistent body. `persistent` is the form in use.
    bool persist_ok = false, persistent = false;
    PersistItem* d_items[2] = {nullptr, nullptr};
    int nitems = 0;
    uint32_t* d_ctl = nullptr;  // 2 counter sets of kPersistCtlHead + n words
    int* d_err = nullptr;       // set when a row item's wait ran out
    size_t persist_smem = 0;
    int persist_grid_n = 0;

    // Captured graphs by substep count and parity.
    std::map<std::pair<uint32_t, int>, cudaGraphExec_t> graphs;
    std::vector<void*> allocs;

    template <typename T>
    cudaError_t alloc(T** p, size_t count) {
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) allocs.push_back(*p);
        return e;
    }
    ~BatchContext() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        for (void* p : allocs) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
    }

    // Each field starts on a 256-byte boundary (the row passes stage fields
    // with 16-byte asynchronous copies; a world of odd size before it must
    // not shift it).
    static size_t field_stride(const lenia_world& w) { return (size_t(w.width) * w.height + 63) / 64 * 64; }
    float* field(int w, int half) { return fields + field_off[size_t(w)] + size_t(half) * field_stride(worlds[w]); }

    int fail(int code, std::string m) {
        message = std::move(m);
        return code;
    }

    cudaError_t launch_step(int parity, cudaStream_t s, bool advance = true);
    cudaError_t launch_r2c(int parity, cudaStream_t s);
    int build_persistent(const std::vector<int>& slot_of);
    void drop_graphs() {
        for (auto& g : graphs) cudaGraphExecDestroy(g.second);
        graphs.clear();
    }
};

namespace {

StepParams world_params(const lenia_world& w) {
    StepParams p;
    std::memset(&p, 0, sizeof p);
    p.dt = w.dt;
    p.num_kernels = 1;
    p.mu[0] = w.mu;
    p.sigma[0] = w.sigma;
    p.weight[0] = 1.0f;
    p.sum_weights = 1.0f;
    p.growth_mode = w.growth_mode;
    p.radius = w.radius;
    p.width = w.width;
    p.height = w.height;
    p.seed = pcg_hash_host(derive_seed(w.seed, 0x4C454E31u) ^ 0u);
    return p;
}

}  // namespace

// One substep of every world. The per-size form leaves the seed advance to
// advance_kernel (launched by the caller); the persistent form does it in
// its last CTA unless `advance` is false (timing).
cudaError_t BatchContext::launch_step(int parity, cudaStream_t s, bool advance) {
    if (persistent)
        return launch_persistent(d_items[parity], nitems, d_ctl, int(worlds.size()), parity, d_param_loc, d_base_seed,
                                 d_frame, advance, d_err, persist_smem, persist_grid_n, s);
    cudaError_t e = cudaSuccess;
    if (ntiles > 0) e = launch_direct_worlds(d_dtab[parity], d_tiles, ntiles, max_r, s);
    for (auto& c : classes) {
        if (e != cudaSuccess) break;
        const int n = int(c.ids.size());
        e = launch_col_fast_worlds(c.H, c.M, c.t, c.col_batch, c.d_stab[parity], n, s);
        if (e == cudaSuccess) e = launch_row_fast_worlds(c.H, c.M, c.t, c.tw_r2c, c.row_batch, c.d_stab[parity], n, s);
    }
    return e;
}

cudaError_t BatchContext::launch_r2c(int parity, cudaStream_t s) {
    cudaError_t e = cudaSuccess;
    for (auto& c : classes) {
        if (e != cudaSuccess) break;
        e = launch_row_fast_worlds(c.H, c.M, c.t, c.tw_r2c, c.row_batch, c.d_r2c[parity], int(c.ids.size()), s);
    }
    return e;
}

// Work lists of the persistent form, one per table parity: every column
// item (world by world, each world's groups in order), then the direct
// tiles, then every row item in the same world order -- a row item comes
// after all column items of its world, which is what its wait relies on.
// Returns LENIA_OK with persist_ok false when some spectral size has no
// persistent body.
int BatchContext::build_persistent(const std::vector<int>& slot_of) {
    persist_ok = false;
    std::vector<int> col_h, row_m;
    for (auto& c : classes) {
        if (persist_col_group(c.H) == 0 || persist_row_group(c.M) == 0) return LENIA_OK;
        col_h.push_back(c.H);
        row_m.push_back(c.M);
    }
    const int n = int(worlds.size());
    // Groups per item: several consecutive column (row) groups share one
    // item's set-up (its descriptor, world entry and dependency check).
    int per_item = 4;
    if (const char* env = std::getenv("LENIA_PERSIST_GROUPS")) per_item = std::max(1, std::atoi(env));
    std::vector<PersistItem> items[2];
    for (int par = 0; par < 2; ++par) {
        std::vector<PersistItem> cols, rows;
        for (auto& c : classes) {
            const int B = persist_col_group(c.H) * per_item, RB = persist_row_group(c.M) * per_item;
            const int ncol = (c.M + B - 1) / B;
            for (int wi : c.ids) {
                PersistItem it{};
                it.world = c.d_stab[par] + slot_of[size_t(wi)];
                it.world_id = wi;
                it.kind = kPersistCol;
                it.count = per_item;
                it.shape = c.H;
                it.tw0 = c.t.col_twf;
                it.tw1 = c.t.col_twi;
                for (int g = 0; g < ncol; ++g) {
                    it.group = g * B;
                    cols.push_back(it);
                }
                it.kind = kPersistRow;
                it.shape = c.M;
                it.tw0 = c.t.row_twi;
                it.tw1 = c.t.row_twf;
                it.tw2 = c.tw_r2c;
                it.need = ncol;
                for (int y = 0; y < c.H; y += RB) {
                    it.group = y;
                    rows.push_back(it);
                }
            }
        }
        std::vector<PersistItem> direct;
        for (int wi : direct_ids) {
            const lenia_world& w = worlds[size_t(wi)];
            PersistItem it{};
            it.world = d_dtab[par] + slot_of[size_t(wi)];
            it.world_id = wi;
            it.kind = kPersistDirect;
            for (int ty = 0; ty < (int(w.height) + 31) / 32; ++ty)
                for (int tx = 0; tx < (int(w.width) + 63) / 64; ++tx) {
                    it.group = tx | (ty << 16);
                    direct.push_back(it);
                }
        }
        items[par] = cols;
        items[par].insert(items[par].end(), direct.begin(), direct.end());
        items[par].insert(items[par].end(), rows.begin(), rows.end());
    }
    nitems = int(items[0].size());
    if (nitems == 0) return LENIA_OK;
    persist_smem = persist_smem_bytes(col_h, row_m, direct_ids.empty() ? 0 : max_r);
    persist_grid_n = persist_grid(persist_smem);
    if (persist_grid_n <= 0) return LENIA_OK;
    for (int par = 0; par < 2; ++par) {
        if (alloc(&d_items[par], items[par].size()) != cudaSuccess) return LENIA_ERR_CUDA;
        cudaMemcpy(d_items[par], items[par].data(), items[par].size() * sizeof(PersistItem), cudaMemcpyHostToDevice);
    }
    if (alloc(&d_ctl, 2 * (size_t(kPersistCtlHead) + n)) != cudaSuccess || alloc(&d_err, 1) != cudaSuccess)
        return LENIA_ERR_CUDA;
    cudaMemset(d_ctl, 0, 2 * (size_t(kPersistCtlHead) + n) * sizeof(uint32_t));
    cudaMemset(d_err, 0, sizeof(int));
    persist_ok = true;
    return LENIA_OK;
}

}  // namespace lenia

struct lenia_batch {
    lenia::BatchContext ctx;
};

using lenia::BatchContext;

namespace {
// Message of the calling thread's last failed lenia_batch_create.
thread_local std::string g_batch_create_error;
}  // namespace

extern "C" {

int lenia_batch_create(const lenia_world* worlds, uint32_t n, uint32_t policy, lenia_batch** out) {
    g_batch_create_error.clear();
    std::unique_ptr<lenia_batch> holder;
    const int rc = lenia::abi_guard(&g_batch_create_error, [&]() -> int {
        using namespace lenia;
        if (!worlds || !out || n == 0) return LENIA_ERR_INVALID_ARG;
        *out = nullptr;
        holder = std::make_unique<lenia_batch>();
        BatchContext& b = holder->ctx;
        b.worlds.assign(worlds, worlds + n);
        if (cudaGetDevice(&b.device) != cudaSuccess) return LENIA_ERR_NO_DEVICE;
        cudaError_t e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return LENIA_ERR_CUDA;

        // Fields.
        size_t total = 0;
        b.field_off.resize(n);
        for (uint32_t i = 0; i < n; ++i) {
            const lenia_world& w = worlds[i];
            if (w.width < 1 || w.height < 1 || !(w.sigma != 0.0f)) return LENIA_ERR_INVALID_ARG;
            if (w.radius > uint32_t(kMaxRadius) && (w.width % 2 || w.width < 2)) return LENIA_ERR_UNSUPPORTED;
            b.field_off[i] = total;
            total += 2 * BatchContext::field_stride(w);
        }
        if ((e = b.alloc(&b.fields, total)) != cudaSuccess) return LENIA_ERR_CUDA;
        cudaMemsetAsync(b.fields, 0, total * sizeof(float), b.stream);

        // Which worlds can take which path.
        std::vector<bool> can_fft(n), can_direct(n);
        for (uint32_t i = 0; i < n; ++i) {
            const lenia_world& w = worlds[i];
            FastPlan cf, ri;
            can_fft[i] = w.width % 2 == 0 && fast_col_plan(int(w.height), cf) && fast_row_plan(int(w.width / 2), ri) &&
                         (w.width / 2) % kSpectralBlock == 0;
            can_direct[i] = w.radius <= uint32_t(kMaxRadius);
            if (!can_fft[i] && !can_direct[i]) {
                b.message = "world " + std::to_string(i) + ": radius > 32 needs a spectral size (see fast plans)";
                return LENIA_ERR_UNSUPPORTED;
            }
        }
        b.path.assign(n, LENIA_CONV_DIRECT);
        for (uint32_t i = 0; i < n; ++i) {
            if (policy == LENIA_BATCH_FFT && !can_fft[i]) return LENIA_ERR_UNSUPPORTED;
            if (policy == LENIA_BATCH_DIRECT && !can_direct[i]) return LENIA_ERR_UNSUPPORTED;
            b.path[i] = (policy == LENIA_BATCH_FFT || !can_direct[i]) ? LENIA_CONV_FFT : LENIA_CONV_DIRECT;
        }

        // Direct LUTs for every world that might take the direct path.
        std::vector<std::vector<float>> luts(n);
        std::vector<uint32_t> nnz(n, 0);
        for (uint32_t i = 0; i < n; ++i)
            if (can_direct[i]) {
                build_direct_lut(worlds[i].radius, worlds[i].shell_mu, worlds[i].shell_sigma, worlds[i].kernel_core,
                                 luts[i]);
                nnz[i] = nnz_taps(luts[i]);
            }

        // Spectral classes for every world that might take the spectral path.
        std::map<std::pair<int, int>, int> class_of;
        std::vector<int> cls(n, -1);
        for (uint32_t i = 0; i < n; ++i)
            if (can_fft[i]) {
                auto key = std::make_pair(int(worlds[i].width), int(worlds[i].height));
                auto it = class_of.find(key);
                if (it == class_of.end()) {
                    BatchContext::SizeClass c;
                    c.W = key.first;
                    c.H = key.second;
                    c.M = c.W / 2;
                    class_of[key] = int(b.classes.size());
                    b.classes.push_back(c);
                    it = class_of.find(key);
                }
                cls[i] = it->second;
            }

        // Per-world parameters and the substep seed base.
        std::vector<StepParams> params(n);
        std::vector<uint32_t> base_seed(n);
        for (uint32_t i = 0; i < n; ++i) {
            params[i] = world_params(worlds[i]);
            base_seed[i] = derive_seed(worlds[i].seed, 0x4C454E31u);
        }
        std::vector<std::vector<int>> class_members(b.classes.size());
        for (uint32_t i = 0; i < n; ++i)
            if (cls[i] >= 0) class_members[size_t(cls[i])].push_back(int(i));

        // Spectral resources of every candidate world of each size class.
        for (size_t ci = 0; ci < b.classes.size(); ++ci) {
            auto& c = b.classes[ci];
            const int cnt = int(class_members[ci].size());
            const size_t spec = size_t(c.M) * c.H;
            const int Hh = c.H / 2 + 1;
            if ((e = b.alloc(&c.S, spec * cnt)) != cudaSuccess) return LENIA_ERR_CUDA;
            if ((e = b.alloc(&c.U, spec * cnt)) != cudaSuccess) return LENIA_ERR_CUDA;
            if ((e = b.alloc(&c.khat, size_t(c.M + 1) * Hh * cnt)) != cudaSuccess) return LENIA_ERR_CUDA;
            std::vector<float> kh(size_t(c.M + 1) * Hh * cnt), img, sp;
            for (int k = 0; k < cnt; ++k) {
                const lenia_world& w = worlds[class_members[ci][size_t(k)]];
                build_ring_image(w.width, w.height, float(w.radius), w.shell_sigma, std::vector<float>{1.0f},
                                 w.kernel_core, img);
                kernel_spectrum(img, w.width, w.height, sp);
                std::copy(sp.begin(), sp.end(), kh.begin() + size_t(k) * (c.M + 1) * Hh);
            }
            cudaMemcpy(c.khat, kh.data(), kh.size() * sizeof(float), cudaMemcpyHostToDevice);
            std::vector<float2> t2;
            fill_twiddles(c.W, t2);
            t2.resize(size_t(c.M) + 1);
            if ((e = b.alloc(&c.tw_r2c, t2.size())) != cudaSuccess) return LENIA_ERR_CUDA;
            cudaMemcpy(c.tw_r2c, t2.data(), t2.size() * sizeof(float2), cudaMemcpyHostToDevice);
            FastPlan cf, ri;
            fast_col_plan(c.H, cf);
            fast_row_plan(c.M, ri);
            FastPlan rcf = cf, rri = ri;
            for (int i = 0; i < cf.np; ++i) rcf.radix[i] = cf.radix[cf.np - 1 - i];
            for (int i = 0; i < ri.np; ++i) rri.radix[i] = ri.radix[ri.np - 1 - i];
            const FastPlan* plans[4] = {&cf, &rcf, &ri, &rri};
            for (int q = 0; q < 4; ++q) {
                std::vector<float2> tw;
                fast_plan_twiddles(*plans[q], tw);
                if (tw.empty()) tw.push_back(make_float2(1.0f, 0.0f));
                if ((e = b.alloc(&c.tw[q], tw.size())) != cudaSuccess) return LENIA_ERR_CUDA;
                cudaMemcpy(c.tw[q], tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice);
            }
            c.t.col_twf = c.tw[0];
            c.t.col_twi = c.tw[1];
            c.t.row_twi = c.tw[2];
            c.t.row_twf = c.tw[3];
        }

        std::vector<int> slot_of(n, 0);
        // Direct tables for a set of worlds (both parities) and their tile list.
        auto build_direct = [&](const std::vector<int>& ids, DirectWorld** dtab, int3** dtiles, int* ntiles,
                                int* max_r) -> int {
            std::vector<float> all_w;
            std::vector<uint32_t> all_s;
            std::vector<DirectWorld> tab;
            std::vector<int3> tiles;
            std::vector<std::pair<size_t, size_t>> offs;
            *max_r = 0;
            for (int i : ids) {
                const int R = int(worlds[i].radius);
                DirectGeometry g{R, 2 * R + 1, (R + 3) / 4 * 4, 0};
                g.wp = 2 * g.xp + 8;
                const size_t wo = all_w.size(), so = all_s.size();
                all_w.resize(wo + size_t(g.ksize) * g.wp, 0.0f);
                all_s.resize(so + size_t(g.ksize), 128u);
                for (int dy = 0; dy < g.ksize; ++dy) {
                    int lo = 1 << 30, hi = -(1 << 30);
                    for (int dx = -R; dx <= R; ++dx) {
                        const float v = luts[size_t(i)][size_t(dy) * g.ksize + size_t(dx + R)];
                        all_w[wo + size_t(dy) * g.wp + size_t(dx + g.xp)] = v;
                        if (v != 0.0f) { lo = std::min(lo, dx); hi = std::max(hi, dx); }
                    }
                    if (lo <= hi) {
                        const int start = (lo >= 0) ? (lo / 4) * 4 : -((-lo + 3) / 4) * 4;
                        all_s[so + size_t(dy)] = uint32_t(start + 128) | (uint32_t((hi - start + 1 + 7) / 8) << 16);
                    }
                }
                offs.push_back({wo, so});
                DirectWorld dw{};
                dw.g = g;
                dw.p = params[size_t(i)];
                slot_of[size_t(i)] = int(tab.size());
                for (int ty = 0; ty < (int(worlds[i].height) + 15) / 16; ++ty)
                    for (int tx = 0; tx < (int(worlds[i].width) + 31) / 32; ++tx)
                        tiles.push_back(make_int3(int(tab.size()), tx, ty));
                tab.push_back(dw);
                *max_r = std::max(*max_r, R);
            }
            *ntiles = int(tiles.size());
            if (tab.empty()) return LENIA_OK;
            float* dw = nullptr;
            uint32_t* ds = nullptr;
            if (b.alloc(&dw, all_w.size()) != cudaSuccess || b.alloc(&ds, all_s.size()) != cudaSuccess ||
                b.alloc(dtiles, tiles.size()) != cudaSuccess || b.alloc(&dtab[0], tab.size()) != cudaSuccess ||
                b.alloc(&dtab[1], tab.size()) != cudaSuccess)
                return LENIA_ERR_CUDA;
            cudaMemcpy(dw, all_w.data(), all_w.size() * sizeof(float), cudaMemcpyHostToDevice);
            cudaMemcpy(ds, all_s.data(), all_s.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
            cudaMemcpy(*dtiles, tiles.data(), tiles.size() * sizeof(int3), cudaMemcpyHostToDevice);
            for (int par = 0; par < 2; ++par) {
                std::vector<DirectWorld> t2 = tab;
                for (size_t k = 0; k < t2.size(); ++k) {
                    t2[k].weights = dw + offs[k].first;
                    t2[k].spans = ds + offs[k].second;
                    t2[k].src = b.field(ids[k], par);
                    t2[k].dst = b.field(ids[k], par ^ 1);
                }
                cudaMemcpy(dtab[par], t2.data(), t2.size() * sizeof(DirectWorld), cudaMemcpyHostToDevice);
            }
            return LENIA_OK;
        };
        // Spectral tables of one class for a subset of its candidate worlds.
        auto build_spectral = [&](size_t ci, const std::vector<int>& ids, SpectralWorld** stab, SpectralWorld** r2c) -> int {
            auto& c = b.classes[ci];
            const size_t spec = size_t(c.M) * c.H;
            const int Hh = c.H / 2 + 1;
            std::vector<SpectralWorld> steady[2], rt[2];
            for (int wi : ids) {
                const size_t k = size_t(std::find(class_members[ci].begin(), class_members[ci].end(), wi) -
                                        class_members[ci].begin());
                slot_of[size_t(wi)] = int(steady[0].size());
                for (int par = 0; par < 2; ++par) {
                    SpectralWorld sw{};
                    sw.S = c.S + spec * k;
                    sw.U = c.U + spec * k;
                    sw.khat = c.khat + size_t(c.M + 1) * Hh * k;
                    sw.A = b.field(wi, par);
                    sw.A_out = b.field(wi, par ^ 1);
                    sw.S_next = c.S + spec * k;
                    sw.M = c.M;
                    sw.nk = 1;
                    sw.p = params[size_t(wi)];
                    steady[par].push_back(sw);
                    SpectralWorld r = sw;
                    r.nk = 0;  // row spectrum of A only
                    r.A_out = nullptr;
                    r.U = nullptr;
                    rt[par].push_back(r);
                }
            }
            if (ids.empty()) return LENIA_OK;
            for (int par = 0; par < 2; ++par) {
                if (b.alloc(&stab[par], steady[par].size()) != cudaSuccess || b.alloc(&r2c[par], rt[par].size()) != cudaSuccess)
                    return LENIA_ERR_CUDA;
                cudaMemcpy(stab[par], steady[par].data(), steady[par].size() * sizeof(SpectralWorld), cudaMemcpyHostToDevice);
                cudaMemcpy(r2c[par], rt[par].data(), rt[par].size() * sizeof(SpectralWorld), cudaMemcpyHostToDevice);
            }
            return LENIA_OK;
        };

        // Autotuner (policy AUTO): time the batched direct launch over every
        // direct candidate (cost per pixel-tap) and each class's spectral step
        // over all its candidates (cost per pixel) -- the batch's own launch
        // shapes, on its own buffers -- and give each world the cheaper path.
        if (policy == LENIA_BATCH_AUTO) {
            cudaEvent_t ea, eb;
            cudaEventCreate(&ea);
            cudaEventCreate(&eb);
            auto time_ms = [&](auto&& fn) {
                float best = 1e30f;
                for (int rep = 0; rep < 3; ++rep) {
                    cudaEventRecord(ea, b.stream);
                    if (fn() != cudaSuccess) return 1e30f;
                    cudaEventRecord(eb, b.stream);
                    cudaEventSynchronize(eb);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, ea, eb);
                    if (rep > 0) best = std::min(best, ms);
                }
                return best;
            };
            // Cost per tap of the batched direct launch over every candidate.
            // That launch sizes its halo tile for the largest radius it holds,
            // which overstates the cost for small radii; so candidates are also
            // timed in radius bands, each with its own halo, and a band with
            // enough work (>= 1e8 pixel-taps, so the launch itself is amortised)
            // uses its own figure.
            const auto band = [&](uint32_t i) { return worlds[i].radius <= 12u ? 0 : worlds[i].radius <= 20u ? 1 : 2; };
            std::vector<int> dall, dcand[3];
            double taps_all = 0.0, taps[3] = {0.0, 0.0, 0.0};
            for (uint32_t i = 0; i < n; ++i)
                if (can_direct[i] && can_fft[i]) {
                    const double t = double(worlds[i].width) * worlds[i].height * nnz[i];
                    dall.push_back(int(i));
                    dcand[band(i)].push_back(int(i));
                    taps_all += t;
                    taps[band(i)] += t;
                }
            const auto time_direct = [&](const std::vector<int>& ids, double t, double& out) {
                DirectWorld* dt[2] = {nullptr, nullptr};
                int3* tl = nullptr;
                int nt = 0, mr = 0;
                if (build_direct(ids, dt, &tl, &nt, &mr) < 0) return false;
                const float ms = time_ms([&] { return launch_direct_worlds(dt[0], tl, nt, mr, b.stream); });
                out = double(ms) / t;
                return true;
            };
            double cost_all = 0.0, cost_tap[3] = {0.0, 0.0, 0.0};
            if (!dall.empty() && !time_direct(dall, taps_all, cost_all)) return LENIA_ERR_CUDA;
            for (int bd = 0; bd < 3; ++bd) {
                cost_tap[bd] = cost_all;
                if (taps[bd] >= 1e8 && !time_direct(dcand[bd], taps[bd], cost_tap[bd])) return LENIA_ERR_CUDA;
            }
            std::vector<double> cost_px(b.classes.size(), 0.0);
            for (size_t ci = 0; ci < b.classes.size(); ++ci) {
                auto& c = b.classes[ci];
                SpectralWorld* st[2] = {nullptr, nullptr};
                SpectralWorld* rt[2] = {nullptr, nullptr};
                if (build_spectral(ci, class_members[ci], st, rt) < 0) return LENIA_ERR_CUDA;
                const int cnt = int(class_members[ci].size());
                const float ms = time_ms([&] {
                    cudaError_t r = launch_col_fast_worlds(c.H, c.M, c.t, c.col_batch, st[0], cnt, b.stream);
                    if (r == cudaSuccess) r = launch_row_fast_worlds(c.H, c.M, c.t, c.tw_r2c, c.row_batch, st[0], cnt, b.stream);
                    return r;
                });
                cost_px[ci] = double(ms) / (double(c.W) * c.H * cnt);
            }
            cudaEventDestroy(ea);
            cudaEventDestroy(eb);
            for (uint32_t i = 0; i < n; ++i)
                if (can_direct[i] && can_fft[i])
                    b.path[i] = (cost_tap[band(i)] * nnz[i] <= cost_px[size_t(cls[i])]) ? LENIA_CONV_DIRECT : LENIA_CONV_FFT;
            cudaMemsetAsync(b.fields, 0, total * sizeof(float), b.stream);
        }

        // Final tables.
        for (uint32_t i = 0; i < n; ++i)
            if (b.path[i] == LENIA_CONV_DIRECT) b.direct_ids.push_back(int(i));
        if (build_direct(b.direct_ids, b.d_dtab, &b.d_tiles, &b.ntiles, &b.max_r) < 0) return LENIA_ERR_CUDA;
        std::vector<BatchContext::SizeClass> kept;
        for (size_t ci = 0; ci < b.classes.size(); ++ci) {
            auto& c = b.classes[ci];
            for (int wi : class_members[ci])
                if (b.path[size_t(wi)] == LENIA_CONV_FFT) c.ids.push_back(wi);
            if (c.ids.empty()) continue;
            if (build_spectral(ci, c.ids, c.d_stab, c.d_r2c) < 0) return LENIA_ERR_CUDA;
            kept.push_back(c);
        }
        b.classes = kept;

        // Columns / rows per CTA iteration of each size's passes: every candidate
        // timed on the class's own tables (the fields are cleared afterwards).
        if (!b.classes.empty()) {
            cudaEvent_t ea, eb;
            cudaEventCreate(&ea);
            cudaEventCreate(&eb);
            auto time_ms = [&](auto&& fn) {
                float best = 1e30f;
                for (int rep = 0; rep < 3; ++rep) {
                    cudaEventRecord(ea, b.stream);
                    if (fn() != cudaSuccess) return 1e30f;
                    cudaEventRecord(eb, b.stream);
                    cudaEventSynchronize(eb);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, ea, eb);
                    if (rep > 0) best = std::min(best, ms);
                }
                return best;
            };
            for (auto& c : b.classes) {
                const int cnt = int(c.ids.size());
                float best = 1e30f;
                for (int cb : kColCandidates) {
                    const float ms = time_ms([&] { return launch_col_fast_worlds(c.H, c.M, c.t, cb, c.d_stab[0], cnt, b.stream); });
                    if (ms < 0.97f * best) { best = ms; c.col_batch = cb; }
                }
                best = 1e30f;
                for (int rb : kRowCandidates) {
                    const float ms = time_ms([&] {
                        return launch_row_fast_worlds(c.H, c.M, c.t, c.tw_r2c, rb, c.d_stab[0], cnt, b.stream);
                    });
                    if (ms < 0.97f * best) { best = ms; c.row_batch = rb; }
                }
            }
            cudaGetLastError();
            cudaEventDestroy(ea);
            cudaEventDestroy(eb);
            cudaMemsetAsync(b.fields, 0, total * sizeof(float), b.stream);
        }

        // Per-world seed/frame state and where each world's parameters live in
        // the two parity tables (device addresses, for the advance kernel).
        std::vector<StepParams*> loc(2 * size_t(n), nullptr);
        for (uint32_t i = 0; i < n; ++i)
            for (int par = 0; par < 2; ++par) {
                char* entry = nullptr;
                size_t member = 0;
                if (b.path[i] == LENIA_CONV_DIRECT) {
                    entry = reinterpret_cast<char*>(b.d_dtab[par] + slot_of[i]);
                    member = offsetof(DirectWorld, p);
                } else {
                    for (auto& c : b.classes)
                        if (c.W == int(worlds[i].width) && c.H == int(worlds[i].height))
                            entry = reinterpret_cast<char*>(c.d_stab[par] + slot_of[i]);
                    member = offsetof(SpectralWorld, p);
                }
                loc[2 * i + size_t(par)] = reinterpret_cast<StepParams*>(entry + member);
            }
        if (b.alloc(&b.d_param_loc, loc.size()) != cudaSuccess || b.alloc(&b.d_base_seed, n) != cudaSuccess ||
            b.alloc(&b.d_frame, n) != cudaSuccess)
            return LENIA_ERR_CUDA;
        cudaMemcpy(b.d_param_loc, loc.data(), loc.size() * sizeof(StepParams*), cudaMemcpyHostToDevice);
        cudaMemcpy(b.d_base_seed, base_seed.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice);
        cudaMemset(b.d_frame, 0, n * sizeof(uint32_t));


        // Stats tables.
        std::vector<const float*> fp0(n), fp1(n);
        std::vector<int> npx(n);
        for (uint32_t i = 0; i < n; ++i) {
            fp0[i] = b.field(int(i), 0);
            fp1[i] = b.field(int(i), 1);
            npx[i] = int(worlds[i].width * worlds[i].height);
        }
        if (b.alloc(&b.d_field_ptrs[0], n) != cudaSuccess || b.alloc(&b.d_field_ptrs[1], n) != cudaSuccess ||
            b.alloc(&b.d_npx, n) != cudaSuccess || b.alloc(&b.d_stats, 2 * size_t(n)) != cudaSuccess)
            return LENIA_ERR_CUDA;
        cudaMemcpy(b.d_field_ptrs[0], fp0.data(), n * sizeof(float*), cudaMemcpyHostToDevice);
        cudaMemcpy(b.d_field_ptrs[1], fp1.data(), n * sizeof(float*), cudaMemcpyHostToDevice);
        cudaMemcpy(b.d_npx, npx.data(), n * sizeof(int), cudaMemcpyHostToDevice);

        // Launch form: one persistent launch per substep where every spectral
        // size has a persistent body, else (or when slower) the per-size
        // launches. The autotuner times a few substeps of each on the batch's
        // own buffers (no seed advance; the fields are cleared afterwards);
        // LENIA_BATCH_PERSISTENT=0/1 forces the choice.
        {
            const int prc = b.build_persistent(slot_of);
            if (prc < 0) return prc;
            const char* env = std::getenv("LENIA_BATCH_PERSISTENT");
            if (b.persist_ok && env && env[0] == '0' && env[1] == '\0') {
                b.persistent = false;
            } else if (b.persist_ok && env && env[0] == '1' && env[1] == '\0') {
                b.persistent = true;
            } else if (b.persist_ok) {
                cudaEvent_t ea, eb;
                cudaEventCreate(&ea);
                cudaEventCreate(&eb);
                float ms[2] = {0.0f, 0.0f};
                for (int form = 0; form < 2; ++form) {
                    b.persistent = form == 1;
                    float best = 1e30f;
                    for (int rep = 0; rep < 4; ++rep) {
                        cudaEventRecord(ea, b.stream);
                        cudaError_t r = cudaSuccess;
                        for (int k = 0; k < 4 && r == cudaSuccess; ++k) r = b.launch_step(k & 1, b.stream, false);
                        cudaEventRecord(eb, b.stream);
                        cudaEventSynchronize(eb);
                        float t = 0.0f;
                        cudaEventElapsedTime(&t, ea, eb);
                        if (r != cudaSuccess) t = 1e30f;
                        if (rep > 0) best = std::min(best, t);
                    }
                    ms[form] = best;
                }
                cudaEventDestroy(ea);
                cudaEventDestroy(eb);
                b.persistent = ms[1] < ms[0];
                cudaGetLastError();
                cudaMemsetAsync(b.fields, 0, total * sizeof(float), b.stream);
            }
            if (b.persist_ok) {
                cudaMemsetAsync(b.d_ctl, 0, 2 * (size_t(kPersistCtlHead) + n) * sizeof(uint32_t), b.stream);
                cudaMemsetAsync(b.d_err, 0, sizeof(int), b.stream);
            }
        }

        cudaStreamSynchronize(b.stream);
        if ((e = cudaGetLastError()) != cudaSuccess) {
            b.message = std::string("batch setup: ") + cudaGetErrorString(e);
            return LENIA_ERR_CUDA;
        }
        *out = holder.release();
        return LENIA_OK;
    });
    // A failure the body reported on the batch it was building.
    if (rc < 0 && holder && g_batch_create_error.empty()) g_batch_create_error = holder->ctx.message;
    return rc;
}

int lenia_batch_destroy(lenia_batch* b) {
    return lenia::abi_guard(b ? &b->ctx.message : nullptr, [&]() -> int {
        if (!b) return LENIA_ERR_INVALID_ARG;
        delete b;
        return LENIA_OK;
    });
}

int lenia_batch_upload(lenia_batch* bb, uint32_t world, const float* host) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !host || world >= bb->ctx.worlds.size()) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        const lenia_world& w = b.worlds[world];
        cudaError_t e = cudaMemcpyAsync(b.field(int(world), b.cur), host, sizeof(float) * w.width * w.height,
                                        cudaMemcpyHostToDevice, b.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b.stream);
        b.spectra_valid = false;
        return e == cudaSuccess ? LENIA_OK : b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
    });
}

int lenia_batch_download(lenia_batch* bb, uint32_t world, float* host) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !host || world >= bb->ctx.worlds.size()) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        const lenia_world& w = b.worlds[world];
        cudaError_t e = cudaDeviceSynchronize();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(host, b.field(int(world), b.cur), sizeof(float) * w.width * w.height,
                                cudaMemcpyDeviceToHost, b.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b.stream);
        return e == cudaSuccess ? LENIA_OK : b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
    });
}

int lenia_batch_step(lenia_batch* bb, uint32_t steps, void* stream) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        using namespace lenia;
        if (!bb) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b.stream;
        const int n = int(b.worlds.size());
        cudaError_t e = cudaSuccess;
        if (!b.spectra_valid) {
            e = b.launch_r2c(b.cur, s);
            if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, std::string("row spectra: ") + cudaGetErrorString(e));
            b.spectra_valid = true;
        }
        if (steps == 0) return LENIA_OK;
        // The graph for (steps, parity): substeps alternate the parity of the
        // tables; after each, the device advances seeds and frames.
        const auto key = std::make_pair(steps, b.cur);
        auto it = b.graphs.find(key);
        if (it == b.graphs.end()) {
            cudaStream_t cap = b.stream;
            cudaGraph_t graph = nullptr;
            e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
            if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
            int par = b.cur;
            for (uint32_t k = 0; k < steps && e == cudaSuccess; ++k) {
                e = b.launch_step(par, cap);
                if (e == cudaSuccess && !b.persistent) {
                    advance_kernel<<<(n + 127) / 128, 128, 0, cap>>>(b.d_param_loc, n, b.d_base_seed, b.d_frame);
                    e = cudaGetLastError();
                }
                par ^= 1;
            }
            cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (e == cudaSuccess) e = e2;
            cudaGraphExec_t exec = nullptr;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
            if (graph) cudaGraphDestroy(graph);
            if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, std::string("graph: ") + cudaGetErrorString(e));
            it = b.graphs.emplace(key, exec).first;
        }
        e = cudaGraphLaunch(it->second, s);
        if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        if (steps % 2) b.cur ^= 1;
        return LENIA_OK;
    });
}

int lenia_batch_stats(lenia_batch* bb, double* mean, double* var) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !mean || !var) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        const int n = int(b.worlds.size());
        cudaError_t e = cudaMemsetAsync(b.d_stats, 0, sizeof(double) * 2 * n, b.stream);
        if (e == cudaSuccess) {
            lenia::stats_kernel<<<dim3(16, unsigned(n)), 256, 0, b.stream>>>(b.d_field_ptrs[b.cur], b.d_npx, b.d_stats, n);
            e = cudaGetLastError();
        }
        std::vector<double> h(2 * size_t(n));
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(h.data(), b.d_stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
        for (int i = 0; i < n; ++i) {
            const double cnt = double(b.worlds[size_t(i)].width) * b.worlds[size_t(i)].height;
            mean[i] = h[2 * size_t(i)] / cnt;
            var[i] = std::max(0.0, h[2 * size_t(i) + 1] / cnt - mean[i] * mean[i]);
        }
        return LENIA_OK;
    });
}

int lenia_batch_activity(lenia_batch* bb, const lenia_colormap* cm, double* mean_luma, double* stddev_luma) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !cm || !mean_luma || !stddev_luma) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        const int n = int(b.worlds.size());
        static_assert(sizeof(lenia_colormap) == sizeof(lenia::ColorMapParams), "colour map layout");
        lenia::ColorMapParams p;
        std::memcpy(&p, cm, sizeof(p));
        cudaError_t e = cudaMemsetAsync(b.d_stats, 0, sizeof(double) * 2 * n, b.stream);
        if (e == cudaSuccess) {
            lenia::activity_kernel<<<dim3(16, unsigned(n)), 256, 0, b.stream>>>(b.d_field_ptrs[b.cur], b.d_npx, p,
                                                                                b.d_stats, n);
            e = cudaGetLastError();
        }
        std::vector<double> h(2 * size_t(n));
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(h.data(), b.d_stats, h.size() * sizeof(double), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
        for (int i = 0; i < n; ++i) {
            const double cnt = double(b.worlds[size_t(i)].width) * b.worlds[size_t(i)].height;
            const double mean = h[2 * size_t(i)] / cnt;
            mean_luma[i] = mean;
            stddev_luma[i] = std::sqrt(std::max(0.0, h[2 * size_t(i) + 1] / cnt - mean * mean));
        }
        return LENIA_OK;
    });
}

int lenia_batch_init_noise(lenia_batch* bb, uint32_t world, uint32_t seed, float init_coverage, float init_scale) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || world >= bb->ctx.worlds.size()) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        const lenia_world& w = b.worlds[world];
        const lenia::InitParams ip{init_coverage, init_scale, lenia::derive_seed(seed, 0x4C454E31u), w.width, w.height};
        cudaError_t e = lenia::launch_init_noise(b.field(int(world), b.cur), ip, b.stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b.stream);
        b.spectra_valid = false;
        return e == cudaSuccess ? LENIA_OK : b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
    });
}

int lenia_batch_world_path(lenia_batch* bb, uint32_t world, uint32_t* path) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !path || world >= bb->ctx.worlds.size()) return LENIA_ERR_INVALID_ARG;
        *path = uint32_t(bb->ctx.path[world]);
        return LENIA_OK;
    });
}

int lenia_batch_sync(lenia_batch* bb) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
        if (b.d_err) {
            int flag = 0;
            e = cudaMemcpy(&flag, b.d_err, sizeof(int), cudaMemcpyDeviceToHost);
            if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
            if (flag) {
                cudaMemset(b.d_err, 0, sizeof(int));
                return b.fail(LENIA_ERR_CUDA,
                              "persistent batch: a row item's wait for its world's column items ran out "
                              "(those rows were not updated)");
            }
        }
        return LENIA_OK;
    });
}

int lenia_batch_launch_form(lenia_batch* bb, uint32_t* form) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || !form) return LENIA_ERR_INVALID_ARG;
        *form = bb->ctx.persistent ? LENIA_BATCH_FORM_PERSISTENT : LENIA_BATCH_FORM_PER_SIZE;
        return LENIA_OK;
    });
}

int lenia_batch_set_launch_form(lenia_batch* bb, uint32_t form) {
    return lenia::abi_guard(bb ? &bb->ctx.message : nullptr, [&]() -> int {
        if (!bb || form > LENIA_BATCH_FORM_PERSISTENT) return LENIA_ERR_INVALID_ARG;
        BatchContext& b = bb->ctx;
        if (form == LENIA_BATCH_FORM_PERSISTENT && !b.persist_ok)
            return b.fail(LENIA_ERR_UNSUPPORTED, "no persistent body for some spectral world size of this batch");
        const bool want = form == LENIA_BATCH_FORM_PERSISTENT;
        if (want != b.persistent) {
            // Graphs hold the other form's launches; the counter sets start clear.
            cudaError_t e = cudaStreamSynchronize(b.stream);
            if (e == cudaSuccess) e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return b.fail(LENIA_ERR_CUDA, cudaGetErrorString(e));
            b.drop_graphs();
            if (b.d_ctl)
                cudaMemset(b.d_ctl, 0, 2 * (size_t(lenia::kPersistCtlHead) + b.worlds.size()) * sizeof(uint32_t));
            b.persistent = want;
        }
        return LENIA_OK;
    });
}

// NULL: the calling thread's last failed lenia_batch_create.
const char* lenia_batch_last_message(lenia_batch* bb) {
    return bb ? bb->ctx.message.c_str() : g_batch_create_error.c_str();
}

}  // extern "C"
