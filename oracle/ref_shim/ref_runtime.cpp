// oracle/ref_shim/ref_runtime.cpp -- a CPU stand-in for the reference's GPU
// runtime, so that the reference's own host module (Modules/FieldModules/
// Lenia.cpp) and parameter bus (LifeCore/Params/ParameterBus.cpp) run
// unmodified on the host and drive the CPU-compiled reference shaders.
//
// TEST INFRASTRUCTURE ONLY. Built into oracle/_ref/ from the reference tree by
// oracle/Makefile; used by tests/golden/make_golden.py to produce fixtures, by
// the oracle cross-check tests, and by bench.py's reference arm. Never linked
// into the product.
//
// What is re-implemented here (declarations are the reference's own headers):
//   ResourcePool  LifeCore/Metal/ResourcePool.h:50-88  -> CPU images
//   CommandGraph  LifeCore/Metal/CommandGraph.h:63-107 -> runs each pass at once
//   ComputePass   LifeCore/Metal/CommandGraph.h:24-61  -> records binds
//   ColorMapPass  LifeCore/Render/ColorMapPass.h:67-  -> no-op (presentation)
// The session API at the bottom mirrors SceneRunner's per-frame flow for one
// Lenia module (LifeCore/Sim/SceneRunner.cpp:138-246): scene numeric params
// become ParameterBus bases (LifeCore/Params/Scene.cpp:96-113), then
// updateCPU(audio) and encode(ctx) once per frame.
#include "LifeCore/Metal/CommandGraph.h"
#include "LifeCore/Metal/ResourcePool.h"
#include "LifeCore/IO/NpyWriter.h"
#include "LifeCore/Params/ParameterBus.h"
#include "LifeCore/Params/Scene.h"
#include "LifeCore/Render/ColorMapPass.h"
#include "LifeCore/Sim/SimulationModule.h"
#include "Modules/FieldModules/Lenia.h"

#include "ref_kernels.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace life {

namespace {

uint32_t channelsOf(PixelFormat f) {
    switch (f) {
    case PixelFormat::R16F:
    case PixelFormat::R32F: return 1;
    case PixelFormat::RG16F:
    case PixelFormat::RG32F: return 2;
    default: return 4;
    }
}

struct CpuTexture {
    TextureDesc desc;
    std::vector<double> store;
    metal::CpuImage img;
    std::vector<float> lastUpload;  // the most recent CPU upload, as floats
};

}  // namespace

struct ResourcePool::Impl {
    std::vector<std::unique_ptr<CpuTexture>> textures;
    CpuTexture* get(TextureHandle h) {
        if (!h.valid() || h.index > textures.size()) return nullptr;
        return textures[h.index - 1].get();
    }
};

ResourcePool::ResourcePool(MetalContext&) : impl_(std::make_unique<Impl>()) {}
ResourcePool::~ResourcePool() = default;

TextureHandle ResourcePool::createTexture(const TextureDesc& desc) {
    auto t = std::make_unique<CpuTexture>();
    t->desc = desc;
    t->img.width = desc.width;
    t->img.height = desc.height;
    t->img.channels = channelsOf(desc.format);
    t->store.assign(size_t(desc.width) * desc.height * t->img.channels, 0.0);
    t->img.data = t->store.data();
    impl_->textures.push_back(std::move(t));
    TextureHandle h;
    h.index = uint32_t(impl_->textures.size());
    h.generation = 1;
    return h;
}

bool ResourcePool::uploadTexture(TextureHandle h, const void* data, size_t bytesPerRow) {
    CpuTexture* t = impl_->get(h);
    if (!t) return false;
    const uint32_t ch = t->img.channels;
    if (bytesPerRow != size_t(t->img.width) * ch * sizeof(float)) return false;
    const float* src = static_cast<const float*>(data);
    const size_t n = size_t(t->img.width) * t->img.height * ch;
    t->lastUpload.assign(src, src + n);
    for (size_t i = 0; i < n; ++i) t->store[i] = double(src[i]);
    return true;
}

struct CommandGraph::Impl {
    ResourcePool* pool = nullptr;
    std::vector<std::string> passLabels;
    // When set, an init pass writes this field instead of running its kernel
    // (used to start the reference from a caller-chosen initial state).
    const std::vector<float>* initOverride = nullptr;
    uint64_t passCount = 0;
    // Row window for the per-pixel update passes (leniaStep,
    // leniaGrowthMulti): a bounded sample of a step for CPU timing.
    uint32_t rowLo = 0, rowHi = ~0u;
};

CommandGraph::CommandGraph(MetalContext&, ResourcePool& pool, PipelineCache&)
    : impl_(std::make_unique<Impl>()) {
    impl_->pool = &pool;
}
CommandGraph::~CommandGraph() = default;

void CommandGraph::copyTexture(TextureHandle src, TextureHandle dst) {
    CpuTexture* s = impl_->pool->impl().get(src);
    CpuTexture* d = impl_->pool->impl().get(dst);
    if (!s || !d || s->store.size() != d->store.size()) {
        std::fprintf(stderr, "[ref] copyTexture: bad handles\n");
        std::abort();
    }
    d->store = s->store;
    d->img.data = d->store.data();
    impl_->passLabels.push_back("blit.copyTexture");
    impl_->passCount++;
}

void CommandGraph::dispatch(ComputePass& pass, uint32_t gridW, uint32_t gridH, uint32_t) {
    metal::CpuImage* tex[8] = {};
    const void* bytes[4] = {};
    size_t nbytes[4] = {};
    CpuTexture* writeTarget = nullptr;
    for (const auto& tb : pass.textures_) {
        CpuTexture* t = impl_->pool->impl().get(tb.handle);
        if (!t || tb.index < 0 || tb.index >= 8) {
            std::fprintf(stderr, "[ref] pass %s: bad texture bind\n", pass.label_.c_str());
            std::abort();
        }
        tex[tb.index] = &t->img;
        if (tb.index == 0) writeTarget = t;
    }
    for (const auto& bb : pass.bytes_) {
        if (bb.index < 0 || bb.index >= 4) std::abort();
        bytes[bb.index] = bb.data.data();
        nbytes[bb.index] = bb.data.size();
    }
    impl_->passLabels.push_back(pass.label_);
    impl_->passCount++;
    const bool isInit = pass.function_ == "leniaInit" || pass.function_ == "leniaStampInit";
    if (isInit && impl_->initOverride && writeTarget) {
        const auto& f = *impl_->initOverride;
        if (f.size() != size_t(writeTarget->img.width) * writeTarget->img.height) std::abort();
        for (size_t i = 0; i < f.size(); ++i) writeTarget->store[i] = double(f[i]);
        return;
    }
    const bool windowed = pass.function_ == "leniaStep" || pass.function_ == "leniaGrowthMulti";
    const uint32_t y0 = windowed ? impl_->rowLo : 0u, y1 = windowed ? impl_->rowHi : ~0u;
    if (!ref_dispatch(pass.function_, tex, bytes, nbytes, gridW, gridH, y0, y1)) {
        std::fprintf(stderr, "[ref] unknown pipeline %s\n", pass.function_.c_str());
        std::abort();
    }
}

ComputePass::ComputePass(CommandGraph& graph, std::string label)
    : graph_(graph), label_(std::move(label)) {}
ComputePass& ComputePass::pipeline(std::string functionName) {
    function_ = std::move(functionName);
    return *this;
}
ComputePass& ComputePass::read(int index, TextureHandle h) {
    textures_.push_back({index, h});
    return *this;
}
ComputePass& ComputePass::write(int index, TextureHandle h) {
    textures_.push_back({index, h});
    return *this;
}
ComputePass& ComputePass::bytes(int index, const void* data, size_t size) {
    const auto* p = static_cast<const uint8_t*>(data);
    bytes_.push_back({index, std::vector<uint8_t>(p, p + size)});
    return *this;
}
void ComputePass::dispatch2D(uint32_t width, uint32_t height) {
    graph_.dispatch(*this, width, height, 1);
}

// Presentation is out of scope for the oracle: the colour map is a no-op.
void ColorMapPass::configure(const nlohmann::json&) {}
void ColorMapPass::encode(CommandGraph&, const std::string&, TextureHandle, TextureHandle,
                          uint32_t, uint32_t, float) {}
void ColorMapPass::encodeScaled(CommandGraph&, const std::string&, TextureHandle, TextureHandle,
                                uint32_t, uint32_t, uint32_t, uint32_t) {}

}  // namespace life

// ---------------------------------------------------------------------------
// Session C API (ctypes-friendly).

namespace {

alignas(64) unsigned char g_dummyDevice[256];  // stands in for MetalContext/PipelineCache

struct RefSession {
    life::ResourcePool pool;
    life::CommandGraph graph;
    life::ParameterBus bus;
    life::LeniaModule module;
    life::SimulationContext ctx;
    std::string instance;
    std::vector<float> initOverride;
    double lastEncodeSeconds = 0.0;

    RefSession()
        : pool(*reinterpret_cast<life::MetalContext*>(g_dummyDevice)),
          graph(*reinterpret_cast<life::MetalContext*>(g_dummyDevice), pool,
                *reinterpret_cast<life::PipelineCache*>(g_dummyDevice)) {}
};

life::CpuTexture* texOf(RefSession* s, life::TextureHandle h) {
    return s->pool.impl().get(h);
}

}  // namespace

extern "C" {

// params_json: the module's scene "params" object. scene_w/h: scene resolution.
void* ref_create(const char* params_json, uint32_t scene_w, uint32_t scene_h,
                 const char* instance) {
    nlohmann::json j;
    try {
        j = nlohmann::json::parse(params_json);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[ref] params JSON parse error: %s\n", e.what());
        return nullptr;
    }
    auto* s = new RefSession();
    s->instance = instance ? instance : "lenia0";
    // Scene.cpp:96-113: numeric and boolean params become bus base values.
    for (auto it = j.begin(); it != j.end(); ++it) {
        if (it.value().is_number())
            s->bus.setBase(s->instance + "." + it.key(), it.value().get<float>());
        else if (it.value().is_boolean())
            s->bus.setBase(s->instance + "." + it.key(), it.value().get<bool>() ? 1.0f : 0.0f);
    }
    s->module.configure(s->instance, j);
    s->ctx.metal = nullptr;
    s->ctx.resources = &s->pool;
    s->ctx.params = &s->bus;
    s->ctx.graph = &s->graph;
    s->ctx.width = scene_w;
    s->ctx.height = scene_h;
    s->module.setup(s->ctx);
    return s;
}

void ref_destroy(void* h) { delete static_cast<RefSession*>(h); }

void ref_set_base(void* h, const char* key, float value) {
    auto* s = static_cast<RefSession*>(h);
    s->bus.setBase(s->instance + "." + key, value);
}

void ref_reset(void* h, uint32_t seed) { static_cast<RefSession*>(h)->module.reset(seed); }

// Makes the next init pass write `field` (sim_w*sim_h floats) instead of the
// noise/stamp kernel. NULL clears the override.
void ref_set_init_field(void* h, const float* field, size_t n) {
    auto* s = static_cast<RefSession*>(h);
    if (field) {
        s->initOverride.assign(field, field + n);
        s->graph.impl().initOverride = &s->initOverride;
    } else {
        s->initOverride.clear();
        s->graph.impl().initOverride = nullptr;
    }
}

// One SceneRunner frame for this module: updateCPU(audio) then encode(ctx).
void ref_encode(void* h, uint32_t frame_index, uint32_t substeps, uint32_t audio_frame_index) {
    auto* s = static_cast<RefSession*>(h);
    life::AudioFeatureState audio;
    audio.frameIndex = audio_frame_index;
    s->ctx.frameIndex = frame_index;
    s->ctx.substeps = substeps;
    s->module.updateCPU(audio);
    auto t0 = std::chrono::steady_clock::now();
    s->module.encode(s->ctx);
    auto t1 = std::chrono::steady_clock::now();
    s->lastEncodeSeconds = std::chrono::duration<double>(t1 - t0).count();
}

double ref_last_encode_seconds(void* h) { return static_cast<RefSession*>(h)->lastEncodeSeconds; }

void ref_field_size(void* h, uint32_t* w, uint32_t* hh) {
    auto* s = static_cast<RefSession*>(h);
    life::CpuTexture* t = texOf(s, s->module.outputField());
    *w = t ? t->img.width : 0;
    *hh = t ? t->img.height : 0;
}

// Copies the current state field (channel 0) to out (sim_w*sim_h floats).
int ref_get_field(void* h, float* out, size_t n) {
    auto* s = static_cast<RefSession*>(h);
    life::CpuTexture* t = texOf(s, s->module.outputField());
    if (!t || n != size_t(t->img.width) * t->img.height) return -1;
    for (size_t i = 0; i < n; ++i) out[i] = float(t->store[i * t->img.channels]);
    return 0;
}

// Overwrites the current state field (channel 0).
int ref_put_field(void* h, const float* in, size_t n) {
    auto* s = static_cast<RefSession*>(h);
    life::CpuTexture* t = texOf(s, s->module.outputField());
    if (!t || n != size_t(t->img.width) * t->img.height) return -1;
    for (size_t i = 0; i < n; ++i) t->store[i * t->img.channels] = double(in[i]);
    return 0;
}

// Fetches the most recent CPU upload into the texture whose label ends with
// `suffix` (e.g. ".kernel", ".kernelImageUpload"). Returns the element count
// (0 if none); copies at most cap floats.
size_t ref_get_upload(void* h, const char* suffix, float* out, size_t cap) {
    auto* s = static_cast<RefSession*>(h);
    const std::string suf(suffix);
    for (auto& t : s->pool.impl().textures) {
        const std::string& l = t->desc.label;
        if (l.size() >= suf.size() && l.compare(l.size() - suf.size(), suf.size(), suf) == 0) {
            size_t n = t->lastUpload.size();
            if (out) std::memcpy(out, t->lastUpload.data(), std::min(n, cap) * sizeof(float));
            return n;
        }
    }
    return 0;
}

// Copies the full contents (all channels) of the texture whose label ends
// with `suffix`. Returns the element count.
size_t ref_get_texture(void* h, const char* suffix, double* out, size_t cap) {
    auto* s = static_cast<RefSession*>(h);
    const std::string suf(suffix);
    for (auto& t : s->pool.impl().textures) {
        const std::string& l = t->desc.label;
        if (l.size() >= suf.size() && l.compare(l.size() - suf.size(), suf.size(), suf) == 0) {
            size_t n = t->store.size();
            if (out) std::memcpy(out, t->store.data(), std::min(n, cap) * sizeof(double));
            return n;
        }
    }
    return 0;
}

// Restricts the per-pixel update passes to rows [y0, y1) (a bounded timing
// sample of a step; rows outside keep their old values). y1 = 0: no window.
void ref_set_row_window(void* h, uint32_t y0, uint32_t y1) {
    auto* s = static_cast<RefSession*>(h);
    s->graph.impl().rowLo = y1 ? y0 : 0u;
    s->graph.impl().rowHi = y1 ? y1 : ~0u;
}

uint64_t ref_pass_count(void* h) { return static_cast<RefSession*>(h)->graph.impl().passCount; }

// Writes the label of pass i (in issue order) into buf; returns its length.
size_t ref_pass_label(void* h, uint64_t i, char* buf, size_t cap) {
    auto* s = static_cast<RefSession*>(h);
    const auto& v = s->graph.impl().passLabels;
    if (i >= v.size()) return 0;
    if (buf && cap) {
        size_t n = std::min(cap - 1, v[i].size());
        std::memcpy(buf, v[i].data(), n);
        buf[n] = 0;
    }
    return v[i].size();
}

void ref_clear_pass_log(void* h) {
    auto* s = static_cast<RefSession*>(h);
    s->graph.impl().passLabels.clear();
}

// ---- The reference's parameter bus alone (LifeCore/Params/ParameterBus.cpp,
// Scene.cpp), driven with synthetic per-frame inputs.
struct RefEventIn {
    char type[32];
    char curve[32];
    float curve_value;
    float progress;
    int32_t started, ended;
};
struct RefFeaturesIn {
    float env[5][5];   // kick, snare, hihat, perc, beat x raw, smoothed, peak, trigger, hold
    float scalars[7];  // rms, low, mid, high, centroid, flux, time
    float lanes[10];   // tension, intensity, wetRatio, kickGate, macroDensity, macroIntensity,
                       // masterRms, drumsRms, spatialActive, seEnv
    int32_t section_index;
    float section_energy, section_progress;
    int32_t section_changed;
    char section_role[32];
    int32_t num_events;
    RefEventIn events[4];
};

void* ref_bus_create(uint32_t seed) {
    auto* b = new life::ParameterBus();
    b->setSeed(seed);
    return b;
}
void ref_bus_destroy(void* b) { delete static_cast<life::ParameterBus*>(b); }

// Scene::parse + applyBaseParams; 0 or -1 with the message in err.
int ref_bus_load_scene(void* b, const char* json_text, char* err, size_t err_n) {
    std::string e;
    try {
        auto j = nlohmann::json::parse(json_text);
        auto sc = life::Scene::parse(j, e);
        if (!sc) {
            std::snprintf(err, err_n, "%s", e.c_str());
            return -1;
        }
        sc->applyBaseParams(*static_cast<life::ParameterBus*>(b));
    } catch (const std::exception& ex) {
        std::snprintf(err, err_n, "%s", ex.what());
        return -1;
    }
    return 0;
}

// Scene::parse's time-source check, then addMapping; 0 or -1.
int ref_bus_add_mapping(void* b, const char* source, const char* target, float in_min, float in_max,
                        float scale, float offset, float smoothing, const char* mode) {
    life::TimeSourceKind k;
    float per, ph;
    std::string e;
    if (!life::parseTimeSource(source, k, per, ph, e)) return -1;
    life::AudioMappingSpec m;
    m.source = source;
    m.target = target;
    m.inMin = in_min;
    m.inMax = in_max;
    m.scale = scale;
    m.offset = offset;
    m.smoothing = smoothing;
    m.mode = life::mappingModeFromString(mode);
    static_cast<life::ParameterBus*>(b)->addMapping(m);
    return 0;
}

void ref_bus_set_base(void* b, const char* key, float v) { static_cast<life::ParameterBus*>(b)->setBase(key, v); }
void ref_bus_set_override(void* b, const char* key, float v) {
    static_cast<life::ParameterBus*>(b)->setOverride(key, v);
}
void ref_bus_clear_override(void* b, const char* key) { static_cast<life::ParameterBus*>(b)->clearOverride(key); }

void ref_bus_update(void* b, const RefFeaturesIn* f, float dt) {
    life::MusicFeatureState m;
    life::ChannelEnvelope* envs[5] = {&m.audio.kickEnv, &m.audio.snareEnv, &m.audio.hihatEnv, &m.audio.percEnv,
                                      &m.audio.beatEnv};
    for (int c = 0; c < 5; ++c) *envs[c] = {f->env[c][0], f->env[c][1], f->env[c][2], f->env[c][3], f->env[c][4]};
    m.audio.rms = f->scalars[0];
    m.audio.low = f->scalars[1];
    m.audio.mid = f->scalars[2];
    m.audio.high = f->scalars[3];
    m.audio.centroid = f->scalars[4];
    m.audio.flux = f->scalars[5];
    m.audio.time = f->scalars[6];
    float* lanes[10] = {&m.lanes.tension, &m.lanes.intensity, &m.lanes.wetRatio, &m.lanes.kickGate,
                        &m.lanes.macroDensity, &m.lanes.macroIntensity, &m.lanes.masterRms, &m.lanes.drumsRms,
                        &m.lanes.spatialActive, &m.lanes.seEnv};
    for (int i = 0; i < 10; ++i) *lanes[i] = f->lanes[i];
    m.sectionIndex = f->section_index;
    m.sectionRole = f->section_role;
    m.sectionEnergy = f->section_energy;
    m.sectionProgress = f->section_progress;
    m.sectionChanged = f->section_changed != 0;
    std::vector<life::MusicEvent> defs(size_t(std::max(0, f->num_events)));
    for (int i = 0; i < f->num_events; ++i) {
        defs[i].type = f->events[i].type;
        defs[i].frameStart = 0;
        defs[i].frameEnd = 1;
        if (f->events[i].curve[0]) defs[i].curves.push_back({f->events[i].curve, {f->events[i].curve_value}});
    }
    for (int i = 0; i < f->num_events; ++i) {
        life::ActiveEvent a;
        a.def = &defs[i];
        a.progress = f->events[i].progress;
        a.justStarted = f->events[i].started != 0;
        a.justEnded = f->events[i].ended != 0;
        m.events.push_back(a);
    }
    m.frame = 0;
    static_cast<life::ParameterBus*>(b)->update(m, dt);
}

// The reference's colour map kernels (Shaders/Render/ColorMap.metal) on a
// w x h single-channel field into an ow x oh RGBA image (floats, before the
// RGBA16F rounding of the texture): colorMapField when the sizes agree, else
// colorMapFieldScaled, as ColorMapPass::encode / encodeScaled choose
// (Lenia.cpp:646-652). cm: the 16 scalars of ColorMapParams in order.
int ref_colormap(const float* field, uint32_t w, uint32_t h, const float* cm, float* rgba, uint32_t ow,
                 uint32_t oh) {
    std::vector<double> src(size_t(w) * h), dst(size_t(ow) * oh * 4);
    for (size_t i = 0; i < src.size(); ++i) src[i] = field[i];
    metal::CpuImage a{w, h, 1, src.data()}, b{ow, oh, 4, dst.data()};
    metal::CpuImage* tex[2] = {&a, &b};
    unsigned char params[16 * 4];
    std::memcpy(params, cm, sizeof(params));
    struct {
        uint32_t w, h;
    } sp{ow, oh};
    const void* bytes[2] = {params, &sp};
    const size_t nb[2] = {sizeof(params), sizeof(sp)};
    const bool same = ow == w && oh == h;
    if (!ref_dispatch(same ? "colorMapField" : "colorMapFieldScaled", tex, bytes, nb, ow, oh, 0, ~0u)) return -1;
    for (size_t i = 0; i < dst.size(); ++i) rgba[i] = float(dst[i]);
    return 0;
}

// The reference's .npy writer and reader (LifeCore/IO/NpyWriter.cpp); 0 or
// -1 with the message in err.
int ref_npy_write(const char* path, const float* data, size_t count, const uint32_t* shape, uint32_t ndim, char* err,
                  size_t err_n) {
    std::string e;
    if (!life::writeNPYFloat32(path, data, count, std::vector<uint32_t>(shape, shape + ndim), e)) {
        std::snprintf(err, err_n, "%s", e.c_str());
        return -1;
    }
    return 0;
}
int ref_npy_read(const char* path, const uint32_t* shape, uint32_t ndim, float* out, size_t count, char* err,
                 size_t err_n) {
    std::string e;
    std::vector<float> data;
    if (!life::readNPYFloat32(path, std::vector<uint32_t>(shape, shape + ndim), data, e)) {
        std::snprintf(err, err_n, "%s", e.c_str());
        return -1;
    }
    if (data.size() != count) return -1;
    std::memcpy(out, data.data(), count * sizeof(float));
    return 0;
}

// The bus a Lenia session reads its parameters from (not to be destroyed).
void* ref_session_bus(void* h) { return &static_cast<RefSession*>(h)->bus; }

float ref_bus_value(void* b, const char* key, float fallback) {
    return static_cast<life::ParameterBus*>(b)->value(key, fallback);
}

uint32_t ref_pcg(uint32_t v) { return ref_pcg_hash(v); }
float ref_rand(uint32_t px, uint32_t py, uint32_t tag, uint32_t seed) {
    return ref_rand01(px, py, tag, seed);
}

}  // extern "C"
