// life_simulation_b200/csrc/lenia_capi.cpp -- the extern "C" boundary
// declared in include/lenia_b200.h. No C++ exception crosses it: every entry
// point converts failures into a status code and a per-context message.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>

#include "../../include/lenia_b200.h"
#include "lenia_module.h"
#include "npy_io.h"

struct lenia_ctx {
    lenia::LeniaModule module;
    lenia::ParameterBus own_bus;               // used unless a shared bus is attached
    lenia::ParameterBus* bus = &own_bus;
    std::string message;
    std::string key(const char* k) const { return module.instance() + "." + k; }
};

// A parameter bus shared by the modules of a scene (SceneRunner's bus).
struct lenia_bus {
    lenia::ParameterBus bus;
    std::string message;
};

namespace {

// Message of the last failed create/inspect on this thread
// (lenia_last_message(NULL)).
thread_local std::string g_create_error;

int set_msg(lenia_ctx* c, int rc) {
    if (c) c->message = c->module.message();
    return rc;
}

template <typename F>
int guarded(lenia_ctx* c, F&& f) {
    try {
        return f();
    } catch (const std::bad_alloc&) {
        if (c) c->message = "host allocation failed";
        return LENIA_ERR_CUDA;
    } catch (const std::exception& e) {
        if (c) c->message = e.what();
        return LENIA_ERR_STATE;
    }
}

template <typename F>
int bus_guarded(lenia_bus* b, F&& f) {
    if (!b) return LENIA_ERR_INVALID_ARG;
    try {
        return f();
    } catch (const std::exception& e) {
        b->message = e.what();
        return LENIA_ERR_STATE;
    }
}

int finish_create(lenia_ctx* c, uint32_t w, uint32_t h, lenia_ctx** out) {
    const int rc = c->module.setup(w, h);
    c->message = c->module.message();
    if (rc < 0) {
        g_create_error = c->message;
        delete c;
        *out = nullptr;
        return rc;
    }
    *out = c;
    return rc;
}

}  // namespace

extern "C" {

void lenia_config_defaults(lenia_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->conv_mode = LENIA_CONV_DIRECT;
    c->radius = 13;
    c->kernel_core = LENIA_CORE_GAUSS_SHELL;
    c->kernel_shell_mu = 0.5f;
    c->kernel_shell_sigma = 0.15f;
    c->init_coverage = 0.4f;
    c->init_scale = 24.0f;
    c->init_mode = LENIA_INIT_NOISE;
    c->org_R = 13.0f;
    c->org_T = 10.0f;
    c->org_mu = 0.15f;
    c->org_sigma = 0.015f;
    c->stamp_count = 6;
    c->stamp_rotate = 1;
    c->use_organism_params = 1;
    for (auto& k : c->kernels) {
        k.radius_scale = 1.0f;
        k.mu = 0.15f;
        k.sigma = 0.017f;
        k.weight = 1.0f;
        k.num_betas = 1;
        k.betas[0] = 1.0f;
    }
}

int lenia_create(const lenia_config* cfg, uint32_t scene_w, uint32_t scene_h, lenia_ctx** out) {
    if (!cfg || !out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        lenia::ModuleConfig mc;
        std::string err;
        const int rc = lenia::config_from_struct(*cfg, mc, err);
        if (rc < 0) {
            g_create_error = err;
            return rc;
        }
        auto* c = new lenia_ctx();
        c->module.configure("lenia0", std::move(mc));
        const int r = finish_create(c, scene_w, scene_h, out);
        if (r < 0) g_create_error = "setup failed";
        return r;
    });
}

int lenia_create_json(const char* params_json, uint32_t scene_w, uint32_t scene_h,
                      const char* base_dir, lenia_ctx** out) {
    if (!params_json || !out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        std::string err;
        lenia::Json j = lenia::Json::parse(params_json, &err);
        if (!err.empty()) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        lenia::ModuleConfig mc;
        int rc = lenia::config_from_json(j, base_dir ? base_dir : "", mc, err);
        if (rc < 0) {
            g_create_error = err;
            return rc;
        }
        auto* c = new lenia_ctx();
        c->module.configure("lenia0", std::move(mc));
        // Scene::applyBaseParams (Scene.cpp:96-113).
        for (const auto& m : j.members()) {
            if (m.second.is_number()) c->own_bus.setBase(c->key(m.first.c_str()), float(m.second.as_number()));
            else if (m.second.is_bool()) c->own_bus.setBase(c->key(m.first.c_str()), m.second.as_bool() ? 1.0f : 0.0f);
        }
        return finish_create(c, scene_w, scene_h, out);
    });
}

int lenia_inspect_json(const char* params_json, uint32_t scene_w, uint32_t scene_h,
                       const char* base_dir, lenia_info* out) {
    if (!params_json || !out) return LENIA_ERR_INVALID_ARG;
    return guarded(nullptr, [&] {
        std::string err;
        lenia::Json j = lenia::Json::parse(params_json, &err);
        if (!err.empty()) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        lenia::ModuleConfig mc;
        int rc = lenia::config_from_json(j, base_dir ? base_dir : "", mc, err);
        if (rc < 0) {
            g_create_error = err;
            return rc;
        }
        lenia::LeniaModule m;
        m.configure("lenia0", std::move(mc));
        rc = m.resolve(scene_w, scene_h);
        g_create_error = m.message();
        if (rc >= 0) m.info(out);
        return rc;
    });
}

int lenia_destroy(lenia_ctx* c) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    delete c;
    return LENIA_OK;
}

int lenia_reset(lenia_ctx* c, uint32_t seed) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    c->module.reset(seed);
    return LENIA_OK;
}

int lenia_set_param(lenia_ctx* c, const char* key, float value) {
    if (!c || !key) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->bus->setBase(c->key(key), value);
        return int(LENIA_OK);
    });
}

int lenia_set_override(lenia_ctx* c, const char* key, float value) {
    if (!c || !key) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->bus->setOverride(c->key(key), value);
        return int(LENIA_OK);
    });
}

int lenia_clear_override(lenia_ctx* c, const char* key) {
    if (!c || !key) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->bus->clearOverride(c->key(key));
        return int(LENIA_OK);
    });
}

int lenia_resolve_frame_params(lenia_ctx* c, uint32_t frame_index, uint32_t audio_frame,
                               lenia_frame_params* out) {
    if (!c || !out) return LENIA_ERR_INVALID_ARG;
    *out = c->module.resolveFrameParams(*c->bus, frame_index, audio_frame);
    return LENIA_OK;
}

int lenia_encode(lenia_ctx* c, uint32_t frame_index, uint32_t substeps, uint32_t audio_frame,
                 void* stream) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->module.updateCPU(audio_frame);
        return set_msg(c, c->module.encode(frame_index, substeps, *c->bus,
                                           static_cast<cudaStream_t>(stream)));
    });
}

int lenia_step(lenia_ctx* c, const lenia_frame_params* fp, uint32_t substeps, void* stream) {
    if (!c || !fp) return LENIA_ERR_INVALID_ARG;
    if (!(fp->growth_sigma != 0.0f)) {
        c->message = "growth_sigma must be nonzero";
        return LENIA_ERR_INVALID_ARG;
    }
    return guarded(c, [&] {
        return set_msg(c, c->module.step(*fp, substeps, static_cast<cudaStream_t>(stream)));
    });
}

int lenia_sync(lenia_ctx* c) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    cudaError_t e = cudaStreamSynchronize(c->module.stream());
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->message = std::string("device error: ") + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    return guarded(c, [&] { return set_msg(c, c->module.checkDeviceFlags()); });
}

int lenia_field_size(lenia_ctx* c, uint32_t* w, uint32_t* h) {
    if (!c || !w || !h) return LENIA_ERR_INVALID_ARG;
    *w = c->module.width();
    *h = c->module.height();
    return LENIA_OK;
}

int lenia_upload(lenia_ctx* c, const float* host, size_t count) {
    if (!c || !host) return LENIA_ERR_INVALID_ARG;
    if (count != size_t(c->module.width()) * c->module.height()) {
        c->message = "upload size does not match the field";
        return LENIA_ERR_INVALID_ARG;
    }
    cudaError_t e = cudaMemcpyAsync(c->module.mutableField(), host, count * sizeof(float),
                                    cudaMemcpyHostToDevice, c->module.stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->module.stream());
    if (e != cudaSuccess) {
        c->message = std::string("upload: ") + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    c->module.fieldWritten();
    return LENIA_OK;
}

int lenia_download(lenia_ctx* c, float* host, size_t count) {
    if (!c || !host) return LENIA_ERR_INVALID_ARG;
    if (count != size_t(c->module.width()) * c->module.height()) {
        c->message = "download size does not match the field";
        return LENIA_ERR_INVALID_ARG;
    }
    // Work may have been queued on a caller stream: wait for the device.
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host, c->module.outputField(), count * sizeof(float), cudaMemcpyDeviceToHost,
                            c->module.stream());
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->module.stream());
    if (e != cudaSuccess) {
        c->message = std::string("download: ") + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    return LENIA_OK;
}

int lenia_upload_device(lenia_ctx* c, const float* dev, size_t count, void* stream) {
    if (!c || !dev) return LENIA_ERR_INVALID_ARG;
    if (count != size_t(c->module.width()) * c->module.height()) return LENIA_ERR_INVALID_ARG;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->module.stream();
    cudaError_t e = cudaMemcpyAsync(c->module.mutableField(), dev, count * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
        c->message = std::string("upload_device: ") + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    c->module.fieldWritten();
    return LENIA_OK;
}

int lenia_download_device(lenia_ctx* c, float* dev, size_t count, void* stream) {
    if (!c || !dev) return LENIA_ERR_INVALID_ARG;
    if (count != size_t(c->module.width()) * c->module.height()) return LENIA_ERR_INVALID_ARG;
    cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->module.stream();
    cudaError_t e = cudaMemcpyAsync(dev, c->module.outputField(), count * sizeof(float),
                                    cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) {
        c->message = std::string("download_device: ") + cudaGetErrorString(e);
        return LENIA_ERR_CUDA;
    }
    return LENIA_OK;
}

int lenia_field_device_ptr(lenia_ctx* c, const float** dev) {
    if (!c || !dev) return LENIA_ERR_INVALID_ARG;
    *dev = c->module.outputField();
    return LENIA_OK;
}

int lenia_get_info(lenia_ctx* c, lenia_info* out) {
    if (!c || !out) return LENIA_ERR_INVALID_ARG;
    c->module.info(out);
    return LENIA_OK;
}

int lenia_get_stream(lenia_ctx* c, void** stream) {
    if (!c || !stream) return LENIA_ERR_INVALID_ARG;
    *stream = static_cast<void*>(c->module.stream());
    return LENIA_OK;
}

int lenia_profile(lenia_ctx* c, int enable) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->module.setProfiling(enable != 0);
        return int(LENIA_OK);
    });
}

int lenia_profile_read(lenia_ctx* c, lenia_profile_data* out) {
    if (!c || !out) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] { return c->module.readProfile(out); });
}

static_assert(LENIA_ROWS_PIPELINED == lenia::kRowPipelined, "pipelined row flag");
static_assert(LENIA_COLS_HALF_THREADS == lenia::kHalfThreads, "half-thread column flag");

int lenia_get_tuning(lenia_ctx* c, int* cols, int* rows) {
    if (!c || !cols || !rows) return LENIA_ERR_INVALID_ARG;
    c->module.tuning(cols, rows);
    return LENIA_OK;
}

int lenia_set_tuning(lenia_ctx* c, int cols, int rows) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] { return set_msg(c, c->module.setTuning(cols, rows)); });
}

// ---------------------------------------------------------- colour map

static_assert(sizeof(lenia_colormap) == sizeof(lenia::ColorMapParams), "colour map layout");

int lenia_get_colormap(lenia_ctx* c, lenia_colormap* out) {
    if (!c || !out) return LENIA_ERR_INVALID_ARG;
    std::memcpy(out, &c->module.colormap(), sizeof(*out));
    return LENIA_OK;
}

int lenia_set_colormap(lenia_ctx* c, const lenia_colormap* cm) {
    if (!c || !cm) return LENIA_ERR_INVALID_ARG;
    lenia::ColorMapParams p;
    std::memcpy(&p, cm, sizeof(p));
    c->module.setColormap(p);
    return LENIA_OK;
}

int lenia_colormap_from_json(const char* params_json, lenia_colormap* out) {
    if (!params_json || !out) return LENIA_ERR_INVALID_ARG;
    return guarded(nullptr, [&] {
        std::string err;
        const lenia::Json j = lenia::Json::parse(params_json, &err);
        if (!err.empty()) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        lenia::ColorMapParams p = lenia::lenia_default_colormap();
        lenia::colormap_from_json(j, p);
        std::memcpy(out, &p, sizeof(*out));
        return int(LENIA_OK);
    });
}

int lenia_render_rgba16f(lenia_ctx* c, void* dst, uint32_t width, uint32_t height, void* stream) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->module.stream();
        return set_msg(c, c->module.render(dst, width, height, s));
    });
}

int lenia_step_render(lenia_ctx* c, const lenia_frame_params* fp, uint32_t substeps, void* dst, uint32_t width,
                      uint32_t height, void* stream) {
    if (!c || !fp) return LENIA_ERR_INVALID_ARG;
    if (!(fp->growth_sigma != 0.0f)) {
        c->message = "growth_sigma must be nonzero";
        return LENIA_ERR_INVALID_ARG;
    }
    return guarded(c, [&] {
        return set_msg(c, c->module.stepRender(*fp, substeps, dst, width, height, static_cast<cudaStream_t>(stream)));
    });
}

// ---------------------------------------------------------- state files

int lenia_npy_write_f32(const char* path, const float* data, size_t count, const uint32_t* shape, uint32_t ndim) {
    if (!path || (!shape && ndim)) return LENIA_ERR_INVALID_ARG;
    return guarded(nullptr, [&] {
        std::string err;
        if (!lenia::write_npy_f32(path, data, count, std::vector<uint32_t>(shape, shape + ndim), err)) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        return int(LENIA_OK);
    });
}

int lenia_npy_read_f32(const char* path, const uint32_t* shape, uint32_t ndim, float* out, size_t count) {
    if (!path || !shape || !out) return LENIA_ERR_INVALID_ARG;
    return guarded(nullptr, [&] {
        std::string err;
        const std::vector<uint32_t> expected(shape, shape + ndim);
        size_t n = 1;
        for (uint32_t s : expected) n *= s;
        if (n != count) {
            g_create_error = "npy read: the expected shape does not hold `count` values";
            return int(LENIA_ERR_INVALID_ARG);
        }
        std::vector<float> data;
        if (!lenia::read_npy_f32(path, expected, data, err)) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        std::memcpy(out, data.data(), n * sizeof(float));
        return int(LENIA_OK);
    });
}

int lenia_save_state(lenia_ctx* c, const char* path) {
    if (!c || !path) return LENIA_ERR_INVALID_ARG;
    uint32_t w = 0, h = 0;
    lenia_field_size(c, &w, &h);
    std::vector<float> host(size_t(w) * h);
    int rc = lenia_download(c, host.data(), host.size());
    if (rc < 0) return rc;
    return guarded(c, [&] {
        std::string err;
        if (!lenia::write_npy_f32(path, host.data(), host.size(), {h, w}, err)) {
            c->message = err;
            return int(LENIA_ERR_PARSE);
        }
        return int(LENIA_OK);
    });
}

int lenia_load_state(lenia_ctx* c, const char* path) {
    if (!c || !path) return LENIA_ERR_INVALID_ARG;
    uint32_t w = 0, h = 0;
    lenia_field_size(c, &w, &h);
    std::vector<float> host;
    const int rc = guarded(c, [&] {
        std::string err;
        if (!lenia::read_npy_f32(path, {h, w}, host, err)) {
            c->message = err;
            return int(LENIA_ERR_PARSE);
        }
        return int(LENIA_OK);
    });
    if (rc < 0) return rc;
    return lenia_upload(c, host.data(), host.size());
}

// ---------------------------------------------------------------- the bus

int lenia_bus_create(uint32_t seed, lenia_bus** out) {
    if (!out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    auto* b = new (std::nothrow) lenia_bus();
    if (!b) return LENIA_ERR_STATE;
    b->bus.setSeed(seed);
    *out = b;
    return LENIA_OK;
}

int lenia_bus_destroy(lenia_bus* b) {
    if (!b) return LENIA_ERR_INVALID_ARG;
    delete b;
    return LENIA_OK;
}

int lenia_bus_load_scene(lenia_bus* b, const char* scene_json, lenia_scene_info* info) {
    if (!scene_json) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        std::string err;
        const lenia::Json j = lenia::Json::parse(scene_json, &err);
        lenia::SceneDoc sc;
        if (!err.empty() || !lenia::parse_scene(j, sc, err)) {
            b->message = err;
            return int(LENIA_ERR_PARSE);
        }
        if (!lenia::apply_scene(sc, b->bus, err)) {
            b->message = err;
            return int(LENIA_ERR_PARSE);
        }
        if (info) {
            info->seed = sc.seed;
            info->width = sc.width;
            info->height = sc.height;
            info->num_modules = uint32_t(sc.modules.size());
            info->num_mappings = uint32_t(sc.mappings.size());
        }
        return int(LENIA_OK);
    });
}

int lenia_bus_add_mapping(lenia_bus* b, const lenia_mapping* m) {
    if (!m || !m->source || !m->target || !m->source[0] || !m->target[0] || m->mode > LENIA_MAP_MUL)
        return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        lenia::MappingSpec spec;
        spec.source = m->source;
        spec.target = m->target;
        spec.in_min = m->in_min;
        spec.in_max = m->in_max;
        spec.scale = m->scale;
        spec.offset = m->offset;
        spec.smoothing = m->smoothing;
        spec.mode = lenia::MapMode(m->mode);
        std::string err;
        if (!b->bus.addMapping(spec, err)) {
            b->message = err;
            return int(LENIA_ERR_INVALID_ARG);
        }
        return int(LENIA_OK);
    });
}

int lenia_bus_set_base(lenia_bus* b, const char* key, float value) {
    if (!key) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        b->bus.setBase(key, value);
        return int(LENIA_OK);
    });
}

int lenia_bus_set_override(lenia_bus* b, const char* key, float value) {
    if (!key) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        b->bus.setOverride(key, value);
        return int(LENIA_OK);
    });
}

int lenia_bus_clear_override(lenia_bus* b, const char* key) {
    if (!key) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        b->bus.clearOverride(key);
        return int(LENIA_OK);
    });
}

int lenia_bus_set_feature(lenia_bus* b, const char* name, float value) {
    if (!name) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        b->bus.setFeature(name, value);
        return int(LENIA_OK);
    });
}

int lenia_bus_set_section(lenia_bus* b, const char* role, int32_t index) {
    return bus_guarded(b, [&] {
        b->bus.setSection(role ? role : "", index);
        return int(LENIA_OK);
    });
}

int lenia_bus_clear_features(lenia_bus* b) {
    return bus_guarded(b, [&] {
        b->bus.clearFeatures();
        return int(LENIA_OK);
    });
}

int lenia_bus_update(lenia_bus* b, float dt) {
    return bus_guarded(b, [&] {
        b->bus.update(dt);
        return int(LENIA_OK);
    });
}

int lenia_bus_value(lenia_bus* b, const char* key, float fallback, float* out) {
    if (!key || !out) return LENIA_ERR_INVALID_ARG;
    return bus_guarded(b, [&] {
        *out = b->bus.value(key, fallback);
        return int(LENIA_OK);
    });
}

const char* lenia_bus_last_message(lenia_bus* b) { return b ? b->message.c_str() : ""; }

int lenia_create_scene_module(const char* scene_json, const char* module_name, lenia_bus* bus,
                              const char* base_dir, lenia_ctx** out) {
    if (!scene_json || !out) return LENIA_ERR_INVALID_ARG;
    *out = nullptr;
    return guarded(nullptr, [&] {
        std::string err;
        const lenia::Json j = lenia::Json::parse(scene_json, &err);
        lenia::SceneDoc sc;
        if (!err.empty() || !lenia::parse_scene(j, sc, err)) {
            g_create_error = err;
            return int(LENIA_ERR_PARSE);
        }
        const lenia::SceneModule* mod = nullptr;
        for (const auto& m : sc.modules)
            if (module_name ? m.name == module_name : m.type == "Lenia") {
                mod = &m;
                break;
            }
        if (!mod) {
            g_create_error = module_name ? "scene has no module named \"" + std::string(module_name) + "\""
                                         : std::string("scene has no module of type \"Lenia\"");
            return int(LENIA_ERR_INVALID_ARG);
        }
        if (mod->type != "Lenia") {
            g_create_error = "module \"" + mod->name + "\" has type \"" + mod->type + "\", not \"Lenia\"";
            return int(LENIA_ERR_INVALID_ARG);
        }
        lenia::ModuleConfig mc;
        int rc = lenia::config_from_json(mod->params, base_dir ? base_dir : "", mc, err);
        if (rc < 0) {
            g_create_error = err;
            return rc;
        }
        auto* c = new lenia_ctx();
        c->module.configure(mod->name, std::move(mc));
        if (bus) {
            c->bus = &bus->bus;
        } else if (!lenia::apply_scene(sc, c->own_bus, err)) {
            g_create_error = err;
            delete c;
            return int(LENIA_ERR_PARSE);
        }
        return finish_create(c, sc.width, sc.height, out);
    });
}

int lenia_attach_bus(lenia_ctx* c, lenia_bus* b) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    c->bus = b ? &b->bus : &c->own_bus;
    return LENIA_OK;
}

const char* lenia_last_message(lenia_ctx* c) {
    if (!c) return g_create_error.c_str();
    return c->message.c_str();
}

const char* lenia_status_string(int s) {
    switch (s) {
    case LENIA_OK: return "ok";
    case LENIA_WARN_FALLBACK: return "ok, with a reference fallback";
    case LENIA_ERR_INVALID_ARG: return "invalid argument";
    case LENIA_ERR_UNSUPPORTED: return "unsupported size or parameter";
    case LENIA_ERR_CUDA: return "CUDA error";
    case LENIA_ERR_TIMEOUT: return "device wait timed out";
    case LENIA_ERR_STATE: return "invalid state";
    case LENIA_ERR_NO_DEVICE: return "no CUDA device";
    case LENIA_ERR_PARSE: return "parameter JSON could not be parsed";
    default: return "unknown status";
    }
}

}  // extern "C"
