// life_simulation_b200/csrc/lenia_capi.cpp -- the extern "C" boundary
// declared in include/lenia_b200.h. No C++ exception crosses it: every entry
// point converts failures into a status code and a per-context message.
#include <cuda_runtime.h>

#include <cstring>
#include <new>
#include <string>

#include "../../include/lenia_b200.h"
#include "lenia_module.h"

struct lenia_ctx {
    lenia::LeniaModule module;
    lenia::ParameterTable params;
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
        // Scene::applyBaseParams (Scene.cpp:96-113).
        for (const auto& m : j.members()) {
            if (m.second.is_number()) c->params.setBase(m.first, float(m.second.as_number()));
            else if (m.second.is_bool()) c->params.setBase(m.first, m.second.as_bool() ? 1.0f : 0.0f);
        }
        c->module.configure("lenia0", std::move(mc));
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
        c->params.setBase(key, value);
        return int(LENIA_OK);
    });
}

int lenia_set_override(lenia_ctx* c, const char* key, float value) {
    if (!c || !key) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->params.setOverride(key, value);
        return int(LENIA_OK);
    });
}

int lenia_clear_override(lenia_ctx* c, const char* key) {
    if (!c || !key) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->params.clearOverride(key);
        return int(LENIA_OK);
    });
}

int lenia_resolve_frame_params(lenia_ctx* c, uint32_t frame_index, uint32_t audio_frame,
                               lenia_frame_params* out) {
    if (!c || !out) return LENIA_ERR_INVALID_ARG;
    *out = c->module.resolveFrameParams(c->params, frame_index, audio_frame);
    return LENIA_OK;
}

int lenia_encode(lenia_ctx* c, uint32_t frame_index, uint32_t substeps, uint32_t audio_frame,
                 void* stream) {
    if (!c) return LENIA_ERR_INVALID_ARG;
    return guarded(c, [&] {
        c->module.updateCPU(audio_frame);
        return set_msg(c, c->module.encode(frame_index, substeps, c->params,
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
    return LENIA_OK;
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
