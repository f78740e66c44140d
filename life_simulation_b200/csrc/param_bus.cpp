// life_simulation_b200/csrc/param_bus.cpp -- parameter bus and scene loader
// (the reference's LifeCore/Params/ParameterBus.cpp and Scene.cpp contract).
#include "param_bus.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>

namespace lenia {

uint32_t pcg_hash_host(uint32_t v);
uint32_t derive_seed(uint32_t global_seed, uint32_t tag);

namespace {

// FNV-1a (32 bit): turns a time source's text into its noise stream's tag.
uint32_t fnv1a(const std::string& s) {
    uint32_t h = 2166136261u;
    for (unsigned char c : s) {
        h ^= c;
        h *= 16777619u;
    }
    return h;
}

// A [0, 1] value per (seed, knot index), from the PCG hash.
float knot_value(uint32_t seed, int64_t index) {
    const uint32_t h = pcg_hash_host(seed ^ pcg_hash_host(uint32_t(index)));
    return float(h) * (1.0f / 4294967295.0f);
}

// A time source at bus time t (ParameterBus.cpp evalTimeSource): the cycle
// position is reduced in double before narrowing, so hours of run time keep
// their phase.
float eval_time(TimeKind kind, float period, float phase, uint32_t noise_seed, double t) {
    if (!(period > 0.0f)) return 0.0f;
    constexpr float kTwoPi = 6.28318530717958647692f;
    const double wide = t / double(period) + double(phase);
    const float x = float(wide - std::floor(wide));
    switch (kind) {
        case TimeKind::Sin: return std::sin(kTwoPi * x);
        case TimeKind::Tri: return (2.0f / 3.14159265358979323846f) * std::asin(std::sin(kTwoPi * x));
        case TimeKind::Ramp: return x;
        case TimeKind::Noise: {
            // Smooth value noise: random knots every period, smoothstep between.
            const double k = std::floor(wide);
            const float f = float(wide - k);
            const float a = knot_value(noise_seed, int64_t(k)) * 2.0f - 1.0f;
            const float b = knot_value(noise_seed, int64_t(k) + 1) * 2.0f - 1.0f;
            const float s = f * f * (3.0f - 2.0f * f);
            return a + (b - a) * s;
        }
        default: return 0.0f;
    }
}

bool strict_float(const std::string& s, float& out) {
    if (s.empty()) return false;
    const char* b = s.c_str();
    char* e = nullptr;
    out = std::strtof(b, &e);
    return e == b + s.size();
}

bool is_envelope(const std::string& ch) {
    return ch == "kick" || ch == "snare" || ch == "hihat" || ch == "perc" || ch == "beat";
}
bool is_scalar_channel(const std::string& ch) {
    return ch == "rms" || ch == "low" || ch == "mid" || ch == "high" || ch == "centroid" || ch == "flux" ||
           ch == "time";
}

MapMode mode_from(const std::string& s) {
    if (s == "set") return MapMode::Set;
    if (s == "mul" || s == "multiply") return MapMode::Mul;
    return MapMode::Add;
}

}  // namespace

bool parse_time_source(const std::string& source, TimeKind& kind, float& period, float& phase,
                       std::string& error) {
    kind = TimeKind::None;
    period = phase = 0.0f;
    if (source.rfind("time.", 0) != 0) return true;
    const std::string rest = source.substr(5);
    const size_t colon = rest.find(':');
    if (colon == std::string::npos) {
        error = "malformed time source (expected \"time.<kind>:<period>\"): \"" + source + "\"";
        return false;
    }
    const std::string k = rest.substr(0, colon);
    std::string per = rest.substr(colon + 1), ph;
    if (const size_t at = per.find('@'); at != std::string::npos) {
        ph = per.substr(at + 1);
        per = per.substr(0, at);
    }
    TimeKind kd;
    if (k == "sin") kd = TimeKind::Sin;
    else if (k == "tri") kd = TimeKind::Tri;
    else if (k == "ramp") kd = TimeKind::Ramp;
    else if (k == "noise") kd = TimeKind::Noise;
    else {
        error = "unknown time source kind \"" + k + "\" in \"" + source + "\" (expected sin, tri, ramp or noise)";
        return false;
    }
    float p = 0.0f, f = 0.0f;
    if (!strict_float(per, p) || !(p > 0.0f)) {
        error = "invalid or non-positive period in time source \"" + source + "\"";
        return false;
    }
    if (!ph.empty() && !strict_float(ph, f)) {
        error = "invalid phase in time source \"" + source + "\"";
        return false;
    }
    kind = kd;
    period = p;
    phase = f;
    return true;
}

float ParameterBus::base(const std::string& key, float fallback) const {
    const auto it = base_.find(key);
    return it != base_.end() ? it->second : fallback;
}

bool ParameterBus::addMapping(const MappingSpec& spec, std::string& error) {
    MapState st;
    st.spec = spec;
    if (!parse_time_source(spec.source, st.kind, st.period, st.phase, error)) return false;
    if (st.kind != TimeKind::None) st.noise_seed = derive_seed(seed_, fnv1a(spec.source));
    specs_.push_back(spec);
    states_.push_back(st);
    return true;
}

void ParameterBus::setFeature(const std::string& name, float v) {
    // An envelope channel named without its part is its smoothed value.
    if (is_envelope(name)) features_[name + ".smoothed"] = v;
    else features_[name] = v;
}

void ParameterBus::clearFeatures() {
    features_.clear();
    section_role_.clear();
    section_index_ = -1;
}

float ParameterBus::featureValue(const std::string& name) const {
    const auto get = [&](const std::string& k) {
        const auto it = features_.find(k);
        return it != features_.end() ? it->second : 0.0f;
    };
    if (name.rfind("lane.", 0) == 0) return get(name);
    if (name.rfind("section.", 0) == 0) {
        const std::string w = name.substr(8);
        if (w.rfind("is:", 0) == 0) return section_role_ == w.substr(3) ? 1.0f : 0.0f;
        if (w.rfind("n:", 0) == 0) return section_index_ == std::atoi(w.c_str() + 2) ? 1.0f : 0.0f;
        if (w == "index") return float(section_index_);
        return get(name);
    }
    if (name.rfind("event:", 0) == 0) {
        const std::string rest = name.substr(6);
        const size_t dot = rest.find('.');
        const std::string type = dot == std::string::npos ? rest : rest.substr(0, dot);
        const bool active = get("event:" + type + ".active") != 0.0f;
        if (dot == std::string::npos || rest.substr(dot + 1) == "active") return active ? 1.0f : 0.0f;
        return active ? get(name) : 0.0f;
    }
    std::string channel = name, part = "smoothed";
    if (const size_t dot = name.find('.'); dot != std::string::npos) {
        channel = name.substr(0, dot);
        part = name.substr(dot + 1);
    }
    if (is_envelope(channel)) {
        if (part != "raw" && part != "peak" && part != "trigger" && part != "hold") part = "smoothed";
        return get(channel + "." + part);
    }
    if (is_scalar_channel(channel)) return get(channel);
    return 0.0f;
}

bool ParameterBus::sourceValue(const std::string& name, float& out) const {
    if (name.rfind("event:", 0) == 0) {
        const std::string rest = name.substr(6);
        const size_t dot = rest.find('.');
        if (dot != std::string::npos) {
            const std::string what = rest.substr(dot + 1);
            const bool meta = what == "active" || what == "started" || what == "ended" || what == "progress";
            if (!meta) {
                // An event's own curve has no value while the event is not running.
                const auto act = features_.find("event:" + rest.substr(0, dot) + ".active");
                if (act == features_.end() || act->second == 0.0f || !features_.count(name)) return false;
            }
        }
    }
    out = featureValue(name);
    return true;
}

void ParameterBus::update(float dt) {
    add_.clear();
    set_.clear();
    mul_.clear();
    for (MapState& ms : states_) {
        const MappingSpec& s = ms.spec;
        float v = 0.0f;
        if (ms.kind != TimeKind::None) {
            v = eval_time(ms.kind, ms.period, ms.phase, ms.noise_seed, clock_);
        } else if (!sourceValue(s.source, v)) {
            continue;  // no contribution at all this frame
        }
        if (s.in_max > s.in_min) v = std::clamp((v - s.in_min) / (s.in_max - s.in_min), 0.0f, 1.0f);
        v = v * s.scale + s.offset;
        if (s.smoothing > 1e-5f && ms.primed) {
            const float k = 1.0f - std::exp(-dt / s.smoothing);
            ms.smoothed += (v - ms.smoothed) * k;
        } else {
            ms.smoothed = v;  // the first value is taken as is (no ramp from 0)
        }
        ms.primed = true;
        switch (s.mode) {
            case MapMode::Set: set_[s.target] = ms.smoothed; break;  // the last one wins
            case MapMode::Mul: {
                const auto it = mul_.find(s.target);
                if (it == mul_.end()) mul_[s.target] = ms.smoothed;
                else it->second *= ms.smoothed;
                break;
            }
            default: add_[s.target] += ms.smoothed; break;
        }
    }
    clock_ += dt;
}

float ParameterBus::value(const std::string& key, float fallback) const {
    if (const auto it = override_.find(key); it != override_.end()) return it->second;
    float v;
    if (const auto it = set_.find(key); it != set_.end()) v = it->second;
    else v = base(key, fallback);
    if (const auto it = add_.find(key); it != add_.end()) v += it->second;
    if (const auto it = mul_.find(key); it != mul_.end()) v *= it->second;
    return v;
}

bool parse_scene(const Json& j, SceneDoc& out, std::string& error) {
    out = SceneDoc();
    if (!j.is_object()) {
        error = "scene must be a JSON object";
        return false;
    }
    out.seed = j.value_u32("seed", 1234u);
    if (const Json* r = j.find("resolution"); r && r->is_array() && r->size() == 2 && r->items()[0].is_number() &&
                                             r->items()[1].is_number()) {
        out.width = uint32_t(r->items()[0].as_number());
        out.height = uint32_t(r->items()[1].as_number());
    }
    if (const Json* ms = j.find("modules"); ms && ms->is_array()) {
        for (const Json& m : ms->items()) {
            SceneModule sm;
            sm.type = m.value_string("type", "");
            sm.name = m.value_string("name", sm.type);
            sm.enabled = m.value_bool("enabled", true);
            if (const Json* p = m.find("params"); p && p->is_object()) sm.params = *p;
            else sm.params = Json::parse("{}", nullptr);
            if (sm.type.empty()) {
                error = "module entry missing \"type\"";
                return false;
            }
            out.modules.push_back(std::move(sm));
        }
    }
    // audioMappings, musicMappings and automation share one form.
    for (const char* key : {"audioMappings", "musicMappings", "automation"}) {
        const Json* arr = j.find(key);
        if (!arr || !arr->is_array()) continue;
        for (const Json& a : arr->items()) {
            MappingSpec s;
            s.source = a.value_string("source", "");
            s.target = a.value_string("target", "");
            s.in_min = a.value_float("inMin", 0.0f);
            s.in_max = a.value_float("inMax", 0.0f);
            s.scale = a.value_float("scale", 1.0f);
            s.offset = a.value_float("offset", 0.0f);
            s.smoothing = a.value_float("smoothing", 0.0f);
            s.mode = mode_from(a.value_string("mode", "add"));
            if (s.source.empty() || s.target.empty()) {
                error = std::string(key) + " entry missing source/target";
                return false;
            }
            TimeKind k;
            float per, ph;
            std::string terr;
            if (!parse_time_source(s.source, k, per, ph, terr)) {
                error = std::string(key) + ": " + terr;
                return false;
            }
            out.mappings.push_back(std::move(s));
        }
    }
    return true;
}

bool apply_scene(const SceneDoc& scene, ParameterBus& bus, std::string& error) {
    bus.setSeed(scene.seed);  // before the mappings: time.noise seeds derive from it
    for (const SceneModule& m : scene.modules) {
        for (const auto& kv : m.params.members()) {
            if (kv.second.is_number()) bus.setBase(m.name + "." + kv.first, float(kv.second.as_number()));
            else if (kv.second.is_bool()) bus.setBase(m.name + "." + kv.first, kv.second.as_bool() ? 1.0f : 0.0f);
        }
    }
    for (const MappingSpec& s : scene.mappings)
        if (!bus.addMapping(s, error)) return false;
    return true;
}

}  // namespace lenia
