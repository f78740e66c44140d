// life_simulation_b200/csrc/param_bus.h -- the parameter bus the Lenia module
// reads its per-frame values from (the reference's ParameterBus,
// LifeCore/Params/ParameterBus.{h,cpp}), and the scene loader that fills it
// (LifeCore/Params/Scene.cpp).
//
// Final value of a key ("<module>.<param>"): the override if set, else
// ((set ?: base) + sum of adds) * product of muls, where set/add/mul come
// from the mappings evaluated by the last update(). A mapping reads a source
// (a named per-frame input value or a time source), normalises it to 0..1
// when in_max > in_min, applies scale and offset and exponential smoothing
// (time constant `smoothing` seconds), and contributes to its target in its
// mode. Sources with no value this frame (an event's own curve while the event
// is not running) contribute nothing.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "json_lite.h"

namespace lenia {

enum class MapMode : uint32_t { Add = 0, Set = 1, Mul = 2 };
enum class TimeKind : uint32_t { None = 0, Sin, Tri, Ramp, Noise };

struct MappingSpec {
    std::string source, target;
    float in_min = 0.0f, in_max = 0.0f;
    float scale = 1.0f, offset = 0.0f;
    float smoothing = 0.0f;
    MapMode mode = MapMode::Add;
};

// Parses "time.<sin|tri|ramp|noise>:<period>[@<phase>]" (ParameterBus.cpp
// parseTimeSource): sources not starting with "time." are kind None (true);
// a malformed time source returns false with a message naming it.
bool parse_time_source(const std::string& source, TimeKind& kind, float& period, float& phase,
                       std::string& error);

class ParameterBus {
public:
    void setSeed(uint32_t seed) { seed_ = seed; }
    uint32_t seed() const { return seed_; }
    void setBase(const std::string& key, float v) { base_[key] = v; }
    float base(const std::string& key, float fallback) const;
    void setOverride(const std::string& key, float v) { override_[key] = v; }
    void clearOverride(const std::string& key) { override_.erase(key); }
    // False (with `error`) for a malformed time source.
    bool addMapping(const MappingSpec& spec, std::string& error);
    const std::vector<MappingSpec>& mappings() const { return specs_; }

    // This frame's input values by source name: audio channels ("kick" is
    // "kick.smoothed"; parts raw, smoothed, peak, trigger, hold), "rms",
    // "low", "mid", "high", "centroid", "flux", "time", "lane.<name>",
    // "section.energy|progress|changed", "event:<type>.<what>" (set only while
    // the event runs). Values persist until changed or cleared.
    void setFeature(const std::string& name, float v);
    void setSection(const std::string& role, int index) {
        section_role_ = role;
        section_index_ = index;
    }
    void clearFeatures();

    // Evaluates every mapping for this frame and advances the bus clock by dt
    // (ParameterBus::update, ParameterBus.cpp:267-343).
    void update(float dt);
    // param(ctx, key, fallback) (ParameterBus.cpp:345-355).
    float value(const std::string& key, float fallback) const;
    double clock() const { return clock_; }

private:
    struct MapState {
        MappingSpec spec;
        float smoothed = 0.0f;
        bool primed = false;
        TimeKind kind = TimeKind::None;
        float period = 0.0f, phase = 0.0f;
        uint32_t noise_seed = 0;
    };
    bool sourceValue(const std::string& name, float& out) const;
    float featureValue(const std::string& name) const;

    std::map<std::string, float> base_, override_, set_, add_, mul_;
    std::map<std::string, float> features_;
    std::string section_role_;
    int section_index_ = -1;
    std::vector<MappingSpec> specs_;
    std::vector<MapState> states_;
    uint32_t seed_ = 0;
    double clock_ = 0.0;  // seconds; double so hours of 1/60 s steps stay exact enough
};

// The scene document (Scene::parse, Scene.cpp:24-93).
struct SceneModule {
    std::string type, name;
    bool enabled = true;
    Json params;  // the module's "params" object
};
struct SceneDoc {
    uint32_t seed = 1234, width = 1920, height = 1080;
    std::vector<SceneModule> modules;
    std::vector<MappingSpec> mappings;  // audioMappings, musicMappings, automation
};
// Returns false with `error` on a structural problem (module without "type",
// mapping without source/target, malformed time source).
bool parse_scene(const Json& j, SceneDoc& out, std::string& error);
// Scene::applyBaseParams (Scene.cpp:96-113): seed, numeric/boolean module
// params as "<module>.<key>" bases, then every mapping.
bool apply_scene(const SceneDoc& scene, ParameterBus& bus, std::string& error);

}  // namespace lenia
