// life_simulation_b200/csrc/json_lite.h -- a small JSON reader for scene
// "params" blocks and organism files (objects, arrays, numbers, strings,
// booleans, null). Numbers keep their double value; value<T>() converts like
// the reference's nlohmann::json::value<T>(key, default) for the types the
// Lenia params use (float, uint32_t, bool, string).
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

namespace lenia {

class Json {
public:
    enum class Type { Null, Bool, Number, String, Array, Object };

    Json() = default;
    static Json parse(const std::string& text, std::string* error);

    Type type() const { return type_; }
    bool is_null() const { return type_ == Type::Null; }
    bool is_bool() const { return type_ == Type::Bool; }
    bool is_number() const { return type_ == Type::Number; }
    bool is_string() const { return type_ == Type::String; }
    bool is_array() const { return type_ == Type::Array; }
    bool is_object() const { return type_ == Type::Object; }

    bool as_bool() const { return b_; }
    double as_number() const { return num_; }
    const std::string& as_string() const { return str_; }
    const std::vector<Json>& items() const { return arr_; }
    const std::vector<std::pair<std::string, Json>>& members() const { return obj_; }

    bool contains(const std::string& key) const { return find(key) != nullptr; }
    const Json* find(const std::string& key) const;
    size_t size() const { return is_array() ? arr_.size() : obj_.size(); }

    float value_float(const std::string& key, float dflt) const;
    uint32_t value_u32(const std::string& key, uint32_t dflt) const;
    bool value_bool(const std::string& key, bool dflt) const;
    std::string value_string(const std::string& key, const std::string& dflt) const;

private:
    friend class JsonParser;
    Type type_ = Type::Null;
    bool b_ = false;
    double num_ = 0.0;
    std::string str_;
    std::vector<Json> arr_;
    std::vector<std::pair<std::string, Json>> obj_;
};

}  // namespace lenia
