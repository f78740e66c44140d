// life_simulation_b200/csrc/json_lite.cpp -- recursive-descent JSON reader.
#include "json_lite.h"

#include <cctype>
#include <cmath>
#include <cstdlib>

namespace lenia {

class JsonParser {
public:
    explicit JsonParser(const std::string& s) : s_(s) {}

    bool parse(Json& out, std::string* err) {
        skip();
        if (!value(out, 0)) {
            if (err) *err = error_ + " at offset " + std::to_string(pos_);
            return false;
        }
        skip();
        if (pos_ != s_.size()) {
            if (err) *err = "trailing characters at offset " + std::to_string(pos_);
            return false;
        }
        return true;
    }

private:
    const std::string& s_;
    size_t pos_ = 0;
    std::string error_;

    void skip() {
        while (pos_ < s_.size() && std::isspace(static_cast<unsigned char>(s_[pos_]))) ++pos_;
    }
    bool fail(const char* m) {
        error_ = m;
        return false;
    }
    bool literal(const char* w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(pos_, n, w) != 0) return false;
        pos_ += n;
        return true;
    }
    bool value(Json& v, int depth) {
        if (depth > 64) return fail("nesting too deep");
        skip();
        if (pos_ >= s_.size()) return fail("unexpected end");
        char c = s_[pos_];
        if (c == '{') return object(v, depth);
        if (c == '[') return array(v, depth);
        if (c == '"') {
            v.type_ = Json::Type::String;
            return string(v.str_);
        }
        if (literal("true")) { v.type_ = Json::Type::Bool; v.b_ = true; return true; }
        if (literal("false")) { v.type_ = Json::Type::Bool; v.b_ = false; return true; }
        if (literal("null")) { v.type_ = Json::Type::Null; return true; }
        return number(v);
    }
    bool number(Json& v) {
        const char* start = s_.c_str() + pos_;
        char* end = nullptr;
        double d = std::strtod(start, &end);
        if (end == start) return fail("invalid value");
        pos_ += size_t(end - start);
        v.type_ = Json::Type::Number;
        v.num_ = d;
        return true;
    }
    bool string(std::string& out) {
        ++pos_;  // opening quote
        out.clear();
        while (pos_ < s_.size()) {
            char c = s_[pos_++];
            if (c == '"') return true;
            if (c == '\\') {
                if (pos_ >= s_.size()) return fail("bad escape");
                char e = s_[pos_++];
                switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    if (pos_ + 4 > s_.size()) return fail("bad unicode escape");
                    unsigned cp = unsigned(std::strtoul(s_.substr(pos_, 4).c_str(), nullptr, 16));
                    pos_ += 4;
                    if (cp >= 0xD800 && cp <= 0xDBFF && pos_ + 6 <= s_.size() && s_[pos_] == '\\' &&
                        s_[pos_ + 1] == 'u') {
                        unsigned lo = unsigned(std::strtoul(s_.substr(pos_ + 2, 4).c_str(), nullptr, 16));
                        pos_ += 6;
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    // UTF-8 encode
                    if (cp < 0x80) out += char(cp);
                    else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
                    else if (cp < 0x10000) {
                        out += char(0xE0 | (cp >> 12));
                        out += char(0x80 | ((cp >> 6) & 0x3F));
                        out += char(0x80 | (cp & 0x3F));
                    } else {
                        out += char(0xF0 | (cp >> 18));
                        out += char(0x80 | ((cp >> 12) & 0x3F));
                        out += char(0x80 | ((cp >> 6) & 0x3F));
                        out += char(0x80 | (cp & 0x3F));
                    }
                    break;
                }
                default: return fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        return fail("unterminated string");
    }
    bool array(Json& v, int depth) {
        ++pos_;
        v.type_ = Json::Type::Array;
        skip();
        if (pos_ < s_.size() && s_[pos_] == ']') { ++pos_; return true; }
        while (true) {
            Json item;
            if (!value(item, depth + 1)) return false;
            v.arr_.push_back(std::move(item));
            skip();
            if (pos_ >= s_.size()) return fail("unterminated array");
            if (s_[pos_] == ',') { ++pos_; continue; }
            if (s_[pos_] == ']') { ++pos_; return true; }
            return fail("expected , or ]");
        }
    }
    bool object(Json& v, int depth) {
        ++pos_;
        v.type_ = Json::Type::Object;
        skip();
        if (pos_ < s_.size() && s_[pos_] == '}') { ++pos_; return true; }
        while (true) {
            skip();
            if (pos_ >= s_.size() || s_[pos_] != '"') return fail("expected key");
            std::string key;
            if (!string(key)) return false;
            skip();
            if (pos_ >= s_.size() || s_[pos_] != ':') return fail("expected :");
            ++pos_;
            Json item;
            if (!value(item, depth + 1)) return false;
            // Last duplicate key wins, as nlohmann does on parse.
            bool replaced = false;
            for (auto& m : v.obj_)
                if (m.first == key) { m.second = std::move(item); replaced = true; break; }
            if (!replaced) v.obj_.emplace_back(std::move(key), std::move(item));
            skip();
            if (pos_ >= s_.size()) return fail("unterminated object");
            if (s_[pos_] == ',') { ++pos_; continue; }
            if (s_[pos_] == '}') { ++pos_; return true; }
            return fail("expected , or }");
        }
    }
};

Json Json::parse(const std::string& text, std::string* error) {
    Json out;
    JsonParser p(text);
    if (!p.parse(out, error)) return Json();
    if (error) error->clear();
    return out;
}

const Json* Json::find(const std::string& key) const {
    if (type_ != Type::Object) return nullptr;
    for (const auto& m : obj_)
        if (m.first == key) return &m.second;
    return nullptr;
}

float Json::value_float(const std::string& key, float dflt) const {
    const Json* j = find(key);
    if (!j) return dflt;
    if (j->is_number()) return float(j->num_);
    if (j->is_bool()) return j->b_ ? 1.0f : 0.0f;
    return dflt;
}

uint32_t Json::value_u32(const std::string& key, uint32_t dflt) const {
    const Json* j = find(key);
    if (!j || !j->is_number()) return j && j->is_bool() ? uint32_t(j->b_) : dflt;
    double d = j->num_;
    // Conversion of a JSON number to uint32_t truncates toward zero.
    if (d < 0) return uint32_t(int64_t(d));
    return uint32_t(uint64_t(d));
}

bool Json::value_bool(const std::string& key, bool dflt) const {
    const Json* j = find(key);
    if (!j) return dflt;
    if (j->is_bool()) return j->b_;
    if (j->is_number()) return j->num_ != 0.0;
    return dflt;
}

std::string Json::value_string(const std::string& key, const std::string& dflt) const {
    const Json* j = find(key);
    if (!j || !j->is_string()) return dflt;
    return j->str_;
}

}  // namespace lenia
