// life_simulation_b200/csrc/npy_io.cpp -- .npy v1.0 float32 reader and writer
// (format: the NumPy .npy specification, version 1.0).
#include "npy_io.h"

#include <cstdio>
#include <memory>

namespace lenia {

namespace {

struct FileCloser {
    void operator()(FILE* f) const {
        if (f) std::fclose(f);
    }
};
using File = std::unique_ptr<FILE, FileCloser>;

std::string shape_text(const std::vector<uint32_t>& shape) {
    std::string s = "(";
    for (size_t i = 0; i < shape.size(); ++i) {
        s += std::to_string(shape[i]);
        if (shape.size() == 1 || i + 1 < shape.size()) s += ", ";
    }
    return s + ")";
}

// The value text that follows `'key':` in a header dict (up to the next
// top-level comma or the closing brace; a tuple is kept whole).
bool dict_value(const std::string& dict, const std::string& key, std::string& out) {
    const size_t k = dict.find("'" + key + "'");
    if (k == std::string::npos) return false;
    size_t p = dict.find(':', k);
    if (p == std::string::npos) return false;
    ++p;
    while (p < dict.size() && (dict[p] == ' ' || dict[p] == '\t')) ++p;
    size_t e = p;
    if (p < dict.size() && dict[p] == '(') {
        e = dict.find(')', p);
        if (e == std::string::npos) return false;
        ++e;
    } else {
        while (e < dict.size() && dict[e] != ',' && dict[e] != '}') ++e;
    }
    out = dict.substr(p, e - p);
    while (!out.empty() && (out.back() == ' ' || out.back() == '\t')) out.pop_back();
    return true;
}

bool parse_shape(const std::string& tuple, std::vector<uint32_t>& shape) {
    if (tuple.size() < 2 || tuple.front() != '(' || tuple.back() != ')') return false;
    shape.clear();
    const std::string inner = tuple.substr(1, tuple.size() - 2);
    size_t p = 0;
    while (p <= inner.size()) {
        size_t c = inner.find(',', p);
        if (c == std::string::npos) c = inner.size();
        const size_t b = inner.find_first_not_of(" \t", p);
        if (b != std::string::npos && b < c) {
            const size_t e = inner.find_last_not_of(" \t", c - 1);
            const std::string t = inner.substr(b, e - b + 1);
            if (t.size() > 10) return false;
            uint64_t v = 0;
            for (char d : t) {
                if (d < '0' || d > '9') return false;
                v = v * 10 + uint64_t(d - '0');
            }
            if (v > 0xFFFFFFFFull) return false;
            shape.push_back(uint32_t(v));
        }
        p = c + 1;
    }
    return true;
}

}  // namespace

bool write_npy_f32(const std::string& path, const float* data, size_t count, const std::vector<uint32_t>& shape,
                   std::string& error) {
    size_t n = 1;
    for (uint32_t s : shape) n *= s;
    if (n != count || (count > 0 && !data)) {
        error = "npy write: shape and element count differ for " + path;
        return false;
    }
    std::string dict = "{'descr': '<f4', 'fortran_order': False, 'shape': " + shape_text(shape) + ", }";
    const size_t preamble = 10 + dict.size() + 1;  // magic, version, length, dict, '\n'
    dict.append((64 - preamble % 64) % 64, ' ');
    dict.push_back('\n');
    if (dict.size() > 0xFFFF) {
        error = "npy write: header too long for " + path;
        return false;
    }
    File f(std::fopen(path.c_str(), "wb"));
    if (!f) {
        error = "cannot open " + path + " for writing";
        return false;
    }
    const unsigned char head[10] = {0x93, 'N', 'U', 'M', 'P', 'Y', 1, 0, uint8_t(dict.size() & 0xFF),
                                    uint8_t(dict.size() >> 8)};
    bool ok = std::fwrite(head, 1, 10, f.get()) == 10 && std::fwrite(dict.data(), 1, dict.size(), f.get()) == dict.size();
    if (ok && count) ok = std::fwrite(data, sizeof(float), count, f.get()) == count;
    if (ok) ok = std::fflush(f.get()) == 0;
    if (!ok) {
        error = "short write on " + path;
        return false;
    }
    return true;
}

bool read_npy_f32(const std::string& path, const std::vector<uint32_t>& expected, std::vector<float>& out,
                  std::string& error) {
    out.clear();
    if (expected.empty()) {
        error = "npy read: the expected shape must not be empty (" + path + ")";
        return false;
    }
    size_t n = 1;
    for (uint32_t s : expected) n *= s;
    File f(std::fopen(path.c_str(), "rb"));
    if (!f) {
        error = "cannot open " + path + " for reading";
        return false;
    }
    unsigned char head[10];
    if (std::fread(head, 1, 10, f.get()) != 10 || head[0] != 0x93 || head[1] != 'N' || head[2] != 'U' ||
        head[3] != 'M' || head[4] != 'P' || head[5] != 'Y' || head[6] != 1) {
        error = "corrupt or truncated npy header: " + path;
        return false;
    }
    const size_t len = size_t(head[8]) | (size_t(head[9]) << 8);
    std::string dict(len, '\0');
    if (len == 0 || std::fread(dict.data(), 1, len, f.get()) != len) {
        error = "truncated npy header dict: " + path;
        return false;
    }
    std::string descr, order, tuple;
    if (!dict_value(dict, "descr", descr) || descr != "'<f4'") {
        error = "unsupported npy dtype (expected <f4): " + path;
        return false;
    }
    if (dict_value(dict, "fortran_order", order) && order != "False") {
        error = "npy array in Fortran order (expected C order): " + path;
        return false;
    }
    std::vector<uint32_t> shape;
    if (!dict_value(dict, "shape", tuple) || !parse_shape(tuple, shape)) {
        error = "cannot parse npy shape: " + path;
        return false;
    }
    if (shape != expected) {
        error = "npy shape mismatch in " + path + ": expected " + shape_text(expected) + ", file has " +
                shape_text(shape);
        return false;
    }
    out.resize(n);
    const size_t got = n ? std::fread(out.data(), sizeof(float), n, f.get()) : 0;
    if (got != n) {
        out.clear();
        error = "truncated npy data in " + path + ": expected " + std::to_string(n) + " float32 values, got " +
                std::to_string(got);
        return false;
    }
    return true;
}

}  // namespace lenia
