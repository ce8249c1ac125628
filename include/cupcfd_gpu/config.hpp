// cupcfd_gpu/config.hpp - reads the parts of a CUP-CFD JSON configuration
// (the cupcfd.json a reference run takes) that the kernel benchmark needs:
//
//   "Mesh": { "Partitioner": { "NaivePartitioner": {} },
//             "MeshSource": { "MeshSourceStructGen": { "CellX": .., "CellY": .., "CellZ": ..,
//                              "SpatialXMin": .., "SpatialXMax": .., (Y, Z likewise) } } }
//   "Benchmarks": [ { "BenchmarkKernels": { "BenchmarkName": "..", "Repetitions": N } }, ... ]
//
// Key names and their meaning follow the reference's JSON readers
// (src/benchmarks/implementation/source/BenchmarkConfigKernelsJSON.cpp:40-70:
// BenchmarkName, Repetitions; src/geometry/mesh/implementation/source/
// MeshSourceStructGenConfigJSON.cpp:66-231: CellX/Y/Z, SpatialX/Y/ZMin/Max;
// MeshConfigSourceJSON.cpp:78-98: the Partitioner choice). A missing key is
// CUPCFD_E_CONFIG_OPT_NOT_FOUND and a value of the wrong kind
// CUPCFD_E_CONFIG_INVALID_VALUE, as in the reference; an unreadable file is
// CUPCFD_E_FILE_MISSING and malformed JSON CUPCFD_E_INVALID_FILE_FORMAT.
// Header-only; a small JSON reader of its own (objects, arrays, strings,
// numbers, true/false/null), no dependencies.
#pragma once

#include <cctype>
#include <cstdlib>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "cupcfd_gpu.h"

namespace cupcfd {
namespace benchmark {
namespace gpu {

// ---------------------------------------------------------------------------
// JSON values
// ---------------------------------------------------------------------------
struct Json {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;  // in file order

    const Json *get(const std::string &key) const {
        if (kind != Object) return nullptr;
        for (const auto &kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

namespace detail {

class JsonReader {
  public:
    explicit JsonReader(const std::string &text) : s_(text) {}

    bool parse(Json &out) {
        ws();
        if (!value(out)) return false;
        ws();
        return p_ == s_.size();
    }

  private:
    const std::string &s_;
    size_t p_ = 0;

    void ws() {
        while (p_ < s_.size() && std::isspace((unsigned char) s_[p_])) p_++;
    }
    bool lit(const char *w) {
        size_t n = std::char_traits<char>::length(w);
        if (s_.compare(p_, n, w) != 0) return false;
        p_ += n;
        return true;
    }
    bool string(std::string &out) {
        if (p_ >= s_.size() || s_[p_] != '"') return false;
        p_++;
        while (p_ < s_.size() && s_[p_] != '"') {
            char c = s_[p_++];
            if (c == '\\') {
                if (p_ >= s_.size()) return false;
                char e = s_[p_++];
                switch (e) {
                    case '"': case '\\': case '/': out.push_back(e); break;
                    case 'b': out.push_back('\b'); break;
                    case 'f': out.push_back('\f'); break;
                    case 'n': out.push_back('\n'); break;
                    case 'r': out.push_back('\r'); break;
                    case 't': out.push_back('\t'); break;
                    case 'u': {  // keep ASCII code points, replace the rest
                        if (p_ + 4 > s_.size()) return false;
                        unsigned v = (unsigned) std::strtoul(s_.substr(p_, 4).c_str(), nullptr, 16);
                        out.push_back(v < 128 ? (char) v : '?');
                        p_ += 4;
                        break;
                    }
                    default: return false;
                }
            } else {
                out.push_back(c);
            }
        }
        if (p_ >= s_.size()) return false;
        p_++;
        return true;
    }
    bool value(Json &v) {
        ws();
        if (p_ >= s_.size()) return false;
        char c = s_[p_];
        if (c == '{') {
            v.kind = Json::Object;
            p_++;
            ws();
            if (p_ < s_.size() && s_[p_] == '}') { p_++; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (p_ >= s_.size() || s_[p_] != ':') return false;
                p_++;
                Json x;
                if (!value(x)) return false;
                v.obj.emplace_back(std::move(k), std::move(x));
                ws();
                if (p_ < s_.size() && s_[p_] == ',') { p_++; continue; }
                if (p_ < s_.size() && s_[p_] == '}') { p_++; return true; }
                return false;
            }
        }
        if (c == '[') {
            v.kind = Json::Array;
            p_++;
            ws();
            if (p_ < s_.size() && s_[p_] == ']') { p_++; return true; }
            for (;;) {
                Json x;
                if (!value(x)) return false;
                v.arr.push_back(std::move(x));
                ws();
                if (p_ < s_.size() && s_[p_] == ',') { p_++; continue; }
                if (p_ < s_.size() && s_[p_] == ']') { p_++; return true; }
                return false;
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            return string(v.str);
        }
        if (lit("true")) { v.kind = Json::Bool; v.b = true; return true; }
        if (lit("false")) { v.kind = Json::Bool; v.b = false; return true; }
        if (lit("null")) { v.kind = Json::Null; return true; }
        const char *b = s_.c_str() + p_;
        char *e = nullptr;
        double d = std::strtod(b, &e);
        if (e == b) return false;
        v.kind = Json::Number;
        v.num = d;
        p_ += (size_t) (e - b);
        return true;
    }
};

inline int number(const Json *o, const char *key, double &out) {
    const Json *v = o ? o->get(key) : nullptr;
    if (!v || v->kind == Json::Null) return CUPCFD_E_CONFIG_OPT_NOT_FOUND;
    if (v->kind != Json::Number) return CUPCFD_E_CONFIG_INVALID_VALUE;
    out = v->num;
    return CUPCFD_E_SUCCESS;
}

}  // namespace detail

// Parses a JSON file.
inline int read_json(const std::string &path, Json &out) {
    std::ifstream f(path);
    if (!f) return CUPCFD_E_FILE_MISSING;
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    out = Json();
    return detail::JsonReader(text).parse(out) ? CUPCFD_E_SUCCESS : CUPCFD_E_INVALID_FILE_FORMAT;
}

// One "BenchmarkKernels" entry of "Benchmarks" (BenchmarkConfigKernels).
struct KernelBenchmarkConfig {
    std::string benchmarkName;
    long repetitions = 0;
};

// Every "BenchmarkKernels" entry of the top-level "Benchmarks" array, in
// file order (other benchmark kinds are skipped).
inline int kernel_benchmarks(const Json &root, std::vector<KernelBenchmarkConfig> &out) {
    out.clear();
    const Json *list = root.get("Benchmarks");
    if (!list) return CUPCFD_E_CONFIG_OPT_NOT_FOUND;
    if (list->kind != Json::Array) return CUPCFD_E_CONFIG_INVALID_VALUE;
    for (const Json &entry : list->arr) {
        const Json *k = entry.get("BenchmarkKernels");
        if (!k) continue;
        KernelBenchmarkConfig c;
        const Json *name = k->get("BenchmarkName");
        if (!name || name->kind == Json::Null) return CUPCFD_E_CONFIG_OPT_NOT_FOUND;
        if (name->kind != Json::String) return CUPCFD_E_CONFIG_INVALID_VALUE;
        c.benchmarkName = name->str;
        double reps = 0;
        int rc = detail::number(k, "Repetitions", reps);
        if (rc != CUPCFD_E_SUCCESS) return rc;
        c.repetitions = (long) reps;
        out.push_back(c);
    }
    return CUPCFD_E_SUCCESS;
}

// "Mesh" -> "MeshSource" -> "MeshSourceStructGen" (MeshSourceStructGenConfig)
// and the partitioner named under "Mesh" -> "Partitioner".
struct StructGenConfig {
    int cellX = 0, cellY = 0, cellZ = 0;
    double sMinX = 0, sMaxX = 0, sMinY = 0, sMaxY = 0, sMinZ = 0, sMaxZ = 0;
    std::string partitioner;  // "NaivePartitioner", "MetisPartitioner", "ParmetisPartitioner" or empty
};

inline int structgen_mesh(const Json &root, StructGenConfig &out) {
    const Json *mesh = root.get("Mesh");
    if (!mesh) return CUPCFD_E_CONFIG_OPT_NOT_FOUND;
    const Json *src = mesh->get("MeshSource");
    const Json *sg = src ? src->get("MeshSourceStructGen") : nullptr;
    if (!sg) return CUPCFD_E_CONFIG_OPT_NOT_FOUND;
    double v[9];
    const char *keys[9] = {"CellX", "CellY", "CellZ", "SpatialXMin", "SpatialXMax",
                           "SpatialYMin", "SpatialYMax", "SpatialZMin", "SpatialZMax"};
    for (int i = 0; i < 9; i++) {
        int rc = detail::number(sg, keys[i], v[i]);
        if (rc != CUPCFD_E_SUCCESS) return rc;
    }
    out.cellX = (int) v[0];
    out.cellY = (int) v[1];
    out.cellZ = (int) v[2];
    out.sMinX = v[3]; out.sMaxX = v[4];
    out.sMinY = v[5]; out.sMaxY = v[6];
    out.sMinZ = v[7]; out.sMaxZ = v[8];
    out.partitioner.clear();
    if (const Json *p = mesh->get("Partitioner"))
        if (p->kind == Json::Object && !p->obj.empty()) out.partitioner = p->obj.front().first;
    return CUPCFD_E_SUCCESS;
}

}  // namespace gpu
}  // namespace benchmark
}  // namespace cupcfd
