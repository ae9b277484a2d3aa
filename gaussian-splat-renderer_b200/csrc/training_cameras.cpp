// INRIA training cameras (cameras.json, written by gaussian-splatting's camera_to_JSON) and the
// two helpers derived from them (src/scene/training_cameras.cpp:1-75), restated. The reference
// parses the file with nlohmann/json 3.11.3 (a dependency absent from its tree); the small JSON
// reader below gives the same values: floating-point numbers through strtod, integers as 64-bit
// integers, and the same narrowing conversions (static_cast) to the camera's fields.
#include "scene_io.h"

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace gsr::io {

namespace {

struct Json {
    enum Kind { Null, Bool, Integer, Unsigned, Float, String, Array, Object } kind = Null;
    bool b = false;
    int64_t i = 0;
    uint64_t u = 0;
    double f = 0.0;
    std::string s;
    std::vector<Json> items;                            // Array
    std::vector<std::pair<std::string, Json>> members;  // Object

    const Json* member(const std::string& key) const {
        for (const auto& m : members)
            if (m.first == key) return &m.second;
        return nullptr;
    }
    const Json& at(const std::string& key) const {
        if (kind != Object) throw std::runtime_error("cannot use at() with " + typeName());
        const Json* m = member(key);
        if (!m) throw std::runtime_error("key '" + key + "' not found");
        return *m;
    }
    const Json& operator[](size_t k) const {
        if (kind != Array) throw std::runtime_error("cannot use operator[] with a numeric argument with " + typeName());
        if (k >= items.size()) throw std::runtime_error("array index " + std::to_string(k) + " is out of range");
        return items[k];
    }
    // nlohmann's size(): elements of an array or object, 0 for null, 1 for any other value
    size_t size() const {
        return kind == Array ? items.size() : kind == Object ? members.size() : kind == Null ? 0 : 1;
    }
    std::string typeName() const {
        static const char* kNames[] = {"null", "boolean", "number", "number", "number", "string", "array", "object"};
        return kNames[kind];
    }
    // get<T>() of an arithmetic T: static_cast from the stored representation
    template <typename T>
    T number() const {
        switch (kind) {
            case Integer: return static_cast<T>(i);
            case Unsigned: return static_cast<T>(u);
            case Float: return static_cast<T>(f);
            case Bool: return static_cast<T>(b);
            default: throw std::runtime_error("type must be number, but is " + typeName());
        }
    }
    std::string string() const {
        if (kind != String) throw std::runtime_error("type must be string, but is " + typeName());
        return s;
    }
};

class JsonReader {
public:
    explicit JsonReader(const std::string& text) : t_(text) {}
    Json document() {
        Json v = value();
        space();
        if (p_ != t_.size()) fail("unexpected content after the value");
        return v;
    }

private:
    const std::string& t_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        throw std::runtime_error("parse error at byte " + std::to_string(p_ + 1) + ": " + what);
    }
    void space() {
        while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t' || t_[p_] == '\n' || t_[p_] == '\r')) ++p_;
    }
    bool literal(const char* word) {
        const size_t n = std::strlen(word);
        if (t_.compare(p_, n, word) != 0) return false;
        p_ += n;
        return true;
    }
    Json value() {
        space();
        if (p_ >= t_.size()) fail("unexpected end of input");
        Json v;
        const char c = t_[p_];
        if (c == '{') {
            v.kind = Json::Object;
            ++p_;
            space();
            if (p_ < t_.size() && t_[p_] == '}') {
                ++p_;
                return v;
            }
            for (;;) {
                space();
                if (p_ >= t_.size() || t_[p_] != '"') fail("expected a string key");
                std::string key = str();
                space();
                if (p_ >= t_.size() || t_[p_] != ':') fail("expected ':'");
                ++p_;
                Json item = value();
                // a repeated key keeps its last value
                bool replaced = false;
                for (auto& m : v.members)
                    if (m.first == key) {
                        m.second = std::move(item);
                        replaced = true;
                        break;
                    }
                if (!replaced) v.members.emplace_back(std::move(key), std::move(item));
                space();
                if (p_ < t_.size() && t_[p_] == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < t_.size() && t_[p_] == '}') {
                    ++p_;
                    return v;
                }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Array;
            ++p_;
            space();
            if (p_ < t_.size() && t_[p_] == ']') {
                ++p_;
                return v;
            }
            for (;;) {
                v.items.push_back(value());
                space();
                if (p_ < t_.size() && t_[p_] == ',') {
                    ++p_;
                    continue;
                }
                if (p_ < t_.size() && t_[p_] == ']') {
                    ++p_;
                    return v;
                }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::String;
            v.s = str();
            return v;
        }
        if (literal("true")) {
            v.kind = Json::Bool;
            v.b = true;
            return v;
        }
        if (literal("false")) {
            v.kind = Json::Bool;
            return v;
        }
        if (literal("null")) return v;
        return number();
    }
    void utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6));
            out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18));
            out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F));
            out += char(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (p_ + 4 > t_.size()) fail("truncated \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char h = t_[p_++];
            v <<= 4;
            if (h >= '0' && h <= '9') v |= uint32_t(h - '0');
            else if (h >= 'a' && h <= 'f') v |= uint32_t(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= uint32_t(h - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string str() {
        ++p_;  // opening quote
        std::string out;
        for (;;) {
            if (p_ >= t_.size()) fail("unterminated string");
            const char c = t_[p_++];
            if (c == '"') return out;
            if (static_cast<unsigned char>(c) < 0x20) fail("control character in a string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (p_ >= t_.size()) fail("unterminated string");
            const char e = t_[p_++];
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
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp <= 0xDBFF) {  // surrogate pair
                        if (p_ + 2 > t_.size() || t_[p_] != '\\' || t_[p_ + 1] != 'u') fail("lone surrogate");
                        p_ += 2;
                        const uint32_t lo = hex4();
                        if (lo < 0xDC00 || lo > 0xDFFF) fail("bad surrogate pair");
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    } else if (cp >= 0xDC00 && cp <= 0xDFFF) {
                        fail("lone surrogate");
                    }
                    utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
    }
    Json number() {
        const size_t b = p_;
        bool isFloat = false;
        if (p_ < t_.size() && t_[p_] == '-') ++p_;
        auto digits = [&] {
            const size_t d = p_;
            while (p_ < t_.size() && t_[p_] >= '0' && t_[p_] <= '9') ++p_;
            return p_ > d;
        };
        if (p_ < t_.size() && t_[p_] == '0') ++p_;
        else if (!digits()) fail("invalid literal");
        if (p_ < t_.size() && t_[p_] == '.') {
            ++p_;
            if (!digits()) fail("invalid number");
            isFloat = true;
        }
        if (p_ < t_.size() && (t_[p_] == 'e' || t_[p_] == 'E')) {
            ++p_;
            if (p_ < t_.size() && (t_[p_] == '+' || t_[p_] == '-')) ++p_;
            if (!digits()) fail("invalid number");
            isFloat = true;
        }
        const std::string tok = t_.substr(b, p_ - b);
        Json v;
        if (!isFloat) {
            errno = 0;
            char* end = nullptr;
            if (tok[0] == '-') {
                const long long x = std::strtoll(tok.c_str(), &end, 10);
                if (errno == 0 && end == tok.c_str() + tok.size()) {
                    v.kind = Json::Integer;
                    v.i = x;
                    return v;
                }
            } else {
                const unsigned long long x = std::strtoull(tok.c_str(), &end, 10);
                if (errno == 0 && end == tok.c_str() + tok.size()) {
                    v.kind = Json::Unsigned;
                    v.u = x;
                    return v;
                }
            }
        }
        // floating point (or an integer outside the 64-bit range)
        v.kind = Json::Float;
        v.f = std::strtod(tok.c_str(), nullptr);
        return v;
    }
};

}  // namespace

std::vector<TrainingCamera> loadTrainingCameras(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Cannot open cameras file: " + path);
    std::stringstream text;
    text << in.rdbuf();
    const std::string body = text.str();
    std::vector<TrainingCamera> cameras;
    try {
        const Json doc = JsonReader(body).document();
        if (doc.kind != Json::Array) throw std::runtime_error("expected a JSON array");
        for (const Json& c : doc.items) {
            TrainingCamera cam;
            cam.id = c.at("id").number<int>();
            const Json* name = c.kind == Json::Object ? c.member("img_name") : nullptr;
            if (c.kind != Json::Object) throw std::runtime_error("cannot use value() with " + c.typeName());
            cam.imageName = name ? name->string() : std::string();
            cam.width = c.at("width").number<uint32_t>();
            cam.height = c.at("height").number<uint32_t>();
            cam.fx = c.at("fx").number<float>();
            cam.fy = c.at("fy").number<float>();
            const Json& p = c.at("position");
            const Json& r = c.at("rotation");
            if (p.size() != 3 || r.size() != 3) throw std::runtime_error("bad position/rotation size");
            for (int k = 0; k < 3; ++k) cam.position[k] = p[size_t(k)].number<float>();
            // JSON rows -> columns: element (row, col) is column col, row `row`
            for (int row = 0; row < 3; ++row) {
                const Json& rr = r[size_t(row)];
                if (rr.size() != 3) throw std::runtime_error("bad rotation row");
                for (int col = 0; col < 3; ++col) cam.cameraToWorld[col * 3 + row] = rr[size_t(col)].number<float>();
            }
            if (cam.width == 0 || cam.height == 0 || !(cam.fy > 0.0f))
                throw std::runtime_error("bad intrinsics for camera " + std::to_string(cam.id));
            cameras.push_back(std::move(cam));
        }
    } catch (const std::exception& e) {
        throw std::runtime_error("Invalid cameras file " + path + ": " + e.what());
    }
    return cameras;
}

float fovYDeg(const TrainingCamera& c) {
    return float(2.0 * std::atan(double(c.height) / (2.0 * double(c.fy))) * 180.0 / 3.14159265358979323846);
}

void meanCameraUp(const TrainingCamera* cams, size_t n, float up[3]) {
    // the average of the cameras' up (-y, the negated down axis), in double
    double sum[3] = {0.0, 0.0, 0.0};
    for (size_t k = 0; k < n; ++k)
        for (int a = 0; a < 3; ++a) sum[a] -= double(cams[k].cameraToWorld[3 + a]);
    const double len = std::sqrt(sum[0] * sum[0] + sum[1] * sum[1] + sum[2] * sum[2]);
    if (len > 1e-9) {
        for (int a = 0; a < 3; ++a) up[a] = float(sum[a] / len);
    } else {
        up[0] = 0.0f;
        up[1] = -1.0f;
        up[2] = 0.0f;
    }
}

void cameraFocusPoint(const TrainingCamera* cams, size_t n, float point[3]) {
    // least squares over the optical axes: sum_i (I - f f^T)(p - c_i) = 0, i.e. A p = b with
    // A = sum (I - f f^T), b = sum (I - f f^T) c (column-major 3x3 in double)
    if (n == 0) {
        point[0] = point[1] = point[2] = 0.0f;
        return;
    }
    double A[3][3] = {}, b[3] = {}, centroid[3] = {};
    for (size_t k = 0; k < n; ++k) {
        const float* fw = &cams[k].cameraToWorld[6];
        double f[3] = {double(fw[0]), double(fw[1]), double(fw[2])};
        const double inv = 1.0 / std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
        for (double& x : f) x *= inv;
        double P[3][3];  // P[col][row]
        for (int col = 0; col < 3; ++col)
            for (int row = 0; row < 3; ++row) P[col][row] = (col == row ? 1.0 : 0.0) - f[row] * f[col];
        const double c[3] = {double(cams[k].position[0]), double(cams[k].position[1]), double(cams[k].position[2])};
        for (int col = 0; col < 3; ++col)
            for (int row = 0; row < 3; ++row) A[col][row] += P[col][row];
        for (int row = 0; row < 3; ++row) b[row] += (P[0][row] * c[0] + P[1][row] * c[1]) + P[2][row] * c[2];
        for (int a = 0; a < 3; ++a) centroid[a] += c[a];
    }
    for (double& x : centroid) x /= double(n);
    auto m = [&](int col, int row) { return A[col][row]; };
    const double c00 = m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2);
    const double c10 = m(0, 1) * m(2, 2) - m(2, 1) * m(0, 2);
    const double c20 = m(0, 1) * m(1, 2) - m(1, 1) * m(0, 2);
    const double det = m(0, 0) * c00 - m(1, 0) * c10 + m(2, 0) * c20;
    // parallel axes (a forward-facing capture) leave A singular: no unique point
    if (std::fabs(det) < 1e-6 * double(n)) {
        for (int a = 0; a < 3; ++a) point[a] = float(centroid[a]);
        return;
    }
    // inverse by cofactors (inverse[col][row]), then p = inverse * b
    const double s = 1.0 / det;
    double inv[3][3];
    inv[0][0] = +(m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2)) * s;
    inv[1][0] = -(m(1, 0) * m(2, 2) - m(2, 0) * m(1, 2)) * s;
    inv[2][0] = +(m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1)) * s;
    inv[0][1] = -(m(0, 1) * m(2, 2) - m(2, 1) * m(0, 2)) * s;
    inv[1][1] = +(m(0, 0) * m(2, 2) - m(2, 0) * m(0, 2)) * s;
    inv[2][1] = -(m(0, 0) * m(2, 1) - m(2, 0) * m(0, 1)) * s;
    inv[0][2] = +(m(0, 1) * m(1, 2) - m(1, 1) * m(0, 2)) * s;
    inv[1][2] = -(m(0, 0) * m(1, 2) - m(1, 0) * m(0, 2)) * s;
    inv[2][2] = +(m(0, 0) * m(1, 1) - m(1, 0) * m(0, 1)) * s;
    for (int row = 0; row < 3; ++row) point[row] = float((inv[0][row] * b[0] + inv[1][row] * b[1]) + inv[2][row] * b[2]);
}

}  // namespace gsr::io
