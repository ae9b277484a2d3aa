// A minimal, self-written stand-in for the GLM 1.0.1 subset that the renderer's CPU sources
// use (vec2/3/4, mat2/3/4, mat3x2/mat2x3, products, transpose, normalize, length, dot,
// outerProduct, min/max). It exists so that the reference's own CPU renderer
// (src/splat/*.cpp, src/scene/*.cpp) can be compiled here as the oracle: GLM itself is a
// FetchContent dependency (CMakeLists.txt:47-48, GIT_TAG 1.0.1) that is absent from the
// reference tree.
//
// This file DEFINES the floating-point evaluation order of every vector/matrix operation,
// and the C restatement (oracle/gsr_oracle.c) and the CUDA kernels follow it operation for
// operation:
//   * matrices are column-major, m[c][r] is column c, row r;
//   * every product sums over the inner index k in ascending order, left to right:
//       (A*B)[c][r] = ((A[0][r]*B[c][0] + A[1][r]*B[c][1]) + A[2][r]*B[c][2]) (+ A[3][r]*B[c][3])
//       (M*v)[r]    = ((M[0][r]*v.x + M[1][r]*v.y) + M[2][r]*v.z) (+ M[3][r]*v.w)
//     including products with entries that happen to be zero (no term is dropped);
//   * dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z for vec3, and for vec4 GLM 1.0.1's generic
//     compute_dot<vec4> (func_geometric.inl, every compiler but MSVC):
//     (a.x*b.x + a.y*b.y) + (a.z*b.z + a.w*b.w);
//   * normalize(v) = v * (1 / sqrt(dot(v, v))); length(v) = sqrt(dot(v, v));
//   * max(a, b) = (a < b) ? b : a and min(a, b) = (b < a) ? b : a per component;
//   * outerProduct(c, r)[i][j] = c[j] * r[i].
// No fused multiply-add: build every user of this header with -ffp-contract=off.
#pragma once

#include <cmath>
#include <cstddef>
#include <cstdint>

namespace glm {

using length_t = int;

struct vec2 {
    union { struct { float x, y; }; struct { float r, g; }; };
    vec2() : x(0.0f), y(0.0f) {}
    explicit vec2(float s) : x(s), y(s) {}
    vec2(float a, float b) : x(a), y(b) {}
    float& operator[](length_t i) { return (&x)[i]; }
    const float& operator[](length_t i) const { return (&x)[i]; }
};

struct vec4;

struct vec3 {
    union { struct { float x, y, z; }; struct { float r, g, b; }; };
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit vec3(const vec4& v);
    float& operator[](length_t i) { return (&x)[i]; }
    const float& operator[](length_t i) const { return (&x)[i]; }
    vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3& operator+=(float s) { x = x + s; y = y + s; z = z + s; return *this; }
    vec3& operator*=(float s) { x = x * s; y = y * s; z = z * s; return *this; }
};

struct vec4 {
    union { struct { float x, y, z, w; }; struct { float r, g, b, a; }; };
    vec4() : x(0.0f), y(0.0f), z(0.0f), w(0.0f) {}
    explicit vec4(float s) : x(s), y(s), z(s), w(s) {}
    vec4(float a_, float b_, float c_, float d_) : x(a_), y(b_), z(c_), w(d_) {}
    vec4(const vec3& v, float s) : x(v.x), y(v.y), z(v.z), w(s) {}
    float& operator[](length_t i) { return (&x)[i]; }
    const float& operator[](length_t i) const { return (&x)[i]; }
    vec4& operator+=(const vec4& o) { x = x + o.x; y = y + o.y; z = z + o.z; w = w + o.w; return *this; }
    vec4& operator*=(float s) { x = x * s; y = y * s; z = z * s; w = w * s; return *this; }
};

inline vec3::vec3(const vec4& v) : x(v.x), y(v.y), z(v.z) {}

struct uvec2 {
    uint32_t x, y;
    uvec2() : x(0), y(0) {}
    uvec2(uint32_t a, uint32_t b) : x(a), y(b) {}
};

// ---- vector arithmetic (component-wise) ---------------------------------------------------
inline vec2 operator+(const vec2& a, const vec2& b) { return {a.x + b.x, a.y + b.y}; }
inline vec2 operator-(const vec2& a, const vec2& b) { return {a.x - b.x, a.y - b.y}; }
inline vec2 operator*(const vec2& a, float s) { return {a.x * s, a.y * s}; }
inline vec2 operator*(float s, const vec2& a) { return {s * a.x, s * a.y}; }

inline vec3 operator-(const vec3& a) { return {-a.x, -a.y, -a.z}; }
inline vec3 operator+(const vec3& a, const vec3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3 operator-(const vec3& a, const vec3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3 operator*(const vec3& a, const vec3& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3 operator/(const vec3& a, const vec3& b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline vec3 operator+(const vec3& a, float s) { return {a.x + s, a.y + s, a.z + s}; }
inline vec3 operator-(const vec3& a, float s) { return {a.x - s, a.y - s, a.z - s}; }
inline vec3 operator*(const vec3& a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline vec3 operator*(float s, const vec3& a) { return {s * a.x, s * a.y, s * a.z}; }
inline vec3 operator/(const vec3& a, float s) { return {a.x / s, a.y / s, a.z / s}; }
inline vec3 operator/(float s, const vec3& a) { return {s / a.x, s / a.y, s / a.z}; }
inline bool operator==(const vec3& a, const vec3& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

inline vec4 operator-(const vec4& a) { return {-a.x, -a.y, -a.z, -a.w}; }
inline vec4 operator+(const vec4& a, const vec4& b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline vec4 operator-(const vec4& a, const vec4& b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline vec4 operator*(const vec4& a, const vec4& b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline vec4 operator*(const vec4& a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline vec4 operator*(float s, const vec4& a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
inline vec4 operator/(const vec4& a, float s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }

// ---- geometric functions ------------------------------------------------------------------
inline float dot(const vec2& a, const vec2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const vec3& a, const vec3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(const vec4& a, const vec4& b) { return (a.x * b.x + a.y * b.y) + (a.z * b.z + a.w * b.w); }
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline float length(const vec4& v) { return std::sqrt(dot(v, v)); }
inline vec3 normalize(const vec3& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline vec4 normalize(const vec4& v) { return v * (1.0f / std::sqrt(dot(v, v))); }
inline vec3 cross(const vec3& a, const vec3& b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}

inline vec3 exp(const vec3& v) { return {std::exp(v.x), std::exp(v.y), std::exp(v.z)}; }

inline float max(float a, float b) { return (a < b) ? b : a; }
inline float min(float a, float b) { return (b < a) ? b : a; }
inline vec3 max(const vec3& a, const vec3& b) { return {max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)}; }
inline vec3 min(const vec3& a, const vec3& b) { return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)}; }
inline vec3 max(const vec3& a, float b) { return max(a, vec3(b)); }
inline vec3 min(const vec3& a, float b) { return min(a, vec3(b)); }

// ---- matrices (column-major) --------------------------------------------------------------
struct mat2 {
    vec2 c[2];
    mat2() : c{vec2(1.0f, 0.0f), vec2(0.0f, 1.0f)} {}
    explicit mat2(float s) : c{vec2(s, 0.0f), vec2(0.0f, s)} {}
    vec2& operator[](length_t i) { return c[i]; }
    const vec2& operator[](length_t i) const { return c[i]; }
};

struct mat3x2 {  // 3 columns, 2 rows
    vec2 c[3];
    mat3x2() : c{vec2(1.0f, 0.0f), vec2(0.0f, 1.0f), vec2(0.0f, 0.0f)} {}
    explicit mat3x2(float s) : c{vec2(s, 0.0f), vec2(0.0f, s), vec2(0.0f, 0.0f)} {}
    vec2& operator[](length_t i) { return c[i]; }
    const vec2& operator[](length_t i) const { return c[i]; }
};

struct mat2x3 {  // 2 columns, 3 rows
    vec3 c[2];
    mat2x3() : c{vec3(1.0f, 0.0f, 0.0f), vec3(0.0f, 1.0f, 0.0f)} {}
    vec3& operator[](length_t i) { return c[i]; }
    const vec3& operator[](length_t i) const { return c[i]; }
};

struct mat4;

struct mat3 {
    vec3 c[3];
    mat3() : c{vec3(1.0f, 0.0f, 0.0f), vec3(0.0f, 1.0f, 0.0f), vec3(0.0f, 0.0f, 1.0f)} {}
    explicit mat3(float s) : c{vec3(s, 0.0f, 0.0f), vec3(0.0f, s, 0.0f), vec3(0.0f, 0.0f, s)} {}
    mat3(const vec3& a, const vec3& b, const vec3& d) : c{a, b, d} {}
    explicit mat3(const mat4& m);
    vec3& operator[](length_t i) { return c[i]; }
    const vec3& operator[](length_t i) const { return c[i]; }
    mat3& operator+=(const mat3& o) {
        for (int i = 0; i < 3; ++i) c[i] += o.c[i];
        return *this;
    }
};

struct mat4 {
    vec4 c[4];
    mat4()
        : c{vec4(1.0f, 0.0f, 0.0f, 0.0f), vec4(0.0f, 1.0f, 0.0f, 0.0f), vec4(0.0f, 0.0f, 1.0f, 0.0f),
            vec4(0.0f, 0.0f, 0.0f, 1.0f)} {}
    explicit mat4(float s)
        : c{vec4(s, 0.0f, 0.0f, 0.0f), vec4(0.0f, s, 0.0f, 0.0f), vec4(0.0f, 0.0f, s, 0.0f), vec4(0.0f, 0.0f, 0.0f, s)} {}
    vec4& operator[](length_t i) { return c[i]; }
    const vec4& operator[](length_t i) const { return c[i]; }
};

inline mat3::mat3(const mat4& m) : c{vec3(m[0]), vec3(m[1]), vec3(m[2])} {}

inline mat3 operator*(float s, const mat3& m) { return {s * m[0], s * m[1], s * m[2]}; }

inline mat3 transpose(const mat3& m) {
    mat3 t;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) t[col][row] = m[row][col];
    return t;
}
inline mat2x3 transpose(const mat3x2& m) {
    mat2x3 t;
    for (int col = 0; col < 2; ++col)
        for (int row = 0; row < 3; ++row) t[col][row] = m[row][col];
    return t;
}
inline mat4 transpose(const mat4& m) {
    mat4 t;
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row) t[col][row] = m[row][col];
    return t;
}

inline vec3 operator*(const mat3& m, const vec3& v) {
    return {m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z, m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
            m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z};
}
inline vec4 operator*(const mat4& m, const vec4& v) {
    vec4 r;
    for (int row = 0; row < 4; ++row)
        r[row] = m[0][row] * v.x + m[1][row] * v.y + m[2][row] * v.z + m[3][row] * v.w;
    return r;
}
inline mat3 operator*(const mat3& a, const mat3& b) {
    mat3 r;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 3; ++row) r[col][row] = a[0][row] * b[col][0] + a[1][row] * b[col][1] + a[2][row] * b[col][2];
    return r;
}
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r;
    for (int col = 0; col < 4; ++col)
        for (int row = 0; row < 4; ++row)
            r[col][row] = a[0][row] * b[col][0] + a[1][row] * b[col][1] + a[2][row] * b[col][2] + a[3][row] * b[col][3];
    return r;
}
inline mat3x2 operator*(const mat3x2& a, const mat3& b) {
    mat3x2 r;
    for (int col = 0; col < 3; ++col)
        for (int row = 0; row < 2; ++row) r[col][row] = a[0][row] * b[col][0] + a[1][row] * b[col][1] + a[2][row] * b[col][2];
    return r;
}
inline mat2 operator*(const mat3x2& a, const mat2x3& b) {
    mat2 r;
    for (int col = 0; col < 2; ++col)
        for (int row = 0; row < 2; ++row) r[col][row] = a[0][row] * b[col][0] + a[1][row] * b[col][1] + a[2][row] * b[col][2];
    return r;
}

inline mat3 outerProduct(const vec3& c, const vec3& r) {
    mat3 m;
    for (int i = 0; i < 3; ++i) m[i] = c * r[i];
    return m;
}

}  // namespace glm
