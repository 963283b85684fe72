// Project-written subset of the glm vector-math API (test infrastructure only).
//
// glm is not installed in this environment, so the oracle harness that compiles the
// reference's own sources supplies this header set in its place.  Only the symbols
// the reference's hot-path files use exist here: vec2, vec3, mat3x3, dot, cross,
// normalize, min, max, transpose and the component-wise operators.  Each function
// restates glm 0.9.9's documented scalar (non-SIMD) definition:
//   dot(a, b)      = (a.x*b.x + a.y*b.y) + a.z*b.z           (sum left to right)
//   cross(a, b)    = (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
//   normalize(v)   = v * (1 / sqrt(dot(v, v)))                (inversesqrt = 1/sqrt)
//   min(x, y)      = (y < x) ? y : x,   max(x, y) = (x < y) ? y : x
//   mat3 * v       = column-major: m[0]*v.x + m[1]*v.y + m[2]*v.z, summed left to right
// Last-bit agreement with a real glm build is unpinned (no glm here to compare with).
#ifndef SPT_ORACLE_GLM_SHIM_CORE_HPP
#define SPT_ORACLE_GLM_SHIM_CORE_HPP

// Standard headers that glm's own headers pull in (glm.hpp, detail/setup.hpp);
// the reference relies on them arriving through <glm/glm.hpp>.
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstddef>
#include <limits>

namespace glm {

struct vec2 {
    union { float x, r, s; };
    union { float y, g, t; };
    vec2() : x(0.0f), y(0.0f) {}
    explicit vec2(float v) : x(v), y(v) {}
    template <typename A, typename B>
    vec2(A a, B b) : x(static_cast<float>(a)), y(static_cast<float>(b)) {}
    float& operator[](std::size_t i) { return i == 0 ? x : y; }
    const float& operator[](std::size_t i) const { return i == 0 ? x : y; }
};

inline vec2 operator+(const vec2& a, const vec2& b) { return vec2(a.x + b.x, a.y + b.y); }
inline vec2 operator-(const vec2& a, const vec2& b) { return vec2(a.x - b.x, a.y - b.y); }
inline vec2 operator*(const vec2& a, float s) { return vec2(a.x * s, a.y * s); }
inline vec2 operator*(float s, const vec2& a) { return vec2(s * a.x, s * a.y); }

struct vec3 {
    union { float x, r, s; };
    union { float y, g, t; };
    union { float z, b, p; };
    vec3() : x(0.0f), y(0.0f), z(0.0f) {}
    explicit vec3(float v) : x(v), y(v), z(v) {}
    template <typename A, typename B, typename C>
    vec3(A a, B b, C c) : x(static_cast<float>(a)), y(static_cast<float>(b)), z(static_cast<float>(c)) {}
    float& operator[](std::size_t i) { return i == 0 ? x : (i == 1 ? y : z); }
    const float& operator[](std::size_t i) const { return i == 0 ? x : (i == 1 ? y : z); }

    vec3& operator+=(const vec3& o) { x = x + o.x; y = y + o.y; z = z + o.z; return *this; }
    vec3& operator-=(const vec3& o) { x = x - o.x; y = y - o.y; z = z - o.z; return *this; }
    vec3& operator*=(const vec3& o) { x = x * o.x; y = y * o.y; z = z * o.z; return *this; }
    vec3& operator/=(const vec3& o) { x = x / o.x; y = y / o.y; z = z / o.z; return *this; }
    template <typename U>
    vec3& operator*=(U s) { const float f = static_cast<float>(s); x = x * f; y = y * f; z = z * f; return *this; }
    template <typename U>
    vec3& operator/=(U s) { const float f = static_cast<float>(s); x = x / f; y = y / f; z = z / f; return *this; }
};

inline vec3 operator-(const vec3& a) { return vec3(-a.x, -a.y, -a.z); }
inline vec3 operator+(const vec3& a, const vec3& b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(const vec3& a, const vec3& b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(const vec3& a, const vec3& b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator/(const vec3& a, const vec3& b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline vec3 operator+(const vec3& a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
inline vec3 operator-(const vec3& a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
inline vec3 operator*(const vec3& a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator/(const vec3& a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator+(float s, const vec3& a) { return vec3(s + a.x, s + a.y, s + a.z); }
inline vec3 operator-(float s, const vec3& a) { return vec3(s - a.x, s - a.y, s - a.z); }
inline vec3 operator*(float s, const vec3& a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(float s, const vec3& a) { return vec3(s / a.x, s / a.y, s / a.z); }

inline float dot(const vec3& a, const vec3& b) {
    const vec3 m = a * b;
    return m.x + m.y + m.z;
}

inline vec3 cross(const vec3& a, const vec3& b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}

inline float inversesqrt(float v) { return 1.0f / std::sqrt(v); }

inline vec3 normalize(const vec3& v) { return v * inversesqrt(dot(v, v)); }

inline float min(float x, float y) { return (y < x) ? y : x; }
inline float max(float x, float y) { return (x < y) ? y : x; }
inline vec3 min(const vec3& a, const vec3& b) { return vec3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline vec3 max(const vec3& a, const vec3& b) { return vec3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }

// Column-major 3x3 matrix: m[c] is column c.
struct mat3x3 {
    vec3 col[3];
    mat3x3() : col{vec3(1.0f, 0.0f, 0.0f), vec3(0.0f, 1.0f, 0.0f), vec3(0.0f, 0.0f, 1.0f)} {}
    vec3& operator[](std::size_t c) { return col[c]; }
    const vec3& operator[](std::size_t c) const { return col[c]; }
};
typedef mat3x3 mat3;

inline vec3 operator*(const mat3x3& m, const vec3& v) {
    return vec3(m[0][0] * v.x + m[1][0] * v.y + m[2][0] * v.z,
                m[0][1] * v.x + m[1][1] * v.y + m[2][1] * v.z,
                m[0][2] * v.x + m[1][2] * v.y + m[2][2] * v.z);
}

inline mat3x3 transpose(const mat3x3& m) {
    mat3x3 r;
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k) r[c][k] = m[k][c];
    return r;
}

}  // namespace glm

#endif  // SPT_ORACLE_GLM_SHIM_CORE_HPP
