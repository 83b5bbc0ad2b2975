// Minimal stand-in for the glm 1.0.1 API that the reference's SVO path
// includes (vec2/3/4, ivec3, uvec3, bvec3, mat3/mat4 and the free functions
// listed below), written for this test build only: it lets
// oracle/ref_build.sh compile the reference's own ray-cast sources here,
// where glm is not installed.  TEST INFRASTRUCTURE ONLY.
//
// Arithmetic follows glm's documented definitions in IEEE binary32, left to
// right, as the oracle's substitution (1) states them:
//   dot(a, b)      = (a.x*b.x + a.y*b.y) + a.z*b.z
//   length(v)      = sqrt(dot(v, v))
//   normalize(v)   = v * (1 / sqrt(dot(v, v)))
//   min(x, y)      = (y < x) ? y : x        max(x, y) = (x < y) ? y : x
//   clamp(x, a, b) = min(max(x, a), b)
//   M * v          = (M[0]*v.x + M[1]*v.y) + (M[2]*v.z + M[3]*v.w)   (mat4)
//                  = (M[0]*v.x + M[1]*v.y) + M[2]*v.z                  (mat3)
//   translate(M, t) sets column 3 to ((M[0]*t.x + M[1]*t.y) + M[2]*t.z) + M[3]
//   scale(M, s)    multiplies columns 0..2 by s.x, s.y, s.z
//   inverse(M)     of an affine matrix whose upper 3x3 is diagonal (the only
//                  form the path builds: translate * scale): columns 0..2 get
//                  1 / s, column 3 gets -(t * (1 / s)); any other matrix
//                  throws (the path does not produce one).
#pragma once

#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>

namespace glm {

template <class T>
struct tvec4;

template <class T>
struct tvec2 {
    T x{}, y{};
    tvec2() = default;
    explicit tvec2(T s) : x(s), y(s) {}
    tvec2(T a, T b) : x(a), y(b) {}
    T& operator[](int i) { return i == 0 ? x : y; }
    const T& operator[](int i) const { return i == 0 ? x : y; }
};

template <class T>
struct tvec3 {
    union { T x; T r; };
    union { T y; T g; };
    union { T z; T b; };
    tvec3() : x(), y(), z() {}
    explicit tvec3(T s) : x(s), y(s), z(s) {}
    tvec3(T a, T b_, T c) : x(a), y(b_), z(c) {}
    template <class U>
    explicit tvec3(const tvec3<U>& o) : x(static_cast<T>(o.x)), y(static_cast<T>(o.y)), z(static_cast<T>(o.z)) {}
    explicit tvec3(const tvec4<T>& o);
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    tvec3& operator+=(const tvec3& o) { x += o.x; y += o.y; z += o.z; return *this; }
    tvec3& operator-=(const tvec3& o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    tvec3& operator*=(const tvec3& o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    tvec3& operator/=(const tvec3& o) { x /= o.x; y /= o.y; z /= o.z; return *this; }
    tvec3& operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
    tvec3& operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
    tvec3& operator+=(T s) { x += s; y += s; z += s; return *this; }
    tvec3& operator-=(T s) { x -= s; y -= s; z -= s; return *this; }
};

template <class T>
struct tvec4 {
    T x{}, y{}, z{}, w{};
    tvec4() = default;
    explicit tvec4(T s) : x(s), y(s), z(s), w(s) {}
    tvec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    tvec4(const tvec3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    T& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    const T& operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
};

using vec2 = tvec2<float>;
using vec3 = tvec3<float>;
using vec4 = tvec4<float>;
using ivec2 = tvec2<int>;
using ivec3 = tvec3<int>;
using ivec4 = tvec4<int>;
using uvec2 = tvec2<unsigned>;
using uvec3 = tvec3<unsigned>;
using uvec4 = tvec4<unsigned>;
using bvec3 = tvec3<bool>;
using dvec3 = tvec3<double>;

#define VXGLM_BIN(OP)                                                                                     \
    template <class T>                                                                                    \
    tvec3<T> operator OP(const tvec3<T>& a, const tvec3<T>& b) { return {a.x OP b.x, a.y OP b.y, a.z OP b.z}; } \
    template <class T>                                                                                    \
    tvec3<T> operator OP(const tvec3<T>& a, T s) { return {a.x OP s, a.y OP s, a.z OP s}; }              \
    template <class T>                                                                                    \
    tvec3<T> operator OP(T s, const tvec3<T>& a) { return {s OP a.x, s OP a.y, s OP a.z}; }              \
    template <class T>                                                                                    \
    tvec4<T> operator OP(const tvec4<T>& a, const tvec4<T>& b) {                                         \
        return {a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w};                                          \
    }                                                                                                     \
    template <class T>                                                                                    \
    tvec4<T> operator OP(const tvec4<T>& a, T s) { return {a.x OP s, a.y OP s, a.z OP s, a.w OP s}; }     \
    template <class T>                                                                                    \
    tvec2<T> operator OP(const tvec2<T>& a, const tvec2<T>& b) { return {a.x OP b.x, a.y OP b.y}; }      \
    template <class T>                                                                                    \
    tvec2<T> operator OP(const tvec2<T>& a, T s) { return {a.x OP s, a.y OP s}; }
VXGLM_BIN(+)
VXGLM_BIN(-)
VXGLM_BIN(*)
VXGLM_BIN(/)
#undef VXGLM_BIN

template <class T>
tvec3<T> operator-(const tvec3<T>& a) { return {-a.x, -a.y, -a.z}; }
template <class T>
tvec3<T> operator&(const tvec3<T>& a, T s) { return {a.x & s, a.y & s, a.z & s}; }
template <class T>
tvec3<T> operator%(const tvec3<T>& a, T s) { return {a.x % s, a.y % s, a.z % s}; }
template <class T>
tvec3<T> operator>>(const tvec3<T>& a, T s) { return {a.x >> s, a.y >> s, a.z >> s}; }
template <class T>
tvec3<T> operator<<(const tvec3<T>& a, T s) { return {a.x << s, a.y << s, a.z << s}; }
template <class T>
bool operator==(const tvec3<T>& a, const tvec3<T>& b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
template <class T>
bool operator!=(const tvec3<T>& a, const tvec3<T>& b) { return !(a == b); }
template <class T>
bool operator==(const tvec2<T>& a, const tvec2<T>& b) { return a.x == b.x && a.y == b.y; }
template <class T>
bool operator==(const tvec4<T>& a, const tvec4<T>& b) { return a.x == b.x && a.y == b.y && a.z == b.z && a.w == b.w; }

// scalar min / max / clamp (glm/func_common)
template <class T>
T min(T x, T y) { return (y < x) ? y : x; }
template <class T>
T max(T x, T y) { return (x < y) ? y : x; }
template <class T>
T clamp(T x, T lo, T hi) { return min(max(x, lo), hi); }
template <class T>
tvec3<T> min(const tvec3<T>& a, const tvec3<T>& b) { return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)}; }
template <class T>
tvec3<T> max(const tvec3<T>& a, const tvec3<T>& b) { return {max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)}; }
template <class T>
tvec3<T> min(const tvec3<T>& a, T s) { return min(a, tvec3<T>(s)); }
template <class T>
tvec3<T> max(const tvec3<T>& a, T s) { return max(a, tvec3<T>(s)); }
template <class T>
tvec3<T> clamp(const tvec3<T>& v, const tvec3<T>& lo, const tvec3<T>& hi) { return min(max(v, lo), hi); }
template <class T>
tvec3<T> clamp(const tvec3<T>& v, T lo, T hi) { return clamp(v, tvec3<T>(lo), tvec3<T>(hi)); }

inline float floor(float x) { return std::floor(x); }
inline vec3 floor(const vec3& v) { return {std::floor(v.x), std::floor(v.y), std::floor(v.z)}; }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline vec3 abs(const vec3& v) { return {std::fabs(v.x), std::fabs(v.y), std::fabs(v.z)}; }
inline ivec3 abs(const ivec3& v) { return {abs(v.x), abs(v.y), abs(v.z)}; }
inline float sign(float x) { return float(0.0f < x) - float(x < 0.0f); }
inline vec3 sign(const vec3& v) { return {sign(v.x), sign(v.y), sign(v.z)}; }

inline float dot(const vec3& a, const vec3& b) {
    const vec3 t = a * b;
    return (t.x + t.y) + t.z;
}
inline float dot(const vec2& a, const vec2& b) {
    const vec2 t = a * b;
    return t.x + t.y;
}
inline float length(const vec3& v) { return std::sqrt(dot(v, v)); }
inline float length(const vec2& v) { return std::sqrt(dot(v, v)); }
inline float distance(const vec3& a, const vec3& b) { return length(b - a); }
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
inline vec3 normalize(const vec3& v) { return v * inversesqrt(dot(v, v)); }
inline vec3 cross(const vec3& a, const vec3& b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline float radians(float d) { return d * 0.01745329251994329576923690768489f; }

template <class T>
bvec3 lessThan(const tvec3<T>& a, const tvec3<T>& b) { return {a.x < b.x, a.y < b.y, a.z < b.z}; }
template <class T>
bvec3 lessThanEqual(const tvec3<T>& a, const tvec3<T>& b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
template <class T>
bvec3 greaterThan(const tvec3<T>& a, const tvec3<T>& b) { return {a.x > b.x, a.y > b.y, a.z > b.z}; }
template <class T>
bvec3 greaterThanEqual(const tvec3<T>& a, const tvec3<T>& b) { return {a.x >= b.x, a.y >= b.y, a.z >= b.z}; }
template <class T>
bvec3 equal(const tvec3<T>& a, const tvec3<T>& b) { return {a.x == b.x, a.y == b.y, a.z == b.z}; }
inline bool all(const bvec3& v) { return v.x && v.y && v.z; }
inline bool any(const bvec3& v) { return v.x || v.y || v.z; }
inline bvec3 isnan(const vec3& v) { return {std::isnan(v.x), std::isnan(v.y), std::isnan(v.z)}; }
inline bvec3 isinf(const vec3& v) { return {std::isinf(v.x), std::isinf(v.y), std::isinf(v.z)}; }
inline bool isnan(float x) { return std::isnan(x); }
inline bool isinf(float x) { return std::isinf(x); }

// Column-major matrices: m[i] is column i.
struct mat4 {
    vec4 c[4];
    mat4() : mat4(1.0f) {}
    explicit mat4(float d) {
        for (int i = 0; i < 4; ++i) c[i] = vec4(0.0f);
        c[0].x = c[1].y = c[2].z = c[3].w = d;
    }
    vec4& operator[](int i) { return c[i]; }
    const vec4& operator[](int i) const { return c[i]; }
};
struct mat3 {
    vec3 c[3];
    mat3() : mat3(1.0f) {}
    explicit mat3(float d) {
        for (int i = 0; i < 3; ++i) c[i] = vec3(0.0f);
        c[0].x = c[1].y = c[2].z = d;
    }
    explicit mat3(const mat4& m) {
        for (int i = 0; i < 3; ++i) c[i] = vec3(m[i].x, m[i].y, m[i].z);
    }
    vec3& operator[](int i) { return c[i]; }
    const vec3& operator[](int i) const { return c[i]; }
};

inline vec4 operator*(const mat4& m, const vec4& v) {
    const vec4 a = m[0] * v.x, b = m[1] * v.y, c2 = m[2] * v.z, d = m[3] * v.w;
    return (a + b) + (c2 + d);
}
inline vec3 operator*(const mat3& m, const vec3& v) {
    return {(m[0].x * v.x + m[1].x * v.y) + m[2].x * v.z, (m[0].y * v.x + m[1].y * v.y) + m[2].y * v.z,
            (m[0].z * v.x + m[1].z * v.y) + m[2].z * v.z};
}
inline mat4 operator*(const mat4& a, const mat4& b) {
    mat4 r(0.0f);
    for (int i = 0; i < 4; ++i) r[i] = a * b[i];
    return r;
}
inline mat4 translate(const mat4& m, const vec3& t) {
    mat4 r = m;
    r[3] = ((m[0] * t.x + m[1] * t.y) + m[2] * t.z) + m[3];
    return r;
}
inline mat4 scale(const mat4& m, const vec3& s) {
    mat4 r = m;
    r[0] = m[0] * s.x;
    r[1] = m[1] * s.y;
    r[2] = m[2] * s.z;
    return r;
}
inline mat4 inverse(const mat4& m) {
    const bool affine_diag = m[0].y == 0.0f && m[0].z == 0.0f && m[1].x == 0.0f && m[1].z == 0.0f &&
                             m[2].x == 0.0f && m[2].y == 0.0f && m[0].w == 0.0f && m[1].w == 0.0f &&
                             m[2].w == 0.0f && m[3].w == 1.0f;
    if (!affine_diag) {
        std::string msg = "glm stand-in: inverse of a general matrix is not provided:";
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) msg += " " + std::to_string(m[i][j]);
        throw std::runtime_error(msg);
    }
    mat4 r(1.0f);
    const vec3 inv(1.0f / m[0].x, 1.0f / m[1].y, 1.0f / m[2].z);
    r[0].x = inv.x;
    r[1].y = inv.y;
    r[2].z = inv.z;
    r[3] = vec4(-(m[3].x * inv.x), -(m[3].y * inv.y), -(m[3].z * inv.z), 1.0f);
    return r;
}

template <class T>
tvec3<T>::tvec3(const tvec4<T>& o) : x(o.x), y(o.y), z(o.z) {}

}  // namespace glm
