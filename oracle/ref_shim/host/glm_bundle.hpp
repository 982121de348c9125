// TEST INFRASTRUCTURE ONLY — stand-in for the reference's include/host/glm_bundle.hpp.  The
// reference links glm 1.0.3 (CMakeLists.txt:40-45), which is not installed here; this header
// restates, in float, the few glm functions its path uses, with glm's published definitions:
//   dot(a, b)      = (a.x*b.x + a.y*b.y) + a.z*b.z      (component product, then summed in order)
//   cross(a, b)    = (a.y*b.z - b.y*a.z, a.z*b.x - b.z*a.x, a.x*b.y - b.x*a.y)
//   normalize(v)   = v * inversesqrt(dot(v, v)),  inversesqrt(x) = 1 / sqrt(x)
//   length(v)      = sqrt(dot(v, v));  radians(d) = d * 0.01745329251994329576923690768489
//   max(a, b)      = (a < b) ? b : a;  abs, tan = the C library's
// plus the reference's own vec3/vec2 <-> float4/float2 helpers (glm_bundle.hpp:10-12).
#pragma once

#include <cmath>

#include "common/typedefs.h"

namespace glm {

struct vec2 {
    float x, y;
    vec2() = default;
    vec2(float a, float b) : x(a), y(b) {}
};

struct vec3 {
    float x, y, z;
    vec3() = default;
    vec3(float a, float b, float c) : x(a), y(b), z(c) {}
    explicit vec3(float s) : x(s), y(s), z(s) {}
};

inline vec3 operator+(vec3 a, vec3 b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline vec3 operator-(vec3 a, vec3 b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline vec3 operator*(vec3 a, vec3 b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline vec3 operator*(vec3 a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
inline vec3 operator*(float s, vec3 a) { return vec3(s * a.x, s * a.y, s * a.z); }
inline vec3 operator/(vec3 a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
inline vec3 operator-(vec3 a) { return vec3(-a.x, -a.y, -a.z); }

inline float dot(vec3 a, vec3 b) {
    vec3 t = a * b;
    return t.x + t.y + t.z;
}
inline vec3 cross(vec3 a, vec3 b) {
    return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
inline float inversesqrt(float x) { return 1.0f / std::sqrt(x); }
inline vec3 normalize(vec3 v) { return v * inversesqrt(dot(v, v)); }
inline float length(vec3 v) { return std::sqrt(dot(v, v)); }
inline float radians(float d) { return d * static_cast<float>(0.01745329251994329576923690768489); }
inline float tan(float x) { return std::tan(x); }
inline float abs(float x) { return std::fabs(x); }
inline float max(float a, float b) { return (a < b) ? b : a; }

} // namespace glm

using glm::vec2, glm::vec3;

inline float4 vec3_to_float4(const vec3 &v) { return float4{{v.x, v.y, v.z, 0.0f}}; }
inline vec3 float4_to_vec3(const float4 &v) { return {v.x, v.y, v.z}; }
inline float2 vec2_to_float2(const vec2 &v) { return float2{{v.x, v.y}}; }
