// dev_common.cuh — device-side vocabulary of the SPPM core: float4 arithmetic with the fixed
// OpenCL builtin semantics, the PCG stream, the photon codecs and the grid hash.
//
// Arithmetic contract (shared with the host-side restatement used in the tests): binary32 with
// no contraction (the library is built with -fmad=false, -prec-div=true, -prec-sqrt=true),
// dot(a,b) = ((ax*bx + ay*by) + az*bz) + aw*bw, normalize(v) = v / sqrt(dot(v,v)) (zero vector
// returned unchanged), rsqrt(x) = 1/sqrt(x), and transcendental builtins from phx_math.h.  With
// these, every kernel reproduces the reference's float expression trees bit for bit.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/phx.h"
#include "../../include/phx_math.h"

namespace phx {

typedef uint32_t u32;
typedef int32_t i32;
typedef uint8_t u8;
typedef uint64_t u64;

#define PHX_DI __device__ __forceinline__
// Large shading routines, by group: compiled out of line (one shared copy, a smaller instruction
// footprint for the state-machine kernels) or inlined.
#define PHX_OUTLINED static __device__ __noinline__
#ifdef PHX_OUTLINE_NEE
#define PHX_SHADE_NEE PHX_OUTLINED
#else
#define PHX_SHADE_NEE PHX_DI
#endif
#ifdef PHX_OUTLINE_BSDF
#define PHX_SHADE_BSDF PHX_OUTLINED
#else
#define PHX_SHADE_BSDF PHX_DI
#endif
#ifdef PHX_OUTLINE_HIT
#define PHX_SHADE_HIT PHX_OUTLINED
#else
#define PHX_SHADE_HIT PHX_DI
#endif
#ifdef PHX_OUTLINE_TEX
#define PHX_SHADE_TEX PHX_OUTLINED
#else
#define PHX_SHADE_TEX PHX_DI
#endif
#ifdef PHX_OUTLINE_LIGHT
#define PHX_SHADE_LIGHT PHX_OUTLINED
#else
#define PHX_SHADE_LIGHT PHX_DI
#endif
#define PHX_HDI __host__ __device__ __forceinline__

// include/common/constants.h:6-45
constexpr float EPS = 1e-5f;
constexpr float INF = 1e9f;
constexpr float PI = 3.141592654f;
constexpr float U32_MAX_F = 4294967296.0f;
constexpr u32 NO_TEXTURE = 0xFFFFFFFFu;
constexpr float AIR_IOR = 1.0f;
constexpr u32 MAX_RAY_BOUNCES = 5u;
constexpr u32 IOR_STACK_SIZE = 8u;
constexpr float MIN_ROUGHNESS = 0.001f;
constexpr u32 GGX_SAMPLING_ATTEMPTS = 8u;
constexpr u32 RR_MIN_RAY_DEPTH = 2u;
constexpr u32 RR_MIN_PHOTON_DEPTH = 2u;
constexpr float RR_MIN_Q = 0.05f;
constexpr float RR_MAX_Q = 1.0f;
constexpr float GAUSS_ALPHA = 1.818f;
constexpr float GAUSS_BETA = 1.953f;
constexpr float GAUSS_DENOM = 0.85815f;

// device error bits (phx_info.error_flags)
constexpr u32 ERR_LOOKBACK_TIMEOUT = 1u;
constexpr u32 ERR_STACK_OVERFLOW = 2u;
constexpr u32 ERR_SLOT_OVERFLOW = 4u;
constexpr u32 ERR_NO_PHOTONS = 8u;
constexpr u32 ERR_DEFER_OVERFLOW = 16u; // a deferred emission term did not fit its pixel's list

// ---- float4 ----------------------------------------------------------------------------------
PHX_HDI float4 f4(float x, float y, float z, float w) { return make_float4(x, y, z, w); }
PHX_HDI float4 f4(const phx_f4 &v) { return make_float4(v.x, v.y, v.z, v.w); }
PHX_HDI float4 operator+(float4 a, float4 b) { return f4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
PHX_HDI float4 operator-(float4 a, float4 b) { return f4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
PHX_HDI float4 operator*(float4 a, float4 b) { return f4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
PHX_HDI float4 operator/(float4 a, float4 b) { return f4(a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w); }
PHX_HDI float4 operator*(float4 a, float s) { return f4(a.x * s, a.y * s, a.z * s, a.w * s); }
PHX_HDI float4 operator*(float s, float4 a) { return f4(s * a.x, s * a.y, s * a.z, s * a.w); }
PHX_HDI float4 operator/(float4 a, float s) { return f4(a.x / s, a.y / s, a.z / s, a.w / s); }
PHX_HDI float4 operator-(float4 a) { return f4(-a.x, -a.y, -a.z, -a.w); }
PHX_HDI float4 &operator+=(float4 &a, float4 b) { return a = a + b; }
PHX_HDI float4 &operator*=(float4 &a, float4 b) { return a = a * b; }
PHX_HDI float4 &operator*=(float4 &a, float s) { return a = a * s; }
PHX_HDI float4 &operator/=(float4 &a, float s) { return a = a / s; }
PHX_HDI float dot(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
PHX_HDI float4 cross(float4 a, float4 b) {
    return f4(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f);
}
PHX_HDI float length(float4 v) { return sqrtf(dot(v, v)); }
PHX_HDI float4 normalize(float4 v) {
    float l = sqrtf(dot(v, v));
    if (l == 0.0f)
        return v;
    return v / l;
}
PHX_HDI float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
PHX_HDI float4 mix(float4 a, float4 b, float t) { return a + (b - a) * t; }
PHX_HDI float4 zero4() { return f4(0.0f, 0.0f, 0.0f, 0.0f); }
PHX_HDI float4 white4() { return f4(1.0f, 1.0f, 1.0f, 0.0f); }

// ---- PCG: include/common/random.h:16-36 --------------------------------------------------------
struct Rng {
    u32 state;
};
PHX_HDI Rng pcg_seed(u32 seed) {
    Rng r;
    r.state = 2891336453u; // 0 * 747796405u + 2891336453u
    r.state += seed;
    r.state = r.state * 747796405u + 2891336453u;
    return r;
}
PHX_HDI u32 random_u32(Rng *rng) {
    u32 old = rng->state;
    rng->state = rng->state * 747796405u + 2891336453u;
    return ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
}
PHX_HDI float random_float(Rng *rng) { return (float)random_u32(rng) / U32_MAX_F; }

// The state after n more draws, in O(log n) steps: the LCG's n-step map x -> A x + C, composed by
// binary powering (Brown, "Random number generation with arbitrary strides", Trans. Am. Nucl. Soc.
// 71, 1994).  All arithmetic is mod 2^32, so the result equals n calls of random_u32 exactly.
PHX_HDI Rng rng_advance(Rng r, u32 n) {
    u32 cur_mult = 747796405u, cur_plus = 2891336453u, acc_mult = 1u, acc_plus = 0u;
    while (n) {
        if (n & 1u) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1u) * cur_plus;
        cur_mult *= cur_mult;
        n >>= 1;
    }
    r.state = acc_mult * r.state + acc_plus;
    return r;
}

// utils.h:59-71
PHX_HDI void make_tbn(float4 normal, float4 *tangent, float4 *bitangent) {
    normal.w = 0.0f;
    float4 tmp = (fabsf(normal.x) > 0.1f) ? f4(0.0f, 1.0f, 0.0f, 0.0f) : f4(1.0f, 0.0f, 0.0f, 0.0f);
    *tangent = cross(normal, tmp);
    if (length(*tangent) < EPS) {
        tmp = f4(0.0f, 0.0f, 1.0f, 0.0f);
        *tangent = cross(normal, tmp);
    }
    *tangent = normalize(*tangent);
    *bitangent = cross(normal, *tangent);
}

// random.h:40-46
PHX_HDI float4 random_unit_vector(Rng *rng) {
    float z = 2.0f * random_float(rng) - 1.0f;
    float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
    float phi = (2.0f * PI) * random_float(rng);
    float sp, cp;
    pm_sincosf(phi, &sp, &cp);
    return f4(r * cp, r * sp, z, 0.0f);
}

// random.h:48-62
// The same with the normal's frame (make_tbn of the normal) given by the caller.
PHX_HDI float4 random_in_unit_hemisphere_tbn(Rng *rng, float4 normal, float4 t, float4 b) {
    normal.w = 0.0f;
    float r1 = random_float(rng);
    float r2 = random_float(rng);
    float phi = (2.0f * PI) * r1;
    float st = sqrtf(r2);
    float ct = sqrtf(1.0f - r2);
    float sp, cp;
    pm_sincosf(phi, &sp, &cp);
    float4 hl = f4(st * cp, st * sp, ct, 0.0f);
    return normalize(hl.x * t + hl.y * b + hl.z * normal);
}
PHX_HDI float4 random_in_unit_hemisphere(Rng *rng, float4 normal) {
    float4 t, b;
    make_tbn(normal, &t, &b); // make_tbn ignores the normal's w, as the sampler does
    return random_in_unit_hemisphere_tbn(rng, normal, t, b);
}

// ---- codecs: include/device/encoding.h:10-74 ---------------------------------------------------
PHX_HDI u32 encode_rgbe(float4 power) {
    float m = fmaxf(power.x, fmaxf(power.y, power.z));
    if (m <= 0.0f)
        return 0u;
    int e;
    frexpf(m, &e);
    float scale = pm_exp2i(e); // ldexp(1.0f, e), exact
    u32 r = (u32)(power.x / scale * 256.0f);
    u32 g = (u32)(power.y / scale * 256.0f);
    u32 b = (u32)(power.z / scale * 256.0f);
    u32 E = (u32)(e + 128);
    r = r < 255u ? r : 255u;
    g = g < 255u ? g : 255u;
    b = b < 255u ? b : 255u;
    return r | (g << 8) | (b << 16) | (E << 24);
}
PHX_HDI float4 decode_rgbe(u32 rgbe) {
    u32 E = rgbe >> 24;
    if (E == 0)
        return zero4();
    float scale = pm_exp2i((i32)E - 136); // ldexp(1.0f, E - 128 - 8)
    return f4((float)(rgbe & 0xFFu) * scale, (float)((rgbe >> 8) & 0xFFu) * scale,
              (float)((rgbe >> 16) & 0xFFu) * scale, 0.0f);
}
PHX_HDI u32 encode_oct(float4 dir) {
    dir = normalize(dir);
    float l = (fabsf(dir.x) + fabsf(dir.y)) + fabsf(dir.z);
    float nx = dir.x / l, ny = dir.y / l;
    if (!(dir.z >= 0.0f)) {
        float sx = nx >= 0.0f ? 1.0f : -1.0f;
        float sy = ny >= 0.0f ? 1.0f : -1.0f;
        float wx = (1.0f - fabsf(ny)) * sx;
        float wy = (1.0f - fabsf(nx)) * sy;
        nx = wx;
        ny = wy;
    }
    u32 ux = (u32)(clampf(nx * 0.5f + 0.5f, 0.0f, 1.0f) * 65535.0f);
    u32 uy = (u32)(clampf(ny * 0.5f + 0.5f, 0.0f, 1.0f) * 65535.0f);
    return ux | (uy << 16);
}
PHX_HDI float4 decode_oct(u32 packed) {
    float fx = (float)(packed & 0xFFFFu) / 65535.0f;
    float fy = (float)((packed >> 16) & 0xFFFFu) / 65535.0f;
    fx = fx * 2.0f - 1.0f;
    fy = fy * 2.0f - 1.0f;
    float4 n = f4(fx, fy, (1.0f - fabsf(fx)) - fabsf(fy), 0.0f);
    float t = clampf(-n.z, 0.0f, 1.0f);
    n.x += n.x >= 0.0f ? -t : t;
    n.y += n.y >= 0.0f ? -t : t;
    return normalize(n);
}

// ---- grid hash: include/common/photon_hash.h:21-37 ---------------------------------------------
struct GridDev {
    float ox, oy, oz;
    float cx, cy, cz;
    u32 g;
    u32 pad;
};
PHX_HDI u32 get_hash(float px, float py, float pz, const GridDev &d) {
    float fx = (px - d.ox) / d.cx;
    float fy = (py - d.oy) / d.cy;
    float fz = (pz - d.oz) / d.cz;
    float gf = (float)d.g;
    if (fx < 0.0f || fy < 0.0f || fz < 0.0f || fx >= gf || fy >= gf || fz >= gf)
        return 0;
    u32 x = (u32)fx, y = (u32)fy, z = (u32)fz;
    return d.g * d.g * x + d.g * y + z + 1;
}

} // namespace phx
