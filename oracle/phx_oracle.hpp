// phx_oracle.hpp — TEST INFRASTRUCTURE ONLY.  CPU restatement of the reference SPPM pipeline.
//
// This is the correctness oracle of the repository.  It follows the reference's OpenCL kernels
// and device headers statement by statement (file:line cited per function) and runs them
// sequentially in a canonical order.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline use it; the library never links or calls it.
//
// PINNED TO THE REFERENCE ITSELF: the reference (alfazet/phosphor) ships no golden vectors and
// has no OpenCL runtime to run on here, so oracle/build_ref_sppm.py compiles its own kernels
// (kernels/*.cl with include/{common,device}/*.h, vector literals and one swizzle rewritten) and
// its host BVH builder, camera, light constructors and image formation for the CPU, with the
// builtins fixed as below.  tests/test_ref_pin.py checks this restatement against that build's
// outputs (tests/golden/ref_sppm_golden.npz): every stage bit for bit on eight scenes.
//
// Fixed choices where OpenCL leaves freedom (the same choices the device code makes):
//  * IEEE-754 binary32 arithmetic with no contraction (build with -ffp-contract=off);
//  * dot(a,b) = ((ax*bx + ay*by) + az*bz) + aw*bw; length = sqrt(dot(v,v)); normalize(v) =
//    v / length(v) (a zero vector is returned unchanged); rsqrt(x) = 1/sqrt(x); mix(a,b,t) =
//    a + (b-a)*t;
//  * transcendental builtins (sin, cos, exp, log, pow, acos, atan2, native_exp) are the
//    portable implementations of include/phx_math.h in float mode, std:: in double mode;
//  * canonical orders for the reference's atomic races: photons are stored in (photon index,
//    bounce) order — a sequential run of emit_photons.cl:98 — and the scatter is stable
//    (source index ascending within a cell) — a sequential run of scatter_photons.cl:13.
// The double instantiation is the FP64 image oracle: the same algorithm, RGBE/octahedral
// quantisation included, in double precision.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "../include/phx.h"
#include "../include/phx_math.h"

namespace orc {

using u32 = uint32_t;
using i32 = int32_t;
using u8 = uint8_t;

// ---- constants: include/common/constants.h:6-45 ----------------------------------------------
constexpr u32 SCAN_WG_SIZE = 256u;
constexpr u32 SCAN_ELEMENTS_PER_THREAD = 16u;
constexpr u32 SCAN_CHUNK_SIZE = SCAN_WG_SIZE * SCAN_ELEMENTS_PER_THREAD;
constexpr float EPS_F = 1e-5f;
constexpr float BBOX_EPS = 1e-3f;
constexpr float INF_F = 1e9f;
constexpr float PI_F = 3.141592654f;
constexpr float U32_MAX_F = 4294967296.0f;
constexpr u32 NO_TEXTURE = 0xFFFFFFFFu;
constexpr float AIR_IOR = 1.0f;
constexpr u32 MAX_RAY_BOUNCES = 5u;
constexpr float MIN_CELL_SIZE = 0.001f;
constexpr u32 BVH_STACK_SIZE = 24u;
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

// ---- scalar math dispatch ----------------------------------------------------------------------
template <class R> struct M;
template <> struct M<float> {
    static float sqrt(float x) { return std::sqrt(x); }
    static float sin(float x) { return pm_sinf(x); }
    static float cos(float x) { return pm_cosf(x); }
    static float exp(float x) { return pm_expf(x); }
    static float log(float x) { return pm_logf(x); }
    static float pow(float x, float y) { return pm_powf(x, y); }
    static float acos(float x) { return pm_acosf(x); }
    static float atan2(float y, float x) { return pm_atan2f(y, x); }
    static float floor(float x) { return std::floor(x); }
    static float ceil(float x) { return std::ceil(x); }
    static float fabs(float x) { return std::fabs(x); }
    static float fmax(float a, float b) { return std::fmax(a, b); }
    static float fmin(float a, float b) { return std::fmin(a, b); }
    static float ldexp(float x, int e) { return std::ldexp(x, e); }
    static float frexp(float x, int *e) { return std::frexp(x, e); }
};
template <> struct M<double> {
    static double sqrt(double x) { return std::sqrt(x); }
    static double sin(double x) { return std::sin(x); }
    static double cos(double x) { return std::cos(x); }
    static double exp(double x) { return std::exp(x); }
    static double log(double x) { return std::log(x); }
    static double pow(double x, double y) { return std::pow(x, y); }
    static double acos(double x) { return std::acos(x); }
    static double atan2(double y, double x) { return std::atan2(y, x); }
    static double floor(double x) { return std::floor(x); }
    static double ceil(double x) { return std::ceil(x); }
    static double fabs(double x) { return std::fabs(x); }
    static double fmax(double a, double b) { return std::fmax(a, b); }
    static double fmin(double a, double b) { return std::fmin(a, b); }
    static double ldexp(double x, int e) { return std::ldexp(x, e); }
    static double frexp(double x, int *e) { return std::frexp(x, e); }
};

// ---- OpenCL float4 with component-wise operators ----------------------------------------------
template <class R> struct V4 {
    R x, y, z, w;
};
template <class R> inline V4<R> mk(R x, R y, R z, R w) { return V4<R>{x, y, z, w}; }
template <class R> inline V4<R> from(const phx_f4 &v) { return V4<R>{(R)v.x, (R)v.y, (R)v.z, (R)v.w}; }
template <class R> inline V4<R> operator+(V4<R> a, V4<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class R> inline V4<R> operator-(V4<R> a, V4<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
template <class R> inline V4<R> operator*(V4<R> a, V4<R> b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class R> inline V4<R> operator/(V4<R> a, V4<R> b) { return {a.x / b.x, a.y / b.y, a.z / b.z, a.w / b.w}; }
template <class R> inline V4<R> operator*(V4<R> a, R s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class R> inline V4<R> operator*(R s, V4<R> a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
template <class R> inline V4<R> operator/(V4<R> a, R s) { return {a.x / s, a.y / s, a.z / s, a.w / s}; }
template <class R> inline V4<R> operator-(V4<R> a) { return {-a.x, -a.y, -a.z, -a.w}; }
template <class R> inline V4<R> &operator+=(V4<R> &a, V4<R> b) { return a = a + b; }
template <class R> inline V4<R> &operator*=(V4<R> &a, V4<R> b) { return a = a * b; }
template <class R> inline V4<R> &operator*=(V4<R> &a, R s) { return a = a * s; }
template <class R> inline V4<R> &operator/=(V4<R> &a, R s) { return a = a / s; }
template <class R> inline R dot(V4<R> a, V4<R> b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
template <class R> inline V4<R> cross(V4<R> a, V4<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, (R)0};
}
template <class R> inline R length(V4<R> v) { return M<R>::sqrt(dot(v, v)); }
template <class R> inline V4<R> normalize(V4<R> v) {
    R l = M<R>::sqrt(dot(v, v));
    if (l == (R)0)
        return v;
    return v / l;
}
template <class R> inline R clampr(R x, R lo, R hi) { return M<R>::fmin(M<R>::fmax(x, lo), hi); }
template <class R> inline V4<R> mix(V4<R> a, V4<R> b, R t) { return a + (b - a) * t; }
template <class R> inline V4<R> zero4() { return {(R)0, (R)0, (R)0, (R)0}; }
template <class R> inline V4<R> white4() { return {(R)1, (R)1, (R)1, (R)0}; }

template <class R> struct C {
    static constexpr R EPS = (R)EPS_F;
    static constexpr R INF = (R)INF_F;
    static constexpr R PI = (R)PI_F;
};

inline float as_float(u32 u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline u32 as_uint(float f) {
    u32 u;
    std::memcpy(&u, &f, 4);
    return u;
}

// ---- RNG: include/common/random.h:16-62 --------------------------------------------------------
struct Rng {
    u32 state;
};
inline Rng pcg_seed(u32 seed) { // random.h:16-24
    Rng r;
    r.state = 0u;
    r.state = r.state * 747796405u + 2891336453u;
    r.state += seed;
    r.state = r.state * 747796405u + 2891336453u;
    return r;
}
inline u32 random_u32(Rng *rng) { // random.h:29-34
    u32 old = rng->state;
    rng->state = rng->state * 747796405u + 2891336453u;
    return ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
}
template <class R> inline R random_float(Rng *rng); // random.h:36
template <> inline float random_float<float>(Rng *rng) { return (float)random_u32(rng) / U32_MAX_F; }
template <> inline double random_float<double>(Rng *rng) { return (double)random_u32(rng) / 4294967296.0; }

template <class R> inline void make_tbn(V4<R> normal, V4<R> *tangent, V4<R> *bitangent) { // utils.h:59-71
    normal.w = (R)0;
    V4<R> tmp = (M<R>::fabs(normal.x) > (R)0.1f) ? mk<R>(0, 1, 0, 0) : mk<R>(1, 0, 0, 0);
    *tangent = cross(normal, tmp);
    if (length(*tangent) < C<R>::EPS) {
        tmp = mk<R>(0, 0, 1, 0);
        *tangent = cross(normal, tmp);
    }
    *tangent = normalize(*tangent);
    *bitangent = cross(normal, *tangent);
}

template <class R> inline V4<R> random_unit_vector(Rng *rng) { // random.h:40-46
    R z = (R)2 * random_float<R>(rng) - (R)1;
    R r = M<R>::sqrt(M<R>::fmax((R)0, (R)1 - z * z));
    R phi = ((R)2 * C<R>::PI) * random_float<R>(rng);
    return mk<R>(r * M<R>::cos(phi), r * M<R>::sin(phi), z, (R)0);
}

template <class R> inline V4<R> random_in_unit_hemisphere(Rng *rng, V4<R> normal) { // random.h:48-62
    normal.w = (R)0;
    R r1 = random_float<R>(rng);
    R r2 = random_float<R>(rng);
    R phi = ((R)2 * C<R>::PI) * r1;
    R sin_theta = M<R>::sqrt(r2);
    R cos_theta = M<R>::sqrt((R)1 - r2);
    V4<R> hl = mk<R>(sin_theta * M<R>::cos(phi), sin_theta * M<R>::sin(phi), cos_theta, (R)0);
    V4<R> t, b;
    make_tbn(normal, &t, &b);
    return normalize(hl.x * t + hl.y * b + hl.z * normal);
}

// ---- codecs: include/device/encoding.h:10-74 ---------------------------------------------------
template <class R> inline u32 encode_rgbe(V4<R> power) { // encoding.h:10-29
    R m = M<R>::fmax(power.x, M<R>::fmax(power.y, power.z));
    if (m <= (R)0)
        return 0u;
    int e;
    M<R>::frexp(m, &e);
    R scale = M<R>::ldexp((R)1, e);
    u32 r = (u32)(power.x / scale * (R)256);
    u32 g = (u32)(power.y / scale * (R)256);
    u32 b = (u32)(power.z / scale * (R)256);
    u32 E = (u32)(e + 128);
    r = std::min(r, 255u);
    g = std::min(g, 255u);
    b = std::min(b, 255u);
    return r | (g << 8) | (b << 16) | (E << 24);
}
template <class R> inline V4<R> decode_rgbe(u32 rgbe) { // encoding.h:31-39
    u32 E = rgbe >> 24;
    if (E == 0)
        return zero4<R>();
    R scale = M<R>::ldexp((R)1, (i32)E - 128 - 8);
    return mk<R>((R)(rgbe & 0xFF) * scale, (R)((rgbe >> 8) & 0xFF) * scale, (R)((rgbe >> 16) & 0xFF) * scale, (R)0);
}
template <class R> inline u32 encode_oct(V4<R> dir) { // encoding.h:47-59
    dir = normalize(dir);
    R l = (M<R>::fabs(dir.x) + M<R>::fabs(dir.y)) + M<R>::fabs(dir.z);
    R nx = dir.x / l, ny = dir.y / l;
    if (!(dir.z >= (R)0)) { // oct_wrap (encoding.h:43-45)
        R sx = nx >= (R)0 ? (R)1 : (R)-1;
        R sy = ny >= (R)0 ? (R)1 : (R)-1;
        R wx = ((R)1 - M<R>::fabs(ny)) * sx;
        R wy = ((R)1 - M<R>::fabs(nx)) * sy;
        nx = wx;
        ny = wy;
    }
    u32 ux = (u32)(clampr<R>(nx * (R)0.5 + (R)0.5, (R)0, (R)1) * (R)65535);
    u32 uy = (u32)(clampr<R>(ny * (R)0.5 + (R)0.5, (R)0, (R)1) * (R)65535);
    return ux | (uy << 16);
}
template <class R> inline V4<R> decode_oct(u32 packed) { // encoding.h:61-74
    R fx = (R)(packed & 0xFFFF) / (R)65535;
    R fy = (R)((packed >> 16) & 0xFFFF) / (R)65535;
    fx = fx * (R)2 - (R)1;
    fy = fy * (R)2 - (R)1;
    V4<R> n = mk<R>(fx, fy, ((R)1 - M<R>::fabs(fx)) - M<R>::fabs(fy), (R)0);
    R t = clampr<R>(-n.z, (R)0, (R)1);
    n.x += n.x >= (R)0 ? -t : t;
    n.y += n.y >= (R)0 ? -t : t;
    return normalize(n);
}

// ---- scene view (pointers into phx_scene arrays; SoA split of geometry.cpp:6-51) -------------
struct Scene {
    const phx_triangle *tris = nullptr;
    u32 n_tris = 0;
    const phx_triangle *etris = nullptr;
    u32 n_etris = 0;
    const phx_material *materials = nullptr;
    const phx_uv_transform_block *uv = nullptr;
    const phx_light *lights = nullptr;
    u32 n_lights = 0;
    const float *lum_pref_sum = nullptr;
    float total_lum = 0.0f;
    const phx_texture_meta *tex_meta = nullptr;
    const u8 *tex_atlas = nullptr;
    const float *envmap = nullptr;
    u32 env_w = 0, env_h = 0;
    u32 has_envmap = 0;
    phx_camera_params camera{};
    const phx_bvh_node *bvh = nullptr;
    phx_f4 scene_center{};
    float scene_radius = 0.0f;
};

// ---- hit.h:13-197 ------------------------------------------------------------------------------
template <class R> struct HitRecord {
    R t, u, v;
    u32 tri_index, mat_index;
};
template <class R> struct SurfaceHit {
    V4<R> position, normal;
    R uvx, uvy;
    R t;
    u32 mat_index, tri_index;
    bool front_face;
};

template <class R> inline V4<R> compute_bary(R bx, R by, V4<R> v0, V4<R> v1, V4<R> v2) { // hit.h:31-43
    R w0 = (R)1 - bx - by;
    R w1 = bx, w2 = by;
    return mk<R>(w0 * v0.x + w1 * v1.x + w2 * v2.x, w0 * v0.y + w1 * v1.y + w2 * v2.y,
                 w0 * v0.z + w1 * v1.z + w2 * v2.z, (R)0);
}

template <class R>
inline bool is_triangle_hit(const Scene &sc, u32 tri_idx, V4<R> origin, V4<R> dir, R t_min, R t_max,
                            HitRecord<R> *rec) { // hit.h:45-78
    const phx_triangle &tr = sc.tris[tri_idx];
    V4<R> v0 = from<R>(tr.v0), v1 = from<R>(tr.v1), v2 = from<R>(tr.v2);
    V4<R> e1 = v1 - v0;
    V4<R> e2 = v2 - v0;
    V4<R> h = cross(dir, e2);
    R a = dot(e1, h);
    if (M<R>::fabs(a) < C<R>::EPS)
        return false;
    R f = (R)1 / a;
    V4<R> s = origin - v0;
    R u = f * dot(s, h);
    if (u < (R)0 || u > (R)1)
        return false;
    V4<R> q = cross(s, e1);
    R v = f * dot(dir, q);
    if (v < (R)0 || u + v > (R)1)
        return false;
    R t = f * dot(e2, q);
    if (t < t_min || t > t_max)
        return false;
    rec->t = t;
    rec->u = u;
    rec->v = v;
    rec->tri_index = tri_idx;
    rec->mat_index = tr.mat_index;
    return true;
}

template <class R>
inline bool bbox_hit(const phx_bvh_node &nd, V4<R> origin, V4<R> dir, R t_min, R t_max) { // hit.h:80-133
    R inv_dx = (R)1 / dir.x;
    R tx0 = ((R)nd.min.x - origin.x) * inv_dx;
    R tx1 = ((R)nd.max.x - origin.x) * inv_dx;
    if (tx0 < tx1) {
        if (tx0 > t_min) t_min = tx0;
        if (tx1 < t_max) t_max = tx1;
    } else {
        if (tx1 > t_min) t_min = tx1;
        if (tx0 < t_max) t_max = tx0;
    }
    if (t_max <= t_min)
        return false;
    R inv_dy = (R)1 / dir.y;
    R ty0 = ((R)nd.min.y - origin.y) * inv_dy;
    R ty1 = ((R)nd.max.y - origin.y) * inv_dy;
    if (ty0 < ty1) {
        if (ty0 > t_min) t_min = ty0;
        if (ty1 < t_max) t_max = ty1;
    } else {
        if (ty1 > t_min) t_min = ty1;
        if (ty0 < t_max) t_max = ty0;
    }
    if (t_max <= t_min)
        return false;
    R inv_dz = (R)1 / dir.z;
    R tz0 = ((R)nd.min.z - origin.z) * inv_dz;
    R tz1 = ((R)nd.max.z - origin.z) * inv_dz;
    if (tz0 < tz1) {
        if (tz0 > t_min) t_min = tz0;
        if (tz1 < t_max) t_max = tz1;
    } else {
        if (tz1 > t_min) t_min = tz1;
        if (tz0 < t_max) t_max = tz0;
    }
    if (t_max <= t_min)
        return false;
    return true;
}

template <class R>
inline bool scene_intersect(const Scene &sc, V4<R> origin, V4<R> dir, R t_min, R t_max,
                            HitRecord<R> *rec) { // hit.h:135-172
    i32 p = 0;
    u32 stack[BVH_STACK_SIZE];
    stack[0] = 0;
    bool found = false;
    R closest = t_max;
    while (p >= 0) {
        u32 index = stack[p];
        const phx_bvh_node &node = sc.bvh[index];
        p--;
        if (!bbox_hit<R>(node, origin, dir, t_min, closest))
            continue;
        u32 triangle_index = as_uint(node.min.w);
        if (triangle_index != 0xFFFFFFFFu) {
            HitRecord<R> cand;
            if (is_triangle_hit<R>(sc, triangle_index, origin, dir, t_min, closest, &cand)) {
                closest = cand.t;
                *rec = cand;
                found = true;
            }
            continue;
        }
        if (p + 2 >= (i32)BVH_STACK_SIZE)
            continue;
        u32 right_child = as_uint(node.max.w);
        stack[++p] = right_child;
        stack[++p] = index + 1;
    }
    return found;
}

template <class R>
inline SurfaceHit<R> process_hit(const Scene &sc, const HitRecord<R> &rec, V4<R> origin, V4<R> dir) { // hit.h:174-197
    SurfaceHit<R> sh;
    sh.t = rec.t;
    sh.mat_index = rec.mat_index;
    sh.tri_index = rec.tri_index;
    sh.position = origin + dir * rec.t;
    R u = rec.u, v = rec.v;
    R w = (R)1 - u - v;
    const phx_triangle &tr = sc.tris[rec.tri_index];
    V4<R> outward = normalize(compute_bary<R>(u, v, from<R>(tr.n0), from<R>(tr.n1), from<R>(tr.n2)));
    bool front = dot(dir, outward) < (R)0;
    sh.normal = front ? outward : -outward;
    sh.front_face = front;
    sh.uvx = w * (R)tr.uv0.x + u * (R)tr.uv1.x + v * (R)tr.uv2.x;
    sh.uvy = w * (R)tr.uv0.y + u * (R)tr.uv1.y + v * (R)tr.uv2.y;
    return sh;
}

// ---- textures: include/common/material.h:66-149 ------------------------------------------------
template <class R> inline V4<R> srgb_to_linear(V4<R> c) { // material.h:66
    return mk<R>(M<R>::pow(c.x, (R)2.2f), M<R>::pow(c.y, (R)2.2f), M<R>::pow(c.z, (R)2.2f), c.w);
}

template <class R>
inline V4<R> naive_sample_texture(const Scene &sc, u32 index, R ux, R uy) { // material.h:77-93
    if (index == NO_TEXTURE)
        return white4<R>();
    const phx_texture_meta &meta = sc.tex_meta[index];
    u32 px = std::min((u32)(ux * (R)meta.width), meta.width - 1);
    u32 py = std::min((u32)(uy * (R)meta.height), meta.height - 1);
    u32 texel = meta.atlas_offset + (py * meta.width + px) * 3u;
    R r = (R)sc.tex_atlas[texel + 0] / (R)255;
    R g = (R)sc.tex_atlas[texel + 1] / (R)255;
    R b = (R)sc.tex_atlas[texel + 2] / (R)255;
    return mk<R>(r, g, b, (R)1);
}

template <class R> inline V4<R> texel4(const Scene &sc, i32 idx) {
    return mk<R>((R)sc.tex_atlas[idx], (R)sc.tex_atlas[idx + 1], (R)sc.tex_atlas[idx + 2], (R)255) / (R)255;
}

template <class R> inline V4<R> sample_texture(const Scene &sc, u32 index, R ux, R uy) { // material.h:95-140
    if (index == NO_TEXTURE)
        return white4<R>();
    const phx_texture_meta &meta = sc.tex_meta[index];
    i32 w = (i32)meta.width;
    i32 h = (i32)meta.height;
    ux = ux - M<R>::floor(ux);
    uy = uy - M<R>::floor(uy);
    uy = (R)1 - uy;
    R x = M<R>::fmin(ux * (R)w, (R)(w - 1));
    R y = M<R>::fmin(uy * (R)h, (R)(h - 1));
    i32 x1 = std::min((i32)x, w - 1);
    i32 x2 = std::min((i32)M<R>::ceil(x), w - 1);
    i32 y1 = std::min((i32)y, h - 1);
    i32 y2 = std::min((i32)M<R>::ceil(y), h - 1);
    i32 ch = (i32)meta.channels;
    i32 off = (i32)meta.atlas_offset;
    V4<R> Q11 = texel4<R>(sc, off + (y1 * w + x1) * ch);
    V4<R> Q12 = texel4<R>(sc, off + (y2 * w + x1) * ch);
    V4<R> Q21 = texel4<R>(sc, off + (y1 * w + x2) * ch);
    V4<R> Q22 = texel4<R>(sc, off + (y2 * w + x2) * ch);
    if (x2 == x1 && y2 == y1)
        return naive_sample_texture<R>(sc, index, ux, uy);
    else if (x2 == x1)
        return mix(Q11, Q12, y - (R)y1);
    else if (y2 == y1)
        return mix(Q11, Q21, x - (R)x1);
    R denom = (R)((x2 - x1) * (y2 - y1));
    R w11 = ((R)x2 - x) * ((R)y2 - y) / denom;
    R w12 = ((R)x2 - x) * (y - (R)y1) / denom;
    R w21 = (x - (R)x1) * ((R)y2 - y) / denom;
    R w22 = (x - (R)x1) * (y - (R)y1) / denom;
    return w11 * Q11 + w12 * Q12 + w21 * Q21 + w22 * Q22;
}

template <class R>
inline V4<R> sample_texture_uv(const Scene &sc, u32 mat_index, u32 tex_index, R ux, R uy, u32 slot) { // material.h:142-149
    const phx_uv_transform *t = &sc.uv[mat_index].diff + slot;
    R sx = ux * (R)t->uv_scale.x, sy = uy * (R)t->uv_scale.y;
    R c = M<R>::cos((R)t->uv_rotation), s = M<R>::sin((R)t->uv_rotation);
    R rx = c * sx - s * sy, ry = s * sx + c * sy;
    return sample_texture<R>(sc, tex_index, rx + (R)t->uv_offset.x, ry + (R)t->uv_offset.y);
}

// ---- shading.h:13-213 --------------------------------------------------------------------------
template <class R> struct ShadingContext {
    V4<R> base_color, emissive, shading_normal;
    R metallic, roughness, transmission, occlusion, ior;
};
template <class R> struct IorStack {
    R ior[IOR_STACK_SIZE];
    u32 cur;
};
template <class R> inline void init_ior_stack(IorStack<R> *s, R initial) { s->cur = 0; s->ior[0] = initial; }
template <class R> inline R current_ior(const IorStack<R> *s) { return s->ior[s->cur]; }
template <class R> inline R target_ior(const IorStack<R> *s, R inside, bool front) { // shading.h:38-42
    if (front)
        return inside;
    return (s->cur == 0) ? (R)AIR_IOR : s->ior[s->cur - 1];
}
template <class R> inline void update_ior_stack(IorStack<R> *s, R inside, bool front) { // shading.h:44-54
    if (front) {
        if (s->cur < IOR_STACK_SIZE - 1) {
            s->cur++;
            s->ior[s->cur] = inside;
        }
    } else {
        if (s->cur > 0)
            s->cur--;
    }
}

template <class R> inline V4<R> apply_normal_map(V4<R> ms, V4<R> gn, V4<R> t, V4<R> b) { // shading.h:56-62
    V4<R> n = mk<R>(ms.x * (R)2 - (R)1, ms.y * (R)2 - (R)1, ms.z * (R)2 - (R)1, (R)0);
    V4<R> p = n.x * t + n.y * b + n.z * gn;
    R len = length(p);
    return (len > C<R>::EPS) ? (p / len) : gn;
}

template <class R>
inline ShadingContext<R> evaluate_material(const Scene &sc, const phx_material &mat, u32 mat_index, R ux, R uy,
                                           V4<R> gn, V4<R> t, V4<R> b) { // shading.h:75-123
    ShadingContext<R> ctx;
    ctx.base_color = from<R>(mat.base_color);
    if (mat.diff_index != NO_TEXTURE)
        ctx.base_color *= srgb_to_linear(sample_texture_uv<R>(sc, mat_index, mat.diff_index, ux, uy, 0));
    ctx.emissive = from<R>(mat.emissive);
    if (mat.emis_index != NO_TEXTURE)
        ctx.emissive *= srgb_to_linear(sample_texture_uv<R>(sc, mat_index, mat.emis_index, ux, uy, 1));
    ctx.metallic = (R)mat.metallic;
    ctx.roughness = (R)mat.roughness;
    if (mat.metal_rough_index != NO_TEXTURE) {
        V4<R> mr = sample_texture_uv<R>(sc, mat_index, mat.metal_rough_index, ux, uy, 4);
        ctx.metallic *= mr.z;
        ctx.roughness *= mr.y;
    }
    ctx.roughness = clampr<R>(ctx.roughness, (R)MIN_ROUGHNESS, (R)1);
    ctx.transmission = (R)mat.transmission;
    if (mat.transmission_index != NO_TEXTURE) {
        V4<R> tx = sample_texture_uv<R>(sc, mat_index, mat.transmission_index, ux, uy, 5);
        ctx.transmission *= tx.x;
    }
    ctx.occlusion = (R)1;
    if (mat.occlusion_index != NO_TEXTURE) {
        V4<R> occ = sample_texture_uv<R>(sc, mat_index, mat.occlusion_index, ux, uy, 3);
        ctx.occlusion = occ.x;
    }
    ctx.ior = (R)mat.ior;
    ctx.shading_normal = gn;
    if (mat.norm_index != NO_TEXTURE) {
        V4<R> ms = sample_texture_uv<R>(sc, mat_index, mat.norm_index, ux, uy, 2);
        ctx.shading_normal = apply_normal_map(ms, gn, t, b);
    }
    return ctx;
}

template <class R> inline V4<R> beer_lambert(V4<R> att_color, R att_dist, R travel) { // shading.h:125-133
    if (att_dist < C<R>::EPS)
        return white4<R>();
    V4<R> sigma = mk<R>(-M<R>::log(M<R>::fmax(att_color.x, C<R>::EPS)), -M<R>::log(M<R>::fmax(att_color.y, C<R>::EPS)),
                        -M<R>::log(M<R>::fmax(att_color.z, C<R>::EPS)), (R)0) /
                  att_dist;
    return mk<R>(M<R>::exp(-sigma.x * travel), M<R>::exp(-sigma.y * travel), M<R>::exp(-sigma.z * travel), (R)0);
}

// ---- bsdfs.h:11-121 ----------------------------------------------------------------------------
template <class R> inline V4<R> reflect(V4<R> in, V4<R> n) { return normalize(in - ((R)2 * dot(in, n)) * n); }
template <class R> inline V4<R> safe_reflect(V4<R> d, V4<R> n, V4<R> gn) { // bsdfs.h:15-22
    V4<R> r = reflect(d, n);
    if (dot(r, gn) <= (R)0) {
        r = r - dot(r, gn) * gn;
        r = normalize(r);
    }
    return r;
}

template <class R>
inline V4<R> ggx_sample_vndf(Rng *rng, V4<R> normal, V4<R> gn, V4<R> view, R roughness) { // bsdfs.h:27-72
    R alpha = roughness * roughness;
    V4<R> t, b;
    make_tbn(normal, &t, &b);
    V4<R> vl = normalize(mk<R>(dot(view, t), dot(view, b), dot(view, normal), (R)0));
    V4<R> vh = normalize(mk<R>(alpha * vl.x, alpha * vl.y, vl.z, (R)0));
    R len_sq = vh.x * vh.x + vh.y * vh.y;
    V4<R> T1 = (len_sq > (R)0) ? mk<R>(-vh.y, vh.x, (R)0, (R)0) * ((R)1 / M<R>::sqrt(len_sq)) : mk<R>(1, 0, 0, 0);
    V4<R> T2 = cross(vh, T1);
    R s = (R)0.5 * ((R)1 + vh.z);
    V4<R> ne;
    for (u32 a = 0; a < GGX_SAMPLING_ATTEMPTS; a++) {
        R u1 = random_float<R>(rng);
        R u2 = random_float<R>(rng);
        R r = M<R>::sqrt(u1);
        R phi = ((R)2 * C<R>::PI) * u2;
        R t1 = r * M<R>::cos(phi);
        R t2 = r * M<R>::sin(phi);
        t2 = ((R)1 - s) * M<R>::sqrt(M<R>::fmax((R)0, (R)1 - t1 * t1)) + s * t2;
        R nz2 = M<R>::fmax((R)0, (R)1 - t1 * t1 - t2 * t2);
        V4<R> nh = t1 * T1 + t2 * T2 + M<R>::sqrt(nz2) * vh;
        V4<R> nel = normalize(mk<R>(alpha * nh.x, alpha * nh.y, M<R>::fmax((R)0, nh.z), (R)0));
        ne = normalize(nel.x * t + nel.y * b + nel.z * normal);
        V4<R> refl = reflect(-view, ne);
        if (dot(refl, gn) >= (R)0)
            return ne;
    }
    return normal;
}

template <class R> inline R smith_g1_ggx(R cos_theta, R alpha) { // bsdfs.h:77-83
    if (cos_theta <= (R)0)
        return (R)0;
    R a2 = alpha * alpha;
    return (R)2 * cos_theta / (cos_theta + M<R>::sqrt(a2 + ((R)1 - a2) * cos_theta * cos_theta));
}
template <class R> inline R fresnel(R r0, V4<R> in, V4<R> n) { // bsdfs.h:86-89
    R c = M<R>::fabs(dot(in, n));
    return r0 + ((R)1 - r0) * M<R>::pow((R)1 - c, (R)5);
}
template <class R> inline V4<R> fresnel4(V4<R> r0, V4<R> in, V4<R> n) { // bsdfs.h:91-94
    R c = M<R>::fabs(dot(in, n));
    R p = M<R>::pow((R)1 - c, (R)5);
    return mk<R>(r0.x + ((R)1 - r0.x) * p, r0.y + ((R)1 - r0.y) * p, r0.z + ((R)1 - r0.z) * p,
                 r0.w + ((R)1 - r0.w) * p);
}
template <class R> inline R fresnel_refracted(R i1, R i2, V4<R> in, V4<R> n) { // bsdfs.h:96-99
    R r0 = M<R>::pow((i1 - i2) / (i1 + i2), (R)2);
    return fresnel(r0, in, n);
}
template <class R> inline V4<R> refract(V4<R> in, V4<R> n, R eta1, R eta2, bool *tir) { // bsdfs.h:101-114
    R eta = eta1 / eta2;
    R ndi = dot(in, n);
    R sin_t2 = eta * eta * ((R)1 - ndi * ndi);
    if (sin_t2 > (R)1) {
        *tir = true;
        return reflect(in, n);
    }
    *tir = false;
    V4<R> rf = eta * in - (eta * ndi + M<R>::sqrt((R)1 - sin_t2)) * n;
    return normalize(rf);
}
template <class R> inline R ggx_ndf(R ndh, R alpha) { // bsdfs.h:117-121
    R a2 = alpha * alpha;
    R d = ndh * ndh * (a2 - (R)1) + (R)1;
    return a2 / M<R>::fmax(C<R>::PI * d * d, C<R>::EPS);
}

enum { BSDF_DIFFUSE = 0, BSDF_METALLIC = 1, BSDF_FRESNEL = 2, BSDF_TRANSMIT = 3 };
template <class R> struct BsdfSample {
    V4<R> dir, throughput;
    u32 event;
};

template <class R>
inline BsdfSample<R> sample_bsdf(Rng *rng, const ShadingContext<R> &ctx, V4<R> sn, V4<R> gn, V4<R> view,
                                 IorStack<R> *ior, bool front) { // shading.h:150-213
    BsdfSample<R> s;
    V4<R> h = ggx_sample_vndf<R>(rng, sn, gn, view, ctx.roughness);
    R alpha = ctx.roughness * ctx.roughness;
    if (random_float<R>(rng) < ctx.metallic) {
        s.dir = safe_reflect(-view, h, gn);
        R cl = M<R>::fmax((R)0, dot(s.dir, sn));
        R g1 = smith_g1_ggx(cl, alpha);
        s.throughput = fresnel4(ctx.base_color, -view, h) * g1;
        s.event = BSDF_METALLIC;
        return s;
    }
    R i1 = current_ior(ior);
    R i2 = target_ior(ior, ctx.ior, front);
    R fr = fresnel_refracted(i1, i2, -view, h);
    R r_diel = random_float<R>(rng);
    if (r_diel < fr) {
        s.dir = safe_reflect(-view, h, gn);
        R cl = M<R>::fmax((R)0, dot(s.dir, sn));
        R g1 = smith_g1_ggx(cl, alpha);
        s.throughput = mk<R>(g1, g1, g1, (R)0);
        s.event = BSDF_FRESNEL;
        return s;
    }
    R r_trans = (r_diel - fr) / M<R>::fmax((R)1 - fr, C<R>::EPS);
    if (r_trans < ctx.transmission) {
        bool tir;
        V4<R> rf = refract(-view, h, i1, i2, &tir);
        if (tir) {
            s.dir = safe_reflect(-view, h, gn);
            R cl = M<R>::fmax((R)0, dot(s.dir, sn));
            R g1 = smith_g1_ggx(cl, alpha);
            s.throughput = mk<R>(g1, g1, g1, (R)0);
            s.event = BSDF_FRESNEL;
            return s;
        }
        bool transmitted = dot(rf, h) < (R)0;
        if (transmitted)
            update_ior_stack(ior, ctx.ior, front);
        s.dir = rf;
        R cl = M<R>::fmax((R)0, M<R>::fabs(dot(rf, sn)));
        R g1 = smith_g1_ggx(cl, alpha);
        s.throughput = ctx.base_color * g1;
        s.event = BSDF_TRANSMIT;
        return s;
    }
    s.dir = random_in_unit_hemisphere(rng, sn);
    if (dot(s.dir, gn) <= (R)0)
        s.dir = random_in_unit_hemisphere(rng, gn);
    s.throughput = ctx.base_color;
    s.event = BSDF_DIFFUSE;
    return s;
}

// ---- light_sampling.h:18-390 -------------------------------------------------------------------
struct Bary {
    double u, v, w;
};
template <class R> struct EmissivePoint {
    u32 tri_idx;
    R bu, bv, bw;
    V4<R> pos, normal;
};
template <class R> struct LightFragment {
    V4<R> radiance, dir;
    R dist, n_dot_dir;
};

template <class R> inline R spotlight_falloff(R c, R ci, R co) { // light_sampling.h:36-39
    R t = clampr<R>((c - co) / (ci - co + C<R>::EPS), (R)0, (R)1);
    return t * t * ((R)3 - (R)2 * t);
}
template <class R> inline V4<R> light_flux(const phx_light &l, R scale) { // light_sampling.h:41-43
    return mk<R>((R)l.power.x, (R)l.power.y, (R)l.power.z, (R)0) / scale;
}
template <class R> inline void fill_light_vecs(V4<R> from_, V4<R> to, V4<R> *dir, R *dist, R *dist_sq) { // :45-50
    V4<R> d = to - from_;
    *dist_sq = M<R>::fmax(dot(d, d), C<R>::EPS);
    *dist = M<R>::sqrt(*dist_sq);
    *dir = d / *dist;
}
template <class R>
inline u32 choose_emissive_triangle(Rng *rng, const Scene &sc, u32 start, u32 n, R total_area) { // :52-67
    if (n <= 1 || total_area <= C<R>::EPS)
        return start;
    R r = random_float<R>(rng) * total_area;
    R accum = (R)0;
    for (u32 i = 0; i < n; i++) {
        const phx_triangle &ev = sc.etris[start + i];
        V4<R> v0 = from<R>(ev.v0), v1 = from<R>(ev.v1), v2 = from<R>(ev.v2);
        accum += (R)0.5 * length(cross(v1 - v0, v2 - v0));
        if (r <= accum)
            return start + i;
    }
    return start + n - 1;
}
template <class R>
inline EmissivePoint<R> sample_emissive_point(Rng *rng, const Scene &sc, u32 start, u32 n, R total_area) { // :82-100
    EmissivePoint<R> p;
    p.tri_idx = choose_emissive_triangle<R>(rng, sc, start, n, total_area);
    R r1 = random_float<R>(rng); // sample_barycentric :69-80
    R r2 = random_float<R>(rng);
    R s = M<R>::sqrt(r1);
    p.bu = (R)1 - s;
    p.bv = r2 * s;
    p.bw = (R)1 - p.bu - p.bv;
    const phx_triangle &ev = sc.etris[p.tri_idx];
    V4<R> v0 = from<R>(ev.v0), v1 = from<R>(ev.v1), v2 = from<R>(ev.v2);
    p.pos = p.bw * v0 + p.bu * v1 + p.bv * v2;
    V4<R> nn = p.bw * from<R>(ev.n0) + p.bu * from<R>(ev.n1) + p.bv * from<R>(ev.n2);
    if (length(nn) > C<R>::EPS)
        p.normal = normalize(nn);
    else
        p.normal = normalize(cross(v1 - v0, v2 - v0));
    return p;
}
template <class R>
inline V4<R> apply_emissive_texture(const Scene &sc, V4<R> color, u32 tex_index, const EmissivePoint<R> &p) { // :102-115
    if (tex_index == NO_TEXTURE)
        return color;
    const phx_triangle &et = sc.etris[p.tri_idx];
    R ux = p.bw * (R)et.uv0.x + p.bu * (R)et.uv1.x + p.bv * (R)et.uv2.x;
    R uy = p.bw * (R)et.uv0.y + p.bu * (R)et.uv1.y + p.bv * (R)et.uv2.y;
    u32 mat_idx = et.mat_index;
    V4<R> tc = sample_texture_uv<R>(sc, mat_idx, tex_index, ux, uy, 1);
    return color * srgb_to_linear(tc);
}
template <class R> inline u32 select_light(Rng *rng, const Scene &sc, R *scale) { // :117-139
    u32 n = sc.n_lights;
    R total = (R)sc.total_lum;
    if (n == 0 || total < C<R>::EPS) {
        *scale = (R)1;
        return 0;
    }
    R r = random_float<R>(rng) * total;
    u32 low = 0, high = n;
    while (low < high) {
        u32 mid = (low + high) / 2;
        if ((R)sc.lum_pref_sum[mid] < r)
            low = mid + 1;
        else
            high = mid;
    }
    if (low >= n)
        low = n - 1;
    R lum = (low == 0) ? (R)sc.lum_pref_sum[0] : ((R)sc.lum_pref_sum[low] - (R)sc.lum_pref_sum[low - 1]);
    *scale = M<R>::fmax(lum / total, C<R>::EPS);
    return low;
}

template <class R>
inline void sample_light(Rng *rng, const Scene &sc, V4<R> *origin, V4<R> *dir, V4<R> *power) { // :200-227
    if (sc.n_lights == 0 || (R)sc.total_lum < C<R>::EPS) {
        *origin = zero4<R>();
        *dir = mk<R>(0, 1, 0, 0);
        *power = zero4<R>();
        return;
    }
    R scale;
    u32 idx = select_light<R>(rng, sc, &scale);
    const phx_light &L = sc.lights[idx];
    if (L.kind == PHX_LIGHT_POINT) { // :141-145
        *origin = from<R>(L.position);
        *dir = random_unit_vector<R>(rng);
        *power = from<R>(L.power) * ((R)4 * C<R>::PI);
    } else if (L.kind == PHX_LIGHT_SPOT) { // :147-167
        *origin = from<R>(L.position);
        R ci = M<R>::cos((R)L.aux.x);
        R co = M<R>::cos((R)L.aux.y);
        R r1 = random_float<R>(rng);
        R r2 = random_float<R>(rng);
        R ct = (R)1 - r1 * ((R)1 - co);
        R st = M<R>::sqrt(M<R>::fmax((R)0, (R)1 - ct * ct));
        R phi = ((R)2 * C<R>::PI) * r2;
        V4<R> ld = mk<R>(st * M<R>::cos(phi), st * M<R>::sin(phi), ct, (R)0);
        V4<R> t, b;
        V4<R> ldir = normalize(from<R>(L.direction));
        make_tbn(ldir, &t, &b);
        *dir = normalize(ld.x * t + ld.y * b + ld.z * ldir);
        R fo = spotlight_falloff(ct, ci, co);
        R sa = ((R)2 * C<R>::PI) * ((R)1 - co);
        *power = from<R>(L.power) * fo * sa;
    } else if (L.kind == PHX_LIGHT_DIRECTIONAL) { // :188-198
        V4<R> center = from<R>(sc.scene_center);
        R radius = (R)sc.scene_radius;
        R r1 = radius * M<R>::sqrt(random_float<R>(rng));
        R r2 = ((R)2 * C<R>::PI) * random_float<R>(rng);
        V4<R> disk = r1 * (M<R>::cos(r2) * from<R>(L.tangent) + M<R>::sin(r2) * from<R>(L.bitangent));
        *dir = from<R>(L.direction);
        *origin = center - from<R>(L.direction) * (R)2 * radius + disk;
        *power = from<R>(L.power) * C<R>::PI * radius * radius;
    } else { // textured :169-186
        u32 tex_idx = as_uint(L.aux.x);
        u32 start = as_uint(L.aux.y);
        u32 ntri = as_uint(L.aux.z);
        R area = (R)L.aux.w;
        EmissivePoint<R> p = sample_emissive_point<R>(rng, sc, start, ntri, area);
        *dir = random_in_unit_hemisphere(rng, p.normal);
        *origin = p.pos + C<R>::EPS * *dir;
        *power = apply_emissive_texture<R>(sc, from<R>(L.power), tex_idx, p);
    }
    *power /= scale;
}

template <class R>
inline bool sample_light_fragment(Rng *rng, const Scene &sc, V4<R> pos, V4<R> normal, LightFragment<R> *out) { // :231-300
    if (sc.n_lights == 0 || (R)sc.total_lum < C<R>::EPS)
        return false;
    R scale;
    u32 li = select_light<R>(rng, sc, &scale);
    const phx_light &L = sc.lights[li];
    V4<R> flux = light_flux<R>(L, scale);
    V4<R> dir;
    R dist, dist_sq, ndd;
    V4<R> radiance;
    if (L.kind == PHX_LIGHT_POINT || L.kind == PHX_LIGHT_SPOT) {
        fill_light_vecs(pos, from<R>(L.position), &dir, &dist, &dist_sq);
        ndd = dot(dir, normal);
        if (ndd <= (R)0)
            return false;
        R cone = (R)1;
        if (L.kind == PHX_LIGHT_SPOT) {
            R cd = dot(-dir, normalize(from<R>(L.direction)));
            cone = spotlight_falloff(cd, M<R>::cos((R)L.aux.x), M<R>::cos((R)L.aux.y));
            if (cone < C<R>::EPS)
                return false;
        }
        radiance = flux * cone * ndd / dist_sq;
    } else if (L.kind == PHX_LIGHT_DIRECTIONAL) {
        dir = normalize(-from<R>(L.direction));
        dist = C<R>::INF;
        ndd = dot(dir, normal);
        if (ndd <= (R)0)
            return false;
        radiance = flux * ndd;
    } else {
        u32 tex_index = as_uint(L.aux.x);
        u32 start = as_uint(L.aux.y);
        u32 ntri = as_uint(L.aux.z);
        R area = (R)L.aux.w;
        if (area < C<R>::EPS)
            return false;
        EmissivePoint<R> p = sample_emissive_point<R>(rng, sc, start, ntri, area);
        fill_light_vecs(pos, p.pos, &dir, &dist, &dist_sq);
        ndd = dot(dir, normal);
        if (ndd <= (R)0)
            return false;
        V4<R> ef = apply_emissive_texture<R>(sc, flux, tex_index, p);
        R cos_l = M<R>::fmax(dot(-dir, p.normal), (R)0);
        radiance = ef * ndd * cos_l / (C<R>::PI * dist_sq);
    }
    if (dot(radiance, radiance) < C<R>::EPS * C<R>::EPS)
        return false;
    out->radiance = radiance;
    out->dir = dir;
    out->dist = dist;
    out->n_dot_dir = ndd;
    return true;
}

template <class R> inline V4<R> shadow_transmittance(const Scene &sc, V4<R> origin, V4<R> dir, R dist) { // :302-333
    V4<R> trans = white4<R>();
    R t_min = C<R>::EPS, t_max = dist - C<R>::EPS;
    for (u32 depth = 0; depth < MAX_RAY_BOUNCES; depth++) {
        HitRecord<R> rec;
        if (!scene_intersect<R>(sc, origin, dir, t_min, t_max, &rec))
            break;
        const phx_material &mat = sc.materials[rec.mat_index];
        if ((R)mat.transmission < C<R>::EPS)
            return zero4<R>();
        V4<R> base = from<R>(mat.base_color);
        if (mat.diff_index != NO_TEXTURE) {
            SurfaceHit<R> sh = process_hit<R>(sc, rec, origin, dir);
            base *= srgb_to_linear(sample_texture_uv<R>(sc, rec.mat_index, mat.diff_index, sh.uvx, sh.uvy, 0));
        }
        if ((R)mat.att_dist > C<R>::EPS)
            trans *= beer_lambert<R>(from<R>(mat.att_color), (R)mat.att_dist, rec.t - t_min);
        trans *= base * (R)mat.transmission;
        if (dot(trans, trans) < C<R>::EPS)
            return zero4<R>();
        t_min = rec.t + C<R>::EPS;
    }
    return trans;
}

template <class R>
inline V4<R> direct_lighting_diffuse(Rng *rng, const Scene &sc, V4<R> pos, V4<R> normal, V4<R> base) { // :335-353
    LightFragment<R> f;
    if (!sample_light_fragment<R>(rng, sc, pos, normal, &f))
        return zero4<R>();
    V4<R> trans = shadow_transmittance<R>(sc, pos, f.dir, f.dist);
    return f.radiance * (base / C<R>::PI) * trans;
}

template <class R>
inline V4<R> direct_lighting_specular(Rng *rng, const Scene &sc, V4<R> pos, V4<R> normal, V4<R> view, V4<R> f0,
                                      R roughness) { // :355-390
    R ndv = dot(view, normal);
    if (ndv < C<R>::EPS)
        return zero4<R>();
    LightFragment<R> f;
    if (!sample_light_fragment<R>(rng, sc, pos, normal, &f))
        return zero4<R>();
    if (f.n_dot_dir < C<R>::EPS)
        return zero4<R>();
    R alpha = roughness * roughness;
    V4<R> h = normalize(f.dir + view);
    R ndh = M<R>::fmax(dot(normal, h), (R)0);
    R g = ggx_ndf(ndh, alpha);
    V4<R> fr = fresnel4(f0, view, h);
    R sm = smith_g1_ggx(f.n_dot_dir, alpha) * smith_g1_ggx(ndv, alpha);
    V4<R> spec = f.radiance * g * fr * sm / ((R)4 * f.n_dot_dir * ndv);
    if (dot(spec, spec) < C<R>::EPS * C<R>::EPS)
        return zero4<R>();
    V4<R> trans = shadow_transmittance<R>(sc, pos, f.dir, f.dist);
    return spec * trans;
}

template <class R> inline V4<R> sample_envmap(const Scene &sc, V4<R> dir) { // envmap.h:9-20
    R theta = M<R>::acos(clampr<R>(dir.z, (R)-1, (R)1));
    R phi = M<R>::atan2(dir.y, dir.x);
    R u = (phi + C<R>::PI) / ((R)2 * C<R>::PI);
    R v = clampr<R>((R)1 - theta / C<R>::PI, (R)0, (R)1);
    u = u - M<R>::floor(u);
    u32 px = std::min((u32)(u * (R)sc.env_w), sc.env_w - 1);
    u32 py = std::min((u32)(v * (R)sc.env_h), sc.env_h - 1);
    u32 idx = 3 * (py * sc.env_w + px);
    return mk<R>((R)sc.envmap[idx], (R)sc.envmap[idx + 1], (R)sc.envmap[idx + 2], (R)0);
}

template <class R>
inline void make_ray(const phx_camera_params &cam, u32 px, u32 py, u32 width, u32 height, Rng *rng, V4<R> *origin,
                     V4<R> *dir) { // camera.h:28-47
    R u = random_float<R>(rng) - (R)0.5;
    R v = random_float<R>(rng) - (R)0.5;
    R s = ((R)px + (R)0.5 + u) / (R)width;
    R t = (R)1 - ((R)py + (R)0.5 + v) / (R)height;
    V4<R> disk = zero4<R>();
    if ((R)cam.defocus_angle > (R)0) {
        R r1 = M<R>::sqrt(random_float<R>(rng));
        R r2 = ((R)2 * C<R>::PI) * random_float<R>(rng);
        R c = M<R>::cos(r2), sn = M<R>::sin(r2);
        disk = r1 * (c * from<R>(cam.defocus_disk_u) + sn * from<R>(cam.defocus_disk_v));
    }
    *origin = from<R>(cam.position) + disk;
    V4<R> d = from<R>(cam.lower_left_corner) + s * from<R>(cam.horizontal) + t * from<R>(cam.vertical) - *origin;
    *dir = normalize(d);
}

// ---- trace_rays.cl:14-169 ----------------------------------------------------------------------
template <class R> struct HitPoint {
    V4<R> pos, normal, throughput, base_color, direct, emission;
};

template <class R>
inline HitPoint<R> trace_pixel(const Scene &sc, u32 width, u32 height, u32 seed, u32 direct_samples, u32 tid) {
    u32 px = tid % width;
    u32 py = tid / width;
    Rng rng = pcg_seed(seed + tid);
    V4<R> origin, dir;
    make_ray<R>(sc.camera, px, py, width, height, &rng, &origin, &dir);
    V4<R> position = zero4<R>(), normal = zero4<R>(), throughput = white4<R>(), base_color = zero4<R>(),
          direct = zero4<R>(), emission = zero4<R>();
    IorStack<R> ior;
    init_ior_stack<R>(&ior, (R)AIR_IOR);
    for (i32 depth = 0; depth < (i32)MAX_RAY_BOUNCES; depth++) {
        HitRecord<R> rec;
        bool hit = scene_intersect<R>(sc, origin, dir, C<R>::EPS, C<R>::INF, &rec);
        if (!hit) {
            if (sc.has_envmap)
                emission += throughput * sample_envmap<R>(sc, dir);
            break;
        }
        SurfaceHit<R> sh = process_hit<R>(sc, rec, origin, dir);
        const phx_material &mat = sc.materials[sh.mat_index];
        V4<R> vol = white4<R>();
        R cur = current_ior(&ior);
        if (cur != (R)AIR_IOR && (R)mat.thickness > C<R>::EPS && (R)mat.att_dist > C<R>::EPS) {
            vol = beer_lambert<R>(from<R>(mat.att_color), (R)mat.att_dist, sh.t);
            throughput *= vol;
        }
        R bw = (R)1 - rec.u - rec.v;
        const phx_triangle &tr = sc.tris[sh.tri_index];
        V4<R> traw = bw * from<R>(tr.t0) + rec.u * from<R>(tr.t1) + rec.v * from<R>(tr.t2);
        V4<R> braw = (length(traw) > C<R>::EPS) ? cross(sh.normal, traw) : zero4<R>();
        V4<R> tangent, bitangent;
        if (length(braw) > C<R>::EPS) {
            bitangent = normalize(braw);
            tangent = cross(bitangent, sh.normal);
        } else {
            make_tbn(sh.normal, &tangent, &bitangent);
        }
        ShadingContext<R> ctx = evaluate_material<R>(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        emission += throughput * ctx.emissive;
        V4<R> view = -dir;
        BsdfSample<R> bs = sample_bsdf<R>(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE) {
            V4<R> sum = zero4<R>();
            for (u32 d = 0; d < direct_samples; d++)
                sum += direct_lighting_diffuse<R>(&rng, sc, sh.position, ctx.shading_normal, ctx.base_color);
            emission = mk<R>(emission.x, emission.y, emission.z, (R)1);
            position = sh.position;
            normal = sh.normal;
            base_color = ctx.base_color;
            direct = throughput * ctx.occlusion * (sum / (R)direct_samples);
            break;
        }
        if (bs.event == BSDF_METALLIC) {
            V4<R> sum = zero4<R>();
            for (u32 d = 0; d < direct_samples; d++)
                sum += direct_lighting_specular<R>(&rng, sc, sh.position, ctx.shading_normal, view, ctx.base_color,
                                                   ctx.roughness);
            emission += throughput * (sum / (R)direct_samples);
        }
        if (bs.event == BSDF_FRESNEL) {
            R ratio = (cur - ctx.ior) / (cur + ctx.ior);
            R r0 = ratio * ratio;
            V4<R> f0 = mk<R>(r0, r0, r0, (R)0);
            V4<R> sum = zero4<R>();
            for (u32 d = 0; d < direct_samples; d++)
                sum += direct_lighting_specular<R>(&rng, sc, sh.position, ctx.shading_normal, view, f0, ctx.roughness);
            emission += throughput * (sum / (R)direct_samples);
        }
        throughput *= bs.throughput;
        if ((u32)depth >= RR_MIN_RAY_DEPTH) {
            R q = M<R>::fmax(throughput.x, M<R>::fmax(throughput.y, throughput.z));
            q = clampr<R>(q, (R)RR_MIN_Q, (R)RR_MAX_Q);
            if (random_float<R>(&rng) > q)
                break;
            throughput *= (R)1 / q;
        }
        V4<R> side = (dot(bs.dir, sh.normal) > (R)0) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * C<R>::EPS + side * C<R>::EPS;
        dir = bs.dir;
    }
    HitPoint<R> hp;
    hp.emission = emission;
    hp.pos = position;
    hp.normal = normal;
    hp.throughput = throughput;
    hp.base_color = base_color;
    hp.direct = direct;
    return hp;
}

// ---- emit_photons.cl:12-114 --------------------------------------------------------------------
template <class R> struct StoredPhoton {
    V4<R> pos;
    u32 power, dir;
};

// Traces photon path `tid` and appends its stored photons (canonical: bounce order) to out.
template <class R>
inline u32 emit_photon(const Scene &sc, u32 tid, u32 max_bounces, u32 seed, StoredPhoton<R> *out) {
    u32 n_out = 0;
    Rng rng = pcg_seed(seed + tid);
    V4<R> origin, dir, power;
    sample_light<R>(&rng, sc, &origin, &dir, &power);
    IorStack<R> ior;
    init_ior_stack<R>(&ior, (R)AIR_IOR);
    V4<R> throughput = mk<R>(1, 1, 1, 0);
    for (u32 depth = 0; depth < max_bounces; depth++) {
        HitRecord<R> rec;
        bool hit = scene_intersect<R>(sc, origin, dir, C<R>::EPS, C<R>::INF, &rec);
        if (!hit)
            return n_out;
        SurfaceHit<R> sh = process_hit<R>(sc, rec, origin, dir);
        const phx_material &mat = sc.materials[sh.mat_index];
        V4<R> vol = white4<R>();
        R cur = current_ior(&ior);
        if (cur != (R)AIR_IOR && (R)mat.thickness > C<R>::EPS && (R)mat.att_dist > C<R>::EPS) {
            vol = beer_lambert<R>(from<R>(mat.att_color), (R)mat.att_dist, sh.t);
            power *= vol;
            throughput *= vol;
        }
        R bw = (R)1 - rec.u - rec.v;
        const phx_triangle &tr = sc.tris[sh.tri_index];
        V4<R> traw = bw * from<R>(tr.t0) + rec.u * from<R>(tr.t1) + rec.v * from<R>(tr.t2);
        V4<R> braw = (length(traw) > C<R>::EPS) ? cross(sh.normal, traw) : zero4<R>();
        V4<R> tangent, bitangent;
        if (length(braw) > C<R>::EPS) {
            bitangent = normalize(braw);
            tangent = cross(bitangent, sh.normal);
        } else {
            make_tbn(sh.normal, &tangent, &bitangent);
        }
        ShadingContext<R> ctx = evaluate_material<R>(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        if (depth >= RR_MIN_PHOTON_DEPTH) {
            R q = M<R>::fmax(throughput.x, M<R>::fmax(throughput.y, throughput.z));
            q = clampr<R>(q, (R)RR_MIN_Q, (R)RR_MAX_Q);
            if (random_float<R>(&rng) > q)
                return n_out;
            R inv_q = (R)1 / q;
            throughput *= inv_q;
            power *= inv_q;
        }
        V4<R> view = -dir;
        BsdfSample<R> bs = sample_bsdf<R>(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE && dot(dir, sh.normal) < (R)0) {
            // the reference's buffer (photons x max_bounces, renderer.cpp:40) never overflows: at most
            // one store per bounce
            out[n_out].pos = sh.position;
            out[n_out].power = encode_rgbe<R>(power);
            out[n_out].dir = encode_oct<R>(dir);
            n_out++;
        }
        power *= bs.throughput;
        throughput *= bs.throughput;
        V4<R> side = (dot(bs.dir, sh.normal) > (R)0) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * C<R>::EPS + side * C<R>::EPS;
        dir = bs.dir;
    }
    return n_out;
}

// ---- photon_hash.h:21-103 ----------------------------------------------------------------------
template <class R> inline u32 get_hash(V4<R> pos, const phx_photon_hash_data &d) { // photon_hash.h:21-37
    u32 g = d.grid_res;
    R fx = (pos.x - (R)d.origin.x) / (R)d.cell_sizes.x;
    R fy = (pos.y - (R)d.origin.y) / (R)d.cell_sizes.y;
    R fz = (pos.z - (R)d.origin.z) / (R)d.cell_sizes.z;
    if (fx < (R)0 || fy < (R)0 || fz < (R)0 || fx >= (R)g || fy >= (R)g || fz >= (R)g)
        return 0;
    u32 x = (u32)fx, y = (u32)fy, z = (u32)fz;
    return g * g * x + g * y + z + 1;
}

template <class R>
inline void gather_photon_flux(V4<R> pos, V4<R> n, const phx_photon_hash_data &d, const u32 *cell_start,
                               const u32 *cell_end, const V4<R> *ph_pos, const u32 *ph_power, const u32 *ph_dir,
                               R r_sq, V4<R> *out_flux, R *out_found) { // photon_hash.h:56-103
    *out_flux = zero4<R>();
    *out_found = (R)0;
    for (u32 i = 0; i < 27; i++) {
        i32 cx = (i32)(i % 3) - 1;
        i32 cy = (i32)((i / 3) % 3) - 1;
        i32 cz = (i32)((i / 9) % 3) - 1;
        V4<R> p2 = pos;
        p2.x += (R)cx * (R)d.cell_sizes.x;
        p2.y += (R)cy * (R)d.cell_sizes.y;
        p2.z += (R)cz * (R)d.cell_sizes.z;
        u32 h = get_hash<R>(p2, d);
        if (h == 0)
            continue;
        u32 start = cell_start[h], end = cell_end[h];
        if (start == end)
            continue;
        for (u32 k = start; k < end; k++) {
            V4<R> dd = pos - ph_pos[k];
            R dsq = dot(dd, dd);
            if (dsq >= r_sq)
                continue;
            V4<R> pd = decode_oct<R>(ph_dir[k]);
            if (dot(pd, n) > (R)0)
                continue;
            R w = (R)GAUSS_ALPHA * ((R)1 - ((R)1 - M<R>::exp((R)(-GAUSS_BETA) * dsq / ((R)2 * r_sq))) / (R)GAUSS_DENOM);
            *out_flux += w * decode_rgbe<R>(ph_power[k]);
            *out_found += w;
        }
    }
}

// gather_flux.cl:5-78 for one pixel; flux/weight/radiance updated in place
template <class R>
inline void gather_pixel(const HitPoint<R> &hp, const phx_photon_hash_data &d, const u32 *cell_start,
                         const u32 *cell_end, const V4<R> *ph_pos, const u32 *ph_power, const u32 *ph_dir, R alpha,
                         V4<R> *flux, R *weight, V4<R> *radiance) {
    V4<R> ge = hp.emission;
    V4<R> rso = *radiance;
    V4<R> r = mk<R>(ge.x, ge.y, ge.z, (R)0);
    if (ge.w == (R)0) {
        *radiance = rso + r;
        return;
    }
    V4<R> direct = hp.direct;
    r.x += direct.x;
    r.y += direct.y;
    r.z += direct.z;
    *radiance = rso + r;
    V4<R> fso = *flux;
    R wso = *weight;
    R r_sq = fso.w;
    if (r_sq < C<R>::EPS) {
        R hx = (R)d.cell_sizes.x * (R)0.5f;
        R hy = (R)d.cell_sizes.y * (R)0.5f;
        R hz = (R)d.cell_sizes.z * (R)0.5f;
        r_sq = hx * hx + hy * hy + hz * hz;
    }
    V4<R> nf;
    R found;
    gather_photon_flux<R>(hp.pos, hp.normal, d, cell_start, cell_end, ph_pos, ph_power, ph_dir, r_sq, &nf, &found);
    if (found > (R)0) {
        R nw = wso + alpha * found;
        R ratio = nw / (wso + found);
        R nr = r_sq * ratio;
        V4<R> albedo = hp.base_color;
        V4<R> contribution = hp.throughput * (albedo / C<R>::PI) * nf;
        V4<R> temp = (fso + contribution) * ratio;
        *flux = mk<R>(temp.x, temp.y, temp.z, nr);
        *weight = nw;
    }
}

// ---- host pieces -------------------------------------------------------------------------------
// bounding_box.h:48-61 + bvh.cpp:18-84 (the reference's median-split builder and flattening)
struct BBox {
    float min[4], max[4];
};
inline bool check_inf(float v) { return v >= INF_F || v <= -INF_F; }

inline bool tri_bbox(const phx_triangle &t, BBox *out) {
    BBox b;
    b.min[0] = b.min[1] = b.min[2] = INF_F;
    b.max[0] = b.max[1] = b.max[2] = -INF_F;
    b.min[3] = b.max[3] = 0.0f;
    const phx_f4 *vs[3] = {&t.v0, &t.v1, &t.v2};
    for (auto *v : vs) {
        b.min[0] = std::min(b.min[0], v->x);
        b.min[1] = std::min(b.min[1], v->y);
        b.min[2] = std::min(b.min[2], v->z);
        b.max[0] = std::max(b.max[0], v->x);
        b.max[1] = std::max(b.max[1], v->y);
        b.max[2] = std::max(b.max[2], v->z);
    }
    for (int i = 0; i < 3; i++)
        if (check_inf(b.min[i]) || check_inf(b.max[i]))
            return false;
    for (int i = 0; i < 3; i++) {
        b.min[i] -= BBOX_EPS;
        b.max[i] += BBOX_EPS;
    }
    if (b.min[0] == b.max[0] || b.min[1] == b.max[1] || b.min[2] == b.max[2])
        return false;
    *out = b;
    return true;
}

inline BBox merge_bbox(const BBox &a, const BBox &b) {
    BBox r;
    for (int i = 0; i < 3; i++) {
        r.min[i] = std::min(a.min[i], b.min[i]);
        r.max[i] = std::max(a.max[i], b.max[i]);
    }
    r.min[3] = a.min[3];
    r.max[3] = a.max[3];
    return r;
}

inline u32 longest_axis(const BBox &b) { // bounding_box.h:63-78
    float xs = b.max[0] - b.min[0], ys = b.max[1] - b.min[1], zs = b.max[2] - b.min[2];
    if (xs > ys) {
        if (xs > zs)
            return 0;
    } else {
        if (ys > zs)
            return 1;
    }
    return 2;
}

struct TmpNode {
    BBox bbox;
    i32 tri;
    u32 left, right;
};

inline u32 build_tmp(const std::vector<BBox> &bbs, std::vector<u32> &idx, u32 start, u32 end,
                     std::vector<TmpNode> &tmp) { // bvh.cpp:18-53
    u32 id = (u32)tmp.size();
    tmp.push_back({});
    if (end == start + 1) {
        tmp[id].tri = (i32)idx[start];
        tmp[id].bbox = bbs[idx[start]];
        tmp[id].left = 0;
        tmp[id].right = 0;
        return id;
    }
    BBox bb = bbs[idx[start]];
    for (u32 i = start + 1; i < end; i++)
        bb = merge_bbox(bb, bbs[idx[i]]);
    tmp[id].bbox = bb;
    tmp[id].tri = -1;
    u32 axis = longest_axis(bb);
    std::sort(idx.begin() + start, idx.begin() + end,
              [&](u32 i, u32 j) { return bbs[i].min[axis] < bbs[j].min[axis]; });
    u32 mid = start + (end - start) / 2;
    u32 l = build_tmp(bbs, idx, start, mid, tmp);
    u32 r = build_tmp(bbs, idx, mid, end, tmp);
    tmp[id].left = l;
    tmp[id].right = r;
    return id;
}

inline void flatten(const std::vector<TmpNode> &tmp, u32 ti, std::vector<phx_bvh_node> &out) { // bvh.cpp:57-72
    u32 id = (u32)out.size();
    out.push_back({});
    const BBox &b = tmp[ti].bbox;
    out[id].min = {b.min[0], b.min[1], b.min[2], as_float((u32)tmp[ti].tri)};
    out[id].max = {b.max[0], b.max[1], b.max[2], as_float(tmp[ti].right)};
    if (tmp[ti].tri == -1) {
        flatten(tmp, tmp[ti].left, out);
        out[id].max.w = as_float((u32)out.size());
        flatten(tmp, tmp[ti].right, out);
    }
}

inline bool build_bvh(const phx_triangle *tris, u32 n, std::vector<phx_bvh_node> &out) { // bvh.cpp:74-84
    std::vector<BBox> bbs(n);
    for (u32 i = 0; i < n; i++)
        if (!tri_bbox(tris[i], &bbs[i]))
            return false;
    std::vector<u32> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::vector<TmpNode> tmp;
    tmp.reserve(2 * (size_t)n);
    build_tmp(bbs, idx, 0, n, tmp);
    out.clear();
    out.reserve(2 * (size_t)n - 1);
    flatten(tmp, 0, out);
    return true;
}

// photon_hash.h:41-50
inline phx_photon_hash_data hash_info(const phx_bvh_node &root, u32 g) {
    phx_photon_hash_data d{};
    d.grid_res = g;
    d.origin = {root.min.x, root.min.y, root.min.z, 0.0f};
    d.cell_sizes.x = std::max((root.max.x - root.min.x) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.y = std::max((root.max.y - root.min.y) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.z = std::max((root.max.z - root.min.z) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.w = 0.0f;
    return d;
}

// shading.cpp:45-58 scene centre and bounding radius from the BVH root box
inline void scene_sphere(const phx_bvh_node &root, phx_f4 *center, float *radius) {
    float cx = 0.5f * (root.min.x + root.max.x);
    float cy = 0.5f * (root.min.y + root.max.y);
    float cz = 0.5f * (root.min.z + root.max.z);
    *center = {cx, cy, cz, 0.0f};
    const float xs[2] = {root.min.x, root.max.x}, ys[2] = {root.min.y, root.max.y}, zs[2] = {root.min.z, root.max.z};
    float r = 0.0f;
    // glm::length(corner - center) for the eight corners, order irrelevant for max
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                float dx = xs[i] - cx, dy = ys[j] - cy, dz = zs[k] - cz;
                r = std::max(r, std::sqrt(dx * dx + dy * dy + dz * dz));
            }
    *radius = r;
}

} // namespace orc
