// ref_kernels.cpp — TEST INFRASTRUCTURE ONLY.  Runs the reference's own SPPM kernels on the CPU.
//
// oracle/build_ref_sppm.py preprocesses the reference's kernels/*.cl (with its include/ tree, as
// OpenCL C: __OPENCL_C_VERSION__ defined) into one translation unit, rewrites the two pieces of
// OpenCL C syntax that C++ cannot parse — vector literals `(float4)(...)` / `(float2)(...)` become
// calls of float4_ctor / float2_ctor, and the rvalue swizzle `.yx` becomes `.yx_()` — and writes
// the result to oracle/_ref/sppm_kernels.inc (git-ignored).  This file supplies what an OpenCL
// runtime would: the vector types with OpenCL's component-wise operators, the builtins, the
// work-item ids and the work-group barrier, and it launches each kernel over its NDRange.
//
// The builtins follow the OpenCL C specification where it is exact, and take the same fixed
// choices as the CPU restatement (oracle/phx_oracle.hpp) and the CUDA library where the
// specification leaves them to the implementation:
//   * IEEE-754 binary32 with no contraction (built with -ffp-contract=off, SSE arithmetic);
//   * dot(a, b) = ((a.x*b.x + a.y*b.y) + a.z*b.z) + a.w*b.w; length(v) = sqrt(dot(v, v));
//     normalize(v) = v / length(v), a zero vector returned unchanged; rsqrt(x) = 1 / sqrt(x);
//     cross(a, b) has w = 0; mix(a, b, t) = a + (b - a) * t; clamp(x, lo, hi) = fmin(fmax(x, lo), hi);
//     min(x, y) = y < x ? y : x;
//   * sin, cos, exp, native_exp, log, pow, acos and atan2 are include/phx_math.h's
//     implementations (OpenCL only bounds their error);
//   * atomic_inc is a plain increment: the kernels that use it (emit_photons, hash_photons,
//     scatter_photons) are launched with their work items in index order, one at a time, which
//     is one of the orders an OpenCL device may produce and the canonical order the GPU library
//     reproduces.
// Nothing here is product code; the CUDA library never links it.
#include <algorithm>
#include <barrier>
#include <cstdint>
#include <cstring>
#include <functional>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../include/phx.h"
#include "../include/phx_math.h"

namespace refk {

// ---- OpenCL C scalar and vector types -----------------------------------------------------------
typedef unsigned char uchar;
typedef unsigned int uint;
typedef unsigned long ulong;

struct float2 {
    union {
        struct {
            float x, y;
        };
        struct {
            float r, g;
        };
    };
    float2 yx_() const;
} __attribute__((aligned(8)));

struct float3s { // the lvalue view .xyz of a float4
    float x, y, z;
};

struct float4 {
    union {
        struct {
            float x, y, z, w;
        };
        struct {
            float r, g, b, a;
        };
        float2 xy;
        float3s xyz;
    };
} __attribute__((aligned(16)));

static_assert(sizeof(float2) == 8 && sizeof(float4) == 16, "OpenCL vector sizes");

inline float2 float2_ctor(float a, float b) {
    float2 v;
    v.x = a;
    v.y = b;
    return v;
}
inline float2 float2_ctor(float s) { return float2_ctor(s, s); }
inline float2 float2::yx_() const { return float2_ctor(y, x); }
inline float4 float4_ctor(float a, float b, float c, float d) {
    float4 v;
    v.x = a;
    v.y = b;
    v.z = c;
    v.w = d;
    return v;
}
inline float4 float4_ctor(float s) { return float4_ctor(s, s, s, s); }
inline float4 float4_ctor(float3s v, float d) { return float4_ctor(v.x, v.y, v.z, d); }
inline float4 float4_ctor(float2 v, float c, float d) { return float4_ctor(v.x, v.y, c, d); }

#define PHX_V4_BINOP(op)                                                                                               \
    inline float4 operator op(float4 a, float4 b) { return float4_ctor(a.x op b.x, a.y op b.y, a.z op b.z, a.w op b.w); } \
    inline float4 operator op(float4 a, float s) { return float4_ctor(a.x op s, a.y op s, a.z op s, a.w op s); }         \
    inline float4 operator op(float s, float4 a) { return float4_ctor(s op a.x, s op a.y, s op a.z, s op a.w); }         \
    inline float2 operator op(float2 a, float2 b) { return float2_ctor(a.x op b.x, a.y op b.y); }                       \
    inline float2 operator op(float2 a, float s) { return float2_ctor(a.x op s, a.y op s); }                            \
    inline float2 operator op(float s, float2 a) { return float2_ctor(s op a.x, s op a.y); }
PHX_V4_BINOP(+)
PHX_V4_BINOP(-)
PHX_V4_BINOP(*)
PHX_V4_BINOP(/)
#undef PHX_V4_BINOP
inline float4 operator-(float4 a) { return float4_ctor(-a.x, -a.y, -a.z, -a.w); }
inline float2 operator-(float2 a) { return float2_ctor(-a.x, -a.y); }
#define PHX_V4_ASSIGN(op, bop)                                                                                         \
    inline float4 &operator op(float4 &a, float4 b) { return a = a bop b; }                                            \
    inline float4 &operator op(float4 &a, float s) { return a = a bop s; }                                             \
    inline float2 &operator op(float2 &a, float2 b) { return a = a bop b; }                                            \
    inline float2 &operator op(float2 &a, float s) { return a = a bop s; }
PHX_V4_ASSIGN(+=, +)
PHX_V4_ASSIGN(-=, -)
PHX_V4_ASSIGN(*=, *)
PHX_V4_ASSIGN(/=, /)
#undef PHX_V4_ASSIGN

// ---- builtins ----------------------------------------------------------------------------------
inline float sqrt(float x) { return __builtin_sqrtf(x); }
inline float fabs(float x) { return __builtin_fabsf(x); }
inline float2 fabs(float2 v) { return float2_ctor(fabs(v.x), fabs(v.y)); }
inline float floor(float x) { return __builtin_floorf(x); }
inline float ceil(float x) { return __builtin_ceilf(x); }
inline float fmax(float a, float b) { return __builtin_fmaxf(a, b); }
inline float fmin(float a, float b) { return __builtin_fminf(a, b); }
inline float min(float x, float y) { return y < x ? y : x; }
inline int min(int x, int y) { return y < x ? y : x; }
inline uint min(uint x, uint y) { return y < x ? y : x; }
inline float clamp(float x, float lo, float hi) { return fmin(fmax(x, lo), hi); }
inline float frexp(float x, int *e) { return __builtin_frexpf(x, e); }
inline float ldexp(float x, int e) { return __builtin_ldexpf(x, e); }
inline float sin(float x) { return pm_sinf(x); }
inline float cos(float x) { return pm_cosf(x); }
inline float exp(float x) { return pm_expf(x); }
inline float native_exp(float x) { return pm_expf(x); }
inline float log(float x) { return pm_logf(x); }
inline float pow(float x, float y) { return pm_powf(x, y); }
inline float acos(float x) { return pm_acosf(x); }
inline float atan2(float y, float x) { return pm_atan2f(y, x); }
inline float rsqrt(float x) { return 1.0f / sqrt(x); }
inline float dot(float4 a, float4 b) { return ((a.x * b.x + a.y * b.y) + a.z * b.z) + a.w * b.w; }
inline float4 cross(float4 a, float4 b) {
    return float4_ctor(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x, 0.0f);
}
inline float length(float4 v) { return sqrt(dot(v, v)); }
inline float4 normalize(float4 v) {
    float l = sqrt(dot(v, v));
    if (l == 0.0f)
        return v;
    return v / l;
}
inline float4 mix(float4 a, float4 b, float t) { return a + (b - a) * t; }
inline uint as_uint(float f) {
    uint u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float as_float(uint u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint atomic_inc(uint *p) { return (*p)++; }

// ---- work-item ids and the work-group barrier ----------------------------------------------------
thread_local uint t_global_id = 0, t_local_id = 0, t_group_id = 0;
thread_local std::barrier<> *t_group_barrier = nullptr;
inline uint get_global_id(uint) { return t_global_id; }
inline uint get_local_id(uint) { return t_local_id; }
inline uint get_group_id(uint) { return t_group_id; }
constexpr int CLK_LOCAL_MEM_FENCE = 1;
inline void barrier(int) {
    if (t_group_barrier)
        t_group_barrier->arrive_and_wait();
}

// ---- the reference's kernels and device headers (generated from its sources) ---------------------
#include "sppm_kernels.inc"

static_assert(sizeof(Material) == sizeof(phx_material) && sizeof(Light) == sizeof(phx_light) &&
                  sizeof(CameraParams) == sizeof(phx_camera_params) && sizeof(BvhNode) == sizeof(phx_bvh_node) &&
                  sizeof(PhotonHashData) == sizeof(phx_photon_hash_data) &&
                  sizeof(UvTransformBlock) == sizeof(phx_uv_transform_block) &&
                  sizeof(TextureMeta) == sizeof(phx_texture_meta) && sizeof(TriangleUvs) == 32,
              "reference layouts");

// ---- NDRange launches ----------------------------------------------------------------------------
// Work items in [0, n): independent items split over host threads (each item sees its own id).
void launch_parallel(uint n, int threads, const std::function<void()> &item) {
    auto run = [&](uint b, uint e) {
        for (uint i = b; i < e; i++) {
            t_global_id = i;
            item();
        }
    };
    if (threads <= 1 || n < 256) {
        run(0, n);
        return;
    }
    std::vector<std::thread> pool;
    const uint chunk = (n + (uint)threads - 1) / (uint)threads;
    for (int t = 0; t < threads; t++) {
        uint b = std::min(n, (uint)t * chunk), e = std::min(n, b + chunk);
        pool.emplace_back(run, b, e);
    }
    for (auto &th : pool)
        th.join();
}

// Work items in index order, one at a time (kernels with atomic_inc: canonical order).
void launch_sequential(uint n, const std::function<void()> &item) {
    for (uint i = 0; i < n; i++) {
        t_global_id = i;
        item();
    }
}

// Work groups of `wg` items that synchronise at barrier(): one host thread per work item, the
// groups run one after another (so the kernel's __local arrays hold one group's data at a time).
void launch_groups(uint groups, uint wg, const std::function<void()> &item) {
    std::barrier<> bar((std::ptrdiff_t)wg);
    std::vector<std::thread> pool;
    for (uint l = 0; l < wg; l++)
        pool.emplace_back([&, l]() {
            t_group_barrier = &bar;
            for (uint g = 0; g < groups; g++) {
                t_local_id = l;
                t_group_id = g;
                t_global_id = g * wg + l;
                item();
                bar.arrive_and_wait();
            }
            t_group_barrier = nullptr;
        });
    for (auto &th : pool)
        th.join();
}

// The scene in the reference's device layout (src/buffers/geometry.cpp:5-55,
// src/buffers/shading.cpp:9-75): structure-of-arrays triangles, the rest byte-compatible.
struct RefScene {
    std::vector<TriangleVertices> tv, etv;
    std::vector<TriangleNormals> tn, etn;
    std::vector<TriangleTangents> tt;
    std::vector<TriangleUvs> tuv, etuv;
    std::vector<uint> tmat, etmat;
    std::vector<BvhNode> bvh;
    const Material *materials = nullptr;
    const UvTransformBlock *uvs = nullptr;
    const Light *lights = nullptr;
    uint n_lights = 0;
    std::vector<float> lum;
    float total_lum = 0.0f;
    std::vector<TextureMeta> tex_meta;
    std::vector<uchar> atlas;
    std::vector<float> envmap;
    uint env_w = 0, env_h = 0, has_env = 0;
    CameraParams camera{};
    float4 center{};
    float radius = 0.0f;
};

template <class T> T cvt(const void *p) {
    T t;
    std::memcpy(&t, p, sizeof(T));
    return t;
}

void split_triangles(const phx_triangle *in, uint n, std::vector<TriangleVertices> &tv,
                     std::vector<TriangleNormals> *tn, std::vector<TriangleTangents> *tt,
                     std::vector<TriangleUvs> &tuv, std::vector<uint> &tmat) {
    tv.resize(std::max(n, 1u));
    tuv.resize(std::max(n, 1u));
    tmat.resize(std::max(n, 1u));
    if (tn)
        tn->resize(std::max(n, 1u));
    if (tt)
        tt->resize(std::max(n, 1u));
    for (uint i = 0; i < n; i++) {
        const phx_triangle &t = in[i];
        tv[i].v0 = cvt<float4>(&t.v0);
        tv[i].v1 = cvt<float4>(&t.v1);
        tv[i].v2 = cvt<float4>(&t.v2);
        if (tn) {
            (*tn)[i].n0 = cvt<float4>(&t.n0);
            (*tn)[i].n1 = cvt<float4>(&t.n1);
            (*tn)[i].n2 = cvt<float4>(&t.n2);
        }
        if (tt) {
            (*tt)[i].t0 = cvt<float4>(&t.t0);
            (*tt)[i].t1 = cvt<float4>(&t.t1);
            (*tt)[i].t2 = cvt<float4>(&t.t2);
        }
        std::memset(&tuv[i], 0, sizeof(TriangleUvs));
        tuv[i].uv0 = cvt<float2>(&t.uv0);
        tuv[i].uv1 = cvt<float2>(&t.uv1);
        tuv[i].uv2 = cvt<float2>(&t.uv2);
        tmat[i] = t.mat_index;
    }
}

} // namespace refk

using namespace refk;

extern "C" {

#define REF_API __attribute__((visibility("default")))

// Scene set-up: `bvh` is the reference tree (2n-1 nodes, from ref_bvh_build), center/radius the
// scene sphere (ref_scene_sphere); lum_pref_sum and the camera come with the scene.
REF_API void *ref_scene_create(const phx_scene *s, const phx_bvh_node *bvh, const float *center, float radius) {
    auto *r = new RefScene();
    split_triangles(s->triangles, s->n_triangles, r->tv, &r->tn, &r->tt, r->tuv, r->tmat);
    split_triangles(s->emissive_triangles, s->n_emissive_triangles, r->etv, &r->etn, nullptr, r->etuv, r->etmat);
    r->bvh.resize(2 * (size_t)s->n_triangles - 1);
    std::memcpy(r->bvh.data(), bvh, r->bvh.size() * sizeof(BvhNode));
    r->materials = reinterpret_cast<const Material *>(s->materials);
    r->uvs = reinterpret_cast<const UvTransformBlock *>(s->uv_transforms);
    r->lights = reinterpret_cast<const Light *>(s->lights);
    r->n_lights = s->n_lights;
    r->lum.assign(s->lum_pref_sum, s->lum_pref_sum + s->n_lights);
    r->total_lum = r->lum.empty() ? 0.0f : r->lum.back(); // shading.cpp:22-23
    if (r->lum.empty())
        r->lum.push_back(0.0f);
    for (uint i = 0; i < s->n_textures; i++)
        r->tex_meta.push_back(cvt<TextureMeta>(&s->tex_meta[i]));
    if (r->tex_meta.empty()) // shading.cpp:37-40
        r->tex_meta.push_back(TextureMeta{});
    r->atlas.assign(s->tex_atlas, s->tex_atlas + s->tex_atlas_bytes);
    if (r->atlas.empty())
        r->atlas.push_back(0);
    if (s->envmap && s->envmap_width && s->envmap_height) {
        r->envmap.assign(s->envmap, s->envmap + 3 * (size_t)s->envmap_width * s->envmap_height);
        r->env_w = s->envmap_width;
        r->env_h = s->envmap_height;
        r->has_env = 1;
    } else {
        r->envmap.push_back(0.0f);
    }
    r->camera = cvt<CameraParams>(&s->camera);
    r->center = float4_ctor(center[0], center[1], center[2], 0.0f);
    r->radius = radius;
    return r;
}

REF_API void ref_scene_destroy(void *h) { delete reinterpret_cast<RefScene *>(h); }

// kernels/trace_rays.cl over width*height work items; out: 6 float4 per pixel (pos, normal,
// throughput, base colour, direct, emission), pixel-major.
REF_API int ref_trace(void *h, uint w, uint hgt, uint seed, uint ds, float *out, int threads) {
    auto *r = reinterpret_cast<RefScene *>(h);
    const uint n = w * hgt;
    std::vector<float4> hp[6];
    for (auto &v : hp)
        v.resize(n);
    launch_parallel(n, threads, [&]() {
        trace_rays(r->camera, w, hgt, seed, ds, r->tv.data(), r->tn.data(), r->tt.data(), r->tuv.data(), r->bvh.data(),
                   r->tmat.data(), (uint)r->tv.size(), r->materials, r->uvs, r->tex_meta.data(), r->atlas.data(),
                   r->lights, r->n_lights, r->lum.data(), r->total_lum, r->center, r->radius, r->etv.data(),
                   r->etn.data(), r->etuv.data(), r->etmat.data(), r->envmap.data(), r->env_w, r->env_h, r->has_env,
                   hp[0].data(), hp[1].data(), hp[2].data(), hp[3].data(), hp[4].data(), hp[5].data());
    });
    for (uint i = 0; i < n; i++)
        for (int k = 0; k < 6; k++)
            std::memcpy(out + 4 * (6 * (size_t)i + k), &hp[k][i], 16);
    return 0;
}

// Renderer::emit_photons (renderer.cpp:97-120): batches of at most `batch` work items of
// kernels/emit_photons.cl, work items in index order.  Writes *n_out = min(count, capacity).
REF_API int ref_emit(void *h, uint photons, uint batch, uint max_bounces, uint seed, uint capacity, float *pos4,
                     uint *power, uint *dir, uint *n_out) {
    auto *r = reinterpret_cast<RefScene *>(h);
    uint count = 0;
    std::vector<float4> p(capacity);
    const uint per_batch = std::min(photons, batch);
    for (uint off = 0; off < photons; off += per_batch) {
        uint to_emit = std::min(per_batch, photons - off);
        launch_sequential(to_emit, [&]() {
            emit_photons(r->lights, r->n_lights, capacity, off, to_emit, max_bounces, seed, r->bvh.data(),
                         r->tv.data(), r->tn.data(), r->tt.data(), r->tuv.data(), r->tmat.data(), (uint)r->tv.size(),
                         r->etv.data(), r->etn.data(), r->etuv.data(), r->etmat.data(), r->materials, r->uvs,
                         r->tex_meta.data(), r->atlas.data(), r->lum.data(), r->total_lum, r->center, r->radius,
                         p.data(), power, dir, &count);
        });
    }
    *n_out = std::min(count, capacity);
    std::memcpy(pos4, p.data(), (size_t)*n_out * 16);
    return 0;
}

// Renderer::hash_and_sort_photons (renderer.cpp:122-151): zeroed counts, hash_photons, the three
// scan kernels, the start->end copy and scatter_photons (work items in index order).
REF_API int ref_hash_sort(const float *pos4, const uint *power, const uint *dir, uint n, const phx_photon_hash_data *hd,
                          uint buckets, uint *keys, uint *counts, uint *starts, uint *ends, float *out_pos4,
                          uint *out_power, uint *out_dir) {
    const PhotonHashData data = cvt<PhotonHashData>(hd);
    std::vector<float4> in_pos((size_t)std::max(n, 1u)), o_pos((size_t)std::max(n, 1u));
    std::memcpy(in_pos.data(), pos4, (size_t)n * 16);
    std::fill(counts, counts + buckets, 0u);
    launch_sequential(n, [&]() { hash_photons(in_pos.data(), n, data, keys, counts); });
    const uint chunks = (buckets + SCAN_CHUNK_SIZE_VALUE - 1) / SCAN_CHUNK_SIZE_VALUE;
    std::vector<uint> small(chunks), big(chunks);
    launch_groups(chunks, SCAN_WG_SIZE_VALUE, [&]() { scan_small_chunks(counts, buckets, starts, small.data()); });
    launch_groups(1, SCAN_WG_SIZE_VALUE, [&]() { scan_big_chunks(small.data(), chunks, big.data()); });
    launch_groups(chunks, SCAN_WG_SIZE_VALUE, [&]() { scan_add_offsets(big.data(), buckets, starts); });
    std::memcpy(ends, starts, (size_t)buckets * 4);
    launch_sequential(n, [&]() {
        scatter_photons(in_pos.data(), power, dir, keys, ends, n, o_pos.data(), out_power, out_dir);
    });
    std::memcpy(out_pos4, o_pos.data(), (size_t)n * 16);
    return 0;
}

// kernels/gather_flux.cl over the pixels; hit points as written by ref_trace; flux (float4),
// weight (float) and radiance (float4) updated in place.
REF_API int ref_gather(const float *hp, uint n_pixels, const float *pos4, const uint *power, const uint *dir, uint n,
                       const uint *starts, const uint *ends, const phx_photon_hash_data *hd, float alpha, float *flux4,
                       float *weight, float *radiance4, int threads) {
    const PhotonHashData data = cvt<PhotonHashData>(hd);
    std::vector<float4> h[6];
    for (int k = 0; k < 6; k++) {
        h[k].resize(std::max(n_pixels, 1u));
        for (uint i = 0; i < n_pixels; i++)
            std::memcpy(&h[k][i], hp + 4 * (6 * (size_t)i + k), 16);
    }
    std::vector<float4> ppos((size_t)std::max(n, 1u)), fl(std::max(n_pixels, 1u)), rad(std::max(n_pixels, 1u));
    std::memcpy(ppos.data(), pos4, (size_t)n * 16);
    std::memcpy(fl.data(), flux4, (size_t)n_pixels * 16);
    std::memcpy(rad.data(), radiance4, (size_t)n_pixels * 16);
    launch_parallel(n_pixels, threads, [&]() {
        gather_flux(h[0].data(), h[1].data(), h[2].data(), h[3].data(), h[4].data(), h[5].data(), n_pixels, ppos.data(),
                    power, dir, n, starts, ends, data, alpha, fl.data(), weight, rad.data());
    });
    std::memcpy(flux4, fl.data(), (size_t)n_pixels * 16);
    std::memcpy(radiance4, rad.data(), (size_t)n_pixels * 16);
    return 0;
}

// The reference's device codecs and hash, for known-answer checks (encoding.h, photon_hash.h).
REF_API void ref_codecs(const float *in4, uint n, uint *rgbe, uint *oct, float *rgbe_dec4, float *oct_dec4) {
    for (uint i = 0; i < n; i++) {
        float4 v = float4_ctor(in4[4 * i], in4[4 * i + 1], in4[4 * i + 2], in4[4 * i + 3]);
        rgbe[i] = encode_rgbe(v);
        oct[i] = encode_oct(v);
        float4 a = decode_rgbe(rgbe[i]), b = decode_oct(oct[i]);
        std::memcpy(rgbe_dec4 + 4 * i, &a, 16);
        std::memcpy(oct_dec4 + 4 * i, &b, 16);
    }
}

REF_API void ref_pcg(uint seed, uint n, uint *out_u32, float *out_f) {
    RngState r = pcg_seed(seed);
    for (uint i = 0; i < n; i++) {
        RngState c = r;
        out_u32[i] = random_u32(&r);
        out_f[i] = random_float(&c);
    }
}

} // extern "C"
