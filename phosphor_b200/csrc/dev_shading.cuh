// dev_shading.cuh — surface interaction, materials, BSDF sampling and light sampling on the
// device.  Each function states the reference file:line it computes; expression trees follow the
// reference's operator order so results match it bit for bit under the arithmetic contract of
// dev_common.cuh.
#pragma once

#include "dev_scene.cuh"

namespace phx {

// hit.h:21-29
struct SurfaceHit {
    float4 position, normal;
    float uvx, uvy;
    float t;
    u32 mat_index;
    i32 tri;
    bool front_face;
};

PHX_DI u32 tri_mat(const SceneDesc &sc, i32 tri) { return __float_as_uint(__ldg(&sc.trirec[3 * (size_t)tri].w)); }

// hit.h:174-197 (compute_bary hit.h:31-43)
// The texture coordinates are interpolated only when need_uv (they feed texture lookups alone).
PHX_SHADE_HIT SurfaceHit process_hit(const SceneDesc &sc, const Hit &h, float4 origin, float4 dir,
                                     bool need_uv = true) {
    SurfaceHit s;
    s.t = h.t;
    s.tri = h.tri;
    s.mat_index = tri_mat(sc, h.tri);
    s.position = origin + dir * h.t;
    float u = h.u, v = h.v;
    float w = 1.0f - u - v;
    const float4 *nn = sc.tri_nrm + 3 * (size_t)h.tri;
    float4 n0 = __ldg(nn), n1 = __ldg(nn + 1), n2 = __ldg(nn + 2);
    float w0 = 1.0f - u - v;
    float4 b = f4(w0 * n0.x + u * n1.x + v * n2.x, w0 * n0.y + u * n1.y + v * n2.y, w0 * n0.z + u * n1.z + v * n2.z,
                  0.0f);
    float4 outward = normalize(b);
    bool front = dot(dir, outward) < 0.0f;
    s.normal = front ? outward : -outward;
    s.front_face = front;
    s.uvx = 0.0f;
    s.uvy = 0.0f;
    if (need_uv) {
        const float4 *uv = sc.tri_uv + 2 * (size_t)h.tri;
        float4 uva = __ldg(uv), uvb = __ldg(uv + 1);
        s.uvx = w * uva.x + u * uva.z + v * uvb.x;
        s.uvy = w * uva.y + u * uva.w + v * uvb.y;
    }
    return s;
}

// Whether a material reads any texture (and so the hit's texture coordinates).
PHX_DI bool mat_textured(const phx_material &m) {
    return m.diff_index != NO_TEXTURE || m.emis_index != NO_TEXTURE || m.norm_index != NO_TEXTURE ||
           m.occlusion_index != NO_TEXTURE || m.metal_rough_index != NO_TEXTURE || m.transmission_index != NO_TEXTURE;
}

// ---- textures: include/common/material.h:66-149 ------------------------------------------------
PHX_DI float4 srgb_to_linear(float4 c) {
    return f4(pm_powf(c.x, 2.2f), pm_powf(c.y, 2.2f), pm_powf(c.z, 2.2f), c.w);
}

PHX_DI float4 naive_sample_texture(const SceneDesc &sc, u32 index, float ux, float uy) {
    if (index == NO_TEXTURE)
        return white4();
    phx_texture_meta m = sc.tex_meta[index];
    u32 px = (u32)(ux * (float)m.width);
    px = px < m.width - 1 ? px : m.width - 1;
    u32 py = (u32)(uy * (float)m.height);
    py = py < m.height - 1 ? py : m.height - 1;
    u32 texel = m.atlas_offset + (py * m.width + px) * 3u;
    float r = (float)sc.tex_atlas[texel + 0] / 255.0f;
    float g = (float)sc.tex_atlas[texel + 1] / 255.0f;
    float b = (float)sc.tex_atlas[texel + 2] / 255.0f;
    return f4(r, g, b, 1.0f);
}

PHX_DI float4 texel4(const SceneDesc &sc, i32 idx) {
    return f4((float)sc.tex_atlas[idx], (float)sc.tex_atlas[idx + 1], (float)sc.tex_atlas[idx + 2], 255.0f) / 255.0f;
}

PHX_DI float4 sample_texture(const SceneDesc &sc, u32 index, float ux, float uy) {
    if (index == NO_TEXTURE)
        return white4();
    phx_texture_meta m = sc.tex_meta[index];
    i32 w = (i32)m.width, h = (i32)m.height;
    ux = ux - floorf(ux);
    uy = uy - floorf(uy);
    uy = 1.0f - uy;
    float x = fminf(ux * (float)w, (float)(w - 1));
    float y = fminf(uy * (float)h, (float)(h - 1));
    i32 x1 = min((i32)x, w - 1);
    i32 x2 = min((i32)ceilf(x), w - 1);
    i32 y1 = min((i32)y, h - 1);
    i32 y2 = min((i32)ceilf(y), h - 1);
    i32 ch = (i32)m.channels, off = (i32)m.atlas_offset;
    float4 Q11 = texel4(sc, off + (y1 * w + x1) * ch);
    float4 Q12 = texel4(sc, off + (y2 * w + x1) * ch);
    float4 Q21 = texel4(sc, off + (y1 * w + x2) * ch);
    float4 Q22 = texel4(sc, off + (y2 * w + x2) * ch);
    if (x2 == x1 && y2 == y1)
        return naive_sample_texture(sc, index, ux, uy);
    else if (x2 == x1)
        return mix(Q11, Q12, y - (float)y1);
    else if (y2 == y1)
        return mix(Q11, Q21, x - (float)x1);
    float denom = (float)((x2 - x1) * (y2 - y1));
    float w11 = ((float)x2 - x) * ((float)y2 - y) / denom;
    float w12 = ((float)x2 - x) * (y - (float)y1) / denom;
    float w21 = (x - (float)x1) * ((float)y2 - y) / denom;
    float w22 = (x - (float)x1) * (y - (float)y1) / denom;
    return w11 * Q11 + w12 * Q12 + w21 * Q21 + w22 * Q22;
}

PHX_SHADE_TEX float4 sample_texture_uv(const SceneDesc &sc, u32 mat_index, u32 tex_index, float ux, float uy, u32 slot) {
    const phx_uv_transform *t = &sc.uvt[mat_index].diff + slot;
    float sx = ux * t->uv_scale.x, sy = uy * t->uv_scale.y;
    float c, s;
    pm_sincosf(t->uv_rotation, &s, &c);
    float rx = c * sx - s * sy, ry = s * sx + c * sy;
    return sample_texture(sc, tex_index, rx + t->uv_offset.x, ry + t->uv_offset.y);
}

// ---- shading.h:13-123 --------------------------------------------------------------------------
struct ShadingContext {
    float4 base_color, emissive, shading_normal;
    float metallic, roughness, transmission, occlusion, ior;
};

struct IorStack {
    float ior[IOR_STACK_SIZE];
    u32 cur;
};
PHX_DI void init_ior_stack(IorStack *s, float v) {
    s->cur = 0;
    s->ior[0] = v;
}
PHX_DI float current_ior(const IorStack *s) { return s->ior[s->cur]; }
PHX_DI float target_ior(const IorStack *s, float inside, bool front) {
    if (front)
        return inside;
    return (s->cur == 0) ? AIR_IOR : s->ior[s->cur - 1];
}
PHX_DI void update_ior_stack(IorStack *s, float inside, bool front) {
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

PHX_DI float4 apply_normal_map(float4 ms, float4 gn, float4 t, float4 b) {
    float4 n = f4(ms.x * 2.0f - 1.0f, ms.y * 2.0f - 1.0f, ms.z * 2.0f - 1.0f, 0.0f);
    float4 p = n.x * t + n.y * b + n.z * gn;
    float len = length(p);
    return (len > EPS) ? (p / len) : gn;
}

PHX_SHADE_HIT ShadingContext evaluate_material(const SceneDesc &sc, const phx_material &mat, u32 mi, float ux, float uy,
                                        float4 gn, float4 t, float4 b) {
    ShadingContext ctx;
    ctx.base_color = f4(mat.base_color);
    if (mat.diff_index != NO_TEXTURE)
        ctx.base_color *= srgb_to_linear(sample_texture_uv(sc, mi, mat.diff_index, ux, uy, 0));
    ctx.emissive = f4(mat.emissive);
    if (mat.emis_index != NO_TEXTURE)
        ctx.emissive *= srgb_to_linear(sample_texture_uv(sc, mi, mat.emis_index, ux, uy, 1));
    ctx.metallic = mat.metallic;
    ctx.roughness = mat.roughness;
    if (mat.metal_rough_index != NO_TEXTURE) {
        float4 mr = sample_texture_uv(sc, mi, mat.metal_rough_index, ux, uy, 4);
        ctx.metallic *= mr.z;
        ctx.roughness *= mr.y;
    }
    ctx.roughness = clampf(ctx.roughness, MIN_ROUGHNESS, 1.0f);
    ctx.transmission = mat.transmission;
    if (mat.transmission_index != NO_TEXTURE) {
        float4 tx = sample_texture_uv(sc, mi, mat.transmission_index, ux, uy, 5);
        ctx.transmission *= tx.x;
    }
    ctx.occlusion = 1.0f;
    if (mat.occlusion_index != NO_TEXTURE) {
        float4 occ = sample_texture_uv(sc, mi, mat.occlusion_index, ux, uy, 3);
        ctx.occlusion = occ.x;
    }
    ctx.ior = mat.ior;
    ctx.shading_normal = gn;
    if (mat.norm_index != NO_TEXTURE) {
        float4 ms = sample_texture_uv(sc, mi, mat.norm_index, ux, uy, 2);
        ctx.shading_normal = apply_normal_map(ms, gn, t, b);
    }
    return ctx;
}

// shading.h:125-133
PHX_DI float4 beer_lambert(float4 att, float att_dist, float travel) {
    if (att_dist < EPS)
        return white4();
    float4 sigma =
        f4(-pm_logf(fmaxf(att.x, EPS)), -pm_logf(fmaxf(att.y, EPS)), -pm_logf(fmaxf(att.z, EPS)), 0.0f) / att_dist;
    return f4(pm_expf(-sigma.x * travel), pm_expf(-sigma.y * travel), pm_expf(-sigma.z * travel), 0.0f);
}

// ---- bsdfs.h:11-121 ----------------------------------------------------------------------------
PHX_DI float4 reflect(float4 in, float4 n) { return normalize(in - (2.0f * dot(in, n)) * n); }
PHX_DI float4 safe_reflect(float4 d, float4 n, float4 gn) {
    float4 r = reflect(d, n);
    if (dot(r, gn) <= 0.0f) {
        r = r - dot(r, gn) * gn;
        r = normalize(r);
    }
    return r;
}

// ggx_sample_vndf with the frame of `normal` (make_tbn) given by the caller; *refl receives
// reflect(-view, h) when the accepted attempt computed it (*has_refl), as it does unless every
// attempt failed and h is the normal.
PHX_DI float4 ggx_sample_vndf_tbn(Rng *rng, float4 normal, float4 t, float4 b, float4 gn, float4 view,
                                  float roughness, float4 *refl_out, bool *has_refl) {
    *has_refl = false;
    float alpha = roughness * roughness;
    float4 vl = normalize(f4(dot(view, t), dot(view, b), dot(view, normal), 0.0f));
    float4 vh = normalize(f4(alpha * vl.x, alpha * vl.y, vl.z, 0.0f));
    float len_sq = vh.x * vh.x + vh.y * vh.y;
    float4 T1 = (len_sq > 0.0f) ? f4(-vh.y, vh.x, 0.0f, 0.0f) * (1.0f / sqrtf(len_sq)) : f4(1.0f, 0.0f, 0.0f, 0.0f);
    float4 T2 = cross(vh, T1);
    float s = 0.5f * (1.0f + vh.z);
    for (u32 a = 0; a < GGX_SAMPLING_ATTEMPTS; a++) {
        float u1 = random_float(rng);
        float u2 = random_float(rng);
        float r = sqrtf(u1);
        float phi = (2.0f * PI) * u2;
        float sp, cp;
        pm_sincosf(phi, &sp, &cp);
        float t1 = r * cp;
        float t2 = r * sp;
        t2 = (1.0f - s) * sqrtf(fmaxf(0.0f, 1.0f - t1 * t1)) + s * t2;
        float nz2 = fmaxf(0.0f, 1.0f - t1 * t1 - t2 * t2);
        float4 nh = t1 * T1 + t2 * T2 + sqrtf(nz2) * vh;
        float4 nel = normalize(f4(alpha * nh.x, alpha * nh.y, fmaxf(0.0f, nh.z), 0.0f));
        float4 ne = normalize(nel.x * t + nel.y * b + nel.z * normal);
        float4 refl = reflect(-view, ne);
        if (dot(refl, gn) >= 0.0f) {
            *refl_out = refl;
            *has_refl = true;
            return ne;
        }
    }
    return normal;
}
PHX_DI float4 ggx_sample_vndf(Rng *rng, float4 normal, float4 gn, float4 view, float roughness) {
    float4 t, b, refl;
    bool has_refl;
    make_tbn(normal, &t, &b);
    return ggx_sample_vndf_tbn(rng, normal, t, b, gn, view, roughness, &refl, &has_refl);
}

PHX_DI float smith_g1_ggx(float c, float alpha) {
    if (c <= 0.0f)
        return 0.0f;
    float a2 = alpha * alpha;
    return 2.0f * c / (c + sqrtf(a2 + (1.0f - a2) * c * c));
}
PHX_DI float fresnel(float r0, float4 in, float4 n) {
    float c = fabsf(dot(in, n));
    return r0 + (1.0f - r0) * pm_powf(1.0f - c, 5.0f);
}
PHX_DI float4 fresnel4(float4 r0, float4 in, float4 n) {
    float c = fabsf(dot(in, n));
    float p = pm_powf(1.0f - c, 5.0f);
    return f4(r0.x + (1.0f - r0.x) * p, r0.y + (1.0f - r0.y) * p, r0.z + (1.0f - r0.z) * p, r0.w + (1.0f - r0.w) * p);
}
PHX_DI float fresnel_refracted(float i1, float i2, float4 in, float4 n) {
    float r0 = pm_powf((i1 - i2) / (i1 + i2), 2.0f);
    return fresnel(r0, in, n);
}
PHX_DI float4 refract(float4 in, float4 n, float eta1, float eta2, bool *tir) {
    float eta = eta1 / eta2;
    float ndi = dot(in, n);
    float sin_t2 = eta * eta * (1.0f - ndi * ndi);
    if (sin_t2 > 1.0f) {
        *tir = true;
        return reflect(in, n);
    }
    *tir = false;
    float4 rf = eta * in - (eta * ndi + sqrtf(1.0f - sin_t2)) * n;
    return normalize(rf);
}
PHX_DI float ggx_ndf(float ndh, float alpha) {
    float a2 = alpha * alpha;
    float d = ndh * ndh * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxf(PI * d * d, EPS);
}

enum { BSDF_DIFFUSE = 0, BSDF_METALLIC = 1, BSDF_FRESNEL = 2, BSDF_TRANSMIT = 3 };
struct BsdfSample {
    float4 dir, throughput;
    u32 event;
};

// shading.h:150-213
PHX_SHADE_BSDF BsdfSample sample_bsdf(Rng *rng, const ShadingContext &ctx, float4 sn, float4 gn, float4 view, IorStack *ior,
                              bool front) {
    BsdfSample s;
    // one frame of the shading normal serves the microfacet sample and a diffuse direction
    float4 tn, bn;
    make_tbn(sn, &tn, &bn);
    float4 hr;
    bool has_hr;
    float4 h = ggx_sample_vndf_tbn(rng, sn, tn, bn, gn, view, ctx.roughness, &hr, &has_hr);
    // safe_reflect(-view, h, gn), reusing reflect(-view, h) from the microfacet sample
    auto reflect_h = [&]() {
        float4 r = has_hr ? hr : reflect(-view, h);
        if (dot(r, gn) <= 0.0f) {
            r = r - dot(r, gn) * gn;
            r = normalize(r);
        }
        return r;
    };
    float alpha = ctx.roughness * ctx.roughness;
    if (random_float(rng) < ctx.metallic) {
        s.dir = reflect_h();
        float cl = fmaxf(0.0f, dot(s.dir, sn));
        float g1 = smith_g1_ggx(cl, alpha);
        s.throughput = fresnel4(ctx.base_color, -view, h) * g1;
        s.event = BSDF_METALLIC;
        return s;
    }
    float i1 = current_ior(ior);
    float i2 = target_ior(ior, ctx.ior, front);
    float fr = fresnel_refracted(i1, i2, -view, h);
    float r_diel = random_float(rng);
    if (r_diel < fr) {
        s.dir = reflect_h();
        float cl = fmaxf(0.0f, dot(s.dir, sn));
        float g1 = smith_g1_ggx(cl, alpha);
        s.throughput = f4(g1, g1, g1, 0.0f);
        s.event = BSDF_FRESNEL;
        return s;
    }
    float r_trans = (r_diel - fr) / fmaxf(1.0f - fr, EPS);
    if (r_trans < ctx.transmission) {
        bool tir;
        float4 rf = refract(-view, h, i1, i2, &tir);
        if (tir) {
            s.dir = reflect_h();
            float cl = fmaxf(0.0f, dot(s.dir, sn));
            float g1 = smith_g1_ggx(cl, alpha);
            s.throughput = f4(g1, g1, g1, 0.0f);
            s.event = BSDF_FRESNEL;
            return s;
        }
        bool transmitted = dot(rf, h) < 0.0f;
        if (transmitted)
            update_ior_stack(ior, ctx.ior, front);
        s.dir = rf;
        float cl = fmaxf(0.0f, fabsf(dot(rf, sn)));
        float g1 = smith_g1_ggx(cl, alpha);
        s.throughput = ctx.base_color * g1;
        s.event = BSDF_TRANSMIT;
        return s;
    }
    s.dir = random_in_unit_hemisphere_tbn(rng, sn, tn, bn);
    if (dot(s.dir, gn) <= 0.0f)
        s.dir = random_in_unit_hemisphere(rng, gn);
    s.throughput = ctx.base_color;
    s.event = BSDF_DIFFUSE;
    return s;
}

// ---- light_sampling.h:18-390 -------------------------------------------------------------------
struct EmissivePoint {
    u32 tri_idx;
    float bu, bv, bw;
    float4 pos, normal;
};
struct LightFragment {
    float4 radiance, dir;
    float dist, n_dot_dir;
};

PHX_DI float spotlight_falloff(float c, float ci, float co) {
    float t = clampf((c - co) / (ci - co + EPS), 0.0f, 1.0f);
    return t * t * (3.0f - 2.0f * t);
}
PHX_DI void fill_light_vecs(float4 from_, float4 to, float4 *dir, float *dist, float *dist_sq) {
    float4 d = to - from_;
    *dist_sq = fmaxf(dot(d, d), EPS);
    *dist = sqrtf(*dist_sq);
    *dir = d / *dist;
}
PHX_DI u32 choose_emissive_triangle(Rng *rng, const SceneDesc &sc, u32 start, u32 n, float total_area) {
    if (n <= 1 || total_area <= EPS)
        return start;
    float r = random_float(rng) * total_area;
    float accum = 0.0f;
    for (u32 i = 0; i < n; i++) {
        const float4 *ev = sc.etri_v + 3 * (size_t)(start + i);
        float4 v0 = __ldg(ev), v1 = __ldg(ev + 1), v2 = __ldg(ev + 2);
        accum += 0.5f * length(cross(v1 - v0, v2 - v0));
        if (r <= accum)
            return start + i;
    }
    return start + n - 1;
}
PHX_DI EmissivePoint sample_emissive_point(Rng *rng, const SceneDesc &sc, u32 start, u32 n, float total_area) {
    EmissivePoint p;
    p.tri_idx = choose_emissive_triangle(rng, sc, start, n, total_area);
    float r1 = random_float(rng);
    float r2 = random_float(rng);
    float s = sqrtf(r1);
    p.bu = 1.0f - s;
    p.bv = r2 * s;
    p.bw = 1.0f - p.bu - p.bv;
    const float4 *ev = sc.etri_v + 3 * (size_t)p.tri_idx;
    float4 v0 = __ldg(ev), v1 = __ldg(ev + 1), v2 = __ldg(ev + 2);
    p.pos = p.bw * v0 + p.bu * v1 + p.bv * v2;
    const float4 *en = sc.etri_n + 3 * (size_t)p.tri_idx;
    float4 nn = p.bw * __ldg(en) + p.bu * __ldg(en + 1) + p.bv * __ldg(en + 2);
    if (length(nn) > EPS)
        p.normal = normalize(nn);
    else
        p.normal = normalize(cross(v1 - v0, v2 - v0));
    return p;
}
PHX_DI float4 apply_emissive_texture(const SceneDesc &sc, float4 color, u32 tex_index, const EmissivePoint &p) {
    if (tex_index == NO_TEXTURE)
        return color;
    const float4 *uv = sc.etri_uv + 2 * (size_t)p.tri_idx;
    float4 a = __ldg(uv), b = __ldg(uv + 1);
    float ux = p.bw * a.x + p.bu * a.z + p.bv * b.x;
    float uy = p.bw * a.y + p.bu * a.w + p.bv * b.y;
    u32 mi = sc.etri_mat[p.tri_idx];
    float4 tc = sample_texture_uv(sc, mi, tex_index, ux, uy, 1);
    return color * srgb_to_linear(tc);
}
PHX_DI u32 select_light(Rng *rng, const SceneDesc &sc, float *scale) {
    u32 n = sc.n_lights;
    float total = sc.total_lum;
    if (n == 0 || total < EPS) {
        *scale = 1.0f;
        return 0;
    }
    float r = random_float(rng) * total;
    u32 low = 0, high = n;
    while (low < high) {
        u32 mid = (low + high) / 2;
        if (__ldg(&sc.lum_pref_sum[mid]) < r)
            low = mid + 1;
        else
            high = mid;
    }
    if (low >= n)
        low = n - 1;
    float lum = (low == 0) ? __ldg(&sc.lum_pref_sum[0])
                           : (__ldg(&sc.lum_pref_sum[low]) - __ldg(&sc.lum_pref_sum[low - 1]));
    *scale = fmaxf(lum / total, EPS);
    return low;
}

// light_sampling.h:200-227
PHX_SHADE_LIGHT void sample_light(Rng *rng, const SceneDesc &sc, float4 *origin, float4 *dir, float4 *power) {
    if (sc.n_lights == 0 || sc.total_lum < EPS) {
        *origin = zero4();
        *dir = f4(0.0f, 1.0f, 0.0f, 0.0f);
        *power = zero4();
        return;
    }
    float scale;
    u32 idx = select_light(rng, sc, &scale);
    const phx_light &L = sc.lights[idx];
    u8 kind = L.kind;
    if (kind == PHX_LIGHT_POINT) {
        *origin = f4(L.position);
        *dir = random_unit_vector(rng);
        *power = f4(L.power) * (4.0f * PI);
    } else if (kind == PHX_LIGHT_SPOT) {
        *origin = f4(L.position);
        float ci = pm_cosf(L.aux.x);
        float co = pm_cosf(L.aux.y);
        float r1 = random_float(rng);
        float r2 = random_float(rng);
        float ct = 1.0f - r1 * (1.0f - co);
        float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
        float phi = (2.0f * PI) * r2;
        float sp, cp;
        pm_sincosf(phi, &sp, &cp);
        float4 ld = f4(st * cp, st * sp, ct, 0.0f);
        float4 t, b;
        float4 ldir = normalize(f4(L.direction));
        make_tbn(ldir, &t, &b);
        *dir = normalize(ld.x * t + ld.y * b + ld.z * ldir);
        float fo = spotlight_falloff(ct, ci, co);
        float sa = (2.0f * PI) * (1.0f - co);
        *power = f4(L.power) * fo * sa;
    } else if (kind == PHX_LIGHT_DIRECTIONAL) {
        float4 center = sc.scene_center;
        float radius = sc.scene_radius;
        float r1 = radius * sqrtf(random_float(rng));
        float r2 = (2.0f * PI) * random_float(rng);
        float s2, c2;
        pm_sincosf(r2, &s2, &c2);
        float4 disk = r1 * (c2 * f4(L.tangent) + s2 * f4(L.bitangent));
        *dir = f4(L.direction);
        *origin = center - f4(L.direction) * 2.0f * radius + disk;
        *power = f4(L.power) * PI * radius * radius;
    } else {
        u32 tex_idx = __float_as_uint(L.aux.x);
        u32 start = __float_as_uint(L.aux.y);
        u32 ntri = __float_as_uint(L.aux.z);
        float area = L.aux.w;
        EmissivePoint p = sample_emissive_point(rng, sc, start, ntri, area);
        *dir = random_in_unit_hemisphere(rng, p.normal);
        *origin = p.pos + EPS * *dir;
        *power = apply_emissive_texture(sc, f4(L.power), tex_idx, p);
    }
    *power /= scale;
}

// light_sampling.h:231-300; always inlined (sample_light_fragment is the possibly out-of-line copy).
PHX_DI bool light_fragment(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, LightFragment *out) {
    if (sc.n_lights == 0 || sc.total_lum < EPS)
        return false;
    float scale;
    u32 li = select_light(rng, sc, &scale);
    const phx_light &L = sc.lights[li];
    u8 kind = L.kind;
    float4 flux = f4(L.power.x, L.power.y, L.power.z, 0.0f) / scale;
    float4 dir;
    float dist, dist_sq, ndd;
    float4 radiance;
    if (kind == PHX_LIGHT_POINT || kind == PHX_LIGHT_SPOT) {
        fill_light_vecs(pos, f4(L.position), &dir, &dist, &dist_sq);
        ndd = dot(dir, normal);
        if (ndd <= 0.0f)
            return false;
        float cone = 1.0f;
        if (kind == PHX_LIGHT_SPOT) {
            float cd = dot(-dir, normalize(f4(L.direction)));
            cone = spotlight_falloff(cd, pm_cosf(L.aux.x), pm_cosf(L.aux.y));
            if (cone < EPS)
                return false;
        }
        radiance = flux * cone * ndd / dist_sq;
    } else if (kind == PHX_LIGHT_DIRECTIONAL) {
        dir = normalize(-f4(L.direction));
        dist = INF;
        ndd = dot(dir, normal);
        if (ndd <= 0.0f)
            return false;
        radiance = flux * ndd;
    } else {
        u32 tex_index = __float_as_uint(L.aux.x);
        u32 start = __float_as_uint(L.aux.y);
        u32 ntri = __float_as_uint(L.aux.z);
        float area = L.aux.w;
        if (area < EPS)
            return false;
        EmissivePoint p = sample_emissive_point(rng, sc, start, ntri, area);
        fill_light_vecs(pos, p.pos, &dir, &dist, &dist_sq);
        ndd = dot(dir, normal);
        if (ndd <= 0.0f)
            return false;
        float4 ef = apply_emissive_texture(sc, flux, tex_index, p);
        float cos_l = fmaxf(dot(-dir, p.normal), 0.0f);
        radiance = ef * ndd * cos_l / (PI * dist_sq);
    }
    if (dot(radiance, radiance) < EPS * EPS)
        return false;
    out->radiance = radiance;
    out->dir = dir;
    out->dist = dist;
    out->n_dot_dir = ndd;
    return true;
}
PHX_SHADE_NEE bool sample_light_fragment(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, LightFragment *out) {
    return light_fragment(rng, sc, pos, normal, out);
}

// light_sampling.h:302-333
// A shadow ray crossing the surface it hit at h (one step of the walk in shadow_transmittance):
// false when the surface blocks the ray (the transmittance is then zero).
// uv_pending: h carries no barycentrics yet (a hit taken from a HitList without them).
// NOTEX: no material of the context has a texture.
template <bool NOTEX = false>
PHX_DI bool shadow_cross(const SceneDesc &sc, const Hit &h, float4 origin, float4 dir, float t_min, float4 *trans,
                         bool uv_pending = false) {
    u32 mi = tri_mat(sc, h.tri);
    const phx_material &mat = sc.materials[mi];
    if (mat.transmission < EPS)
        return false;
    float4 base = f4(mat.base_color);
    if (!NOTEX && mat.diff_index != NO_TEXTURE) {
        Hit hh = h;
        if (uv_pending)
            hit_uv(sc, h.tri, origin, dir, &hh.u, &hh.v);
        SurfaceHit s = process_hit(sc, hh, origin, dir);
        base *= srgb_to_linear(sample_texture_uv(sc, mi, mat.diff_index, s.uvx, s.uvy, 0));
    }
    float4 tr = *trans;
    if (mat.att_dist > EPS)
        tr *= beer_lambert(f4(mat.att_color), mat.att_dist, h.t - t_min);
    tr *= base * mat.transmission;
    *trans = tr;
    return !(dot(tr, tr) < EPS);
}

// The walk of shadow_transmittance by closest-hit queries (any-hit where no material transmits),
// from step `depth` at t_min with the transmittance so far.  (Compiled out of line it freed the
// shadow kernels' spills but measured 5 % slower.)
template <bool NOTEX = false>
PHX_DI float4 shadow_walk(const SceneDesc &sc, float4 origin, float4 dir, float t_min, float t_max, u32 depth,
                                  float4 trans, u32 *overflow) {
    for (; depth < MAX_RAY_BOUNCES; depth++) {
        Hit h;
        if (!intersect(sc, origin, dir, t_min, t_max, &h, overflow, sc.any_transmissive == 0))
            break;
        if (!shadow_cross<NOTEX>(sc, h, origin, dir, t_min, &trans))
            return zero4();
        t_min = h.t + EPS;
    }
    return trans;
}

#ifndef PHX_SHADOW_LIST
// Hits a shadow ray's single traversal collects in scenes with transmissive materials: 2 holds a
// crossing of a closed glass surface (in and out) and measured fastest (shadow stage 8.3 ms with no
// list, 6.3 ms with 2, 7.1 with 3, 7.8 with 4: each entry costs registers).
#define PHX_SHADOW_LIST 2
#endif

// The reference walks the segment with one closest-hit query per surface crossed, each starting
// EPS past the previous hit (light_sampling.h).  In scenes with transmissive materials one
// traversal lists the nearest hits instead (intersect_list): a hit's t, u, v and rank do not
// depend on the query's bounds, so the query of each step returns the first listed hit at or
// beyond its t_min, provided the list holds every hit up to that one.  Where it cannot vouch for
// that, the walk goes on with closest-hit queries from there: the result is the reference's.
template <int KIND = SHADOW_GENERAL>
PHX_DI float4 shadow_transmittance(const SceneDesc &sc, float4 origin, float4 dir, float dist, u32 *overflow) {
    float4 trans = white4();
    float t_min = EPS, t_max = dist - EPS;
    if constexpr (KIND == SHADOW_OPAQUE) { // every surface blocks: any hit on the segment gives zero
        return occluded(sc, origin, dir, t_min, t_max, overflow) ? zero4() : trans;
    } else {
    u32 depth = 0;
#if PHX_SHADOW_LIST > 0
    if (sc.any_transmissive != 0) {
        constexpr int K = PHX_SHADOW_LIST;
        HitList<K> L;
        intersect_list(sc, origin, dir, t_min, t_max, &L, overflow);
        const bool whole = !(L.lost < __int_as_float(0x7f800000)) && L.bound == t_max; // every hit listed
        for (; depth < MAX_RAY_BOUNCES; depth++) {
            Hit h;
            bool found = false;
#pragma unroll
            for (int i = 0; i < K; i++) {
                if (!found && i < L.n && !(L.t[i] < t_min)) {
                    h.t = L.t[i];
                    h.u = h.v = 0.0f; // recomputed by shadow_cross where a texture needs them
                    h.tri = L.tri[i];
                    found = true;
                }
            }
            if (found ? !(h.t < L.lost && h.t <= L.bound) : !whole)
                break; // not vouched for: closest-hit queries from here on
            if (!found)
                return trans; // no surface left on the segment
            if (!shadow_cross<KIND == SHADOW_CLEAR>(sc, h, origin, dir, t_min, &trans, true))
                return zero4();
            t_min = h.t + EPS;
        }
    }
#endif
    return shadow_walk<KIND == SHADOW_CLEAR>(sc, origin, dir, t_min, t_max, depth, trans, overflow);
    }
}

PHX_DI float4 direct_lighting_diffuse(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, float4 base,
                                      u32 *overflow) { // light_sampling.h:335-353
    LightFragment f;
    if (!sample_light_fragment(rng, sc, pos, normal, &f))
        return zero4();
    float4 trans = shadow_transmittance(sc, pos, f.dir, f.dist, overflow);
    return f.radiance * (base / PI) * trans;
}

PHX_DI float4 direct_lighting_specular(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, float4 view,
                                       float4 f0, float roughness, u32 *overflow) { // light_sampling.h:355-390
    float ndv = dot(view, normal);
    if (ndv < EPS)
        return zero4();
    LightFragment f;
    if (!sample_light_fragment(rng, sc, pos, normal, &f))
        return zero4();
    if (f.n_dot_dir < EPS)
        return zero4();
    float alpha = roughness * roughness;
    float4 h = normalize(f.dir + view);
    float ndh = fmaxf(dot(normal, h), 0.0f);
    float g = ggx_ndf(ndh, alpha);
    float4 fr = fresnel4(f0, view, h);
    float sm = smith_g1_ggx(f.n_dot_dir, alpha) * smith_g1_ggx(ndv, alpha);
    float4 spec = f.radiance * g * fr * sm / (4.0f * f.n_dot_dir * ndv);
    if (dot(spec, spec) < EPS * EPS)
        return zero4();
    float4 trans = shadow_transmittance(sc, pos, f.dir, f.dist, overflow);
    return spec * trans;
}

// envmap.h:9-20
PHX_DI float4 sample_envmap(const SceneDesc &sc, float4 dir) {
    float theta = pm_acosf(clampf(dir.z, -1.0f, 1.0f));
    float phi = pm_atan2f(dir.y, dir.x);
    float u = (phi + PI) / (2.0f * PI);
    float v = clampf(1.0f - theta / PI, 0.0f, 1.0f);
    u = u - floorf(u);
    u32 px = (u32)(u * (float)sc.env_w);
    px = px < sc.env_w - 1 ? px : sc.env_w - 1;
    u32 py = (u32)(v * (float)sc.env_h);
    py = py < sc.env_h - 1 ? py : sc.env_h - 1;
    u32 idx = 3 * (py * sc.env_w + px);
    return f4(__ldg(&sc.envmap[idx]), __ldg(&sc.envmap[idx + 1]), __ldg(&sc.envmap[idx + 2]), 0.0f);
}

// camera.h:28-47
PHX_DI void make_ray(const phx_camera_params &cam, u32 px, u32 py, u32 width, u32 height, Rng *rng, float4 *origin,
                     float4 *dir) {
    float u = random_float(rng) - 0.5f;
    float v = random_float(rng) - 0.5f;
    float s = ((float)px + 0.5f + u) / (float)width;
    float t = 1.0f - ((float)py + 0.5f + v) / (float)height;
    float4 disk = zero4();
    if (cam.defocus_angle > 0.0f) {
        float r1 = sqrtf(random_float(rng));
        float r2 = (2.0f * PI) * random_float(rng);
        float c, sn;
        pm_sincosf(r2, &sn, &c);
        disk = r1 * (c * f4(cam.defocus_disk_u) + sn * f4(cam.defocus_disk_v));
    }
    *origin = f4(cam.position) + disk;
    float4 d = f4(cam.lower_left_corner) + s * f4(cam.horizontal) + t * f4(cam.vertical) - *origin;
    *dir = normalize(d);
}

// tangent frame at a hit (trace_rays.cl:83-93, emit_photons.cl:66-76)
PHX_DI void hit_frame(const SceneDesc &sc, const Hit &h, const SurfaceHit &s, float4 *tangent, float4 *bitangent) {
    float bw = 1.0f - h.u - h.v;
    const float4 *tt = sc.tri_tan + 3 * (size_t)h.tri;
    float4 traw = bw * __ldg(tt) + h.u * __ldg(tt + 1) + h.v * __ldg(tt + 2);
    float4 braw = (length(traw) > EPS) ? cross(s.normal, traw) : zero4();
    if (length(braw) > EPS) {
        *bitangent = normalize(braw);
        *tangent = cross(*bitangent, s.normal);
    } else {
        make_tbn(s.normal, tangent, bitangent);
    }
}

} // namespace phx
