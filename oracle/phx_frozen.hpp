// phx_frozen.hpp — TEST INFRASTRUCTURE ONLY (part of the oracle): the frozen-path SPPM estimator
// F(θ') that the library's adjoint differentiates, evaluated in double (its central finite
// differences are one reference gradient) or, with the scalar type S = Dual<N> of phx_dual.hpp,
// in forward-mode dual numbers (the analytic FP64 gradient, all partials in one evaluation).
// Every function is a template on S; with S = double it performs exactly the double operations
// of the untemplated estimator.  Never linked into the product.
//
// Everything random or discrete is frozen at the scene's own parameters θ0 — the float render of
// phx_oracle.hpp replayed draw for draw: camera and photon paths, hit points, photon positions and
// directions, BSDF events, microfacet normals, Russian-roulette decisions and factors, light
// selections and their probabilities, NEE directions, shadow-ray hit lists, gather neighbourhoods,
// kernel weights, radii and SPPM ratios.  Only the weights depend on θ' = (per-material base colour
// and roughness, per-light power):
//   * a BSDF bounce with frozen view v, direction l and microfacet normal h has weight
//     W(θ') = W(θ0) · f(θ')/f(θ0) (detached sampling): the base-colour factor of the reference's
//     weight (shading.h:150-213: base for diffuse and transmission, Schlick F(base) for metal) taken
//     at θ', times D(h;α')G1(v;α')G1(l;α') / (D(h;α0)G1(v;α0)G1(l;α0)) with α = roughness²
//     (a factor whose cosine is 0 is left out);
//   * light power enters linearly: photon power and NEE radiance scale by L'/L0 per channel;
//   * NEE samples are re-evaluated at θ' along their frozen directions (light_sampling.h:335-390:
//     base'/π for diffuse, D·F·G1·G1/(4 n·l n·v) at α' with f0 = base' for metal), and a
//     transmissive occluder contributes base'·transmission (light_sampling.h:302-333);
//   * photon power is carried unquantised (no RGBE).
// The image is I(θ') = radiance'/R + flux'.xyz / (π r_R² N_emitted) with
// flux'_{n+1} = (flux'_n + T'·A'/π·Σ_k w_k Φ'_k)·ratio_n over the θ0 neighbourhoods and ratios
// (gather_flux.cl:5-78, output.cpp:62-76).  At θ' = θ0, F differs from the float render only by
// precision and by the photon-power quantisation.
#pragma once

#include "phx_dual.hpp"
#include "phx_oracle.hpp"

namespace orc {
namespace frozen {

template <class S> inline V4<S> dd(const V4<float> &v) { return mk<S>(S(v.x), S(v.y), S(v.z), S(v.w)); }
template <class S> inline V4<S> dd(const phx_f4 &v) { return mk<S>(S(v.x), S(v.y), S(v.z), S(v.w)); }

// θ': per material base colour (xyz) and roughness, per light power (xyz), in the scalar type S
// (with tangents for S = Dual); the tables hold every other field of θ' (the scene's counts).
template <class S> struct Primed {
    const phx_material *mats;
    const phx_light *lights;
    const V4<S> *base;  // per material
    const S *rough;     // per material
    const V4<S> *power; // per light
};

// Primed<double> over float tables (the θ' of orc_frozen_render)
struct PrimedTables {
    std::vector<V4<double>> base, power;
    std::vector<double> rough;
    PrimedTables(const phx_material *m, u32 nm, const phx_light *l, u32 nl) {
        for (u32 i = 0; i < nm; i++) {
            base.push_back(dd<double>(m[i].base_color));
            rough.push_back(m[i].roughness);
        }
        for (u32 i = 0; i < nl; i++)
            power.push_back(dd<double>(l[i].power));
    }
};

// L'/L0 per channel for light li (0 where the θ0 power is 0)
template <class S> inline V4<S> light_ratio(const Scene &sc, const Primed<S> &pr, u32 li) {
    if (sc.n_lights == 0)
        return zero4<S>();
    const phx_f4 &a = sc.lights[li].power;
    const V4<S> &b = pr.power[li];
    return mk<S>(a.x != 0.0f ? b.x / S(a.x) : S(0.0), a.y != 0.0f ? b.y / S(a.y) : S(0.0),
                 a.z != 0.0f ? b.z / S(a.z) : S(0.0), S(0.0));
}

// base colour and roughness of material mi at θ', with the same texture factors as θ0
template <class S> inline V4<S> base_primed(const Scene &sc, const Primed<S> &pr, u32 mi, float uvx, float uvy) {
    const phx_material &m = pr.mats[mi];
    V4<S> b = pr.base[mi];
    if (m.diff_index != NO_TEXTURE)
        b = b * dd<S>(srgb_to_linear(sample_texture_uv<float>(sc, mi, m.diff_index, uvx, uvy, 0)));
    return b;
}
template <class S> inline S rough_primed(const Scene &sc, const Primed<S> &pr, u32 mi, float uvx, float uvy) {
    const phx_material &m = pr.mats[mi];
    S r = pr.rough[mi];
    if (m.metal_rough_index != NO_TEXTURE)
        r = r * S((double)sample_texture_uv<float>(sc, mi, m.metal_rough_index, uvx, uvy, 4).y);
    if (r < S((double)MIN_ROUGHNESS)) // clamp to [MIN_ROUGHNESS, 1] (a clamped value is constant)
        return S((double)MIN_ROUGHNESS);
    if (S(1.0) < r)
        return S(1.0);
    return r;
}

template <class S> inline S rough_ratio(double ch, double cv, double cl, double a0, S a1) {
    S r = ggx_ndf<S>(S(ch), a1) / S(ggx_ndf<double>(ch, a0));
    if (cv > 0.0)
        r = r * (smith_g1_ggx<S>(S(cv), a1) / S(smith_g1_ggx<double>(cv, a0)));
    if (cl > 0.0)
        r = r * (smith_g1_ggx<S>(S(cl), a1) / S(smith_g1_ggx<double>(cl, a0)));
    return r;
}

// W(θ') of a frozen BSDF bounce (sample_bsdf at θ0 gave bs from microfacet normal h)
template <class S>
inline V4<S> bounce_primed(const BsdfSample<float> &bs, V4<float> h, V4<float> view, V4<float> sn, float rough0,
                           S rough1, V4<S> base1) {
    if (bs.event == BSDF_DIFFUSE)
        return base1;
    const double a0 = (double)rough0 * rough0;
    const S a1 = rough1 * rough1;
    const V4<double> H = dd<double>(h), V = dd<double>(view), N = dd<double>(sn), L = dd<double>(bs.dir);
    const double ch = dot(N, H), cv = std::fabs(dot(V, N));
    const double cl = bs.event == BSDF_TRANSMIT ? std::fabs(dot(L, N)) : std::max(0.0, dot(L, N));
    const S w = S(smith_g1_ggx<double>(cl, a0)) * rough_ratio<S>(ch, cv, cl, a0, a1);
    if (bs.event == BSDF_METALLIC)
        return fresnel4<S>(base1, -dd<S>(view), dd<S>(h)) * w;
    if (bs.event == BSDF_TRANSMIT)
        return base1 * w;
    return mk<S>(w, w, w, S(0.0));
}

// shadow_transmittance<float> (θ0 decisions) and the same product at θ' in *out1
template <class S>
inline V4<float> shadow_tr(const Scene &sc, const Primed<S> &pr, V4<float> origin, V4<float> dir, float dist,
                           V4<S> *out1) {
    V4<float> trans = white4<float>();
    V4<S> t1 = white4<S>();
    float t_min = C<float>::EPS, t_max = dist - C<float>::EPS;
    for (u32 depth = 0; depth < MAX_RAY_BOUNCES; depth++) {
        HitRecord<float> rec;
        if (!scene_intersect<float>(sc, origin, dir, t_min, t_max, &rec))
            break;
        const phx_material &mat = sc.materials[rec.mat_index];
        if (mat.transmission < C<float>::EPS) {
            *out1 = zero4<S>();
            return zero4<float>();
        }
        V4<float> base = from<float>(mat.base_color);
        V4<S> b1 = pr.base[rec.mat_index];
        if (mat.diff_index != NO_TEXTURE) {
            SurfaceHit<float> sh = process_hit<float>(sc, rec, origin, dir);
            V4<float> tex = srgb_to_linear(sample_texture_uv<float>(sc, rec.mat_index, mat.diff_index, sh.uvx, sh.uvy, 0));
            base *= tex;
            b1 = b1 * dd<S>(tex);
        }
        if (mat.att_dist > C<float>::EPS) {
            V4<float> bl = beer_lambert<float>(from<float>(mat.att_color), mat.att_dist, rec.t - t_min);
            trans *= bl;
            t1 = t1 * dd<S>(bl);
        }
        trans *= base * mat.transmission;
        t1 = t1 * b1 * S((double)mat.transmission);
        if (dot(trans, trans) < C<float>::EPS) {
            *out1 = zero4<S>();
            return zero4<float>();
        }
        t_min = rec.t + C<float>::EPS;
    }
    *out1 = t1;
    return trans;
}

// sample_light_fragment<float> plus the index of the light it selected
inline bool light_fragment(Rng *rng, const Scene &sc, V4<float> pos, V4<float> normal, LightFragment<float> *f,
                           u32 *li) {
    Rng c = *rng;
    float scale;
    *li = select_light<float>(&c, sc, &scale);
    return sample_light_fragment<float>(rng, sc, pos, normal, f);
}

// direct_lighting_diffuse<float> and its value at θ' in *out1
template <class S>
inline V4<float> nee_diffuse(Rng *rng, const Scene &sc, const Primed<S> &pr, V4<float> pos, V4<float> normal,
                             V4<float> base, V4<S> base1, V4<S> *out1) {
    *out1 = zero4<S>();
    LightFragment<float> f;
    u32 li;
    if (!light_fragment(rng, sc, pos, normal, &f, &li))
        return zero4<float>();
    V4<S> tr1;
    V4<float> trans = shadow_tr<S>(sc, pr, pos, f.dir, f.dist, &tr1);
    *out1 = dd<S>(f.radiance) * light_ratio<S>(sc, pr, li) * (base1 / S((double)C<float>::PI)) * tr1;
    return f.radiance * (base / C<float>::PI) * trans;
}

// direct_lighting_specular<float> and its value at θ' (f0', roughness') in *out1
template <class S>
inline V4<float> nee_specular(Rng *rng, const Scene &sc, const Primed<S> &pr, V4<float> pos, V4<float> normal,
                              V4<float> view, V4<float> f0, float roughness, V4<S> f0_1, S rough1, V4<S> *out1) {
    *out1 = zero4<S>();
    float ndv = dot(view, normal);
    if (ndv < C<float>::EPS)
        return zero4<float>();
    LightFragment<float> f;
    u32 li;
    if (!light_fragment(rng, sc, pos, normal, &f, &li))
        return zero4<float>();
    if (f.n_dot_dir < C<float>::EPS)
        return zero4<float>();
    float alpha = roughness * roughness;
    V4<float> h = normalize(f.dir + view);
    float ndh = M<float>::fmax(dot(normal, h), 0.0f);
    float g = ggx_ndf(ndh, alpha);
    V4<float> fr = fresnel4(f0, view, h);
    float sm = smith_g1_ggx(f.n_dot_dir, alpha) * smith_g1_ggx(ndv, alpha);
    V4<float> spec = f.radiance * g * fr * sm / (4.0f * f.n_dot_dir * ndv);
    if (dot(spec, spec) < C<float>::EPS * C<float>::EPS)
        return zero4<float>();
    V4<S> tr1;
    V4<float> trans = shadow_tr<S>(sc, pr, pos, f.dir, f.dist, &tr1);
    const S a1 = rough1 * rough1;
    const double nl = f.n_dot_dir, nv = ndv;
    V4<S> spec1 = dd<S>(f.radiance) * light_ratio<S>(sc, pr, li) * ggx_ndf<S>(S((double)ndh), a1) *
                  fresnel4<S>(f0_1, dd<S>(view), dd<S>(h)) *
                  (smith_g1_ggx<S>(S(nl), a1) * smith_g1_ggx<S>(S(nv), a1) / S(4.0 * nl * nv));
    *out1 = spec1 * tr1;
    return spec * trans;
}

template <class S> struct HitPrimed {
    V4<S> throughput, base_color, direct, emission;
};

// trace_pixel<float> (identical result) with the θ' quantities of the same path in *p1
template <class S>
inline HitPoint<float> trace_pixel(const Scene &sc, const Primed<S> &pr, u32 width, u32 height, u32 seed,
                                   u32 direct_samples, u32 tid, HitPrimed<S> *p1) {
    u32 px = tid % width;
    u32 py = tid / width;
    Rng rng = pcg_seed(seed + tid);
    V4<float> origin, dir;
    make_ray<float>(sc.camera, px, py, width, height, &rng, &origin, &dir);
    V4<float> position = zero4<float>(), normal = zero4<float>(), throughput = white4<float>(),
              base_color = zero4<float>(), direct = zero4<float>(), emission = zero4<float>();
    V4<S> thr1 = white4<S>(), emi1 = zero4<S>(), dir1 = zero4<S>(), base_out1 = zero4<S>();
    IorStack<float> ior;
    init_ior_stack<float>(&ior, AIR_IOR);
    for (i32 depth = 0; depth < (i32)MAX_RAY_BOUNCES; depth++) {
        HitRecord<float> rec;
        bool hit = scene_intersect<float>(sc, origin, dir, C<float>::EPS, C<float>::INF, &rec);
        if (!hit) {
            if (sc.has_envmap) {
                V4<float> env = sample_envmap<float>(sc, dir);
                emission += throughput * env;
                emi1 += thr1 * dd<S>(env);
            }
            break;
        }
        SurfaceHit<float> sh = process_hit<float>(sc, rec, origin, dir);
        const phx_material &mat = sc.materials[sh.mat_index];
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > C<float>::EPS && mat.att_dist > C<float>::EPS) {
            V4<float> vol = beer_lambert<float>(from<float>(mat.att_color), mat.att_dist, sh.t);
            throughput *= vol;
            thr1 = thr1 * dd<S>(vol);
        }
        float bw = 1.0f - rec.u - rec.v;
        const phx_triangle &tr = sc.tris[sh.tri_index];
        V4<float> traw = bw * from<float>(tr.t0) + rec.u * from<float>(tr.t1) + rec.v * from<float>(tr.t2);
        V4<float> braw = (length(traw) > C<float>::EPS) ? cross(sh.normal, traw) : zero4<float>();
        V4<float> tangent, bitangent;
        if (length(braw) > C<float>::EPS) {
            bitangent = normalize(braw);
            tangent = cross(bitangent, sh.normal);
        } else {
            make_tbn(sh.normal, &tangent, &bitangent);
        }
        ShadingContext<float> ctx =
            evaluate_material<float>(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        const V4<S> base1 = base_primed<S>(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        const S rough1 = rough_primed<S>(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        emission += throughput * ctx.emissive;
        emi1 += thr1 * dd<S>(ctx.emissive);
        V4<float> view = -dir;
        Rng peek = rng; // sample_bsdf draws the microfacet normal first
        V4<float> h = ggx_sample_vndf<float>(&peek, ctx.shading_normal, sh.normal, view, ctx.roughness);
        BsdfSample<float> bs = sample_bsdf<float>(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE) {
            V4<float> sum = zero4<float>();
            V4<S> sum1 = zero4<S>();
            for (u32 d = 0; d < direct_samples; d++) {
                V4<S> v1;
                sum += nee_diffuse<S>(&rng, sc, pr, sh.position, ctx.shading_normal, ctx.base_color, base1, &v1);
                sum1 += v1;
            }
            emission = mk<float>(emission.x, emission.y, emission.z, 1.0f);
            position = sh.position;
            normal = sh.normal;
            base_color = ctx.base_color;
            base_out1 = base1;
            direct = throughput * ctx.occlusion * (sum / (float)direct_samples);
            dir1 = thr1 * S((double)ctx.occlusion) * (sum1 / S((double)direct_samples));
            break;
        }
        if (bs.event == BSDF_METALLIC || bs.event == BSDF_FRESNEL) {
            V4<float> f0 = ctx.base_color;
            V4<S> f0_1 = base1;
            if (bs.event == BSDF_FRESNEL) {
                float ratio = (cur - ctx.ior) / (cur + ctx.ior);
                float r0 = ratio * ratio;
                f0 = mk<float>(r0, r0, r0, 0.0f);
                f0_1 = dd<S>(f0);
            }
            V4<float> sum = zero4<float>();
            V4<S> sum1 = zero4<S>();
            for (u32 d = 0; d < direct_samples; d++) {
                V4<S> v1;
                sum += nee_specular<S>(&rng, sc, pr, sh.position, ctx.shading_normal, view, f0, ctx.roughness, f0_1,
                                       rough1, &v1);
                sum1 += v1;
            }
            emission += throughput * (sum / (float)direct_samples);
            emi1 += thr1 * (sum1 / S((double)direct_samples));
        }
        throughput *= bs.throughput;
        thr1 = thr1 * bounce_primed<S>(bs, h, view, ctx.shading_normal, ctx.roughness, rough1, base1);
        if ((u32)depth >= RR_MIN_RAY_DEPTH) {
            float q = M<float>::fmax(throughput.x, M<float>::fmax(throughput.y, throughput.z));
            q = clampr<float>(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float<float>(&rng) > q)
                break;
            throughput *= 1.0f / q;
            thr1 = thr1 * S((double)(1.0f / q));
        }
        V4<float> side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * C<float>::EPS + side * C<float>::EPS;
        dir = bs.dir;
    }
    HitPoint<float> hp;
    hp.emission = emission;
    hp.pos = position;
    hp.normal = normal;
    hp.throughput = throughput;
    hp.base_color = base_color;
    hp.direct = direct;
    p1->throughput = thr1;
    p1->base_color = base_out1;
    p1->direct = dir1;
    p1->emission = emi1;
    return hp;
}

// emit_photon<float> (identical stored photons) with each stored photon's power at θ' in pow1
template <class S>
inline u32 emit_photon(const Scene &sc, const Primed<S> &pr, u32 tid, u32 max_bounces, u32 seed,
                       StoredPhoton<float> *out, V4<S> *pow1) {
    u32 n_out = 0;
    Rng rng = pcg_seed(seed + tid);
    V4<float> origin, dir, power;
    Rng peek = rng; // sample_light selects the light first
    float scale;
    const u32 li = select_light<float>(&peek, sc, &scale);
    sample_light<float>(&rng, sc, &origin, &dir, &power);
    V4<S> p1 = dd<S>(power) * light_ratio<S>(sc, pr, li);
    IorStack<float> ior;
    init_ior_stack<float>(&ior, AIR_IOR);
    V4<float> throughput = mk<float>(1, 1, 1, 0);
    for (u32 depth = 0; depth < max_bounces; depth++) {
        HitRecord<float> rec;
        bool hit = scene_intersect<float>(sc, origin, dir, C<float>::EPS, C<float>::INF, &rec);
        if (!hit)
            return n_out;
        SurfaceHit<float> sh = process_hit<float>(sc, rec, origin, dir);
        const phx_material &mat = sc.materials[sh.mat_index];
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > C<float>::EPS && mat.att_dist > C<float>::EPS) {
            V4<float> vol = beer_lambert<float>(from<float>(mat.att_color), mat.att_dist, sh.t);
            power *= vol;
            throughput *= vol;
            p1 = p1 * dd<S>(vol);
        }
        float bw = 1.0f - rec.u - rec.v;
        const phx_triangle &tr = sc.tris[sh.tri_index];
        V4<float> traw = bw * from<float>(tr.t0) + rec.u * from<float>(tr.t1) + rec.v * from<float>(tr.t2);
        V4<float> braw = (length(traw) > C<float>::EPS) ? cross(sh.normal, traw) : zero4<float>();
        V4<float> tangent, bitangent;
        if (length(braw) > C<float>::EPS) {
            bitangent = normalize(braw);
            tangent = cross(bitangent, sh.normal);
        } else {
            make_tbn(sh.normal, &tangent, &bitangent);
        }
        ShadingContext<float> ctx =
            evaluate_material<float>(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        if (depth >= RR_MIN_PHOTON_DEPTH) {
            float q = M<float>::fmax(throughput.x, M<float>::fmax(throughput.y, throughput.z));
            q = clampr<float>(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float<float>(&rng) > q)
                return n_out;
            float inv_q = 1.0f / q;
            throughput *= inv_q;
            power *= inv_q;
            p1 = p1 * S((double)inv_q);
        }
        const V4<S> base1 = base_primed<S>(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        const S rough1 = rough_primed<S>(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        V4<float> view = -dir;
        Rng peek2 = rng;
        V4<float> h = ggx_sample_vndf<float>(&peek2, ctx.shading_normal, sh.normal, view, ctx.roughness);
        BsdfSample<float> bs = sample_bsdf<float>(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE && dot(dir, sh.normal) < 0.0f) {
            out[n_out].pos = sh.position;
            out[n_out].power = encode_rgbe<float>(power);
            out[n_out].dir = encode_oct<float>(dir);
            pow1[n_out] = p1;
            n_out++;
        }
        power *= bs.throughput;
        throughput *= bs.throughput;
        p1 = p1 * bounce_primed<S>(bs, h, view, ctx.shading_normal, ctx.roughness, rough1, base1);
        V4<float> side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * C<float>::EPS + side * C<float>::EPS;
        dir = bs.dir;
    }
    return n_out;
}

// gather_pixel<float> (identical float state) and the θ' flux / radiance of the same pixel
template <class S>
inline void gather_pixel(const HitPoint<float> &hp, const HitPrimed<S> &p1, const phx_photon_hash_data &d,
                         const u32 *cell_start, const u32 *cell_end, const V4<float> *ph_pos, const u32 *ph_power,
                         const u32 *ph_dir, const V4<S> *ph_pow1, float alpha, V4<float> *flux, float *weight,
                         V4<float> *radiance, V4<S> *flux1, V4<S> *rad1) {
    V4<float> ge = hp.emission;
    V4<float> rso = *radiance;
    V4<float> r = mk<float>(ge.x, ge.y, ge.z, 0.0f);
    V4<S> e1 = p1.emission;
    e1.w = S(0.0);
    if (ge.w == 0.0f) {
        *radiance = rso + r;
        *rad1 += e1;
        return;
    }
    V4<float> direct = hp.direct;
    r.x += direct.x;
    r.y += direct.y;
    r.z += direct.z;
    *radiance = rso + r;
    V4<S> d1 = p1.direct;
    d1.w = S(0.0);
    *rad1 += e1 + d1;
    V4<float> fso = *flux;
    float wso = *weight;
    float r_sq = fso.w;
    if (r_sq < C<float>::EPS) {
        float hx = d.cell_sizes.x * 0.5f;
        float hy = d.cell_sizes.y * 0.5f;
        float hz = d.cell_sizes.z * 0.5f;
        r_sq = hx * hx + hy * hy + hz * hz;
    }
    V4<float> nf;
    float found;
    gather_photon_flux<float>(hp.pos, hp.normal, d, cell_start, cell_end, ph_pos, ph_power, ph_dir, r_sq, &nf,
                              &found);
    if (found > 0.0f) {
        V4<S> nf1 = zero4<S>(); // the same neighbourhood and kernel weights, θ' power
        for (u32 i = 0; i < 27; i++) {
            V4<float> p2 = hp.pos;
            p2.x += (float)((i32)(i % 3) - 1) * d.cell_sizes.x;
            p2.y += (float)((i32)((i / 3) % 3) - 1) * d.cell_sizes.y;
            p2.z += (float)((i32)((i / 9) % 3) - 1) * d.cell_sizes.z;
            u32 hsh = get_hash<float>(p2, d);
            if (hsh == 0)
                continue;
            for (u32 k = cell_start[hsh]; k < cell_end[hsh]; k++) {
                V4<float> dd4 = hp.pos - ph_pos[k];
                float dsq = dot(dd4, dd4);
                if (dsq >= r_sq)
                    continue;
                if (dot(decode_oct<float>(ph_dir[k]), hp.normal) > 0.0f)
                    continue;
                float w = GAUSS_ALPHA * (1.0f - (1.0f - M<float>::exp(-GAUSS_BETA * dsq / (2.0f * r_sq))) / GAUSS_DENOM);
                nf1 += S((double)w) * ph_pow1[k];
            }
        }
        float nw = wso + alpha * found;
        float ratio = nw / (wso + found);
        float nr = r_sq * ratio;
        V4<float> contribution = hp.throughput * (hp.base_color / C<float>::PI) * nf;
        V4<float> temp = (fso + contribution) * ratio;
        *flux = mk<float>(temp.x, temp.y, temp.z, nr);
        *weight = nw;
        V4<S> c1 = p1.throughput * (p1.base_color / S((double)C<float>::PI)) * nf1;
        c1.w = S(0.0);
        *flux1 = (*flux1 + c1) * S((double)ratio);
    }
}

} // namespace frozen
} // namespace orc
