// phx_frozen.hpp — TEST INFRASTRUCTURE ONLY (part of the oracle): the frozen-path SPPM estimator
// F(θ') that the library's adjoint differentiates, evaluated in double so that central finite
// differences of it give the reference gradient.  Never linked into the product.
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

#include "phx_oracle.hpp"

namespace orc {
namespace frozen {

using D4 = V4<double>;
inline D4 dd(const V4<float> &v) { return mk<double>(v.x, v.y, v.z, v.w); }
inline D4 dd(const phx_f4 &v) { return mk<double>(v.x, v.y, v.z, v.w); }

struct Primed {
    const phx_material *mats; // θ' materials (the scene's count and order)
    const phx_light *lights;  // θ' lights
};

// L'/L0 per channel for light li (0 where the θ0 power is 0)
inline D4 light_ratio(const Scene &sc, const Primed &pr, u32 li) {
    if (sc.n_lights == 0)
        return zero4<double>();
    const phx_f4 &a = sc.lights[li].power, &b = pr.lights[li].power;
    return mk<double>(a.x != 0.0f ? (double)b.x / a.x : 0.0, a.y != 0.0f ? (double)b.y / a.y : 0.0,
                      a.z != 0.0f ? (double)b.z / a.z : 0.0, 0.0);
}

// base colour and roughness of material mi at θ', with the same texture factors as θ0
inline D4 base_primed(const Scene &sc, const Primed &pr, u32 mi, float uvx, float uvy) {
    const phx_material &m = pr.mats[mi];
    D4 b = dd(m.base_color);
    if (m.diff_index != NO_TEXTURE)
        b = b * dd(srgb_to_linear(sample_texture_uv<float>(sc, mi, m.diff_index, uvx, uvy, 0)));
    return b;
}
inline double rough_primed(const Scene &sc, const Primed &pr, u32 mi, float uvx, float uvy) {
    const phx_material &m = pr.mats[mi];
    double r = m.roughness;
    if (m.metal_rough_index != NO_TEXTURE)
        r *= (double)sample_texture_uv<float>(sc, mi, m.metal_rough_index, uvx, uvy, 4).y;
    return std::min(std::max(r, (double)MIN_ROUGHNESS), 1.0);
}

inline double rough_ratio(double ch, double cv, double cl, double a0, double a1) {
    double r = ggx_ndf<double>(ch, a1) / ggx_ndf<double>(ch, a0);
    if (cv > 0.0)
        r *= smith_g1_ggx<double>(cv, a1) / smith_g1_ggx<double>(cv, a0);
    if (cl > 0.0)
        r *= smith_g1_ggx<double>(cl, a1) / smith_g1_ggx<double>(cl, a0);
    return r;
}

// W(θ') of a frozen BSDF bounce (sample_bsdf at θ0 gave bs from microfacet normal h)
inline D4 bounce_primed(const BsdfSample<float> &bs, V4<float> h, V4<float> view, V4<float> sn, float rough0,
                        double rough1, D4 base1) {
    if (bs.event == BSDF_DIFFUSE)
        return base1;
    const double a0 = (double)rough0 * rough0, a1 = rough1 * rough1;
    const D4 H = dd(h), V = dd(view), N = dd(sn), L = dd(bs.dir);
    const double ch = dot(N, H), cv = std::fabs(dot(V, N));
    const double cl = bs.event == BSDF_TRANSMIT ? std::fabs(dot(L, N)) : std::max(0.0, dot(L, N));
    const double w = smith_g1_ggx<double>(cl, a0) * rough_ratio(ch, cv, cl, a0, a1);
    if (bs.event == BSDF_METALLIC)
        return fresnel4<double>(base1, -V, H) * w;
    if (bs.event == BSDF_TRANSMIT)
        return base1 * w;
    return mk<double>(w, w, w, 0.0);
}

// shadow_transmittance<float> (θ0 decisions) and the same product at θ' in *out1
inline V4<float> shadow_tr(const Scene &sc, const Primed &pr, V4<float> origin, V4<float> dir, float dist,
                           D4 *out1) {
    V4<float> trans = white4<float>();
    D4 t1 = white4<double>();
    float t_min = C<float>::EPS, t_max = dist - C<float>::EPS;
    for (u32 depth = 0; depth < MAX_RAY_BOUNCES; depth++) {
        HitRecord<float> rec;
        if (!scene_intersect<float>(sc, origin, dir, t_min, t_max, &rec))
            break;
        const phx_material &mat = sc.materials[rec.mat_index];
        if (mat.transmission < C<float>::EPS) {
            *out1 = zero4<double>();
            return zero4<float>();
        }
        V4<float> base = from<float>(mat.base_color);
        D4 b1 = dd(pr.mats[rec.mat_index].base_color);
        if (mat.diff_index != NO_TEXTURE) {
            SurfaceHit<float> sh = process_hit<float>(sc, rec, origin, dir);
            V4<float> tex = srgb_to_linear(sample_texture_uv<float>(sc, rec.mat_index, mat.diff_index, sh.uvx, sh.uvy, 0));
            base *= tex;
            b1 = b1 * dd(tex);
        }
        if (mat.att_dist > C<float>::EPS) {
            V4<float> bl = beer_lambert<float>(from<float>(mat.att_color), mat.att_dist, rec.t - t_min);
            trans *= bl;
            t1 = t1 * dd(bl);
        }
        trans *= base * mat.transmission;
        t1 = t1 * b1 * (double)mat.transmission;
        if (dot(trans, trans) < C<float>::EPS) {
            *out1 = zero4<double>();
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
inline V4<float> nee_diffuse(Rng *rng, const Scene &sc, const Primed &pr, V4<float> pos, V4<float> normal,
                             V4<float> base, D4 base1, D4 *out1) {
    *out1 = zero4<double>();
    LightFragment<float> f;
    u32 li;
    if (!light_fragment(rng, sc, pos, normal, &f, &li))
        return zero4<float>();
    D4 tr1;
    V4<float> trans = shadow_tr(sc, pr, pos, f.dir, f.dist, &tr1);
    *out1 = dd(f.radiance) * light_ratio(sc, pr, li) * (base1 / (double)C<float>::PI) * tr1;
    return f.radiance * (base / C<float>::PI) * trans;
}

// direct_lighting_specular<float> and its value at θ' (f0', roughness') in *out1
inline V4<float> nee_specular(Rng *rng, const Scene &sc, const Primed &pr, V4<float> pos, V4<float> normal,
                              V4<float> view, V4<float> f0, float roughness, D4 f0_1, double rough1, D4 *out1) {
    *out1 = zero4<double>();
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
    D4 tr1;
    V4<float> trans = shadow_tr(sc, pr, pos, f.dir, f.dist, &tr1);
    const double a1 = rough1 * rough1, nl = f.n_dot_dir, nv = ndv;
    D4 spec1 = dd(f.radiance) * light_ratio(sc, pr, li) * ggx_ndf<double>((double)ndh, a1) *
               fresnel4<double>(f0_1, dd(view), dd(h)) *
               (smith_g1_ggx<double>(nl, a1) * smith_g1_ggx<double>(nv, a1) / (4.0 * nl * nv));
    *out1 = spec1 * tr1;
    return spec * trans;
}

struct HitPrimed {
    D4 throughput, base_color, direct, emission;
};

// trace_pixel<float> (identical result) with the θ' quantities of the same path in *p1
inline HitPoint<float> trace_pixel(const Scene &sc, const Primed &pr, u32 width, u32 height, u32 seed,
                                   u32 direct_samples, u32 tid, HitPrimed *p1) {
    u32 px = tid % width;
    u32 py = tid / width;
    Rng rng = pcg_seed(seed + tid);
    V4<float> origin, dir;
    make_ray<float>(sc.camera, px, py, width, height, &rng, &origin, &dir);
    V4<float> position = zero4<float>(), normal = zero4<float>(), throughput = white4<float>(),
              base_color = zero4<float>(), direct = zero4<float>(), emission = zero4<float>();
    D4 thr1 = white4<double>(), emi1 = zero4<double>(), dir1 = zero4<double>(), base_out1 = zero4<double>();
    IorStack<float> ior;
    init_ior_stack<float>(&ior, AIR_IOR);
    for (i32 depth = 0; depth < (i32)MAX_RAY_BOUNCES; depth++) {
        HitRecord<float> rec;
        bool hit = scene_intersect<float>(sc, origin, dir, C<float>::EPS, C<float>::INF, &rec);
        if (!hit) {
            if (sc.has_envmap) {
                V4<float> env = sample_envmap<float>(sc, dir);
                emission += throughput * env;
                emi1 += thr1 * dd(env);
            }
            break;
        }
        SurfaceHit<float> sh = process_hit<float>(sc, rec, origin, dir);
        const phx_material &mat = sc.materials[sh.mat_index];
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > C<float>::EPS && mat.att_dist > C<float>::EPS) {
            V4<float> vol = beer_lambert<float>(from<float>(mat.att_color), mat.att_dist, sh.t);
            throughput *= vol;
            thr1 = thr1 * dd(vol);
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
        const D4 base1 = base_primed(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        const double rough1 = rough_primed(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        emission += throughput * ctx.emissive;
        emi1 += thr1 * dd(ctx.emissive);
        V4<float> view = -dir;
        Rng peek = rng; // sample_bsdf draws the microfacet normal first
        V4<float> h = ggx_sample_vndf<float>(&peek, ctx.shading_normal, sh.normal, view, ctx.roughness);
        BsdfSample<float> bs = sample_bsdf<float>(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE) {
            V4<float> sum = zero4<float>();
            D4 sum1 = zero4<double>();
            for (u32 d = 0; d < direct_samples; d++) {
                D4 v1;
                sum += nee_diffuse(&rng, sc, pr, sh.position, ctx.shading_normal, ctx.base_color, base1, &v1);
                sum1 += v1;
            }
            emission = mk<float>(emission.x, emission.y, emission.z, 1.0f);
            position = sh.position;
            normal = sh.normal;
            base_color = ctx.base_color;
            base_out1 = base1;
            direct = throughput * ctx.occlusion * (sum / (float)direct_samples);
            dir1 = thr1 * (double)ctx.occlusion * (sum1 / (double)direct_samples);
            break;
        }
        if (bs.event == BSDF_METALLIC || bs.event == BSDF_FRESNEL) {
            V4<float> f0 = ctx.base_color;
            D4 f0_1 = base1;
            if (bs.event == BSDF_FRESNEL) {
                float ratio = (cur - ctx.ior) / (cur + ctx.ior);
                float r0 = ratio * ratio;
                f0 = mk<float>(r0, r0, r0, 0.0f);
                f0_1 = dd(f0);
            }
            V4<float> sum = zero4<float>();
            D4 sum1 = zero4<double>();
            for (u32 d = 0; d < direct_samples; d++) {
                D4 v1;
                sum += nee_specular(&rng, sc, pr, sh.position, ctx.shading_normal, view, f0, ctx.roughness, f0_1,
                                    rough1, &v1);
                sum1 += v1;
            }
            emission += throughput * (sum / (float)direct_samples);
            emi1 += thr1 * (sum1 / (double)direct_samples);
        }
        throughput *= bs.throughput;
        thr1 = thr1 * bounce_primed(bs, h, view, ctx.shading_normal, ctx.roughness, rough1, base1);
        if ((u32)depth >= RR_MIN_RAY_DEPTH) {
            float q = M<float>::fmax(throughput.x, M<float>::fmax(throughput.y, throughput.z));
            q = clampr<float>(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float<float>(&rng) > q)
                break;
            throughput *= 1.0f / q;
            thr1 = thr1 * (double)(1.0f / q);
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
inline u32 emit_photon(const Scene &sc, const Primed &pr, u32 tid, u32 max_bounces, u32 seed,
                       StoredPhoton<float> *out, D4 *pow1) {
    u32 n_out = 0;
    Rng rng = pcg_seed(seed + tid);
    V4<float> origin, dir, power;
    Rng peek = rng; // sample_light selects the light first
    float scale;
    const u32 li = select_light<float>(&peek, sc, &scale);
    sample_light<float>(&rng, sc, &origin, &dir, &power);
    D4 p1 = dd(power) * light_ratio(sc, pr, li);
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
            p1 = p1 * dd(vol);
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
            p1 = p1 * (double)inv_q;
        }
        const D4 base1 = base_primed(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
        const double rough1 = rough_primed(sc, pr, sh.mat_index, sh.uvx, sh.uvy);
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
        p1 = p1 * bounce_primed(bs, h, view, ctx.shading_normal, ctx.roughness, rough1, base1);
        V4<float> side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * C<float>::EPS + side * C<float>::EPS;
        dir = bs.dir;
    }
    return n_out;
}

// gather_pixel<float> (identical float state) and the θ' flux / radiance of the same pixel
inline void gather_pixel(const HitPoint<float> &hp, const HitPrimed &p1, const phx_photon_hash_data &d,
                         const u32 *cell_start, const u32 *cell_end, const V4<float> *ph_pos, const u32 *ph_power,
                         const u32 *ph_dir, const D4 *ph_pow1, float alpha, V4<float> *flux, float *weight,
                         V4<float> *radiance, D4 *flux1, D4 *rad1) {
    V4<float> ge = hp.emission;
    V4<float> rso = *radiance;
    V4<float> r = mk<float>(ge.x, ge.y, ge.z, 0.0f);
    D4 e1 = p1.emission;
    e1.w = 0.0;
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
    D4 d1 = p1.direct;
    d1.w = 0.0;
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
        D4 nf1 = zero4<double>(); // the same neighbourhood and kernel weights, θ' power
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
                nf1 += (double)w * ph_pow1[k];
            }
        }
        float nw = wso + alpha * found;
        float ratio = nw / (wso + found);
        float nr = r_sq * ratio;
        V4<float> contribution = hp.throughput * (hp.base_color / C<float>::PI) * nf;
        V4<float> temp = (fso + contribution) * ratio;
        *flux = mk<float>(temp.x, temp.y, temp.z, nr);
        *weight = nw;
        D4 c1 = p1.throughput * (p1.base_color / (double)C<float>::PI) * nf1;
        c1.w = 0.0;
        *flux1 = (*flux1 + c1) * (double)ratio;
    }
}

} // namespace frozen
} // namespace orc
