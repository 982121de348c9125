// k_adjoint.cu — reverse-mode derivative of the SPPM image with respect to per-material base
// colour and roughness and per-light power: the adjoint of gather_flux (gather_flux.cl:5-78) and of
// the BSDF / direct-lighting weights (shading.h:150-213, bsdfs.h:77-121, light_sampling.h:302-390)
// along camera and photon paths replayed from their RNG seeds.  No counterpart in the reference.
//
// What is differentiated is the frozen-path estimator: every random or discrete choice of the
// forward render stays fixed — paths, BSDF events, microfacet normals, Russian-roulette factors,
// light-selection probabilities, shadow-ray hit lists, gather neighbourhoods, kernel weights,
// radii and SPPM ratios — and only the weights depend on the parameters.  A BSDF bounce with
// frozen directions has weight W(θ0)·f(θ)/f(θ0) (detached sampling), so
//   d log W / d base_c     = 1/base_c (diffuse, transmission; base = material base × texture)
//                          = (1-p)·base_c/(mb_c·F_c) (metal, Schlick F = base + (1-base)·p)
//   d log W / d roughness  = (d log D(h) + d log G1(v) + d log G1(l)) / dα · dα/d roughness,
// with α = roughness² and roughness = clamp(mb_rough × texture, 0.001, 1).  Light power enters
// linearly; photon power is carried unquantised.  The oracle's frozen estimator
// (oracle/phx_frozen.hpp) evaluates exactly this function in double for the finite-difference
// checks.
//
// The image is I = radiance/R + flux.xyz/(π r_R² N) with flux_R = Σ_n c_n Π_{m>=n} ratio_m
// (ratio 1 in a round without photons), so dI/dc_n = K_n = Π_{m>=n} ratio_m / (π r_R² N).
// Per round n of the backward pass (hit points and photons re-created by the ordinary kernels):
//   k_gather_adj  a = dL/dI·K_n, S = Σ w_k Φ_k over the round's neighbourhood:
//                 dL/dT = a·A/π·S, dL/dA = a·T/π·S, dL/dΦ_k += w_k·a·T·A/π (float atomics)
//   k_trace_adj   replays the camera path with inline NEE and adds, for every term X it produces
//                 with adjoint u (emission and direct light: dL/dI/R; final throughput: dL/dT;
//                 base colour: dL/dA), Σ_c u_c X_c · d log X_c/dθ
//   k_emit_adj    replays the photon path; at stored photon k, u = dL/dΦ_k ⊙ Φ_k times
//                 d log Φ_k/dθ (the bounces before the store and 1/L of its light)
// Gradients are summed per block in shared memory (float) and then into doubles.
#include "dev_shading.cuh"
#include "kernels.hpp"

namespace phx {

// ---- gradient accumulation ---------------------------------------------------------------------
struct GradAcc {
    float *sm;  // per-block partial sums (nullptr: straight to global)
    double *gl;
    PHX_DI void add(u32 i, float v) const {
        if (v == 0.0f)
            return;
        if (sm)
            atomicAdd(&sm[i], v);
        else
            atomicAdd(&gl[i], (double)v);
    }
};

PHX_DI GradAcc grad_begin(const AdjBufs &ab, float *smem) {
    GradAcc g{ab.block_sums ? smem : nullptr, ab.grad};
    if (g.sm) {
        for (u32 i = threadIdx.x; i < ab.n_params; i += blockDim.x)
            g.sm[i] = 0.0f;
        __syncthreads();
    }
    return g;
}
PHX_DI void grad_end(const AdjBufs &ab, const GradAcc &g) {
    if (!g.sm)
        return;
    __syncthreads();
    for (u32 i = threadIdx.x; i < ab.n_params; i += blockDim.x)
        if (g.sm[i] != 0.0f)
            atomicAdd(&ab.grad[i], (double)g.sm[i]);
}

// ---- log-derivatives of the weights ------------------------------------------------------------
PHX_DI float dlog_ndf(float c, float a) { // d log D(c; α) / dα, D = α²/max(π d², EPS) (bsdfs.h:117-121)
    float a2 = a * a;
    float d = c * c * (a2 - 1.0f) + 1.0f;
    if (PI * d * d <= EPS)
        return 2.0f / a;
    return 2.0f / a - 4.0f * a * c * c / d;
}
PHX_DI float dlog_g1(float c, float a) { // d log G1(c; α) / dα (bsdfs.h:77-83); 0 where G1 = 0
    if (c <= 0.0f)
        return 0.0f;
    float a2 = a * a;
    float s = sqrtf(a2 + (1.0f - a2) * c * c);
    return -a * (1.0f - c * c) / (s * (c + s));
}
PHX_DI float4 inv_nonzero(float4 v) {
    return f4(v.x != 0.0f ? 1.0f / v.x : 0.0f, v.y != 0.0f ? 1.0f / v.y : 0.0f, v.z != 0.0f ? 1.0f / v.z : 0.0f,
              0.0f);
}
// dα / d(material roughness) where the clamp is inactive: α = r², r = mb_r·t  =>  2r·t = 2r²/mb_r
PHX_DI float dalpha_drough(float r, float mb_r) {
    return (r > MIN_ROUGHNESS && r < 1.0f && mb_r > 0.0f) ? 2.0f * r * r / mb_r : 0.0f;
}

// d log W of one bounce: per base colour channel of its material, and per material roughness
struct BounceRec {
    u32 mat;
    float db0, db1, db2, dr;
};

PHX_DI BounceRec bounce_dlog(const BsdfSample &bs, float4 h, float4 view, float4 sn, const ShadingContext &ctx,
                             const phx_material &mat, u32 mi) {
    BounceRec r{mi, 0.0f, 0.0f, 0.0f, 0.0f};
    const float4 imb = inv_nonzero(f4(mat.base_color));
    if (bs.event == BSDF_DIFFUSE || bs.event == BSDF_TRANSMIT) {
        r.db0 = imb.x;
        r.db1 = imb.y;
        r.db2 = imb.z;
    } else if (bs.event == BSDF_METALLIC) {
        const float p = pm_powf(1.0f - fabsf(dot(-view, h)), 5.0f);
        const float4 b = ctx.base_color;
        const float fx = b.x + (1.0f - b.x) * p, fy = b.y + (1.0f - b.y) * p, fz = b.z + (1.0f - b.z) * p;
        r.db0 = fx != 0.0f ? (1.0f - p) * b.x * imb.x / fx : 0.0f;
        r.db1 = fy != 0.0f ? (1.0f - p) * b.y * imb.y / fy : 0.0f;
        r.db2 = fz != 0.0f ? (1.0f - p) * b.z * imb.z / fz : 0.0f;
    }
    if (bs.event != BSDF_DIFFUSE) {
        const float a = ctx.roughness * ctx.roughness;
        const float ch = dot(sn, h), cv = fabsf(dot(view, sn));
        const float cl = bs.event == BSDF_TRANSMIT ? fabsf(dot(bs.dir, sn)) : fmaxf(0.0f, dot(bs.dir, sn));
        r.dr = (dlog_ndf(ch, a) + dlog_g1(cv, a) + dlog_g1(cl, a)) * dalpha_drough(ctx.roughness, mat.roughness);
    }
    return r;
}

// Adds Σ_c z_c · d log W_i,c/dθ for every recorded bounce i (z = u ⊙ X of a term X that carries
// the product of those bounce weights).
PHX_DI void add_prefix(const GradAcc &acc, const BounceRec *br, u32 nb, float4 z) {
    if (z.x == 0.0f && z.y == 0.0f && z.z == 0.0f)
        return;
    const float zs = z.x + z.y + z.z;
    for (u32 i = 0; i < nb; i++) {
        const u32 o = 4 * br[i].mat;
        acc.add(o + 0, z.x * br[i].db0);
        acc.add(o + 1, z.y * br[i].db1);
        acc.add(o + 2, z.z * br[i].db2);
        acc.add(o + 3, zs * br[i].dr);
    }
}

// ---- direct lighting with the pieces the adjoint needs -----------------------------------------
struct NeeRec {
    u32 light;          // selected light
    u32 n_occ;          // transmissive occluders on the shadow ray
    u32 occ[MAX_RAY_BOUNCES];
    float dlog_a;       // specular: d log (D G1 G1) / dα
    float4 dlog_f0;     // specular: d log F_c / d f0_c (f0 = base: metal)
};

// shadow_transmittance (light_sampling.h:302-333) recording the transmissive occluders
PHX_DI float4 shadow_tr_rec(const SceneDesc &sc, float4 origin, float4 dir, float dist, u32 *overflow, NeeRec *nr) {
    float4 trans = white4();
    float t_min = EPS, t_max = dist - EPS;
    nr->n_occ = 0;
    for (u32 depth = 0; depth < MAX_RAY_BOUNCES; depth++) {
        Hit h;
        if (!intersect(sc, origin, dir, t_min, t_max, &h, overflow, sc.any_transmissive == 0))
            break;
        u32 mi = tri_mat(sc, h.tri);
        const phx_material &mat = sc.materials[mi];
        if (mat.transmission < EPS)
            return zero4();
        float4 base = f4(mat.base_color);
        if (mat.diff_index != NO_TEXTURE) {
            SurfaceHit s = process_hit(sc, h, origin, dir);
            base *= srgb_to_linear(sample_texture_uv(sc, mi, mat.diff_index, s.uvx, s.uvy, 0));
        }
        if (mat.att_dist > EPS)
            trans *= beer_lambert(f4(mat.att_color), mat.att_dist, h.t - t_min);
        trans *= base * mat.transmission;
        if (dot(trans, trans) < EPS)
            return zero4();
        nr->occ[nr->n_occ++] = mi;
        t_min = h.t + EPS;
    }
    return trans;
}

PHX_DI u32 peek_light(const Rng *rng, const SceneDesc &sc) {
    Rng c = *rng;
    float scale;
    return select_light(&c, sc, &scale);
}

// direct_lighting_diffuse (light_sampling.h:335-353)
PHX_DI float4 nee_diffuse_adj(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, float4 base, u32 *overflow,
                              NeeRec *nr) {
    nr->light = peek_light(rng, sc);
    nr->n_occ = 0;
    LightFragment f;
    if (!sample_light_fragment(rng, sc, pos, normal, &f))
        return zero4();
    float4 trans = shadow_tr_rec(sc, pos, f.dir, f.dist, overflow, nr);
    return f.radiance * (base / PI) * trans;
}

// direct_lighting_specular (light_sampling.h:355-390)
PHX_DI float4 nee_specular_adj(Rng *rng, const SceneDesc &sc, float4 pos, float4 normal, float4 view, float4 f0,
                               float roughness, u32 *overflow, NeeRec *nr) {
    nr->n_occ = 0;
    nr->light = 0;
    float ndv = dot(view, normal);
    if (ndv < EPS)
        return zero4();
    nr->light = peek_light(rng, sc);
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
    float4 trans = shadow_tr_rec(sc, pos, f.dir, f.dist, overflow, nr);
    nr->dlog_a = dlog_ndf(ndh, alpha) + dlog_g1(f.n_dot_dir, alpha) + dlog_g1(ndv, alpha);
    const float p = pm_powf(1.0f - fabsf(dot(view, h)), 5.0f);
    nr->dlog_f0 = f4(fr.x != 0.0f ? (1.0f - p) / fr.x : 0.0f, fr.y != 0.0f ? (1.0f - p) / fr.y : 0.0f,
                     fr.z != 0.0f ? (1.0f - p) / fr.z : 0.0f, 0.0f);
    return spec * trans;
}

// per-sample derivatives of a NEE term z = u ⊙ X: its light and its transmissive occluders
PHX_DI void add_nee_common(const SceneDesc &sc, const AdjBufs &ab, const GradAcc &acc, const NeeRec &nr, float4 z) {
    if (sc.n_lights > 0) {
        const float4 il = inv_nonzero(f4(sc.lights[nr.light].power));
        const u32 o = 4 * ab.n_mat + 3 * nr.light;
        acc.add(o + 0, z.x * il.x);
        acc.add(o + 1, z.y * il.y);
        acc.add(o + 2, z.z * il.z);
    }
    for (u32 i = 0; i < nr.n_occ; i++) {
        const float4 imb = inv_nonzero(f4(sc.materials[nr.occ[i]].base_color));
        const u32 o = 4 * nr.occ[i];
        acc.add(o + 0, z.x * imb.x);
        acc.add(o + 1, z.y * imb.y);
        acc.add(o + 2, z.z * imb.z);
    }
}

// ---- camera paths (trace_rays.cl:14-169, inline NEE) -------------------------------------------
PHX_DI void trace_adj_pixel(const SceneDesc &sc, u32 seed, u32 tid, u32 gpix, const AdjBufs &ab, const GradAcc &acc,
                            u32 *overflow) {
    const float4 ur = ab.g_img[gpix] * ab.inv_rounds; // dL / d(this round's radiance increment)
    const float4 uT = ab.gT[gpix], uA = ab.gA[gpix];
    if (ur.x == 0.0f && ur.y == 0.0f && ur.z == 0.0f && uT.x == 0.0f && uT.y == 0.0f && uT.z == 0.0f &&
        uA.x == 0.0f && uA.y == 0.0f && uA.z == 0.0f)
        return;
    u32 width = sc.width, height = sc.height;
    u32 px = tid % width;
    u32 py = tid / width;
    Rng rng = pcg_seed(seed + tid);
    float4 origin, dir;
    make_ray(sc.camera, px, py, width, height, &rng, &origin, &dir);
    float4 throughput = white4();
    IorStack ior;
    init_ior_stack(&ior, AIR_IOR);
    BounceRec br[MAX_RAY_BOUNCES];
    u32 nb = 0;
    const float inv_ds = 1.0f / (float)sc.direct_samples;
    for (i32 depth = 0; depth < (i32)MAX_RAY_BOUNCES; depth++) {
        Hit h;
        bool hit = intersect(sc, origin, dir, EPS, INF, &h, overflow);
        if (!hit) {
            if (sc.has_env)
                add_prefix(acc, br, nb, ur * throughput * sample_envmap(sc, dir));
            break;
        }
        SurfaceHit sh = process_hit(sc, h, origin, dir);
        const phx_material mat = sc.materials[sh.mat_index];
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS)
            throughput *= beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
        float4 tangent, bitangent;
        hit_frame(sc, h, sh, &tangent, &bitangent);
        ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        add_prefix(acc, br, nb, ur * throughput * ctx.emissive);
        float4 view = -dir;
        Rng peek = rng; // sample_bsdf draws the microfacet normal first
        const float4 hm = ggx_sample_vndf(&peek, ctx.shading_normal, sh.normal, view, ctx.roughness);
        BsdfSample bs = sample_bsdf(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        const u32 mo = 4 * sh.mat_index;
        const float4 imb = inv_nonzero(f4(mat.base_color));
        if (bs.event == BSDF_DIFFUSE) {
            // direct = T·occlusion·mean_s NEE_s, NEE_s = L_s·base/π·trans_s
            const float4 w = ur * throughput * (ctx.occlusion * inv_ds);
            float4 zsum = zero4();
            for (u32 d = 0; d < sc.direct_samples; d++) {
                NeeRec nr;
                float4 v = nee_diffuse_adj(&rng, sc, sh.position, ctx.shading_normal, ctx.base_color, overflow, &nr);
                const float4 z = w * v;
                if (z.x == 0.0f && z.y == 0.0f && z.z == 0.0f)
                    continue;
                zsum += z;
                add_nee_common(sc, ab, acc, nr, z);
                acc.add(mo + 0, z.x * imb.x);
                acc.add(mo + 1, z.y * imb.y);
                acc.add(mo + 2, z.z * imb.z);
            }
            add_prefix(acc, br, nb, zsum);
            add_prefix(acc, br, nb, uT * throughput); // the hit point's throughput
            const float4 b = ctx.base_color;          // the hit point's base colour (mb × texture)
            acc.add(mo + 0, uA.x * b.x * imb.x);
            acc.add(mo + 1, uA.y * b.y * imb.y);
            acc.add(mo + 2, uA.z * b.z * imb.z);
            break;
        }
        if (bs.event == BSDF_METALLIC || bs.event == BSDF_FRESNEL) {
            float4 f0 = ctx.base_color;
            if (bs.event == BSDF_FRESNEL) {
                float ratio = (cur - ctx.ior) / (cur + ctx.ior);
                float r0 = ratio * ratio;
                f0 = f4(r0, r0, r0, 0.0f);
            }
            const float dadr = dalpha_drough(ctx.roughness, mat.roughness);
            const float4 w = ur * throughput * inv_ds;
            float4 zsum = zero4();
            for (u32 d = 0; d < sc.direct_samples; d++) {
                NeeRec nr;
                float4 v = nee_specular_adj(&rng, sc, sh.position, ctx.shading_normal, view, f0, ctx.roughness,
                                            overflow, &nr);
                const float4 z = w * v;
                if (z.x == 0.0f && z.y == 0.0f && z.z == 0.0f)
                    continue;
                zsum += z;
                add_nee_common(sc, ab, acc, nr, z);
                acc.add(mo + 3, (z.x + z.y + z.z) * nr.dlog_a * dadr);
                if (bs.event == BSDF_METALLIC) { // f0 = base = mb × texture
                    const float4 b = ctx.base_color;
                    acc.add(mo + 0, z.x * nr.dlog_f0.x * b.x * imb.x);
                    acc.add(mo + 1, z.y * nr.dlog_f0.y * b.y * imb.y);
                    acc.add(mo + 2, z.z * nr.dlog_f0.z * b.z * imb.z);
                }
            }
            add_prefix(acc, br, nb, zsum);
        }
        br[nb++] = bounce_dlog(bs, hm, view, ctx.shading_normal, ctx, mat, sh.mat_index);
        throughput *= bs.throughput;
        if ((u32)depth >= RR_MIN_RAY_DEPTH) {
            float q = fmaxf(throughput.x, fmaxf(throughput.y, throughput.z));
            q = clampf(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float(&rng) > q)
                break;
            throughput *= 1.0f / q;
        }
        float4 side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * EPS + side * EPS;
        dir = bs.dir;
    }
}

__global__ void __launch_bounds__(128) k_trace_adj(LaunchCtx lc, AdjBufs ab) {
    extern __shared__ float s_grad[];
    const GradAcc acc = grad_begin(ab, s_grad);
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < lc.total_pixels) {
        const SceneDesc &sc = lc.scenes[0];
        u32 ovf = 0;
        trace_adj_pixel(sc, __ldg(&lc.seeds[0]), gid, gid, ab, acc, &ovf);
        if (ovf)
            atomicAdd(lc.overflow, ovf);
    }
    grad_end(ab, acc);
}

// ---- photon paths (emit_photons.cl:12-114) -----------------------------------------------------
constexpr u32 MAX_PHOTON_BOUNCES = 32;

PHX_DI void emit_adj_path(const SceneDesc &sc, u32 seed, u32 tid, const AdjBufs &ab, const GradAcc &acc,
                          u32 *overflow) {
    u32 k = ab.offsets[tid];
    const u32 n_stored = ab.offsets[tid + 1] - k;
    if (n_stored == 0)
        return;
    Rng rng = pcg_seed(seed + tid);
    const u32 li = peek_light(&rng, sc);
    float4 origin, dir, power;
    sample_light(&rng, sc, &origin, &dir, &power);
    const float4 il = sc.n_lights > 0 ? inv_nonzero(f4(sc.lights[li].power)) : zero4();
    const u32 lo = 4 * ab.n_mat + 3 * li;
    IorStack ior;
    init_ior_stack(&ior, AIR_IOR);
    float4 throughput = f4(1.0f, 1.0f, 1.0f, 0.0f);
    BounceRec br[MAX_PHOTON_BOUNCES];
    u32 nb = 0, seen = 0;
    for (u32 depth = 0; depth < sc.max_bounces && seen < n_stored; depth++) {
        Hit h;
        bool hit = intersect(sc, origin, dir, EPS, INF, &h, overflow);
        if (!hit)
            return;
        SurfaceHit sh = process_hit(sc, h, origin, dir);
        const phx_material mat = sc.materials[sh.mat_index];
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS) {
            float4 vol = beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
            power *= vol;
            throughput *= vol;
        }
        float4 tangent, bitangent;
        hit_frame(sc, h, sh, &tangent, &bitangent);
        ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        if (depth >= RR_MIN_PHOTON_DEPTH) {
            float q = fmaxf(throughput.x, fmaxf(throughput.y, throughput.z));
            q = clampf(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float(&rng) > q)
                return;
            float inv_q = 1.0f / q;
            throughput *= inv_q;
            power *= inv_q;
        }
        float4 view = -dir;
        Rng peek = rng;
        const float4 hm = ggx_sample_vndf(&peek, ctx.shading_normal, sh.normal, view, ctx.roughness);
        BsdfSample bs = sample_bsdf(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE && dot(dir, sh.normal) < 0.0f) {
            const float4 u = ab.gphi[k] * power; // dL/dΦ ⊙ Φ of this stored photon
            k++;
            seen++;
            add_prefix(acc, br, nb, u);
            acc.add(lo + 0, u.x * il.x);
            acc.add(lo + 1, u.y * il.y);
            acc.add(lo + 2, u.z * il.z);
        }
        br[nb++] = bounce_dlog(bs, hm, view, ctx.shading_normal, ctx, mat, sh.mat_index);
        power *= bs.throughput;
        throughput *= bs.throughput;
        float4 side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * EPS + side * EPS;
        dir = bs.dir;
    }
}

__global__ void __launch_bounds__(128) k_emit_adj(LaunchCtx lc, AdjBufs ab) {
    extern __shared__ float s_grad[];
    const GradAcc acc = grad_begin(ab, s_grad);
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid < lc.total_emit) {
        const SceneDesc &sc = lc.scenes[0];
        u32 ovf = 0;
        emit_adj_path(sc, __ldg(&lc.seeds[0]), gid, ab, acc, &ovf);
        if (ovf)
            atomicAdd(lc.overflow, ovf);
    }
    grad_end(ab, acc);
}

// ---- gather adjoint (gather_flux.cl:5-78, photon_hash.h:56-103) --------------------------------
__global__ void __launch_bounds__(128) k_gather_adj(LaunchCtx lc, GatherBufs g, AdjBufs ab) {
    u32 gpix = blockIdx.x * blockDim.x + threadIdx.x;
    if (gpix >= lc.total_pixels)
        return;
    const SceneDesc &sc = lc.scenes[0];
    const float4 ge = g.hp_emission[gpix];
    const float4 a = ab.g_img[gpix] * ab.kscale[gpix];
    if (ge.w == 0.0f || (a.x == 0.0f && a.y == 0.0f && a.z == 0.0f)) {
        ab.gT[gpix] = zero4();
        ab.gA[gpix] = zero4();
        return;
    }
    const GridDev grid = sc.grid;
    const float r_sq = ab.r2[gpix];
    const float4 pos = g.hp_pos[gpix];
    const float4 nrm = g.hp_normal[gpix];
    const float4 T = g.hp_throughput[gpix], A = g.hp_base_color[gpix];
    const float4 pa = a * T * (A / PI); // dL/dΦ_k = w_k · pa
    const float denom = 2.0f * r_sq;
    const float qx = (pos.x - grid.ox) / grid.cx, qy = (pos.y - grid.oy) / grid.cy, qz = (pos.z - grid.oz) / grid.cz;
    const u32 G = grid.g;
    constexpr float M = 1.0f / 1024.0f;
    float4 S = zero4();
    const u32 *cs = g.cell_start + sc.cell_base;
    for (u32 i = 0; i < 27; i++) {
        float px = pos.x, py = pos.y, pz = pos.z;
        px += (float)((i32)(i % 3) - 1) * grid.cx;
        py += (float)((i32)((i / 3) % 3) - 1) * grid.cy;
        pz += (float)((i32)((i / 9) % 3) - 1) * grid.cz;
        const u32 hsh = get_hash(px, py, pz, grid);
        if (hsh == 0)
            continue;
        const u32 hz = (hsh - 1) % G, hy = ((hsh - 1) / G) % G, hx = (hsh - 1) / (G * G);
        const float gx = fmaxf(fmaxf(((float)hx - M) - qx, qx - ((float)hx + (1.0f + M))), 0.0f) * grid.cx;
        const float gy = fmaxf(fmaxf(((float)hy - M) - qy, qy - ((float)hy + (1.0f + M))), 0.0f) * grid.cy;
        const float gz = fmaxf(fmaxf(((float)hz - M) - qz, qz - ((float)hz + (1.0f + M))), 0.0f) * grid.cz;
        if ((gx * gx + gy * gy) + gz * gz > r_sq)
            continue;
        const u32 end = min(__ldg(&cs[hsh + 1]), g.n_cap);
        for (u32 k = min(__ldg(&cs[hsh]), g.n_cap); k < end; k++) {
            const float4 p = __ldg(&g.s_posdir[k]);
            const float dx = pos.x - p.x, dy = pos.y - p.y, dz = pos.z - p.z, dw = pos.w - 0.0f;
            const float dsq = ((dx * dx + dy * dy) + dz * dz) + dw * dw;
            if (!(dsq < r_sq))
                continue;
            if (dot(decode_oct(__float_as_uint(p.w)), nrm) > 0.0f)
                continue;
            const float w = GAUSS_ALPHA * (1.0f - (1.0f - pm_expf((-GAUSS_BETA) * dsq / denom)) / GAUSS_DENOM);
            const u32 c = __ldg(&ab.perm[k]);
            S += w * __ldg(&ab.ph_pow[c]);
            atomicAdd(&ab.gphi[c].x, w * pa.x);
            atomicAdd(&ab.gphi[c].y, w * pa.y);
            atomicAdd(&ab.gphi[c].z, w * pa.z);
        }
    }
    ab.gT[gpix] = a * (A / PI) * S;
    ab.gA[gpix] = a * (T / PI) * S;
}

// ---- small kernels -------------------------------------------------------------------------------
// unquantised power of the canonical photons (the compaction of k_compact for the power slots)
__global__ void __launch_bounds__(256) k_compact_pow(LaunchCtx lc, const float4 *slot_pow, const u32 *counts,
                                                     const u32 *offsets, float4 *ph_pow) {
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.total_emit)
        return;
    const SceneDesc &sc = lc.scenes[0];
    const u32 c = counts[gid], off = offsets[gid];
    u64 slot = sc.slot_base + gid;
    for (u32 j = 0; j < c; j++, slot += sc.n_emit)
        ph_pow[off + j] = slot_pow[slot];
}

// K_n = Π_{m>=n} ratio_m / (π r_R² N) per pixel, rounds stored round-major
__global__ void __launch_bounds__(256) k_adj_scale(const float *ratio, float *kscale, const float4 *flux, u32 n_pix,
                                                   u32 rounds, float inv_n) {
    u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pix)
        return;
    const float area = PI * flux[p].w;
    float k = area > 0.0f ? inv_n / area : 0.0f;
    for (u32 n = rounds; n-- > 0;) {
        k *= ratio[(size_t)n * n_pix + p];
        kscale[(size_t)n * n_pix + p] = k;
    }
}

// linear image radiance/R + flux/(π r² N) (output.cpp:62-76 before the display transform)
__global__ void __launch_bounds__(256) k_adj_image(const float4 *flux, const float4 *radiance, u32 n_pix,
                                                   float inv_rounds, float inv_n, float *img) {
    u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_pix)
        return;
    const float4 f = flux[p], r = radiance[p];
    const float area = PI * f.w;
    const float per = area > 0.0f ? inv_n / area : 0.0f;
    img[3 * (size_t)p + 0] = r.x * inv_rounds + f.x * per;
    img[3 * (size_t)p + 1] = r.y * inv_rounds + f.y * per;
    img[3 * (size_t)p + 2] = r.z * inv_rounds + f.z * per;
}

static size_t grad_smem(const AdjBufs &ab) { return ab.block_sums ? 4 * (size_t)ab.n_params : 0; }

void launch_trace_adj(const LaunchCtx &lc, const AdjBufs &ab, cudaStream_t st) {
    if (lc.total_pixels)
        k_trace_adj<<<(lc.total_pixels + 127) / 128, 128, grad_smem(ab), st>>>(lc, ab);
}
void launch_emit_adj(const LaunchCtx &lc, const AdjBufs &ab, cudaStream_t st) {
    if (lc.total_emit)
        k_emit_adj<<<(lc.total_emit + 127) / 128, 128, grad_smem(ab), st>>>(lc, ab);
}
void launch_gather_adj(const LaunchCtx &lc, const GatherBufs &g, const AdjBufs &ab, cudaStream_t st) {
    if (lc.total_pixels)
        k_gather_adj<<<(lc.total_pixels + 127) / 128, 128, 0, st>>>(lc, g, ab);
}
void launch_compact_pow(const LaunchCtx &lc, const float4 *slot_pow, const u32 *counts, const u32 *offsets,
                        float4 *ph_pow, cudaStream_t st) {
    if (lc.total_emit)
        k_compact_pow<<<(lc.total_emit + 255) / 256, 256, 0, st>>>(lc, slot_pow, counts, offsets, ph_pow);
}
void launch_adj_scale(const float *ratio, float *kscale, const float4 *flux, u32 n_pix, u32 rounds, float inv_n,
                      cudaStream_t st) {
    if (n_pix)
        k_adj_scale<<<(n_pix + 255) / 256, 256, 0, st>>>(ratio, kscale, flux, n_pix, rounds, inv_n);
}
void launch_adj_image(const float4 *flux, const float4 *radiance, u32 n_pix, float inv_rounds, float inv_n, float *img,
                      cudaStream_t st) {
    if (n_pix)
        k_adj_image<<<(n_pix + 255) / 256, 256, 0, st>>>(flux, radiance, n_pix, inv_rounds, inv_n, img);
}

} // namespace phx
