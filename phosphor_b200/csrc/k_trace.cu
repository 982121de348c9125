// k_trace.cu — camera paths to the first diffuse hit with explicit direct lighting
// (kernels/trace_rays.cl:14-169), for every pixel of every scene of an engine.
//
// Two forms produce identical results:
//  * k_trace: one thread per pixel, the reference's nested loops as written.  A warp then runs
//    the traversal from several call sites (camera ray, diffuse-NEE shadow ray, specular-NEE
//    shadow ray, shadow continuation) one after another, and every lane waits for the longest
//    path of its warp.
//  * k_trace_persistent: each lane runs its pixel as a state machine that issues ONE ray query
//    per step (camera ray or shadow ray), so all lanes of a warp traverse together from a single
//    call site; when a lane's path ends, the warp refills its free lanes with new pixels in one
//    shot (__ballot_sync / __popc over the free mask, one atomicAdd per refill).  The state
//    machine replays the reference's statements in the same order with the same RNG draws, only
//    split at the ray queries.
// Pixel i of a scene uses pcg_seed(round_seed + i), so results do not depend on which lane or
// block traces it.
//
// This file compiles the light sampling of NEE, the texture lookups and the BSDF sampler out of
// line: the camera-path kernels call them from several places, and one shared copy keeps their
// instruction footprint small (measured: warps stalled on instruction fetch dominated, and the
// persistent camera kernel ran 18 % faster out of line).  The photon kernels (k_emit.cu) measure
// faster with everything inlined and keep it so.
#define PHX_OUTLINE_NEE
#define PHX_OUTLINE_TEX
#define PHX_OUTLINE_BSDF
#include "dev_shading.cuh"
#include "kernels.hpp"

// Minimum resident blocks per SM asked of the compiler, which caps registers per thread (64 at 8
// blocks of 128 threads).  Both traversal kernels are latency-bound: 8 blocks per SM (with a few
// hundred bytes of spills to L1) measured faster than 4-7 register-limited blocks, and faster than
// 10-12 blocks with heavier spills (camera kernel 8.5 -> 7.7 ms, shadow 8.8 -> 7.8 ms).
#ifndef PHX_TRACE_MINB
#define PHX_TRACE_MINB 8
#endif
#ifndef PHX_SHADOW_MINB
#define PHX_SHADOW_MINB 8
#endif

namespace phx {

struct TraceResult {
    float4 position, normal, throughput, base_color, direct, emission;
};

PHX_DI void write_result(const TraceOut &out, u32 gpix, const TraceResult &r) {
    out.emission[gpix] = r.emission;
    out.pos[gpix] = r.position;
    out.normal[gpix] = r.normal;
    out.throughput[gpix] = r.throughput;
    out.base_color[gpix] = r.base_color;
    out.direct[gpix] = r.direct;
}

// Deferred diffuse-hit NEE (trace_rays.cl:103-118).  The reference's path ends after this loop
// and its RNG draws (light choice, light point) never depend on the shadow rays' outcome, so the
// loop is split in three kernels: k_nee_sample draws the samples in order and records each shadow
// ray; the shadow wavefront traces them; the resolve kernel sums the contributions in sample order.
// The camera kernels only leave the pixel's RNG state and shading normal in its first sample slot
// (stash_nee): drawing the samples there would run the light-sampling code for one lane of a warp
// at a time, while k_nee_sample runs it for 32 diffuse hit points together.
PHX_DI void stash_nee(const TraceOut &out, u32 gpix, Rng rng, float4 sn) {
    out.stash_sn[gpix] = sn;
    out.stash_rng[gpix] = rng.state;
}

PHX_DI void record_nee(const SceneDesc &sc, Rng *rng, float4 pos, float4 sn, float4 base, const TraceOut &out,
                       u32 slot) {
    for (u32 d = 0; d < sc.direct_samples; d++, slot++) {
        LightFragment f;
        if (sample_light_fragment(rng, sc, pos, sn, &f)) { // direct_lighting_diffuse, light_sampling.h:345-352
            out.nee_ray[slot] = f4(f.dir.x, f.dir.y, f.dir.z, f.dist);
            out.nee_val[slot] = f.radiance * (base / PI);
        } else {
            out.nee_ray[slot] = f4(0.0f, 0.0f, 0.0f, -1.0f); // returns BLACK
            out.nee_val[slot] = zero4();
        }
    }
}

// ---- one thread per pixel ---------------------------------------------------------------------
PHX_DI void trace_pixel(const SceneDesc &sc, u32 seed, u32 tid, const TraceOut &out, u32 gpix, u32 *overflow,
                        bool defer) {
    u32 width = sc.width, height = sc.height;
    u32 px = tid % width;
    u32 py = tid / width;
    Rng rng = pcg_seed(seed + tid);
    float4 origin, dir;
    make_ray(sc.camera, px, py, width, height, &rng, &origin, &dir);
    float4 position = zero4(), normal = zero4(), throughput = white4(), base_color = zero4(), direct = zero4(),
           emission = zero4();
    IorStack ior;
    init_ior_stack(&ior, AIR_IOR);
    for (i32 depth = 0; depth < (i32)MAX_RAY_BOUNCES; depth++) {
        Hit h;
        bool hit = intersect(sc, origin, dir, EPS, INF, &h, overflow);
        if (!hit) {
            if (sc.has_env)
                emission += throughput * sample_envmap(sc, dir);
            break;
        }
        const phx_material mat = sc.materials[tri_mat(sc, h.tri)];
        SurfaceHit sh = process_hit(sc, h, origin, dir, mat_textured(mat));
        float4 vol = white4();
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS) {
            vol = beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
            throughput *= vol;
        }
        float4 tangent = zero4(), bitangent = zero4(); // the frame only serves a normal map
        if (mat.norm_index != NO_TEXTURE)
            hit_frame(sc, h, sh, &tangent, &bitangent);
        ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        emission += throughput * ctx.emissive;
        float4 view = -dir;
        BsdfSample bs = sample_bsdf(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE) {
            if (defer) {
                stash_nee(out, gpix, rng, ctx.shading_normal);
                direct = f4(ctx.occlusion, 0.0f, 0.0f, 0.0f); // the resolve kernel completes it
            } else {
                float4 sum = zero4();
                for (u32 d = 0; d < sc.direct_samples; d++)
                    sum += direct_lighting_diffuse(&rng, sc, sh.position, ctx.shading_normal, ctx.base_color,
                                                   overflow);
                direct = throughput * ctx.occlusion * (sum / (float)sc.direct_samples);
            }
            emission = f4(emission.x, emission.y, emission.z, 1.0f);
            position = sh.position;
            normal = sh.normal;
            base_color = ctx.base_color;
            break;
        }
        if (bs.event == BSDF_METALLIC) {
            float4 sum = zero4();
            for (u32 d = 0; d < sc.direct_samples; d++)
                sum += direct_lighting_specular(&rng, sc, sh.position, ctx.shading_normal, view, ctx.base_color,
                                                ctx.roughness, overflow);
            emission += throughput * (sum / (float)sc.direct_samples);
        }
        if (bs.event == BSDF_FRESNEL) {
            float ratio = (cur - ctx.ior) / (cur + ctx.ior);
            float r0 = ratio * ratio;
            float4 f0 = f4(r0, r0, r0, 0.0f);
            float4 sum = zero4();
            for (u32 d = 0; d < sc.direct_samples; d++)
                sum += direct_lighting_specular(&rng, sc, sh.position, ctx.shading_normal, view, f0, ctx.roughness,
                                                overflow);
            emission += throughput * (sum / (float)sc.direct_samples);
        }
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
    TraceResult r{position, normal, throughput, base_color, direct, emission};
    write_result(out, gpix, r);
}

__global__ void __launch_bounds__(128) k_trace(LaunchCtx lc, TraceOut out) {
    u32 gid = lc.pix_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.pix_hi)
        return;
    u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
    const SceneDesc &sc = lc.scenes[s];
    if (!sc.active)
        return;
    u32 ovf = 0;
    trace_pixel(sc, __ldg(&lc.seeds[s]), gid - sc.pixel_base, out, gid, &ovf, lc.nee_defer != 0);
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

// ---- state machine ------------------------------------------------------------------------------
enum : u32 { PH_CAMERA = 0, PH_SHADOW = 1 };
enum : u32 { NEE_DIFFUSE = 0, NEE_SPECULAR = 1, NEE_NONE = 2 };

struct CameraPath {
    const SceneDesc *sc;
    u32 gpix, tid;
    Rng rng;
    u32 phase, nee_kind, nee_i, depth;
    float4 origin, dir;         // current query ray
    float t_min, t_max;
    float4 throughput, emission;
    IorStack ior;
    // shading state kept across the NEE loop (trace_rays.cl:99-147)
    float4 pos, sn, gn, base, view, f0, bs_dir, bs_thr, nee_sum;
    float occl, rough;
    // pending shadow query (shadow_transmittance, light_sampling.h:302-333)
    float4 m, trans;
    u32 sh_depth;
    u32 def_n; // emission terms listed for the deferred specular NEE (0: none deferred yet)
};

// Adds one term to the path's emission.  Once the path has deferred a specular NEE term, the sum
// is completed after the shadow pass (k_spec_resolve), so its later terms are listed in order
// instead.  A zero term is left out: the sum starts at +0 and only ever adds, so it is never -0 and
// e + (+-0) == e bit for bit.
PHX_DI void cp_add_emission(CameraPath &p, const TraceOut &out, float4 a) {
    if (p.def_n == 0) {
        p.emission += a;
        return;
    }
    if (a.x == 0.0f && a.y == 0.0f && a.z == 0.0f && a.w == 0.0f)
        return;
    if (p.def_n >= DEF_MAX) { // cannot happen (at most 10 terms follow a deferred one); reported
        p.def_n |= DEF_OVERFLOW;
        return;
    }
    const size_t k = (size_t)p.gpix * DEF_MAX + p.def_n++;
    out.def_val[k] = a;
    out.def_tag[k] = DEF_KNOWN;
}

PHX_DI void cp_finish(CameraPath &p, const TraceOut &out, bool diffuse_hit, bool deferred = false) {
    if (out.def_cnt) {
        out.def_cnt[p.gpix] = p.def_n | (diffuse_hit ? DEF_DIFFUSE : 0u);
        if (p.def_n)
            out.def_prefix[p.gpix] = p.emission;
    }
    TraceResult r;
    r.throughput = p.throughput;
    if (diffuse_hit) {
        r.emission = f4(p.emission.x, p.emission.y, p.emission.z, 1.0f);
        r.position = p.pos;
        r.normal = p.gn;
        r.base_color = p.base;
        r.direct = deferred ? f4(p.occl, 0.0f, 0.0f, 0.0f)
                            : p.throughput * p.occl * (p.nee_sum / (float)p.sc->direct_samples);
    } else {
        r.emission = p.emission;
        r.position = zero4();
        r.normal = zero4();
        r.base_color = zero4();
        r.direct = zero4();
    }
    write_result(out, p.gpix, r);
}

PHX_DI void cp_start(CameraPath &p, const SceneDesc *sc, u32 seed, u32 tid, u32 gpix) {
    p.sc = sc;
    p.gpix = gpix;
    p.tid = tid;
    p.rng = pcg_seed(seed + tid);
    make_ray(sc->camera, tid % sc->width, tid / sc->width, sc->width, sc->height, &p.rng, &p.origin, &p.dir);
    p.throughput = white4();
    p.emission = zero4();
    p.def_n = 0;
    init_ior_stack(&p.ior, AIR_IOR);
    p.depth = 0;
    p.phase = PH_CAMERA;
    p.t_min = EPS;
    p.t_max = INF;
}

// Whether a scene's specular NEE samples are drawn by the shadow kernel (each thread its own
// sample, from the event's RNG state advanced past the samples before it): possible when every
// light sample takes the same number of draws; the event record needs four sample slots.
PHX_DI bool spec_drawn_in_shadow(const SceneDesc &sc) {
    return sc.light_draws != LIGHT_DRAWS_VARY && sc.direct_samples >= 4;
}

// One sample of direct_lighting_specular (light_sampling.h:355-390) up to its shadow query: false
// when it contributes nothing (no RNG draw depends on a shadow query's outcome), else the light
// fragment and the weight m of its transmittance.
// INL: the light sampler inlined (the shadow kernel) instead of called out of line.
template <bool INL = false>
PHX_DI bool spec_light_sample(Rng *rng, const SceneDesc &sc, float4 pos, float4 sn, float4 view, float4 f0,
                              float rough, LightFragment *f, float4 *m) {
    float ndv = dot(view, sn);
    if (ndv < EPS)
        return false;
    if (!(INL ? light_fragment(rng, sc, pos, sn, f) : sample_light_fragment(rng, sc, pos, sn, f)) ||
        f->n_dot_dir < EPS)
        return false;
    float alpha = rough * rough;
    float4 h = normalize(f->dir + view);
    float ndh = fmaxf(dot(sn, h), 0.0f);
    float g = ggx_ndf(ndh, alpha);
    float4 fr = fresnel4(f0, view, h);
    float sm = smith_g1_ggx(f->n_dot_dir, alpha) * smith_g1_ggx(ndv, alpha);
    float4 spec = f->radiance * g * fr * sm / (4.0f * f->n_dot_dir * ndv);
    if (dot(spec, spec) < EPS * EPS)
        return false;
    *m = spec;
    return true;
}

PHX_DI bool spec_sample(CameraPath &p, LightFragment *f, float4 *m) {
    return spec_light_sample(&p.rng, *p.sc, p.pos, p.sn, p.view, p.f0, p.rough, f, m);
}

// Runs the NEE loop from sample nee_i until a shadow query is needed (returns true with the query
// in origin/dir/t_min/t_max) or all samples are done (returns false).
PHX_DI bool cp_next_shadow(CameraPath &p) {
    const SceneDesc &sc = *p.sc;
    while (p.nee_i < sc.direct_samples) {
        if (p.nee_kind == NEE_DIFFUSE) { // direct_lighting_diffuse, light_sampling.h:335-353
            LightFragment f;
            if (!sample_light_fragment(&p.rng, sc, p.pos, p.sn, &f)) {
                p.nee_sum += zero4();
                p.nee_i++;
                continue;
            }
            p.m = f.radiance * (p.base / PI);
            p.dir = f.dir;
            p.t_max = f.dist - EPS;
        } else {
            LightFragment f;
            if (!spec_sample(p, &f, &p.m)) {
                p.nee_sum += zero4();
                p.nee_i++;
                continue;
            }
            p.dir = f.dir;
            p.t_max = f.dist - EPS;
        }
        p.origin = p.pos;
        p.t_min = EPS;
        p.trans = white4();
        p.sh_depth = 0;
        p.phase = PH_SHADOW;
        return true;
    }
    return false;
}

// Continues the camera path after its BSDF sample (trace_rays.cl:149-160).  Returns true when a
// new camera query is pending, false when the path has ended (outputs written).
PHX_DI bool cp_continue(CameraPath &p, const TraceOut &out) {
    p.throughput *= p.bs_thr;
    if (p.depth >= RR_MIN_RAY_DEPTH) {
        float q = fmaxf(p.throughput.x, fmaxf(p.throughput.y, p.throughput.z));
        q = clampf(q, RR_MIN_Q, RR_MAX_Q);
        if (random_float(&p.rng) > q) {
            cp_finish(p, out, false);
            return false;
        }
        p.throughput *= 1.0f / q;
    }
    float4 side = (dot(p.bs_dir, p.gn) > 0.0f) ? p.gn : -p.gn;
    p.origin = p.pos + p.bs_dir * EPS + side * EPS;
    p.dir = p.bs_dir;
    p.depth++;
    if (p.depth >= MAX_RAY_BOUNCES) {
        cp_finish(p, out, false);
        return false;
    }
    p.phase = PH_CAMERA;
    p.t_min = EPS;
    p.t_max = INF;
    return true;
}

// After the NEE loop of a bounce: finish (diffuse) or continue (specular events).
PHX_DI bool cp_after_nee(CameraPath &p, const TraceOut &out) {
    if (p.nee_kind == NEE_DIFFUSE) {
        cp_finish(p, out, true);
        return false;
    }
    if (p.nee_kind == NEE_SPECULAR)
        cp_add_emission(p, out, p.throughput * (p.nee_sum / (float)p.sc->direct_samples));
    return cp_continue(p, out);
}

// Claims n consecutive slots of a counter for each calling lane; the converged lanes asking for the
// same n share one atomic.
PHX_DI u32 claim_slots(u32 *counter, u32 n) {
    const u32 lane = threadIdx.x & 31u;
    const u32 same = __match_any_sync(__activemask(), n);
    const u32 leader = __ffs(same) - 1;
    u32 base = 0;
    if (lane == leader)
        base = atomicAdd(counter, n * (u32)__popc(same));
    base = __shfl_sync(same, base, leader);
    return base + n * (u32)__popc(same & ((1u << lane) - 1u));
}

// Specular NEE without the shadow queries: draws the event's samples in order (the path's RNG
// advances exactly as in the traced form), records each shadow ray with its weight in claimed
// sample slots and lists the NEE term (throughput * mean of the samples' contributions) for
// k_spec_resolve.  Returns false, having changed nothing, when the sample slots are exhausted.
// Out of line: it runs once per specular event and would otherwise add its registers to every
// step of the camera kernel's loop.
static __device__ __noinline__ bool cp_defer_specular(CameraPath &p, const TraceOut &out) {
    const u32 ds = p.sc->direct_samples;
    if (p.def_n >= DEF_MAX)
        return false;
    const bool drawn_later = spec_drawn_in_shadow(*p.sc);
    const u32 base = claim_slots(out.spec_next, ds);
    if (ds > out.spec_cap || base > out.spec_cap - ds) {
        // no room: the slots of this claim that lie below the capacity carry no ray
        for (u32 slot = base; slot < out.spec_cap && slot - base < ds; slot++) {
            out.spec_ray[slot] = drawn_later ? f4(__uint_as_float(slot), 0.0f, 0.0f, __uint_as_float(1u))
                                             : f4(0.0f, 0.0f, 0.0f, -1.0f);
            out.spec_val[slot] = zero4();
            out.spec_org[slot] = zero4();
            out.spec_pix[slot] = p.gpix;
        }
        return false;
    }
    if (drawn_later) {
        // k_shadow draws sample i from this state advanced by i * light_draws; here the event is
        // recorded in its first four slots' origins and every slot's header, and the path's RNG
        // skips the event's draws (none when the view grazes: every sample fails before drawing)
        const bool grazing = dot(p.view, p.sn) < EPS;
        out.spec_org[base] = p.pos;
        out.spec_org[base + 1] = p.sn;
        out.spec_org[base + 2] = p.view;
        out.spec_org[base + 3] = p.f0;
        const float4 hdr = f4(__uint_as_float(base), p.rough, __uint_as_float(p.rng.state),
                              __uint_as_float(grazing ? 1u : 0u));
        for (u32 i = 0; i < ds; i++) {
            out.spec_ray[base + i] = hdr;
            out.spec_pix[base + i] = p.gpix;
        }
        if (!grazing)
            p.rng = rng_advance(p.rng, ds * p.sc->light_draws);
    } else {
    for (u32 i = 0; i < ds; i++) {
        LightFragment f;
        float4 m;
        const u32 slot = base + i;
        if (spec_sample(p, &f, &m)) {
            out.spec_ray[slot] = f4(f.dir.x, f.dir.y, f.dir.z, f.dist);
            out.spec_val[slot] = m;
        } else {
            out.spec_ray[slot] = f4(0.0f, 0.0f, 0.0f, -1.0f);
            out.spec_val[slot] = zero4();
        }
        out.spec_org[slot] = p.pos;
        out.spec_pix[slot] = p.gpix;
    }
    }
    const size_t k = (size_t)p.gpix * DEF_MAX + p.def_n++;
    out.def_val[k] = p.throughput;
    out.def_tag[k] = base;
    return true;
}

// Consumes the result of the pending query; returns true while the path needs another query.
// NOTEX: no material of the context has a texture (texture indices never change after set-up), so
// the texture branches are compiled out of this instance.
template <bool NOTEX>
PHX_DI bool cp_advance(CameraPath &p, bool hit, const Hit &h, const TraceOut &out, bool defer) {
    const SceneDesc &sc = *p.sc;
    if (p.phase == PH_SHADOW) {
        bool done_ray = false;
        float4 contrib;
        if (!hit) {
            contrib = p.trans;
            done_ray = true;
        } else {
            u32 mi = tri_mat(sc, h.tri);
            const phx_material &mat = sc.materials[mi];
            if (mat.transmission < EPS) {
                contrib = zero4();
                done_ray = true;
            } else {
                float4 base = f4(mat.base_color);
                if (!NOTEX && mat.diff_index != NO_TEXTURE) {
                    SurfaceHit s = process_hit(sc, h, p.origin, p.dir);
                    base *= srgb_to_linear(sample_texture_uv(sc, mi, mat.diff_index, s.uvx, s.uvy, 0));
                }
                if (mat.att_dist > EPS)
                    p.trans *= beer_lambert(f4(mat.att_color), mat.att_dist, h.t - p.t_min);
                p.trans *= base * mat.transmission;
                if (dot(p.trans, p.trans) < EPS) {
                    contrib = zero4();
                    done_ray = true;
                } else {
                    p.t_min = h.t + EPS;
                    p.sh_depth++;
                    if (p.sh_depth >= MAX_RAY_BOUNCES) {
                        contrib = p.trans;
                        done_ray = true;
                    }
                }
            }
        }
        if (!done_ray)
            return true; // next transmittance query along the same shadow ray
        p.nee_sum += p.m * contrib;
        p.nee_i++;
        if (cp_next_shadow(p))
            return true;
        return cp_after_nee(p, out);
    }
    // camera query (trace_rays.cl:64-147)
    if (!hit) {
        if (sc.has_env)
            cp_add_emission(p, out, p.throughput * sample_envmap(sc, p.dir));
        cp_finish(p, out, false);
        return false;
    }
    phx_material mat = sc.materials[tri_mat(sc, h.tri)];
    if constexpr (NOTEX)
        mat.diff_index = mat.emis_index = mat.norm_index = mat.occlusion_index = mat.metal_rough_index =
            mat.transmission_index = NO_TEXTURE;
    SurfaceHit sh = process_hit(sc, h, p.origin, p.dir, mat_textured(mat));
    float cur = current_ior(&p.ior);
    if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS)
        p.throughput *= beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
    float4 tangent = zero4(), bitangent = zero4(); // the frame only serves a normal map
    if (mat.norm_index != NO_TEXTURE)
        hit_frame(sc, h, sh, &tangent, &bitangent);
    ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
    cp_add_emission(p, out, p.throughput * ctx.emissive);
    p.view = -p.dir;
    BsdfSample bs = sample_bsdf(&p.rng, ctx, ctx.shading_normal, sh.normal, p.view, &p.ior, sh.front_face);
    p.pos = sh.position;
    p.sn = ctx.shading_normal;
    p.gn = sh.normal;
    p.base = ctx.base_color;
    p.occl = ctx.occlusion;
    p.rough = ctx.roughness;
    p.bs_dir = bs.dir;
    p.bs_thr = bs.throughput;
    p.nee_sum = zero4();
    p.nee_i = 0;
    if (bs.event == BSDF_DIFFUSE) {
        p.nee_kind = NEE_DIFFUSE;
        if (defer) {
            stash_nee(out, p.gpix, p.rng, p.sn);
            cp_finish(p, out, true, true);
            return false;
        }
    } else if (bs.event == BSDF_METALLIC) {
        p.nee_kind = NEE_SPECULAR;
        p.f0 = ctx.base_color;
    } else if (bs.event == BSDF_FRESNEL) {
        float ratio = (cur - ctx.ior) / (cur + ctx.ior);
        float r0 = ratio * ratio;
        p.nee_kind = NEE_SPECULAR;
        p.f0 = f4(r0, r0, r0, 0.0f);
    } else {
        p.nee_kind = NEE_NONE;
        return cp_continue(p, out);
    }
    if (defer && out.spec_ray && cp_defer_specular(p, out))
        return cp_continue(p, out);
    if (cp_next_shadow(p))
        return true;
    return cp_after_nee(p, out);
}

template <bool NOTEX>
__global__ void __launch_bounds__(128, PHX_TRACE_MINB) k_trace_persistent(LaunchCtx lc, TraceOut out, u32 *queue) {
    const u32 lane = threadIdx.x & 31u;
    const u32 lt_mask = (1u << lane) - 1u;
    u32 ovf = 0;
    CameraPath p;
    bool active = false, exhausted = false;
    for (;;) {
        // refill free lanes with new pixels: one atomic per warp
        const u32 need = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (need) {
            const u32 leader = __ffs(need) - 1;
            u32 base = 0;
            if (lane == leader)
                base = atomicAdd(queue, (u32)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                const u32 gid = lc.pix_lo + base + __popc(need & lt_mask);
                if (gid < lc.pix_hi) {
                    const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
                    const SceneDesc *sc = lc.scenes + s;
                    if (sc->active) { // a retired scene's pixel is skipped; the lane refills next step
                        cp_start(p, sc, __ldg(&lc.seeds[s]), gid - sc->pixel_base, gid);
                        active = true;
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted))
            break;
        if (active) {
            Hit h;
            const bool any = p.phase == PH_SHADOW && p.sc->any_transmissive == 0;
            const bool hit = intersect(*p.sc, p.origin, p.dir, p.t_min, p.t_max, &h, &ovf, any);
            active = cp_advance<NOTEX>(p, hit, h, out, lc.nee_defer != 0);
        }
    }
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

// ---- shadow wavefront ---------------------------------------------------------------------------
// One thread per recorded NEE sample; the ds samples of a pixel are consecutive threads, so a warp
// traces shadow rays from one or two hit points toward the same light: coherent traversal.
template <int KIND, bool PER_PIXEL, bool ONE>
PHX_DI void shadow_spec_slots(const LaunchCtx &lc, const TraceOut &out, u32 first_block, const SceneDesc &one);

// Blocks [0, nee_blocks): one diffuse sample slot per thread.  Blocks from nee_blocks on (only when
// the specular NEE is deferred): the specular sample slots, grid-stride; being last in the grid
// they start as the diffuse blocks drain and fill the launch's tail.  KIND: the scenes' kind
// (SHADOW_*), chosen on the host.
// per_pixel (a single scene whose only light is a point, spot or directional light): choosing that
// light is a sample's only random draw, so all ds samples of a hit point are the same ray with the
// same weight; one thread per pixel traces sample 0 and writes its contribution to the pixel's ds
// slots, which k_nee_resolve then sums as before (the same values in the same order).
// ONE: a single-scene context whose scene descriptor comes as a kernel parameter (`one`), so the
// traversal reads its pointers and sizes from the constant bank instead of holding them in
// registers (caustic shadow stage 6.80 -> 6.71 ms; the same form of the photon kernel measured no
// gain).  A captured graph then holds the descriptor by value: the engine re-captures after any
// change of a single scene's descriptor.
template <int KIND, bool PER_PIXEL, bool ONE>
__global__ void __launch_bounds__(128, PHX_SHADOW_MINB)
    k_shadow(LaunchCtx lc, TraceOut out, u32 nee_blocks, const __grid_constant__ SceneDesc one) {
    constexpr bool per_pixel = PER_PIXEL;
    if (blockIdx.x >= nee_blocks) {
        shadow_spec_slots<KIND, PER_PIXEL, ONE>(lc, out, nee_blocks, one);
        return;
    }
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (per_pixel ? (ONE ? one : lc.scenes[0]).n_pixels : lc.total_nee))
        return;
    const u32 s = per_pixel || ONE || lc.n_scenes == 1 ? 0 : find_scene(lc.nee_bases, lc.n_scenes, t);
    const SceneDesc &sc = ONE ? one : lc.scenes[s];
    if (!sc.active)
        return;
    const u32 ds = sc.direct_samples;
    const u32 pixel = per_pixel ? t : (t - sc.nee_base) / ds;
    const u32 g = per_pixel ? sc.nee_base + pixel * ds : t; // this thread's (first) sample slot
    const u32 gpix = sc.pixel_base + pixel;
    if (out.emission[gpix].w != 1.0f)
        return; // no diffuse hit point: the slot was not used this round
    const float4 pos = out.pos[gpix];
    float4 dir = zero4(), w = zero4();
    float dist = -1.0f; // < 0: sample_light_fragment failed, direct_lighting_diffuse returns BLACK
    if (sc.light_draws != LIGHT_DRAWS_VARY) {
        // this slot's sample, drawn here: the pixel's stream advanced past the samples before it
        Rng rng;
        rng.state = out.stash_rng[gpix];
        rng = rng_advance(rng, (g - sc.nee_base - pixel * ds) * sc.light_draws);
        LightFragment f;
        // the light sampler inlined here (out of line in the camera kernels): shadow stage 6.59 -> 6.47 ms
        if (light_fragment(&rng, sc, pos, out.stash_sn[gpix], &f)) { // light_sampling.h:345-352
            dir = f4(f.dir.x, f.dir.y, f.dir.z, 0.0f);
            dist = f.dist;
            w = f.radiance * (out.base_color[gpix] / PI);
        }
    } else { // drawn by k_nee_sample
        const float4 ray = out.nee_ray[g];
        if (!(ray.w < 0.0f)) {
            dir = f4(ray.x, ray.y, ray.z, 0.0f);
            dist = ray.w;
            w = out.nee_val[g];
        }
    }
    float4 contrib = zero4();
    if (!(dist < 0.0f)) {
        u32 ovf = 0;
        contrib = w * shadow_transmittance<KIND>(sc, pos, dir, dist, &ovf); // frag.radiance * (base / PI) * trans
        if (ovf)
            atomicAdd(lc.overflow, per_pixel ? ovf * ds : ovf);
    }
    if (per_pixel) {
        for (u32 i = 0; i < ds; i++)
            out.nee_val[g + i] = contrib;
    } else {
        out.nee_val[g] = contrib;
    }
}

// Deferred specular NEE samples: one thread per claimed sample slot.  An event's samples are
// consecutive, so a warp traces rays from one or two hit points toward the lights together.  The
// contribution is the traced form's: weight * transmittance, zero for a sample without a ray.
// per_pixel (see k_shadow): an event's ds samples, ds consecutive slots from a multiple of ds, are
// one ray with one weight: one thread per event traces its first slot and fills all ds.
template <int KIND, bool PER_PIXEL, bool ONE>
PHX_DI void shadow_spec_slots(const LaunchCtx &lc, const TraceOut &out, u32 first_block, const SceneDesc &one) {
    const u32 n = min(*out.spec_next, out.spec_cap);
    const u32 stride = (gridDim.x - first_block) * blockDim.x;
    const u32 step = PER_PIXEL ? (ONE ? one : lc.scenes[0]).direct_samples : 1u;
    u32 ovf = 0;
    for (u32 e = (blockIdx.x - first_block) * blockDim.x + threadIdx.x; (u64)e * step < n; e += stride) {
        const u32 g = e * step;
        const u32 gpix = out.spec_pix[g];
        const SceneDesc &sc = ONE ? one : lc.scenes[lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gpix)];
        const float4 hdr = out.spec_ray[g];
        float4 org, dir = zero4(), w = zero4();
        float dist = -1.0f; // < 0: no contribution
        if (spec_drawn_in_shadow(sc)) {
            // the event recorded by the camera pass: header (first slot, roughness, RNG state,
            // grazing view), origin / shading normal / view / f0 in its first four slots
            const u32 base = __float_as_uint(hdr.x);
            org = out.spec_org[base];
            if (__float_as_uint(hdr.w) == 0u) {
                Rng rng;
                rng.state = __float_as_uint(hdr.z);
                rng = rng_advance(rng, (g - base) * sc.light_draws);
                LightFragment f;
                float4 m;
                if (spec_light_sample<true>(&rng, sc, org, out.spec_org[base + 1], out.spec_org[base + 2],
                                      out.spec_org[base + 3], hdr.y, &f, &m)) {
                    dir = f4(f.dir.x, f.dir.y, f.dir.z, 0.0f);
                    dist = f.dist;
                    w = m;
                }
            }
        } else { // drawn by the camera pass
            org = out.spec_org[g];
            if (!(hdr.w < 0.0f)) {
                dir = f4(hdr.x, hdr.y, hdr.z, 0.0f);
                dist = hdr.w;
                w = out.spec_val[g];
            }
        }
        float4 contrib = zero4();
        if (!(dist < 0.0f)) {
            u32 o_ = 0;
            contrib = w * shadow_transmittance<KIND>(sc, org, dir, dist, &o_);
            ovf += o_ * step;
        }
        for (u32 i = 0; i < step; i++)
            out.spec_val[g + i] = contrib;
    }
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}



// Completes the emission of every pixel that deferred a specular NEE term: its listed terms are
// added to the prefix in path order, an NEE term as throughput * (sum of its samples in sample
// order / direct_samples) — the traced form's float operations, in the same order.
__global__ void __launch_bounds__(256) k_spec_resolve(LaunchCtx lc, TraceOut out) {
    const u32 gpix = lc.pix_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (gpix >= lc.pix_hi)
        return;
    const SceneDesc &sc = lc.scenes[lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gpix)];
    if (!sc.active)
        return;
    const u32 c = out.def_cnt[gpix];
    if (c & DEF_OVERFLOW) {
        atomicOr(lc.err, ERR_DEFER_OVERFLOW);
        return;
    }
    const u32 n = c & 0xffu;
    if (n == 0)
        return;
    const u32 ds = sc.direct_samples;
    float4 e = out.def_prefix[gpix];
    for (u32 i = 0; i < n; i++) {
        const size_t k = (size_t)gpix * DEF_MAX + i;
        const u32 tag = out.def_tag[k];
        const float4 v = out.def_val[k];
        if (tag == DEF_KNOWN) {
            e += v;
            continue;
        }
        float4 sum = zero4();
        for (u32 j = 0; j < ds; j++)
            sum += out.spec_val[tag + j];
        e += v * (sum / (float)ds);
    }
    out.emission[gpix] = (c & DEF_DIFFUSE) ? f4(e.x, e.y, e.z, 1.0f) : e;
}


void launch_spec_resolve(const LaunchCtx &lc, const TraceOut &out, cudaStream_t st) {
    if (!out.def_cnt || lc.pix_hi <= lc.pix_lo)
        return;
    k_spec_resolve<<<(lc.pix_hi - lc.pix_lo + 255) / 256, 256, 0, st>>>(lc, out);
}

// Sums each pixel's samples in sample order (trace_rays.cl:104-118).
__global__ void __launch_bounds__(256) k_nee_resolve(LaunchCtx lc, TraceOut out) {
    const u32 gpix = blockIdx.x * blockDim.x + threadIdx.x;
    if (gpix >= lc.total_pixels)
        return;
    if (out.emission[gpix].w != 1.0f)
        return;
    const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gpix);
    const SceneDesc &sc = lc.scenes[s];
    if (!sc.active)
        return;
    const u32 ds = sc.direct_samples;
    const float4 *v = out.nee_val + sc.nee_base + (size_t)(gpix - sc.pixel_base) * ds;
    float4 sum = zero4();
    for (u32 d = 0; d < ds; d++)
        sum += v[d];
    const float occl = out.direct[gpix].x;
    out.direct[gpix] = out.throughput[gpix] * occl * (sum / (float)ds);
}

// Draws the diffuse-NEE samples of every pixel with a diffuse hit point (one thread per pixel),
// from the RNG state and shading normal the camera pass left in the pixel's first sample slot.
__global__ void __launch_bounds__(128) k_nee_sample(LaunchCtx lc, TraceOut out) {
    const u32 gpix = lc.pix_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (gpix >= lc.pix_hi)
        return;
    if (out.emission[gpix].w != 1.0f)
        return; // no diffuse hit point
    const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gpix);
    const SceneDesc &sc = lc.scenes[s];
    if (!sc.active || sc.light_draws != LIGHT_DRAWS_VARY) // fixed draws: k_shadow draws each sample
        return;
    const u32 slot = sc.nee_base + (gpix - sc.pixel_base) * sc.direct_samples;
    Rng rng;
    rng.state = out.stash_rng[gpix];
    record_nee(sc, &rng, out.pos[gpix], out.stash_sn[gpix], out.base_color[gpix], out, slot);
}

template <int KIND, bool PER_PIXEL>
static void launch_shadow_kind(const LaunchCtx &lc, const TraceOut &out, u32 grid, u32 nee_blocks, const SceneDesc *one,
                               cudaStream_t st) {
    if (one)
        k_shadow<KIND, PER_PIXEL, true><<<grid, 128, 0, st>>>(lc, out, nee_blocks, *one);
    else
        k_shadow<KIND, PER_PIXEL, false><<<grid, 128, 0, st>>>(lc, out, nee_blocks, SceneDesc{});
}

void launch_shadow(const LaunchCtx &lc, const TraceOut &out, int kind, bool presample, bool per_pixel,
                   u32 n_pixels, const SceneDesc *one, cudaStream_t st) {
    if (!lc.nee_defer || lc.total_nee == 0)
        return;
    if (presample && lc.pix_hi > lc.pix_lo)
        k_nee_sample<<<(lc.pix_hi - lc.pix_lo + 127) / 128, 128, 0, st>>>(lc, out);
    per_pixel = per_pixel && !presample && lc.n_scenes == 1;
    const u32 nee_blocks = ((per_pixel ? n_pixels : lc.total_nee) + 127) / 128;
    const u32 spec_blocks = out.spec_ray && out.spec_cap ? (u32)g_sm_count * 8u : 0u;
    const u32 grid = nee_blocks + spec_blocks;
    if (lc.n_scenes != 1)
        one = nullptr;
    if (kind == SHADOW_OPAQUE && per_pixel)
        launch_shadow_kind<SHADOW_OPAQUE, true>(lc, out, grid, nee_blocks, one, st);
    else if (kind == SHADOW_OPAQUE)
        launch_shadow_kind<SHADOW_OPAQUE, false>(lc, out, grid, nee_blocks, one, st);
    else if (kind == SHADOW_CLEAR && per_pixel)
        launch_shadow_kind<SHADOW_CLEAR, true>(lc, out, grid, nee_blocks, one, st);
    else if (kind == SHADOW_CLEAR)
        launch_shadow_kind<SHADOW_CLEAR, false>(lc, out, grid, nee_blocks, one, st);
    else if (per_pixel)
        launch_shadow_kind<SHADOW_GENERAL, true>(lc, out, grid, nee_blocks, one, st);
    else
        launch_shadow_kind<SHADOW_GENERAL, false>(lc, out, grid, nee_blocks, one, st);
}

void launch_nee_resolve(const LaunchCtx &lc, const TraceOut &out, cudaStream_t st) {
    if (!lc.nee_defer || lc.total_pixels == 0)
        return;
    k_nee_resolve<<<(lc.total_pixels + 255) / 256, 256, 0, st>>>(lc, out);
}

void launch_trace(const LaunchCtx &lc, const TraceOut &out, int block, int persistent, int blocks_per_sm, u32 *queue,
                  bool untextured, cudaStream_t st) {
    if (lc.pix_hi <= lc.pix_lo)
        return;
    if (persistent && queue) {
        cudaMemsetAsync(queue, 0, sizeof(u32), st);
        int grid = g_sm_count * (blocks_per_sm > 0 ? blocks_per_sm : 8);
        if (untextured) // camera kernel 2.77 -> 2.44 ms (atrium), 1.04 -> 0.90 ms (caustic)
            k_trace_persistent<true><<<grid, 128, 0, st>>>(lc, out, queue);
        else
            k_trace_persistent<false><<<grid, 128, 0, st>>>(lc, out, queue);
    } else {
        (void)block;
        u32 grid = (lc.pix_hi - lc.pix_lo + 127) / 128;
        k_trace<<<grid, 128, 0, st>>>(lc, out);
    }
}

} // namespace phx
