// k_trace.cu — camera paths to the first diffuse hit with explicit direct lighting
// (kernels/trace_rays.cl:14-169), for every pixel of every scene of an engine.
//
// Two launch forms share one per-pixel body:
//  * one thread per pixel;
//  * persistent warps that drain a global pixel queue 32 pixels at a time.
// Pixel i of a scene uses pcg_seed(round_seed + i) exactly like the reference, so the result is
// independent of which lane or block traces it.
#include "dev_shading.cuh"
#include "kernels.hpp"

namespace phx {

PHX_DI void trace_pixel(const SceneDesc &sc, u32 seed, u32 tid, const TraceOut &out, u32 gpix, u32 *overflow) {
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
        SurfaceHit sh = process_hit(sc, h, origin, dir);
        const phx_material mat = sc.materials[sh.mat_index];
        float4 vol = white4();
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS) {
            vol = beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
            throughput *= vol;
        }
        float4 tangent, bitangent;
        hit_frame(sc, h, sh, &tangent, &bitangent);
        ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        emission += throughput * ctx.emissive;
        float4 view = -dir;
        BsdfSample bs = sample_bsdf(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE) {
            float4 sum = zero4();
            for (u32 d = 0; d < sc.direct_samples; d++)
                sum += direct_lighting_diffuse(&rng, sc, sh.position, ctx.shading_normal, ctx.base_color, overflow);
            emission = f4(emission.x, emission.y, emission.z, 1.0f);
            position = sh.position;
            normal = sh.normal;
            base_color = ctx.base_color;
            direct = throughput * ctx.occlusion * (sum / (float)sc.direct_samples);
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
    out.emission[gpix] = emission;
    out.pos[gpix] = position;
    out.normal[gpix] = normal;
    out.throughput[gpix] = throughput;
    out.base_color[gpix] = base_color;
    out.direct[gpix] = direct;
}

__global__ void __launch_bounds__(128) k_trace(LaunchCtx lc, TraceOut out) {
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.total_pixels)
        return;
    u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
    const SceneDesc &sc = lc.scenes[s];
    u32 ovf = 0;
    trace_pixel(sc, __ldg(&lc.seeds[s]), gid - sc.pixel_base, out, gid, &ovf);
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

// Persistent form: warps pull pixel indices from *queue until it is drained.
__global__ void __launch_bounds__(128) k_trace_persistent(LaunchCtx lc, TraceOut out, u32 *queue) {
    const u32 lane = threadIdx.x & 31u;
    u32 ovf = 0;
    for (;;) {
        u32 base = 0;
        if (lane == 0)
            base = atomicAdd(queue, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= lc.total_pixels)
            break;
        u32 gid = base + lane;
        if (gid < lc.total_pixels) {
            u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
            const SceneDesc &sc = lc.scenes[s];
            trace_pixel(sc, __ldg(&lc.seeds[s]), gid - sc.pixel_base, out, gid, &ovf);
        }
    }
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

void launch_trace(const LaunchCtx &lc, const TraceOut &out, int block, int persistent, int blocks_per_sm, u32 *queue,
                  cudaStream_t st) {
    if (lc.total_pixels == 0)
        return;
    if (persistent && queue) {
        cudaMemsetAsync(queue, 0, sizeof(u32), st);
        int grid = g_sm_count * (blocks_per_sm > 0 ? blocks_per_sm : 8);
        k_trace_persistent<<<grid, 128, 0, st>>>(lc, out, queue);
    } else {
        (void)block;
        u32 grid = (lc.total_pixels + 127) / 128;
        k_trace<<<grid, 128, 0, st>>>(lc, out);
    }
}

} // namespace phx
