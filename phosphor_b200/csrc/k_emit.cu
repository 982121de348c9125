// k_emit.cu — photon paths from the lights, stored at diffuse bounces
// (kernels/emit_photons.cl:12-114).
//
// Canonical order instead of atomic compaction.  The reference appends each stored photon at
// atomic_inc(n_photons) (emit_photons.cl:98), so its photon order depends on scheduling.  Here
// path t writes its j-th stored photon to slot (j, t) of a slot array laid out slot-major
// (slot_base + j*n_emit + t: lanes of a warp store to consecutive addresses) and its store count
// to counts[t].  An exclusive scan of the counts then places photon (t, j) at offsets[t] + j —
// the order a sequential run of emit_photons.cl produces — and the compaction is fused into the
// hash kernel.  A path stores at most one photon per bounce, so max_bounces slots per path
// always suffice, exactly like the reference's photons*max_bounces buffer (renderer.cpp:40).
//
// Two forms produce identical results: k_emit (one thread per path) and k_emit_persistent, where
// each lane runs one path as a state machine (one ray query per step) and the warp refills lanes
// whose path ended with new paths (__ballot_sync / __popc, one atomicAdd per refill), so short
// paths (escapes, Russian roulette) do not leave lanes idle while long ones bounce.
#include "dev_shading.cuh"
#include "kernels.hpp"

// Minimum resident blocks per SM asked of the compiler (caps registers per thread at 64): 8 blocks
// per SM measured fastest for the photon kernel (6.3 -> 5.4 ms; 10 or 12 spill too much).
#ifndef PHX_EMIT_MINB
#define PHX_EMIT_MINB 8
#endif

namespace phx {

PHX_DI u32 emit_path(const SceneDesc &sc, u32 seed, u32 tid, const EmitOut &out, u32 *overflow) {
    u32 n_out = 0;
    const u64 stride = sc.n_emit;
    u64 slot = sc.slot_base + tid;
    Rng rng = pcg_seed(seed + tid);
    float4 origin, dir, power;
    sample_light(&rng, sc, &origin, &dir, &power);
    IorStack ior;
    init_ior_stack(&ior, AIR_IOR);
    float4 throughput = f4(1.0f, 1.0f, 1.0f, 0.0f);
    for (u32 depth = 0; depth < sc.max_bounces; depth++) {
        Hit h;
        bool hit = intersect(sc, origin, dir, EPS, INF, &h, overflow);
        if (!hit)
            return n_out;
        const phx_material mat = sc.materials[tri_mat(sc, h.tri)];
        SurfaceHit sh = process_hit(sc, h, origin, dir, mat_textured(mat));
        float4 vol = white4();
        float cur = current_ior(&ior);
        if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS) {
            vol = beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
            power *= vol;
            throughput *= vol;
        }
        float4 tangent = zero4(), bitangent = zero4(); // the frame only serves a normal map
        if (mat.norm_index != NO_TEXTURE)
            hit_frame(sc, h, sh, &tangent, &bitangent);
        ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
        if (depth >= RR_MIN_PHOTON_DEPTH) {
            float q = fmaxf(throughput.x, fmaxf(throughput.y, throughput.z));
            q = clampf(q, RR_MIN_Q, RR_MAX_Q);
            if (random_float(&rng) > q)
                return n_out;
            float inv_q = 1.0f / q;
            throughput *= inv_q;
            power *= inv_q;
        }
        float4 view = -dir;
        BsdfSample bs = sample_bsdf(&rng, ctx, ctx.shading_normal, sh.normal, view, &ior, sh.front_face);
        if (bs.event == BSDF_DIFFUSE && dot(dir, sh.normal) < 0.0f) {
            out.slot_pos[slot] = sh.position;
            out.slot_pd[slot] = make_uint2(encode_rgbe(power), encode_oct(dir));
            if (out.slot_pow)
                out.slot_pow[slot] = power;
            slot += stride;
            n_out++;
        }
        power *= bs.throughput;
        throughput *= bs.throughput;
        float4 side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
        origin = sh.position + bs.dir * EPS + side * EPS;
        dir = bs.dir;
    }
    return n_out;
}

__global__ void __launch_bounds__(128) k_emit(LaunchCtx lc, EmitOut out) {
    u32 gid = lc.emit_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.emit_hi)
        return;
    u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.emit_bases, lc.n_scenes, gid);
    const SceneDesc &sc = lc.scenes[s];
    if (!sc.active) { // retired batch scene: no photons
        out.counts[gid] = 0;
        return;
    }
    u32 ovf = 0;
    out.counts[gid] = emit_path(sc, __ldg(&lc.seeds[s]), gid - sc.emit_base, out, &ovf);
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

// ---- state machine with lane refill -------------------------------------------------------------
// One photon path per lane, one ray query per step (emit_photons.cl:49-113 split at
// scene_intersect); a lane whose path ends is refilled with the next path of the queue.
struct PhotonPath {
    const SceneDesc *sc;
    u32 gid, n_out, depth;
    u64 slot;
    Rng rng;
    float4 origin, dir, power, throughput;
    IorStack ior;
};

// PRE: the path starts from the state k_emit_start left in its own first three photon slots — its
// light sample (origin, direction, power) and the RNG state after it; the path overwrites them only
// when it stores photons, later.  Otherwise it draws its light sample here.
template <bool PRE>
PHX_DI void pp_start(PhotonPath &p, const SceneDesc *sc, u32 seed, u32 tid, u32 gid, const EmitOut &out) {
    p.sc = sc;
    p.gid = gid;
    p.n_out = 0;
    p.depth = 0;
    p.slot = sc->slot_base + tid;
    if constexpr (PRE) {
        const u64 n = sc->n_emit;
        p.origin = out.slot_pos[p.slot];
        p.dir = out.slot_pos[p.slot + n];
        p.power = out.slot_pos[p.slot + 2 * n];
        p.rng.state = out.slot_pd[p.slot].x;
    } else {
        p.rng = pcg_seed(seed + tid);
        sample_light(&p.rng, *sc, &p.origin, &p.dir, &p.power);
    }
    init_ior_stack(&p.ior, AIR_IOR);
    p.throughput = f4(1.0f, 1.0f, 1.0f, 0.0f);
}

// The light samples that start the photon paths, drawn for every path at once (one thread per
// path, all lanes busy) before the lane-refill kernel, which would otherwise draw them for the few
// lanes it refills at a time.  The same draws from the same streams: the paths are unchanged.
// Needs three photon slots per path (max_bounces >= 3) in every scene.  Photon kernel 4.43 -> 4.01
// ms on the caustic workload, 2.73 -> 2.68 ms on the atrium one.
__global__ void __launch_bounds__(128) k_emit_start(LaunchCtx lc, EmitOut out) {
    const u32 gid = lc.emit_lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.emit_hi)
        return;
    const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.emit_bases, lc.n_scenes, gid);
    const SceneDesc &sc = lc.scenes[s];
    if (!sc.active)
        return;
    const u32 tid = gid - sc.emit_base;
    Rng rng = pcg_seed(__ldg(&lc.seeds[s]) + tid);
    float4 origin, dir, power;
    sample_light(&rng, sc, &origin, &dir, &power);
    const u64 b = sc.slot_base + tid, n = sc.n_emit;
    out.slot_pos[b] = origin;
    out.slot_pos[b + n] = dir;
    out.slot_pos[b + 2 * n] = power;
    out.slot_pd[b].x = rng.state;
}

// Consumes the pending query; returns true while the path continues.  NOTEX: no material of the
// context has a texture (texture indices never change after set-up), so every texture branch is
// compiled out of this instance.
template <bool NOTEX>
PHX_DI bool pp_advance(PhotonPath &p, bool hit, const Hit &h, const EmitOut &out) {
    const SceneDesc &sc = *p.sc;
    if (!hit)
        return false;
    phx_material mat = sc.materials[tri_mat(sc, h.tri)];
    if constexpr (NOTEX)
        mat.diff_index = mat.emis_index = mat.norm_index = mat.occlusion_index = mat.metal_rough_index =
            mat.transmission_index = NO_TEXTURE;
    SurfaceHit sh = process_hit(sc, h, p.origin, p.dir, mat_textured(mat));
    float cur = current_ior(&p.ior);
    if (cur != AIR_IOR && mat.thickness > EPS && mat.att_dist > EPS) {
        float4 vol = beer_lambert(f4(mat.att_color), mat.att_dist, sh.t);
        p.power *= vol;
        p.throughput *= vol;
    }
    float4 tangent = zero4(), bitangent = zero4(); // the frame only serves a normal map
    if (mat.norm_index != NO_TEXTURE)
        hit_frame(sc, h, sh, &tangent, &bitangent);
    ShadingContext ctx = evaluate_material(sc, mat, sh.mat_index, sh.uvx, sh.uvy, sh.normal, tangent, bitangent);
    if (p.depth >= RR_MIN_PHOTON_DEPTH) {
        float q = fmaxf(p.throughput.x, fmaxf(p.throughput.y, p.throughput.z));
        q = clampf(q, RR_MIN_Q, RR_MAX_Q);
        if (random_float(&p.rng) > q)
            return false;
        float inv_q = 1.0f / q;
        p.throughput *= inv_q;
        p.power *= inv_q;
    }
    float4 view = -p.dir;
    BsdfSample bs = sample_bsdf(&p.rng, ctx, ctx.shading_normal, sh.normal, view, &p.ior, sh.front_face);
    if (bs.event == BSDF_DIFFUSE && dot(p.dir, sh.normal) < 0.0f) {
        out.slot_pos[p.slot] = sh.position;
        out.slot_pd[p.slot] = make_uint2(encode_rgbe(p.power), encode_oct(p.dir));
        p.slot += sc.n_emit;
        p.n_out++;
    }
    p.power *= bs.throughput;
    p.throughput *= bs.throughput;
    float4 side = (dot(bs.dir, sh.normal) > 0.0f) ? sh.normal : -sh.normal;
    p.origin = sh.position + bs.dir * EPS + side * EPS;
    p.dir = bs.dir;
    p.depth++;
    return p.depth < sc.max_bounces;
}

template <bool NOTEX, bool PRE>
__global__ void __launch_bounds__(128, PHX_EMIT_MINB) k_emit_persistent(LaunchCtx lc, EmitOut out, u32 *queue) {
    const u32 lane = threadIdx.x & 31u;
    const u32 lt_mask = (1u << lane) - 1u;
    u32 ovf = 0;
    PhotonPath p;
    bool active = false, exhausted = false;
    for (;;) {
        const u32 need = __ballot_sync(0xffffffffu, !active && !exhausted);
        if (need) {
            const u32 leader = __ffs(need) - 1;
            u32 base = 0;
            if (lane == leader)
                base = atomicAdd(queue, (u32)__popc(need));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!active && !exhausted) {
                const u32 gid = lc.emit_lo + base + __popc(need & lt_mask);
                if (gid < lc.emit_hi) {
                    const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.emit_bases, lc.n_scenes, gid);
                    const SceneDesc *sc = lc.scenes + s;
                    pp_start<PRE>(p, sc, __ldg(&lc.seeds[s]), gid - sc->emit_base, gid, out);
                    active = true;
                    if (sc->max_bounces == 0 || !sc->active) { // retired batch scene: no photons
                        out.counts[gid] = 0;
                        active = false;
                    }
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active))
            break;
        if (active) {
            Hit h;
            const bool hit = intersect(*p.sc, p.origin, p.dir, EPS, INF, &h, &ovf);
            if (!pp_advance<NOTEX>(p, hit, h, out)) {
                out.counts[p.gid] = p.n_out;
                active = false;
            }
        }
    }
    if (ovf)
        atomicAdd(lc.overflow, ovf);
}

void launch_emit(const LaunchCtx &lc, const EmitOut &out, int block, int persistent, int blocks_per_sm, u32 *queue,
                 bool untextured, bool prestart, cudaStream_t st) {
    if (lc.emit_hi <= lc.emit_lo)
        return;
    if (persistent && queue && !out.slot_pow) {
        cudaMemsetAsync(queue, 0, sizeof(u32), st);
        if (prestart)
            k_emit_start<<<(lc.emit_hi - lc.emit_lo + 127) / 128, 128, 0, st>>>(lc, out);
        int grid = g_sm_count * (blocks_per_sm > 0 ? blocks_per_sm : 8);
        // untextured: emit 4.52 -> 4.44 ms (caustic), 2.82 -> 2.73 ms (atrium)
        if (untextured && prestart)
            k_emit_persistent<true, true><<<grid, 128, 0, st>>>(lc, out, queue);
        else if (untextured)
            k_emit_persistent<true, false><<<grid, 128, 0, st>>>(lc, out, queue);
        else if (prestart)
            k_emit_persistent<false, true><<<grid, 128, 0, st>>>(lc, out, queue);
        else
            k_emit_persistent<false, false><<<grid, 128, 0, st>>>(lc, out, queue);
    } else {
        (void)block;
        u32 grid = (lc.emit_hi - lc.emit_lo + 127) / 128;
        k_emit<<<grid, 128, 0, st>>>(lc, out);
    }
}

} // namespace phx
