// engine_adjoint.cu — parameter updates and the forward / backward passes of the adjoint
// (kernels in k_adjoint.cu).  No counterpart in the reference.
//
// Forward: a fresh render of R rounds (state cleared) through the ordinary round, recording per
// round the seed, and per pixel the search radius² and the SPPM ratio its gather applied; returns
// the linear image radiance/R + flux/(π r² N).  Backward: for each round, restores its seed,
// re-creates its hit points and photons with the ordinary kernels (the emit pass also keeps the
// unquantised photon power), then runs the gather adjoint and the camera- and photon-path replays.
// Nothing per path vertex is stored between the passes.  Any later round, gather, state write or
// parameter change invalidates the recording.
#include "engine.hpp"

#include <cstring>

namespace phx {

#define CK(x)                                                                                                          \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return fail(PHX_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
    } while (0)

namespace {
int ensure(DevBuf &b, size_t bytes) {
    if (b.p && b.bytes >= bytes)
        return PHX_OK;
    return b.alloc(bytes);
}
} // namespace

uint32_t Engine::n_params() const {
    return sc.size() == 1 ? 4 * (uint32_t)sc[0].mats.size() + 3 * (uint32_t)sc[0].lights.size() : 0;
}

int Engine::set_materials(const phx_material *m, uint32_t n) {
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "materials can only be replaced on single-scene contexts");
    SceneSlot &S = sc[0];
    if (!m || n != S.mats.size())
        return fail(PHX_E_INVALID, "material count differs from the scene's");
    for (uint32_t i = 0; i < n; i++) {
        const phx_material &a = S.mats[i], &b = m[i];
        if (a.diff_index != b.diff_index || a.emis_index != b.emis_index || a.norm_index != b.norm_index ||
            a.occlusion_index != b.occlusion_index || a.metal_rough_index != b.metal_rough_index ||
            a.transmission_index != b.transmission_index)
            return fail(PHX_E_INVALID, "texture indices of a material cannot change");
    }
    adjoint_invalidate();
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(S.bufs[9].p, m, sizeof(phx_material) * n, cudaMemcpyHostToDevice));
    S.mats.assign(m, m + n);
    S.desc.any_transmissive = 0;
    for (const auto &mm : S.mats)
        if (!(mm.transmission < 1e-5f)) // not blocking a shadow ray (NaN included)
            S.desc.any_transmissive = 1;
    invalidate_graph(); // the shadow kernel captured for the scene's kind may no longer fit
    return upload_descs();
}

int Engine::set_lights(const phx_light *l, uint32_t n) {
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "lights can only be replaced on single-scene contexts");
    SceneSlot &S = sc[0];
    if ((n && !l) || n != S.lights.size())
        return fail(PHX_E_INVALID, "light count differs from the scene's");
    for (uint32_t i = 0; i < n; i++)
        if (l[i].kind != S.lights[i].kind ||
            (l[i].kind == PHX_LIGHT_TEXTURED && std::memcmp(&l[i].aux, &S.lights[i].aux, sizeof(phx_f4)) != 0))
            return fail(PHX_E_INVALID, "light kinds and emissive-triangle ranges cannot change");
    if (n == 0)
        return PHX_OK;
    adjoint_invalidate();
    std::vector<float> lum(n);
    lum_pref_sum(l, n, lum.data()); // scene_data.cpp:14-23
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(S.bufs[13].p, l, sizeof(phx_light) * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.bufs[14].p, lum.data(), 4 * (size_t)n, cudaMemcpyHostToDevice));
    S.lights.assign(l, l + n);
    S.desc.total_lum = lum[n - 1]; // shading.cpp:26
    S.desc.light_draws = light_sample_draws(l, n, S.desc.total_lum);
    invalidate_graph(); // the captured shadow stage depends on the draw count
    return upload_descs();
}

int Engine::adjoint_forward(uint32_t rounds, float *image) {
    if (sc.size() != 1 || shard.world > 1)
        return fail(PHX_E_UNSUPPORTED, "the adjoint is only available on single-scene, unsharded contexts");
    if (rounds == 0 || rounds > 4096)
        return fail(PHX_E_INVALID, "rounds must be 1..4096");
    SceneSlot &S = sc[0];
    const uint32_t P = total_pixels;
    const size_t rp = (size_t)rounds * P;
    int r;
    if ((r = ensure(adj_seeds, 4 * (size_t)rounds)) || (r = ensure(adj_r2, 4 * rp)) ||
        (r = ensure(adj_ratio, 4 * rp)) || (r = ensure(adj_k, 4 * rp)) || (r = ensure(adj_img, 12 * (size_t)P)))
        return r;
    adj_ready = false;
    CK(cudaStreamSynchronize(st));
    CK(cudaMemsetAsync(flux.p, 0, 16 * (size_t)P, st));
    CK(cudaMemsetAsync(weight.p, 0, 4 * (size_t)P, st));
    CK(cudaMemsetAsync(radiance.p, 0, 16 * (size_t)P, st));
    S.rounds = 0;
    S.total_emitted = 0;
    in_adjoint = true;
    for (uint32_t n = 0; n < rounds; n++) {
        rec_r2 = adj_r2.as<float>() + (size_t)n * P;
        rec_ratio = adj_ratio.as<float>() + (size_t)n * P;
        r = plain_round();
        if (!r && cudaMemcpyAsync(adj_seeds.as<u32>() + n, d_seeds.p, 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            r = fail(PHX_E_CUDA, "seed copy failed");
        if (r) {
            rec_r2 = rec_ratio = nullptr;
            in_adjoint = false;
            return r;
        }
    }
    rec_r2 = rec_ratio = nullptr;
    in_adjoint = false;
    const float inv_n = 1.0f / ((float)S.prm.photons_per_round * (float)rounds);
    launch_adj_image(flux.as<float4>(), radiance.as<float4>(), P, 1.0f / (float)rounds, inv_n, adj_img.as<float>(), st);
    CK(cudaGetLastError());
    if (image)
        CK(cudaMemcpyAsync(image, adj_img.p, 12 * (size_t)P, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    adj_rounds = rounds;
    adj_ready = true;
    adj_k_ready = false;
    return PHX_OK;
}

int Engine::adjoint_backward(const float *dl_dimage, float *grad, uint32_t n_grad) {
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "the adjoint is only available on single-scene contexts");
    if (!adj_ready)
        return fail(PHX_E_STATE, "adjoint_backward needs an adjoint_forward with no round, gather, state write or "
                                 "parameter change in between");
    const uint32_t np = n_params();
    if (!dl_dimage || !grad || n_grad < np)
        return fail(PHX_E_INVALID, "need dL/dI for every pixel and room for every parameter");
    SceneSlot &S = sc[0];
    const uint32_t P = total_pixels, R = adj_rounds;
    int r;
    if ((r = ensure(adj_g, 16 * (size_t)P)) || (r = ensure(adj_gT, 16 * (size_t)P)) ||
        (r = ensure(adj_gA, 16 * (size_t)P)) || (r = ensure(adj_gphi, 16 * max_photons)) ||
        (r = ensure(adj_slot_pow, 16 * total_slots)) || (r = ensure(adj_ph_pow, 16 * max_photons)) ||
        (r = ensure(adj_grad, 8 * (size_t)std::max(np, 1u))))
        return r;
    std::vector<float4> g(P);
    for (uint32_t i = 0; i < P; i++)
        g[i] = make_float4(dl_dimage[3 * (size_t)i], dl_dimage[3 * (size_t)i + 1], dl_dimage[3 * (size_t)i + 2], 0.0f);
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(adj_g.p, g.data(), 16 * (size_t)P, cudaMemcpyHostToDevice));
    if (!adj_k_ready) {
        const float inv_n = 1.0f / ((float)S.prm.photons_per_round * (float)R);
        launch_adj_scale(adj_ratio.as<float>(), adj_k.as<float>(), flux.as<float4>(), P, R, inv_n, st);
        adj_k_ready = true;
    }
    CK(cudaMemsetAsync(adj_grad.p, 0, 8 * (size_t)std::max(np, 1u), st));
    AdjBufs ab{};
    ab.g_img = adj_g.as<float4>();
    ab.gT = adj_gT.as<float4>();
    ab.gA = adj_gA.as<float4>();
    ab.gphi = adj_gphi.as<float4>();
    ab.ph_pow = adj_ph_pow.as<float4>();
    ab.offsets = offsets.as<u32>();
    ab.grad = adj_grad.as<double>();
    ab.n_params = np;
    ab.n_mat = (u32)S.mats.size();
    ab.inv_rounds = 1.0f / (float)R;
    ab.block_sums = 4 * (size_t)np <= 32768 ? 1u : 0u;
    in_adjoint = true;
    for (uint32_t n = 0; n < R && !r; n++) {
        if (cudaMemcpyAsync(d_seeds.p, adj_seeds.as<u32>() + n, 4, cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
            r = fail(PHX_E_CUDA, "seed copy failed");
            break;
        }
        enq_trace();
        // photons of the round, keeping their unquantised power
        EmitOut eo{slot_pos.as<float4>(), slot_pd.as<uint2>(), counts.as<u32>(), adj_slot_pow.as<float4>()};
        launch_emit(lc(), eo, (int)tune.emit_block, 0, 0, nullptr, untextured(), false, st);
        launch_scan(counts.as<u32>(), offsets.as<u32>(), (u64)total_emit + 1, scan_scr.p, d_ntotal.as<u32>(),
                    d_err.as<u32>(), st);
        launch_compact(lc(), gb(), st);
        launch_compact_pow(lc(), adj_slot_pow.as<float4>(), counts.as<u32>(), offsets.as<u32>(),
                           adj_ph_pow.as<float4>(), st);
        stage_state |= 2;
        enq_hash_sort();
        if (cudaMemsetAsync(adj_gphi.p, 0, 16 * max_photons, st) != cudaSuccess) {
            r = fail(PHX_E_CUDA, "memset failed");
            break;
        }
        ab.kscale = adj_k.as<float>() + (size_t)n * P;
        ab.r2 = adj_r2.as<float>() + (size_t)n * P;
        ab.perm = perm;
        GatherBufs gbuf{hp[0].as<float4>(), hp[1].as<float4>(), hp[2].as<float4>(), hp[3].as<float4>(),
                        hp[4].as<float4>(), hp[5].as<float4>(), s_posdir.as<float4>(), s_power.as<u32>(),
                        s_dir.as<float4>(), s_pow.as<float4>(), cell_start.as<u32>(), (u32)max_photons,
                        flux.as<float4>(), weight.as<float>(), radiance.as<float4>(), nullptr, nullptr};
        launch_gather_adj(lc(), gbuf, ab, st);
        launch_trace_adj(lc(), ab, st);
        launch_emit_adj(lc(), ab, st);
        if (cudaGetLastError() != cudaSuccess)
            r = fail(PHX_E_CUDA, "adjoint kernel launch failed");
    }
    in_adjoint = false;
    if (r)
        return r;
    if ((r = sync_and_check()))
        return r;
    std::vector<double> gd(std::max(np, 1u));
    CK(cudaMemcpy(gd.data(), adj_grad.p, 8 * (size_t)np, cudaMemcpyDeviceToHost));
    for (uint32_t i = 0; i < np; i++)
        grad[i] = (float)gd[i];
    return PHX_OK;
}

} // namespace phx
