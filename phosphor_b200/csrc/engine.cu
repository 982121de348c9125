// engine.cu — Engine: scene upload, device memory, stage enqueueing, the plain per-pass form
// (Renderer::run, src/renderer/renderer.cpp:59-161, with its two host syncs per round) and the
// graph form (one captured round replayed with no host sync).
#include "engine.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <chrono>
#include <thread>

namespace phx {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define CK(x)                                                                                                          \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return fail(PHX_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
    } while (0)

void init_kernels(int device);

int DevBuf::alloc(size_t b) {
    release();
    bytes = b;
    if (cudaMalloc(&p, b ? b : 16) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return fail(PHX_E_OOM, "device allocation of " + std::to_string(b) + " bytes failed");
    }
    return PHX_OK;
}

void DevBuf::release() {
    if (p)
        cudaFree(p);
    p = nullptr;
    bytes = 0;
}

Engine::~Engine() {
    if (st)
        cudaStreamSynchronize(st);
    shard_release();
    invalidate_graph();
    for (auto &v : xbufs)
        for (auto &b : v)
            b.release();
    for (auto s : pipe_st)
        if (s)
            cudaStreamDestroy(s);
    for (auto e : pipe_ev)
        if (e)
            cudaEventDestroy(e);
    for (auto &e : events)
        if (e)
            cudaEventDestroy(e);
    for (auto &e : seed_ev)
        if (e)
            cudaEventDestroy(e);
    if (h_seed_ring)
        cudaFreeHost(h_seed_ring);
    for (auto &s : sc)
        for (auto &b : s.bufs)
            b.release();
    DevBuf *all[] = {&d_desc, &d_pix_bases, &d_emit_bases, &d_nee_bases, &nee_ray, &nee_val, &stash_sn, &stash_rng,
                     &spec_ray, &spec_val,
                     &spec_org, &spec_pix, &spec_next, &def_cnt, &def_prefix, &def_val, &def_tag, &d_seeds, &d_rng,
                     &d_err, &d_ovf, &d_queue, &d_ntotal,
                     &flux, &weight, &radiance, &slot_pos, &slot_pd, &counts, &offsets, &ph_pos, &ph_pd, &keys,
                     &cell_count, &cell_start, &sk0, &sk1, &sv0, &sv1, &s_posdir, &s_power, &s_dir, &s_pow, &scan_scr, &radix_scr,
                     &img_rgb, &img_ldr, &pk_keys, &pk_t0, &pk_t1, &pk_v0, &pk_v1, &pk_scr, &d_npix, &adj_seeds, &adj_r2, &adj_ratio, &adj_k, &adj_img, &adj_g, &adj_gT,
                     &adj_gA, &adj_gphi, &adj_slot_pow, &adj_ph_pow, &adj_grad};
    for (auto *b : all)
        b->release();
    for (auto &b : hp)
        b.release();
    if (h_pinned)
        cudaFreeHost(h_pinned);
    if (fork_ev)
        cudaEventDestroy(fork_ev);
    if (join_ev)
        cudaEventDestroy(join_ev);
    if (st_side)
        cudaStreamDestroy(st_side);
    if (st)
        cudaStreamDestroy(st);
}

static int upload(DevBuf &b, const void *src, size_t bytes) {
    int r = b.alloc(bytes);
    if (r)
        return r;
    if (bytes && src)
        CK(cudaMemcpy(b.p, src, bytes, cudaMemcpyHostToDevice));
    else
        CK(cudaMemset(b.p, 0, bytes ? bytes : 16));
    return PHX_OK;
}

static int check_params(const phx_params &p) {
    if (p.width == 0 || p.height == 0 || (uint64_t)p.width * p.height > 0x7fffffffull)
        return fail(PHX_E_INVALID, "image size out of range");
    if (p.photons_per_round == 0)
        return fail(PHX_E_INVALID, "photons_per_round must be positive");
    if (p.max_photon_bounces < 1 || p.max_photon_bounces > 32)
        return fail(PHX_E_INVALID, "max_photon_bounces must be in 1..32 (cmd_args.hpp:49)");
    if (p.grid_res < 1 || p.grid_res > 255)
        return fail(PHX_E_INVALID, "grid_res must be in 1..255 (cmd_args.hpp:51)");
    if (p.direct_samples < 1 || p.direct_samples > 128)
        return fail(PHX_E_INVALID, "direct_samples must be in 1..128 (cmd_args.hpp:59)");
    if (!(p.sppm_alpha >= 0.0f))
        return fail(PHX_E_INVALID, "sppm_alpha must be non-negative");
    return PHX_OK;
}

// RNG draws one light sample takes (sample_light_fragment): none without light, one to choose the
// light, and for an area light of nonzero area one more to choose its triangle (when it has
// several) and two for the point.  LIGHT_DRAWS_VARY when the lights differ: a sample's draws then
// depend on which light it chose.
uint32_t light_sample_draws(const phx_light *l, uint32_t n, float total_lum) {
    const float eps = 1e-5f;
    if (n == 0 || total_lum < eps)
        return 0;
    uint32_t draws = LIGHT_DRAWS_VARY;
    for (uint32_t k = 0; k < n; k++) {
        uint32_t d = 1;
        if (l[k].kind != PHX_LIGHT_POINT && l[k].kind != PHX_LIGHT_SPOT && l[k].kind != PHX_LIGHT_DIRECTIONAL) {
            const float area = l[k].aux.w;
            uint32_t ntri;
            std::memcpy(&ntri, &l[k].aux.z, 4);
            if (!(area < eps))
                d = 1 + ((ntri <= 1 || area <= eps) ? 0 : 1) + 2;
        }
        if (k == 0)
            draws = d;
        else if (d != draws)
            return LIGHT_DRAWS_VARY;
    }
    return draws;
}

static float ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// The SAH traversal tree built on the device (k_bvh.cu) while a host thread builds the reference
// tree, whose leaf ranks only the last step needs.  done = false: the caller builds on the host
// (force_ref: the SAH tree is too deep for the traversal stack, use the reference tree).
static int device_traversal(SceneSlot &S, const phx_scene &s, const phx_params &p, cudaStream_t st, bool &ref_built,
                            bool &done, bool &force_ref, int32_t &root, bool &wide) {
    const uint32_t n = s.n_triangles;
    DevBuf tris, rank;
    int r;
    if ((r = upload(tris, s.triangles, sizeof(phx_triangle) * (size_t)n)))
        return r;
    bool ref_ok = false;
    std::vector<uint32_t> ranks;
    std::thread ref([&] {
        ref_ok = bvh_build(s.triangles, n, S.nodes, &S.depth);
        if (ref_ok)
            ranks = reference_leaf_ranks(S.nodes, n);
    });
    DeviceBvh db;
    std::string msg;
    const bool want_wide = !(p.flags & PHX_F_BINARY_BVH);
    const int rc =
        bvh_device_build(tris.as<phx_triangle>(), n, p.bvh_leaf_size ? p.bvh_leaf_size : 4u, want_wide, st, db, msg);
    ref.join();
    ref_built = ref_ok;
    struct Release {
        DeviceBvh &b;
        ~Release() { b.release(); }
    } release{db};
    if (!ref_ok)
        return fail(PHX_E_INVALID, "degenerate or infinite triangle bounding box (bounding_box.h:17-28)");
    if (rc)
        return fail(rc == 2 ? PHX_E_OOM : rc == 1 ? PHX_E_INVALID : PHX_E_CUDA, msg);
    if (!(db.depth + 2 < (uint32_t)TRAV_STACK)) {
        force_ref = true;
        return PHX_OK;
    }
    wide = want_wide && 3 * db.wdepth + 4 < (uint32_t)TRAV_STACK;
    const bool quant = wide && (p.flags & PHX_F_QUANT_BVH);
    const float *nodes = wide ? db.wnodes : db.cnodes;
    const uint32_t n_nodes = wide ? db.n_wide : db.n_inner, per = quant ? 16u : wide ? 28u : 16u;
    S.trav_depth = wide ? db.wdepth : db.depth;
    S.trav_inner = n_nodes;
    root = wide ? db.wroot : db.root;
    if ((r = upload(S.bufs[0], nullptr, std::max<size_t>((size_t)n_nodes * per, 4) * 4)) ||
        (r = S.bufs[1].alloc((size_t)n * 48)) || (r = S.bufs[2].alloc((size_t)n * 48)) ||
        (r = S.bufs[3].alloc((size_t)n * 48)) || (r = S.bufs[4].alloc((size_t)n * 32)) ||
        (r = upload(rank, ranks.data(), 4 * (size_t)n)))
        return r;
    if (n_nodes && quant)
        CK(bvh_device_quantize(db.wnodes, n_nodes, S.bufs[0].as<u32>(), st));
    else if (n_nodes)
        CK(cudaMemcpyAsync(S.bufs[0].p, nodes, (size_t)n_nodes * per * 4, cudaMemcpyDeviceToDevice, st));
    if (bvh_device_finish(tris.as<phx_triangle>(), rank.as<u32>(), n, db, S.bufs[1].as<float4>(),
                          S.bufs[2].as<float4>(), S.bufs[3].as<float4>(), S.bufs[4].as<float4>(), st))
        return fail(PHX_E_CUDA, "device BVH triangle records: launch failed");
    CK(cudaStreamSynchronize(st));
    done = true;
    return PHX_OK;
}

int Engine::upload_scene(uint32_t i, const phx_scene &s, const phx_params &p, uint32_t *pix, uint32_t *emit,
                         uint32_t *cell, uint64_t *slot) {
    SceneSlot &S = sc[i];
    S.prm = p;
    const auto t_setup = std::chrono::steady_clock::now();
    if (!s.triangles || s.n_triangles == 0)
        return fail(PHX_E_INVALID, "scene has no triangles");
    if (!s.materials || s.n_materials == 0)
        return fail(PHX_E_INVALID, "scene has no materials");
    for (uint32_t t = 0; t < s.n_triangles; t++)
        if (s.triangles[t].mat_index >= s.n_materials)
            return fail(PHX_E_INVALID, "triangle material index out of range");
    for (uint32_t l = 0; l < s.n_lights; l++)
        if (s.lights[l].kind == PHX_LIGHT_TEXTURED) {
            uint32_t a, b;
            std::memcpy(&a, &s.lights[l].aux.y, 4);
            std::memcpy(&b, &s.lights[l].aux.z, 4);
            if ((uint64_t)a + b > s.n_emissive_triangles)
                return fail(PHX_E_INVALID, "emissive light triangle range out of bounds");
        }
    if (s.n_textures && (!s.tex_meta || !s.tex_atlas))
        return fail(PHX_E_INVALID, "textures declared without data");
    for (uint32_t k = 0; k < s.n_textures; k++) {
        const phx_texture_meta &m = s.tex_meta[k];
        // texel reads stay inside the atlas (material.h:84-122 index width*height*channels bytes, and
        // naive_sample_texture assumes 3 channels)
        if (m.width == 0 || m.height == 0 || m.channels < 3 ||
            (uint64_t)m.atlas_offset + (uint64_t)m.width * m.height * m.channels > s.tex_atlas_bytes)
            return fail(PHX_E_INVALID, "texture extends past the atlas or has fewer than 3 channels");
    }
    if (s.envmap && (s.envmap_width == 0) != (s.envmap_height == 0))
        return fail(PHX_E_INVALID, "envmap with a zero dimension");
    for (uint32_t m = 0; m < s.n_materials; m++) {
        const phx_material &mm = s.materials[m];
        const uint32_t idx[6] = {mm.diff_index, mm.emis_index, mm.norm_index, mm.occlusion_index,
                                 mm.metal_rough_index, mm.transmission_index};
        for (uint32_t k : idx)
            if (k != PHX_NO_TEXTURE && k >= s.n_textures)
                return fail(PHX_E_INVALID, "material texture index out of range");
    }
    const uint32_t n = s.n_triangles;
    S.n_tris = n;
    S.bufs.resize(16);
    int r;
    int32_t trav_root = 0;
    bool wide = false, trav_done = false, ref_built = false, force_ref = false;
    if (!(p.flags & PHX_F_HOST_BVH) && !(p.flags & PHX_F_REFERENCE_BVH) &&
        (r = device_traversal(S, s, p, st, ref_built, trav_done, force_ref, trav_root, wide)))
        return r;
    const bool quant_req = (p.flags & PHX_F_QUANT_BVH) != 0;
    if (!trav_done) {
        if (!ref_built && !bvh_build(s.triangles, s.n_triangles, S.nodes, &S.depth))
            return fail(PHX_E_INVALID, "degenerate or infinite triangle bounding box (bounding_box.h:17-28)");
        // Traversal tree: binned SAH over the same expanded boxes (fewer node visits), or the
        // reference tree itself.  Either returns the reference's hit for every ray: the closest t,
        // ties broken by the reference leaf rank carried in each triangle record.
        PackedBvh pk;
        bool sah = !(p.flags & PHX_F_REFERENCE_BVH) && !force_ref;
        if (sah) {
            std::vector<uint32_t> ranks = reference_leaf_ranks(S.nodes, s.n_triangles);
            sah = bvh_build_sah(s.triangles, s.n_triangles, ranks, p.bvh_leaf_size ? p.bvh_leaf_size : 4u, pk) &&
                  pk.depth + 2 < (uint32_t)TRAV_STACK;
        }
        if (!sah)
            bvh_pack(S.nodes, s.triangles, pk);
        // 4-wide nodes over the SAH tree (half the dependent node fetches per ray) unless asked for
        // the binary form or the worst-case stack (3 pushes per level) could exceed the traversal stack
        if (sah && !(p.flags & PHX_F_BINARY_BVH)) {
            bvh_widen(pk);
            wide = 3 * pk.wdepth + 4 < (uint32_t)TRAV_STACK;
        }
        S.trav_depth = wide ? pk.wdepth : sah ? pk.depth : S.depth;
        S.trav_inner = wide ? (uint32_t)(pk.wnodes.size() / 28) : (uint32_t)(pk.cnodes.size() / 16);
        trav_root = wide ? pk.wroot : pk.root;
        std::vector<float> nrm((size_t)n * 12), tan((size_t)n * 12), uv((size_t)n * 8);
        for (uint32_t k = 0; k < n; k++) {
            const phx_triangle &t = s.triangles[pk.leaf_tri[k]];
            const phx_f4 *nn[3] = {&t.n0, &t.n1, &t.n2}, *tt[3] = {&t.t0, &t.t1, &t.t2};
            for (int j = 0; j < 3; j++) {
                std::memcpy(&nrm[(size_t)k * 12 + 4 * j], nn[j], 16);
                std::memcpy(&tan[(size_t)k * 12 + 4 * j], tt[j], 16);
            }
            float u8v[8] = {t.uv0.x, t.uv0.y, t.uv1.x, t.uv1.y, t.uv2.x, t.uv2.y, 0.0f, 0.0f};
            std::memcpy(&uv[(size_t)k * 8], u8v, 32);
        }
        std::vector<uint32_t> qn;
        if (wide && quant_req)
            qn = bvh_quantize(pk);
        const void *inner = wide && quant_req ? (const void *)qn.data()
                            : wide           ? (const void *)pk.wnodes.data()
                                             : (const void *)pk.cnodes.data();
        const size_t inner_words = wide && quant_req ? qn.size() : wide ? pk.wnodes.size() : pk.cnodes.size();
        if ((r = upload(S.bufs[0], inner, std::max<size_t>(inner_words, 4) * 4)) ||
            (r = upload(S.bufs[1], pk.trirec.data(), pk.trirec.size() * 4)) ||
            (r = upload(S.bufs[2], nrm.data(), nrm.size() * 4)) ||
            (r = upload(S.bufs[3], tan.data(), tan.size() * 4)) || (r = upload(S.bufs[4], uv.data(), uv.size() * 4)))
            return r;
    }
    S.bvh_ms = ms_since(t_setup);
    const uint32_t ne = s.n_emissive_triangles;
    std::vector<float> ev((size_t)std::max(ne, 1u) * 12, 0.0f), en((size_t)std::max(ne, 1u) * 12, 0.0f),
        euv((size_t)std::max(ne, 1u) * 8, 0.0f);
    std::vector<uint32_t> emat(std::max(ne, 1u), 0u);
    for (uint32_t k = 0; k < ne; k++) {
        const phx_triangle &t = s.emissive_triangles[k];
        const phx_f4 *vv[3] = {&t.v0, &t.v1, &t.v2}, *nn[3] = {&t.n0, &t.n1, &t.n2};
        for (int j = 0; j < 3; j++) {
            std::memcpy(&ev[(size_t)k * 12 + 4 * j], vv[j], 16);
            std::memcpy(&en[(size_t)k * 12 + 4 * j], nn[j], 16);
        }
        float u8v[8] = {t.uv0.x, t.uv0.y, t.uv1.x, t.uv1.y, t.uv2.x, t.uv2.y, 0.0f, 0.0f};
        std::memcpy(&euv[(size_t)k * 8], u8v, 32);
        emat[k] = t.mat_index;
    }
    std::vector<phx_uv_transform_block> uvt(s.n_materials);
    if (s.uv_transforms) {
        std::memcpy(uvt.data(), s.uv_transforms, sizeof(phx_uv_transform_block) * s.n_materials);
    } else {
        phx_uv_transform id{};
        id.uv_scale = {1.0f, 1.0f};
        for (auto &b : uvt)
            b.diff = b.emis = b.norm = b.occlusion = b.metal_rough = b.transmission = id;
    }
    std::vector<float> lum(std::max(s.n_lights, 1u), 0.0f);
    if (s.n_lights) {
        if (s.lum_pref_sum)
            std::memcpy(lum.data(), s.lum_pref_sum, 4 * s.n_lights);
        else
            lum_pref_sum(s.lights, s.n_lights, lum.data());
    }
    if ((r = upload(S.bufs[5], ev.data(), ev.size() * 4)) ||
        (r = upload(S.bufs[6], en.data(), en.size() * 4)) || (r = upload(S.bufs[7], euv.data(), euv.size() * 4)) ||
        (r = upload(S.bufs[8], emat.data(), emat.size() * 4)) ||
        (r = upload(S.bufs[9], s.materials, sizeof(phx_material) * s.n_materials)) ||
        (r = upload(S.bufs[10], uvt.data(), sizeof(phx_uv_transform_block) * uvt.size())) ||
        (r = upload(S.bufs[11], s.tex_meta, sizeof(phx_texture_meta) * std::max(s.n_textures, 1u))) ||
        (r = upload(S.bufs[12], s.tex_atlas, std::max<uint64_t>(s.tex_atlas_bytes, 16))) ||
        (r = upload(S.bufs[13], s.lights, sizeof(phx_light) * std::max(s.n_lights, 1u))) ||
        (r = upload(S.bufs[14], lum.data(), lum.size() * 4)))
        return r;
    const bool has_env = s.envmap && s.envmap_width > 0 && s.envmap_height > 0;
    if ((r = upload(S.bufs[15], has_env ? s.envmap : nullptr,
                    has_env ? (size_t)s.envmap_width * s.envmap_height * 3 * 4 : 16)))
        return r;

    S.mats.assign(s.materials, s.materials + s.n_materials);
    S.lights.assign(s.lights, s.lights + s.n_lights);
    SceneDesc &d = S.desc;
    std::memset(&d, 0, sizeof(d));
    d.cnodes = S.bufs[0].as<float4>();
    d.trirec = S.bufs[1].as<float4>();
    d.tri_nrm = S.bufs[2].as<float4>();
    d.tri_tan = S.bufs[3].as<float4>();
    d.tri_uv = S.bufs[4].as<float4>();
    d.etri_v = S.bufs[5].as<float4>();
    d.etri_n = S.bufs[6].as<float4>();
    d.etri_uv = S.bufs[7].as<float4>();
    d.etri_mat = S.bufs[8].as<u32>();
    d.materials = S.bufs[9].as<phx_material>();
    d.uvt = S.bufs[10].as<phx_uv_transform_block>();
    d.tex_meta = S.bufs[11].as<phx_texture_meta>();
    d.tex_atlas = S.bufs[12].as<u8>();
    d.lights = S.bufs[13].as<phx_light>();
    d.lum_pref_sum = S.bufs[14].as<float>();
    d.envmap = S.bufs[15].as<float>();
    d.root = trav_root;
    d.wide = wide ? (quant_req ? 2u : 1u) : 0u;
    d.n_tris = n;
    d.n_lights = s.n_lights;
    d.total_lum = s.n_lights ? lum[s.n_lights - 1] : 0.0f; // shading.cpp:26
    d.light_draws = light_sample_draws(s.lights, s.n_lights, d.total_lum);
    phx_f4 ctr;
    float rad;
    scene_sphere(S.nodes[0], &ctr, &rad);
    d.scene_center = make_float4(ctr.x, ctr.y, ctr.z, ctr.w);
    d.scene_radius = rad;
    d.env_w = has_env ? s.envmap_width : 0;
    d.env_h = has_env ? s.envmap_height : 0;
    d.has_env = has_env ? 1u : 0u;
    d.camera = s.camera;
    d.width = p.width;
    d.height = p.height;
    d.n_pixels = p.width * p.height;
    d.n_emit = p.photons_per_round;
    d.max_bounces = p.max_photon_bounces;
    d.direct_samples = p.direct_samples;
    d.alpha = p.sppm_alpha;
    d.n_cells = p.grid_res * p.grid_res * p.grid_res + 1; // renderer.cpp:38
    S.hash = hash_info(S.nodes[0], p.grid_res);
    d.grid = GridDev{S.hash.origin.x, S.hash.origin.y, S.hash.origin.z, S.hash.cell_sizes.x,
                     S.hash.cell_sizes.y, S.hash.cell_sizes.z, p.grid_res, 0u};
    d.pixel_base = *pix;
    d.emit_base = *emit;
    d.cell_base = *cell;
    d.slot_base = *slot;
    d.nee_base = total_nee;
    if ((uint64_t)total_nee + (uint64_t)d.n_pixels * d.direct_samples > 0x7fffffffull)
        return fail(PHX_E_INVALID, "too many direct-lighting samples per round for 31-bit slot indices");
    total_nee += d.n_pixels * d.direct_samples;
    d.flags = p.flags;
    d.active = 1;
    d.any_transmissive = 0;
    for (uint32_t m = 0; m < s.n_materials; m++)
        if (!(s.materials[m].transmission < 1e-5f)) // not blocking a shadow ray (NaN included)
            d.any_transmissive = 1;
    if ((uint64_t)*pix + d.n_pixels > 0x7fffffffull || (uint64_t)*emit + d.n_emit > 0x7fffffffull ||
        (uint64_t)*cell + d.n_cells > 0x7fffffffull)
        return fail(PHX_E_INVALID, "batch too large for 31-bit global indices");
    *pix += d.n_pixels;
    *emit += d.n_emit;
    *cell += d.n_cells;
    *slot += (uint64_t)d.n_emit * d.max_bounces;
    S.setup_ms = ms_since(t_setup);
    return PHX_OK;
}

int Engine::create(const phx_scene *scenes, const phx_params *params, uint32_t n, int dev) {
    if (!scenes || !params || n == 0)
        return fail(PHX_E_INVALID, "no scenes");
    for (uint32_t i = 0; i < n; i++) {
        int r = check_params(params[i]);
        if (r)
            return r;
    }
    device = dev;
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&st_side, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&join_ev, cudaEventDisableTiming));
    init_kernels(device);
    sc.resize(n);
    uint32_t pix = 0, emit = 0, cell = 0;
    uint64_t slot = 0;
    for (uint32_t i = 0; i < n; i++) {
        int r = upload_scene(i, scenes[i], params[i], &pix, &emit, &cell, &slot);
        if (r)
            return r;
    }
    total_pixels = pix;
    total_emit = emit;
    total_cells = cell;
    total_slots = slot;
    max_photons = slot; // <= one stored photon per bounce (renderer.cpp:40)
    if (max_photons > 0x7fffffffull)
        return fail(PHX_E_INVALID, "photon buffer exceeds 2^31 entries");
    uint32_t kmax = total_cells - 1;
    key_bits = 1;
    while (key_bits < 32 && (kmax >> key_bits) != 0)
        key_bits++;

    std::vector<SceneDesc> descs(n);
    std::vector<uint32_t> pb(n + 1), eb(n + 1), nb(n + 1), rng(n);
    for (uint32_t i = 0; i < n; i++) {
        descs[i] = sc[i].desc;
        pb[i] = sc[i].desc.pixel_base;
        eb[i] = sc[i].desc.emit_base;
        nb[i] = sc[i].desc.nee_base;
        rng[i] = pcg_seed(sc[i].prm.seed).state; // renderer.cpp:54
    }
    pb[n] = total_pixels;
    eb[n] = total_emit;
    nb[n] = total_nee;
    int r;
    if ((r = upload(d_desc, descs.data(), sizeof(SceneDesc) * n)) || (r = upload(d_pix_bases, pb.data(), 4 * pb.size())) ||
        (r = upload(d_emit_bases, eb.data(), 4 * eb.size())) || (r = upload(d_nee_bases, nb.data(), 4 * nb.size())) ||
        (r = nee_ray.alloc(16 * (size_t)total_nee)) || (r = nee_val.alloc(16 * (size_t)total_nee)) ||
        (r = stash_sn.alloc(16 * (size_t)total_pixels)) || (r = stash_rng.alloc(4 * (size_t)total_pixels)) ||
        (r = spec_ray.alloc(16 * (size_t)total_nee)) || (r = spec_val.alloc(16 * (size_t)total_nee)) ||
        (r = spec_org.alloc(16 * (size_t)total_nee)) || (r = spec_pix.alloc(4 * (size_t)total_nee)) ||
        (r = upload(spec_next, nullptr, 16)) || (r = upload(def_cnt, nullptr, 4 * (size_t)total_pixels)) ||
        (r = def_prefix.alloc(16 * (size_t)total_pixels)) ||
        (r = def_val.alloc(16 * (size_t)DEF_MAX * total_pixels)) ||
        (r = def_tag.alloc(4 * (size_t)DEF_MAX * total_pixels)) ||
        (r = upload(d_rng, rng.data(), 4 * n)) ||
        (r = upload(d_seeds, nullptr, 4 * n)) || (r = upload(d_err, nullptr, 16)) || (r = upload(d_ovf, nullptr, 16)) ||
        (r = upload(d_queue, nullptr, 16)) || (r = upload(d_ntotal, nullptr, 16)))
        return r;
    const size_t P = total_pixels, E = total_emit, C = (size_t)total_cells + 1, N = max_photons;
    for (auto &b : hp)
        if ((r = upload(b, nullptr, 16 * P))) // ImageBuffers::alloc zero-fills (image.cpp:11-21)
            return r;
    if ((r = upload(flux, nullptr, 16 * P)) || (r = upload(weight, nullptr, 4 * P)) || (r = upload(radiance, nullptr, 16 * P)) ||
        (r = slot_pos.alloc(16 * N)) || (r = slot_pd.alloc(8 * N)) || (r = upload(counts, nullptr, 4 * (E + 1))) ||
        (r = upload(offsets, nullptr, 4 * (E + 1))) || (r = upload(ph_pos, nullptr, 16 * N)) ||
        (r = upload(ph_pd, nullptr, 8 * N)) || (r = upload(keys, nullptr, 4 * N)) ||
        (r = upload(cell_count, nullptr, 4 * C)) || (r = upload(cell_start, nullptr, 4 * C)) ||
        (r = sk0.alloc(4 * N)) || (r = sk1.alloc(4 * N)) || (r = upload(sv0, nullptr, 4 * N)) ||
        (r = upload(sv1, nullptr, 4 * N)) || (r = upload(s_posdir, nullptr, 16 * N)) ||
        (r = upload(s_power, nullptr, 4 * N)) || (r = upload(s_dir, nullptr, 16 * N)) ||
        (r = upload(s_pow, nullptr, 16 * N)) ||
        (r = scan_scr.alloc(std::max(scan_scratch_bytes(E + 1), scan_scratch_bytes(C)))) ||
        (r = radix_scr.alloc(radix_scratch_bytes(N, key_bits))))
        return r;
    perm = sv0.as<u32>();
    rs0 = view_own_buffers();
    // gather order: sort the pixels by (cell, octant) key; needs the composite key to fit 32 bits
    pix_key_bits = key_bits + 3 <= 32 ? key_bits + 3 : 0;
    if (pix_key_bits) {
        const uint32_t Pn = total_pixels;
        if ((r = pk_keys.alloc(4 * (size_t)Pn)) || (r = pk_t0.alloc(4 * (size_t)Pn)) ||
            (r = pk_t1.alloc(4 * (size_t)Pn)) || (r = pk_v0.alloc(4 * (size_t)Pn)) ||
            (r = pk_v1.alloc(4 * (size_t)Pn)) || (r = pk_scr.alloc(radix_scratch_bytes(Pn, pix_key_bits))) ||
            (r = upload(d_npix, &Pn, 4)))
            return r;
    }
    CK(cudaMallocHost((void **)&h_pinned, 4096));
    tune.trace_block = 128;
    tune.emit_block = 128;
    tune.gather_block = 128;
    tune.trace_blocks_per_sm = 8;
    tune.emit_blocks_per_sm = 8;
    tune.persistent = 1;
    tune.nee_wavefront = 1;
    tune.concurrent_passes = 0;
    tune.gather_sorted = 1;
    tune.gather_coop = 0; // the per-thread gather measured faster (caustic 2.28 vs 3.15 ms, atrium 3.52 vs 4.19)
    tune.pipeline_rounds = 2; // two rounds in flight per graph replay (measured faster, bit-identical)
    for (uint32_t i = 0; i < n; i++)
        if (params[i].flags & PHX_F_SIMPLE_TRAVERSAL)
            tune.persistent = 0;
    CK(cudaDeviceSynchronize());
    return PHX_OK;
}

LaunchCtx Engine::lc(const RoundSet &R) const {
    LaunchCtx l;
    l.scenes = d_desc.as<SceneDesc>();
    l.n_scenes = (u32)sc.size();
    l.pix_bases = d_pix_bases.as<u32>();
    l.emit_bases = d_emit_bases.as<u32>();
    l.total_pixels = total_pixels;
    l.total_emit = total_emit;
    l.seeds = R.seeds;
    l.err = d_err.as<u32>();
    l.overflow = d_ovf.as<u32>();
    l.nee_bases = d_nee_bases.as<u32>();
    l.total_nee = total_nee;
    l.nee_defer = tune.nee_wavefront ? 1u : 0u;
    l.pix_lo = shard.world > 1 ? shard.pix_lo : 0u;
    l.pix_hi = shard.world > 1 ? shard.pix_hi : total_pixels;
    l.emit_lo = shard.world > 1 ? shard.emit_lo : 0u;
    l.emit_hi = shard.world > 1 ? shard.emit_hi : total_emit;
    return l;
}

GridBufs Engine::gb(const RoundSet &R) const {
    GridBufs g;
    g.counts = R.counts;
    g.offsets = R.offsets;
    g.slot_pos = R.slot_pos;
    g.slot_pd = R.slot_pd;
    g.ph_pos = R.ph_pos;
    g.ph_pd = R.ph_pd;
    g.keys = R.keys;
    g.cell_count = R.cell_count;
    return g;
}

RoundSet Engine::view_own_buffers() {
    RoundSet R;
    R.seeds = d_seeds.as<u32>();
    R.queue = d_queue.as<u32>();
    R.ntotal = d_ntotal.as<u32>();
    for (int k = 0; k < 6; k++)
        R.hp[k] = hp[k].as<float4>();
    R.nee_ray = nee_ray.as<float4>();
    R.nee_val = nee_val.as<float4>();
    R.stash_sn = stash_sn.as<float4>();
    R.stash_rng = stash_rng.as<u32>();
    R.spec_ray = spec_ray.as<float4>();
    R.spec_val = spec_val.as<float4>();
    R.spec_org = spec_org.as<float4>();
    R.spec_pix = spec_pix.as<u32>();
    R.spec_next = spec_next.as<u32>();
    R.def_cnt = def_cnt.as<u32>();
    R.def_prefix = def_prefix.as<float4>();
    R.def_val = def_val.as<float4>();
    R.def_tag = def_tag.as<u32>();
    R.slot_pos = slot_pos.as<float4>();
    R.slot_pd = slot_pd.as<uint2>();
    R.counts = counts.as<u32>();
    R.offsets = offsets.as<u32>();
    R.ph_pos = ph_pos.as<float4>();
    R.ph_pd = ph_pd.as<uint2>();
    R.keys = keys.as<u32>();
    R.cell_count = cell_count.as<u32>();
    R.cell_start = cell_start.as<u32>();
    R.sk0 = sk0.as<u32>();
    R.sk1 = sk1.as<u32>();
    R.sv0 = sv0.as<u32>();
    R.sv1 = sv1.as<u32>();
    R.s_posdir = s_posdir.as<float4>();
    R.s_power = s_power.as<u32>();
    R.s_dir = s_dir.as<float4>();
    R.s_pow = s_pow.as<float4>();
    R.scan_scr = scan_scr.p;
    R.radix_scr = radix_scr.p;
    R.perm = sv0.as<u32>();
    return R;
}

void Engine::ev(int stage, bool end, cudaStream_t s) {
    if (!profiling)
        return;
    cudaEvent_t &e = events[2 * stage + (end ? 1 : 0)];
    if (!e)
        cudaEventCreate(&e);
    if (capturing)
        cudaEventRecordWithFlags(e, s ? s : st, cudaEventRecordExternal);
    else
        cudaEventRecord(e, s ? s : st);
}

void Engine::enq_seeds_r(RoundSet &R, cudaStream_t s) {
    ev(ST_SEEDS, false, s);
    launch_next_seeds(d_rng.as<u32>(), R.seeds, (u32)sc.size(), s);
    ev(ST_SEEDS, true, s);
}

void Engine::enq_trace_r(RoundSet &R, cudaStream_t s) {
    ev(ST_TRACE, false, s);
    TraceOut o{R.hp[0], R.hp[1], R.hp[2], R.hp[3], R.hp[4], R.hp[5], R.nee_ray, R.nee_val, R.stash_sn, R.stash_rng};
    const LaunchCtx l = lc(R);
    const bool spec = spec_deferred();
    if (spec) {
        o.spec_ray = R.spec_ray;
        o.spec_val = R.spec_val;
        o.spec_org = R.spec_org;
        o.spec_pix = R.spec_pix;
        o.spec_next = R.spec_next;
        o.spec_cap = total_nee;
        o.def_cnt = R.def_cnt;
        o.def_prefix = R.def_prefix;
        o.def_val = R.def_val;
        o.def_tag = R.def_tag;
        cudaMemsetAsync(R.spec_next, 0, sizeof(u32), s);
    }
    launch_trace(l, o, (int)tune.trace_block, (int)tune.persistent, (int)tune.trace_blocks_per_sm, R.queue,
                 untextured(), s);
    ev(ST_TRACE, true, s);
    ev(ST_SHADOW, false, s);
    bool transmissive = false, presample = false;
    for (const auto &sl : sc) {
        transmissive = transmissive || sl.desc.any_transmissive != 0;
        presample = presample || sl.desc.light_draws == LIGHT_DRAWS_VARY;
    }
    // every sample of a hit point is one ray when the only light is a point, spot or directional one
    const bool per_pixel = sc.size() == 1 && shard.world == 1 && sc[0].lights.size() == 1 &&
                           sc[0].lights[0].kind != PHX_LIGHT_TEXTURED;
    const int kind = !transmissive ? SHADOW_OPAQUE : untextured() ? SHADOW_CLEAR : SHADOW_GENERAL;
    launch_shadow(l, o, kind, presample, per_pixel, sc[0].desc.n_pixels,
                  sc.size() == 1 ? &sc[0].desc : nullptr, s);
    launch_nee_resolve(l, o, s);
    if (spec)
        launch_spec_resolve(l, o, s);
    ev(ST_SHADOW, true, s);
    stage_state |= 1;
}

void Engine::enq_emit_r(RoundSet &R, cudaStream_t s) {
    ev(ST_EMIT, false, s);
    EmitOut o{R.slot_pos, R.slot_pd, R.counts};
    launch_emit(lc(R), o, (int)tune.emit_block, (int)tune.persistent, (int)tune.emit_blocks_per_sm, R.queue + 1,
                untextured(), photon_prestart(), s);
    ev(ST_EMIT, true, s);
    ev(ST_EMIT_SCAN, false, s);
    launch_scan(R.counts, R.offsets, (u64)total_emit + 1, R.scan_scr, R.ntotal, d_err.as<u32>(), s);
    launch_compact(lc(R), gb(R), s);
    ev(ST_EMIT_SCAN, true, s);
    stage_state |= 2;
}

void Engine::enq_hash_sort_r(RoundSet &R, cudaStream_t s) {
    ev(ST_HASH, false, s);
    cudaMemsetAsync(R.cell_count, 0, 4 * ((size_t)total_cells + 1), s);
    launch_hash(lc(R), gb(R), R.ntotal, max_photons, s);
    ev(ST_HASH, true, s);
    ev(ST_CELL_SCAN, false, s);
    launch_scan(R.cell_count, R.cell_start, (u64)total_cells + 1, R.scan_scr, nullptr, d_err.as<u32>(), s);
    ev(ST_CELL_SCAN, true, s);
    ev(ST_SORT, false, s);
    launch_radix_sort(R.keys, R.sk0, R.sk1, R.sv0, R.sv1, &R.perm, R.ntotal, max_photons, key_bits, R.radix_scr,
                      d_err.as<u32>(), s);
    ev(ST_SORT, true, s);
    ev(ST_RECORDS, false, s);
    launch_sorted_records(R.perm, R.ph_pos, R.ph_pd, R.ntotal, max_photons, R.s_posdir, R.s_power, R.s_dir, R.s_pow,
                          d_err.as<u32>(), s);
    ev(ST_RECORDS, true, s);
    stage_state |= 4;
}

void Engine::enq_gather_r(RoundSet &R, cudaStream_t s) {
    adjoint_invalidate();
    ev(ST_GATHER, false, s);
    const u32 *order = nullptr;
    if (tune.gather_sorted && pix_key_bits) {
        launch_pixel_keys(lc(R), R.hp[0], R.hp[5], pix_key_bits, pk_keys.as<u32>(), s);
        launch_radix_sort(pk_keys.as<u32>(), pk_t0.as<u32>(), pk_t1.as<u32>(), pk_v0.as<u32>(), pk_v1.as<u32>(),
                          &pix_order, d_npix.as<u32>(), total_pixels, pix_key_bits, pk_scr.p, d_err.as<u32>(), s);
        order = pix_order;
    }
    GatherBufs g{R.hp[0], R.hp[1], R.hp[2], R.hp[3], R.hp[4], R.hp[5], R.s_posdir, R.s_power, R.s_dir, R.s_pow,
                 R.cell_start, (u32)max_photons, flux.as<float4>(), weight.as<float>(), radiance.as<float4>(), rec_r2,
                 rec_ratio, order};
    launch_gather(lc(R), g, (int)tune.gather_block, tune.gather_coop != 0, s);
    ev(ST_GATHER, true, s);
}

void Engine::enq_round() {
    enq_seeds();
    enq_trace();
    enq_emit();
    enq_hash_sort();
    enq_gather();
}

void Engine::accumulate_profile() {
    if (!profiling)
        return;
    for (int s = 0; s < ST__N; s++) {
        if (!events[2 * s] || !events[2 * s + 1])
            continue;
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, events[2 * s], events[2 * s + 1]) == cudaSuccess)
            prof_ms[s] += ms;
        else
            cudaGetLastError();
    }
    prof_rounds++;
}

void Engine::invalidate_graph() {
    if (st)
        cudaStreamSynchronize(st);
    if (gexec)
        cudaGraphExecDestroy(gexec);
    if (graph)
        cudaGraphDestroy(graph);
    if (gexec_host)
        cudaGraphExecDestroy(gexec_host);
    if (graph_host)
        cudaGraphDestroy(graph_host);
    if (gexec_pipe)
        cudaGraphExecDestroy(gexec_pipe);
    if (graph_pipe)
        cudaGraphDestroy(graph_pipe);
    gexec = nullptr;
    graph = nullptr;
    gexec_host = nullptr;
    graph_host = nullptr;
    gexec_pipe = nullptr;
    graph_pipe = nullptr;
    pipe_k = 0;
}

void Engine::set_profiling(bool on) {
    if (on != profiling) // re-capture so the graph carries (or drops) the event nodes
        invalidate_graph();
    profiling = on;
    for (auto &m : prof_ms)
        m = 0.0;
    prof_rounds = 0;
}

void Engine::stage_ms(float *out) const {
    for (int s = 0; s < ST__N; s++)
        out[s] = prof_rounds ? (float)(prof_ms[s] / prof_rounds) : 0.0f;
}

int Engine::sync_and_check() {
    CK(cudaStreamSynchronize(st));
    CK(cudaGetLastError());
    CK(cudaMemcpy(h_pinned, d_err.p, 8, cudaMemcpyDeviceToHost));
    uint32_t err = h_pinned[0];
    if (err & ERR_LOOKBACK_TIMEOUT)
        return fail(PHX_E_TIMEOUT, "a decoupled look-back wait gave up (device error flag set)");
    if (err & ERR_NO_PHOTONS)
        return fail(PHX_E_NO_PHOTONS, "no photon was stored in a round (renderer.cpp:117-118)");
    if (err & ERR_DEFER_OVERFLOW)
        return fail(PHX_E_STATE, "a deferred specular emission term did not fit its pixel's list");
    return PHX_OK;
}

int Engine::read_total(uint32_t *n) {
    CK(cudaMemcpyAsync(h_pinned, d_ntotal.p, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    *n = h_pinned[0];
    return PHX_OK;
}

int Engine::set_seed(uint32_t seed) {
    std::vector<uint32_t> s(sc.size(), seed);
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(d_seeds.p, s.data(), 4 * s.size(), cudaMemcpyHostToDevice));
    return PHX_OK;
}

int Engine::scene_photon_range(uint32_t s, uint32_t *off, uint32_t *n) {
    CK(cudaStreamSynchronize(st));
    if (sc.size() == 1) {
        uint32_t v[1];
        CK(cudaMemcpy(v, d_ntotal.p, 4, cudaMemcpyDeviceToHost));
        *off = 0;
        *n = v[0];
        return PHX_OK;
    }
    uint32_t a = 0, b = 0;
    CK(cudaMemcpy(&a, offsets.as<u32>() + sc[s].desc.emit_base, 4, cudaMemcpyDeviceToHost));
    uint32_t next = s + 1 < sc.size() ? sc[s + 1].desc.emit_base : total_emit;
    CK(cudaMemcpy(&b, offsets.as<u32>() + next, 4, cudaMemcpyDeviceToHost));
    *off = a;
    *n = b - a;
    return PHX_OK;
}

bool Engine::untextured() const {
    for (const auto &s : sc)
        for (const auto &m : s.mats)
            if (m.diff_index != PHX_NO_TEXTURE || m.emis_index != PHX_NO_TEXTURE || m.norm_index != PHX_NO_TEXTURE ||
                m.occlusion_index != PHX_NO_TEXTURE || m.metal_rough_index != PHX_NO_TEXTURE ||
                m.transmission_index != PHX_NO_TEXTURE)
                return false;
    return true;
}

bool Engine::photon_prestart() const {
    for (const auto &s : sc)
        if (s.desc.max_bounces < 3)
            return false;
    return true;
}

bool Engine::any_active() const {
    for (const auto &s : sc)
        if (s.desc.active)
            return true;
    return false;
}

int Engine::set_active(uint32_t scene, bool on) {
    if (scene >= sc.size())
        return fail(PHX_E_INVALID, "scene index out of range");
    if ((sc[scene].desc.active != 0) == on)
        return PHX_OK;
    adjoint_invalidate();
    CK(cudaStreamSynchronize(st));
    sc[scene].desc.active = on ? 1u : 0u;
    return upload_descs();
}

int Engine::plain_round() {
    if (shard.world > 1)
        return fail(PHX_E_STATE, "a sharded context renders with phx_shard_round or phx_shard_begin/_end");
    if (!any_active())
        return PHX_OK;
    enq_seeds();
    enq_trace();
    enq_emit();
    // renderer.cpp:113-118: blocking read of the stored-photon count
    uint32_t total = 0;
    int r = read_total(&total);
    if (r)
        return r;
    for (uint32_t s = 0; s < sc.size(); s++) {
        uint32_t off, n;
        if ((r = scene_photon_range(s, &off, &n)))
            return r;
        if (n == 0 && sc[s].desc.active)
            return fail(PHX_E_NO_PHOTONS, "no photon hit (renderer.cpp:117-118)");
        sc[s].n_photons_last = n;
    }
    enq_hash_sort();
    enq_gather();
    r = sync_and_check(); // renderer.cpp:160 queue.finish()
    if (r)
        return r;
    accumulate_profile();
    count_round(1);
    return PHX_OK;
}

// Captures one round (optionally without the device-side seed step) into an executable graph.
int Engine::capture(bool with_seeds, cudaGraph_t *g, cudaGraphExec_t *ge) {
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    if (with_seeds)
        enq_seeds();
    if (tune.concurrent_passes) {
        // the photon pass only shares the round seed with the camera pass: fork it onto a second
        // branch of the graph and join before the hash stage
        cudaEventRecord(fork_ev, st);
        cudaStreamWaitEvent(st_side, fork_ev, 0);
        enq_emit(st_side);
        enq_trace();
        cudaEventRecord(join_ev, st_side);
        cudaStreamWaitEvent(st, join_ev, 0);
    } else {
        enq_trace();
        enq_emit();
    }
    enq_hash_sort();
    enq_gather();
    capturing = false;
    cudaError_t e = cudaStreamEndCapture(st, g);
    if (e != cudaSuccess) {
        *g = nullptr;
        return fail(PHX_E_CUDA, std::string("stream capture failed: ") + cudaGetErrorString(e));
    }
    CK(cudaGraphInstantiate(ge, *g, 0));
    return PHX_OK;
}

void Engine::count_round(uint32_t rounds) {
    for (auto &s : sc) {
        if (!s.desc.active)
            continue;
        s.rounds += rounds;
        s.total_emitted += (uint64_t)rounds * s.prm.photons_per_round;
    }
}

// Rounds per pipelined graph: the tuning's, but 1 (off) while profiling stage times, while the
// adjoint records its forward pass, for a sharded context, or with rounds of the one-thread
// kernels' inline NEE form (their buffers are the same, this keeps the forms few).
uint32_t Engine::pipeline_rounds() const {
    if (tune.pipeline_rounds <= 1 || profiling || rec_r2 || shard.world > 1)
        return 1;
    return std::min(tune.pipeline_rounds, 8u);
}

// Allocates `sets` more sets of per-round buffers, sized like the engine's own (zero-filled where
// those are).
int Engine::alloc_round_sets(uint32_t sets) {
    const size_t P = total_pixels, E = total_emit, C = (size_t)total_cells + 1, N = max_photons,
                 NE = total_nee, n = sc.size();
    while (xsets.size() < sets) {
        std::vector<DevBuf> b(44);
        RoundSet R;
        int k = 0, r = 0;
        auto get = [&](size_t bytes, bool zero) -> void * {
            DevBuf &d = b[k++];
            if (r)
                return nullptr;
            r = zero ? upload(d, nullptr, bytes) : d.alloc(bytes);
            return d.p;
        };
        R.seeds = (u32 *)get(4 * n, true);
        R.queue = (u32 *)get(16, true);
        R.ntotal = (u32 *)get(16, true);
        for (int h = 0; h < 6; h++)
            R.hp[h] = (float4 *)get(16 * P, true);
        R.nee_ray = (float4 *)get(16 * NE, false);
        R.nee_val = (float4 *)get(16 * NE, false);
        R.stash_sn = (float4 *)get(16 * P, false);
        R.stash_rng = (u32 *)get(4 * P, false);
        R.spec_ray = (float4 *)get(16 * NE, false);
        R.spec_val = (float4 *)get(16 * NE, false);
        R.spec_org = (float4 *)get(16 * NE, false);
        R.spec_pix = (u32 *)get(4 * NE, false);
        R.spec_next = (u32 *)get(16, true);
        R.def_cnt = (u32 *)get(4 * P, true);
        R.def_prefix = (float4 *)get(16 * P, false);
        R.def_val = (float4 *)get(16 * (size_t)DEF_MAX * P, false);
        R.def_tag = (u32 *)get(4 * (size_t)DEF_MAX * P, false);
        R.slot_pos = (float4 *)get(16 * N, false);
        R.slot_pd = (uint2 *)get(8 * N, false);
        R.counts = (u32 *)get(4 * (E + 1), true);
        R.offsets = (u32 *)get(4 * (E + 1), true);
        R.ph_pos = (float4 *)get(16 * N, true);
        R.ph_pd = (uint2 *)get(8 * N, true);
        R.keys = (u32 *)get(4 * N, true);
        R.cell_count = (u32 *)get(4 * C, true);
        R.cell_start = (u32 *)get(4 * C, true);
        R.sk0 = (u32 *)get(4 * N, false);
        R.sk1 = (u32 *)get(4 * N, false);
        R.sv0 = (u32 *)get(4 * N, true);
        R.sv1 = (u32 *)get(4 * N, true);
        R.s_posdir = (float4 *)get(16 * N, true);
        R.s_power = (u32 *)get(4 * N, true);
        R.s_dir = (float4 *)get(16 * N, true);
        R.s_pow = (float4 *)get(16 * N, true);
        R.scan_scr = get(std::max(scan_scratch_bytes(E + 1), scan_scratch_bytes(C)), false);
        R.radix_scr = get(radix_scratch_bytes(N, key_bits), false);
        R.perm = R.sv0;
        if (r) {
            for (auto &d : b)
                d.release();
            return r;
        }
        xbufs.push_back(std::move(b));
        xsets.push_back(R);
    }
    return PHX_OK;
}

// Captures k rounds.  Round i (0..k-1) uses buffer set k-1-i, so the last round leaves its results
// in the engine's own buffers (read-back and every other form see the latest round).  The seed
// steps stay in order on the engine's stream (they advance one RNG state); each round's passes
// (camera + shadow, photon + hash + sort) run on a branch of their own from its seed step; the
// gathers run in round order, each after its round's passes.  Rounds thus overlap wherever a
// round's paths leave the GPU partly idle; every round computes exactly what it computes alone.
int Engine::capture_pipelined(uint32_t k) {
    int r;
    if ((r = alloc_round_sets(k - 1)))
        return r;
    while (pipe_st.size() < 2 * k) {
        cudaStream_t s2;
        CK(cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        pipe_st.push_back(s2);
    }
    while (pipe_ev.size() < 3 * k) {
        cudaEvent_t e;
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        pipe_ev.push_back(e);
    }
    auto set = [&](uint32_t i) -> RoundSet & { return i == k - 1 ? rs0 : xsets[k - 2 - i]; };
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    for (uint32_t i = 0; i < k; i++) {
        RoundSet &R = set(i);
        enq_seeds_r(R, st);
        cudaEventRecord(pipe_ev[3 * i], st); // round i's seeds
        cudaStream_t a = pipe_st[2 * i], b = pipe_st[2 * i + 1];
        cudaStreamWaitEvent(a, pipe_ev[3 * i], 0);
        if (tune.concurrent_passes) {
            cudaStreamWaitEvent(b, pipe_ev[3 * i], 0);
            enq_emit_r(R, b);
            enq_trace_r(R, a);
            cudaEventRecord(pipe_ev[3 * i + 1], b);
            cudaStreamWaitEvent(a, pipe_ev[3 * i + 1], 0);
        } else {
            enq_trace_r(R, a);
            enq_emit_r(R, a);
        }
        enq_hash_sort_r(R, a);
        cudaEventRecord(pipe_ev[3 * i + 2], a); // round i's passes
    }
    for (uint32_t i = 0; i < k; i++) {
        cudaStreamWaitEvent(st, pipe_ev[3 * i + 2], 0);
        enq_gather_r(set(i), st);
    }
    perm = rs0.perm;
    capturing = false;
    cudaError_t e = cudaStreamEndCapture(st, &graph_pipe);
    if (e != cudaSuccess) {
        graph_pipe = nullptr;
        return fail(PHX_E_CUDA, std::string("stream capture failed: ") + cudaGetErrorString(e));
    }
    CK(cudaGraphInstantiate(&gexec_pipe, graph_pipe, 0));
    pipe_k = k;
    return PHX_OK;
}

int Engine::graph_rounds(uint32_t rounds) {
    if (shard.world > 1)
        return fail(PHX_E_STATE, "a sharded context renders with phx_shard_round or phx_shard_begin/_end");
    adjoint_invalidate();
    if (!any_active())
        return PHX_OK;
    int r;
    const uint32_t k = pipeline_rounds();
    uint32_t single = rounds;
    if (k > 1 && rounds >= k) {
        if (pipe_k != k) {
            if (gexec_pipe)
                cudaGraphExecDestroy(gexec_pipe);
            if (graph_pipe)
                cudaGraphDestroy(graph_pipe);
            gexec_pipe = nullptr;
            graph_pipe = nullptr;
            pipe_k = 0;
            if ((r = capture_pipelined(k)))
                return r;
        }
        for (uint32_t i = 0; i < rounds / k; i++)
            CK(cudaGraphLaunch(gexec_pipe, st));
        single = rounds % k;
    }
    if (single && !gexec && (r = capture(true, &graph, &gexec)))
        return r;
    for (uint32_t i = 0; i < single; i++) {
        CK(cudaGraphLaunch(gexec, st));
        if (profiling) {
            CK(cudaStreamSynchronize(st));
            accumulate_profile();
        }
    }
    r = sync_and_check();
    if (r)
        return r;
    count_round(rounds);
    for (uint32_t s = 0; s < sc.size(); s++) {
        uint32_t off, n;
        if ((r = scene_photon_range(s, &off, &n)))
            return r;
        sc[s].n_photons_last = n;
    }
    return PHX_OK;
}

int Engine::seeded_round(uint32_t seed) {
    if (shard.world > 1)
        return fail(PHX_E_STATE, "a sharded context renders with phx_shard_round or phx_shard_begin/_end");
    adjoint_invalidate();
    if (!any_active())
        return PHX_OK;
    int r;
    if (!gexec_host && (r = capture(false, &graph_host, &gexec_host)))
        return r;
    if (!h_seed_ring)
        CK(cudaMallocHost((void **)&h_seed_ring, sizeof(u32) * SEED_RING * sc.size()));
    const uint32_t slot = seed_slot++ % SEED_RING;
    if (seed_ev[slot])
        CK(cudaEventSynchronize(seed_ev[slot])); // the staging slot's previous copy has been consumed
    else
        CK(cudaEventCreateWithFlags(&seed_ev[slot], cudaEventDisableTiming));
    u32 *h = h_seed_ring + slot * sc.size();
    for (size_t s = 0; s < sc.size(); s++)
        h[s] = seed;
    CK(cudaMemcpyAsync(d_seeds.p, h, sizeof(u32) * sc.size(), cudaMemcpyHostToDevice, st));
    CK(cudaEventRecord(seed_ev[slot], st));
    CK(cudaGraphLaunch(gexec_host, st));
    count_round(1);
    return PHX_OK;
}

int Engine::upload_descs() {
    if (sc.size() == 1)
        invalidate_graph(); // the captured shadow launch holds the descriptor by value
    std::vector<SceneDesc> d(sc.size());
    for (size_t i = 0; i < sc.size(); i++)
        d[i] = sc[i].desc;
    CK(cudaMemcpy(d_desc.p, d.data(), sizeof(SceneDesc) * d.size(), cudaMemcpyHostToDevice));
    return PHX_OK;
}

int Engine::autotune(uint32_t rounds, phx_tuning *chosen) {
    if (shard.world > 1)
        return fail(PHX_E_STATE, "a sharded context renders with phx_shard_round or phx_shard_begin/_end");
    if (!any_active())
        return fail(PHX_E_STATE, "no active scene to tune on");
    if (rounds == 0 || rounds > 64)
        return fail(PHX_E_INVALID, "rounds_per_trial must be 1..64");
    adjoint_invalidate();
    CK(cudaStreamSynchronize(st));
    // the trials render real rounds: keep the state they overwrite
    const size_t P = total_pixels, ns = sc.size();
    DevBuf keep;
    int r;
    if ((r = keep.alloc(36 * P + 4 * ns)))
        return r;
    char *k = keep.as<char>();
    CK(cudaMemcpy(k, flux.p, 16 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(k + 16 * P, radiance.p, 16 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(k + 32 * P, weight.p, 4 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(k + 36 * P, d_rng.p, 4 * ns, cudaMemcpyDeviceToDevice));
    std::vector<SceneSlot> counters(ns);
    for (size_t i = 0; i < ns; i++) {
        counters[i].rounds = sc[i].rounds;
        counters[i].total_emitted = sc[i].total_emitted;
        counters[i].n_photons_last = sc[i].n_photons_last;
    }
    const int kept_state = stage_state;
    const bool was_profiling = profiling;
    if (was_profiling)
        set_profiling(false);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // milliseconds per round of `rounds` graph-replayed rounds (rounded up to whole pipelined groups,
    // after a warm-up that captures the graph)
    auto trial = [&](const phx_tuning &tt, float *ms) -> int {
        tune = tt;
        invalidate_graph();
        const uint32_t k = pipeline_rounds();
        const uint32_t n = (rounds + k - 1) / k * k;
        int rr = graph_rounds(k); // capture + warm-up
        if (rr)
            return rr;
        if (cudaEventRecord(e0, st) != cudaSuccess)
            return fail(PHX_E_CUDA, "event record failed");
        if ((rr = graph_rounds(n)))
            return rr;
        if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(ms, e0, e1) != cudaSuccess)
            return fail(PHX_E_CUDA, "event timing failed");
        *ms /= (float)n;
        return PHX_OK;
    };
    phx_tuning best = tune;
    float best_ms = 0.0f;
    r = trial(best, &best_ms);
    // coordinate descent over the knobs that leave every result bit-identical
    auto knob = [&](uint32_t phx_tuning::*f, std::initializer_list<uint32_t> values) {
        for (uint32_t v : values) {
            if (r || best.*f == v)
                continue;
            phx_tuning c = best;
            c.*f = v;
            float ms = 0.0f;
            r = trial(c, &ms);
            if (!r && ms < best_ms) {
                best_ms = ms;
                best = c;
            }
        }
    };
    knob(&phx_tuning::persistent, {1u, 0u});
    knob(&phx_tuning::nee_wavefront, {1u, 0u});
    if (best.persistent) {
        knob(&phx_tuning::trace_blocks_per_sm, {2u, 4u, 6u, 8u, 12u, 16u});
        knob(&phx_tuning::emit_blocks_per_sm, {2u, 4u, 6u, 8u, 12u, 16u});
    }
    knob(&phx_tuning::concurrent_passes, {0u, 1u});
    knob(&phx_tuning::gather_sorted, {1u, 0u});
    knob(&phx_tuning::gather_coop, {1u, 0u});
    // rounds in flight: each more needs another set of per-round buffers; a candidate whose sets do
    // not fit in device memory is skipped
    for (uint32_t v : {1u, 2u, 4u}) {
        if (r || best.pipeline_rounds == v)
            continue;
        phx_tuning c = best;
        c.pipeline_rounds = v;
        float ms = 0.0f;
        r = trial(c, &ms);
        if (r == PHX_E_OOM) {
            r = PHX_OK;
            cudaGetLastError();
            continue;
        }
        if (!r && ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    tune = best;
    invalidate_graph();
    // restore the state
    CK(cudaMemcpy(flux.p, k, 16 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(radiance.p, k + 16 * P, 16 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(weight.p, k + 32 * P, 4 * P, cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(d_rng.p, k + 36 * P, 4 * ns, cudaMemcpyDeviceToDevice));
    for (size_t i = 0; i < ns; i++) {
        sc[i].rounds = counters[i].rounds;
        sc[i].total_emitted = counters[i].total_emitted;
        sc[i].n_photons_last = counters[i].n_photons_last;
    }
    stage_state = kept_state;
    if (was_profiling)
        set_profiling(true);
    if (r)
        return r;
    if (chosen)
        *chosen = best;
    return PHX_OK;
}

int Engine::set_alpha(float alpha) {
    adjoint_invalidate();
    CK(cudaStreamSynchronize(st));
    for (auto &s : sc) {
        s.desc.alpha = alpha;
        s.prm.sppm_alpha = alpha;
    }
    return upload_descs();
}

int Engine::set_n_photons(uint32_t n) {
    adjoint_invalidate();
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "photon injection is only available on single-scene contexts");
    if (n > max_photons)
        return fail(PHX_E_INVALID, "n_photons exceeds the photon buffer (photons_per_round * max_bounces)");
    CK(cudaStreamSynchronize(st));
    CK(cudaMemcpy(d_ntotal.p, &n, 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(offsets.as<u32>() + total_emit, &n, 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(cell_start.as<u32>() + total_cells, &n, 4, cudaMemcpyHostToDevice));
    sc[0].n_photons_last = n;
    stage_state |= 2;
    return PHX_OK;
}

namespace {
struct BufDesc {
    size_t esize;   // logical element size (reference layout)
    uint64_t count; // logical elements
};
} // namespace

int Engine::read_buffer(uint32_t s, int which, void *dst, uint64_t off, uint64_t bytes) {
    if (s >= sc.size())
        return fail(PHX_E_INVALID, "scene index out of range");
    if (!dst && bytes)
        return fail(PHX_E_INVALID, "null destination");
    const SceneDesc &d = sc[s].desc;
    uint32_t poff = 0, pn = 0;
    int r;
    if (which >= PHX_BUF_PHOTON_POS && which <= PHX_BUF_SORTED_DIR && which != PHX_BUF_CELL_COUNT)
        if ((r = scene_photon_range(s, &poff, &pn)))
            return r;
    if (which == PHX_BUF_SORT_PERM && (r = scene_photon_range(s, &poff, &pn)))
        return r;
    CK(cudaStreamSynchronize(st));
    BufDesc bd{0, 0};
    switch (which) {
    case PHX_BUF_HP_POS: case PHX_BUF_HP_NORMAL: case PHX_BUF_HP_THROUGHPUT: case PHX_BUF_HP_BASE_COLOR:
    case PHX_BUF_HP_DIRECT: case PHX_BUF_HP_EMISSION: case PHX_BUF_FLUX: case PHX_BUF_RADIANCE:
        bd = {16, d.n_pixels};
        break;
    case PHX_BUF_PHOTON_WEIGHT:
        bd = {4, d.n_pixels};
        break;
    case PHX_BUF_PHOTON_POS: case PHX_BUF_SORTED_POS:
        bd = {16, pn};
        break;
    case PHX_BUF_PHOTON_POWER: case PHX_BUF_PHOTON_DIR: case PHX_BUF_PHOTON_HASH: case PHX_BUF_SORTED_POWER:
    case PHX_BUF_SORTED_DIR: case PHX_BUF_SORT_PERM:
        bd = {4, pn};
        break;
    case PHX_BUF_CELL_COUNT: case PHX_BUF_CELL_START: case PHX_BUF_CELL_END:
        bd = {4, d.n_cells};
        break;
    case PHX_BUF_EMIT_COUNT:
        bd = {4, d.n_emit};
        break;
    case PHX_BUF_BVH_NODES:
        bd = {sizeof(phx_bvh_node), sc[s].nodes.size()};
        break;
    case PHX_BUF_ROUND_RNG:
        bd = {4, 1};
        break;
    default:
        return fail(PHX_E_INVALID, "unknown buffer id");
    }
    if (off + bytes > bd.esize * bd.count)
        return fail(PHX_E_INVALID, "read past the end of the buffer");
    if (bytes == 0)
        return PHX_OK;
    const uint64_t e0 = off / bd.esize, e1 = (off + bytes + bd.esize - 1) / bd.esize, ne = e1 - e0;
    std::vector<uint8_t> tmp(ne * bd.esize);
    auto dcopy = [&](const void *src, size_t b) -> int {
        CK(cudaMemcpy(tmp.data(), src, b, cudaMemcpyDeviceToHost));
        return PHX_OK;
    };
    auto fetch32 = [&](const u32 *src, std::vector<uint32_t> &v) -> int {
        v.resize(ne);
        CK(cudaMemcpy(v.data(), src, 4 * ne, cudaMemcpyDeviceToHost));
        return PHX_OK;
    };
    std::vector<uint32_t> v;
    std::vector<uint2> v2;
    std::vector<float4> v4;
    switch (which) {
    case PHX_BUF_HP_POS: case PHX_BUF_HP_NORMAL: case PHX_BUF_HP_THROUGHPUT: case PHX_BUF_HP_BASE_COLOR:
    case PHX_BUF_HP_DIRECT: case PHX_BUF_HP_EMISSION:
        r = dcopy(hp[which].as<float4>() + d.pixel_base + e0, 16 * ne);
        break;
    case PHX_BUF_FLUX:
        r = dcopy(flux.as<float4>() + d.pixel_base + e0, 16 * ne);
        break;
    case PHX_BUF_RADIANCE:
        r = dcopy(radiance.as<float4>() + d.pixel_base + e0, 16 * ne);
        break;
    case PHX_BUF_PHOTON_WEIGHT:
        r = dcopy(weight.as<float>() + d.pixel_base + e0, 4 * ne);
        break;
    case PHX_BUF_PHOTON_POS:
        r = dcopy(ph_pos.as<float4>() + poff + e0, 16 * ne);
        break;
    case PHX_BUF_PHOTON_POWER: case PHX_BUF_PHOTON_DIR:
        v2.resize(ne);
        CK(cudaMemcpy(v2.data(), ph_pd.as<uint2>() + poff + e0, 8 * ne, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < ne; i++)
            ((uint32_t *)tmp.data())[i] = which == PHX_BUF_PHOTON_POWER ? v2[i].x : v2[i].y;
        r = PHX_OK;
        break;
    case PHX_BUF_PHOTON_HASH:
        if (!(r = fetch32(keys.as<u32>() + poff + e0, v)))
            for (uint64_t i = 0; i < ne; i++)
                ((uint32_t *)tmp.data())[i] = v[i] - d.cell_base;
        break;
    case PHX_BUF_CELL_COUNT:
        r = dcopy(cell_count.as<u32>() + d.cell_base + e0, 4 * ne);
        break;
    case PHX_BUF_CELL_START: case PHX_BUF_CELL_END:
        if (!(r = fetch32(cell_start.as<u32>() + d.cell_base + e0 + (which == PHX_BUF_CELL_END ? 1 : 0), v)))
            for (uint64_t i = 0; i < ne; i++)
                ((uint32_t *)tmp.data())[i] = v[i] - poff;
        break;
    case PHX_BUF_SORTED_POS: case PHX_BUF_SORTED_DIR:
        v4.resize(ne);
        CK(cudaMemcpy(v4.data(), s_posdir.as<float4>() + poff + e0, 16 * ne, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < ne; i++) {
            if (which == PHX_BUF_SORTED_POS) {
                float q[4] = {v4[i].x, v4[i].y, v4[i].z, 0.0f};
                std::memcpy(tmp.data() + 16 * i, q, 16);
            } else {
                std::memcpy(tmp.data() + 4 * i, &v4[i].w, 4);
            }
        }
        r = PHX_OK;
        break;
    case PHX_BUF_SORTED_POWER:
        r = dcopy(s_power.as<u32>() + poff + e0, 4 * ne);
        break;
    case PHX_BUF_EMIT_COUNT:
        r = dcopy(counts.as<u32>() + d.emit_base + e0, 4 * ne);
        break;
    case PHX_BUF_BVH_NODES:
        std::memcpy(tmp.data(), sc[s].nodes.data() + e0, sizeof(phx_bvh_node) * ne);
        r = PHX_OK;
        break;
    case PHX_BUF_ROUND_RNG:
        r = dcopy(d_rng.as<u32>() + s, 4);
        break;
    case PHX_BUF_SORT_PERM:
        if (!(r = fetch32(perm + poff + e0, v)))
            for (uint64_t i = 0; i < ne; i++)
                ((uint32_t *)tmp.data())[i] = v[i] - poff;
        break;
    default:
        return fail(PHX_E_INVALID, "unknown buffer id");
    }
    if (r)
        return r;
    std::memcpy(dst, tmp.data() + (off - e0 * bd.esize), bytes);
    return PHX_OK;
}

int Engine::write_buffer(uint32_t s, int which, const void *src, uint64_t off, uint64_t bytes) {
    adjoint_invalidate();
    if (sc.size() != 1 || s != 0)
        return fail(PHX_E_UNSUPPORTED, "buffer writes are only available on single-scene contexts");
    if (!src && bytes)
        return fail(PHX_E_INVALID, "null source");
    const SceneDesc &d = sc[0].desc;
    CK(cudaStreamSynchronize(st));
    auto put = [&](void *base, size_t cap) -> int {
        if (off + bytes > cap)
            return fail(PHX_E_INVALID, "write past the end of the buffer");
        CK(cudaMemcpy((char *)base + off, src, bytes, cudaMemcpyHostToDevice));
        return PHX_OK;
    };
    // the gather reads each record's decoded direction and power: refresh them after host writes
    auto decode_records = [&]() -> int {
        launch_decode_records(s_posdir.as<float4>(), s_power.as<u32>(), max_photons, s_dir.as<float4>(),
                              s_pow.as<float4>(), st);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(st));
        return PHX_OK;
    };
    const size_t P = d.n_pixels, N = max_photons;
    switch (which) {
    case PHX_BUF_HP_POS: case PHX_BUF_HP_NORMAL: case PHX_BUF_HP_THROUGHPUT: case PHX_BUF_HP_BASE_COLOR:
    case PHX_BUF_HP_DIRECT: case PHX_BUF_HP_EMISSION:
        stage_state |= 1;
        return put(hp[which].p, 16 * P);
    case PHX_BUF_FLUX:
        return put(flux.p, 16 * P);
    case PHX_BUF_RADIANCE:
        return put(radiance.p, 16 * P);
    case PHX_BUF_PHOTON_WEIGHT:
        return put(weight.p, 4 * P);
    case PHX_BUF_PHOTON_POS:
        return put(ph_pos.p, 16 * N);
    case PHX_BUF_SORTED_POWER: {
        stage_state |= 4;
        const int r = put(s_power.p, 4 * N);
        return r ? r : decode_records();
    }
    case PHX_BUF_CELL_START:
        stage_state |= 4;
        return put(cell_start.p, 4 * (size_t)d.n_cells);
    case PHX_BUF_ROUND_RNG:
        return put(d_rng.p, 4);
    case PHX_BUF_PHOTON_POWER: case PHX_BUF_PHOTON_DIR: case PHX_BUF_SORTED_POS: case PHX_BUF_SORTED_DIR: {
        const bool sorted = which == PHX_BUF_SORTED_POS || which == PHX_BUF_SORTED_DIR;
        const size_t es = which == PHX_BUF_SORTED_POS ? 16 : 4;
        if (off % es || bytes % es)
            return fail(PHX_E_INVALID, "unaligned partial write");
        const uint64_t e0 = off / es, ne = bytes / es;
        if (e0 + ne > N)
            return fail(PHX_E_INVALID, "write past the end of the buffer");
        if (sorted) {
            std::vector<float4> v(ne);
            CK(cudaMemcpy(v.data(), s_posdir.as<float4>() + e0, 16 * ne, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < ne; i++) {
                if (which == PHX_BUF_SORTED_POS) {
                    const float *q = (const float *)src + 4 * i;
                    v[i].x = q[0];
                    v[i].y = q[1];
                    v[i].z = q[2];
                } else {
                    std::memcpy(&v[i].w, (const uint32_t *)src + i, 4);
                }
            }
            CK(cudaMemcpy(s_posdir.as<float4>() + e0, v.data(), 16 * ne, cudaMemcpyHostToDevice));
            stage_state |= 4;
            if (int r = decode_records())
                return r;
        } else {
            std::vector<uint2> v(ne);
            CK(cudaMemcpy(v.data(), ph_pd.as<uint2>() + e0, 8 * ne, cudaMemcpyDeviceToHost));
            for (uint64_t i = 0; i < ne; i++) {
                uint32_t x = ((const uint32_t *)src)[i];
                if (which == PHX_BUF_PHOTON_POWER)
                    v[i].x = x;
                else
                    v[i].y = x;
            }
            CK(cudaMemcpy(ph_pd.as<uint2>() + e0, v.data(), 8 * ne, cudaMemcpyHostToDevice));
        }
        return PHX_OK;
    }
    default:
        return fail(PHX_E_UNSUPPORTED, "buffer is not writable");
    }
}

int Engine::info(uint32_t s, phx_info *o) {
    if (s >= sc.size() || !o)
        return fail(PHX_E_INVALID, "bad info request");
    std::memset(o, 0, sizeof(*o));
    const SceneSlot &S = sc[s];
    o->n_pixels = S.desc.n_pixels;
    o->width = S.desc.width;
    o->height = S.desc.height;
    o->photons_per_round = S.prm.photons_per_round;
    o->photon_buf_size = S.prm.photons_per_round * S.prm.max_photon_bounces;
    o->bucket_count = S.desc.n_cells;
    o->n_photons = S.n_photons_last;
    o->n_bvh_nodes = (uint32_t)S.nodes.size();
    o->bvh_depth = S.depth;
    o->rounds_done = S.rounds;
    o->total_photons_emitted = S.total_emitted;
    o->hash = S.hash;
    o->sort_passes = radix_passes(key_bits);
    o->trav_depth = S.trav_depth;
    o->trav_inner_nodes = S.trav_inner;
    o->setup_ms = S.setup_ms;
    o->bvh_build_ms = S.bvh_ms;
    // seeds, trace, [sample, shadow, resolve], emit, count scan, compaction, hash, cell scan, 3 per
    // sort pass, records, gather (+1 with the specular NEE deferred: its resolve; k_shadow traces
    // its rays; +1 for the photon start pre-pass of the lane-refill form).  The sampling kernel runs
    // only for scenes whose light samples vary in RNG draws.
    bool presample = false;
    for (const auto &sl : sc)
        presample = presample || sl.desc.light_draws == LIGHT_DRAWS_VARY;
    o->kernels_per_round = 9 + 3 * o->sort_passes + (tune.nee_wavefront ? (presample ? 3 : 2) : 0) +
                           (spec_deferred() ? 1 : 0) + (tune.persistent && photon_prestart() ? 1 : 0) +
                           (tune.gather_sorted && pix_key_bits ? 1 + 3 * radix_passes(pix_key_bits) : 0);
    CK(cudaStreamSynchronize(st));
    uint32_t v[3] = {0, 0, 0};
    CK(cudaMemcpy(&v[0], d_ovf.p, 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&v[1], d_err.p, 4, cudaMemcpyDeviceToHost));
    if (spec_next.p)
        CK(cudaMemcpy(&v[2], spec_next.p, 4, cudaMemcpyDeviceToHost));
    o->stack_overflows = v[0];
    o->error_flags = v[1];
    o->spec_samples = spec_deferred() ? std::min(v[2], total_nee) : 0u; // claimed slots, capped as traced
    return PHX_OK;
}

int Engine::image(uint32_t s, float exposure, int tonemap, uint64_t total_photons, uint32_t rounds, float *rgb,
                  uint8_t *ldr) {
    if (s >= sc.size())
        return fail(PHX_E_INVALID, "scene index out of range");
    const SceneSlot &S = sc[s];
    if (total_photons == 0 && rounds == 0) {
        total_photons = S.total_emitted;
        rounds = S.rounds;
    }
    const uint32_t n = S.desc.n_pixels;
    int r;
    if (img_rgb.bytes < (size_t)n * 12 && (r = img_rgb.alloc((size_t)n * 12)))
        return r;
    if (img_ldr.bytes < (size_t)n * 3 && (r = img_ldr.alloc((size_t)n * 3)))
        return r;
    float inv_ph = total_photons > 0 ? 1.0f / (float)total_photons : 0.0f; // output.cpp:56-57
    float inv_r = rounds > 0 ? 1.0f / (float)rounds : 0.0f;
    launch_image(flux.as<float4>() + S.desc.pixel_base, radiance.as<float4>() + S.desc.pixel_base, n, exposure, tonemap,
                 inv_ph, inv_r, rgb ? img_rgb.as<float>() : nullptr, ldr ? img_ldr.as<uint8_t>() : nullptr, st);
    if (rgb)
        CK(cudaMemcpyAsync(rgb, img_rgb.p, (size_t)n * 12, cudaMemcpyDeviceToHost, st));
    if (ldr)
        CK(cudaMemcpyAsync(ldr, img_ldr.p, (size_t)n * 3, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return PHX_OK;
}

} // namespace phx
