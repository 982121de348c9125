// capi.cu — the extern "C" boundary of libphx.so (declared in include/phx.h).  Every entry point
// validates its handle and arguments, catches every C++ exception and reports failures as status
// codes with a message in phx_last_error(); nothing traps or throws across the boundary.
#include "engine.hpp"
#include "nccl_dl.hpp"

#include <chrono>
#include <cstring>
#include <new>

using namespace phx;

// byte layouts shared with the reference (include/common/*.h) and with the ctypes mirror
static_assert(sizeof(phx_triangle) == 176, "Triangle layout");
static_assert(sizeof(phx_material) == 96, "Material layout");
static_assert(sizeof(phx_uv_transform_block) == 192, "UvTransformBlock layout");
static_assert(sizeof(phx_light) == 128, "Light layout");
static_assert(sizeof(phx_camera_params) == 112, "CameraParams layout");
static_assert(sizeof(phx_bvh_node) == 32, "BvhNode layout");
static_assert(sizeof(phx_photon_hash_data) == 48, "PhotonHashData layout");
static_assert(sizeof(phx_texture_meta) == 16, "TextureMeta layout");
static_assert(offsetof(phx_scene, camera) == 128 && sizeof(phx_scene) == 240, "phx_scene layout");
static_assert(offsetof(phx_info, hash) == 64 && sizeof(phx_info) == 144, "phx_info layout");
static_assert(sizeof(phx_params) == 64 && sizeof(phx_tuning) == 48 && sizeof(phx_scene_spec) == 40, "param layout");

namespace {

template <class F> int guard(F &&f) {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        return fail(PHX_E_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        return fail(PHX_E_INVALID, e.what());
    } catch (...) {
        return fail(PHX_E_INVALID, "unknown C++ exception");
    }
}

Engine *eng(void *h) { return reinterpret_cast<Engine *>(h); }

struct SceneHandle {
    SceneStore store;
};

} // namespace

extern "C" {

PHX_API const char *phx_last_error(void) { return g_last_error.c_str(); }
PHX_API const char *phx_version(void) { return "phx 0.1 (sm_100a)"; }

PHX_API int phx_create(const phx_scene *scene, const phx_params *params, int device, void **out_ctx) {
    return guard([&]() -> int {
        if (!out_ctx || !scene || !params)
            return fail(PHX_E_INVALID, "null argument");
        *out_ctx = nullptr;
        auto *e = new Engine();
        int r = e->create(scene, params, 1, device);
        if (r) {
            std::string msg = g_last_error;
            delete e;
            return fail(r, msg);
        }
        *out_ctx = e;
        return PHX_OK;
    });
}

PHX_API int phx_destroy(void *ctx) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        delete eng(ctx);
        return PHX_OK;
    });
}

PHX_API int phx_get_info(void *ctx, phx_info *out) {
    return guard([&]() -> int { return ctx ? eng(ctx)->info(0, out) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_trace_rays(void *ctx, uint32_t seed) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        Engine *e = eng(ctx);
        int r = e->set_seed(seed);
        if (r)
            return r;
        e->enq_trace();
        cudaError_t c = cudaGetLastError();
        return c == cudaSuccess ? PHX_OK : fail(PHX_E_CUDA, cudaGetErrorString(c));
    });
}

PHX_API int phx_emit_photons(void *ctx, uint32_t seed) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        Engine *e = eng(ctx);
        int r = e->set_seed(seed);
        if (r)
            return r;
        e->enq_emit();
        uint32_t n = 0;
        if ((r = e->read_total(&n))) // renderer.cpp:113-115
            return r;
        e->sc[0].n_photons_last = n;
        if (n == 0)
            return fail(PHX_E_NO_PHOTONS, "no photon hit (renderer.cpp:117-118)");
        return PHX_OK;
    });
}

PHX_API int phx_hash_sort(void *ctx) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        Engine *e = eng(ctx);
        if (!(e->stage_state & 2))
            return fail(PHX_E_STATE, "hash_sort before emit_photons");
        e->enq_hash_sort();
        return e->sync_and_check();
    });
}

PHX_API int phx_gather(void *ctx, float alpha) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        Engine *e = eng(ctx);
        if ((e->stage_state & 5) != 5)
            return fail(PHX_E_STATE, "gather before trace_rays and hash_sort");
        if (!(alpha >= 0.0f))
            return fail(PHX_E_INVALID, "sppm_alpha must be non-negative");
        if (alpha != e->sc[0].desc.alpha) {
            int r = e->set_alpha(alpha);
            if (r)
                return r;
        }
        e->enq_gather();
        return e->sync_and_check(); // renderer.cpp:160
    });
}

PHX_API int phx_round(void *ctx) {
    return guard([&]() -> int { return ctx ? eng(ctx)->plain_round() : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_iterate(void *ctx, uint32_t rounds) {
    return guard([&]() -> int { return ctx ? eng(ctx)->graph_rounds(rounds) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_round_seeded(void *ctx, uint32_t seed) {
    return guard([&]() -> int { return ctx ? eng(ctx)->seeded_round(seed) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_sync(void *ctx) {
    return guard([&]() -> int { return ctx ? eng(ctx)->sync_and_check() : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_read_buffer(void *ctx, int which, void *dst, uint64_t off, uint64_t bytes) {
    return guard([&]() -> int { return ctx ? eng(ctx)->read_buffer(0, which, dst, off, bytes) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_write_buffer(void *ctx, int which, const void *src, uint64_t off, uint64_t bytes) {
    return guard([&]() -> int { return ctx ? eng(ctx)->write_buffer(0, which, src, off, bytes) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_set_n_photons(void *ctx, uint32_t n) {
    return guard([&]() -> int { return ctx ? eng(ctx)->set_n_photons(n) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_image(void *ctx, float exposure, int tonemap, uint64_t total_photons, uint32_t rounds, float *rgb,
                      uint8_t *ldr) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->image(0, exposure, tonemap, total_photons, rounds, rgb, ldr)
                   : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_bvh_build(const phx_triangle *tris, uint32_t n, phx_bvh_node *out, uint32_t *depth) {
    return guard([&]() -> int {
        if (!tris || !out || n == 0)
            return fail(PHX_E_INVALID, "bad arguments");
        std::vector<phx_bvh_node> nodes;
        if (!bvh_build(tris, n, nodes, depth))
            return fail(PHX_E_INVALID, "degenerate or infinite triangle bounding box");
        std::memcpy(out, nodes.data(), nodes.size() * sizeof(phx_bvh_node));
        return PHX_OK;
    });
}

#ifndef CK
#define CK(x)                                                                                                          \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return fail(PHX_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
    } while (0)
#endif

PHX_API int phx_traversal_bvh_build(const phx_triangle *tris, uint32_t n, uint32_t max_leaf, int wide, int device,
                                    phx_bvh_packed *out) {
    return guard([&]() -> int {
        if (!tris || !out || !out->nodes || !out->trirec || !out->leaf_tri || n == 0 || max_leaf < 1 ||
            max_leaf > 16 || wide < 0 || wide > 2)
            return fail(PHX_E_INVALID, "bad arguments");
        const bool quant = wide == 2;
        std::vector<phx_bvh_node> ref;
        if (!bvh_build(tris, n, ref, nullptr))
            return fail(PHX_E_INVALID, "degenerate or infinite triangle bounding box");
        const std::vector<uint32_t> ranks = reference_leaf_ranks(ref, n);
        const uint32_t per = quant ? 16u : wide ? 28u : 16u;
        if (device < 0) {
            const auto t0 = std::chrono::steady_clock::now();
            PackedBvh pk;
            if (!bvh_build_sah(tris, n, ranks, max_leaf, pk))
                return fail(PHX_E_INVALID, "SAH build failed");
            if (wide)
                bvh_widen(pk);
            std::vector<uint32_t> qn;
            if (quant)
                qn = bvh_quantize(pk);
            out->build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
            const std::vector<float> &nodes = wide ? pk.wnodes : pk.cnodes;
            if (quant)
                std::memcpy(out->nodes, qn.data(), qn.size() * 4);
            else
                std::memcpy(out->nodes, nodes.data(), nodes.size() * 4);
            std::memcpy(out->trirec, pk.trirec.data(), pk.trirec.size() * 4);
            std::memcpy(out->leaf_tri, pk.leaf_tri.data(), pk.leaf_tri.size() * 4);
            out->n_nodes = (uint32_t)(nodes.size() / (wide ? 28u : 16u));
            out->root = wide ? pk.wroot : pk.root;
            out->depth = pk.depth;
            out->wdepth = wide ? pk.wdepth : 0u;
            return PHX_OK;
        }
        CK(cudaSetDevice(device));
        cudaStream_t st;
        CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct Cleanup {
            cudaStream_t st;
            std::vector<void *> p;
            DeviceBvh db;
            ~Cleanup() {
                db.release();
                for (void *q : p)
                    cudaFree(q);
                cudaStreamDestroy(st);
            }
        } c{st, {}, {}};
        auto dalloc = [&](size_t bytes) -> void * {
            void *q = nullptr;
            if (cudaMalloc(&q, std::max<size_t>(bytes, 16)) != cudaSuccess)
                return nullptr;
            c.p.push_back(q);
            return q;
        };
        auto *d_tris = static_cast<phx_triangle *>(dalloc(sizeof(phx_triangle) * (size_t)n));
        auto *d_rank = static_cast<uint32_t *>(dalloc(4 * (size_t)n));
        auto *d_rec = static_cast<float4 *>(dalloc(48 * (size_t)n));
        auto *d_nrm = static_cast<float4 *>(dalloc(48 * (size_t)n));
        auto *d_tan = static_cast<float4 *>(dalloc(48 * (size_t)n));
        auto *d_uv = static_cast<float4 *>(dalloc(32 * (size_t)n));
        auto *d_q = static_cast<uint32_t *>(dalloc(quant ? 64 * (size_t)n : 16));
        if (!d_tris || !d_rank || !d_rec || !d_nrm || !d_tan || !d_uv || !d_q)
            return fail(PHX_E_OOM, "device allocation failed");
        CK(cudaMemcpy(d_tris, tris, sizeof(phx_triangle) * (size_t)n, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(d_rank, ranks.data(), 4 * (size_t)n, cudaMemcpyHostToDevice));
        const auto t0 = std::chrono::steady_clock::now();
        std::string msg;
        const int rc = bvh_device_build(d_tris, n, max_leaf, wide != 0, st, c.db, msg);
        if (rc)
            return fail(rc == 2 ? PHX_E_OOM : rc == 1 ? PHX_E_INVALID : PHX_E_CUDA, msg);
        if (bvh_device_finish(d_tris, d_rank, n, c.db, d_rec, d_nrm, d_tan, d_uv, st))
            return fail(PHX_E_CUDA, "device BVH triangle records: launch failed");
        if (quant && c.db.n_wide)
            CK(bvh_device_quantize(c.db.wnodes, c.db.n_wide, d_q, st));
        CK(cudaStreamSynchronize(st));
        out->build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
        out->n_nodes = wide ? c.db.n_wide : c.db.n_inner;
        out->root = wide ? c.db.wroot : c.db.root;
        out->depth = c.db.depth;
        out->wdepth = wide ? c.db.wdepth : 0u;
        if (out->n_nodes)
            CK(cudaMemcpy(out->nodes, quant ? (const void *)d_q : wide ? (const void *)c.db.wnodes : c.db.cnodes,
                          (size_t)out->n_nodes * per * 4, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(out->trirec, d_rec, 48 * (size_t)n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(out->leaf_tri, c.db.leaf_tri, 4 * (size_t)n, cudaMemcpyDeviceToHost));
        return PHX_OK;
    });
}

PHX_API int phx_hash_info(const phx_bvh_node *root, uint32_t grid_res, phx_photon_hash_data *out) {
    return guard([&]() -> int {
        if (!root || !out || grid_res < 1 || grid_res > 255)
            return fail(PHX_E_INVALID, "bad arguments");
        *out = hash_info(*root, grid_res);
        return PHX_OK;
    });
}

PHX_API int phx_camera_make(const float position[3], const float look_at[3], const float up[3], float hfov_deg,
                            float aspect, float defocus_angle, float focus_distance, phx_camera_params *out) {
    return guard([&]() -> int {
        if (!position || !look_at || !up || !out || !(aspect > 0.0f))
            return fail(PHX_E_INVALID, "bad arguments");
        return camera_make(position, look_at, up, hfov_deg, aspect, defocus_angle, focus_distance, out);
    });
}

PHX_API int phx_lum_pref_sum(const phx_light *lights, uint32_t n, float *out) {
    return guard([&]() -> int {
        if ((!lights || !out) && n)
            return fail(PHX_E_INVALID, "bad arguments");
        lum_pref_sum(lights, n, out);
        return PHX_OK;
    });
}

PHX_API int phx_scene_generate(const phx_scene_spec *spec, phx_scene *out, void **handle) {
    return guard([&]() -> int {
        if (!spec || !out || !handle)
            return fail(PHX_E_INVALID, "null argument");
        auto *h = new SceneHandle();
        std::string err;
        int r = scene_generate(*spec, h->store, err);
        if (r) {
            delete h;
            return fail(r, err);
        }
        h->store.view(out);
        *handle = h;
        return PHX_OK;
    });
}

PHX_API int phx_scene_load_gltf(const char *path, const phx_gltf_options *options, phx_scene *out, void **handle) {
    return guard([&]() -> int {
        if (!path || !out || !handle)
            return fail(PHX_E_INVALID, "null argument");
        phx_gltf_options opt{};
        if (options)
            opt = *options;
        auto *h = new SceneHandle();
        std::string err;
        int r = scene_load_gltf(path, opt, h->store, err);
        if (r) {
            delete h;
            return fail(r, err);
        }
        h->store.view(out);
        *handle = h;
        return PHX_OK;
    });
}

PHX_API int phx_scene_free(void *handle) {
    return guard([&]() -> int {
        if (!handle)
            return fail(PHX_E_INVALID, "null handle");
        delete reinterpret_cast<SceneHandle *>(handle);
        return PHX_OK;
    });
}

PHX_API int phx_batch_create(const phx_scene *scenes, const phx_params *params, uint32_t n, int device,
                             void **out_batch) {
    return guard([&]() -> int {
        if (!out_batch || !scenes || !params || n == 0)
            return fail(PHX_E_INVALID, "bad arguments");
        *out_batch = nullptr;
        auto *e = new Engine();
        int r = e->create(scenes, params, n, device);
        if (r) {
            std::string msg = g_last_error;
            delete e;
            return fail(r, msg);
        }
        *out_batch = e;
        return PHX_OK;
    });
}

PHX_API int phx_batch_destroy(void *b) { return phx_destroy(b); }

PHX_API int phx_batch_iterate(void *b, uint32_t rounds, int mode) {
    return guard([&]() -> int {
        if (!b)
            return fail(PHX_E_INVALID, "null batch");
        Engine *e = eng(b);
        if (mode == 1)
            return e->graph_rounds(rounds);
        if (mode != 0)
            return fail(PHX_E_INVALID, "mode must be 0 or 1");
        for (uint32_t i = 0; i < rounds; i++) {
            int r = e->plain_round();
            if (r)
                return r;
        }
        return PHX_OK;
    });
}

PHX_API int phx_batch_set_active(void *b, uint32_t scene, int active) {
    return guard([&]() -> int {
        return b ? eng(b)->set_active(scene, active != 0) : fail(PHX_E_INVALID, "null batch");
    });
}

PHX_API int phx_batch_read_buffer(void *b, uint32_t scene, int which, void *dst, uint64_t off, uint64_t bytes) {
    return guard([&]() -> int { return b ? eng(b)->read_buffer(scene, which, dst, off, bytes) : fail(PHX_E_INVALID, "null batch"); });
}

PHX_API int phx_batch_get_info(void *b, uint32_t scene, phx_info *out) {
    return guard([&]() -> int { return b ? eng(b)->info(scene, out) : fail(PHX_E_INVALID, "null batch"); });
}

PHX_API int phx_batch_image(void *b, uint32_t scene, float exposure, int tonemap, float *rgb) {
    return guard([&]() -> int { return b ? eng(b)->image(scene, exposure, tonemap, 0, 0, rgb, nullptr) : fail(PHX_E_INVALID, "null batch"); });
}

PHX_API int phx_get_tuning(void *ctx, phx_tuning *out) {
    return guard([&]() -> int {
        if (!ctx || !out)
            return fail(PHX_E_INVALID, "null argument");
        *out = eng(ctx)->tune;
        return PHX_OK;
    });
}

PHX_API int phx_set_tuning(void *ctx, const phx_tuning *in) {
    return guard([&]() -> int {
        if (!ctx || !in)
            return fail(PHX_E_INVALID, "null argument");
        const uint32_t blocks[3] = {in->trace_block, in->emit_block, in->gather_block};
        for (uint32_t b : blocks)
            if (b != 0 && (b % 32 != 0 || b > 1024))
                return fail(PHX_E_INVALID, "block sizes must be multiples of 32 up to 1024");
        if (in->trace_blocks_per_sm > 64 || in->emit_blocks_per_sm > 64)
            return fail(PHX_E_INVALID, "blocks_per_sm out of range");
        if (in->pipeline_rounds > 8)
            return fail(PHX_E_INVALID, "pipeline_rounds must be at most 8");
        Engine *e = eng(ctx);
        e->tune = *in;
        e->invalidate_graph(); // the next replay is captured with the new launch shape
        return PHX_OK;
    });
}

PHX_API int phx_autotune(void *ctx, uint32_t rounds_per_trial, phx_tuning *chosen) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->autotune(rounds_per_trial, chosen) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_profile(void *ctx, int enable) {
    return guard([&]() -> int {
        if (!ctx)
            return fail(PHX_E_INVALID, "null context");
        eng(ctx)->set_profiling(enable != 0);
        return PHX_OK;
    });
}

PHX_API int phx_stage_ms(void *ctx, float *out, uint32_t n) {
    return guard([&]() -> int {
        if (!ctx || !out || n < (uint32_t)ST__N)
            return fail(PHX_E_INVALID, "need room for every stage");
        eng(ctx)->stage_ms(out);
        return PHX_OK;
    });
}

PHX_API uint64_t phx_get_stream(void *ctx) { return ctx ? (uint64_t)(uintptr_t)eng(ctx)->st : 0; }

PHX_API int phx_selftest_lookback_timeout(int device, uint32_t n, uint32_t *err_flags) {
    return guard([&]() -> int {
        if (!err_flags || n == 0 || n > (1u << 26))
            return fail(PHX_E_INVALID, "bad arguments");
        *err_flags = 0;
        int rc = selftest_lookback_timeout(device, n, err_flags);
        if (rc == 2)
            return fail(PHX_E_OOM, "self-test allocation failed");
        if (rc == 3)
            return fail(PHX_E_CUDA, "self-test kernel failed");
        if (*err_flags & ERR_LOOKBACK_TIMEOUT)
            return fail(PHX_E_TIMEOUT, "look-back wait gave up as intended (tile 0 withheld)");
        return PHX_OK;
    });
}

PHX_API int phx_set_materials(void *ctx, const phx_material *materials, uint32_t n) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->set_materials(materials, n) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_set_lights(void *ctx, const phx_light *lights, uint32_t n) {
    return guard([&]() -> int { return ctx ? eng(ctx)->set_lights(lights, n) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_adjoint_n_params(void *ctx, uint32_t *n) {
    return guard([&]() -> int {
        if (!ctx || !n)
            return fail(PHX_E_INVALID, "null argument");
        *n = eng(ctx)->n_params();
        return PHX_OK;
    });
}

PHX_API int phx_adjoint_forward(void *ctx, uint32_t rounds, float *image) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->adjoint_forward(rounds, image) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_adjoint_backward(void *ctx, const float *dl_dimage, float *grad, uint32_t n_grad) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->adjoint_backward(dl_dimage, grad, n_grad) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_shard(void *ctx, uint32_t rank, uint32_t world) {
    return guard([&]() -> int { return ctx ? eng(ctx)->set_shard(rank, world) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_shard_begin(void *ctx, uint32_t *n_local) {
    return guard([&]() -> int { return ctx ? eng(ctx)->shard_begin(n_local) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_shard_get_photons(void *ctx, float *pos4, uint32_t *pd2, uint32_t n) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->shard_get_photons(pos4, pd2, n) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_shard_put_photons(void *ctx, const float *pos4, const uint32_t *pd2, uint32_t n_all) {
    return guard([&]() -> int {
        return ctx ? eng(ctx)->shard_put_photons(pos4, pd2, n_all) : fail(PHX_E_INVALID, "null context");
    });
}

PHX_API int phx_shard_end(void *ctx) {
    return guard([&]() -> int { return ctx ? eng(ctx)->shard_end() : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_nccl_unique_id(uint8_t *out, uint32_t n) {
    return guard([&]() -> int {
        std::string why;
        const NcclApi *api = nccl_api(&why);
        if (!api)
            return fail(PHX_E_UNSUPPORTED, why);
        if (!out || n < sizeof(ncclUniqueId))
            return fail(PHX_E_INVALID, "need 128 bytes for the NCCL unique id");
        ncclUniqueId id;
        ncclResult_t r = api->GetUniqueId(&id);
        if (r != ncclSuccess)
            return fail(PHX_E_CUDA, std::string("ncclGetUniqueId: ") + api->GetErrorString(r));
        std::memcpy(out, &id, sizeof(id));
        return PHX_OK;
    });
}

PHX_API int phx_shard_nccl(void *ctx, const uint8_t *id) {
    return guard([&]() -> int { return ctx ? eng(ctx)->shard_nccl_init(id) : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_shard_round(void *ctx) {
    return guard([&]() -> int { return ctx ? eng(ctx)->shard_round() : fail(PHX_E_INVALID, "null context"); });
}

PHX_API int phx_scan_noalloc(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *total, uint64_t stream) {
    return guard([&]() -> int {
        if (n && (!in || !out))
            return fail(PHX_E_INVALID, "null buffer");
        std::string msg;
        int rc = scan_noalloc(in, out, n, total, (cudaStream_t)(uintptr_t)stream, msg);
        if (rc == 1)
            return fail(PHX_E_INVALID, msg);
        if (rc == 3)
            return fail(PHX_E_CUDA, msg);
        if (rc == 4)
            return fail(PHX_E_TIMEOUT, msg);
        return PHX_OK;
    });
}

static int filter_entry(int mode, const int32_t *in, float *out, const float *weights, uint32_t width,
                        uint32_t height, uint32_t k, float *kernel_ms) {
    return guard([&]() -> int {
        std::string msg;
        const int rc = denoise_filter(mode, in, out, weights, width, height, k, kernel_ms, msg);
        if (rc == 1)
            return fail(PHX_E_INVALID, msg);
        if (rc == 3)
            return fail(PHX_E_CUDA, msg);
        return PHX_OK;
    });
}

PHX_API int phx_mean_filter(const int32_t *in, float *out, uint32_t width, uint32_t height, uint32_t k,
                            float *kernel_ms) {
    return filter_entry(0, in, out, nullptr, width, height, k, kernel_ms);
}

PHX_API int phx_median_filter(const int32_t *in, float *out, uint32_t width, uint32_t height, uint32_t k,
                              float *kernel_ms) {
    return filter_entry(1, in, out, nullptr, width, height, k, kernel_ms);
}

PHX_API int phx_weighted_filter(const int32_t *in, float *out, const float *weights, uint32_t width, uint32_t height,
                                uint32_t k, float *kernel_ms) {
    return filter_entry(2, in, out, weights, width, height, k, kernel_ms);
}

} // extern "C"
