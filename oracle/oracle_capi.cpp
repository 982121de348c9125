// oracle_capi.cpp — TEST INFRASTRUCTURE ONLY: extern "C" entry points of the CPU oracle
// (liboracle.so), called through ctypes by tests/ and by bench.py's CPU-baseline leg.
// Pinned to the reference's own code compiled for the CPU (see phx_oracle.hpp).
#include "phx_frozen.hpp"
#include "phx_oracle.hpp"

// the procedural scene generators (phosphor_b200/csrc/scenes.cpp, compiled into this library too):
// the seeded synthetic inputs, so that a CPU-only run of the oracle never loads the CUDA library
#include "../phosphor_b200/csrc/host.hpp"

#include <atomic>
#include <chrono>
#include <functional>
#include <thread>

using namespace orc;

namespace {

void parallel_for(uint32_t n, int threads, const std::function<void(uint32_t, uint32_t)> &fn) {
    if (threads <= 1 || n < 64) {
        fn(0, n);
        return;
    }
    std::atomic<uint32_t> next{0};
    const uint32_t chunk = std::max<uint32_t>(16, n / (uint32_t)(threads * 16));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; t++)
        pool.emplace_back([&]() {
            for (;;) {
                uint32_t b = next.fetch_add(chunk);
                if (b >= n)
                    break;
                fn(b, std::min(n, b + chunk));
            }
        });
    for (auto &th : pool)
        th.join();
}

struct OrcCtx {
    Scene sc;
    u32 n_materials = 0;
    std::vector<phx_bvh_node> bvh;
    u32 depth = 0;
};

template <class R> void store4(void *out, size_t i, const V4<R> &v) {
    R *o = (R *)out + 4 * i;
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
template <class R> V4<R> load4(const void *in, size_t i) {
    const R *p = (const R *)in + 4 * i;
    return mk<R>(p[0], p[1], p[2], p[3]);
}

u32 tree_depth(const std::vector<phx_bvh_node> &n, u32 i, u32 d) {
    if (as_uint(n[i].min.w) != 0xFFFFFFFFu)
        return d;
    return std::max(tree_depth(n, i + 1, d + 1), tree_depth(n, as_uint(n[i].max.w), d + 1));
}

template <class R>
void trace_impl(OrcCtx *o, u32 w, u32 h, u32 seed, u32 ds, const u32 *ids, u32 n_ids, void *out, int threads) {
    parallel_for(n_ids, threads, [&](u32 b, u32 e) {
        for (u32 i = b; i < e; i++) {
            u32 tid = ids ? ids[i] : i;
            HitPoint<R> hp = trace_pixel<R>(o->sc, w, h, seed, ds, tid);
            // PHX_BUF order: pos, normal, throughput, base_color, direct, emission (6 per pixel)
            store4<R>(out, (size_t)i * 6 + 0, hp.pos);
            store4<R>(out, (size_t)i * 6 + 1, hp.normal);
            store4<R>(out, (size_t)i * 6 + 2, hp.throughput);
            store4<R>(out, (size_t)i * 6 + 3, hp.base_color);
            store4<R>(out, (size_t)i * 6 + 4, hp.direct);
            store4<R>(out, (size_t)i * 6 + 5, hp.emission);
        }
    });
}

template <class R>
int emit_impl(OrcCtx *o, u32 tb, u32 te, u32 maxb, u32 seed, u32 *counts, void *pos, u32 *power, u32 *dir,
              uint64_t cap, uint64_t *n_out, int threads) {
    u32 n = te - tb;
    std::vector<StoredPhoton<R>> slots((size_t)n * maxb);
    std::vector<u32> cnt(n);
    parallel_for(n, threads, [&](u32 b, u32 e) {
        for (u32 i = b; i < e; i++)
            cnt[i] = emit_photon<R>(o->sc, tb + i, maxb, seed, &slots[(size_t)i * maxb]);
    });
    uint64_t k = 0;
    for (u32 i = 0; i < n; i++) {
        if (counts)
            counts[i] = cnt[i];
        for (u32 j = 0; j < cnt[i]; j++) {
            if (k < cap) {
                store4<R>(pos, k, slots[(size_t)i * maxb + j].pos);
                power[k] = slots[(size_t)i * maxb + j].power;
                dir[k] = slots[(size_t)i * maxb + j].dir;
            }
            k++;
        }
    }
    *n_out = k;
    return k > cap ? PHX_E_OVERFLOW : PHX_OK;
}

// scan_small_chunks.cl + scan_big_chunks.cl + scan_add_offsets.cl, restated with their chunking
void reference_scan(const u32 *counts, u32 n_cells, u32 *cell_start) {
    u32 n_chunks = (n_cells + SCAN_CHUNK_SIZE - 1) / SCAN_CHUNK_SIZE;
    std::vector<u32> chunk_sums(n_chunks), big(n_chunks);
    std::vector<u32> sh(SCAN_CHUNK_SIZE), sums(SCAN_WG_SIZE);
    for (u32 wg = 0; wg < n_chunks; wg++) { // scan_small_chunks.cl:6-51
        u32 cs = wg * SCAN_CHUNK_SIZE;
        for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++)
            for (u32 i = 0; i < SCAN_ELEMENTS_PER_THREAD; i++) {
                u32 idx = cs + lt + i * SCAN_WG_SIZE;
                sh[lt + i * SCAN_WG_SIZE] = idx < n_cells ? counts[idx] : 0;
            }
        for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++) {
            u32 s = 0, st = lt * SCAN_ELEMENTS_PER_THREAD;
            for (u32 i = 0; i < SCAN_ELEMENTS_PER_THREAD; i++) {
                u32 prev = sh[st + i];
                sh[st + i] = s;
                s += prev;
            }
            sums[lt] = s;
        }
        for (u32 stride = 1; stride < SCAN_WG_SIZE; stride *= 2) {
            std::vector<u32> prev(SCAN_WG_SIZE);
            for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++)
                prev[lt] = lt >= stride ? sums[lt - stride] : 0;
            for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++)
                sums[lt] += prev[lt];
        }
        for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++) {
            u32 off = lt > 0 ? sums[lt - 1] : 0;
            for (u32 i = 0; i < SCAN_ELEMENTS_PER_THREAD; i++)
                sh[lt * SCAN_ELEMENTS_PER_THREAD + i] += off;
        }
        chunk_sums[wg] = sums[SCAN_WG_SIZE - 1];
        for (u32 lt = 0; lt < SCAN_WG_SIZE; lt++)
            for (u32 i = 0; i < SCAN_ELEMENTS_PER_THREAD; i++) {
                u32 idx = cs + lt + i * SCAN_WG_SIZE;
                if (idx < n_cells)
                    cell_start[idx] = sh[lt + i * SCAN_WG_SIZE];
            }
    }
    { // scan_big_chunks.cl:6-46 (one work group: n_chunks <= SCAN_CHUNK_SIZE)
        u32 run = 0;
        for (u32 i = 0; i < n_chunks; i++) {
            big[i] = run;
            run += chunk_sums[i];
        }
    }
    for (u32 wg = 0; wg < n_chunks; wg++) // scan_add_offsets.cl:5-18
        for (u32 i = 0; i < SCAN_CHUNK_SIZE; i++) {
            u32 idx = wg * SCAN_CHUNK_SIZE + i;
            if (idx < n_cells)
                cell_start[idx] += big[wg];
        }
}

template <class R>
void hash_impl(const void *pos, u32 n, const phx_photon_hash_data &d, u32 buckets, u32 *keys, u32 *counts) {
    std::fill(counts, counts + buckets, 0u);
    for (u32 i = 0; i < n; i++) { // hash_photons.cl:4-13
        u32 h = get_hash<R>(load4<R>(pos, i), d);
        keys[i] = h;
        counts[h]++;
    }
}

template <class R>
void scatter_impl(const void *pos, const u32 *power, const u32 *dir, const u32 *keys, u32 n, const u32 *start,
                  u32 buckets, void *spos, u32 *spower, u32 *sdir, u32 *end, u32 *perm) {
    std::memcpy(end, start, sizeof(u32) * buckets); // renderer.cpp:147
    for (u32 i = 0; i < n; i++) { // scatter_photons.cl:4-18, sequential = stable
        u32 dst = end[keys[i]]++;
        R *o = (R *)spos + 4 * (size_t)dst;
        const R *p = (const R *)pos + 4 * (size_t)i;
        o[0] = p[0];
        o[1] = p[1];
        o[2] = p[2];
        o[3] = p[3];
        spower[dst] = power[i];
        sdir[dst] = dir[i];
        if (perm)
            perm[dst] = i;
    }
}

template <class R>
void gather_impl(const void *hp6, u32 n_pixels, const void *spos, const u32 *spower, const u32 *sdir,
                 const u32 *start, const u32 *end, const phx_photon_hash_data &d, R alpha, void *flux, void *weight,
                 void *radiance, int threads) {
    const V4<R> *sp = (const V4<R> *)spos;
    parallel_for(n_pixels, threads, [&](u32 b, u32 e) {
        for (u32 i = b; i < e; i++) {
            HitPoint<R> hp;
            hp.pos = load4<R>(hp6, (size_t)i * 6 + 0);
            hp.normal = load4<R>(hp6, (size_t)i * 6 + 1);
            hp.throughput = load4<R>(hp6, (size_t)i * 6 + 2);
            hp.base_color = load4<R>(hp6, (size_t)i * 6 + 3);
            hp.direct = load4<R>(hp6, (size_t)i * 6 + 4);
            hp.emission = load4<R>(hp6, (size_t)i * 6 + 5);
            V4<R> f = load4<R>(flux, i), rad = load4<R>(radiance, i);
            R w = ((R *)weight)[i];
            gather_pixel<R>(hp, d, start, end, sp, spower, sdir, alpha, &f, &w, &rad);
            store4<R>(flux, i, f);
            store4<R>(radiance, i, rad);
            ((R *)weight)[i] = w;
        }
    });
}

// Renderer::run (renderer.cpp:59-88) for `rounds` rounds, state in precision R.
template <class R>
int render_impl(OrcCtx *o, const phx_params *p, u32 rounds, int threads, void *flux, void *weight, void *radiance,
                uint64_t *total_emitted, u32 *n_last, double *stage_seconds) {
    u32 npx = p->width * p->height;
    u32 buckets = p->grid_res * p->grid_res * p->grid_res + 1;
    uint64_t cap = (uint64_t)p->photons_per_round * p->max_photon_bounces;
    phx_photon_hash_data hd = hash_info(o->bvh[0], p->grid_res);
    std::vector<R> hp((size_t)npx * 24);
    std::vector<R> pos(cap * 4), spos(cap * 4);
    std::vector<u32> power(cap), dir(cap), spower(cap), sdir(cap), keys(cap);
    std::vector<u32> counts(buckets), start(buckets), end(buckets);
    Rng rng = pcg_seed(p->seed);
    uint64_t total = total_emitted ? *total_emitted : 0;
    using clk = std::chrono::steady_clock;
    for (u32 round = 0; round < rounds; round++) {
        u32 seed = random_u32(&rng);
        auto t0 = clk::now();
        trace_impl<R>(o, p->width, p->height, seed, p->direct_samples, nullptr, npx, hp.data(), threads);
        auto t1 = clk::now();
        uint64_t n = 0;
        int st = emit_impl<R>(o, 0, p->photons_per_round, p->max_photon_bounces, seed, nullptr, pos.data(),
                              power.data(), dir.data(), cap, &n, threads);
        if (st != PHX_OK)
            return st;
        if (n == 0)
            return PHX_E_NO_PHOTONS;
        auto t2 = clk::now();
        hash_impl<R>(pos.data(), (u32)n, hd, buckets, keys.data(), counts.data());
        reference_scan(counts.data(), buckets, start.data());
        scatter_impl<R>(pos.data(), power.data(), dir.data(), keys.data(), (u32)n, start.data(), buckets,
                        spos.data(), spower.data(), sdir.data(), end.data(), nullptr);
        auto t3 = clk::now();
        gather_impl<R>(hp.data(), npx, spos.data(), spower.data(), sdir.data(), start.data(), end.data(), hd,
                       (R)p->sppm_alpha, flux, weight, radiance, threads);
        auto t4 = clk::now();
        total += p->photons_per_round;
        if (n_last)
            *n_last = (u32)n;
        if (stage_seconds) {
            stage_seconds[0] += std::chrono::duration<double>(t1 - t0).count();
            stage_seconds[1] += std::chrono::duration<double>(t2 - t1).count();
            stage_seconds[2] += std::chrono::duration<double>(t3 - t2).count();
            stage_seconds[3] += std::chrono::duration<double>(t4 - t3).count();
        }
    }
    if (total_emitted)
        *total_emitted = total;
    return PHX_OK;
}

// The frozen-path estimator F(θ') (phx_frozen.hpp) over `rounds` rounds from a fresh state:
// linear image (radiance/R + flux/(π r² N)) in the scalar type S into img1 (npx x 3); the θ0 float
// state (bit-identical to render_impl<float>) into flux0/radiance0 when given.
template <class S>
int frozen_render_impl(OrcCtx *o, const phx_params *p, u32 rounds, const frozen::Primed<S> &pr, int threads,
                       S *img1, float *flux0, float *radiance0) {
    u32 npx = p->width * p->height;
    u32 buckets = p->grid_res * p->grid_res * p->grid_res + 1;
    u32 maxb = p->max_photon_bounces, ne = p->photons_per_round;
    phx_photon_hash_data hd = hash_info(o->bvh[0], p->grid_res);
    std::vector<HitPoint<float>> hp(npx);
    std::vector<frozen::HitPrimed<S>> hp1(npx);
    std::vector<StoredPhoton<float>> slots((size_t)ne * maxb);
    std::vector<V4<S>> slot_pow1((size_t)ne * maxb);
    std::vector<u32> cnt(ne);
    std::vector<V4<float>> flux(npx, zero4<float>()), radiance(npx, zero4<float>());
    std::vector<float> weight(npx, 0.0f);
    std::vector<V4<S>> flux1(npx, zero4<S>()), rad1(npx, zero4<S>());
    std::vector<u32> counts(buckets), start(buckets), end(buckets);
    Rng rng = pcg_seed(p->seed);
    for (u32 round = 0; round < rounds; round++) {
        u32 seed = random_u32(&rng);
        parallel_for(npx, threads, [&](u32 b, u32 e) {
            for (u32 i = b; i < e; i++)
                hp[i] = frozen::trace_pixel<S>(o->sc, pr, p->width, p->height, seed, p->direct_samples, i, &hp1[i]);
        });
        parallel_for(ne, threads, [&](u32 b, u32 e) {
            for (u32 i = b; i < e; i++)
                cnt[i] = frozen::emit_photon<S>(o->sc, pr, i, maxb, seed, &slots[(size_t)i * maxb],
                                                &slot_pow1[(size_t)i * maxb]);
        });
        std::vector<float> pos;
        std::vector<u32> power, dir;
        std::vector<V4<S>> pow1;
        for (u32 i = 0; i < ne; i++) // canonical order: path, then bounce
            for (u32 j = 0; j < cnt[i]; j++) {
                const StoredPhoton<float> &s = slots[(size_t)i * maxb + j];
                pos.insert(pos.end(), {s.pos.x, s.pos.y, s.pos.z, s.pos.w});
                power.push_back(s.power);
                dir.push_back(s.dir);
                pow1.push_back(slot_pow1[(size_t)i * maxb + j]);
            }
        u32 n = (u32)power.size();
        if (n == 0)
            return PHX_E_NO_PHOTONS;
        std::vector<u32> keys(n), spower(n), sdir(n), perm(n);
        std::vector<float> spos((size_t)n * 4);
        hash_impl<float>(pos.data(), n, hd, buckets, keys.data(), counts.data());
        reference_scan(counts.data(), buckets, start.data());
        scatter_impl<float>(pos.data(), power.data(), dir.data(), keys.data(), n, start.data(), buckets, spos.data(),
                            spower.data(), sdir.data(), end.data(), perm.data());
        std::vector<V4<S>> spow1(n);
        for (u32 k = 0; k < n; k++)
            spow1[k] = pow1[perm[k]];
        const V4<float> *sp = (const V4<float> *)spos.data();
        parallel_for(npx, threads, [&](u32 b, u32 e) {
            for (u32 i = b; i < e; i++)
                frozen::gather_pixel<S>(hp[i], hp1[i], hd, start.data(), end.data(), sp, spower.data(), sdir.data(),
                                        spow1.data(), p->sppm_alpha, &flux[i], &weight[i], &radiance[i], &flux1[i],
                                        &rad1[i]);
        });
    }
    const double n_total = (double)p->photons_per_round * rounds;
    for (u32 i = 0; i < npx; i++) {
        const double area = (double)PI_F * flux[i].w;
        const double per = area > 0.0 ? 1.0 / (area * n_total) : 0.0;
        img1[3 * (size_t)i + 0] = rad1[i].x / S((double)rounds) + flux1[i].x * S(per);
        img1[3 * (size_t)i + 1] = rad1[i].y / S((double)rounds) + flux1[i].y * S(per);
        img1[3 * (size_t)i + 2] = rad1[i].z / S((double)rounds) + flux1[i].z * S(per);
        if (flux0)
            store4<float>(flux0, i, flux[i]);
        if (radiance0)
            store4<float>(radiance0, i, radiance[i]);
    }
    return PHX_OK;
}

// output.cpp:40-83 in float (u8 quantisation left to the caller)
template <class R>
void image_impl(const void *flux, const void *radiance, u32 n, float exposure, int tonemap, uint64_t total_photons,
                u32 rounds, double *rgb) {
    R inv_ph = total_photons > 0 ? (R)1 / (R)total_photons : (R)0;
    R inv_r = rounds > 0 ? (R)1 / (R)rounds : (R)0;
    for (u32 p = 0; p < n; p++) {
        V4<R> f = load4<R>(flux, p), rad = load4<R>(radiance, p);
        R area = C<R>::PI * f.w;
        R ir = 0, ig = 0, ib = 0;
        if (area > (R)0) {
            R per = inv_ph / area;
            ir = f.x * per;
            ig = f.y * per;
            ib = f.z * per;
        }
        R c[3] = {rad.x * inv_r + ir, rad.y * inv_r + ig, rad.z * inv_r + ib};
        for (int k = 0; k < 3; k++) {
            R x = c[k] * (R)exposure;
            R out = x;
            if (tonemap) {
                R a = (R)2.51f, b = (R)0.03f, cc = (R)2.43f, dd = (R)0.59f, e = (R)0.14f;
                out = (x * (a * x + b)) / (x * (cc * x + dd) + e);
            }
            out = M<R>::pow(out, (R)1 / (R)2.2f);
            rgb[(size_t)p * 3 + k] = (double)clampr<R>(out, (R)0, (R)1);
        }
    }
}

} // namespace

extern "C" {

__attribute__((visibility("default"))) int orc_scene_generate(const phx_scene_spec *spec, phx_scene *out,
                                                             void **handle) {
    if (!spec || !out || !handle)
        return PHX_E_INVALID;
    auto *st = new phx::SceneStore();
    std::string err;
    int r = phx::scene_generate(*spec, *st, err);
    if (r) {
        delete st;
        return r;
    }
    st->view(out);
    *handle = st;
    return PHX_OK;
}

__attribute__((visibility("default"))) void orc_scene_free(void *handle) {
    delete reinterpret_cast<phx::SceneStore *>(handle);
}

// the generators' camera (Camera + focus + to_params) and light luminance prefix sum, for checks
// against the reference's own camera.cpp and scene_data.cpp
__attribute__((visibility("default"))) void orc_camera_make(const float *pos, const float *at, const float *up,
                                                           float hfov, float aspect, float defocus, float focus,
                                                           phx_camera_params *out) {
    phx::camera_make(pos, at, up, hfov, aspect, defocus, focus, out);
}

__attribute__((visibility("default"))) void orc_lum_pref_sum(const phx_light *lights, uint32_t n, float *out) {
    phx::lum_pref_sum(lights, n, out);
}

__attribute__((visibility("default"))) int orc_bvh_build(const phx_triangle *tris, uint32_t n, phx_bvh_node *out,
                                                        uint32_t *depth) {
    std::vector<phx_bvh_node> nodes;
    if (!tris || n == 0 || !build_bvh(tris, n, nodes))
        return PHX_E_INVALID;
    std::memcpy(out, nodes.data(), nodes.size() * sizeof(phx_bvh_node));
    if (depth)
        *depth = tree_depth(nodes, 0, 0);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_hash_info(const phx_bvh_node *root, uint32_t g,
                                                        phx_photon_hash_data *out) {
    *out = hash_info(*root, g);
    return PHX_OK;
}

__attribute__((visibility("default"))) void *orc_create(const phx_scene *s) {
    auto *o = new OrcCtx();
    if (!build_bvh(s->triangles, s->n_triangles, o->bvh)) {
        delete o;
        return nullptr;
    }
    o->depth = tree_depth(o->bvh, 0, 0);
    Scene &sc = o->sc;
    sc.tris = s->triangles;
    sc.n_tris = s->n_triangles;
    sc.etris = s->emissive_triangles;
    sc.n_etris = s->n_emissive_triangles;
    sc.materials = s->materials;
    o->n_materials = s->n_materials;
    sc.uv = s->uv_transforms;
    sc.lights = s->lights;
    sc.n_lights = s->n_lights;
    sc.lum_pref_sum = s->lum_pref_sum;
    sc.total_lum = s->n_lights ? s->lum_pref_sum[s->n_lights - 1] : 0.0f; // shading.cpp:26
    sc.tex_meta = s->tex_meta;
    sc.tex_atlas = s->tex_atlas;
    sc.envmap = s->envmap;
    sc.env_w = s->envmap_width;
    sc.env_h = s->envmap_height;
    sc.has_envmap = s->envmap != nullptr && s->envmap_width > 0 && s->envmap_height > 0;
    sc.camera = s->camera;
    sc.bvh = o->bvh.data();
    scene_sphere(o->bvh[0], &sc.scene_center, &sc.scene_radius);
    return o;
}

__attribute__((visibility("default"))) void orc_destroy(void *o) { delete (OrcCtx *)o; }

__attribute__((visibility("default"))) uint32_t orc_bvh_depth(void *o) { return ((OrcCtx *)o)->depth; }

__attribute__((visibility("default"))) int orc_get_bvh(void *o, phx_bvh_node *out, uint32_t cap) {
    auto *c = (OrcCtx *)o;
    if (cap < c->bvh.size())
        return PHX_E_INVALID;
    std::memcpy(out, c->bvh.data(), c->bvh.size() * sizeof(phx_bvh_node));
    return PHX_OK;
}

/* hp output: n_ids x 6 x 4 values (float or double per prec) */
__attribute__((visibility("default"))) int orc_trace(void *o, uint32_t w, uint32_t h, uint32_t seed, uint32_t ds,
                                                    const uint32_t *ids, uint32_t n_ids, int prec, void *out,
                                                    int threads) {
    if (prec)
        trace_impl<double>((OrcCtx *)o, w, h, seed, ds, ids, n_ids, out, threads);
    else
        trace_impl<float>((OrcCtx *)o, w, h, seed, ds, ids, n_ids, out, threads);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_emit(void *o, uint32_t tb, uint32_t te, uint32_t maxb, uint32_t seed,
                                                   int prec, uint32_t *counts, void *pos, uint32_t *power,
                                                   uint32_t *dir, uint64_t cap, uint64_t *n_out, int threads) {
    if (prec)
        return emit_impl<double>((OrcCtx *)o, tb, te, maxb, seed, counts, pos, power, dir, cap, n_out, threads);
    return emit_impl<float>((OrcCtx *)o, tb, te, maxb, seed, counts, pos, power, dir, cap, n_out, threads);
}

__attribute__((visibility("default"))) int orc_hash(const float *pos4, uint32_t n, const phx_photon_hash_data *d,
                                                   uint32_t buckets, uint32_t *keys, uint32_t *counts) {
    hash_impl<float>(pos4, n, *d, buckets, keys, counts);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_scan(const uint32_t *counts, uint32_t n, uint32_t *start) {
    if (n > SCAN_CHUNK_SIZE * SCAN_CHUNK_SIZE)
        return PHX_E_INVALID; // constants.h:8-9
    reference_scan(counts, n, start);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_scatter(const float *pos4, const uint32_t *power, const uint32_t *dir,
                                                      const uint32_t *keys, uint32_t n, const uint32_t *start,
                                                      uint32_t buckets, float *spos4, uint32_t *spower,
                                                      uint32_t *sdir, uint32_t *end, uint32_t *perm) {
    scatter_impl<float>(pos4, power, dir, keys, n, start, buckets, spos4, spower, sdir, end, perm);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_gather(const float *hp6, uint32_t n_pixels, const float *spos4,
                                                     const uint32_t *spower, const uint32_t *sdir,
                                                     const uint32_t *start, const uint32_t *end,
                                                     const phx_photon_hash_data *d, float alpha, float *flux4,
                                                     float *weight, float *radiance4, int threads) {
    gather_impl<float>(hp6, n_pixels, spos4, spower, sdir, start, end, *d, alpha, flux4, weight, radiance4, threads);
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_render(void *o, const phx_params *p, uint32_t rounds, int prec,
                                                     int threads, void *flux4, void *weight, void *radiance4,
                                                     uint64_t *total_emitted, uint32_t *n_last,
                                                     double *stage_seconds) {
    if (prec)
        return render_impl<double>((OrcCtx *)o, p, rounds, threads, flux4, weight, radiance4, total_emitted, n_last,
                                   stage_seconds);
    return render_impl<float>((OrcCtx *)o, p, rounds, threads, flux4, weight, radiance4, total_emitted, n_last,
                              stage_seconds);
}

/* F(θ') of phx_frozen.hpp: mats1 / lights1 are θ' (the scene's counts), img1 npx x 3 doubles */
__attribute__((visibility("default"))) int orc_frozen_render(void *o, const phx_params *p, uint32_t rounds,
                                                            const phx_material *mats1, uint32_t n_mats,
                                                            const phx_light *lights1, uint32_t n_lights,
                                                            int threads, double *img1, float *flux4,
                                                            float *radiance4) {
    auto *c = (OrcCtx *)o;
    if (!c || !p || !img1 || rounds == 0 || n_mats != c->n_materials || n_lights != c->sc.n_lights ||
        (n_mats && !mats1) || (n_lights && !lights1))
        return PHX_E_INVALID;
    frozen::PrimedTables t(mats1, n_mats, lights1, n_lights);
    frozen::Primed<double> pr{mats1, lights1, t.base.data(), t.rough.data(), t.power.data()};
    return frozen_render_impl<double>(c, p, rounds, pr, threads, img1, flux4, radiance4);
}

/* The analytic gradient of L(θ) = Σ g · F(θ) at θ = (mats1, lights1), in double, by forward-mode
 * dual numbers (phx_dual.hpp): θ is laid out as 4 per material (base colour r, g, b, roughness),
 * then 3 per light (power r, g, b); g_img holds npx x 3 doubles; grad receives the θ-sized
 * gradient and *loss (optional) L.  The parameters are seeded DUAL_CHUNK at a time, one frozen
 * evaluation per chunk. */
constexpr int DUAL_CHUNK = 8;
__attribute__((visibility("default"))) int orc_frozen_grad(void *o, const phx_params *p, uint32_t rounds,
                                                          const phx_material *mats1, uint32_t n_mats,
                                                          const phx_light *lights1, uint32_t n_lights,
                                                          const double *g_img, int threads, double *grad,
                                                          double *loss) {
    auto *c = (OrcCtx *)o;
    if (!c || !p || !g_img || !grad || rounds == 0 || n_mats != c->n_materials || n_lights != c->sc.n_lights ||
        (n_mats && !mats1) || (n_lights && !lights1))
        return PHX_E_INVALID;
    using DD = Dual<DUAL_CHUNK>;
    const u32 np = 4 * n_mats + 3 * n_lights, npx = p->width * p->height;
    std::vector<DD> img((size_t)npx * 3);
    for (u32 c0 = 0; c0 < np; c0 += DUAL_CHUNK) {
        std::vector<V4<DD>> base(n_mats), power(n_lights);
        std::vector<DD> rough(n_mats);
        auto seeded = [&](double v, u32 param) {
            DD d(v);
            if (param >= c0 && param < c0 + DUAL_CHUNK)
                d.d[param - c0] = 1.0;
            return d;
        };
        for (u32 m = 0; m < n_mats; m++) {
            const phx_f4 &b = mats1[m].base_color;
            base[m] = mk<DD>(seeded(b.x, 4 * m), seeded(b.y, 4 * m + 1), seeded(b.z, 4 * m + 2), DD((double)b.w));
            rough[m] = seeded(mats1[m].roughness, 4 * m + 3);
        }
        for (u32 l = 0; l < n_lights; l++) {
            const phx_f4 &w = lights1[l].power;
            const u32 k = 4 * n_mats + 3 * l;
            power[l] = mk<DD>(seeded(w.x, k), seeded(w.y, k + 1), seeded(w.z, k + 2), DD((double)w.w));
        }
        frozen::Primed<DD> pr{mats1, lights1, base.data(), rough.data(), power.data()};
        int r = frozen_render_impl<DD>(c, p, rounds, pr, threads, img.data(), nullptr, nullptr);
        if (r)
            return r;
        double l = 0.0;
        double acc[DUAL_CHUNK] = {};
        for (size_t i = 0; i < img.size(); i++) {
            l += g_img[i] * img[i].v;
            for (int j = 0; j < DUAL_CHUNK; j++)
                acc[j] += g_img[i] * img[i].d[j];
        }
        for (u32 j = 0; j < DUAL_CHUNK && c0 + j < np; j++)
            grad[c0 + j] = acc[j];
        if (loss)
            *loss = l;
    }
    return PHX_OK;
}

__attribute__((visibility("default"))) int orc_image(const void *flux4, const void *radiance4, uint32_t n, int prec,
                                                    float exposure, int tonemap, uint64_t total_photons,
                                                    uint32_t rounds, double *rgb) {
    if (prec)
        image_impl<double>(flux4, radiance4, n, exposure, tonemap, total_photons, rounds, rgb);
    else
        image_impl<float>(flux4, radiance4, n, exposure, tonemap, total_photons, rounds, rgb);
    return PHX_OK;
}

/* known-answer helpers */
__attribute__((visibility("default"))) void orc_pcg(uint32_t seed, uint32_t n, uint32_t *out, float *outf) {
    Rng r = pcg_seed(seed);
    for (uint32_t i = 0; i < n; i++) {
        Rng c = r;
        out[i] = random_u32(&r);
        if (outf)
            outf[i] = random_float<float>(&c);
    }
}
__attribute__((visibility("default"))) void orc_encode_rgbe(const float *p4, uint32_t n, uint32_t *out) {
    for (uint32_t i = 0; i < n; i++)
        out[i] = encode_rgbe<float>(mk<float>(p4[4 * i], p4[4 * i + 1], p4[4 * i + 2], p4[4 * i + 3]));
}
__attribute__((visibility("default"))) void orc_decode_rgbe(const uint32_t *in, uint32_t n, float *out4) {
    for (uint32_t i = 0; i < n; i++)
        store4<float>(out4, i, decode_rgbe<float>(in[i]));
}
__attribute__((visibility("default"))) void orc_encode_oct(const float *d4, uint32_t n, uint32_t *out) {
    for (uint32_t i = 0; i < n; i++)
        out[i] = encode_oct<float>(mk<float>(d4[4 * i], d4[4 * i + 1], d4[4 * i + 2], d4[4 * i + 3]));
}
__attribute__((visibility("default"))) void orc_decode_oct(const uint32_t *in, uint32_t n, float *out4) {
    for (uint32_t i = 0; i < n; i++)
        store4<float>(out4, i, decode_oct<float>(in[i]));
}
__attribute__((visibility("default"))) void orc_get_hash(const float *p4, uint32_t n, const phx_photon_hash_data *d,
                                                        uint32_t *out) {
    for (uint32_t i = 0; i < n; i++)
        out[i] = get_hash<float>(mk<float>(p4[4 * i], p4[4 * i + 1], p4[4 * i + 2], p4[4 * i + 3]), *d);
}
__attribute__((visibility("default"))) float orc_math(int fn, float x, float y) {
    switch (fn) {
    case 0: return pm_sinf(x);
    case 1: return pm_cosf(x);
    case 2: return pm_expf(x);
    case 3: return pm_logf(x);
    case 4: return pm_powf(x, y);
    case 5: return pm_acosf(x);
    case 6: return pm_atan2f(x, y);
    default: return 0.0f;
    }
}

} // extern "C"
