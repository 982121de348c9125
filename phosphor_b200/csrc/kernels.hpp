// kernels.hpp — host-side launchers of the SPPM device kernels (one translation unit each).
#pragma once

#include <cstdint>
#include <string>
#include <cuda_runtime.h>

#include "dev_scene.cuh"

namespace phx {

// Global index spaces of an engine: pixels, photon paths, photon slots and grid cells of all
// scenes concatenated in scene order.  bases arrays hold n_scenes+1 prefix offsets.
struct LaunchCtx {
    const SceneDesc *scenes; // device array
    u32 n_scenes;
    const u32 *pix_bases;    // device
    const u32 *emit_bases;   // device
    u32 total_pixels;
    u32 total_emit;
    const u32 *seeds;        // device, one round seed per scene
    u32 *err;                // device error word
    u32 *overflow;           // device traversal-overflow counter
    const u32 *nee_bases;    // device, n_scenes+1 prefix offsets of deferred-NEE sample slots
    u32 total_nee;           // sum over scenes of pixels * direct_samples
    u32 nee_defer;           // 1: diffuse-hit NEE shadow rays go to the shadow wavefront
    u32 pix_lo, pix_hi;      // global pixels the camera pass traces (all, or one shard's range)
    u32 emit_lo, emit_hi;    // global photon paths the photon pass emits
};

// Deferred specular NEE: per pixel at most two emission terms per camera bounce (the surface's
// emission, the NEE mean) and one for an escaped ray.
constexpr u32 DEF_MAX = 11;
constexpr u32 DEF_KNOWN = 0xffffffffu; // def_tag of a term whose value is known
constexpr u32 DEF_DIFFUSE = 0x100u;    // def_cnt flag: the path ended at a diffuse hit point
constexpr u32 DEF_OVERFLOW = 0x40000000u; // def_cnt flag: a term did not fit (never expected)

struct TraceOut {
    float4 *pos, *normal, *throughput, *base_color, *direct, *emission;
    float4 *nee_ray; // per NEE sample slot: (dir.xyz, light distance), w < 0 = no contribution
    float4 *nee_val; // per slot: radiance * (base / pi); replaced by the contribution in the shadow pass
    float4 *stash_sn = nullptr; // per pixel with a diffuse hit point: shading normal for its NEE samples
    u32 *stash_rng = nullptr;   // per pixel: RNG state at its NEE samples
    // Deferred specular NEE (lane-refill camera kernel; null: traced in place).  Each specular
    // event claims direct_samples consecutive sample slots; from a pixel's first deferred event on,
    // its nonzero emission terms are listed in order and summed once the samples are traced.
    float4 *spec_ray = nullptr; // per sample: (dir.xyz, light distance), w < 0 = no contribution
    float4 *spec_val = nullptr; // per sample: the NEE weight; replaced by weight * transmittance
    float4 *spec_org = nullptr; // per sample: shadow ray origin (the specular hit point)
    u32 *spec_pix = nullptr;    // per sample: global pixel (its scene)
    u32 *spec_next = nullptr;   // claimed sample slots this round (zeroed before the camera pass)
    u32 spec_cap = 0;           // sample slots
    u32 *def_cnt = nullptr;     // per pixel: listed terms | DEF_DIFFUSE
    float4 *def_prefix = nullptr; // per pixel: the emission before its first listed term
    float4 *def_val = nullptr;  // per pixel x DEF_MAX: a known term, or the throughput of an NEE term
    u32 *def_tag = nullptr;     // per pixel x DEF_MAX: DEF_KNOWN, or the first sample slot of an NEE term
};

// Persistent work queue (lane refill): a device counter the kernel drains.
// untextured: no material of the context has a texture
void launch_trace(const LaunchCtx &lc, const TraceOut &out, int block, int persistent, int blocks_per_sm,
                  u32 *queue, bool untextured, cudaStream_t st);
// Deferred diffuse-hit NEE: trace every recorded shadow ray (one thread per sample slot), then sum
// each pixel's samples in sample order into hp_direct.
// kind: SHADOW_OPAQUE when no scene has a transmissive material, else SHADOW_CLEAR when no material
// has a texture, else SHADOW_GENERAL.  presample:
// some scene's light samples take varying RNG draws, so k_nee_sample draws its samples first.
// per_pixel: a single scene whose only light is not an area light (one shadow ray per hit point)
// one: the scene descriptor of a single-scene context (passed to the kernel by value), or null
void launch_shadow(const LaunchCtx &lc, const TraceOut &out, int kind, bool presample, bool per_pixel,
                   u32 n_pixels, const SceneDesc *one, cudaStream_t st);
void launch_nee_resolve(const LaunchCtx &lc, const TraceOut &out, cudaStream_t st);
// Deferred specular NEE: complete each listed pixel's emission once k_shadow has traced the
// claimed sample slots.
void launch_spec_resolve(const LaunchCtx &lc, const TraceOut &out, cudaStream_t st);

struct EmitOut {
    float4 *slot_pos;
    uint2 *slot_pd;    // (rgbe power, octahedral direction)
    u32 *counts;       // per photon path (global emit index)
    float4 *slot_pow;  // optional (one-thread-per-path form only): unquantised power per slot
};
// untextured: no material of the context has a texture.  prestart: every scene has at least three
// photon slots per path (max_bounces >= 3), so the lane-refill form can draw the paths' light
// samples in a pre-pass (k_emit_start) and keep them in those slots.
void launch_emit(const LaunchCtx &lc, const EmitOut &out, int block, int persistent, int blocks_per_sm, u32 *queue,
                 bool untextured, bool prestart, cudaStream_t st);

// grid build
struct GridBufs {
    const u32 *counts;   // per photon path
    const u32 *offsets;  // exclusive scan of counts, total_emit+1 entries
    const float4 *slot_pos;
    const uint2 *slot_pd;
    float4 *ph_pos;      // canonical photons
    uint2 *ph_pd;
    u32 *keys;           // composite cell key per canonical photon
    u32 *cell_count;     // total_cells+1
};
void launch_compact(const LaunchCtx &lc, const GridBufs &g, cudaStream_t st);
void launch_hash(const LaunchCtx &lc, const GridBufs &g, const u32 *n_dev, u64 n_max, cudaStream_t st);

// exclusive scan of n u32 (decoupled look-back).  total (optional) receives the sum.
// scratch: ScanScratch sized by scan_scratch_words(n).
size_t scan_scratch_bytes(u64 n);
// n_dyn (optional): scan only min(n, dyn_mul * ceil(*n_dyn / dyn_div)) items, read on the device
void launch_scan(const u32 *in, u32 *out, u64 n, void *scratch, u32 *total, u32 *err, cudaStream_t st,
                 const u32 *n_dyn = nullptr, u32 dyn_div = 1, u32 dyn_mul = 1);
// failure-detection self-test: scan with tile 0 withheld; returns 0 ok, 2 alloc, 3 CUDA error
int selftest_lookback_timeout(int device, u32 n, u32 *err_out);
// exclusive scan with its scratch in a static device array (no allocation); synchronous.
// returns 0 ok, 1 too large, 3 CUDA error, 4 look-back timeout (message in err)
int scan_noalloc(const u32 *in, u32 *out, u32 n, u32 *total, cudaStream_t st, std::string &err);
// k_denoise.cu: mode 0 mean, 1 median, 2 weighted; 0 = ok, 1 = invalid argument, 3 = CUDA error
int denoise_filter(int mode, const int32_t *in, float *out, const float *weights, uint32_t width, uint32_t height,
                   uint32_t k, float *kernel_ms, std::string &msg);

// k_bvh.cu: the binned-SAH traversal tree built on the device, identical to the host builder's
// (bvh_build_sah, then bvh_widen when `widen`).  Topology first; bvh_device_finish then orders each
// leaf by reference rank and writes the per-triangle records (trirec 3, nrm 3, tan 3, uv 2 float4
// per triangle, leaf order).  Returns 0 ok, 1 invalid input, 2 out of memory, 3 CUDA error.
struct DeviceBvh {
    float *cnodes = nullptr; // 16 floats per inner node, pre-order (max(n_inner, 1) records)
    float *wnodes = nullptr; // 28 floats per 4-wide node, pre-order (when widened)
    u32 *leaf_tri = nullptr; // triangle index per leaf position
    uint2 *leaves = nullptr; // (first, count) per leaf
    u32 n_inner = 0, depth = 0, n_leaves = 0, levels = 0;
    int root = 0;            // 0 or a leaf reference
    u32 n_wide = 0, wdepth = 0;
    int wroot = 0;
    void release();
};
int bvh_device_build(const phx_triangle *tris, u32 n, u32 max_leaf, bool widen, cudaStream_t st, DeviceBvh &out,
                     std::string &err);
// 4-wide nodes -> 8-bit child boxes (bvh_quant.hpp), one thread per node
cudaError_t bvh_device_quantize(const float *wnodes, u32 n, u32 *out, cudaStream_t st);
int bvh_device_finish(const phx_triangle *tris, const u32 *rank, u32 n, DeviceBvh &b, float4 *trirec, float4 *nrm,
                      float4 *tan, float4 *uv, cudaStream_t st);

// stable LSD radix sort of (key, canonical index) by key; n read from device *n_dev (<= n_max)
size_t radix_scratch_bytes(u64 n_max, u32 key_bits);
u32 radix_passes(u32 key_bits);
void launch_radix_sort(const u32 *keys_in, u32 *keys_tmp0, u32 *keys_tmp1, u32 *vals0, u32 *vals1, u32 **perm_out,
                       const u32 *n_dev, u64 n_max, u32 key_bits, void *scratch, u32 *err, cudaStream_t st);

void launch_sorted_records(const u32 *perm, const float4 *ph_pos, const uint2 *ph_pd, const u32 *n_dev, u64 n_max,
                           float4 *s_posdir, u32 *s_power, float4 *s_dir, float4 *s_pow, u32 *err, cudaStream_t st);
void launch_decode_records(const float4 *s_posdir, const u32 *s_power, u64 n, float4 *s_dir, float4 *s_pow,
                           cudaStream_t st);

struct GatherBufs {
    const float4 *hp_pos, *hp_normal, *hp_throughput, *hp_base_color, *hp_direct, *hp_emission;
    const float4 *s_posdir;
    const u32 *s_power;
    const float4 *s_dir, *s_pow; // per record: decode_oct(direction bits), decode_rgbe(power)
    const u32 *cell_start; // total_cells+1
    u32 n_cap;             // photon buffer capacity: cell ranges are clamped to it
    float4 *flux;
    float *weight;
    float4 *radiance;
    float *rec_r2;         // optional: per pixel, the search radius² used this round
    float *rec_ratio;      // optional: per pixel, the SPPM ratio applied to the flux (1 if none)
    const u32 *order;      // optional: thread t gathers pixel order[t] (pixels grouped by grid cell)
};
// coop: the warp-cooperative kernel (k_gather_coop), else one thread per pixel (k_gather)
void launch_gather(const LaunchCtx &lc, const GatherBufs &g, int block, bool coop, cudaStream_t st);
// Per pixel a sort key that groups hit points by photon-grid cell: ((cell_base + cell) << 3 | octant
// of the point inside its cell), 0 for pixels without a diffuse hit point.
void launch_pixel_keys(const LaunchCtx &lc, const float4 *hp_pos, const float4 *hp_emission, u32 key_bits, u32 *keys,
                       cudaStream_t st);

// adjoint (single scene): gather adjoint, camera / photon path replays, helpers
struct AdjBufs {
    const float4 *g_img;   // dL/dI per pixel (linear radiance; .w unused)
    const float *kscale;   // K_n per pixel for the round being replayed
    const float *r2;       // search radius² per pixel in that round
    float4 *gT, *gA;       // dL/d throughput and dL/d base colour of each hit point
    float4 *gphi;          // dL/d power per canonical photon
    const float4 *ph_pow;  // unquantised power per canonical photon
    const u32 *perm;       // cell-order index -> canonical index
    const u32 *offsets;    // first canonical photon of each path (total_emit + 1 entries)
    double *grad;          // 4 per material (base r, g, b, roughness), then 3 per light (power r, g, b)
    u32 n_params, n_mat;
    float inv_rounds;
    u32 block_sums;        // 1: per-block partial sums in 4*n_params bytes of shared memory
};
void launch_gather_adj(const LaunchCtx &lc, const GatherBufs &g, const AdjBufs &ab, cudaStream_t st);
void launch_trace_adj(const LaunchCtx &lc, const AdjBufs &ab, cudaStream_t st);
void launch_emit_adj(const LaunchCtx &lc, const AdjBufs &ab, cudaStream_t st);
void launch_compact_pow(const LaunchCtx &lc, const float4 *slot_pow, const u32 *counts, const u32 *offsets,
                        float4 *ph_pow, cudaStream_t st);
void launch_adj_scale(const float *ratio, float *kscale, const float4 *flux, u32 n_pix, u32 rounds, float inv_n,
                      cudaStream_t st);
void launch_adj_image(const float4 *flux, const float4 *radiance, u32 n_pix, float inv_rounds, float inv_n, float *img,
                      cudaStream_t st);

// image formation (output.cpp:52-83) for one scene's pixel range
void launch_image(const float4 *flux, const float4 *radiance, u32 n, float exposure, int tonemap, float inv_photons,
                  float inv_rounds, float *rgb, uint8_t *ldr, cudaStream_t st);

// per-scene round seeds: seeds[s] = random_u32(&state[s])
void launch_next_seeds(u32 *state, u32 *seeds, u32 n, cudaStream_t st);

// SM count of the current device (set by init_kernels, called once per engine outside capture)
extern int g_sm_count;
void init_kernels(int device);

} // namespace phx
