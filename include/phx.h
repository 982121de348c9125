/*
 * phx.h — C ABI of the B200-native SPPM renderer core (libphx.so).
 *
 * The reference (alfazet/phosphor) has no plugin or FFI: its hot path sits behind the private
 * methods Renderer::trace_rays / emit_photons / hash_and_sort_photons / gather_flux
 * (include/host/renderer.hpp:63-69), fed by RenderingBuffers::set_*_args
 * (src/buffers/rendering.cpp:32-77) and the scene upload in Renderer::set_scene
 * (src/renderer/renderer.cpp:22-57).  Each entry point below names the reference interface it
 * replaces.  Only plain C types cross this boundary: POD structs byte-compatible with the
 * reference's shared host/device structs (include/common/ headers, 16-byte aligned like GPU_ALIGN at
 * include/common/constants.h:4), host pointers and sizes.  No device pointer, C++ exception or
 * trap ever crosses it; every call returns an int status and phx_last_error() explains failures.
 *
 * Threading: one context owns one CUDA stream and all of its device memory.  A context is not
 * safe to use from two threads at once; distinct contexts are independent.
 */
#ifndef PHX_H
#define PHX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__) || defined(__CUDACC__)
#define PHX_ALIGN16 __attribute__((aligned(16)))
#define PHX_API __attribute__((visibility("default")))
#else
#define PHX_ALIGN16
#define PHX_API
#endif

/* ---- status codes ------------------------------------------------------------------------ */
enum {
    PHX_OK = 0,
    PHX_E_INVALID = 1,     /* bad argument, size or handle */
    PHX_E_OOM = 2,         /* device or host allocation failed */
    PHX_E_CUDA = 3,        /* a CUDA runtime call failed (message in phx_last_error) */
    PHX_E_TIMEOUT = 4,     /* a bounded device-side wait gave up (decoupled look-back) */
    PHX_E_NO_PHOTONS = 5,  /* no photon was stored this round (renderer.cpp:117-118 traps here) */
    PHX_E_STATE = 6,       /* call out of order (e.g. gather before trace) */
    PHX_E_OVERFLOW = 7,    /* a fixed-capacity device structure overflowed (traversal stack) */
    PHX_E_UNSUPPORTED = 8  /* feature not available in this build / on this device */
};

/* ---- POD layouts shared with the reference (byte-compatible) ----------------------------- */
typedef struct PHX_ALIGN16 phx_f4 { float x, y, z, w; } phx_f4;
typedef struct phx_f2 { float x, y; } __attribute__((aligned(8))) phx_f2;

/* include/common/triangle.h:30-44 — 176 bytes */
typedef struct PHX_ALIGN16 phx_triangle {
    phx_f4 v0, v1, v2;
    phx_f4 n0, n1, n2;
    phx_f4 t0, t1, t2;
    phx_f2 uv0, uv1, uv2;
    uint32_t mat_index;
    uint8_t _padding[4];
} phx_triangle;

/* include/common/material.h:7-27 */
typedef struct PHX_ALIGN16 phx_uv_transform {
    phx_f2 uv_offset;
    phx_f2 uv_scale;
    float uv_rotation;
    uint8_t _padding[12];
} phx_uv_transform;

typedef struct PHX_ALIGN16 phx_uv_transform_block {
    phx_uv_transform diff, emis, norm, occlusion, metal_rough, transmission;
} phx_uv_transform_block;

#define PHX_NO_TEXTURE 0xFFFFFFFFu

/* include/common/material.h:36-59 — 96 bytes */
typedef struct PHX_ALIGN16 phx_material {
    phx_f4 base_color;
    phx_f4 emissive;
    phx_f4 att_color;
    float metallic, roughness, transmission, ior, att_dist, thickness;
    uint32_t diff_index, emis_index, norm_index, occlusion_index, metal_rough_index, transmission_index;
} phx_material;

/* include/common/light.h:9-31 — 128 bytes */
#define PHX_LIGHT_POINT 0
#define PHX_LIGHT_SPOT 1
#define PHX_LIGHT_DIRECTIONAL 2
#define PHX_LIGHT_TEXTURED 3
typedef struct PHX_ALIGN16 phx_light {
    phx_f4 position, power, direction, tangent, bitangent, origin;
    phx_f4 aux; /* spot: x inner, y outer angle; textured: x tex (u32 bits), y tri_start, z tri_count, w area */
    uint8_t kind;
    uint8_t _padding[15];
} phx_light;

/* include/common/texture_meta.h:7-15 */
typedef struct PHX_ALIGN16 phx_texture_meta {
    uint32_t atlas_offset, width, height, channels;
} phx_texture_meta;

/* include/common/camera.h:7-22 — 112 bytes */
typedef struct PHX_ALIGN16 phx_camera_params {
    phx_f4 position, lower_left_corner, horizontal, vertical, defocus_disk_u, defocus_disk_v;
    float defocus_angle;
    float focus_distance;
    uint8_t _padding[8];
} phx_camera_params;

/* include/common/bvh_node.h:6-8 — min.w = triangle index bits (-1 = inner), max.w = skip index */
typedef struct PHX_ALIGN16 phx_bvh_node {
    phx_f4 min;
    phx_f4 max;
} phx_bvh_node;

/* include/common/photon_hash.h:11-19 — 48 bytes */
typedef struct PHX_ALIGN16 phx_photon_hash_data {
    phx_f4 origin;
    phx_f4 cell_sizes;
    uint32_t grid_res;
    uint8_t _padding[12];
} phx_photon_hash_data;

/* Scene handed to phx_create: the SceneData arrays (include/host/scene_data.hpp:21-42) with the
 * camera already resolved to CameraParams (Camera::to_params, src/renderer/camera.cpp:44-56).
 * All arrays are copied at create time; the caller keeps ownership. */
typedef struct phx_scene {
    const phx_triangle *triangles;
    uint32_t n_triangles;
    const phx_triangle *emissive_triangles;
    uint32_t n_emissive_triangles;
    const phx_material *materials;
    const phx_uv_transform_block *uv_transforms; /* one block per material */
    uint32_t n_materials;
    const phx_light *lights;
    uint32_t n_lights;
    const float *lum_pref_sum; /* n_lights entries (scene_data.cpp:14-23) */
    const phx_texture_meta *tex_meta;
    uint32_t n_textures;
    const uint8_t *tex_atlas;
    uint64_t tex_atlas_bytes;
    const float *envmap; /* RGB f32, width*height*3, NULL for none */
    uint32_t envmap_width, envmap_height; /* `camera` lands on offset 128: no implicit padding */
    phx_camera_params camera;
} phx_scene;

/* The per-render knobs of ArgsList (include/host/cmd_args.hpp:36-65) that the pipeline uses. */
typedef struct phx_params {
    uint32_t width, height;        /* -w -h */
    uint32_t photons_per_round;    /* -p */
    uint32_t max_photon_bounces;   /* --max-bounces (1..32) */
    uint32_t grid_res;             /* --grid-res (1..255) */
    float sppm_alpha;              /* --sppm-alpha */
    uint32_t direct_samples;       /* --direct-samples (1..128) */
    uint32_t seed;                 /* --seed */
    uint32_t flags;                /* PHX_F_* */
    uint32_t bvh_leaf_size;        /* max triangles per leaf of the traversal tree (0 = 4) */
    uint32_t reserved[6];
} phx_params;

/* flags */
#define PHX_F_DEFAULT 0u
#define PHX_F_SIMPLE_TRAVERSAL 1u /* one-thread-per-ray kernels instead of the persistent ones */
#define PHX_F_REFERENCE_BVH 2u    /* traverse the reference's median-split tree instead of the SAH tree */
#define PHX_F_BINARY_BVH 4u       /* traverse the SAH tree as child pairs instead of 4-wide nodes */
#define PHX_F_QUANT_BVH 16u       /* 4-wide nodes with 8-bit child boxes (64 instead of 112 bytes) */
#define PHX_F_DEVICE_BVH 8u       /* build the SAH traversal tree on the GPU: the default (the same
                                     tree as the host build, bit for bit; the reference tree for the
                                     tie-break ranks is built on host threads meanwhile) */
#define PHX_F_HOST_BVH 32u        /* build the SAH traversal tree on the host instead */

/* Counters and sizes of a context. */
typedef struct phx_info {
    uint32_t n_pixels;
    uint32_t width, height;
    uint32_t photons_per_round;
    uint32_t photon_buf_size;     /* photons_per_round * max_photon_bounces (renderer.cpp:40) */
    uint32_t bucket_count;        /* grid_res^3 + 1 (renderer.cpp:38) */
    uint32_t n_photons;           /* photons stored by the last emit (device value, synced) */
    uint32_t n_bvh_nodes;
    uint32_t bvh_depth;
    uint32_t rounds_done;
    uint64_t total_photons_emitted;
    uint32_t stack_overflows;     /* traversal stack overflows seen (0 expected) */
    uint32_t error_flags;         /* device error bits (look-back timeouts etc.) */
    uint32_t _pad0[2];            /* keeps `hash` 16-byte aligned without implicit padding */
    phx_photon_hash_data hash;
    uint32_t kernels_per_round;   /* CUDA kernels one round launches (all scenes of an engine) */
    uint32_t sort_passes;         /* counting-sort digit passes per round */
    uint32_t trav_depth;          /* depth of the device traversal tree */
    uint32_t trav_inner_nodes;    /* inner (child-pair) nodes of the device traversal tree */
    uint32_t spec_samples;        /* specular-NEE shadow rays the last camera pass deferred (all scenes) */
    float setup_ms;               /* wall time of this scene's setup (trees, uploads) */
    float bvh_build_ms;           /* of which: building the reference and traversal trees */
    uint32_t reserved[1];
} phx_info;

/* Buffers readable / writable through phx_read_buffer / phx_write_buffer, always in the
 * reference's layout (element sizes in parentheses). */
enum {
    PHX_BUF_HP_POS = 0,        /* float4 per pixel */
    PHX_BUF_HP_NORMAL = 1,     /* float4 */
    PHX_BUF_HP_THROUGHPUT = 2, /* float4 */
    PHX_BUF_HP_BASE_COLOR = 3, /* float4 */
    PHX_BUF_HP_DIRECT = 4,     /* float4 */
    PHX_BUF_HP_EMISSION = 5,   /* float4 (.w = 1 when the pixel has a diffuse hit point) */
    PHX_BUF_FLUX = 6,          /* float4 (.w = search radius squared) */
    PHX_BUF_PHOTON_WEIGHT = 7, /* f32 */
    PHX_BUF_RADIANCE = 8,      /* float4 */
    PHX_BUF_PHOTON_POS = 9,    /* float4 per stored photon, canonical emission order */
    PHX_BUF_PHOTON_POWER = 10, /* u32 RGBE */
    PHX_BUF_PHOTON_DIR = 11,   /* u32 octahedral */
    PHX_BUF_PHOTON_HASH = 12,  /* u32 cell key per stored photon (canonical order) */
    PHX_BUF_CELL_COUNT = 13,   /* u32 per cell (bucket_count) */
    PHX_BUF_CELL_START = 14,   /* u32 per cell */
    PHX_BUF_CELL_END = 15,     /* u32 per cell */
    PHX_BUF_SORTED_POS = 16,   /* float4 per stored photon, cell order */
    PHX_BUF_SORTED_POWER = 17, /* u32 */
    PHX_BUF_SORTED_DIR = 18,   /* u32 */
    PHX_BUF_EMIT_COUNT = 19,   /* u32 photons stored by each emitted photon path */
    PHX_BUF_BVH_NODES = 20,    /* phx_bvh_node, reference layout */
    PHX_BUF_SORT_PERM = 21,    /* u32 canonical index of each cell-ordered photon */
    PHX_BUF_ROUND_RNG = 22,    /* u32: the state of the round-seed PCG stream (Renderer::rng, renderer.cpp:49,65);
                                  writing a saved state makes the following rounds reuse its seeds */
    PHX_BUF__COUNT = 23
};

/* ---- context lifecycle -------------------------------------------------------------------- */

/* Replaces Renderer::Renderer + Renderer::set_scene (renderer.cpp:9-57): builds the BVH on the
 * host with the reference's median split (bvh.cpp:18-84), uploads the scene, sizes every buffer
 * like set_scene does, seeds the round RNG with pcg_seed(params->seed) (renderer.cpp:54).
 * device = CUDA ordinal. */
PHX_API int phx_create(const phx_scene *scene, const phx_params *params, int device, void **out_ctx);
PHX_API int phx_destroy(void *ctx);
PHX_API int phx_get_info(void *ctx, phx_info *out);

/* ---- per-pass stages (the plain form: one launch sequence per pass, like the reference) ---- */

/* Renderer::trace_rays (renderer.cpp:90-95) -> kernels/trace_rays.cl:14-169. */
PHX_API int phx_trace_rays(void *ctx, uint32_t seed);
/* Renderer::emit_photons (renderer.cpp:97-121) -> kernels/emit_photons.cl:12-114; photons are
 * stored in canonical order (path index, then bounce).  Reads the stored count back to the host
 * like renderer.cpp:114 and returns PHX_E_NO_PHOTONS when it is zero. */
PHX_API int phx_emit_photons(void *ctx, uint32_t seed);
/* Renderer::hash_and_sort_photons (renderer.cpp:123-153): hash_photons.cl, the scan_*.cl trio and
 * scatter_photons.cl, as hash + decoupled-look-back scan + stable counting sort. */
PHX_API int phx_hash_sort(void *ctx);
/* Renderer::gather_flux (renderer.cpp:155-161) -> kernels/gather_flux.cl:5-78. */
PHX_API int phx_gather(void *ctx, float sppm_alpha);
/* One round of Renderer::run's loop body (renderer.cpp:64-78) in the plain form: draws the round
 * seed from the context RNG, then the four stages above with the reference's two host syncs. */
PHX_API int phx_round(void *ctx);
/* `rounds` rounds with every stage of a round replayed from one captured CUDA graph and no host
 * sync inside; numerically identical to calling phx_round `rounds` times. */
PHX_API int phx_iterate(void *ctx, uint32_t rounds);
/* One round replayed from a captured graph with the round seed given by the host, as in
 * renderer.cpp:65 (the seed is copied from pinned memory on the context stream).  Asynchronous:
 * returns after enqueueing; phx_sync or any read waits for it. */
PHX_API int phx_round_seeded(void *ctx, uint32_t seed);
PHX_API int phx_sync(void *ctx);

/* Device state access in the reference layouts (for parity checks and snapshots). */
PHX_API int phx_read_buffer(void *ctx, int which, void *dst, uint64_t offset_bytes, uint64_t bytes);
PHX_API int phx_write_buffer(void *ctx, int which, const void *src, uint64_t offset_bytes, uint64_t bytes);
/* Sets the stored-photon count (after writing PHOTON_POS/POWER/DIR for a stage-isolated run). */
PHX_API int phx_set_n_photons(void *ctx, uint32_t n_photons);

/* Image formation of src/renderer/output.cpp:52-83 on the device (flux / (pi r^2 N_emitted) plus
 * radiance / rounds, exposure, optional ACES, gamma 1/2.2, clamp).  Writes width*height*3 floats
 * in [0,1] to rgb_out (host) when rgb_out != NULL, and the u8 quantisation to ldr_out when != NULL. */
PHX_API int phx_image(void *ctx, float exposure, int tonemap, uint64_t total_photons, uint32_t rounds,
                      float *rgb_out, uint8_t *ldr_out);

/* Host-side helpers (no GPU needed). */
/* Bvh::Bvh (src/renderer/bvh.cpp:74-84): writes 2n-1 nodes; returns the tree depth in *depth. */
PHX_API int phx_bvh_build(const phx_triangle *tris, uint32_t n, phx_bvh_node *out_nodes, uint32_t *depth);
/* The traversal tree the kernels walk (no reference counterpart: the reference traverses the tree of
 * bvh.cpp): a binned-SAH tree over the reference's expanded triangle boxes with leaves of up to
 * max_leaf (1..16) triangles, as child pairs (wide = 0: 16 floats per inner node), collapsed to
 * 4-wide nodes (wide = 1: 28 floats) or 4-wide nodes with 8-bit child boxes (wide = 2: 16 words),
 * each triangle record (12 floats, leaf order) carrying its leaf rank in the
 * reference tree.  device < 0 builds on the host; device >= 0 builds on that GPU (PHX_F_DEVICE_BVH)
 * and returns the same arrays bit for bit.  nodes needs room for 16 (or 28) floats per triangle,
 * trirec 12 floats and leaf_tri one entry per triangle.  build_ms: wall time of the traversal tree
 * (for the GPU: its build with the triangles resident on the device and the records written there),
 * excluding the reference tree that supplies the ranks. */
typedef struct phx_bvh_packed {
    float *nodes;
    float *trirec;
    uint32_t *leaf_tri;
    uint32_t n_nodes;  /* out: inner (child-pair or 4-wide) nodes */
    int32_t root;      /* out: root reference (>= 0 inner node, < 0 leaf ~(first | (count-1) << 27)) */
    uint32_t depth;    /* out: depth of the child-pair tree */
    uint32_t wdepth;   /* out: depth of the 4-wide tree (0 for child pairs) */
    float build_ms;    /* out */
    uint32_t reserved[3];
} phx_bvh_packed;
PHX_API int phx_traversal_bvh_build(const phx_triangle *tris, uint32_t n, uint32_t max_leaf, int wide, int device,
                                    phx_bvh_packed *out);
/* build_photon_hash_info (include/common/photon_hash.h:41-50) from the BVH root box. */
PHX_API int phx_hash_info(const phx_bvh_node *root, uint32_t grid_res, phx_photon_hash_data *out);
/* Camera::Camera + Camera::focus + Camera::to_params (src/renderer/camera.cpp:3-56). */
PHX_API int phx_camera_make(const float position[3], const float look_at[3], const float up[3], float hfov_deg,
                            float aspect, float defocus_angle, float focus_distance, phx_camera_params *out);
/* SceneData::build_lum_pref_sum (src/renderer/scene_data.cpp:14-23). */
PHX_API int phx_lum_pref_sum(const phx_light *lights, uint32_t n, float *out);

/* ---- procedural scenes (the reference's .glb assets are not available) --------------------- */
enum {
    PHX_SCENE_CORNELL = 0,       /* empty Cornell box, 12 triangles */
    PHX_SCENE_CAUSTIC = 1,       /* Cornell box + sine-wave water + conductor sphere */
    PHX_SCENE_ATRIUM = 2,        /* procedural courtyard, columns, arches, boxes, sky */
};
typedef struct phx_scene_spec {
    int kind;
    uint32_t seed;
    uint32_t width, height;      /* used for the camera aspect */
    uint32_t detail;             /* generator-specific size knob, 0 = the configuration's size */
    uint32_t reserved[5];
} phx_scene_spec;
/* Generates a scene; *out points into library-owned host memory until phx_scene_free(handle). */
PHX_API int phx_scene_generate(const phx_scene_spec *spec, phx_scene *out, void **handle);
PHX_API int phx_scene_free(void *handle);

/* ---- glTF 2.0 scene ingest (src/parsers/scene.cpp:206-233 read_gltf_scene, material.cpp:157-184,
 * texture.cpp:19-92) -------------------------------------------------------------------------
 * Loads a .gltf (with .bin files or data URIs) or .glb file into library-owned host arrays and
 * fills *out like phx_scene_generate (free with phx_scene_free).  The reference reads the file
 * through assimp; this reads the glTF document directly with the same conversions: node
 * transforms, one material per mesh primitive, emissive primitives as area lights of power
 * π·emissive·area, KHR_lights_punctual power = colour·intensity/683, perspective cameras
 * (hfov = 2·atan(aspect·tan(yfov/2))), KHR materials transmission / ior / volume / emissive
 * strength, KHR_texture_transform, PNG textures as 8-bit RGB (other image formats are skipped:
 * the material then has no texture).  The camera `camera` (the reference takes the first) gets
 * the render's aspect width/height (when both are nonzero) and focus(defocus_angle,
 * focus_distance) (renderer.cpp:24-28).  PHX_E_INVALID (with the reason in phx_last_error) for
 * an unreadable file, a malformed document, a scene without triangles or without that camera. */
typedef struct phx_gltf_options {
    uint32_t width, height;   /* render size (0, 0: the camera's own aspect) */
    float defocus_angle;      /* --defocus-angle (degrees) */
    float focus_distance;     /* --focus-distance (0 = 1) */
    uint32_t camera;          /* camera index in traversal order (0 = the reference's choice) */
    uint32_t reserved[3];
} phx_gltf_options;
PHX_API int phx_scene_load_gltf(const char *path, const phx_gltf_options *options, phx_scene *out, void **handle);

/* ---- batched scenes: one launch per stage for many scenes ---------------------------------- */
/* Creates one engine over n scenes with per-scene params (uneven sizes allowed). */
PHX_API int phx_batch_create(const phx_scene *scenes, const phx_params *params, uint32_t n, int device,
                             void **out_batch);
PHX_API int phx_batch_destroy(void *batch);
/* mode 0: plain form, scenes one at a time with per-pass launches and host syncs;
 * mode 1: all scenes per launch, each round replayed from a captured CUDA graph. */
PHX_API int phx_batch_iterate(void *batch, uint32_t rounds, int mode);
/* Retires (active = 0) or resumes a scene of the batch: every stage skips a retired scene, its
 * state and round count stay as they are, and the captured graph stays valid.  No counterpart in
 * the reference (a scene that has converged stops costing work in the batched form). */
PHX_API int phx_batch_set_active(void *batch, uint32_t scene, int active);
PHX_API int phx_batch_read_buffer(void *batch, uint32_t scene, int which, void *dst, uint64_t offset_bytes,
                                  uint64_t bytes);
PHX_API int phx_batch_get_info(void *batch, uint32_t scene, phx_info *out);
PHX_API int phx_batch_image(void *batch, uint32_t scene, float exposure, int tonemap, float *rgb_out);

/* ---- launch tuning -------------------------------------------------------------------------- */
typedef struct phx_tuning {
    uint32_t trace_block;       /* threads per block, trace kernel */
    uint32_t emit_block;        /* threads per block, photon kernel */
    uint32_t gather_block;      /* threads per block, gather kernel */
    uint32_t trace_blocks_per_sm;  /* persistent grid: resident blocks per SM */
    uint32_t emit_blocks_per_sm;
    uint32_t persistent;        /* 1 = persistent lane-refill kernels, 0 = one thread per item */
    uint32_t nee_wavefront;     /* 1 = diffuse-hit NEE shadow rays traced by a separate wavefront */
    uint32_t concurrent_passes; /* 1 = in the captured graph the camera pass and the photon pass of a
                                   round run on two branches (they only share the round seed) */
    uint32_t gather_sorted;     /* 1 = the gather visits pixels grouped by photon-grid cell */
    uint32_t pipeline_rounds;   /* k > 1: graph replays capture k rounds at a time, each round's camera
                                   and photon passes on branches of their own (they depend only on
                                   the round seed) and the gathers in round order, so rounds overlap;
                                   k - 1 extra sets of per-round buffers (1..8, 1 = off) */
    uint32_t gather_coop;       /* 1 = a warp stages each cell's photon records in shared memory and its
                                   lanes that need the cell walk them; 0 = one thread per pixel */
    uint32_t reserved[1];
} phx_tuning;
PHX_API int phx_get_tuning(void *ctx, phx_tuning *out);
PHX_API int phx_set_tuning(void *ctx, const phx_tuning *in);
/* Autotuner (no counterpart in the reference): times graph-replayed rounds of this context or batch
 * under candidate tunings — lane refill on/off, NEE wavefront on/off, persistent grid sizes of the
 * camera and photon kernels, concurrent passes on/off, 1/2/4 rounds in flight — by coordinate
 * descent, keeps the fastest and writes it to *chosen (may be NULL).  Every candidate gives
 * bit-identical results; the SPPM state, seeds and round counters are restored afterwards.  Each
 * trial renders a warm-up group and rounds_per_trial rounds rounded up to whole groups
 * (rounds_per_trial 1..64); a rounds-in-flight candidate whose buffers do not fit is skipped. */
PHX_API int phx_autotune(void *ctx, uint32_t rounds_per_trial, phx_tuning *chosen);

/* ---- measurement ------------------------------------------------------------------------------ */
/* Records CUDA events around every stage of every later round (in graph replays too) and keeps
 * per-stage averages; enabling or disabling drops the captured graph. */
PHX_API int phx_profile(void *ctx, int enable);
/* Average milliseconds per round of each stage since phx_profile(ctx, 1), in the order
 * seeds, trace, shadow (NEE wavefront + resolve), emit, emit scan + compaction, hash, cell scan,
 * sort, records, gather (n >= 10). */
PHX_API int phx_stage_ms(void *ctx, float *out, uint32_t n);
/* The CUDA stream (cudaStream_t) every stage of the context or batch is enqueued on. */
PHX_API uint64_t phx_get_stream(void *ctx);

/* ---- one image over several GPUs (single-scene contexts) -------------------------------------------
 * No counterpart in the reference (single device).  Each process creates a context for the same
 * scene and params on its own GPU and calls phx_shard(ctx, rank, world): rank r traces the pixel
 * range [P*r/W, P*(r+1)/W) and emits the photon paths [E*r/W, E*(r+1)/W).  In each round the ranks
 * exchange their stored photons once; concatenated in rank order they are the global canonical
 * photons, so every rank hashes, sorts and gathers exactly what a single GPU would, and each pixel's
 * flux, weight and radiance are bit-identical to a single-GPU render (pixels outside a rank's range
 * stay zero there).  A sharded context renders only through these calls (phx_round, phx_iterate and
 * phx_round_seeded return PHX_E_STATE).
 *   NCCL transport: rank 0 calls phx_nccl_unique_id, the id reaches every rank by any host channel,
 *   every rank calls phx_shard_nccl (collective), then phx_shard_round per round.  NCCL is loaded at
 *   run time (the process's own libnccl.so.2 if one is loaded); PHX_E_UNSUPPORTED without it.
 *   Host transport: phx_shard_begin (seed, camera pass, photon pass; *n_local = photons stored by this
 *   rank), phx_shard_get_photons (this rank's photons: float4 positions, uint32 pairs of RGBE power and
 *   octahedral direction), the caller concatenates all ranks' photons in rank order and hands them to
 *   every rank with phx_shard_put_photons, then phx_shard_end (hash, sort, gather). */
PHX_API int phx_shard(void *ctx, uint32_t rank, uint32_t world);
PHX_API int phx_shard_begin(void *ctx, uint32_t *n_local);
PHX_API int phx_shard_get_photons(void *ctx, float *pos4, uint32_t *pd2, uint32_t n);
PHX_API int phx_shard_put_photons(void *ctx, const float *pos4, const uint32_t *pd2, uint32_t n_all);
PHX_API int phx_shard_end(void *ctx);
PHX_API int phx_nccl_unique_id(uint8_t *out, uint32_t n);
PHX_API int phx_shard_nccl(void *ctx, const uint8_t *id);
PHX_API int phx_shard_round(void *ctx);

/* ---- differentiation (single-scene contexts) -------------------------------------------------------
 * No counterpart in the reference.  Parameters θ: per material its base colour (r, g, b) and
 * roughness, per light its power (r, g, b); gradients are laid out as 4 floats per material
 * (base r, g, b, roughness) followed by 3 per light (power r, g, b).
 * What is differentiated is the frozen-path estimator of the image: every random or discrete choice
 * of the forward render (paths, BSDF events, microfacet normals, Russian roulette, light selection,
 * gather neighbourhoods, kernel weights, radii, SPPM ratios) is held fixed and only the weights move
 * with θ — a BSDF bounce weighs W(θ0)·f(θ)/f(θ0) along its frozen directions, light power enters
 * linearly and photon power is taken unquantised.  The gradient is exact for that function (up to
 * float rounding); the oracle evaluates the same function in double for finite-difference checks.
 * Paths are replayed from their RNG seeds in the backward pass; nothing per vertex is stored.
 * A gradient with respect to a base-colour channel or light-power channel whose current value is 0,
 * or a roughness at its clamp (0.001 or 1), is reported as 0. */
/* Replaces the material table (same count; texture indices unchanged). */
PHX_API int phx_set_materials(void *ctx, const phx_material *materials, uint32_t n);
/* Replaces the lights (same count and kinds); the light-selection CDF is rebuilt
 * (scene_data.cpp:14-23). */
PHX_API int phx_set_lights(void *ctx, const phx_light *lights, uint32_t n);
/* Number of parameters: 4 * materials + 3 * lights. */
PHX_API int phx_adjoint_n_params(void *ctx, uint32_t *n);
/* Clears the SPPM state, renders `rounds` rounds (1..4096) recording what the backward pass needs,
 * and writes the linear image radiance/R + flux/(π r² N) (width*height*3 floats, before exposure and
 * gamma) to `image` (may be NULL). */
PHX_API int phx_adjoint_forward(void *ctx, uint32_t rounds, float *image);
/* Gradient of L with respect to θ given dL/dI (width*height*3 floats, same layout as the image) for
 * the last phx_adjoint_forward; n_grad >= phx_adjoint_n_params.  PHX_E_STATE if a round, gather,
 * buffer write or parameter change came in between.  May be called again with another dL/dI. */
PHX_API int phx_adjoint_backward(void *ctx, const float *dl_dimage, float *grad, uint32_t n_grad);

/* ---- failure detection self-test ----------------------------------------------------------------
 * Runs the decoupled look-back scan over n elements with tile 0 withheld (the tile ticket counter
 * starts at 1), so every other tile waits on a predecessor that never publishes.  The bounded
 * wait must give up, set the device error flag and let the kernel finish; the call returns
 * PHX_E_TIMEOUT with the flag in *err_flags.  No reference counterpart (the reference has no
 * device-side waits). */
PHX_API int phx_selftest_lookback_timeout(int device, uint32_t n, uint32_t *err_flags);

/* ---- allocation-free exclusive scan -------------------------------------------------------------
 * No counterpart in the reference.  out[i] = in[0] + ... + in[i-1] over n uint32 elements (sums
 * wrap mod 2^32), the same decoupled look-back scan the rounds use for photon offsets and cell
 * starts, and *total (device pointer, optional) receives the sum of all n.  For callers that may
 * not allocate device memory: a host whose device memory belongs to a caching or arena allocator
 * that has reserved the HBM, a plugin held to a fixed memory budget, or a latency-bound loop that
 * may not pay cudaMalloc/cudaFree's implicit synchronisation after start-up.  The scan's scratch
 * (tile tickets and look-back status words) is a static device array of 33,024 bytes per device
 * instead of a caller-provided buffer, so the call allocates nothing; it clears that scratch itself
 * on every call, so in/out need no initial contents.
 *   - in, out, total: device pointers on the current device (in and out may not overlap).
 *   - n <= 16,777,216 (2^24); larger n returns PHX_E_INVALID.  n == 0 writes *total = 0.
 *   - stream: a cudaStream_t (0 = legacy default stream).  The call enqueues its work there and
 *     then waits for that stream to finish, so the result is ready on return.
 *   - the first call on each device looks up the scratch array's address (cudaGetSymbolAddress)
 *     with that device current; make it before any stream capture on that device.  The address
 *     is kept per CUDA context: the first call after cudaDeviceReset, or under another driver-API
 *     context, looks it up again (so it too should precede any capture).
 *   - calls share the one scratch array per device: two calls whose scans overlap on the GPU
 *     (different streams, or different host threads) race on it and give wrong results.
 * Returns PHX_E_TIMEOUT if a bounded look-back wait gave up (results then invalid). */
PHX_API int phx_scan_noalloc(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *total, uint64_t stream);

/* ---- denoise filters (denoise/filters_gpu.py:9-86) ----------------------------------------------
 * The reference denoiser's three OpenCL image kernels, replacing mean_filter_gpu /
 * median_filter_gpu / gaussian_filter_gpu's kernel launches (filters_gpu.py:128-161).  `in` is an
 * (height, width, 3) int32 image and `out` an (height, width, 3) float32 one, both host memory;
 * each output value is taken over the window [x-k, x+k] x [y-k, y+k] clamped to the image (border
 * windows shrink), summing in the kernels' order (x outer, y inner) with one rounding per float
 * operation: the reference kernels' results bit for bit.
 *   mean:      window sum / window pixel count;
 *   median:    window median, the mean of the two middle values for an even count (k <= 2, as
 *              the reference raises for k > 2: PHX_E_INVALID);
 *   weighted:  sum of value * weights[(yy - y + k) * (2k + 1) + (xx - x + k)]; `weights` holds
 *              (2k+1)^2 floats (gaussian_filter_gpu passes the normalised Gaussian).
 * k <= 32.  Synchronous on a stream of its own on the current device.  kernel_ms, if not NULL,
 * receives the filter kernel's CUDA-event time (copies excluded). */
PHX_API int phx_mean_filter(const int32_t *in, float *out, uint32_t width, uint32_t height, uint32_t k,
                            float *kernel_ms);
PHX_API int phx_median_filter(const int32_t *in, float *out, uint32_t width, uint32_t height, uint32_t k,
                              float *kernel_ms);
PHX_API int phx_weighted_filter(const int32_t *in, float *out, const float *weights, uint32_t width, uint32_t height,
                                uint32_t k, float *kernel_ms);

PHX_API const char *phx_last_error(void);
PHX_API const char *phx_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PHX_H */
