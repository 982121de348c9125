// engine.hpp — device memory layout and stage orchestration for one or many scenes.
//
// HBM layout (all scenes concatenated in scene order; sizes per buffer below):
//   per pixel    hit point SoA: 6 x float4 (pos, normal, throughput, base colour, direct,
//                emission) + SPPM state flux float4, weight f32, radiance float4   (132 B)
//   per path     stored-photon count u32, exclusive offset u32
//   per slot     photon slot (max_bounces per path, slot-major): float4 pos + uint2 (rgbe, oct)
//   per photon   canonical float4 pos + uint2, u32 key, sort keys/values, cell-ordered
//                float4 {x,y,z,dir bits} + u32 power
//   per cell     count u32, start u32 (one extra trailing cell holds the total)
// A context is an engine with one scene; a batch is an engine with many, every stage of every
// scene in one launch.
#pragma once

#include <string>
#include <vector>

#include "host.hpp"
#include "kernels.hpp"

namespace phx {

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    int alloc(size_t b);
    void release();
    template <class T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct SceneSlot {
    phx_params prm{};
    phx_photon_hash_data hash{};
    std::vector<phx_bvh_node> nodes; // the reference tree (read-back, grid box, tie-break ranks)
    uint32_t depth = 0;
    uint32_t trav_depth = 0, trav_inner = 0; // the device traversal tree
    float setup_ms = 0.0f, bvh_ms = 0.0f;     // wall time of the scene setup, of which the trees
    uint32_t n_tris = 0;
    std::vector<DevBuf> bufs;
    SceneDesc desc{};
    uint64_t total_emitted = 0;
    uint32_t rounds = 0;
    uint32_t n_photons_last = 0;
    std::vector<phx_material> mats; // host copies of the parameters the adjoint differentiates
    std::vector<phx_light> lights;
};

enum Stage {
    ST_SEEDS = 0,
    ST_TRACE,
    ST_SHADOW,
    ST_EMIT,
    ST_EMIT_SCAN,
    ST_HASH,
    ST_CELL_SCAN,
    ST_SORT,
    ST_RECORDS,
    ST_GATHER,
    ST__N
};

// One image over several GPUs: this rank's pixel and photon-path ranges (engine_shard.cu).
struct ShardState {
    uint32_t rank = 0, world = 1;
    uint32_t pix_lo = 0, pix_hi = 0, emit_lo = 0, emit_hi = 0;
};

// The buffers one round writes and then reads: round seeds, persistent-kernel queues, camera-path
// outputs and NEE slots, photon slots and canonical photons, cell counts and starts, sort buffers,
// sorted records, scan and sort scratch.  Set 0 views the engine's own buffers; the pipelined
// graph form allocates further sets for the earlier rounds of a captured group.  The SPPM state,
// the error words and the gather's pixel-order buffers stay shared (the gathers run in order).
struct RoundSet {
    u32 *seeds = nullptr, *queue = nullptr, *ntotal = nullptr;
    float4 *hp[6] = {};
    float4 *nee_ray = nullptr, *nee_val = nullptr, *stash_sn = nullptr;
    u32 *stash_rng = nullptr;
    float4 *spec_ray = nullptr, *spec_val = nullptr, *spec_org = nullptr;
    u32 *spec_pix = nullptr, *spec_next = nullptr, *def_cnt = nullptr;
    float4 *def_prefix = nullptr, *def_val = nullptr;
    u32 *def_tag = nullptr;
    float4 *slot_pos = nullptr;
    uint2 *slot_pd = nullptr;
    u32 *counts = nullptr, *offsets = nullptr;
    float4 *ph_pos = nullptr;
    uint2 *ph_pd = nullptr;
    u32 *keys = nullptr, *cell_count = nullptr, *cell_start = nullptr;
    u32 *sk0 = nullptr, *sk1 = nullptr, *sv0 = nullptr, *sv1 = nullptr;
    float4 *s_posdir = nullptr;
    u32 *s_power = nullptr;
    float4 *s_dir = nullptr, *s_pow = nullptr;
    void *scan_scr = nullptr, *radix_scr = nullptr;
    u32 *perm = nullptr; // the photon sort's permutation (set by the hash stage)
};

uint32_t light_sample_draws(const phx_light *l, uint32_t n, float total_lum);

class Engine {
  public:
    ~Engine();
    int create(const phx_scene *scenes, const phx_params *params, uint32_t n, int device);

    // enqueue (no host sync) on the engine's buffers (set 0)
    void enq_seeds() { enq_seeds_r(rs0, st); }
    void enq_trace() { enq_trace_r(rs0, st); }
    void enq_emit(cudaStream_t s = nullptr) { enq_emit_r(rs0, s ? s : st); } // nullptr: the engine's stream
    void enq_hash_sort() {
        enq_hash_sort_r(rs0, st);
        perm = rs0.perm;
    }
    void enq_gather() { enq_gather_r(rs0, st); }
    void enq_round();

    int plain_round();                // reference form: two host syncs per round
    int graph_rounds(uint32_t rounds); // captured round replayed `rounds` times
    int seeded_round(uint32_t seed);   // one replay, seed copied from pinned host memory (async)
    int sync_and_check();
    int set_seed(uint32_t seed);      // explicit seed for the per-stage API (all scenes)
    int read_total(uint32_t *n);      // blocking read of the stored-photon total
    int read_buffer(uint32_t scene, int which, void *dst, uint64_t off, uint64_t bytes);
    int write_buffer(uint32_t scene, int which, const void *src, uint64_t off, uint64_t bytes);
    int set_n_photons(uint32_t n);
    int info(uint32_t scene, phx_info *out);
    int image(uint32_t scene, float exposure, int tonemap, uint64_t total_photons, uint32_t rounds, float *rgb,
              uint8_t *ldr);
    int set_alpha(float alpha);
    void set_profiling(bool on);
    void stage_ms(float *out) const;
    void invalidate_graph();
    int set_active(uint32_t scene, bool on); // retire / resume a scene of a batch
    // Picks the launch tuning that minimises the time of a graph-replayed round (coordinate descent
    // over the result-neutral knobs); the SPPM state is saved and restored around the trials.
    int autotune(uint32_t rounds_per_trial, phx_tuning *chosen);

    // sharded rendering of one image (engine_shard.cu)
    ShardState shard;
    int set_shard(uint32_t rank, uint32_t world);
    int shard_begin(uint32_t *n_local);
    int shard_get_photons(float *pos4, uint32_t *pd2, uint32_t n);
    int shard_put_photons(const float *pos4, const uint32_t *pd2, uint32_t n_all);
    int shard_end();
    int shard_nccl_init(const uint8_t *id);
    int shard_round();
    bool any_active() const;
    bool untextured() const; // no material of any scene has a texture (indices are fixed at set-up)
    bool photon_prestart() const; // every scene keeps >= 3 photon slots per path (k_emit_start)

    // differentiation (single-scene engines; engine_adjoint.cu)
    int set_materials(const phx_material *m, uint32_t n);
    int set_lights(const phx_light *l, uint32_t n);
    uint32_t n_params() const;
    int adjoint_forward(uint32_t rounds, float *image);
    int adjoint_backward(const float *dl_dimage, float *grad, uint32_t n_grad);
    void adjoint_invalidate() {
        if (!in_adjoint)
            adj_ready = false;
    }

    int device = 0;
    cudaStream_t st = nullptr;
    std::vector<SceneSlot> sc;
    uint32_t total_pixels = 0, total_emit = 0, total_cells = 0, total_nee = 0;
    uint64_t total_slots = 0, max_photons = 0;
    uint32_t key_bits = 1;
    phx_tuning tune{};
    int stage_state = 0;

  private:
    LaunchCtx lc() const { return lc(rs0); }
    GridBufs gb() const { return gb(rs0); }
    LaunchCtx lc(const RoundSet &R) const;
    GridBufs gb(const RoundSet &R) const;
    void enq_seeds_r(RoundSet &R, cudaStream_t s);
    void enq_trace_r(RoundSet &R, cudaStream_t s);
    void enq_emit_r(RoundSet &R, cudaStream_t s);
    void enq_hash_sort_r(RoundSet &R, cudaStream_t s);
    void enq_gather_r(RoundSet &R, cudaStream_t s);
    RoundSet view_own_buffers();
    RoundSet rs0;
    // pipelined graph form: `pipe_k` rounds per captured graph, each round's passes on branches of
    // their own, the gathers in round order; extra buffer sets for all but the last round
    uint32_t pipeline_rounds() const;
    int alloc_round_sets(uint32_t sets);
    int capture_pipelined(uint32_t k);
    std::vector<std::vector<DevBuf>> xbufs;
    std::vector<RoundSet> xsets;
    std::vector<cudaStream_t> pipe_st;
    std::vector<cudaEvent_t> pipe_ev;
    cudaGraph_t graph_pipe = nullptr;
    cudaGraphExec_t gexec_pipe = nullptr;
    uint32_t pipe_k = 0;
    int upload_scene(uint32_t i, const phx_scene &s, const phx_params &p, uint32_t *pix, uint32_t *emit,
                     uint32_t *cell, uint64_t *slot);
    int scene_photon_range(uint32_t s, uint32_t *off, uint32_t *n);
    void ev(int stage, bool end, cudaStream_t s = nullptr);
    cudaStream_t st_side = nullptr;          // second branch of a captured round (photon pass)
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    void accumulate_profile();

    DevBuf d_desc, d_pix_bases, d_emit_bases, d_nee_bases, d_seeds, d_rng, d_err, d_ovf, d_queue, d_ntotal;
    DevBuf nee_ray, nee_val, stash_sn, stash_rng;
    // deferred specular NEE: sample slots (as many as the diffuse ones) and per-pixel term lists
    DevBuf spec_ray, spec_val, spec_org, spec_pix, spec_next, def_cnt, def_prefix, def_val, def_tag;
    bool spec_deferred() const { return tune.persistent && tune.nee_wavefront && total_nee > 0; }
    DevBuf hp[6], flux, weight, radiance;
    DevBuf slot_pos, slot_pd, counts, offsets, ph_pos, ph_pd, keys, cell_count, cell_start;
    DevBuf sk0, sk1, sv0, sv1, s_posdir, s_power, s_dir, s_pow, scan_scr, radix_scr, img_rgb, img_ldr;
    int capture(bool with_seeds, cudaGraph_t *g, cudaGraphExec_t *ge);
    void count_round(uint32_t rounds);

    int upload_descs();
    int set_photon_total(uint32_t n);
    void shard_release();
    void *nccl_comm = nullptr; // ncclComm_t once attached
    DevBuf sh_pos, sh_pd, sh_cnt;
    uint32_t shard_n_local = 0, shard_n_all = 0;
    int shard_phase = 0;
    // adjoint state: per round seeds, search radii² and SPPM ratios of the forward pass
    DevBuf adj_seeds, adj_r2, adj_ratio, adj_k, adj_img, adj_g, adj_gT, adj_gA, adj_gphi, adj_slot_pow, adj_ph_pow,
        adj_grad;
    uint32_t adj_rounds = 0;
    bool adj_ready = false, adj_k_ready = false, in_adjoint = false;
    float *rec_r2 = nullptr, *rec_ratio = nullptr; // recording targets of the gather (forward pass)

    // pixel order of the gather (pixels grouped by photon-grid cell)
    DevBuf pk_keys, pk_t0, pk_t1, pk_v0, pk_v1, pk_scr, d_npix;
    uint32_t pix_key_bits = 0; // 0: the gather runs in pixel order
    u32 *pix_order = nullptr;

    u32 *perm = nullptr;
    u32 *h_pinned = nullptr;
    cudaGraph_t graph = nullptr, graph_host = nullptr;
    cudaGraphExec_t gexec = nullptr, gexec_host = nullptr;
    static constexpr int SEED_RING = 64;
    u32 *h_seed_ring = nullptr; // pinned staging for host-given round seeds
    cudaEvent_t seed_ev[SEED_RING] = {};
    uint32_t seed_slot = 0;
    uint32_t pending_seeded = 0;
    bool profiling = false, capturing = false;
    cudaEvent_t events[2 * ST__N] = {};
    double prof_ms[ST__N] = {};
    uint32_t prof_rounds = 0;
};

extern thread_local std::string g_last_error;
int fail(int code, const std::string &msg);

} // namespace phx
