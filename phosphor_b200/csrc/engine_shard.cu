// engine_shard.cu — one image rendered by several GPUs (one process and one context per GPU).
// No counterpart in the reference (single device).
//
// Rank r of W owns the contiguous pixel range [P*r/W, P*(r+1)/W) and the photon paths
// [E*r/W, E*(r+1)/W).  A round on every rank: the round seed (identical on all ranks: same seed
// state), the camera pass over its pixels, the photon pass over its paths, the scan and compaction
// of its stored photons — which are the global canonical photons of those paths, in canonical order
// — then the one exchange of the round: an all-gather of every rank's stored photons (24 B each)
// concatenated in rank order, which is exactly the global canonical order.  Every rank then hashes
// and sorts all photons and gathers its own pixels, so each pixel's flux, weight and radiance are
// bit-identical to a single-GPU render.  The exchange runs over NCCL (phx_shard_round), or through
// the host with phx_shard_begin / phx_shard_get_photons / phx_shard_put_photons / phx_shard_end,
// which lets any transport (or a test running all ranks on one GPU) move the photons.
#include "engine.hpp"
#include "nccl_dl.hpp"

#include <dlfcn.h>

#include <cstdlib>
#include <cstring>
#include <mutex>

namespace phx {

#define CK(x)                                                                                                          \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess)                                                                                         \
            return fail(PHX_E_CUDA, std::string(#x) + ": " + cudaGetErrorString(e_));                                  \
    } while (0)

const NcclApi *nccl_api(std::string *why) {
    static std::mutex mu;
    static NcclApi api;
    static int state = 0; // 0 untried, 1 loaded, -1 failed
    static std::string reason;
    std::lock_guard<std::mutex> lock(mu);
    if (state == 0) {
        // the process's own NCCL first, then PHX_NCCL_LIB (a path), then the system library
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        const char *env = getenv("PHX_NCCL_LIB");
        if (!h && env && *env)
            h = dlopen(env, RTLD_NOW | RTLD_GLOBAL);
        if (!h)
            h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            state = -1;
            const char *e = dlerror();
            reason = std::string("libnccl.so.2 not found: ") + (e ? e : "");
        } else {
            bool ok = true;
            auto sym = [&](auto &fn, const char *name) {
                fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
                if (!fn) {
                    ok = false;
                    reason = std::string("NCCL symbol missing: ") + name;
                }
            };
            sym(api.GetUniqueId, "ncclGetUniqueId");
            sym(api.CommInitRank, "ncclCommInitRank");
            sym(api.CommDestroy, "ncclCommDestroy");
            sym(api.AllGather, "ncclAllGather");
            sym(api.Broadcast, "ncclBroadcast");
            sym(api.GroupStart, "ncclGroupStart");
            sym(api.GroupEnd, "ncclGroupEnd");
            sym(api.GetErrorString, "ncclGetErrorString");
            state = ok ? 1 : -1;
        }
    }
    if (state != 1) {
        if (why)
            *why = reason;
        return nullptr;
    }
    return &api;
}

namespace {
int nccl_fail(const NcclApi *api, ncclResult_t r, const char *what) {
    return fail(PHX_E_CUDA, std::string(what) + ": " + (api->GetErrorString ? api->GetErrorString(r) : "NCCL error"));
}
} // namespace

int Engine::set_shard(uint32_t rank, uint32_t world) {
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "sharding is only available on single-scene contexts");
    if (world == 0 || rank >= world || world > total_pixels || world > total_emit)
        return fail(PHX_E_INVALID, "need rank < world <= pixels and photons per round");
    if (nccl_comm)
        return fail(PHX_E_STATE, "the shard layout is fixed once NCCL is attached");
    adjoint_invalidate();
    invalidate_graph(); // launch ranges are baked into captured rounds
    shard.rank = rank;
    shard.world = world;
    shard.pix_lo = (uint32_t)((uint64_t)total_pixels * rank / world);
    shard.pix_hi = (uint32_t)((uint64_t)total_pixels * (rank + 1) / world);
    shard.emit_lo = (uint32_t)((uint64_t)total_emit * rank / world);
    shard.emit_hi = (uint32_t)((uint64_t)total_emit * (rank + 1) / world);
    shard_phase = 0;
    return PHX_OK;
}

int Engine::set_photon_total(uint32_t n) {
    CK(cudaMemcpy(d_ntotal.p, &n, 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(offsets.as<u32>() + total_emit, &n, 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(cell_start.as<u32>() + total_cells, &n, 4, cudaMemcpyHostToDevice));
    return PHX_OK;
}

int Engine::shard_begin(uint32_t *n_local) {
    if (sc.size() != 1)
        return fail(PHX_E_UNSUPPORTED, "sharding is only available on single-scene contexts");
    adjoint_invalidate();
    enq_seeds();
    enq_trace();
    // paths outside this rank's range store nothing: their counts must read 0 in the scan
    CK(cudaMemsetAsync(counts.p, 0, 4 * ((size_t)total_emit + 1), st));
    enq_emit();
    uint32_t n = 0;
    int r = read_total(&n);
    if (r)
        return r;
    shard_n_local = n;
    shard_phase = 1;
    if (n_local)
        *n_local = n;
    return PHX_OK;
}

int Engine::shard_get_photons(float *pos4, uint32_t *pd2, uint32_t n) {
    if (shard_phase != 1)
        return fail(PHX_E_STATE, "shard_get_photons needs a preceding shard_begin");
    if (n != shard_n_local || (n && (!pos4 || !pd2)))
        return fail(PHX_E_INVALID, "n must be the photon count shard_begin returned");
    if (n) {
        CK(cudaMemcpy(pos4, ph_pos.p, 16 * (size_t)n, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(pd2, ph_pd.p, 8 * (size_t)n, cudaMemcpyDeviceToHost));
    }
    return PHX_OK;
}

int Engine::shard_put_photons(const float *pos4, const uint32_t *pd2, uint32_t n_all) {
    if (shard_phase != 1)
        return fail(PHX_E_STATE, "shard_put_photons needs a preceding shard_begin");
    if (n_all > max_photons || (n_all && (!pos4 || !pd2)))
        return fail(PHX_E_INVALID, "photon count exceeds the photon buffer");
    if (n_all) {
        CK(cudaMemcpy(ph_pos.p, pos4, 16 * (size_t)n_all, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(ph_pd.p, pd2, 8 * (size_t)n_all, cudaMemcpyHostToDevice));
    }
    int r = set_photon_total(n_all);
    if (r)
        return r;
    shard_n_all = n_all;
    shard_phase = 2;
    return PHX_OK;
}

int Engine::shard_end() {
    if (shard_phase != 2)
        return fail(PHX_E_STATE, "shard_end needs the round's photons (shard_put_photons or the NCCL exchange)");
    shard_phase = 0;
    if (shard_n_all == 0)
        return fail(PHX_E_NO_PHOTONS, "no photon hit on any rank (renderer.cpp:117-118)");
    sc[0].n_photons_last = shard_n_all;
    stage_state |= 2;
    enq_hash_sort();
    enq_gather();
    int r = sync_and_check();
    if (r)
        return r;
    count_round(1);
    return PHX_OK;
}

int Engine::shard_nccl_init(const uint8_t *id) {
    std::string why;
    const NcclApi *api = nccl_api(&why);
    if (!api)
        return fail(PHX_E_UNSUPPORTED, why);
    if (!id)
        return fail(PHX_E_INVALID, "null NCCL unique id");
    if (nccl_comm)
        return fail(PHX_E_STATE, "NCCL already attached");
    ncclUniqueId uid;
    std::memcpy(&uid, id, sizeof(uid));
    CK(cudaSetDevice(device));
    ncclComm_t comm = nullptr;
    ncclResult_t nr = api->CommInitRank(&comm, (int)shard.world, uid, (int)shard.rank);
    if (nr != ncclSuccess)
        return nccl_fail(api, nr, "ncclCommInitRank");
    nccl_comm = comm;
    int r;
    if ((r = sh_pos.alloc(16 * max_photons)) || (r = sh_pd.alloc(8 * max_photons)) ||
        (r = sh_cnt.alloc(4 * (size_t)shard.world)))
        return r;
    return PHX_OK;
}

void Engine::shard_release() {
    if (nccl_comm) {
        if (const NcclApi *api = nccl_api(nullptr))
            api->CommDestroy((ncclComm_t)nccl_comm);
        nccl_comm = nullptr;
    }
    sh_pos.release();
    sh_pd.release();
    sh_cnt.release();
}

int Engine::shard_round() {
    if (!nccl_comm)
        return fail(PHX_E_STATE, "shard_round needs NCCL attached (phx_shard_nccl)");
    const NcclApi *api = nccl_api(nullptr);
    uint32_t n = 0;
    int r = shard_begin(&n);
    if (r)
        return r;
    const uint32_t W = shard.world;
    ncclComm_t comm = (ncclComm_t)nccl_comm;
    ncclResult_t nr = api->AllGather(d_ntotal.p, sh_cnt.p, 1, ncclUint32, comm, st);
    if (nr != ncclSuccess)
        return nccl_fail(api, nr, "ncclAllGather (photon counts)");
    std::vector<uint32_t> cnt(W);
    CK(cudaMemcpyAsync(cnt.data(), sh_cnt.p, 4 * (size_t)W, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    uint64_t total = 0;
    std::vector<uint64_t> off(W);
    for (uint32_t q = 0; q < W; q++) {
        off[q] = total;
        total += cnt[q];
    }
    if (total > max_photons)
        return fail(PHX_E_OVERFLOW, "gathered photons exceed the photon buffer");
    // all-gather of unequal segments: one broadcast per rank, in one group
    if ((nr = api->GroupStart()) != ncclSuccess)
        return nccl_fail(api, nr, "ncclGroupStart");
    for (uint32_t q = 0; q < W; q++) {
        if (!cnt[q])
            continue;
        char *dpos = sh_pos.as<char>() + 16 * off[q];
        char *dpd = sh_pd.as<char>() + 8 * off[q];
        const void *spos = q == shard.rank ? ph_pos.p : dpos;
        const void *spd = q == shard.rank ? ph_pd.p : dpd;
        if ((nr = api->Broadcast(spos, dpos, 4 * (size_t)cnt[q], ncclFloat32, (int)q, comm, st)) != ncclSuccess ||
            (nr = api->Broadcast(spd, dpd, 2 * (size_t)cnt[q], ncclUint32, (int)q, comm, st)) != ncclSuccess) {
            api->GroupEnd();
            return nccl_fail(api, nr, "ncclBroadcast (photons)");
        }
    }
    if ((nr = api->GroupEnd()) != ncclSuccess)
        return nccl_fail(api, nr, "ncclGroupEnd");
    if (total) {
        CK(cudaMemcpyAsync(ph_pos.p, sh_pos.p, 16 * total, cudaMemcpyDeviceToDevice, st));
        CK(cudaMemcpyAsync(ph_pd.p, sh_pd.p, 8 * total, cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaStreamSynchronize(st));
    if ((r = set_photon_total((uint32_t)total)))
        return r;
    shard_n_all = (uint32_t)total;
    shard_phase = 2;
    return shard_end();
}

} // namespace phx
