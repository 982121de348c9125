// k_grid.cu — photon grid build: compaction + cell hashing, the single-pass exclusive scan and
// the stable counting sort that puts photons in cell order.
//
// Reference: hash_photons.cl:4-13 (key = get_hash, atomic count), scan_small_chunks.cl /
// scan_big_chunks.cl / scan_add_offsets.cl (three-kernel exclusive scan, capped at 4096^2 cells by
// constants.h:8-9), the start->end copy (renderer.cpp:147) and scatter_photons.cl:4-18 (atomic
// cursor per cell, so the in-cell order depends on scheduling).
//
// Here:
//  * k_compact_hash reads each path's stored-photon slots, writes the photons in canonical order
//    (offsets from the scan of per-path counts), hashes them to 32-bit keys and counts keys with
//    atomics (counts are order-independent, hence deterministic).  Keys of batched scenes are
//    offset by the scene's first cell so all scenes share one key space.
//  * k_scan is a single-pass decoupled look-back scan (Merrill & Garland, "Single-pass Parallel
//    Prefix Scan with Decoupled Look-back", 2016): each 4096-element tile reduces with warp
//    shuffles, publishes its aggregate, then warp 0 looks back over 32 predecessors at a time.
//    Tiles are numbered by an atomic ticket so a tile only waits on tiles already running; every
//    wait is bounded and sets an error bit instead of hanging.  No cap on the cell count.
//  * the scatter is a stable LSD counting sort of (key, canonical index): one counting pass per
//    digit of at most 11 bits (reduce: per-tile digit histograms; scan: the same look-back scan;
//    downsweep: warp-level stable ranks with __match_any_sync).  Within a cell photons keep
//    canonical order, which is what a sequential run of scatter_photons.cl produces, so keys,
//    counts, starts and the permutation are deterministic and bit-exact.
#include "kernels.hpp"

#include <cuda/atomic>
#include <mutex>
#include <string>

namespace phx {

// ---- compaction --------------------------------------------------------------------------------
// Path t's j-th stored photon goes to canonical index offsets[t] + j.
__global__ void __launch_bounds__(256) k_compact(LaunchCtx lc, GridBufs g) {
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.total_emit)
        return;
    u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.emit_bases, lc.n_scenes, gid);
    const SceneDesc &sc = lc.scenes[s];
    const u32 c = g.counts[gid];
    const u32 off = g.offsets[gid];
    u64 slot = sc.slot_base + (gid - sc.emit_base);
    for (u32 j = 0; j < c; j++, slot += sc.n_emit) {
        g.ph_pos[off + j] = g.slot_pos[slot];
        g.ph_pd[off + j] = g.slot_pd[slot];
    }
}

void launch_compact(const LaunchCtx &lc, const GridBufs &g, cudaStream_t st) {
    if (lc.total_emit == 0)
        return;
    k_compact<<<(lc.total_emit + 255) / 256, 256, 0, st>>>(lc, g);
}

// ---- hash (hash_photons.cl:4-13) ---------------------------------------------------------------
// Canonical photon i belongs to the scene whose photon range [offsets[emit_base], ...) holds it.
// The grid is sized for the photon capacity (photons_per_round * max_bounces, often 10-100x the
// photons stored), so the threads stride over the stored ones instead of one block per 256 slots
// of capacity: the empty blocks alone took most of the stage (atrium workload).
PHX_DI void hash_one(const LaunchCtx &lc, const GridBufs &g, u64 i) {
    u32 s = 0;
    if (lc.n_scenes > 1) {
        u32 lo = 0, hi = lc.n_scenes;
        while (hi - lo > 1) {
            u32 mid = (lo + hi) >> 1;
            if (g.offsets[__ldg(&lc.emit_bases[mid])] <= i)
                lo = mid;
            else
                hi = mid;
        }
        s = lo;
    }
    const SceneDesc &sc = lc.scenes[s];
    float4 p = g.ph_pos[i];
    u32 key = sc.cell_base + get_hash(p.x, p.y, p.z, sc.grid);
    g.keys[i] = key;
    atomicAdd(&g.cell_count[key], 1u);
}

__global__ void __launch_bounds__(256) k_hash(LaunchCtx lc, GridBufs g, const u32 *n_dev, u64 n_max) {
    const u64 n = min((u64)*n_dev, n_max);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        hash_one(lc, g, i);
}

// blocks for a grid-stride loop over at most n_max items: enough to fill every SM several times
static unsigned stride_blocks(u64 n_max, unsigned threads) {
    const u64 need = (n_max + threads - 1) / threads, cap = (u64)(g_sm_count > 0 ? g_sm_count : 148) * 16;
    return (unsigned)(need < cap ? (need > 0 ? need : 1) : cap);
}

void launch_hash(const LaunchCtx &lc, const GridBufs &g, const u32 *n_dev, u64 n_max, cudaStream_t st) {
    if (n_max == 0)
        return;
    k_hash<<<stride_blocks(n_max, 256), 256, 0, st>>>(lc, g, n_dev, n_max);
}

// ---- decoupled look-back exclusive scan --------------------------------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr u64 SCAN_TILE = (u64)SCAN_THREADS * SCAN_ITEMS;
constexpr u64 FLAG_A = 1ull << 32;
constexpr u64 FLAG_P = 2ull << 32;
constexpr u32 LOOKBACK_SPIN_LIMIT = 1u << 21;

static inline u64 scan_tiles(u64 n) { return (n + SCAN_TILE - 1) / SCAN_TILE; }

size_t scan_scratch_bytes(u64 n) { return 256 + 8 * (size_t)scan_tiles(n > 0 ? n : 1); }

PHX_DI void publish(u64 *status, u64 word) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(*reinterpret_cast<unsigned long long *>(status));
    a.store(word, cuda::memory_order_release);
}
PHX_DI u64 peek(u64 *status) {
    cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> a(*reinterpret_cast<unsigned long long *>(status));
    return a.load(cuda::memory_order_acquire);
}

// n_dyn (optional): the length is only n' = min(n, dyn_mul * ceil(*n_dyn / dyn_div)), read on the
// device (a graph replays one launch shape for every round); tiles past n' return at once, and
// since a tile only waits on lower ones, no tile waits on them.
__global__ void __launch_bounds__(SCAN_THREADS) k_scan(const u32 *__restrict__ in, u32 *__restrict__ out, u64 n,
                                                      u32 *tile_counter, u64 *status, u32 *total, u32 *err,
                                                      const u32 *n_dyn, u32 dyn_div, u32 dyn_mul) {
    __shared__ u32 s_tile;
    __shared__ u32 s_warp[SCAN_THREADS / 32];
    __shared__ u32 s_prefix;
    if (threadIdx.x == 0)
        s_tile = atomicAdd(tile_counter, 1u);
    if (n_dyn)
        n = min(n, (u64)dyn_mul * (((u64)*n_dyn + dyn_div - 1) / dyn_div));
    __syncthreads();
    const u32 tile = s_tile;
    if ((u64)tile * SCAN_TILE >= n && !(tile == 0 && total)) // past the length (tile 0 still writes the total)
        return;
    const u64 base = (u64)tile * SCAN_TILE;
    const u64 i0 = base + (u64)threadIdx.x * SCAN_ITEMS;
    u32 v[SCAN_ITEMS];
    const bool full = i0 + SCAN_ITEMS <= n && ((reinterpret_cast<uintptr_t>(in + i0) & 15u) == 0) &&
                      ((reinterpret_cast<uintptr_t>(out + i0) & 15u) == 0);
    if (full) {
        const uint4 *p = reinterpret_cast<const uint4 *>(in + i0);
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS / 4; k++) {
            uint4 q = p[k];
            v[4 * k] = q.x;
            v[4 * k + 1] = q.y;
            v[4 * k + 2] = q.z;
            v[4 * k + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++)
            v[k] = (i0 + k < n) ? in[i0 + k] : 0u;
    }
    u32 sum = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) {
        u32 x = v[k];
        v[k] = sum;
        sum += x;
    }
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    u32 incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (u32)o)
            incl += y;
    }
    if (lane == 31)
        s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        u32 w = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0u;
#pragma unroll
        for (int o = 1; o < SCAN_THREADS / 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= (u32)o)
                w += y;
        }
        if (lane < SCAN_THREADS / 32)
            s_warp[lane] = w;
    }
    __syncthreads();
    const u32 thread_excl = (warp ? s_warp[warp - 1] : 0u) + incl - sum;
    const u32 aggregate = s_warp[SCAN_THREADS / 32 - 1];
    if (warp == 0) {
        u32 excl = 0;
        if (tile == 0) {
            if (lane == 0)
                publish(&status[0], FLAG_P | aggregate);
        } else {
            if (lane == 0)
                publish(&status[tile], FLAG_A | aggregate);
            long long pred = (long long)tile - 1;
            u32 spins = 0;
            for (;;) {
                long long idx = pred - (long long)lane;
                u64 word = idx >= 0 ? peek(&status[idx]) : FLAG_P;
                u32 flag = (u32)(word >> 32);
                u32 pmask = __ballot_sync(0xffffffffu, flag == 2u);
                u32 xmask = __ballot_sync(0xffffffffu, flag == 0u);
                u32 limit = pmask ? (u32)(__ffs(pmask) - 1) : 31u;
                u32 needed = limit == 31u ? 0xffffffffu : ((1u << (limit + 1)) - 1u);
                if (xmask & needed) {
                    if (++spins > LOOKBACK_SPIN_LIMIT) {
                        if (lane == 0)
                            atomicOr(err, ERR_LOOKBACK_TIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                u32 val = lane <= limit ? (u32)word : 0u;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1)
                    val += __shfl_xor_sync(0xffffffffu, val, o);
                excl += val;
                if (pmask)
                    break;
                pred -= 32;
            }
            if (lane == 0)
                publish(&status[tile], FLAG_P | (u32)(excl + aggregate));
        }
        if (lane == 0)
            s_prefix = excl;
    }
    __syncthreads();
    const u32 prefix = s_prefix + thread_excl;
    if (full) {
        uint4 *p = reinterpret_cast<uint4 *>(out + i0);
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS / 4; k++)
            p[k] = make_uint4(v[4 * k] + prefix, v[4 * k + 1] + prefix, v[4 * k + 2] + prefix, v[4 * k + 3] + prefix);
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++)
            if (i0 + k < n)
                out[i0 + k] = v[k] + prefix;
    }
    if (total && threadIdx.x == 0 && base + SCAN_TILE >= n)
        *total = s_prefix + aggregate;
}

void launch_scan(const u32 *in, u32 *out, u64 n, void *scratch, u32 *total, u32 *err, cudaStream_t st,
                 const u32 *n_dyn, u32 dyn_div, u32 dyn_mul) {
    if (n == 0)
        return;
    u64 tiles = scan_tiles(n);
    cudaMemsetAsync(scratch, 0, scan_scratch_bytes(n), st);
    u32 *counter = reinterpret_cast<u32 *>(scratch);
    u64 *status = reinterpret_cast<u64 *>(reinterpret_cast<char *>(scratch) + 256);
    k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, counter, status, total, err, n_dyn, dyn_div, dyn_mul);
}

// Withholds tile 0: the ticket counter starts at 1, so tiles 1..T wait on a tile that never
// publishes.  The grid still has T blocks (tickets 1..T); the status array has T+1 entries and
// the data arrays one spare tile, so the extra ticket T stays in bounds (its loads and stores are
// guarded by n anyway).
int selftest_lookback_timeout(int device, u32 n, u32 *err_out) {
    if (cudaSetDevice(device) != cudaSuccess)
        return 3;
    u64 tiles = scan_tiles(n ? n : 1);
    size_t data = (size_t)(tiles + 1) * SCAN_TILE * 4;
    size_t scr = 256 + 8 * (size_t)(tiles + 1);
    void *in = nullptr, *out = nullptr, *scratch = nullptr, *err = nullptr;
    int rc = 0;
    if (cudaMalloc(&in, data) || cudaMalloc(&out, data) || cudaMalloc(&scratch, scr) || cudaMalloc(&err, 4)) {
        rc = 2;
    } else {
        cudaMemset(in, 0, data);
        cudaMemset(scratch, 0, scr);
        cudaMemset(err, 0, 4);
        u32 one = 1;
        cudaMemcpy(scratch, &one, 4, cudaMemcpyHostToDevice); // ticket 0 is never handed out
        k_scan<<<(unsigned)tiles, SCAN_THREADS>>>((const u32 *)in, (u32 *)out, n, (u32 *)scratch,
                                                  (u64 *)((char *)scratch + 256), nullptr, (u32 *)err, nullptr, 1u, 1u);
        if (cudaDeviceSynchronize() != cudaSuccess)
            rc = 3;
        cudaMemcpy(err_out, err, 4, cudaMemcpyDeviceToHost);
    }
    cudaFree(in);
    cudaFree(out);
    cudaFree(scratch);
    cudaFree(err);
    cudaGetLastError();
    return rc;
}

// ---- stable LSD counting sort ------------------------------------------------------------------
constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ITEMS = 16;
constexpr u64 RS_TILE = (u64)RS_THREADS * RS_ITEMS; // 4096; warp w owns [w*512, w*512+512)
constexpr u32 RS_MAX_BITS = 11;

struct RadixPlan {
    u32 passes, bits;
};
static RadixPlan radix_plan(u32 key_bits) {
    if (key_bits == 0)
        key_bits = 1;
    u32 passes = (key_bits + RS_MAX_BITS - 1) / RS_MAX_BITS;
    u32 bits = (key_bits + passes - 1) / passes;
    return {passes, bits};
}

u32 radix_passes(u32 key_bits) { return radix_plan(key_bits).passes; }

size_t radix_scratch_bytes(u64 n_max, u32 key_bits) {
    RadixPlan p = radix_plan(key_bits);
    u64 tiles = (n_max + RS_TILE - 1) / RS_TILE;
    if (tiles == 0)
        tiles = 1;
    u64 hist = ((u64)1 << p.bits) * tiles;
    // hist + scanned hist + scan scratch
    return 2 * hist * 4 + scan_scratch_bytes(hist) + 512;
}

// The launch covers the capacity's tiles; only the first T = ceil(n / RS_TILE) hold keys, and the
// digit histograms are laid out [digit][T] for those alone, so the scan between the passes runs over
// bins * T counters instead of bins * (capacity / RS_TILE).
PHX_DI u32 radix_tiles(const u32 *n_dev) { return (u32)(((u64)*n_dev + RS_TILE - 1) / RS_TILE); }

__global__ void __launch_bounds__(RS_THREADS) k_radix_hist(const u32 *__restrict__ keys, const u32 *n_dev, u32 shift,
                                                          u32 bits, u32 *__restrict__ hist, u32 n_tiles) {
    extern __shared__ u32 sh[];
    const u32 bins = 1u << bits, mask = bins - 1u;
    const u32 t_used = min(radix_tiles(n_dev), n_tiles);
    if (blockIdx.x >= t_used)
        return; // uniform for the block
    for (u32 d = threadIdx.x; d < bins; d += RS_THREADS)
        sh[d] = 0;
    __syncthreads();
    const u64 n = *n_dev;
    const u64 base = (u64)blockIdx.x * RS_TILE;
    if (base < n) {
#pragma unroll 4
        for (int k = 0; k < RS_ITEMS; k++) {
            u64 idx = base + (u64)k * RS_THREADS + threadIdx.x;
            if (idx < n)
                atomicAdd(&sh[(keys[idx] >> shift) & mask], 1u);
        }
    }
    __syncthreads();
    for (u32 d = threadIdx.x; d < bins; d += RS_THREADS)
        hist[(u64)d * t_used + blockIdx.x] = sh[d];
}

__global__ void __launch_bounds__(RS_THREADS) k_radix_scatter(const u32 *__restrict__ keys_in,
                                                             const u32 *__restrict__ vals_in, u32 *__restrict__ keys_out,
                                                             u32 *__restrict__ vals_out, const u32 *n_dev, u32 shift,
                                                             u32 bits, const u32 *__restrict__ hist_scanned,
                                                             u32 n_tiles) {
    extern __shared__ u32 sh[];
    const u32 bins = 1u << bits, mask = bins - 1u;
    const u32 t_used = min(radix_tiles(n_dev), n_tiles);
    if (blockIdx.x >= t_used)
        return; // uniform for the block
    u32 *cnt = sh;                     // [RS_WARPS][bins]
    u32 *gofs = sh + RS_WARPS * bins;  // [bins]
    for (u32 i = threadIdx.x; i < RS_WARPS * bins; i += RS_THREADS)
        cnt[i] = 0;
    for (u32 d = threadIdx.x; d < bins; d += RS_THREADS)
        gofs[d] = hist_scanned[(u64)d * t_used + blockIdx.x];
    __syncthreads();
    const u64 n = *n_dev;
    const u64 base = (u64)blockIdx.x * RS_TILE;
    const u32 lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const u32 lt_mask = (1u << lane) - 1u;
    u32 *wc = cnt + warp * bins;
    u32 dig[RS_ITEMS], rnk[RS_ITEMS], key[RS_ITEMS], val[RS_ITEMS];
#pragma unroll
    for (int k = 0; k < RS_ITEMS; k++) {
        u64 idx = base + (u64)warp * (RS_ITEMS * 32) + (u64)k * 32 + lane;
        bool valid = idx < n;
        u32 kk = valid ? keys_in[idx] : 0u;
        u32 d = valid ? ((kk >> shift) & mask) : bins;
        u32 peers = __match_any_sync(0xffffffffu, d);
        u32 r = __popc(peers & lt_mask);
        u32 b = valid ? wc[d] : 0u;
        __syncwarp();
        if (valid && r == 0)
            wc[d] = b + __popc(peers);
        __syncwarp();
        dig[k] = d;
        rnk[k] = b + r;
        key[k] = kk;
        val[k] = valid ? (vals_in ? vals_in[idx] : (u32)idx) : 0u;
    }
    __syncthreads();
    for (u32 d = threadIdx.x; d < bins; d += RS_THREADS) {
        u32 run = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; w++) {
            u32 c = cnt[w * bins + d];
            cnt[w * bins + d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < RS_ITEMS; k++) {
        if (dig[k] < bins) {
            u32 pos = gofs[dig[k]] + wc[dig[k]] + rnk[k];
            if (keys_out)
                keys_out[pos] = key[k];
            vals_out[pos] = val[k];
        }
    }
}

void launch_radix_sort(const u32 *keys_in, u32 *keys_tmp0, u32 *keys_tmp1, u32 *vals0, u32 *vals1, u32 **perm_out,
                       const u32 *n_dev, u64 n_max, u32 key_bits, void *scratch, u32 *err, cudaStream_t st) {
    RadixPlan p = radix_plan(key_bits);
    u64 tiles = (n_max + RS_TILE - 1) / RS_TILE;
    if (tiles == 0)
        tiles = 1;
    const u32 bins = 1u << p.bits;
    u64 hist_n = (u64)bins * tiles;
    u32 *hist = reinterpret_cast<u32 *>(scratch);
    u32 *hist_scanned = hist + hist_n;
    void *scan_scr = reinterpret_cast<char *>(scratch) + 2 * hist_n * 4 + 256;
    size_t smem_hist = bins * 4;
    size_t smem_scatter = (size_t)(RS_WARPS + 1) * bins * 4;
    u32 *kt[2] = {keys_tmp0, keys_tmp1};
    u32 *vt[2] = {vals0, vals1};
    const u32 *src_k = keys_in;
    const u32 *src_v = nullptr;
    for (u32 pass = 0; pass < p.passes; pass++) {
        u32 shift = pass * p.bits;
        k_radix_hist<<<(unsigned)tiles, RS_THREADS, smem_hist, st>>>(src_k, n_dev, shift, p.bits, hist, (u32)tiles);
        launch_scan(hist, hist_scanned, hist_n, scan_scr, nullptr, err, st, n_dev, (u32)RS_TILE, bins);
        bool last = pass + 1 == p.passes;
        k_radix_scatter<<<(unsigned)tiles, RS_THREADS, smem_scatter, st>>>(
            src_k, src_v, last ? nullptr : kt[pass & 1], vt[pass & 1], n_dev, shift, p.bits, hist_scanned, (u32)tiles);
        src_k = kt[pass & 1];
        src_v = vt[pass & 1];
    }
    *perm_out = vt[(p.passes - 1) & 1];
}

// ---- cell-ordered photon records ---------------------------------------------------------------
// Besides the packed records, each photon's direction and power are decoded here once per round
// (the same decode_oct / decode_rgbe the gather would apply per pixel and photon), so the gather's
// per-pixel branch only loads them.
__global__ void __launch_bounds__(256) k_sorted_records(const u32 *__restrict__ perm, const float4 *__restrict__ ph_pos,
                                                       const uint2 *__restrict__ ph_pd, const u32 *n_dev,
                                                       float4 *__restrict__ s_posdir, u32 *__restrict__ s_power,
                                                       float4 *__restrict__ s_dir, float4 *__restrict__ s_pow,
                                                       u64 n_max, u32 *err) {
    const u64 n = min((u64)*n_dev, n_max);
    if (blockIdx.x == 0 && threadIdx.x == 0 && n == 0)
        atomicOr(err, ERR_NO_PHOTONS); // renderer.cpp:117-118 traps here
    for (u64 p = (u64)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (u64)gridDim.x * blockDim.x) {
        const u32 i = perm[p];
        const float4 pos = ph_pos[i];
        const uint2 pd = ph_pd[i];
        s_posdir[p] = make_float4(pos.x, pos.y, pos.z, __uint_as_float(pd.y));
        s_power[p] = pd.x;
        s_dir[p] = decode_oct(pd.y);
        s_pow[p] = decode_rgbe(pd.x);
    }
}

void launch_sorted_records(const u32 *perm, const float4 *ph_pos, const uint2 *ph_pd, const u32 *n_dev, u64 n_max,
                           float4 *s_posdir, u32 *s_power, float4 *s_dir, float4 *s_pow, u32 *err, cudaStream_t st) {
    if (n_max == 0)
        return;
    k_sorted_records<<<stride_blocks(n_max, 256), 256, 0, st>>>(perm, ph_pos, ph_pd, n_dev, s_posdir, s_power, s_dir,
                                                                s_pow, n_max, err);
}

// The decoded direction and power of records written from the host.
__global__ void __launch_bounds__(256) k_decode_records(const float4 *__restrict__ s_posdir,
                                                       const u32 *__restrict__ s_power, u64 n,
                                                       float4 *__restrict__ s_dir, float4 *__restrict__ s_pow) {
    const u64 p = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n)
        return;
    s_dir[p] = decode_oct(__float_as_uint(s_posdir[p].w));
    s_pow[p] = decode_rgbe(s_power[p]);
}

void launch_decode_records(const float4 *s_posdir, const u32 *s_power, u64 n, float4 *s_dir, float4 *s_pow,
                           cudaStream_t st) {
    if (n == 0)
        return;
    k_decode_records<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s_posdir, s_power, n, s_dir, s_pow);
}

// ---- allocation-free exclusive scan --------------------------------------------------------------
// Some callers cannot allocate device memory: hosts whose device memory is owned by a caching or
// arena allocator that has reserved most of HBM (a side cudaMalloc fails or fragments it), plugins
// whose host enforces a fixed memory budget, and latency-critical loops that may not pay
// cudaMalloc/cudaFree's implicit device synchronisation after start-up.  For them the scan's
// scratch — the tile ticket counter and one 8-byte look-back status word per 4096-element tile —
// lives in this file-scope device array instead of a buffer the caller provides.  It is sized for
// NOALLOC_SCAN_MAX_N elements (33,024 bytes per device, held by every GPU that loads the library
// until the process exits).  All calls share it: each call clears it first, and two calls whose
// kernels overlap on the GPU (different streams, or different host threads) race on it.
constexpr u32 NOALLOC_SCAN_MAX_N = 1u << 24;
constexpr u32 NOALLOC_SCAN_MAX_TILES = NOALLOC_SCAN_MAX_N / (u32)SCAN_TILE;
constexpr size_t NOALLOC_SCRATCH_BYTES = 256 + 8 * (size_t)NOALLOC_SCAN_MAX_TILES;
static __device__ __align__(256) unsigned char g_noalloc_scan_scratch[NOALLOC_SCRATCH_BYTES];

// Host-side address of g_noalloc_scan_scratch on each device.  The array's name in host code is a
// stand-in, not a device address, so the address is looked up (with the device current) through
// cudaGetSymbolAddress and passed to the kernel.  The look-up is the set-up of the first call on each
// device, which should therefore come before any stream capture on it.  The cached address belongs
// to the CUDA context it was looked up in: after cudaDeviceReset, or under another driver-API
// context on the same device, the module is loaded anew and the address changes, so each entry
// records its context and a call made under a different one repeats the set-up.
using CtxGetCurrentFn = int (*)(void **);
static std::mutex g_noalloc_mu;
struct NoallocScratch {
    void *ctx = nullptr;
    void *ptr = nullptr;
};
static NoallocScratch g_noalloc[128];

static void *current_context() {
    static CtxGetCurrentFn fn = []() -> CtxGetCurrentFn {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess) {
            cudaGetLastError();
            f = nullptr;
        } else if (q != cudaDriverEntryPointSuccess) {
            f = nullptr;
        }
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    void *ctx = nullptr;
    if (!fn || fn(&ctx) != 0)
        return nullptr;
    return ctx;
}

int scan_noalloc(const u32 *in, u32 *out, u32 n, u32 *total, cudaStream_t st, std::string &err) {
    if (n > NOALLOC_SCAN_MAX_N) {
        err = "n = " + std::to_string(n) + " exceeds the allocation-free scan's maximum of " +
              std::to_string(NOALLOC_SCAN_MAX_N) + " elements";
        return 1;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 128) {
        err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return 3;
    }
    void *scr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        void *ctx = current_context();
        NoallocScratch &c = g_noalloc[dev];
        if (!c.ptr || !ctx || c.ctx != ctx) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scan_scratch); // also makes the primary context current
            if (e != cudaSuccess || !p) {
                err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return 3;
            }
            c.ptr = p;
            c.ctx = current_context();
        }
        scr = c.ptr;
    }
    if (n == 0) {
        // like every other size, the call returns with the result written
        if (total && ((e = cudaMemsetAsync(total, 0, 4, st)) != cudaSuccess ||
                      (e = cudaStreamSynchronize(st)) != cudaSuccess)) {
            err = std::string("scan (n = 0): ") + cudaGetErrorString(e);
            return 3;
        }
        return 0;
    }
    const u64 tiles = scan_tiles(n);
    // ticket counter (offset 0), error word (offset 4) and the status words must start at zero
    if ((e = cudaMemsetAsync(scr, 0, 256 + 8 * (size_t)tiles, st)) != cudaSuccess) {
        err = std::string("cudaMemsetAsync: ") + cudaGetErrorString(e);
        return 3;
    }
    u32 *counter = reinterpret_cast<u32 *>(scr);
    u32 *errw = counter + 1;
    u64 *status = reinterpret_cast<u64 *>(reinterpret_cast<char *>(scr) + 256);
    k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, out, n, counter, status, total, errw, nullptr, 1u, 1u);
    if ((e = cudaGetLastError()) != cudaSuccess) {
        err = std::string("scan launch: ") + cudaGetErrorString(e);
        return 3;
    }
    u32 flags = 0;
    if ((e = cudaMemcpyAsync(&flags, errw, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        err = std::string("scan: ") + cudaGetErrorString(e);
        return 3;
    }
    if (flags & ERR_LOOKBACK_TIMEOUT) {
        err = "a decoupled look-back wait gave up";
        return 4;
    }
    return 0;
}

// ---- one-time kernel set-up (outside any stream capture) ---------------------------------------
int g_sm_count = 148;

void init_kernels(int device) {
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) == cudaSuccess && sms > 0)
        g_sm_count = sms;
    cudaFuncSetAttribute(k_radix_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (RS_WARPS + 1) * (1 << RS_MAX_BITS) * 4);
    cudaGetLastError();
}

// ---- round seeds (renderer.cpp:65) -------------------------------------------------------------
__global__ void k_next_seeds(u32 *state, u32 *seeds, u32 n) {
    u32 s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        Rng r{state[s]};
        seeds[s] = random_u32(&r);
        state[s] = r.state;
    }
}

void launch_next_seeds(u32 *state, u32 *seeds, u32 n, cudaStream_t st) {
    k_next_seeds<<<(n + 63) / 64, 64, 0, st>>>(state, seeds, n);
}

} // namespace phx
