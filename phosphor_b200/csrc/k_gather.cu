// k_gather.cu — per-pixel photon gather with the SPPM radius/flux update
// (kernels/gather_flux.cl:5-78, gather_photon_flux in include/common/photon_hash.h:56-103), and
// the image formation of src/renderer/output.cpp:40-83.
//
// Photons are read in cell order from the sorted records {x, y, z, octahedral dir bits} (16 B, one
// load answers the radius test); the direction and power, decoded once per round when the records
// are written, are only loaded for photons inside the radius.  Each pixel accumulates its 27 cells in the
// reference's cell order and each cell in sorted (= canonical) order, in one thread with no float
// atomics, so the sum is deterministic and equal to the reference's sequential sum.  cell_end is
// not materialised: the cells are contiguous, so end(h) = start(h+1).
#include "kernels.hpp"

// Photon records loaded ahead per step of a cell's loop (4: gather 2.40 -> 2.30 ms on the caustic
// workload, 3.93 -> 3.56 ms on the atrium one, against 2).
#ifndef PHX_GATHER_AHEAD
#define PHX_GATHER_AHEAD 4
#endif

// Each cell's photon range loaded while the previous cell's photons are summed (1), or after
// (0: one more dependent load round trip per searched cell).
#ifndef PHX_GATHER_NEXT_CELL
#define PHX_GATHER_NEXT_CELL 1
#endif

namespace phx {

PHX_DI void gather_pixel(const SceneDesc &sc, u32 gpix, const GatherBufs &g) {
    float4 ge = g.hp_emission[gpix];
    float4 rso = g.radiance[gpix];
    float4 r = f4(ge.x, ge.y, ge.z, 0.0f);
    if (ge.w == 0.0f) {
        g.radiance[gpix] = rso + r;
        if (g.rec_r2) {
            g.rec_r2[gpix] = 0.0f;
            g.rec_ratio[gpix] = 1.0f;
        }
        return;
    }
    float4 direct = g.hp_direct[gpix];
    r.x += direct.x;
    r.y += direct.y;
    r.z += direct.z;
    g.radiance[gpix] = rso + r;
    float4 fso = g.flux[gpix];
    float wso = g.weight[gpix];
    const GridDev grid = sc.grid;
    float r_sq = fso.w;
    if (r_sq < EPS) {
        float hx = grid.cx * 0.5f, hy = grid.cy * 0.5f, hz = grid.cz * 0.5f;
        r_sq = hx * hx + hy * hy + hz * hz;
    }
    const float4 pos = g.hp_pos[gpix];
    const float4 nrm = g.hp_normal[gpix];
    float4 nf = zero4();
    float found = 0.0f;
    const u32 *cs = g.cell_start + sc.cell_base;
    const float denom = 2.0f * r_sq;
    // hit point in cell units, for the cell-distance test below
    const float qx = (pos.x - grid.ox) / grid.cx, qy = (pos.y - grid.oy) / grid.cy, qz = (pos.z - grid.oz) / grid.cz;
    const u32 G = grid.g;
    // One photon's contribution, in the reference's arithmetic (photon_hash.h:84-101).
    auto add = [&](const float4 p, u32 k) {
        const float dx = pos.x - p.x, dy = pos.y - p.y, dz = pos.z - p.z, dw = pos.w - 0.0f;
        const float dsq = ((dx * dx + dy * dy) + dz * dz) + dw * dw;
        if (dsq < r_sq) {
            const float4 pd = __ldg(&g.s_dir[k]); // decode_oct(p.w), decoded once per round
            if (!(dot(pd, nrm) > 0.0f)) {
                const float w = GAUSS_ALPHA * (1.0f - (1.0f - pm_expf((-GAUSS_BETA) * dsq / denom)) / GAUSS_DENOM);
                nf += w * __ldg(&g.s_pow[k]); // decode_rgbe(s_power[k])
                found += w;
            }
        }
    };
    // The 27 cells in the reference's order (photon_hash.h:65-82), each in sorted (canonical)
    // photon order.  A cell whose box lies farther than the search radius from the hit point holds
    // no photon with dsq < r_sq, so it adds nothing and is skipped; the box is widened by 1/1024
    // of a cell on every side so that rounding in get_hash (which decides a photon's cell) and in
    // this test can never skip a photon that would count.
    constexpr float M = 1.0f / 1024.0f;
    // cell hash of neighbour offset i (0 outside the grid), and whether its box can hold a photon
    // within the radius
    // get_hash of a neighbour position works axis by axis, and an axis's coordinate only takes the
    // three values pos + {-1, 0, 1} * cell: each axis's three cell coordinates are computed once,
    // with the same operations get_hash applies (0xff: outside the grid, which has at most 255
    // cells per axis), and packed one byte per offset.
    const float gf = (float)G;
    auto axis_cells = [&](float p, float o, float c) -> u32 {
        u32 w = 0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float q = p;
            q += (float)(k - 1) * c;
            const float f = (q - o) / c;
            const u32 ci = (f < 0.0f || f >= gf) ? 0xffu : (u32)f;
            w |= ci << (8 * k);
        }
        return w;
    };
    const u32 wx = axis_cells(pos.x, grid.ox, grid.cx), wy = axis_cells(pos.y, grid.oy, grid.cy),
              wz = axis_cells(pos.z, grid.oz, grid.cz);
    auto cell_of = [&](u32 i, bool *near) -> u32 {
        const u32 hx = (wx >> (8 * (i % 3))) & 0xffu;
        const u32 hy = (wy >> (8 * ((i / 3) % 3))) & 0xffu;
        const u32 hz = (wz >> (8 * ((i / 9) % 3))) & 0xffu;
        if (hx == 0xffu || hy == 0xffu || hz == 0xffu) {
            *near = false;
            return 0;
        }
        const u32 h = G * G * hx + G * hy + hz + 1; // get_hash's cell index
        const float gx = fmaxf(fmaxf(((float)hx - M) - qx, qx - ((float)hx + (1.0f + M))), 0.0f) * grid.cx;
        const float gy = fmaxf(fmaxf(((float)hy - M) - qy, qy - ((float)hy + (1.0f + M))), 0.0f) * grid.cy;
        const float gz = fmaxf(fmaxf(((float)hz - M) - qz, qz - ((float)hz + (1.0f + M))), 0.0f) * grid.cz;
        *near = !((gx * gx + gy * gy) + gz * gz > r_sq);
        return h;
    };
    auto cell_photons = [&](u32 k, const u32 end) {
        // PHX_GATHER_AHEAD records in flight per step; contributions still added in photon order
#if PHX_GATHER_AHEAD == 4
        for (; k + 3 < end; k += 4) {
            const float4 p0 = __ldg(&g.s_posdir[k]);
            const float4 p1 = __ldg(&g.s_posdir[k + 1]);
            const float4 p2 = __ldg(&g.s_posdir[k + 2]);
            const float4 p3 = __ldg(&g.s_posdir[k + 3]);
            add(p0, k);
            add(p1, k + 1);
            add(p2, k + 2);
            add(p3, k + 3);
        }
#endif
        for (; k + 1 < end; k += 2) {
            const float4 p0 = __ldg(&g.s_posdir[k]);
            const float4 p1 = __ldg(&g.s_posdir[k + 1]);
            add(p0, k);
            add(p1, k + 1);
        }
        if (k < end)
            add(__ldg(&g.s_posdir[k]), k);
    };
#if PHX_GATHER_NEXT_CELL
    // Each cell's photon range is loaded while the previous cell's photons are summed: the scan for
    // the next cell to search (each neighbour's hash computed once, as before) runs ahead by one.
    auto next_cell = [&](u32 from, u32 *h) -> u32 {
        for (u32 c = from; c < 27; c++) {
            bool near;
            *h = cell_of(c, &near);
            if (near)
                return c;
        }
        return 27u;
    };
    u32 h = 0;
    u32 i = next_cell(0, &h);
    u32 k0 = 0, k1 = 0;
    if (i < 27) {
        k0 = __ldg(&cs[h]);
        k1 = __ldg(&cs[h + 1]);
    }
    while (i < 27) {
        u32 hn = 0, n0 = 0, n1 = 0;
        const u32 j = next_cell(i + 1, &hn);
        if (j < 27) {
            n0 = __ldg(&cs[hn]);
            n1 = __ldg(&cs[hn + 1]);
        }
        cell_photons(min(k0, g.n_cap), min(k1, g.n_cap));
        i = j;
        k0 = n0;
        k1 = n1;
    }
#else
    for (u32 i = 0; i < 27; i++) {
        bool near;
        const u32 h = cell_of(i, &near);
        if (!near)
            continue;
        cell_photons(min(__ldg(&cs[h]), g.n_cap), min(__ldg(&cs[h + 1]), g.n_cap));
    }
#endif
    if (g.rec_r2) {
        g.rec_r2[gpix] = r_sq;
        g.rec_ratio[gpix] = found > 0.0f ? (wso + sc.alpha * found) / (wso + found) : 1.0f;
    }
    if (found > 0.0f) {
        float nw = wso + sc.alpha * found;
        float ratio = nw / (wso + found);
        float nr = r_sq * ratio;
        float4 albedo = g.hp_base_color[gpix];
        float4 contribution = g.hp_throughput[gpix] * (albedo / PI) * nf;
        float4 temp = (fso + contribution) * ratio;
        g.flux[gpix] = f4(temp.x, temp.y, temp.z, nr);
        g.weight[gpix] = nw;
    }
}

// 12 resident blocks per SM (42 registers, ~100 bytes of spills): the photon loop is latency-bound
// and more warps hide it better (7.3 -> 6.4 ms; 16 blocks spill more and measured slower).
#ifndef PHX_GATHER_MINB
#define PHX_GATHER_MINB 12
#endif
__global__ void __launch_bounds__(128, PHX_GATHER_MINB) k_gather(LaunchCtx lc, GatherBufs g) {
    u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.total_pixels)
        return;
    if (g.order)
        gid = __ldg(&g.order[gid]);
    u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
    if (lc.scenes[s].active)
        gather_pixel(lc.scenes[s], gid, g);
}

// Cooperative form of the same gather.  The pixels arrive grouped by photon-grid cell (k_pixel_keys),
// so the lanes of a warp mostly need the same cells.  For each of the 27 neighbour offsets the warp
// forms groups of lanes that need the same (global) cell; for each group all 32 lanes load the
// cell's photon records 32 at a time — one coalesced 16-byte load per lane per record array — into
// the warp's shared-memory stage, and the lanes of the group walk the staged records in order.  A
// pixel still sums its cells in the reference's order and each cell in sorted (canonical) order
// with the same operations, so its result is the per-thread kernel's bit for bit; what changes is
// that one load round trip now serves 32 records instead of one.
constexpr u32 COOP_WARPS = 4;
#ifndef PHX_GATHER_STAGE_ALL
#define PHX_GATHER_STAGE_ALL 1 // stage the decoded direction and power too (else load them per lane)
#endif

__global__ void __launch_bounds__(32 * COOP_WARPS, PHX_GATHER_MINB) k_gather_coop(LaunchCtx lc, GatherBufs g) {
    __shared__ float4 st_pd[COOP_WARPS][32];
#if PHX_GATHER_STAGE_ALL
    __shared__ float4 st_dir[COOP_WARPS][32];
    __shared__ float4 st_pow[COOP_WARPS][32];
#endif
    constexpr u32 FULL = 0xffffffffu, NONE = 0xffffffffu;
    const u32 lane = threadIdx.x & 31u, wq = threadIdx.x >> 5;
    const u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    const SceneDesc *scp = nullptr;
    u32 gpix = 0;
    bool gathering = false;
    float4 pos = zero4(), nrm = zero4(), fso = zero4(), nf = zero4();
    float wso = 0.0f, r_sq = 0.0f, found = 0.0f, denom = 1.0f, qx = 0.0f, qy = 0.0f, qz = 0.0f;
    if (gid < lc.total_pixels) {
        gpix = g.order ? __ldg(&g.order[gid]) : gid;
        const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gpix);
        scp = &lc.scenes[s];
        if (scp->active) {
            const float4 ge = g.hp_emission[gpix];
            const float4 rso = g.radiance[gpix];
            float4 r = f4(ge.x, ge.y, ge.z, 0.0f);
            if (ge.w == 0.0f) {
                g.radiance[gpix] = rso + r;
                if (g.rec_r2) {
                    g.rec_r2[gpix] = 0.0f;
                    g.rec_ratio[gpix] = 1.0f;
                }
            } else {
                const float4 direct = g.hp_direct[gpix];
                r.x += direct.x;
                r.y += direct.y;
                r.z += direct.z;
                g.radiance[gpix] = rso + r;
                fso = g.flux[gpix];
                wso = g.weight[gpix];
                const GridDev &grid = scp->grid;
                r_sq = fso.w;
                if (r_sq < EPS) {
                    float hx = grid.cx * 0.5f, hy = grid.cy * 0.5f, hz = grid.cz * 0.5f;
                    r_sq = hx * hx + hy * hy + hz * hz;
                }
                pos = g.hp_pos[gpix];
                nrm = g.hp_normal[gpix];
                denom = 2.0f * r_sq;
                qx = (pos.x - grid.ox) / grid.cx;
                qy = (pos.y - grid.oy) / grid.cy;
                qz = (pos.z - grid.oz) / grid.cz;
                gathering = true;
            }
        }
    }
    constexpr float M = 1.0f / 1024.0f;
    for (u32 i = 0; i < 27; i++) {
        u32 key = NONE;
        if (gathering) { // the per-thread kernel's cell and cell-distance tests
            const GridDev &grid = scp->grid;
            const i32 ox = (i32)(i % 3) - 1;
            const i32 oy = (i32)((i / 3) % 3) - 1;
            const i32 oz = (i32)((i / 9) % 3) - 1;
            float px = pos.x, py = pos.y, pz = pos.z;
            px += (float)ox * grid.cx;
            py += (float)oy * grid.cy;
            pz += (float)oz * grid.cz;
            const u32 h = get_hash(px, py, pz, grid);
            if (h != 0) {
                const u32 G = grid.g;
                const u32 hz = (h - 1) % G, hy = ((h - 1) / G) % G, hx = (h - 1) / (G * G);
                const float gx = fmaxf(fmaxf(((float)hx - M) - qx, qx - ((float)hx + (1.0f + M))), 0.0f) * grid.cx;
                const float gy = fmaxf(fmaxf(((float)hy - M) - qy, qy - ((float)hy + (1.0f + M))), 0.0f) * grid.cy;
                const float gz = fmaxf(fmaxf(((float)hz - M) - qz, qz - ((float)hz + (1.0f + M))), 0.0f) * grid.cz;
                if (!((gx * gx + gy * gy) + gz * gz > r_sq))
                    key = scp->cell_base + h;
            }
        }
        u32 pending = __ballot_sync(FULL, key != NONE);
        while (pending) {
            const u32 cell = __shfl_sync(FULL, key, __ffs(pending) - 1);
            const u32 grp = __ballot_sync(FULL, key == cell);
            pending &= ~grp;
            const bool mine = (grp >> lane) & 1u;
            const u32 start = min(__ldg(&g.cell_start[cell]), g.n_cap);
            const u32 end = min(__ldg(&g.cell_start[cell + 1]), g.n_cap);
            for (u32 base = start; base < end; base += 32) {
                const u32 k = base + lane;
                if (k < end) {
                    st_pd[wq][lane] = __ldg(&g.s_posdir[k]);
#if PHX_GATHER_STAGE_ALL
                    st_dir[wq][lane] = __ldg(&g.s_dir[k]);
                    st_pow[wq][lane] = __ldg(&g.s_pow[k]);
#endif
                }
                __syncwarp();
                if (mine) {
                    const u32 n = min(32u, end - base);
                    for (u32 j = 0; j < n; j++) { // one photon (photon_hash.h:84-101), in sorted order
                        const float4 p = st_pd[wq][j];
                        const float dx = pos.x - p.x, dy = pos.y - p.y, dz = pos.z - p.z, dw = pos.w - 0.0f;
                        const float dsq = ((dx * dx + dy * dy) + dz * dz) + dw * dw;
                        if (dsq < r_sq) {
#if PHX_GATHER_STAGE_ALL
                            const float4 pd = st_dir[wq][j];
#else
                            const float4 pd = __ldg(&g.s_dir[base + j]);
#endif
                            if (!(dot(pd, nrm) > 0.0f)) {
                                const float w =
                                    GAUSS_ALPHA * (1.0f - (1.0f - pm_expf((-GAUSS_BETA) * dsq / denom)) / GAUSS_DENOM);
#if PHX_GATHER_STAGE_ALL
                                nf += w * st_pow[wq][j];
#else
                                nf += w * __ldg(&g.s_pow[base + j]);
#endif
                                found += w;
                            }
                        }
                    }
                }
                __syncwarp();
            }
        }
    }
    if (!gathering)
        return;
    if (g.rec_r2) {
        g.rec_r2[gpix] = r_sq;
        g.rec_ratio[gpix] = found > 0.0f ? (wso + scp->alpha * found) / (wso + found) : 1.0f;
    }
    if (found > 0.0f) {
        float nw = wso + scp->alpha * found;
        float ratio = nw / (wso + found);
        float nr = r_sq * ratio;
        float4 albedo = g.hp_base_color[gpix];
        float4 contribution = g.hp_throughput[gpix] * (albedo / PI) * nf;
        float4 temp = (fso + contribution) * ratio;
        g.flux[gpix] = f4(temp.x, temp.y, temp.z, nr);
        g.weight[gpix] = nw;
    }
}

// Pixels whose hit points share a photon-grid cell (and an octant of it) visit the same cells and
// skip the same ones, so gathering them in one warp keeps its lanes in step and lets them share
// every photon record load.  Pixels without a diffuse hit point (nothing to gather) sort last.
// Each pixel's own computation does not change.
__global__ void __launch_bounds__(256) k_pixel_keys(LaunchCtx lc, const float4 *hp_pos, const float4 *hp_emission,
                                                    u32 key_bits, u32 *keys) {
    const u32 gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= lc.total_pixels)
        return;
    u32 key = key_bits >= 32 ? 0xffffffffu : (1u << key_bits) - 1u;
    if (hp_emission[gid].w == 1.0f) {
        key = 0; // outside the grid
        const u32 s = lc.n_scenes == 1 ? 0 : find_scene(lc.pix_bases, lc.n_scenes, gid);
        const SceneDesc &sc = lc.scenes[s];
        const float4 p = hp_pos[gid];
        const u32 h = get_hash(p.x, p.y, p.z, sc.grid);
        if (h) {
            const GridDev &gd = sc.grid;
            const float fx = (p.x - gd.ox) / gd.cx, fy = (p.y - gd.oy) / gd.cy, fz = (p.z - gd.oz) / gd.cz;
            const u32 oct = (fx - floorf(fx) >= 0.5f ? 1u : 0u) | (fy - floorf(fy) >= 0.5f ? 2u : 0u) |
                            (fz - floorf(fz) >= 0.5f ? 4u : 0u);
            key = ((sc.cell_base + h) << 3) | oct;
        }
    }
    keys[gid] = key;
}

void launch_pixel_keys(const LaunchCtx &lc, const float4 *hp_pos, const float4 *hp_emission, u32 key_bits, u32 *keys,
                       cudaStream_t st) {
    if (lc.total_pixels)
        k_pixel_keys<<<(lc.total_pixels + 255) / 256, 256, 0, st>>>(lc, hp_pos, hp_emission, key_bits, keys);
}

void launch_gather(const LaunchCtx &lc, const GatherBufs &g, int block, bool coop, cudaStream_t st) {
    if (lc.total_pixels == 0)
        return;
    (void)block;
    if (coop)
        k_gather_coop<<<(lc.total_pixels + 32 * COOP_WARPS - 1) / (32 * COOP_WARPS), 32 * COOP_WARPS, 0, st>>>(lc, g);
    else
        k_gather<<<(lc.total_pixels + 127) / 128, 128, 0, st>>>(lc, g);
}

// output.cpp:40-50 tone_map and :52-83 apply_tonemap, before/after u8 quantisation
__global__ void k_image(const float4 *flux, const float4 *radiance, u32 n, float exposure, int tonemap,
                        float inv_photons, float inv_rounds, float *rgb, uint8_t *ldr) {
    u32 p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n)
        return;
    float4 f = flux[p], rad = radiance[p];
    float area = PI * f.w;
    float ir = 0.0f, ig = 0.0f, ib = 0.0f;
    if (area > 0.0f) {
        float per = inv_photons / area;
        ir = f.x * per;
        ig = f.y * per;
        ib = f.z * per;
    }
    float c[3] = {rad.x * inv_rounds + ir, rad.y * inv_rounds + ig, rad.z * inv_rounds + ib};
    for (int k = 0; k < 3; k++) {
        float x = c[k] * exposure;
        float out = x;
        if (tonemap)
            out = (x * (2.51f * x + 0.03f)) / (x * (2.43f * x + 0.59f) + 0.14f);
        out = pm_powf(out, 1.0f / 2.2f);
        out = clampf(out, 0.0f, 1.0f);
        if (rgb)
            rgb[(size_t)p * 3 + k] = out;
        if (ldr)
            ldr[(size_t)p * 3 + k] = (uint8_t)(out * 255.0f);
    }
}

void launch_image(const float4 *flux, const float4 *radiance, u32 n, float exposure, int tonemap, float inv_photons,
                  float inv_rounds, float *rgb, uint8_t *ldr, cudaStream_t st) {
    if (n == 0)
        return;
    k_image<<<(n + 255) / 256, 256, 0, st>>>(flux, radiance, n, exposure, tonemap, inv_photons, inv_rounds, rgb, ldr);
}

} // namespace phx
