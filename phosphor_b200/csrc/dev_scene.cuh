// dev_scene.cuh — per-scene device descriptor and closest-hit BVH traversal.
//
// BVH layout.  The host builds the reference's tree (median split, one triangle per leaf,
// depth-first flattening: src/renderer/bvh.cpp:18-84) and re-packs it for the device:
//  * inner nodes in pre-order, each a 64-byte "child pair" of four float4: both children's
//    boxes side by side so one node fetch (four coalesced 16-byte loads) tests both children;
//  * child references: >= 0 inner node index, < 0 ~leaf rank;
//  * triangles in leaf (pre-)order as 48-byte records {v0 | mat bits, v1-v0, v2-v0}, so the leaf
//    rank is also the triangle's device index and all per-triangle shading data is stored in
//    that order.
// Traversal visits the nearer child first and culls popped entries whose entry distance exceeds
// the current closest hit.  The reference's depth-first left-first order (hit.h:135-172) keeps
// the LAST tested triangle among hits at exactly equal t (`t > t_max` rejects, equality passes,
// hit.h:68); with left-first pre-order that is the equal-t hit with the largest leaf rank, so an
// equal-t candidate replaces the current hit only when its rank is larger.  Boxes are expanded by
// 1e-3 (bounding_box.h:30-37), so no box that holds the closest hit is ever culled by either
// order, and the result is the reference's hit for every ray.  The reference drops children when
// its 24-entry stack is full (hit.h:163-164), which only happens for trees deeper than 22 levels;
// the host reports the depth and this traversal counts (instead of silently dropping) overflows
// of its own 64-entry stack.
#pragma once

#include <type_traits>

#include "dev_common.cuh"

namespace phx {

struct __align__(16) SceneDesc {
    // geometry, device pointers
    const float4 *cnodes;   // inner nodes: 4 float4 per child pair, or 7 per 4-wide node
    const float4 *trirec;   // 3 float4 per triangle (leaf order)
    const float4 *tri_nrm;  // n0,n1,n2 per triangle (leaf order)
    const float4 *tri_tan;  // t0,t1,t2
    const float4 *tri_uv;   // (uv0.xy, uv1.xy), (uv2.xy, 0, 0)
    const float4 *etri_v;   // emissive triangles v0,v1,v2
    const float4 *etri_n;   // n0,n1,n2
    const float4 *etri_uv;  // 2 float4 per emissive triangle
    const u32 *etri_mat;
    const phx_material *materials;
    const phx_uv_transform_block *uvt;
    const phx_texture_meta *tex_meta;
    const u8 *tex_atlas;
    const phx_light *lights;
    const float *lum_pref_sum;
    const float *envmap;
    i32 root;       // root reference (>= 0 inner, < 0 ~leaf)
    u32 n_tris;
    u32 n_lights;
    float total_lum;
    float4 scene_center;
    float scene_radius;
    u32 env_w, env_h, has_env;
    phx_camera_params camera;
    // image and photon budget
    u32 width, height, n_pixels;
    u32 n_emit;           // photons emitted per round
    u32 max_bounces;
    u32 direct_samples;
    float alpha;
    u32 n_cells;          // grid_res^3 + 1
    GridDev grid;
    // bases in the engine's concatenated arrays
    u32 pixel_base;       // first pixel of this scene
    u32 emit_base;        // first photon path of this scene
    u32 cell_base;        // first cell of this scene
    u32 wide;             // 2: 4-wide nodes with 8-bit child boxes (4 uint4 each), 1: 4-wide nodes (7
                          // float4), 0: child pairs (4 float4)
    u64 slot_base;        // first photon slot of this scene (slot j of path t at slot_base + j*n_emit + t)
    u32 flags;
    u32 any_transmissive; // 0 -> shadow rays can stop at the first hit
    u32 nee_base;         // first deferred-NEE sample slot of this scene (pixel i, sample d at nee_base + i*ds + d)
    u32 active;           // 0: a batch scene that has been retired; every stage skips it
    u32 light_draws;      // RNG draws of one light sample when the same for every light, else LIGHT_DRAWS_VARY
};
constexpr u32 LIGHT_DRAWS_VARY = 0xffffffffu;

// scene of global index gid: bases[s] <= gid < bases[s+1] (n+1 prefix offsets)
PHX_DI u32 find_scene(const u32 *bases, u32 n, u32 gid) {
    u32 lo = 0, hi = n;
    while (hi - lo > 1) {
        u32 mid = (lo + hi) >> 1;
        if (__ldg(&bases[mid]) <= gid)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// ---- closest hit ------------------------------------------------------------------------------
struct Hit {
    float t, u, v;
    i32 tri; // device triangle index (leaf rank), -1 = none
};

#ifndef PHX_TRAV_STACK
#define PHX_TRAV_STACK 64
#endif
constexpr int TRAV_STACK = PHX_TRAV_STACK;
constexpr u32 LEAF_FIRST_BITS = 27; // leaf reference: ~(first | (count-1) << 27)

// Möller–Trumbore test of hit.h:45-78 with the reference's dot(float4) including w terms.
// ow, dw: w components of the ray origin and direction (always +-0 in practice).  The record's
// w lanes carry the material index (r0.w) and the reference leaf rank (r1.w); the test itself
// uses the reference's zero w components of the edge vectors.
PHX_DI bool tri_test(const float4 *rec, float ox, float oy, float oz, float ow, float dx, float dy, float dz, float dw,
                     float t_min, float t_max, float *tt, float *tu, float *tv, u32 *rank) {
    float4 r0 = __ldg(rec + 0), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2);
    *rank = __float_as_uint(r1.w);
    // e1 = r1.xyz, e2 = r2.xyz (precomputed v1-v0, v2-v0 with the same float subtraction)
    float hx = dy * r2.z - dz * r2.y;
    float hy = dz * r2.x - dx * r2.z;
    float hz = dx * r2.y - dy * r2.x;
    float a = ((r1.x * hx + r1.y * hy) + r1.z * hz) + 0.0f * 0.0f;
    if (fabsf(a) < EPS)
        return false;
    float sx = ox - r0.x, sy = oy - r0.y, sz = oz - r0.z, sw = ow - 0.0f;
    const float un = ((sx * hx + sy * hy) + sz * hz) + sw * 0.0f;
    // Division-free rejections, each implied by the exact test below (u = fl(un * fl(1/a)) carries
    // a relative error below 2^-22): |un| > 1.0001|a| gives |u| > 1, so u > 1 or u < 0; a sign
    // opposite to a's with |un| >= 2^-60|a| gives u < 0 (no underflow to -0).  NaNs fail every
    // comparison and fall through to the exact test.
    const float aa = fabsf(a), th = aa * 8.6736174e-19f; // 2^-60
    if (fabsf(un) > aa * 1.0001f || ((un > 0.0f) != (a > 0.0f) && fabsf(un) >= th))
        return false;
    float qx = sy * r1.z - sz * r1.y;
    float qy = sz * r1.x - sx * r1.z;
    float qz = sx * r1.y - sy * r1.x;
    const float vn = ((dx * qx + dy * qy) + dz * qz) + dw * 0.0f;
    // the same for v, and u + v > 1 when |un| + |vn| > 1.0001|a| with u, v >= 0
    if (fabsf(vn) > aa * 1.0001f || ((vn > 0.0f) != (a > 0.0f) && fabsf(vn) >= th) ||
        fabsf(un) + fabsf(vn) > aa * 1.0001f)
        return false;
    float f = 1.0f / a;
    float u = f * un;
    if (u < 0.0f || u > 1.0f)
        return false;
    float v = f * vn;
    if (v < 0.0f || u + v > 1.0f)
        return false;
    float t = f * (((r2.x * qx + r2.y * qy) + r2.z * qz) + 0.0f * 0.0f);
    if (t < t_min || t > t_max)
        return false;
    *tt = t;
    *tu = u;
    *tv = v;
    return true;
}

// Reference leaf rank of device triangle tri (the w lane of its second record).
PHX_DI i32 tri_rank(const SceneDesc &sc, i32 tri) { return __float_as_int(__ldg(&sc.trirec[3 * (size_t)tri + 1].w)); }

// u, v of the hit of (o, d) on triangle tri that tri_test accepted before: the same operations on
// the same inputs give the same values.
PHX_DI void hit_uv(const SceneDesc &sc, i32 tri, float4 o, float4 d, float *u, float *v) {
    float t;
    u32 rank;
    const float INF = __int_as_float(0x7f800000);
    tri_test(sc.trirec + 3 * (size_t)tri, o.x, o.y, o.z, o.w, d.x, d.y, d.z, d.w, -INF, INF, &t, u, v, &rank);
}

// Slab test of both children of a node.  Box tests only decide what is skipped, never which
// triangle is hit (boxes are expanded by 1e-3, far above rounding), so they use fused
// multiply-add t = box*inv - origin*inv: one instruction per plane.
PHX_DI void box2(const float4 &a, const float4 &b, const float4 &c, float ix, float iy, float iz, float oix, float oiy,
                 float oiz, float t_min, float t_max, float *tl, float *tr, bool *hl, bool *hr) {
    // left child: a = (minx, maxx, miny, maxy), c.xy = (minz, maxz); right: b, c.zw
    float lx0 = __fmaf_rn(a.x, ix, -oix), lx1 = __fmaf_rn(a.y, ix, -oix);
    float ly0 = __fmaf_rn(a.z, iy, -oiy), ly1 = __fmaf_rn(a.w, iy, -oiy);
    float lz0 = __fmaf_rn(c.x, iz, -oiz), lz1 = __fmaf_rn(c.y, iz, -oiz);
    float rx0 = __fmaf_rn(b.x, ix, -oix), rx1 = __fmaf_rn(b.y, ix, -oix);
    float ry0 = __fmaf_rn(b.z, iy, -oiy), ry1 = __fmaf_rn(b.w, iy, -oiy);
    float rz0 = __fmaf_rn(c.z, iz, -oiz), rz1 = __fmaf_rn(c.w, iz, -oiz);
    float lnear = fmaxf(fmaxf(fminf(lx0, lx1), fminf(ly0, ly1)), fmaxf(fminf(lz0, lz1), t_min));
    float lfar = fminf(fminf(fmaxf(lx0, lx1), fmaxf(ly0, ly1)), fminf(fmaxf(lz0, lz1), t_max));
    float rnear = fmaxf(fmaxf(fminf(rx0, rx1), fminf(ry0, ry1)), fmaxf(fminf(rz0, rz1), t_min));
    float rfar = fminf(fminf(fmaxf(rx0, rx1), fmaxf(ry0, ry1)), fminf(fmaxf(rz0, rz1), t_max));
    *tl = lnear;
    *tr = rnear;
    *hl = lnear <= lfar;
    *hr = rnear <= rfar;
}

// Slab test of one child of a 4-wide node, given per axis the plane the ray enters first (nx, ny,
// nz) and the one it leaves by (fx, fy, fz), picked once per ray from the sign of its direction;
// returns the entry distance, or +inf on a miss.  A slab whose distances are NaN (a zero direction
// component with the origin's inf products) is ignored by fmaxf / fminf: never pruned wrongly.
PHX_DI float box1(float nx, float fx, float ny, float fy, float nz, float fz, float ix, float iy, float iz,
                  float oix, float oiy, float oiz, float t_min, float t_max) {
    float tn = fmaxf(fmaxf(__fmaf_rn(nx, ix, -oix), __fmaf_rn(ny, iy, -oiy)), fmaxf(__fmaf_rn(nz, iz, -oiz), t_min));
    float tf = fminf(fminf(__fmaf_rn(fx, ix, -oix), __fmaf_rn(fy, iy, -oiy)), fminf(__fmaf_rn(fz, iz, -oiz), t_max));
    return tn <= tf ? tn : __int_as_float(0x7f800000);
}

// Byte k of w as a float: the byte under the exponent of 2^23, minus 2^23 (exact).
PHX_DI float qbyte(u32 w, int k) { return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440 + k)) - 8388608.0f; }

// Slab test of child k of an 8-bit node: per axis the entry and exit byte words (picked by the
// direction's sign), the distance of one quantisation step (s) and of the node origin (b); the plane
// of byte q lies at distance q * s + b.  Returns the entry distance, or +inf on a miss.
PHX_DI float qbox(u32 nxw, u32 fxw, u32 nyw, u32 fyw, u32 nzw, u32 fzw, int k, float sx, float sy, float sz, float bx,
                  float by, float bz, float t_min, float t_max) {
    const float tn = fmaxf(fmaxf(__fmaf_rn(qbyte(nxw, k), sx, bx), __fmaf_rn(qbyte(nyw, k), sy, by)),
                           fmaxf(__fmaf_rn(qbyte(nzw, k), sz, bz), t_min));
    const float tf = fminf(fminf(__fmaf_rn(qbyte(fxw, k), sx, bx), __fmaf_rn(qbyte(fyw, k), sy, by)),
                           fminf(__fmaf_rn(qbyte(fzw, k), sz, bz), t_max));
    return tn <= tf ? tn : __int_as_float(0x7f800000);
}

// The slab tests' inverse direction component 1/dc, except that the +-inf of a zero component
// becomes +-1e30 while the origin's coordinate oc is below 1e4 in magnitude.  A ray with dc = 0
// keeps the coordinate oc.  With +-inf, every plane on the same side of zero as oc gave
// inf - inf = NaN, which the slab tests ignore: that axis pruned nothing, and an axis-aligned ray
// visited most of the tree — 62,533 steps for one photon of the 1920x1080 atrium workload emitted
// straight down, direction (0, 0, -1), from its point light: 26-40 ms added to about one round in
// ten.  With 1e30 a slab's distances are (plane - oc) * 1e30 up to a rounding
// of |oc| * 2^-24 * 1e30, so their signs are exact for every plane farther than 6e-4 from oc, as
// is every plane of a box holding a triangle the ray can hit (triangle boxes are widened by 1e-3
// and the ray's coordinate must lie within the triangle's range).  A box that oc lies outside of
// gets two distances of one sign, at least ~1e27 in magnitude, and is pruned.  NaN and finite
// inverses are unchanged.
PHX_DI float slab_inv(float dc, float oc) {
    const float r = 1.0f / dc;
    return (fabsf(r) == __int_as_float(0x7f800000) && fabsf(oc) < 1e4f) ? copysignf(1e30f, r) : r;
}

// The hits of a ray on [t_min, t_max] that one traversal collects for a shadow ray crossing
// transmissive surfaces: the K first in the order of (t ascending, reference leaf rank descending)
// — the order in which closest-hit queries with a rising t_min return them.  Every hit with
// t <= bound and t < lost is listed: bound is the final culling distance (the K-th listed t once
// the list is full, or the nearest opaque hit), lost the smallest t of a hit that did not fit.
// The list keeps no barycentrics and no reference ranks (registers of the shadow kernel's hot
// loop): the one consumer that needs u, v (a textured transmissive crossing) recomputes them with
// hit_uv, and a rank is read back from the triangle records when two hits tie at exactly equal t.
// Shadow stage 7.25 -> 6.80 ms on the caustic workload.
template <int K> struct HitList {
    float t[K];
    i32 tri[K];
    int n;
    float lost, bound;
};
struct NoHitList {};
template <int K> constexpr int list_capacity(const HitList<K> *) { return K; }
constexpr int list_capacity(const NoHitList *) { return 0; }

template <int K>
PHX_DI void hit_list_insert(const SceneDesc &sc, HitList<K> &L, float t, i32 tri, i32 rank) {
    auto before = [&](int i) { return t < L.t[i] || (t == L.t[i] && rank > tri_rank(sc, L.tri[i])); };
    if (L.n == K) {
        if (!before(K - 1)) { // sorts after the whole list: dropped
            L.lost = fminf(L.lost, t);
            return;
        }
        L.lost = fminf(L.lost, L.t[K - 1]); // the last entry makes room
    }
    bool placed = false;
#pragma unroll
    for (int i = K - 1; i >= 0; i--) {
        if (placed)
            continue;
        if (i > 0 && i - 1 < L.n && before(i - 1)) { // shift the entry after the new hit
            L.t[i] = L.t[i - 1];
            L.tri[i] = L.tri[i - 1];
        } else if (i <= L.n) {
            L.t[i] = t;
            L.tri[i] = tri;
            placed = true;
        }
    }
    if (L.n < K)
        L.n++;
}

// Closest hit in [t_min, t_max] (scene_intersect, hit.h:135-172).  Returns false on a miss.
// `any` stops at the first accepted hit (only valid where the caller needs no specific hit).
// With a HitList (LIST), every accepted hit is offered to the list instead and the culling
// distance follows the list's bound; the return value is then meaningless.
//
// Warp-synchronous single-step loop: the lanes that call intersect together stay in lockstep,
// each iteration advancing every unfinished lane by exactly one node (an inner child pair or a
// leaf), so neighbouring rays share every node fetch and the warp never runs one lane's inner
// loop while the others wait.
// ORDERED: a 4-wide node's nearest hit child is visited first (the others in slot order);
// otherwise all in slot order.  The result never depends on the order (closest hit and tie rank,
// the hit list, or for `any` whether there is a hit); the order only decides how early far
// subtrees are culled.
template <class LIST, bool ORDERED = true>
PHX_DI bool intersect_t(const SceneDesc &sc, float4 o, float4 d, float t_min, float t_max, Hit *hit, u32 *overflow,
                        bool any, LIST *list) {
    constexpr bool LISTED = !std::is_same<LIST, NoHitList>::value;
    float opaque = t_max; // LISTED: nearest opaque hit so far
    constexpr i32 POP = 0x7fffffff;
    const float ix = slab_inv(d.x, o.x), iy = slab_inv(d.y, o.y), iz = slab_inv(d.z, o.z);
    const float oix = o.x * ix, oiy = o.y * iy, oiz = o.z * iz;
    // 4-wide nodes: offsets of the entry-plane rows {minx, maxx, miny, maxy, minz, maxz}
    const int px = ix >= 0.0f ? 0 : 1, py = iy >= 0.0f ? 2 : 3, pz = iz >= 0.0f ? 4 : 5;
    float closest = t_max;
    i32 best = -1, best_rank = -1;
    float bu = 0.0f, bv = 0.0f;
    i32 stack_ref[TRAV_STACK];
    float stack_t[TRAV_STACK];
    int sp = 0;
    i32 node = sc.root;
    bool done = false;
    const u32 mask = __activemask();
    while (__any_sync(mask, !done)) {
        if (done)
            continue;
        if (node >= 0 && sc.wide) { // 4-wide node: descend into the nearest hit child, stack the rest
            const float NOHIT = __int_as_float(0x7f800000);
            float t0, t1, t2, t3;
            int4 ch;
            if (sc.wide == 2) { // 8-bit child boxes (bvh_quant.hpp)
                const uint4 *qn = reinterpret_cast<const uint4 *>(sc.cnodes) + 4 * (size_t)node;
                const uint4 h = __ldg(qn), qx = __ldg(qn + 1), qz = __ldg(qn + 2);
                ch = __ldg(reinterpret_cast<const int4 *>(qn + 3));
                // per axis: distance of the origin plane and of one step; entry / exit bytes by sign
                const float sx = __uint_as_float((h.w & 0xffu) << 23) * ix;
                const float sy = __uint_as_float(((h.w >> 8) & 0xffu) << 23) * iy;
                const float sz = __uint_as_float(((h.w >> 16) & 0xffu) << 23) * iz;
                const float bx = __fmaf_rn(__uint_as_float(h.x), ix, -oix);
                const float by = __fmaf_rn(__uint_as_float(h.y), iy, -oiy);
                const float bz = __fmaf_rn(__uint_as_float(h.z), iz, -oiz);
                const u32 nxw = px == 0 ? qx.x : qx.y, fxw = px == 0 ? qx.y : qx.x;
                const u32 nyw = py == 2 ? qx.z : qx.w, fyw = py == 2 ? qx.w : qx.z;
                const u32 nzw = pz == 4 ? qz.x : qz.y, fzw = pz == 4 ? qz.y : qz.x;
                t0 = ch.x == POP ? NOHIT : qbox(nxw, fxw, nyw, fyw, nzw, fzw, 0, sx, sy, sz, bx, by, bz, t_min, closest);
                t1 = ch.y == POP ? NOHIT : qbox(nxw, fxw, nyw, fyw, nzw, fzw, 1, sx, sy, sz, bx, by, bz, t_min, closest);
                t2 = ch.z == POP ? NOHIT : qbox(nxw, fxw, nyw, fyw, nzw, fzw, 2, sx, sy, sz, bx, by, bz, t_min, closest);
                t3 = ch.w == POP ? NOHIT : qbox(nxw, fxw, nyw, fyw, nzw, fzw, 3, sx, sy, sz, bx, by, bz, t_min, closest);
            } else {
                const float4 *wn = sc.cnodes + 7 * (size_t)node;
                const float4 mnx = __ldg(wn + px), mxx = __ldg(wn + (1 - px)), mny = __ldg(wn + py);
                const float4 mxy = __ldg(wn + (5 - py)), mnz = __ldg(wn + pz), mxz = __ldg(wn + (9 - pz));
                ch = __ldg(reinterpret_cast<const int4 *>(wn + 6));
                // (mnx.. now hold the entry planes, mxx.. the exit planes.)
                // Empty slots carry the box (1e30, -1e30), which no ray with a finite inverse
                // direction component enters (a NaN slab is ignored, and not all three can be NaN);
                // their reference is still checked where a child is stacked, and descending into it
                // pops the next entry, so it is never used as a node index.  Testing the reference
                // here instead measured 4 % slower in the shadow and photon kernels.
                t0 = box1(mnx.x, mxx.x, mny.x, mxy.x, mnz.x, mxz.x, ix, iy, iz, oix, oiy, oiz, t_min, closest);
                t1 = box1(mnx.y, mxx.y, mny.y, mxy.y, mnz.y, mxz.y, ix, iy, iz, oix, oiy, oiz, t_min, closest);
                t2 = box1(mnx.z, mxx.z, mny.z, mxy.z, mnz.z, mxz.z, ix, iy, iz, oix, oiy, oiz, t_min, closest);
                t3 = box1(mnx.w, mxx.w, mny.w, mxy.w, mnz.w, mxz.w, ix, iy, iz, oix, oiy, oiz, t_min, closest);
            }
            i32 r0 = ch.x, r1 = ch.y, r2 = ch.z, r3 = ch.w;
            if constexpr (!ORDERED) {
                // slot order: descend into the first hit child, stack the other hit ones
                const float ts[4] = {t0, t1, t2, t3};
                const i32 rs[4] = {r0, r1, r2, r3};
                i32 nxt = POP;
                float tn = NOHIT;
#pragma unroll
                for (int c = 3; c >= 0; c--) {
                    if (ts[c] == NOHIT || rs[c] == POP)
                        continue;
                    if (nxt != POP) {
                        if (sp < TRAV_STACK) {
                            stack_ref[sp] = nxt;
                            stack_t[sp] = tn;
                            sp++;
                        } else {
                            *overflow += 1;
                        }
                    }
                    nxt = rs[c];
                    tn = ts[c];
                }
                node = nxt;
            } else {
                // the nearest hit child first; the others stacked in slot order.  A full sort of the
                // four (stacked farthest first) culled little more and cost more instructions: shadow
                // stage 6.22 -> 6.09 ms, photon kernel 3.86 -> 3.74 ms on the caustic workload.
                float tm = t0;
                i32 rm = r0;
                if (t1 < tm) { tm = t1; rm = r1; }
                if (t2 < tm) { tm = t2; rm = r2; }
                if (t3 < tm) { tm = t3; rm = r3; }
                const float ts[4] = {t3, t2, t1, t0};
                const i32 rs[4] = {r3, r2, r1, r0};
                node = tm == NOHIT ? POP : rm;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    if (ts[k] == NOHIT || rs[k] == POP || rs[k] == rm)
                        continue;
                    if (sp < TRAV_STACK) {
                        stack_ref[sp] = rs[k];
                        stack_t[sp] = ts[k];
                        sp++;
                    } else {
                        *overflow += 1;
                    }
                }
            }
        } else if (node >= 0) { // child pair: test both children, descend into the nearer hit one
            const float4 *cn = sc.cnodes + 4 * (size_t)node;
            float4 a = __ldg(cn + 0), b = __ldg(cn + 1), c = __ldg(cn + 2);
            int4 ch = __ldg(reinterpret_cast<const int4 *>(cn + 3));
            float tl, tr;
            bool hl, hr;
            box2(a, b, c, ix, iy, iz, oix, oiy, oiz, t_min, closest, &tl, &tr, &hl, &hr);
            if (hl && hr) {
                i32 nearr = ch.x, farr = ch.y;
                float tfar = tr;
                if (tr < tl) {
                    nearr = ch.y;
                    farr = ch.x;
                    tfar = tl;
                }
                if (sp < TRAV_STACK) {
                    stack_ref[sp] = farr;
                    stack_t[sp] = tfar;
                    sp++;
                } else {
                    *overflow += 1;
                }
                node = nearr;
            } else {
                node = hl ? ch.x : (hr ? ch.y : POP);
            }
        } else { // leaf: triangles [first, first + count)
            const u32 enc = (u32)~node;
            const u32 first = enc & ((1u << LEAF_FIRST_BITS) - 1u);
            const u32 count = (enc >> LEAF_FIRST_BITS) + 1u;
            for (u32 k = 0; k < count; k++) {
                float t, u, v;
                u32 rank;
                if (tri_test(sc.trirec + 3 * (size_t)(first + k), o.x, o.y, o.z, o.w, d.x, d.y, d.z, d.w, t_min,
                             closest, &t, &u, &v, &rank)) {
                    if constexpr (LISTED) {
                        hit_list_insert(sc, *list, t, (i32)(first + k), (i32)rank);
                        const u32 mi = __float_as_uint(__ldg(&sc.trirec[3 * (size_t)(first + k)].w));
                        if (sc.materials[mi].transmission < EPS)
                            opaque = fminf(opaque, t); // nothing beyond it can be reached
                        closest = fminf(list->n == list_capacity(list) ? list->t[list_capacity(list) - 1] : t_max,
                                        opaque);
                        continue;
                    }
                    // t <= closest here; at equal t the reference keeps the larger leaf rank
                    if (t < closest || (i32)rank > best_rank) {
                        closest = t;
                        best = (i32)(first + k);
                        best_rank = (i32)rank;
                        bu = u;
                        bv = v;
                        if (any)
                            done = true;
                    }
                }
            }
            node = POP;
        }
        if (node == POP && !done) { // pop the next entry that can still hold a hit
            done = true;
            while (sp > 0) {
                sp--;
                if (stack_t[sp] <= closest) {
                    node = stack_ref[sp];
                    done = false;
                    break;
                }
            }
        }
    }
    if constexpr (LISTED) {
        list->bound = closest;
        return false;
    }
    hit->t = closest;
    hit->u = bu;
    hit->v = bv;
    hit->tri = best;
    return best >= 0;
}

PHX_DI bool intersect(const SceneDesc &sc, float4 o, float4 d, float t_min, float t_max, Hit *hit, u32 *overflow,
                      bool any = false) {
    return intersect_t<NoHitList>(sc, o, d, t_min, t_max, hit, overflow, any, nullptr);
}

// Shadow kernels: general (each scene's materials decide at run time between the listing traversal
// with its walk and the walk's any-hit query), for contexts whose scenes have no transmissive
// material (a single any-hit query in slot order, and nothing else compiled in), or general for
// contexts with no texture at all (SHADOW_CLEAR: the textured crossing compiled out, which frees
// most of the general kernel's spills).
enum : int { SHADOW_GENERAL = 0, SHADOW_OPAQUE = 1, SHADOW_CLEAR = 2 };

// Any-hit query of a shadow ray in a scene where no material transmits.  It visits a 4-wide node's
// children in slot order: an unoccluded ray visits every box on its segment whatever the order,
// and the nearest-first sort only costs it instructions (shadow stage 3.61 -> 3.21 ms on the
// atrium workload).  Closest-hit and listing queries keep the order, which culls behind a hit.
PHX_DI bool occluded(const SceneDesc &sc, float4 o, float4 d, float t_min, float t_max, u32 *overflow) {
    Hit h;
    return intersect_t<NoHitList, false>(sc, o, d, t_min, t_max, &h, overflow, true, nullptr);
}

// Collects the hits of (o, d) on [t_min, t_max] into L (see HitList).
template <int K>
PHX_DI void intersect_list(const SceneDesc &sc, float4 o, float4 d, float t_min, float t_max, HitList<K> *L,
                           u32 *overflow) {
    L->n = 0;
    L->lost = __int_as_float(0x7f800000);
    L->bound = t_max;
    Hit unused;
    intersect_t<HitList<K>>(sc, o, d, t_min, t_max, &unused, overflow, false, L); // nearest first: culls behind the list
}

} // namespace phx
