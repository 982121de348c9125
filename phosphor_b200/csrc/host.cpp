// host.cpp — BVH construction and packing, photon-grid box and scene sphere.
#include "host.hpp"
#include "bvh_quant.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>

namespace phx {

namespace {

constexpr float BBOX_EPS = 1e-3f;
constexpr float INF = 1e9f;
constexpr float MIN_CELL_SIZE = 0.001f;
constexpr float PI = 3.141592654f;

inline uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}
inline float u2f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

struct Box {
    float lo[3], hi[3];
};

// get_bounding_box (bounding_box.h:48-61)
bool triangle_box(const phx_triangle &t, Box &b) {
    for (int i = 0; i < 3; i++) {
        b.lo[i] = INF;
        b.hi[i] = -INF;
    }
    const phx_f4 *v[3] = {&t.v0, &t.v1, &t.v2};
    for (int k = 0; k < 3; k++) {
        const float c[3] = {v[k]->x, v[k]->y, v[k]->z};
        for (int i = 0; i < 3; i++) {
            b.lo[i] = std::min(b.lo[i], c[i]);
            b.hi[i] = std::max(b.hi[i], c[i]);
        }
    }
    for (int i = 0; i < 3; i++)
        if (b.lo[i] >= INF || b.lo[i] <= -INF || b.hi[i] >= INF || b.hi[i] <= -INF)
            return false;
    for (int i = 0; i < 3; i++) {
        b.lo[i] -= BBOX_EPS;
        b.hi[i] += BBOX_EPS;
    }
    for (int i = 0; i < 3; i++)
        if (b.lo[i] == b.hi[i])
            return false;
    return true;
}

// build_tmp + flatten (bvh.cpp:18-72) in one pass: one triangle per leaf, median split of the
// longest axis of the node box on the triangle boxes' minimum corner, written straight into the
// flattened pre-order array.  A subtree over m triangles takes 2m-1 slots, so a node at slot p has
// its left child at p+1 and its right child at p + 2*(mid-start): disjoint subtrees are written by
// independent threads.  Each range is sorted exactly as the sequential build sorts it (same
// comparator, same input order), so the nodes do not depend on the threading.
struct Builder {
    const std::vector<Box> &boxes;
    std::vector<uint32_t> order;
    phx_bvh_node *out;

    Builder(const std::vector<Box> &b, phx_bvh_node *o) : boxes(b), order(b.size()), out(o) {
        std::iota(order.begin(), order.end(), 0u);
    }

    void build(uint32_t start, uint32_t end, uint32_t pos, int spawn_depth) {
        phx_bvh_node &nd = out[pos];
        if (end == start + 1) {
            const Box &bx = boxes[order[start]];
            nd.min = {bx.lo[0], bx.lo[1], bx.lo[2], u2f(order[start])};
            nd.max = {bx.hi[0], bx.hi[1], bx.hi[2], u2f(0u)};
            return;
        }
        Box nb = boxes[order[start]];
        for (uint32_t i = start + 1; i < end; i++) {
            const Box &o = boxes[order[i]];
            for (int a = 0; a < 3; a++) {
                nb.lo[a] = std::min(nb.lo[a], o.lo[a]);
                nb.hi[a] = std::max(nb.hi[a], o.hi[a]);
            }
        }
        // get_longest_axis (bounding_box.h:63-78)
        float xs = nb.hi[0] - nb.lo[0], ys = nb.hi[1] - nb.lo[1], zs = nb.hi[2] - nb.lo[2];
        int axis = 2;
        if (xs > ys) {
            if (xs > zs)
                axis = 0;
        } else if (ys > zs) {
            axis = 1;
        }
        const std::vector<Box> &bx = boxes;
        std::sort(order.begin() + start, order.begin() + end,
                  [&bx, axis](uint32_t i, uint32_t j) { return bx[i].lo[axis] < bx[j].lo[axis]; });
        const uint32_t mid = start + (end - start) / 2;
        const uint32_t right = pos + 2 * (mid - start);
        nd.min = {nb.lo[0], nb.lo[1], nb.lo[2], u2f(0xFFFFFFFFu)};
        nd.max = {nb.hi[0], nb.hi[1], nb.hi[2], u2f(right)};
        if (spawn_depth > 0 && end - start >= 4096) {
            std::thread t([&] { build(start, mid, pos + 1, spawn_depth - 1); });
            build(mid, end, right, spawn_depth - 1);
            t.join();
        } else {
            build(start, mid, pos + 1, 0);
            build(mid, end, right, 0);
        }
    }
};

uint32_t depth_of(const std::vector<phx_bvh_node> &n, uint32_t i) {
    // iterative: (node, depth) stack
    uint32_t best = 0;
    std::vector<std::pair<uint32_t, uint32_t>> st{{i, 0}};
    while (!st.empty()) {
        auto [k, d] = st.back();
        st.pop_back();
        if (f2u(n[k].min.w) != 0xFFFFFFFFu) {
            best = std::max(best, d);
            continue;
        }
        st.push_back({k + 1, d + 1});
        st.push_back({f2u(n[k].max.w), d + 1});
    }
    return best;
}

} // namespace

bool bvh_build(const phx_triangle *tris, uint32_t n, std::vector<phx_bvh_node> &nodes, uint32_t *depth) {
    if (!tris || n == 0)
        return false;
    std::vector<Box> boxes(n);
    for (uint32_t i = 0; i < n; i++)
        if (!triangle_box(tris[i], boxes[i]))
            return false;
    nodes.assign(2 * (size_t)n - 1, phx_bvh_node{});
    Builder b(boxes, nodes.data());
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    int spawn = 0;
    while (spawn < 4 && (2u << spawn) <= hw)
        spawn++;
    b.build(0, n, 0, spawn);
    if (depth)
        *depth = depth_of(nodes, 0);
    return true;
}

namespace {

// 48-byte triangle record: {v0 | material bits}, {v1-v0 | reference rank bits}, {v2-v0 | 0}.  The
// edge vectors use the same float subtraction as hit.h:48-49, so the device test is bit-identical.
void put_trirec(float *r, const phx_triangle &tr, uint32_t ref_rank) {
    r[0] = tr.v0.x; r[1] = tr.v0.y; r[2] = tr.v0.z; r[3] = u2f(tr.mat_index);
    r[4] = tr.v1.x - tr.v0.x; r[5] = tr.v1.y - tr.v0.y; r[6] = tr.v1.z - tr.v0.z; r[7] = u2f(ref_rank);
    r[8] = tr.v2.x - tr.v0.x; r[9] = tr.v2.y - tr.v0.y; r[10] = tr.v2.z - tr.v0.z; r[11] = 0.0f;
}

// leaf reference: ~(first | (count-1) << 27)
constexpr uint32_t LEAF_FIRST_BITS = 27;
int32_t leaf_ref(uint32_t first, uint32_t count) { return ~(int32_t)(first | ((count - 1u) << LEAF_FIRST_BITS)); }

void put_pair(float *c, const float lo0[3], const float hi0[3], const float lo1[3], const float hi1[3], int32_t r0,
              int32_t r1) {
    c[0] = lo0[0]; c[1] = hi0[0]; c[2] = lo0[1]; c[3] = hi0[1];
    c[4] = lo1[0]; c[5] = hi1[0]; c[6] = lo1[1]; c[7] = hi1[1];
    c[8] = lo0[2]; c[9] = hi0[2]; c[10] = lo1[2]; c[11] = hi1[2];
    int32_t refs[2] = {r0, r1};
    std::memcpy(&c[12], refs, 8);
}

} // namespace

std::vector<uint32_t> reference_leaf_ranks(const std::vector<phx_bvh_node> &nodes, uint32_t n_tris) {
    std::vector<uint32_t> rank(n_tris, 0);
    uint32_t k = 0;
    for (const auto &nd : nodes) { // pre-order = the reference's left-first visiting order of leaves
        uint32_t t = f2u(nd.min.w);
        if (t != 0xFFFFFFFFu && t < n_tris)
            rank[t] = k++;
    }
    return rank;
}

void bvh_pack(const std::vector<phx_bvh_node> &nodes, const phx_triangle *tris, PackedBvh &out) {
    const size_t nn = nodes.size();
    std::vector<int32_t> ref(nn);
    uint32_t n_inner = 0, n_leaf = 0;
    for (size_t i = 0; i < nn; i++) {
        if (f2u(nodes[i].min.w) == 0xFFFFFFFFu)
            ref[i] = (int32_t)n_inner++;
        else
            ref[i] = leaf_ref(n_leaf++, 1);
    }
    out.cnodes.assign((size_t)n_inner * 16, 0.0f);
    out.trirec.assign((size_t)n_leaf * 12, 0.0f);
    out.leaf_tri.assign(n_leaf, 0);
    out.root = ref[0];
    out.max_leaf = 1;
    for (size_t i = 0; i < nn; i++) {
        const phx_bvh_node &nd = nodes[i];
        if (ref[i] >= 0) {
            const phx_bvh_node &L = nodes[i + 1];
            uint32_t ri = f2u(nd.max.w);
            const phx_bvh_node &R = nodes[ri];
            const float lo0[3] = {L.min.x, L.min.y, L.min.z}, hi0[3] = {L.max.x, L.max.y, L.max.z};
            const float lo1[3] = {R.min.x, R.min.y, R.min.z}, hi1[3] = {R.max.x, R.max.y, R.max.z};
            put_pair(&out.cnodes[(size_t)ref[i] * 16], lo0, hi0, lo1, hi1, ref[i + 1], ref[ri]);
        } else {
            uint32_t rank = (uint32_t)(~ref[i]) & ((1u << LEAF_FIRST_BITS) - 1u);
            uint32_t t = f2u(nd.min.w);
            out.leaf_tri[rank] = t;
            put_trirec(&out.trirec[(size_t)rank * 12], tris[t], rank);
        }
    }
}

// Binned SAH (surface area heuristic, MacDonald & Booth 1990; binning after Wald 2007): 32 bins
// per axis over the primitive centroids, cost = 1 + (A_l N_l + A_r N_r) / A, leaf cost = N.
bool bvh_build_sah(const phx_triangle *tris, uint32_t n, const std::vector<uint32_t> &ref_rank, uint32_t max_leaf,
                   PackedBvh &out) {
    if (!tris || n == 0 || n >= (1u << LEAF_FIRST_BITS))
        return false;
    max_leaf = std::max(1u, std::min(max_leaf, 16u));
    struct Prim {
        float lo[3], hi[3], c[3];
        uint32_t tri;
    };
    std::vector<Prim> P(n);
    for (uint32_t i = 0; i < n; i++) {
        Box b;
        if (!triangle_box(tris[i], b))
            return false;
        for (int a = 0; a < 3; a++) {
            P[i].lo[a] = b.lo[a];
            P[i].hi[a] = b.hi[a];
            P[i].c[a] = 0.5f * (b.lo[a] + b.hi[a]);
        }
        P[i].tri = i;
    }
    auto area = [](const float *l, const float *h) {
        float x = h[0] - l[0], y = h[1] - l[1], z = h[2] - l[2];
        return x * y + y * z + z * x;
    };
    // centroid bins per axis: 128 for ranges of 256 triangles or more (shadow stage 7.18 -> 7.10 ms on
    // the caustic workload, 3.19 -> 3.09 ms on the atrium one, against 32 everywhere), 32 below
    constexpr int NB = 128;
    out.cnodes.clear();
    out.cnodes.reserve((size_t)n * 16);
    out.trirec.assign((size_t)n * 12, 0.0f);
    out.leaf_tri.assign(n, 0);
    out.max_leaf = max_leaf;
    uint32_t next_tri = 0, depth = 0;
    int32_t root = 0;
    // work item: primitive range [b, e) at depth d whose reference goes to child `side` of `node`
    // (node == ~0u: the root).  Indices, not pointers: cnodes grows while building.
    struct Frame {
        uint32_t b, e, d;
        uint32_t node;
        int side;
    };
    std::vector<Frame> work{{0, n, 0, 0xFFFFFFFFu, 0}};
    while (!work.empty()) {
        Frame f = work.back();
        work.pop_back();
        const Frame &pd = f;
        const uint32_t b = f.b, e = f.e, cnt = e - b;
        depth = std::max(depth, f.d);
        float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
        float clo[3] = {1e30f, 1e30f, 1e30f}, chi[3] = {-1e30f, -1e30f, -1e30f};
        for (uint32_t i = b; i < e; i++)
            for (int a = 0; a < 3; a++) {
                lo[a] = std::min(lo[a], P[i].lo[a]);
                hi[a] = std::max(hi[a], P[i].hi[a]);
                clo[a] = std::min(clo[a], P[i].c[a]);
                chi[a] = std::max(chi[a], P[i].c[a]);
            }
        int32_t ref;
        // choose a split
        const int nb = cnt >= 256 ? NB : 32;
        float best = 1e30f;
        int bax = -1, bbin = 0;
        if (cnt > 1) {
            for (int a = 0; a < 3; a++) {
                float ext = chi[a] - clo[a];
                if (!(ext > 0.0f))
                    continue;
                int bc[NB] = {0};
                float bl[NB][3], bh[NB][3];
                for (int k = 0; k < nb; k++)
                    for (int j = 0; j < 3; j++) {
                        bl[k][j] = 1e30f;
                        bh[k][j] = -1e30f;
                    }
                const float sc = nb / ext;
                for (uint32_t i = b; i < e; i++) {
                    int k = std::min(nb - 1, (int)((P[i].c[a] - clo[a]) * sc));
                    bc[k]++;
                    for (int j = 0; j < 3; j++) {
                        bl[k][j] = std::min(bl[k][j], P[i].lo[j]);
                        bh[k][j] = std::max(bh[k][j], P[i].hi[j]);
                    }
                }
                float ra[NB];
                int rn[NB];
                float rl[3] = {1e30f, 1e30f, 1e30f}, rh[3] = {-1e30f, -1e30f, -1e30f};
                int acc = 0;
                for (int k = nb - 1; k > 0; k--) {
                    acc += bc[k];
                    for (int j = 0; j < 3; j++) {
                        rl[j] = std::min(rl[j], bl[k][j]);
                        rh[j] = std::max(rh[j], bh[k][j]);
                    }
                    rn[k] = acc;
                    ra[k] = acc ? area(rl, rh) : 0.0f;
                }
                float ll[3] = {1e30f, 1e30f, 1e30f}, lh[3] = {-1e30f, -1e30f, -1e30f};
                int ln = 0;
                for (int k = 1; k < nb; k++) {
                    ln += bc[k - 1];
                    for (int j = 0; j < 3; j++) {
                        ll[j] = std::min(ll[j], bl[k - 1][j]);
                        lh[j] = std::max(lh[j], bh[k - 1][j]);
                    }
                    if (ln == 0 || rn[k] == 0)
                        continue;
                    float c = ln * area(ll, lh) + rn[k] * ra[k];
                    if (c < best) {
                        best = c;
                        bax = a;
                        bbin = k;
                    }
                }
            }
        }
        const float parea = area(lo, hi);
        const bool make_leaf = cnt == 1 || (cnt <= max_leaf && (bax < 0 || 1.0f + best / parea >= (float)cnt));
        if (make_leaf && cnt <= max_leaf) {
            uint32_t first = next_tri;
            // keep triangles of a leaf in reference-rank order (irrelevant for results, stable)
            std::sort(P.begin() + b, P.begin() + e,
                      [&](const Prim &x, const Prim &y) { return ref_rank[x.tri] < ref_rank[y.tri]; });
            for (uint32_t i = b; i < e; i++) {
                out.leaf_tri[next_tri] = P[i].tri;
                put_trirec(&out.trirec[(size_t)next_tri * 12], tris[P[i].tri], ref_rank[P[i].tri]);
                next_tri++;
            }
            ref = leaf_ref(first, cnt);
            if (pd.node == 0xFFFFFFFFu)
                root = ref;
            else
                std::memcpy(&out.cnodes[(size_t)pd.node * 16 + 12 + pd.side], &ref, 4);
            continue;
        }
        uint32_t mid;
        if (bax >= 0) {
            const float ext = chi[bax] - clo[bax], sc = nb / ext;
            // stable: every range keeps ascending triangle order, so the object-median fallback
            // below splits a defined sequence (the device builder makes the same tree)
            auto it = std::stable_partition(P.begin() + b, P.begin() + e, [&](const Prim &p) {
                return std::min(nb - 1, (int)((p.c[bax] - clo[bax]) * sc)) < bbin;
            });
            mid = (uint32_t)(it - P.begin());
            if (mid == b || mid == e)
                mid = b + cnt / 2;
        } else { // all centroids coincide: object median
            mid = b + cnt / 2;
        }
        uint32_t node = (uint32_t)(out.cnodes.size() / 16);
        out.cnodes.resize(out.cnodes.size() + 16, 0.0f);
        ref = (int32_t)node;
        if (pd.node == 0xFFFFFFFFu)
            root = ref;
        else
            std::memcpy(&out.cnodes[(size_t)pd.node * 16 + 12 + pd.side], &ref, 4);
        // child boxes
        float l0[3] = {1e30f, 1e30f, 1e30f}, h0[3] = {-1e30f, -1e30f, -1e30f};
        float l1[3] = {1e30f, 1e30f, 1e30f}, h1[3] = {-1e30f, -1e30f, -1e30f};
        for (uint32_t i = b; i < mid; i++)
            for (int a = 0; a < 3; a++) {
                l0[a] = std::min(l0[a], P[i].lo[a]);
                h0[a] = std::max(h0[a], P[i].hi[a]);
            }
        for (uint32_t i = mid; i < e; i++)
            for (int a = 0; a < 3; a++) {
                l1[a] = std::min(l1[a], P[i].lo[a]);
                h1[a] = std::max(h1[a], P[i].hi[a]);
            }
        put_pair(&out.cnodes[(size_t)node * 16], l0, h0, l1, h1, 0, 0);
        // depth-first: left child processed next (pre-order layout)
        work.push_back({mid, e, f.d + 1, node, 1});
        work.push_back({b, mid, f.d + 1, node, 0});
    }
    out.root = root;
    out.depth = depth;
    return next_tri == n;
}

void bvh_widen(PackedBvh &pk) {
    struct Child {
        float lo[3], hi[3];
        int32_t ref;
    };
    auto pair = [&](int32_t node, Child *out) {
        const float *c = &pk.cnodes[(size_t)node * 16];
        int32_t refs[2];
        std::memcpy(refs, &c[12], 8);
        out[0] = {{c[0], c[2], c[8]}, {c[1], c[3], c[9]}, refs[0]};
        out[1] = {{c[4], c[6], c[10]}, {c[5], c[7], c[11]}, refs[1]};
    };
    auto area = [](const Child &c) {
        float x = c.hi[0] - c.lo[0], y = c.hi[1] - c.lo[1], z = c.hi[2] - c.lo[2];
        return x * y + y * z + z * x;
    };
    pk.wnodes.clear();
    pk.wdepth = 0;
    pk.wroot = pk.root;
    if (pk.root < 0)
        return; // a single leaf
    struct Item {
        int32_t bin;
        int32_t parent;
        int slot;
        uint32_t depth;
    };
    std::vector<Item> work{{pk.root, -1, 0, 0}};
    while (!work.empty()) {
        const Item it = work.back();
        work.pop_back();
        Child ch[4];
        pair(it.bin, ch);
        int n = 2;
        while (n < 4) { // open the inner child with the largest surface
            int best = -1;
            float ba = -1.0f;
            for (int k = 0; k < n; k++)
                if (ch[k].ref >= 0 && area(ch[k]) > ba) {
                    ba = area(ch[k]);
                    best = k;
                }
            if (best < 0)
                break;
            Child two[2];
            pair(ch[best].ref, two);
            ch[best] = two[0];
            ch[n++] = two[1];
        }
        const int32_t w = (int32_t)(pk.wnodes.size() / 28);
        pk.wnodes.resize(pk.wnodes.size() + 28, 0.0f);
        pk.wdepth = std::max(pk.wdepth, it.depth);
        if (it.parent < 0)
            pk.wroot = w;
        else
            std::memcpy(&pk.wnodes[(size_t)it.parent * 28 + 24 + it.slot], &w, 4);
        float *o = &pk.wnodes[(size_t)w * 28];
        for (int k = 0; k < 4; k++) {
            const bool has = k < n;
            for (int a = 0; a < 3; a++) {
                o[8 * a + k] = has ? ch[k].lo[a] : 1e30f;
                o[8 * a + 4 + k] = has ? ch[k].hi[a] : -1e30f;
            }
            const int32_t ref = has ? ch[k].ref : 0x7fffffff;
            std::memcpy(&o[24 + k], &ref, 4);
        }
        for (int k = n - 1; k >= 0; k--) // pre-order: the first child is laid out next
            if (ch[k].ref >= 0)
                work.push_back({ch[k].ref, w, k, it.depth + 1});
    }
}

std::vector<uint32_t> bvh_quantize(const PackedBvh &pk) {
    const size_t n = pk.wnodes.size() / 28;
    std::vector<uint32_t> q(n * QNODE_WORDS);
    for (size_t w = 0; w < n; w++)
        quantize_wide_node(&pk.wnodes[w * 28], &q[w * QNODE_WORDS]);
    return q;
}

// build_photon_hash_info (photon_hash.h:41-50)
phx_photon_hash_data hash_info(const phx_bvh_node &root, uint32_t g) {
    phx_photon_hash_data d{};
    d.grid_res = g;
    d.origin = {root.min.x, root.min.y, root.min.z, 0.0f};
    d.cell_sizes.x = std::max((root.max.x - root.min.x) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.y = std::max((root.max.y - root.min.y) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.z = std::max((root.max.z - root.min.z) / (float)g, MIN_CELL_SIZE);
    d.cell_sizes.w = 0.0f;
    return d;
}

// ShadingBuffers::upload scene centre / radius (src/buffers/shading.cpp:45-58)
void scene_sphere(const phx_bvh_node &root, phx_f4 *center, float *radius) {
    float c[3] = {0.5f * (root.min.x + root.max.x), 0.5f * (root.min.y + root.max.y), 0.5f * (root.min.z + root.max.z)};
    *center = {c[0], c[1], c[2], 0.0f};
    float lo[3] = {root.min.x, root.min.y, root.min.z}, hi[3] = {root.max.x, root.max.y, root.max.z};
    float r = 0.0f;
    for (int m = 0; m < 8; m++) {
        float dx = ((m & 1) ? hi[0] : lo[0]) - c[0];
        float dy = ((m & 2) ? hi[1] : lo[1]) - c[1];
        float dz = ((m & 4) ? hi[2] : lo[2]) - c[2];
        r = std::max(r, std::sqrt(dx * dx + dy * dy + dz * dz));
    }
    *radius = r;
}

} // namespace phx
