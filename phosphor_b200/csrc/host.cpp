// host.cpp — BVH construction and packing, camera, light prefix sums, scene generators.
#include "host.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

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

struct BuildNode {
    Box box;
    int32_t tri;
    uint32_t left, right;
};

struct Builder {
    const std::vector<Box> &boxes;
    std::vector<uint32_t> order;
    std::vector<BuildNode> tmp;

    explicit Builder(const std::vector<Box> &b) : boxes(b), order(b.size()) {
        std::iota(order.begin(), order.end(), 0u);
        tmp.reserve(2 * b.size());
    }

    // build_tmp (bvh.cpp:18-53): one triangle per leaf, median split of the longest axis of the
    // node box on the triangle boxes' minimum corner.
    uint32_t build(uint32_t start, uint32_t end) {
        uint32_t id = (uint32_t)tmp.size();
        tmp.push_back({});
        if (end == start + 1) {
            tmp[id].tri = (int32_t)order[start];
            tmp[id].box = boxes[order[start]];
            tmp[id].left = tmp[id].right = 0;
            return id;
        }
        Box nb = boxes[order[start]];
        for (uint32_t i = start + 1; i < end; i++) {
            const Box &o = boxes[order[i]];
            for (int a = 0; a < 3; a++) {
                nb.lo[a] = std::min(nb.lo[a], o.lo[a]);
                nb.hi[a] = std::max(nb.hi[a], o.hi[a]);
            }
        }
        tmp[id].box = nb;
        tmp[id].tri = -1;
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
        uint32_t mid = start + (end - start) / 2;
        uint32_t l = build(start, mid);
        uint32_t r = build(mid, end);
        tmp[id].left = l;
        tmp[id].right = r;
        return id;
    }

    // flatten (bvh.cpp:57-72): pre-order, left child follows its parent, right child index kept
    // in max.w, triangle index (or -1) in min.w.
    void flatten(uint32_t ti, std::vector<phx_bvh_node> &out) const {
        uint32_t id = (uint32_t)out.size();
        out.push_back({});
        const BuildNode &n = tmp[ti];
        out[id].min = {n.box.lo[0], n.box.lo[1], n.box.lo[2], u2f((uint32_t)n.tri)};
        out[id].max = {n.box.hi[0], n.box.hi[1], n.box.hi[2], u2f(n.right)};
        if (n.tri == -1) {
            flatten(n.left, out);
            out[id].max.w = u2f((uint32_t)out.size());
            flatten(n.right, out);
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
    Builder b(boxes);
    b.build(0, n);
    nodes.clear();
    nodes.reserve(2 * (size_t)n - 1);
    b.flatten(0, nodes);
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
            auto it = std::partition(P.begin() + b, P.begin() + e, [&](const Prim &p) {
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

void SceneStore::view(phx_scene *s) const {
    std::memset(s, 0, sizeof(*s));
    s->triangles = tris.data();
    s->n_triangles = (uint32_t)tris.size();
    s->emissive_triangles = etris.empty() ? nullptr : etris.data();
    s->n_emissive_triangles = (uint32_t)etris.size();
    s->materials = mats.data();
    s->uv_transforms = uvs.data();
    s->n_materials = (uint32_t)mats.size();
    s->lights = lights.empty() ? nullptr : lights.data();
    s->n_lights = (uint32_t)lights.size();
    s->lum_pref_sum = lum.empty() ? nullptr : lum.data();
    s->tex_meta = tex_meta.empty() ? nullptr : tex_meta.data();
    s->n_textures = (uint32_t)tex_meta.size();
    s->tex_atlas = atlas.empty() ? nullptr : atlas.data();
    s->tex_atlas_bytes = atlas.size();
    s->envmap = envmap.empty() ? nullptr : envmap.data();
    s->envmap_width = env_w;
    s->envmap_height = env_h;
    s->camera = camera;
}

// ---- procedural scenes --------------------------------------------------------------------------
namespace {

struct V3 {
    double x, y, z;
};
inline V3 operator+(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator*(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 vcross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 vnorm(V3 a) {
    double l = std::sqrt(vdot(a, a));
    return l > 0 ? a * (1.0 / l) : a;
}

struct Pcg { // the renderer's PCG stream (random.h:16-36) drives every generator choice
    uint32_t s;
    explicit Pcg(uint32_t seed) {
        s = 2891336453u + seed;
        s = s * 747796405u + 2891336453u;
    }
    uint32_t next() {
        uint32_t old = s;
        s = s * 747796405u + 2891336453u;
        return ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
    }
    double uni() { return (double)next() / 4294967296.0; }
    double uni(double a, double b) { return a + (b - a) * uni(); }
};

phx_f4 F4(V3 v) { return {(float)v.x, (float)v.y, (float)v.z, 0.0f}; }

phx_material make_material(float r, float g, float b, float metallic, float roughness) {
    // make_default_material (src/parsers/material.cpp:9-30) with the given factors
    phx_material m{};
    m.base_color = {r, g, b, 1.0f};
    m.emissive = {0.0f, 0.0f, 0.0f, 0.0f};
    m.att_color = {1.0f, 1.0f, 1.0f, 0.0f};
    m.metallic = metallic;
    m.roughness = roughness;
    m.transmission = 0.0f;
    m.ior = 1.5f;
    m.att_dist = INF;
    m.thickness = 0.0f;
    m.diff_index = m.emis_index = m.norm_index = m.occlusion_index = m.metal_rough_index = m.transmission_index =
        PHX_NO_TEXTURE;
    return m;
}

phx_uv_transform_block identity_uv() {
    phx_uv_transform id{};
    id.uv_offset = {0.0f, 0.0f};
    id.uv_scale = {1.0f, 1.0f};
    id.uv_rotation = 0.0f;
    phx_uv_transform_block b{};
    b.diff = b.emis = b.norm = b.occlusion = b.metal_rough = b.transmission = id;
    return b;
}

struct Gen {
    SceneStore &s;
    explicit Gen(SceneStore &st) : s(st) {}

    uint32_t material(const phx_material &m) {
        s.mats.push_back(m);
        s.uvs.push_back(identity_uv());
        return (uint32_t)s.mats.size() - 1;
    }

    // one triangle with per-vertex normals; tangent as parse_mesh computes it without UVs
    // (scene.cpp:83-95: det = 0 -> (1,0,0))
    void tri(V3 p0, V3 p1, V3 p2, V3 n0, V3 n1, V3 n2, uint32_t mat) {
        phx_triangle t{};
        t.v0 = F4(p0);
        t.v1 = F4(p1);
        t.v2 = F4(p2);
        t.n0 = F4(vnorm(n0));
        t.n1 = F4(vnorm(n1));
        t.n2 = F4(vnorm(n2));
        t.t0 = t.t1 = t.t2 = {1.0f, 0.0f, 0.0f, 0.0f};
        t.uv0 = t.uv1 = t.uv2 = {0.0f, 0.0f};
        t.mat_index = mat;
        s.tris.push_back(t);
    }
    void flat_tri(V3 p0, V3 p1, V3 p2, V3 n, uint32_t mat) { tri(p0, p1, p2, n, n, n, mat); }
    // quad a-b-c-d (counter-clockwise seen from the normal side)
    void quad(V3 a, V3 b, V3 c, V3 d, V3 n, uint32_t mat) {
        flat_tri(a, b, c, n, mat);
        flat_tri(a, c, d, n, mat);
    }
    // emissive mesh -> LIGHT_TEXTURED (scene.cpp:115-130): power = pi * emissive * area
    void emissive_quad(V3 a, V3 b, V3 c, V3 d, V3 n, uint32_t mat, V3 emissive) {
        uint32_t start_tri = (uint32_t)s.tris.size();
        quad(a, b, c, d, n, mat);
        uint32_t estart = (uint32_t)s.etris.size();
        float area = 0.0f;
        for (uint32_t j = start_tri; j < (uint32_t)s.tris.size(); j++) {
            const phx_triangle &t = s.tris[j];
            s.etris.push_back(t);
            float e1[3] = {t.v1.x - t.v0.x, t.v1.y - t.v0.y, t.v1.z - t.v0.z};
            float e2[3] = {t.v2.x - t.v0.x, t.v2.y - t.v0.y, t.v2.z - t.v0.z};
            float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2],
                  cz = e1[0] * e2[1] - e1[1] * e2[0];
            area += 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
        }
        phx_light l{};
        l.kind = PHX_LIGHT_TEXTURED;
        l.power = {PI * (float)emissive.x * area, PI * (float)emissive.y * area, PI * (float)emissive.z * area, 0.0f};
        l.aux = {u2f(PHX_NO_TEXTURE), u2f(estart), u2f((uint32_t)s.tris.size() - start_tri), area};
        s.lights.push_back(l);
    }
    void box(V3 lo, V3 hi, double yaw, uint32_t mat) {
        V3 c = (lo + hi) * 0.5, h = (hi - lo) * 0.5;
        double cs = std::cos(yaw), sn = std::sin(yaw);
        auto P = [&](double sx, double sy, double sz) {
            double x = sx * h.x, z = sz * h.z;
            return V3{c.x + cs * x - sn * z, c.y + sy * h.y, c.z + sn * x + cs * z};
        };
        auto N = [&](double x, double y, double z) { return V3{cs * x - sn * z, y, sn * x + cs * z}; };
        quad(P(-1, -1, 1), P(1, -1, 1), P(1, 1, 1), P(-1, 1, 1), N(0, 0, 1), mat);
        quad(P(1, -1, -1), P(-1, -1, -1), P(-1, 1, -1), P(1, 1, -1), N(0, 0, -1), mat);
        quad(P(1, -1, 1), P(1, -1, -1), P(1, 1, -1), P(1, 1, 1), N(1, 0, 0), mat);
        quad(P(-1, -1, -1), P(-1, -1, 1), P(-1, 1, 1), P(-1, 1, -1), N(-1, 0, 0), mat);
        quad(P(-1, 1, 1), P(1, 1, 1), P(1, 1, -1), P(-1, 1, -1), N(0, 1, 0), mat);
        quad(P(-1, -1, -1), P(1, -1, -1), P(1, -1, 1), P(-1, -1, 1), N(0, -1, 0), mat);
    }
    // cylinder along +y, segments around, with caps
    void cylinder(V3 base, double r, double hgt, int seg, uint32_t mat) {
        for (int i = 0; i < seg; i++) {
            double a0 = 2 * M_PI * i / seg, a1 = 2 * M_PI * (i + 1) / seg;
            V3 n0{std::cos(a0), 0, std::sin(a0)}, n1{std::cos(a1), 0, std::sin(a1)};
            V3 b0 = base + n0 * r, b1 = base + n1 * r;
            V3 t0 = b0 + V3{0, hgt, 0}, t1 = b1 + V3{0, hgt, 0};
            tri(b0, b1, t1, n0, n1, n1, mat);
            tri(b0, t1, t0, n0, n1, n0, mat);
            V3 top = base + V3{0, hgt, 0};
            flat_tri(top, t1, t0, V3{0, 1, 0}, mat);
            flat_tri(base, b0, b1, V3{0, -1, 0}, mat);
        }
    }
    // UV sphere: stacks x slices, poles as fans
    void sphere(V3 c, double r, int stacks, int slices, uint32_t mat) {
        auto P = [&](int i, int j) {
            double th = M_PI * i / stacks, ph = 2 * M_PI * j / slices;
            return V3{std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)};
        };
        for (int i = 0; i < stacks; i++)
            for (int j = 0; j < slices; j++) {
                V3 a = P(i, j), b = P(i + 1, j), cc = P(i + 1, j + 1), d = P(i, j + 1);
                if (i != 0)
                    tri(c + a * r, c + b * r, c + d * r, a, b, d, mat);
                if (i != stacks - 1)
                    tri(c + d * r, c + b * r, c + cc * r, d, b, cc, mat);
            }
    }
    // half torus standing in the vertical plane through p0-p1 (an arch between two points)
    void arch(V3 p0, V3 p1, double minor, int seg_major, int seg_minor, uint32_t mat) {
        V3 mid = (p0 + p1) * 0.5;
        V3 ax = p1 - p0;
        double R = 0.5 * std::sqrt(vdot(ax, ax));
        V3 u = vnorm(ax), up{0, 1, 0};
        V3 w = vnorm(vcross(u, up));
        auto P = [&](int i, int j, V3 *n) {
            double a = M_PI * i / seg_major, b = 2 * M_PI * j / seg_minor;
            V3 radial = u * std::cos(a) + up * std::sin(a);
            V3 nn = radial * std::cos(b) + w * std::sin(b);
            *n = nn;
            return mid + radial * R + nn * minor;
        };
        for (int i = 0; i < seg_major; i++)
            for (int j = 0; j < seg_minor; j++) {
                V3 na, nb, nc, nd;
                V3 a = P(i, j, &na), b = P(i + 1, j, &nb), c = P(i + 1, j + 1, &nc), d = P(i, j + 1, &nd);
                tri(a, b, c, na, nb, nc, mat);
                tri(a, c, d, na, nc, nd, mat);
            }
    }
};

// Camera::Camera + focus + to_params (src/renderer/camera.cpp:3-56) with glm's float semantics:
// normalize(v) = v * (1/sqrt(dot)), radians(d) = d * 0.017453292...
void make_camera(const float pos[3], const float at[3], const float up[3], float hfov, float aspect, float defocus,
                 float focus, phx_camera_params *out) {
    struct G {
        float x, y, z;
    };
    auto sub = [](G a, G b) { return G{a.x - b.x, a.y - b.y, a.z - b.z}; };
    auto mul = [](G a, float s) { return G{a.x * s, a.y * s, a.z * s}; };
    auto dotg = [](G a, G b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
    auto nrm = [&](G a) { return mul(a, 1.0f / std::sqrt(dotg(a, a))); };
    auto crs = [](G a, G b) { return G{a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; };
    const float deg2rad = (float)0.01745329251994329576923690768489;
    G P{pos[0], pos[1], pos[2]}, T{at[0], at[1], at[2]}, U{up[0], up[1], up[2]};
    float fd = 1.0f, da = 0.0f;
    G dd_u{0, 0, 0}, dd_v{0, 0, 0};
    G hor, ver, ll, uu, vv, ww;
    auto recalc = [&]() {
        ww = nrm(sub(P, T));
        uu = nrm(crs(U, ww));
        vv = crs(ww, uu);
        float hf = hfov * deg2rad;
        float hw = std::tan(hf * 0.5f) * fd;
        float hh = hw / aspect;
        hor = mul(uu, 2.0f * hw);
        ver = mul(vv, 2.0f * hh);
        ll = sub(sub(sub(P, mul(hor, 0.5f)), mul(ver, 0.5f)), mul(ww, fd));
    };
    recalc();
    // focus()
    da = defocus;
    fd = focus;
    float dr = fd * std::tan((da / 2.0f) * deg2rad);
    dd_u = mul(uu, dr);
    dd_v = mul(vv, dr);
    recalc();
    auto f4 = [](G g) { return phx_f4{g.x, g.y, g.z, 0.0f}; };
    std::memset(out, 0, sizeof(*out));
    out->position = f4(P);
    out->lower_left_corner = f4(ll);
    out->horizontal = f4(hor);
    out->vertical = f4(ver);
    out->defocus_disk_u = f4(dd_u);
    out->defocus_disk_v = f4(dd_v);
    out->defocus_angle = da;
    out->focus_distance = fd;
}

void finish_lights(SceneStore &s) { // SceneData::build_lum_pref_sum (scene_data.cpp:14-23)
    s.lum.clear();
    float run = 0.0f;
    for (const auto &l : s.lights) {
        float lum = l.power.x * 0.2126f + l.power.y * 0.7152f + l.power.z * 0.0722f;
        run += std::max(lum, 0.0f);
        s.lum.push_back(run);
    }
}

void cornell(Gen &g, bool with_light = true) {
    uint32_t white = g.material(make_material(0.73f, 0.71f, 0.68f, 0.0f, 1.0f));
    uint32_t red = g.material(make_material(0.63f, 0.06f, 0.04f, 0.0f, 1.0f));
    uint32_t green = g.material(make_material(0.14f, 0.45f, 0.09f, 0.0f, 1.0f));
    g.quad({0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1}, {0, 1, 0}, white);   // floor
    g.quad({0, 1, 0}, {0, 1, 1}, {1, 1, 1}, {1, 1, 0}, {0, -1, 0}, white);  // ceiling
    g.quad({0, 0, 0}, {0, 1, 0}, {1, 1, 0}, {1, 0, 0}, {0, 0, 1}, white);   // back
    g.quad({0, 0, 0}, {0, 0, 1}, {0, 1, 1}, {0, 1, 0}, {1, 0, 0}, red);     // left
    g.quad({1, 0, 0}, {1, 1, 0}, {1, 1, 1}, {1, 0, 1}, {-1, 0, 0}, green);  // right
    if (with_light) {
        phx_material lm = make_material(0.78f, 0.78f, 0.78f, 0.0f, 1.0f);
        lm.emissive = {15.0f, 15.0f, 15.0f, 0.0f};
        uint32_t light = g.material(lm);
        double y = 0.999, a = 0.375, b = 0.625;
        g.emissive_quad({a, y, a}, {a, y, b}, {b, y, b}, {b, y, a}, {0, -1, 0}, light, {15.0, 15.0, 15.0});
    }
}

void caustic_extras(Gen &g, Pcg &rng, uint32_t n_side, int sph_seg) {
    phx_material wm = make_material(1.0f, 1.0f, 1.0f, 0.0f, 0.05f);
    wm.transmission = 1.0f;
    wm.ior = 1.33f;
    uint32_t water = g.material(wm);
    uint32_t copper = g.material(make_material(0.95f, 0.64f, 0.54f, 1.0f, 0.2f));
    struct Wave {
        double a, k, dx, dz, ph;
    } w[8];
    for (auto &wv : w) {
        wv.a = rng.uni(0.002, 0.01);
        double lambda = rng.uni(0.05, 0.3);
        wv.k = 2 * M_PI / lambda;
        double th = rng.uni(0.0, 2 * M_PI);
        wv.dx = std::cos(th);
        wv.dz = std::sin(th);
        wv.ph = rng.uni(0.0, 2 * M_PI);
    }
    auto height = [&](double x, double z, double *gx, double *gz) {
        double h = 0.4;
        *gx = *gz = 0;
        for (auto &wv : w) {
            double arg = wv.k * (wv.dx * x + wv.dz * z) + wv.ph;
            h += wv.a * std::sin(arg);
            *gx += wv.a * wv.k * wv.dx * std::cos(arg);
            *gz += wv.a * wv.k * wv.dz * std::cos(arg);
        }
        return h;
    };
    std::vector<V3> P((size_t)n_side * n_side), N((size_t)n_side * n_side);
    for (uint32_t j = 0; j < n_side; j++)
        for (uint32_t i = 0; i < n_side; i++) {
            double x = (double)i / (n_side - 1), z = (double)j / (n_side - 1), gx, gz;
            double y = height(x, z, &gx, &gz);
            P[(size_t)j * n_side + i] = {x, y, z};
            N[(size_t)j * n_side + i] = vnorm(V3{-gx, 1.0, -gz});
        }
    for (uint32_t j = 0; j + 1 < n_side; j++)
        for (uint32_t i = 0; i + 1 < n_side; i++) {
            size_t a = (size_t)j * n_side + i, b = a + 1, c = a + n_side + 1, d = a + n_side;
            g.tri(P[a], P[d], P[c], N[a], N[d], N[c], water);
            g.tri(P[a], P[c], P[b], N[a], N[c], N[b], water);
        }
    g.sphere({0.66, 0.62, 0.42}, 0.15, sph_seg, sph_seg, copper);
}

void sky_envmap(SceneStore &s, uint32_t w, uint32_t h, V3 sun_dir) {
    // analytic sky: horizon-to-zenith gradient plus a Gaussian sun lobe; stored in the
    // reference's z-up equirect layout (envmap.h:9-20), scene up = +y
    s.env_w = w;
    s.env_h = h;
    s.envmap.resize((size_t)w * h * 3);
    V3 sd = vnorm(sun_dir);
    for (uint32_t py = 0; py < h; py++) {
        double v = (py + 0.5) / h;
        double theta = (1.0 - v) * M_PI; // v = 1 - theta/pi
        for (uint32_t px = 0; px < w; px++) {
            double u = (px + 0.5) / w;
            double phi = u * 2 * M_PI - M_PI;
            V3 d{std::sin(theta) * std::cos(phi), std::sin(theta) * std::sin(phi), std::cos(theta)};
            double up = d.y; // scene up
            double t = std::max(0.0, up);
            V3 horizon{0.9, 0.85, 0.8}, zenith{0.25, 0.45, 0.85}, ground{0.3, 0.28, 0.25};
            V3 c = up >= 0 ? horizon * (1 - t) + zenith * t : ground;
            double cosang = vdot(d, sd);
            double lobe = 40.0 * std::exp(-(1.0 - cosang) / 0.0015);
            float *o = &s.envmap[((size_t)py * w + px) * 3];
            o[0] = (float)(c.x + lobe * 1.0);
            o[1] = (float)(c.y + lobe * 0.95);
            o[2] = (float)(c.z + lobe * 0.85);
        }
    }
}

void atrium(Gen &g, Pcg &rng, int arch_seg, int env_w, int env_h) {
    std::vector<uint32_t> mats;
    for (int i = 0; i < 32; i++) {
        float r = (float)rng.uni(0.05, 0.9), gg = (float)rng.uni(0.05, 0.9), b = (float)rng.uni(0.05, 0.9);
        float rough = (float)rng.uni(0.05, 0.9);
        float metal = rng.uni() < 0.3 ? 1.0f : 0.0f;
        mats.push_back(g.material(make_material(r, gg, b, metal, rough)));
    }
    auto pick = [&]() { return mats[rng.next() % 32u]; };
    double X = 8, Z = 6;
    g.quad({-12, 0, -10}, {-12, 0, 10}, {12, 0, 10}, {12, 0, -10}, {0, 1, 0}, mats[0]);
    // 24 columns around the courtyard perimeter: 8 per long side, 4 per short side (corners shared)
    std::vector<V3> ring;
    for (int i = 0; i < 8; i++)
        ring.push_back({-X + 2 * X * i / 7.0, 0, -Z});
    for (int i = 1; i <= 4; i++)
        ring.push_back({X, 0, -Z + 2 * Z * i / 5.0});
    for (int i = 7; i >= 0; i--)
        ring.push_back({-X + 2 * X * i / 7.0, 0, Z});
    for (int i = 4; i >= 1; i--)
        ring.push_back({-X, 0, -Z + 2 * Z * i / 5.0});
    const double col_r = 0.35, col_h = 4.0, slab_y = 5.3, slab_t = 0.3;
    const double floors[2] = {0.0, slab_y + slab_t};
    int minor_seg = std::max(8, arch_seg * 40 / 64);
    for (double fy : floors) {
        uint32_t cm = pick(), am = pick();
        for (const V3 &p : ring)
            g.cylinder({p.x, fy, p.z}, col_r, col_h, 64, cm);
        for (size_t i = 0; i < ring.size(); i++) {
            const V3 &a = ring[i], &b = ring[(i + 1) % ring.size()];
            g.arch({a.x, fy + col_h, a.z}, {b.x, fy + col_h, b.z}, 0.25, arch_seg, minor_seg, am);
        }
    }
    uint32_t sm = pick();
    g.box({-X - 0.6, slab_y, -Z - 0.6}, {X + 0.6, slab_y + slab_t, -Z + 0.6}, 0, sm);
    g.box({-X - 0.6, slab_y, Z - 0.6}, {X + 0.6, slab_y + slab_t, Z + 0.6}, 0, sm);
    g.box({-X - 0.6, slab_y, -Z + 0.6}, {-X + 0.6, slab_y + slab_t, Z - 0.6}, 0, sm);
    g.box({X - 0.6, slab_y, -Z + 0.6}, {X + 0.6, slab_y + slab_t, Z - 0.6}, 0, sm);
    for (int i = 0; i < 400; i++) {
        double sx = rng.uni(0.05, 0.5), sy = rng.uni(0.05, 0.5), sz = rng.uni(0.05, 0.5);
        double cx = rng.uni(-X + 1, X - 1), cz = rng.uni(-Z + 1, Z - 1), yaw = rng.uni(0, M_PI);
        g.box({cx - sx / 2, 0, cz - sz / 2}, {cx + sx / 2, sy, cz + sz / 2}, yaw, pick());
    }
    phx_light sun{};
    sun.kind = PHX_LIGHT_POINT;
    V3 sun_pos{2.0, 14.0, 3.0};
    sun.position = F4(sun_pos);
    sun.power = {200.0f, 190.0f, 170.0f, 0.0f};
    g.s.lights.push_back(sun);
    sky_envmap(g.s, (uint32_t)env_w, (uint32_t)env_h, sun_pos);
}

} // namespace

int scene_generate(const phx_scene_spec &spec, SceneStore &s, std::string &err) {
    s = SceneStore{};
    Gen g(s);
    Pcg rng(spec.seed);
    float aspect = spec.height ? (float)spec.width / (float)spec.height : 1.0f;
    switch (spec.kind) {
    case PHX_SCENE_CORNELL: {
        cornell(g);
        float pos[3] = {0.5f, 0.5f, 2.4f}, at[3] = {0.5f, 0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 40.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    case PHX_SCENE_CAUSTIC: {
        cornell(g);
        uint32_t side = spec.detail ? spec.detail : 256u;
        if (side < 2)
            side = 2;
        int seg = spec.detail ? std::max(6, (int)(side * 100 / 256)) : 100;
        caustic_extras(g, rng, side, seg);
        float pos[3] = {0.5f, 0.5f, 2.4f}, at[3] = {0.5f, 0.5f, 0.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 40.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    case PHX_SCENE_ATRIUM: {
        int seg = spec.detail ? (int)spec.detail : 64;
        int ew = spec.detail ? 512 : 2048, eh = spec.detail ? 256 : 1024;
        atrium(g, rng, std::max(4, seg), ew, eh);
        float pos[3] = {-6.2f, 1.7f, -4.6f}, at[3] = {5.0f, 3.2f, 4.0f}, up[3] = {0.0f, 1.0f, 0.0f};
        make_camera(pos, at, up, 75.0f, aspect, 0.0f, 1.0f, &s.camera);
        break;
    }
    default:
        err = "unknown scene kind";
        return PHX_E_INVALID;
    }
    finish_lights(s);
    return PHX_OK;
}

} // namespace phx

namespace phx {
int camera_make(const float p[3], const float a[3], const float u[3], float hfov, float aspect, float defocus,
                float focus, phx_camera_params *out) {
    make_camera(p, a, u, hfov, aspect, defocus, focus, out);
    return PHX_OK;
}
void lum_pref_sum(const phx_light *l, uint32_t n, float *out) {
    float run = 0.0f;
    for (uint32_t i = 0; i < n; i++) {
        float lum = l[i].power.x * 0.2126f + l[i].power.y * 0.7152f + l[i].power.z * 0.0722f;
        run += std::max(lum, 0.0f);
        out[i] = run;
    }
}
} // namespace phx
