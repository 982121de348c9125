// k_bvh.cu — the traversal BVH built on the device.
//
// The same tree as the host's binned-SAH builder (host.cpp bvh_build_sah + bvh_widen), bit for
// bit: the same expanded triangle boxes (bounding_box.h:48-61), 128 centroid bins per axis for
// ranges of 256 triangles or more and 32 below, cost 1 + (A_l N_l + A_r N_r) / A against a leaf
// cost N, the first minimum in (axis, bin) order, a stable partition, the object median when every
// centroid coincides, nodes in pre-order with the left child first, and leaf triangles in
// reference-leaf-rank order.  Every float the split decisions read is computed with the host's
// operation order through round-to-nearest intrinsics, and min/max reductions are exact, so the
// order in which threads contribute cannot change a bit.
//
// Construction is breadth first, one level of the tree per step:
//   * a task is a primitive range [b, e) whose node (inner or leaf) is decided this level;
//   * tasks of up to 32 triangles run one per warp, of up to CHUNK one per 256-thread block, and
//     larger ones are cut into CHUNK-sized chunks whose per-chunk bounds and bins merge through
//     global atomics before one block decides the split;
//   * each task reduces its own box (which it writes into its parent's child slot), bins the
//     centroids in shared memory, evaluates the split on three lanes (one per axis, sequential
//     over the bins like the host loop), then scatters its range stably into the other buffer;
//   * inner nodes are numbered in allocation order; a bottom-up count of inner nodes per subtree
//     and a top-down pass give each its pre-order index, and a last pass writes the child-pair
//     records in that order.
// The 4-wide collapse runs the same way, one thread per wide node and level.  Reference leaf
// ranks (the tie-break of equal-t hits) come from the reference's median-split tree, which is
// built on the host; only the last step (leaf order, triangle records) needs them, so the host
// builds that tree while the device builds this one.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bvh_quant.hpp"
#include "kernels.hpp"

namespace phx {

namespace {

constexpr u32 CHUNK = 2048;        // triangles per block of a large task
constexpr u32 TINY = 32;           // tasks of up to this many triangles run one per warp
constexpr int NB_LARGE = 128;      // centroid bins per axis for ranges of 256 or more
constexpr int NB_SMALL = 32;       // and below
constexpr u32 NB_SWITCH = 256;
constexpr u32 NO_PARENT = 0xFFFFFFFFu;
constexpr u32 MAX_LEVELS = 1u << 16;
constexpr float BBOX_EPS = 1e-3f;  // bounding_box.h expansion
constexpr float BOX_INF = 1e9f;    // bounding_box.h "infinite" coordinate
constexpr float BIG = 1e30f;       // the host builder's empty-box bounds

enum : u32 { ERR_DEGENERATE = 1u, ERR_RANGE = 2u };

// order-preserving int image of a float (for atomicMin / atomicMax; -0 never occurs here)
PHX_DI int f2o(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
PHX_DI float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// x*y + y*z + z*x of the box extents, in the host's order
PHX_DI float box_area(const float *lo, const float *hi) {
    const float x = __fsub_rn(hi[0], lo[0]), y = __fsub_rn(hi[1], lo[1]), z = __fsub_rn(hi[2], lo[2]);
    return __fadd_rn(__fadd_rn(__fmul_rn(x, y), __fmul_rn(y, z)), __fmul_rn(z, x));
}

PHX_DI int leaf_ref(u32 first, u32 count) { return ~(int)(first | ((count - 1u) << LEAF_FIRST_BITS)); }

// A primitive: expanded triangle box, triangle index in lo.w.
struct Prim {
    float4 lo, hi;
};

PHX_DI float centroid(const Prim &p, int a) {
    const float l = a == 0 ? p.lo.x : a == 1 ? p.lo.y : p.lo.z;
    const float h = a == 0 ? p.hi.x : a == 1 ? p.hi.y : p.hi.z;
    return __fmul_rn(0.5f, __fadd_rn(l, h));
}

struct Task {
    u32 b, e, parent, side;
};

// a task larger than CHUNK: bounds (ordered ints) and the decided split
struct BigTask {
    u32 b, e, parent, side;
    int red[12]; // lo[3], hi[3], clo[3], chi[3]
    int bax;     // split axis, -1: object median
    u32 bbin, mid, node;
    float clo, sc;
    u32 pad[2];
};

struct Counters {
    u32 n_task[3];   // next level: tiny, medium, large tasks
    u32 n_nodes;     // inner nodes allocated
    u32 n_leaves;
    int root;        // reference of the root (set by the root task)
    u32 err;
    u32 leaf_tris;   // triangles placed in leaves (n when the leaves tile [0, n))
};

struct Lists {
    Task *tiny, *med;
    BigTask *big;
};

struct BuildArgs {
    const Prim *src;
    Prim *dst;
    float *rec;      // 16 floats per inner node, allocation order (child-pair layout of put_pair)
    u32 *leaf_tri;   // triangle index per position (leaf ranges)
    uint2 *leaves;   // (first, count) per leaf
    Counters *ctr;
    Lists next;
    u32 n;
    u32 max_leaf;
    u32 big_cap;     // capacity of the large-task list (the others hold n)
};

// Writes a child's box and reference into its parent's record (child-pair layout: x bounds of
// both children, y bounds, then z bounds of both, then the two references).
PHX_DI void put_child(const BuildArgs &A, u32 parent, u32 side, const float *lo, const float *hi, int ref) {
    if (parent == NO_PARENT) {
        A.ctr->root = ref;
        return;
    }
    float *c = A.rec + (size_t)parent * 16;
    c[4 * side + 0] = lo[0];
    c[4 * side + 1] = hi[0];
    c[4 * side + 2] = lo[1];
    c[4 * side + 3] = hi[1];
    c[8 + 2 * side] = lo[2];
    c[9 + 2 * side] = hi[2];
    c[12 + side] = __int_as_float(ref);
}

PHX_DI void push_task(const BuildArgs &A, u32 b, u32 e, u32 parent, u32 side) {
    const u32 cnt = e - b;
    const u32 cls = cnt <= TINY ? 0u : cnt <= CHUNK ? 1u : 2u;
    const u32 slot = atomicAdd(&A.ctr->n_task[cls], 1u);
    if (slot >= (cls == 2 ? A.big_cap : A.n)) { // cannot happen: a level's tasks are disjoint ranges
        atomicOr(&A.ctr->err, ERR_RANGE);
        return;
    }
    if (cls == 0) {
        A.next.tiny[slot] = {b, e, parent, side};
    } else if (cls == 1) {
        A.next.med[slot] = {b, e, parent, side};
    } else {
        BigTask t;
        t.b = b;
        t.e = e;
        t.parent = parent;
        t.side = side;
        for (int k = 0; k < 3; k++) {
            t.red[k] = f2o(BIG);
            t.red[3 + k] = f2o(-BIG);
            t.red[6 + k] = f2o(BIG);
            t.red[9 + k] = f2o(-BIG);
        }
        t.bax = -1;
        t.bbin = t.mid = t.node = 0;
        t.clo = t.sc = 0.0f;
        t.pad[0] = t.pad[1] = 0;
        A.next.big[slot] = t;
    }
}

// bins: [axis][bin][7] = count, lo[3], hi[3] (ordered ints)
PHX_DI int *bin_at(int *bins, int nb, int a, int k) { return bins + ((size_t)a * nb + k) * 7; }

PHX_DI void bin_prim(int *bins, int nb, const Prim &p, const float *clo, const float *sc, const bool *live) {
    const float lo[3] = {p.lo.x, p.lo.y, p.lo.z}, hi[3] = {p.hi.x, p.hi.y, p.hi.z};
    for (int a = 0; a < 3; a++) {
        if (!live[a])
            continue;
        const int k = max(0, min(nb - 1, __float2int_rz(__fmul_rn(__fsub_rn(centroid(p, a), clo[a]), sc[a]))));
        int *bn = bin_at(bins, nb, a, k);
        atomicAdd(&bn[0], 1);
        for (int j = 0; j < 3; j++) {
            atomicMin(&bn[1 + j], f2o(lo[j]));
            atomicMax(&bn[4 + j], f2o(hi[j]));
        }
    }
}

// Split search over one axis's bins, in the host loop's order: right-hand counts and areas from
// the top bin down, then left-hand sweeps keeping the first strict minimum.  ra/rn: nb scratch.
PHX_DI void sah_axis(const int *bins, int nb, int a, float *ra, int *rn, float *best_c, int *best_k, int *best_ln) {
    float rl[3] = {BIG, BIG, BIG}, rh[3] = {-BIG, -BIG, -BIG};
    int acc = 0;
    for (int k = nb - 1; k > 0; k--) {
        const int *bn = bin_at(const_cast<int *>(bins), nb, a, k);
        const int cnt = *(volatile const int *)&bn[0];
        acc += cnt;
        if (cnt) {
            for (int j = 0; j < 3; j++) {
                rl[j] = fminf(rl[j], o2f(*(volatile const int *)&bn[1 + j]));
                rh[j] = fmaxf(rh[j], o2f(*(volatile const int *)&bn[4 + j]));
            }
        }
        rn[k] = acc;
        ra[k] = acc ? box_area(rl, rh) : 0.0f;
    }
    float ll[3] = {BIG, BIG, BIG}, lh[3] = {-BIG, -BIG, -BIG};
    int ln = 0;
    float best = BIG;
    int bk = -1, bln = 0;
    for (int k = 1; k < nb; k++) {
        const int *bn = bin_at(const_cast<int *>(bins), nb, a, k - 1);
        const int cnt = *(volatile const int *)&bn[0];
        ln += cnt;
        if (cnt) {
            for (int j = 0; j < 3; j++) {
                ll[j] = fminf(ll[j], o2f(*(volatile const int *)&bn[1 + j]));
                lh[j] = fmaxf(lh[j], o2f(*(volatile const int *)&bn[4 + j]));
            }
        }
        if (ln == 0 || rn[k] == 0)
            continue;
        const float c = __fadd_rn(__fmul_rn(__int2float_rn(ln), box_area(ll, lh)),
                                  __fmul_rn(__int2float_rn(rn[k]), ra[k]));
        if (c < best) {
            best = c;
            bk = k;
            bln = ln;
        }
    }
    *best_c = best;
    *best_k = bk;
    *best_ln = bln;
}

struct Split {
    int bax, bbin, ln;
    float best;
};

// the three per-axis results combined in axis order (strict <: the first minimum)
PHX_DI Split combine(const float *c, const int *k, const int *ln, const bool *live) {
    Split s{-1, 0, 0, BIG};
    for (int a = 0; a < 3; a++)
        if (live[a] && k[a] >= 0 && c[a] < s.best) {
            s.best = c[a];
            s.bax = a;
            s.bbin = k[a];
            s.ln = ln[a];
        }
    return s;
}

PHX_DI bool goes_left(const Prim &p, u32 pos, int bax, int bbin, int nb, float clo, float sc, u32 mid) {
    if (bax < 0)
        return pos < mid;
    const int k = max(0, min(nb - 1, __float2int_rz(__fmul_rn(__fsub_rn(centroid(p, bax), clo), sc))));
    return k < bbin;
}

// ---- one task per group of G threads (a warp, or a whole block) ----------------------------

// Shared state of one group.  A warp's tasks hold at most TINY (< NB_SWITCH) triangles, so they bin
// with NB_SMALL bins per axis; a block's may need NB_LARGE.
template <int G> struct GroupSmem {
    static constexpr int NB = G == 32 ? NB_SMALL : NB_LARGE;
    int bins[3 * NB * 7];   // [axis][bin]: count, lo[3], hi[3] (ordered ints)
    float ra[3][NB];        // split search scratch: right-hand areas and counts per bin
    int rn[3][NB];
    float red[G / 32][12];  // per-warp bounds
    float box[12];          // lo, hi, clo, chi of the task
    float ax_c[3];          // best cost, bin and left count per axis
    int ax_k[3], ax_ln[3];
    u32 node;               // the inner node allocated for the task
    u32 wtot[G / 32];       // per-warp left | valid counts of a partition tile
};
static_assert(TINY < NB_SWITCH, "warp tasks bin with NB_SMALL bins");

template <int G> PHX_DI void gsync() {
    if (G == 32)
        __syncwarp();
    else
        __syncthreads();
}

template <int G> PHX_DI void process_task(const Task t, const BuildArgs &A, GroupSmem<G> &sm, int tid) {
    static_assert(G == 32 || GroupSmem<G>::NB == NB_LARGE, "a block-sized group bins up to 128 per axis");
    const u32 b = t.b, e = t.e, cnt = e - b;
    const int lane = tid & 31, warp = tid >> 5;
    // 1. bounds of the boxes and of the centroids
    float r[12];
    for (int k = 0; k < 3; k++) {
        r[k] = BIG;
        r[3 + k] = -BIG;
        r[6 + k] = BIG;
        r[9 + k] = -BIG;
    }
    for (u32 i = b + tid; i < e; i += G) {
        const Prim p = A.src[i];
        const float lo[3] = {p.lo.x, p.lo.y, p.lo.z}, hi[3] = {p.hi.x, p.hi.y, p.hi.z};
        for (int k = 0; k < 3; k++) {
            const float c = centroid(p, k);
            r[k] = fminf(r[k], lo[k]);
            r[3 + k] = fmaxf(r[3 + k], hi[k]);
            r[6 + k] = fminf(r[6 + k], c);
            r[9 + k] = fmaxf(r[9 + k], c);
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 3; k++) {
            r[k] = fminf(r[k], __shfl_xor_sync(0xffffffffu, r[k], off));
            r[3 + k] = fmaxf(r[3 + k], __shfl_xor_sync(0xffffffffu, r[3 + k], off));
            r[6 + k] = fminf(r[6 + k], __shfl_xor_sync(0xffffffffu, r[6 + k], off));
            r[9 + k] = fmaxf(r[9 + k], __shfl_xor_sync(0xffffffffu, r[9 + k], off));
        }
    if (lane == 0)
        for (int k = 0; k < 12; k++)
            sm.red[warp][k] = r[k];
    gsync<G>();
    if (tid < 12) {
        float v = sm.red[0][tid];
        for (int w = 1; w < G / 32; w++)
            v = (tid % 6) < 3 ? fminf(v, sm.red[w][tid]) : fmaxf(v, sm.red[w][tid]);
        sm.box[tid] = v;
    }
    gsync<G>();
    const float lo[3] = {sm.box[0], sm.box[1], sm.box[2]}, hi[3] = {sm.box[3], sm.box[4], sm.box[5]};
    const float clo[3] = {sm.box[6], sm.box[7], sm.box[8]}, chi[3] = {sm.box[9], sm.box[10], sm.box[11]};
    const int nb = cnt >= NB_SWITCH ? NB_LARGE : NB_SMALL;
    bool live[3];
    float sc[3];
    for (int a = 0; a < 3; a++) {
        const float ext = __fsub_rn(chi[a], clo[a]);
        live[a] = cnt > 1 && ext > 0.0f;
        sc[a] = live[a] ? __fdiv_rn(__int2float_rn(nb), ext) : 0.0f;
    }
    // 2. centroid bins
    Split s{-1, 0, 0, BIG};
    if (cnt > 1) {
        for (int i = tid; i < 3 * nb; i += G) {
            int *bn = &sm.bins[i * 7];
            bn[0] = 0;
            for (int j = 0; j < 3; j++) {
                bn[1 + j] = f2o(BIG);
                bn[4 + j] = f2o(-BIG);
            }
        }
        gsync<G>();
        for (u32 i = b + tid; i < e; i += G)
            bin_prim(sm.bins, nb, A.src[i], clo, sc, live);
        gsync<G>();
        // 3. split search: one lane per axis
        if (tid < 3) {
            sm.ax_k[tid] = -1;
            if (live[tid])
                sah_axis(sm.bins, nb, tid, sm.ra[tid], sm.rn[tid], &sm.ax_c[tid], &sm.ax_k[tid], &sm.ax_ln[tid]);
        }
        gsync<G>();
        s = combine(sm.ax_c, sm.ax_k, sm.ax_ln, live);
    }
    const float parea = box_area(lo, hi);
    const bool make_leaf =
        cnt == 1 || (cnt <= A.max_leaf &&
                     (s.bax < 0 || __fadd_rn(1.0f, __fdiv_rn(s.best, parea)) >= __int2float_rn((int)cnt)));
    if (make_leaf) {
        for (u32 i = b + tid; i < e; i += G)
            A.leaf_tri[i] = __float_as_uint(A.src[i].lo.w);
        if (tid == 0) {
            put_child(A, t.parent, t.side, lo, hi, leaf_ref(b, cnt));
            const u32 li = atomicAdd(&A.ctr->n_leaves, 1u);
            atomicAdd(&A.ctr->leaf_tris, cnt);
            if (li < A.n)
                A.leaves[li] = make_uint2(b, cnt);
            else
                atomicOr(&A.ctr->err, ERR_RANGE);
        }
        return;
    }
    const u32 mid = s.bax >= 0 ? b + (u32)s.ln : b + cnt / 2;
    if (tid == 0) {
        const u32 node = atomicAdd(&A.ctr->n_nodes, 1u);
        sm.node = node;
        put_child(A, t.parent, t.side, lo, hi, (int)node);
    }
    // 4. stable partition into the other buffer
    const float pclo = s.bax >= 0 ? clo[s.bax] : 0.0f, psc = s.bax >= 0 ? sc[s.bax] : 0.0f;
    u32 lbase = 0, rbase = 0;
    for (u32 base = b; base < e; base += G) {
        const u32 i = base + tid;
        const bool valid = i < e;
        Prim p;
        bool left = false;
        if (valid) {
            p = A.src[i];
            left = goes_left(p, i, s.bax, s.bbin, nb, pclo, psc, mid);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, left);
        const unsigned vbal = __ballot_sync(0xffffffffu, valid);
        const u32 lrank = __popc(bal & ((1u << lane) - 1u));
        const u32 vrank = __popc(vbal & ((1u << lane) - 1u));
        u32 wl = 0, wv = 0; // lefts / valid in earlier warps of this tile
        u32 tl = __popc(bal), tv = __popc(vbal);
        if (G > 32) {
            if (lane == 0)
                sm.wtot[warp] = (u32)__popc(bal) | ((u32)__popc(vbal) << 16);
            gsync<G>();
            tl = tv = 0;
            for (int w = 0; w < G / 32; w++) {
                const u32 x = sm.wtot[w];
                if (w < warp) {
                    wl += x & 0xffffu;
                    wv += x >> 16;
                }
                tl += x & 0xffffu;
                tv += x >> 16;
            }
            gsync<G>();
        }
        if (valid) {
            const u32 lpos = lbase + wl + lrank;
            const u32 rpos = rbase + (wv + vrank) - (wl + lrank);
            const u32 o = left ? b + lpos : mid + rpos;
            if (o >= b && o < e && (left ? o < mid : o >= mid))
                A.dst[o] = p;
            else
                atomicOr(&A.ctr->err, ERR_RANGE);
        }
        lbase += tl;
        rbase += tv - tl;
    }
    gsync<G>();
    if (tid == 0) {
        push_task(A, b, mid, sm.node, 0);
        push_task(A, mid, e, sm.node, 1);
    }
}

__global__ void __launch_bounds__(256) k_task_block(const Task *tasks, u32 n_tasks, BuildArgs A) {
    __shared__ GroupSmem<256> sm;
    if (blockIdx.x >= n_tasks)
        return;
    process_task<256>(tasks[blockIdx.x], A, sm, threadIdx.x);
}

__global__ void __launch_bounds__(128) k_task_warp(const Task *tasks, u32 n_tasks, BuildArgs A) {
    __shared__ GroupSmem<32> sm[4];
    const u32 w = threadIdx.x >> 5;
    const u32 t = blockIdx.x * 4 + w;
    if (t >= n_tasks)
        return; // whole warps leave together; the group is one warp
    process_task<32>(tasks[t], A, sm[w], threadIdx.x & 31);
}

// ---- large tasks: chunked bounds and bins, one block decides, chunked stable scatter ----------

struct Chunk {
    u32 task, cb, ce, first; // first: the task's first chunk index
};

__global__ void __launch_bounds__(256) k_big_reduce(const Chunk *chunks, BigTask *big, int *gbins, BuildArgs A) {
    const Chunk ch = chunks[blockIdx.x];
    BigTask &t = big[ch.task];
    if (blockIdx.x == ch.first) { // this task's global bins
        int *bins = gbins + (size_t)ch.task * 3 * NB_LARGE * 7;
        for (int i = threadIdx.x; i < 3 * NB_LARGE; i += blockDim.x) {
            bins[i * 7] = 0;
            for (int j = 0; j < 3; j++) {
                bins[i * 7 + 1 + j] = f2o(BIG);
                bins[i * 7 + 4 + j] = f2o(-BIG);
            }
        }
    }
    float r[12];
    for (int k = 0; k < 3; k++) {
        r[k] = BIG;
        r[3 + k] = -BIG;
        r[6 + k] = BIG;
        r[9 + k] = -BIG;
    }
    for (u32 i = ch.cb + threadIdx.x; i < ch.ce; i += blockDim.x) {
        const Prim p = A.src[i];
        const float lo[3] = {p.lo.x, p.lo.y, p.lo.z}, hi[3] = {p.hi.x, p.hi.y, p.hi.z};
        for (int k = 0; k < 3; k++) {
            const float c = centroid(p, k);
            r[k] = fminf(r[k], lo[k]);
            r[3 + k] = fmaxf(r[3 + k], hi[k]);
            r[6 + k] = fminf(r[6 + k], c);
            r[9 + k] = fmaxf(r[9 + k], c);
        }
    }
    for (int off = 16; off > 0; off >>= 1)
        for (int k = 0; k < 12; k++) {
            const float o = __shfl_xor_sync(0xffffffffu, r[k], off);
            r[k] = (k % 6) < 3 ? fminf(r[k], o) : fmaxf(r[k], o);
        }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 12; k++) {
            if ((k % 6) < 3)
                atomicMin(&t.red[k], f2o(r[k]));
            else
                atomicMax(&t.red[k], f2o(r[k]));
        }
}

PHX_DI void big_bounds(const BigTask &t, float *lo, float *hi, float *clo, float *chi) {
    for (int k = 0; k < 3; k++) {
        lo[k] = o2f(t.red[k]);
        hi[k] = o2f(t.red[3 + k]);
        clo[k] = o2f(t.red[6 + k]);
        chi[k] = o2f(t.red[9 + k]);
    }
}

__global__ void __launch_bounds__(256) k_big_bin(const Chunk *chunks, const BigTask *big, int *gbins, BuildArgs A) {
    __shared__ int bins[3 * NB_LARGE * 7];
    const Chunk ch = chunks[blockIdx.x];
    const BigTask &t = big[ch.task];
    float lo[3], hi[3], clo[3], chi[3], sc[3];
    bool live[3];
    big_bounds(t, lo, hi, clo, chi);
    for (int a = 0; a < 3; a++) {
        const float ext = __fsub_rn(chi[a], clo[a]);
        live[a] = ext > 0.0f;
        sc[a] = live[a] ? __fdiv_rn((float)NB_LARGE, ext) : 0.0f;
    }
    for (int i = threadIdx.x; i < 3 * NB_LARGE; i += blockDim.x) {
        bins[i * 7] = 0;
        for (int j = 0; j < 3; j++) {
            bins[i * 7 + 1 + j] = f2o(BIG);
            bins[i * 7 + 4 + j] = f2o(-BIG);
        }
    }
    __syncthreads();
    for (u32 i = ch.cb + threadIdx.x; i < ch.ce; i += blockDim.x)
        bin_prim(bins, NB_LARGE, A.src[i], clo, sc, live);
    __syncthreads();
    int *g = gbins + (size_t)ch.task * 3 * NB_LARGE * 7;
    for (int i = threadIdx.x; i < 3 * NB_LARGE; i += blockDim.x) {
        if (bins[i * 7] == 0)
            continue;
        atomicAdd(&g[i * 7], bins[i * 7]);
        for (int j = 0; j < 3; j++) {
            atomicMin(&g[i * 7 + 1 + j], bins[i * 7 + 1 + j]);
            atomicMax(&g[i * 7 + 4 + j], bins[i * 7 + 4 + j]);
        }
    }
}

// one warp per large task: split search on three lanes, node allocation, child tasks
__global__ void __launch_bounds__(32) k_big_decide(BigTask *big, const int *gbins, BuildArgs A) {
    __shared__ float ra[3][NB_LARGE];
    __shared__ int rn[3][NB_LARGE];
    __shared__ float ax_c[3];
    __shared__ int ax_k[3], ax_ln[3];
    BigTask &t = big[blockIdx.x];
    float lo[3], hi[3], clo[3], chi[3];
    bool live[3];
    big_bounds(t, lo, hi, clo, chi);
    for (int a = 0; a < 3; a++)
        live[a] = __fsub_rn(chi[a], clo[a]) > 0.0f;
    // the task's merged bins, staged in shared memory by the whole warp: the split search walks
    // them sequentially on three lanes, which from global memory took ~0.1 ms per task
    __shared__ int bins[3 * NB_LARGE * 7];
    const int *gb = gbins + (size_t)blockIdx.x * 3 * NB_LARGE * 7;
    const int tid = threadIdx.x;
    for (int i = tid; i < 3 * NB_LARGE * 7; i += 32)
        bins[i] = __ldcg(&gb[i]);
    __syncwarp();
    if (tid < 3) {
        ax_k[tid] = -1;
        if (live[tid])
            sah_axis(bins, NB_LARGE, tid, ra[tid], rn[tid], &ax_c[tid], &ax_k[tid], &ax_ln[tid]);
    }
    __syncwarp();
    if (tid != 0)
        return;
    const Split s = combine(ax_c, ax_k, ax_ln, live);
    const u32 b = t.b, e = t.e, cnt = e - b;
    // cnt > CHUNK > max_leaf: never a leaf
    const u32 mid = s.bax >= 0 ? b + (u32)s.ln : b + cnt / 2;
    const u32 node = atomicAdd(&A.ctr->n_nodes, 1u);
    put_child(A, t.parent, t.side, lo, hi, (int)node);
    t.bax = s.bax;
    t.bbin = (u32)s.bbin;
    t.mid = mid;
    t.node = node;
    t.clo = s.bax >= 0 ? clo[s.bax] : 0.0f;
    t.sc = s.bax >= 0 ? __fdiv_rn((float)NB_LARGE, __fsub_rn(chi[s.bax], clo[s.bax])) : 0.0f;
    push_task(A, b, mid, node, 0);
    push_task(A, mid, e, node, 1);
}

__global__ void __launch_bounds__(256) k_big_count(const Chunk *chunks, const BigTask *big, u32 *chunk_left,
                                                   BuildArgs A) {
    __shared__ u32 wsum[8];
    const Chunk ch = chunks[blockIdx.x];
    const BigTask &t = big[ch.task];
    u32 c = 0;
    for (u32 i = ch.cb + threadIdx.x; i < ch.ce; i += blockDim.x)
        c += goes_left(A.src[i], i, t.bax, (int)t.bbin, NB_LARGE, t.clo, t.sc, t.mid) ? 1u : 0u;
    for (int off = 16; off > 0; off >>= 1)
        c += __shfl_xor_sync(0xffffffffu, c, off);
    if ((threadIdx.x & 31) == 0)
        wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        u32 s = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            s += wsum[w];
        chunk_left[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(256) k_big_scatter(const Chunk *chunks, const BigTask *big, const u32 *chunk_left,
                                                     BuildArgs A) {
    __shared__ u32 wtot[8];
    __shared__ u32 before;
    const Chunk ch = chunks[blockIdx.x];
    const BigTask &t = big[ch.task];
    if (threadIdx.x == 0) {
        u32 s = 0;
        for (u32 k = ch.first; k < blockIdx.x; k++)
            s += chunk_left[k];
        before = s;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u32 lbase = before, rbase = (ch.cb - t.b) - before;
    for (u32 base = ch.cb; base < ch.ce; base += blockDim.x) {
        const u32 i = base + threadIdx.x;
        const bool valid = i < ch.ce;
        Prim p;
        bool left = false;
        if (valid) {
            p = A.src[i];
            left = goes_left(p, i, t.bax, (int)t.bbin, NB_LARGE, t.clo, t.sc, t.mid);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, left);
        const unsigned vbal = __ballot_sync(0xffffffffu, valid);
        if (lane == 0)
            wtot[warp] = (u32)__popc(bal) | ((u32)__popc(vbal) << 16);
        __syncthreads();
        u32 wl = 0, wv = 0, tl = 0, tv = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
            const u32 x = wtot[w];
            if (w < warp) {
                wl += x & 0xffffu;
                wv += x >> 16;
            }
            tl += x & 0xffffu;
            tv += x >> 16;
        }
        __syncthreads();
        if (valid) {
            const u32 lrank = __popc(bal & ((1u << lane) - 1u)) + wl;
            const u32 vrank = __popc(vbal & ((1u << lane) - 1u)) + wv;
            const u32 o = left ? t.b + lbase + lrank : t.mid + rbase + (vrank - lrank);
            if (o >= t.b && o < t.e && (left ? o < t.mid : o >= t.mid))
                A.dst[o] = p;
            else
                atomicOr(&A.ctr->err, ERR_RANGE);
        }
        lbase += tl;
        rbase += tv - tl;
    }
}

// ---- primitives, numbering, records ---------------------------------------------------------

// get_bounding_box (bounding_box.h:48-61) of every triangle, expanded by BBOX_EPS
__global__ void k_prims(const phx_triangle *tris, u32 n, Prim *out, u32 *err) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const phx_triangle &t = tris[i];
    const float v[3][3] = {{t.v0.x, t.v0.y, t.v0.z}, {t.v1.x, t.v1.y, t.v1.z}, {t.v2.x, t.v2.y, t.v2.z}};
    float lo[3], hi[3];
    bool bad = false;
    for (int a = 0; a < 3; a++) {
        lo[a] = BOX_INF;
        hi[a] = -BOX_INF;
        for (int k = 0; k < 3; k++) {
            lo[a] = v[k][a] < lo[a] ? v[k][a] : lo[a];
            hi[a] = hi[a] < v[k][a] ? v[k][a] : hi[a];
        }
        bad |= lo[a] >= BOX_INF || lo[a] <= -BOX_INF || hi[a] >= BOX_INF || hi[a] <= -BOX_INF;
    }
    for (int a = 0; a < 3; a++) {
        lo[a] = __fsub_rn(lo[a], BBOX_EPS);
        hi[a] = __fadd_rn(hi[a], BBOX_EPS);
        bad |= lo[a] == hi[a];
    }
    if (bad)
        atomicOr(err, ERR_DEGENERATE);
    out[i].lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(i));
    out[i].hi = make_float4(hi[0], hi[1], hi[2], 0.0f);
}

// inner nodes under each node of one level (children are deeper, already counted)
__global__ void k_subtree(const float *rec, u32 lo, u32 hi, u32 *sub) {
    const u32 i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi)
        return;
    const int r0 = __float_as_int(rec[(size_t)i * 16 + 12]), r1 = __float_as_int(rec[(size_t)i * 16 + 13]);
    sub[i] = 1u + (r0 >= 0 ? sub[r0] : 0u) + (r1 >= 0 ? sub[r1] : 0u);
}

__global__ void k_preorder(const float *rec, u32 lo, u32 hi, const u32 *sub, u32 *pre) {
    const u32 i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi)
        return;
    const int r0 = __float_as_int(rec[(size_t)i * 16 + 12]), r1 = __float_as_int(rec[(size_t)i * 16 + 13]);
    const u32 p = pre[i];
    if (r0 >= 0)
        pre[r0] = p + 1u;
    if (r1 >= 0)
        pre[r1] = p + 1u + (r0 >= 0 ? sub[r0] : 0u);
}

__global__ void k_remap(const float *rec, u32 n_nodes, const u32 *pre, float *out, u32 *err) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes)
        return;
    const float *c = rec + (size_t)i * 16;
    if (pre[i] >= n_nodes) { // every node is reached by the pre-order pass
        atomicOr(err, ERR_RANGE);
        return;
    }
    float *o = out + (size_t)pre[i] * 16;
    for (int k = 0; k < 12; k++)
        o[k] = c[k];
    for (int s = 0; s < 2; s++) {
        const int r = __float_as_int(c[12 + s]);
        if (r >= (int)n_nodes)
            atomicOr(err, ERR_RANGE);
        o[12 + s] = __int_as_float(r >= 0 && r < (int)n_nodes ? (int)pre[r] : r);
    }
    o[14] = 0.0f;
    o[15] = 0.0f;
}

// ---- 4-wide collapse (host.cpp bvh_widen), one thread per wide node and level ---------------

struct WTask {
    int bin;      // child-pair node (pre-order index)
    u32 parent;   // wide node in allocation order, NO_PARENT for the root
    u32 slot;
    u32 pad;
};

struct WideChild {
    float lo[3], hi[3];
    int ref;
};

PHX_DI void load_pair(const float *cn, int node, WideChild *out) {
    const float *c = cn + (size_t)node * 16;
    const int r0 = __float_as_int(c[12]), r1 = __float_as_int(c[13]);
    out[0] = {{c[0], c[2], c[8]}, {c[1], c[3], c[9]}, r0};
    out[1] = {{c[4], c[6], c[10]}, {c[5], c[7], c[11]}, r1};
}

__global__ void k_widen_level(const float *cn, const WTask *tasks, u32 n_tasks, float *wrec, WTask *next,
                              u32 *ctr /* [0] next tasks, [1] wide nodes, [2] error */, int *wroot, u32 cap) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_tasks)
        return;
    const WTask t = tasks[i];
    if (t.bin < 0 || (u32)t.bin >= cap) { // cap = child-pair nodes
        atomicOr(&ctr[2], ERR_RANGE);
        return;
    }
    WideChild ch[4];
    load_pair(cn, t.bin, ch);
    int n = 2;
    while (n < 4) { // open the inner child with the largest surface (first maximum)
        int best = -1;
        float ba = -1.0f;
        for (int k = 0; k < n; k++)
            if (ch[k].ref >= 0) {
                const float a = box_area(ch[k].lo, ch[k].hi);
                if (a > ba) {
                    ba = a;
                    best = k;
                }
            }
        if (best < 0)
            break;
        if ((u32)ch[best].ref >= cap) {
            atomicOr(&ctr[2], ERR_RANGE);
            return;
        }
        WideChild two[2];
        load_pair(cn, ch[best].ref, two);
        ch[best] = two[0];
        ch[n++] = two[1];
    }
    const u32 w = atomicAdd(&ctr[1], 1u);
    if (w >= cap) {
        atomicOr(&ctr[2], ERR_RANGE);
        return;
    }
    if (t.parent == NO_PARENT)
        *wroot = (int)w;
    else
        wrec[(size_t)t.parent * 28 + 24 + t.slot] = __int_as_float((int)w);
    float *o = wrec + (size_t)w * 28;
    for (int k = 0; k < 4; k++) {
        const bool has = k < n;
        for (int a = 0; a < 3; a++) {
            o[8 * a + k] = has ? ch[k].lo[a] : BIG;
            o[8 * a + 4 + k] = has ? ch[k].hi[a] : -BIG;
        }
        // inner children: replaced by the child's wide index when it is allocated
        o[24 + k] = __int_as_float(has ? ch[k].ref : 0x7fffffff);
    }
    for (int k = 0; k < n; k++)
        if (ch[k].ref >= 0) {
            const u32 s = atomicAdd(&ctr[0], 1u);
            if (s < cap)
                next[s] = {ch[k].ref, w, (u32)k, 0u};
            else
                atomicOr(&ctr[2], ERR_RANGE);
        }
}

// inner (wide) children of wide node i: slots whose reference is a wide node
PHX_DI bool wide_inner(const float *wrec, u32 i, int k, int *ref) {
    *ref = __float_as_int(wrec[(size_t)i * 28 + 24 + k]);
    return *ref >= 0 && *ref != 0x7fffffff;
}

__global__ void k_wsubtree(const float *wrec, u32 lo, u32 hi, u32 *sub) {
    const u32 i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi)
        return;
    u32 s = 1;
    for (int k = 0; k < 4; k++) {
        int r;
        if (wide_inner(wrec, i, k, &r))
            s += sub[r];
    }
    sub[i] = s;
}

__global__ void k_wpreorder(const float *wrec, u32 lo, u32 hi, const u32 *sub, u32 *pre) {
    const u32 i = lo + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= hi)
        return;
    u32 next = pre[i] + 1u;
    for (int k = 0; k < 4; k++) {
        int r;
        if (wide_inner(wrec, i, k, &r)) {
            pre[r] = next;
            next += sub[r];
        }
    }
}

__global__ void k_wremap(const float *wrec, u32 n, const u32 *pre, float *out, u32 *err) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float *c = wrec + (size_t)i * 28;
    if (pre[i] >= n) {
        atomicOr(err, ERR_RANGE);
        return;
    }
    float *o = out + (size_t)pre[i] * 28;
    for (int k = 0; k < 24; k++)
        o[k] = c[k];
    for (int k = 0; k < 4; k++) {
        int r;
        const bool inner = wide_inner(wrec, i, k, &r);
        if (inner && r >= (int)n)
            atomicOr(err, ERR_RANGE);
        o[24 + k] = inner && r < (int)n ? __int_as_float((int)pre[r]) : c[24 + k];
    }
}

// ---- leaf order and triangle records --------------------------------------------------------

// triangles of each leaf in reference-rank order (ranks are a permutation: one result)
__global__ void k_leaf_sort(const uint2 *leaves, u32 n_leaves, const u32 *rank, u32 *leaf_tri) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_leaves)
        return;
    const uint2 L = leaves[i];
    u32 *t = leaf_tri + L.x;
    for (u32 a = 1; a < L.y; a++) {
        const u32 v = t[a], rv = rank[v];
        u32 j = a;
        while (j > 0 && rank[t[j - 1]] > rv) {
            t[j] = t[j - 1];
            j--;
        }
        t[j] = v;
    }
}

// put_trirec (48 B: {v0 | material bits}, {v1-v0 | rank bits}, {v2-v0 | 0}) and the per-triangle
// normals, tangents and uvs in leaf order
__global__ void k_tri_records(const phx_triangle *tris, const u32 *leaf_tri, const u32 *rank, u32 n, float4 *trirec,
                              float4 *nrm, float4 *tan, float4 *uv) {
    const u32 r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n)
        return;
    const u32 ti = leaf_tri[r];
    const phx_triangle &t = tris[ti];
    trirec[3 * (size_t)r + 0] = make_float4(t.v0.x, t.v0.y, t.v0.z, __uint_as_float(t.mat_index));
    trirec[3 * (size_t)r + 1] = make_float4(__fsub_rn(t.v1.x, t.v0.x), __fsub_rn(t.v1.y, t.v0.y),
                                            __fsub_rn(t.v1.z, t.v0.z), __uint_as_float(rank[ti]));
    trirec[3 * (size_t)r + 2] =
        make_float4(__fsub_rn(t.v2.x, t.v0.x), __fsub_rn(t.v2.y, t.v0.y), __fsub_rn(t.v2.z, t.v0.z), 0.0f);
    const phx_f4 *nn[3] = {&t.n0, &t.n1, &t.n2}, *tt[3] = {&t.t0, &t.t1, &t.t2};
    for (int k = 0; k < 3; k++) {
        nrm[3 * (size_t)r + k] = make_float4(nn[k]->x, nn[k]->y, nn[k]->z, nn[k]->w);
        tan[3 * (size_t)r + k] = make_float4(tt[k]->x, tt[k]->y, tt[k]->z, tt[k]->w);
    }
    uv[2 * (size_t)r + 0] = make_float4(t.uv0.x, t.uv0.y, t.uv1.x, t.uv1.y);
    uv[2 * (size_t)r + 1] = make_float4(t.uv2.x, t.uv2.y, 0.0f, 0.0f);
}

__global__ void k_quantize(const float *wnodes, u32 n, u32 *out) {
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        quantize_wide_node(wnodes + (size_t)i * 28, out + (size_t)i * QNODE_WORDS);
}

__global__ void k_push_root(BuildArgs A, u32 n) { push_task(A, 0, n, NO_PARENT, 0); }

u32 blocks_for(u64 n, u32 bs) { return (u32)std::max<u64>(1, (n + bs - 1) / bs); }

// Device scratch of one build: the buffers of a layout are carved from one allocation (a build made
// twenty cudaMalloc / cudaFree calls, each synchronising the device, before it had done any work).
// The layout runs twice: once to size the arena, once to hand out the pointers.
struct Scratch {
    std::vector<void *> arenas;
    char *base = nullptr;
    size_t used = 0;
    bool sizing = false;
    ~Scratch() {
        for (void *p : arenas)
            cudaFree(p);
    }
    template <class T> T *get(size_t count) {
        const size_t off = used;
        used += (std::max<size_t>(count * sizeof(T), 16) + 255) & ~size_t(255);
        return sizing ? nullptr : reinterpret_cast<T *>(base + off);
    }
    // runs layout() to size an arena, allocates it, and runs layout() again with real pointers
    template <class F> bool carve(F &&layout) {
        sizing = true;
        used = 0;
        layout();
        void *p = nullptr;
        if (cudaMalloc(&p, used) != cudaSuccess)
            return false;
        arenas.push_back(p);
        base = static_cast<char *>(p);
        sizing = false;
        used = 0;
        layout();
        return true;
    }
};

int sync_read(void *h, const void *d, size_t bytes, cudaStream_t st, std::string &err) {
    cudaError_t e = cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        err = std::string("device BVH build: ") + cudaGetErrorString(e);
        return 3;
    }
    return 0;
}

} // namespace

void DeviceBvh::release() {
    cudaFree(cnodes);
    cudaFree(wnodes);
    cudaFree(leaf_tri);
    cudaFree(leaves);
    cnodes = wnodes = nullptr;
    leaf_tri = nullptr;
    leaves = nullptr;
}

int bvh_device_build(const phx_triangle *tris, u32 n, u32 max_leaf, bool widen, cudaStream_t st, DeviceBvh &out,
                     std::string &err) {
    out.release();
    out = DeviceBvh{};
    if (!tris || n == 0 || n >= (1u << LEAF_FIRST_BITS)) {
        err = "device BVH build: no triangles, or too many";
        return 1;
    }
    max_leaf = std::max(1u, std::min(max_leaf, 16u));
    Scratch S;
    const u32 big_cap = n / CHUNK + 2, chunk_cap = n / CHUNK + big_cap + 2;
    Prim *pa, *pb;
    float *rec;
    Task *tiny[2], *med[2];
    BigTask *big[2];
    int *gbins;
    Chunk *chunks;
    u32 *chunk_left, *sub, *pre;
    Counters *ctr;
    const bool carved = S.carve([&] {
        pa = S.get<Prim>(n);
        pb = S.get<Prim>(n);
        rec = S.get<float>((size_t)n * 16);
        tiny[0] = S.get<Task>(n);
        tiny[1] = S.get<Task>(n);
        med[0] = S.get<Task>(n);
        med[1] = S.get<Task>(n);
        big[0] = S.get<BigTask>(big_cap);
        big[1] = S.get<BigTask>(big_cap);
        gbins = S.get<int>((size_t)big_cap * 3 * NB_LARGE * 7);
        chunks = S.get<Chunk>(chunk_cap);
        chunk_left = S.get<u32>(chunk_cap);
        ctr = S.get<Counters>(1);
        sub = S.get<u32>(n);
        pre = S.get<u32>(n);
    });
    if (!carved || cudaMalloc(&out.leaf_tri, (size_t)n * 4) != cudaSuccess ||
        cudaMalloc(&out.leaves, (size_t)n * 8) != cudaSuccess) {
        out.release();
        err = "device BVH build: out of device memory";
        return 2;
    }
    Counters host_ctr{};
    Counters *hc = &host_ctr; // read back with a synchronous copy per level (a few words)
    u32 hw[4] = {0, 0, 0, 0};
    auto fail = [&](int code, const char *msg) {
        out.release();
        err = msg;
        return code;
    };
    int r;
    cudaMemsetAsync(rec, 0, (size_t)n * 16 * 4, st);
    cudaMemsetAsync(out.leaf_tri, 0, (size_t)n * 4, st);
    cudaMemsetAsync(ctr, 0, sizeof(Counters), st);
    k_prims<<<blocks_for(n, 256), 256, 0, st>>>(tris, n, pa, &ctr->err);
    {
        BuildArgs A{};
        A.ctr = ctr;
        A.n = n;
        A.big_cap = big_cap;
        A.next = {tiny[0], med[0], big[0]};
        k_push_root<<<1, 1, 0, st>>>(A, n);
    }
    if ((r = sync_read(hc, ctr, sizeof(Counters), st, err)))
        return out.release(), r;
    if (hc->err & ERR_DEGENERATE)
        return fail(1, "degenerate or infinite triangle bounding box (bounding_box.h:17-28)");

    std::vector<u32> level_nodes{0};
    std::vector<BigTask> hbig;
    std::vector<Chunk> hch;
    Prim *src = pa, *dst = pb;
    int cur = 0;
    u32 levels = 0;
    for (;;) {
        const u32 nt = hc->n_task[0], nm = hc->n_task[1], nbg = hc->n_task[2];
        if (nt + nm + nbg == 0)
            break;
        if (++levels > MAX_LEVELS)
            return fail(1, "device BVH build: tree deeper than 65536 levels");
        cudaMemsetAsync(ctr->n_task, 0, sizeof(ctr->n_task), st);
        BuildArgs A{src, dst, rec, out.leaf_tri, out.leaves, ctr, {tiny[cur ^ 1], med[cur ^ 1], big[cur ^ 1]},
                    n, max_leaf, big_cap};
        if (nbg) {
            hbig.resize(nbg);
            if ((r = sync_read(hbig.data(), big[cur], nbg * sizeof(BigTask), st, err)))
                return out.release(), r;
            hch.clear();
            for (u32 k = 0; k < nbg; k++) {
                const u32 first = (u32)hch.size();
                for (u32 cb = hbig[k].b; cb < hbig[k].e; cb += CHUNK)
                    hch.push_back({k, cb, std::min(cb + CHUNK, hbig[k].e), first});
            }
            if (hch.size() > chunk_cap)
                return fail(3, "device BVH build: chunk table overflow");
            const u32 nch = (u32)hch.size();
            cudaMemcpyAsync(chunks, hch.data(), nch * sizeof(Chunk), cudaMemcpyHostToDevice, st);
            k_big_reduce<<<nch, 256, 0, st>>>(chunks, big[cur], gbins, A);
            k_big_bin<<<nch, 256, 0, st>>>(chunks, big[cur], gbins, A);
            k_big_decide<<<nbg, 32, 0, st>>>(big[cur], gbins, A);
            k_big_count<<<nch, 256, 0, st>>>(chunks, big[cur], chunk_left, A);
            k_big_scatter<<<nch, 256, 0, st>>>(chunks, big[cur], chunk_left, A);
        }
        if (nm)
            k_task_block<<<nm, 256, 0, st>>>(med[cur], nm, A);
        if (nt)
            k_task_warp<<<blocks_for(nt, 4), 128, 0, st>>>(tiny[cur], nt, A);
        if ((r = sync_read(hc, ctr, sizeof(Counters), st, err)))
            return out.release(), r;
        if (hc->err)
            return fail(3, "device BVH build: a task range was inconsistent");
        level_nodes.push_back(hc->n_nodes);
        std::swap(src, dst);
        cur ^= 1;
    }
    if (hc->leaf_tris != n)
        return fail(3, "device BVH build: the leaves do not cover every triangle");
    const u32 N = hc->n_nodes;
    out.n_inner = N;
    out.n_leaves = hc->n_leaves;
    out.depth = levels ? levels - 1 : 0;
    out.levels = levels;
    out.root = hc->root;
    if (cudaMalloc(&out.cnodes, (size_t)std::max(N, 1u) * 16 * 4) != cudaSuccess)
        return fail(2, "device BVH build: out of device memory");
    if (N > 0) {
        if (out.root != 0)
            return fail(3, "device BVH build: the root is not the first inner node");
        for (u32 d = levels; d-- > 0;) {
            const u32 lo = level_nodes[d], hi = level_nodes[d + 1];
            if (hi > lo)
                k_subtree<<<blocks_for(hi - lo, 256), 256, 0, st>>>(rec, lo, hi, sub);
        }
        cudaMemsetAsync(pre, 0xff, (size_t)N * 4, st); // unreached nodes stay out of range
        cudaMemsetAsync(pre, 0, 4, st);
        for (u32 d = 0; d < levels; d++) {
            const u32 lo = level_nodes[d], hi = level_nodes[d + 1];
            if (hi > lo)
                k_preorder<<<blocks_for(hi - lo, 256), 256, 0, st>>>(rec, lo, hi, sub, pre);
        }
        k_remap<<<blocks_for(N, 256), 256, 0, st>>>(rec, N, pre, out.cnodes, &ctr->err);
    }
    if (N > 0) {
        if ((r = sync_read(hc, ctr, sizeof(Counters), st, err)))
            return out.release(), r;
        if (hc->err)
            return fail(3, "device BVH build: node numbering inconsistent");
    }
    out.wroot = out.root;
    if (widen && N > 0) {
        // the child-pair records, numbered, are the input; the wide tree has at most N nodes
        float *wrec;
        WTask *wt[2];
        u32 *wctr, *wsub, *wpre;
        int *wroot;
        const bool wcarved = S.carve([&] {
            wrec = S.get<float>((size_t)N * 28);
            wt[0] = S.get<WTask>(N);
            wt[1] = S.get<WTask>(N);
            wctr = S.get<u32>(4);
            wroot = S.get<int>(1);
            wsub = S.get<u32>(N);
            wpre = S.get<u32>(N);
        });
        if (!wcarved || cudaMalloc(&out.wnodes, (size_t)N * 28 * 4) != cudaSuccess)
            return fail(2, "device BVH build: out of device memory");
        const WTask root_task{0, NO_PARENT, 0u, 0u};
        cudaMemcpyAsync(wt[0], &root_task, sizeof(WTask), cudaMemcpyHostToDevice, st);
        cudaMemsetAsync(wctr, 0, 16, st);
        std::vector<u32> wlevel{0};
        u32 ncur = 1, wl = 0;
        int c = 0;
        while (ncur) {
            cudaMemsetAsync(wctr, 0, 4, st);
            k_widen_level<<<blocks_for(ncur, 128), 128, 0, st>>>(out.cnodes, wt[c], ncur, wrec, wt[c ^ 1], wctr,
                                                               wroot, N);
            if ((r = sync_read(hw, wctr, 12, st, err)))
                return out.release(), r;
            if (hw[2])
                return fail(3, "device BVH build: 4-wide collapse overflow");
            wlevel.push_back(hw[1]);
            ncur = hw[0];
            c ^= 1;
            wl++;
        }
        const u32 W = wlevel.back();
        for (u32 d = wl; d-- > 0;) {
            const u32 lo = wlevel[d], hi = wlevel[d + 1];
            if (hi > lo)
                k_wsubtree<<<blocks_for(hi - lo, 256), 256, 0, st>>>(wrec, lo, hi, wsub);
        }
        cudaMemsetAsync(wpre, 0xff, (size_t)W * 4, st);
        cudaMemsetAsync(wpre, 0, 4, st);
        for (u32 d = 0; d < wl; d++) {
            const u32 lo = wlevel[d], hi = wlevel[d + 1];
            if (hi > lo)
                k_wpreorder<<<blocks_for(hi - lo, 256), 256, 0, st>>>(wrec, lo, hi, wsub, wpre);
        }
        k_wremap<<<blocks_for(W, 256), 256, 0, st>>>(wrec, W, wpre, out.wnodes, &wctr[2]);
        if ((r = sync_read(hw, wctr, 12, st, err)))
            return out.release(), r;
        if (hw[2])
            return fail(3, "device BVH build: 4-wide numbering inconsistent");
        out.n_wide = W;
        out.wdepth = wl ? wl - 1 : 0;
        out.wroot = 0;
    }
    cudaError_t e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
        e = cudaGetLastError();
    if (e != cudaSuccess) {
        out.release();
        err = std::string("device BVH build: ") + cudaGetErrorString(e);
        return 3;
    }
    return 0;
}

cudaError_t bvh_device_quantize(const float *wnodes, u32 n, u32 *out, cudaStream_t st) {
    k_quantize<<<blocks_for(n, 128), 128, 0, st>>>(wnodes, n, out);
    return cudaGetLastError();
}

int bvh_device_finish(const phx_triangle *tris, const u32 *rank, u32 n, DeviceBvh &b, float4 *trirec, float4 *nrm,
                      float4 *tan, float4 *uv, cudaStream_t st) {
    if (b.n_leaves)
        k_leaf_sort<<<blocks_for(b.n_leaves, 128), 128, 0, st>>>(b.leaves, b.n_leaves, rank, b.leaf_tri);
    k_tri_records<<<blocks_for(n, 128), 128, 0, st>>>(tris, b.leaf_tri, rank, n, trirec, nrm, tan, uv);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

} // namespace phx
