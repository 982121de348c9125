"""The traversal tree: the host builder's tree is valid (CPU), and the GPU builder (the default;
PHX_F_HOST_BVH selects the host one) returns the same arrays bit for bit and renders the same
images (needs a GPU).

The SAH tree is the kernels' own structure (the reference traverses the median-split tree of
src/renderer/bvh.cpp); what it must preserve is the reference's hit for every ray, which the
tie-break rank carried in each triangle record guarantees for any tree over the same boxes.  Here
the checks are structural: every triangle sits in exactly one leaf, every child box bounds its
subtree, leaves keep the reference-rank order, and the device build equals the host build.
"""
import ctypes as C

import numpy as np
import pytest

import phosphor_b200 as P
from phosphor_b200 import _capi as A
from phosphor_b200 import renderer as R

LEAF_BITS = 27
EMPTY = 0x7FFFFFFF


def soup(verts: np.ndarray) -> P.SceneData:
    """A scene of bare triangles (n, 3, 3) for the tree builders (no materials needed)."""
    n = len(verts)
    rec = np.zeros((n, 44), np.float32)
    rec[:, 0:3], rec[:, 4:7], rec[:, 8:11] = verts[:, 0], verts[:, 1], verts[:, 2]
    rec[:, 12:15] = rec[:, 16:19] = rec[:, 20:23] = (0.0, 0.0, 1.0)
    sc = A.Scene()
    sc.triangles = rec.ctypes.data_as(C.POINTER(A.Triangle))
    sc.n_triangles = n
    return P.SceneData(sc, keep=(rec,))


def random_soup(n, seed=0, scale=10.0, size=0.3):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-scale, scale, (n, 1, 3))
    return soup((c + rng.normal(0, size, (n, 3, 3))).astype(np.float32))


def coincident_soup(n_same, n_other, seed=1):
    """n_same copies of one triangle (every centroid equal: the object-median fallback) + others."""
    rng = np.random.default_rng(seed)
    same = np.repeat(np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]]], np.float32), n_same, axis=0)
    c = rng.uniform(-5, 5, (n_other, 1, 3))
    other = (c + rng.normal(0, 0.2, (n_other, 3, 3))).astype(np.float32)
    return soup(np.concatenate([same, other]).astype(np.float32))


def grid_soup(side):
    """A height-field-like sheet: rows of triangles whose centroids tie on two axes."""
    xs, zs = np.meshgrid(np.arange(side, dtype=np.float32), np.arange(side, dtype=np.float32))
    p00 = np.stack([xs, np.zeros_like(xs), zs], -1).reshape(-1, 3)
    t1 = np.stack([p00, p00 + (1, 0, 0), p00 + (0, 0, 1)], 1)
    t2 = np.stack([p00 + (1, 0, 0), p00 + (1, 0, 1), p00 + (0, 0, 1)], 1)
    return soup(np.concatenate([t1, t2]).astype(np.float32))


def ref_ranks(scene):
    nodes, _ = R.bvh_build(scene)
    tri = nodes[:, 3].view(np.uint32)
    leaves = tri[tri != 0xFFFFFFFF]
    rank = np.empty(scene.n_triangles, np.uint32)
    rank[leaves] = np.arange(len(leaves), dtype=np.uint32)
    return rank


def expanded_boxes(scene):
    v = scene.triangle_vertices().astype(np.float32)
    return v.min(axis=1) - np.float32(1e-3), v.max(axis=1) + np.float32(1e-3)


def check_tree(scene, b: R.TraversalBvh, wide: bool, max_leaf: int):
    n = scene.n_triangles
    lo_t, hi_t = expanded_boxes(scene)
    rank = ref_ranks(scene)
    seen = np.zeros(n, np.int32)
    per = 28 if wide else 16
    refs_at = (24, 28) if wide else (12, 14)

    def children(node):
        row = b.nodes[node]
        refs = row[refs_at[0]:refs_at[1]].view(np.int32)
        out = []
        for k, r in enumerate(refs):
            if wide and r == EMPTY:
                continue
            if wide:
                lo = np.array([row[8 * a + k] for a in range(3)])
                hi = np.array([row[8 * a + 4 + k] for a in range(3)])
            else:
                lo = np.array([row[4 * k], row[4 * k + 2], row[8 + 2 * k]])
                hi = np.array([row[4 * k + 1], row[4 * k + 3], row[9 + 2 * k]])
            out.append((int(r), lo, hi))
        return out

    def leaf_range(r):
        enc = ~r & 0xFFFFFFFF
        return enc & ((1 << LEAF_BITS) - 1), (enc >> LEAF_BITS) + 1

    def visit_leaf(r, lo, hi):
        first, cnt = leaf_range(r)
        assert 1 <= cnt <= max_leaf
        tris = b.leaf_tri[first:first + cnt]
        seen[tris] += 1
        assert np.all(np.diff(rank[tris].astype(np.int64)) > 0), "leaf not in reference-rank order"
        if lo is not None:
            assert np.all(lo_t[tris] >= lo) and np.all(hi_t[tris] <= hi), "leaf box does not bound its triangles"
        assert np.array_equal(b.trirec[first:first + cnt, 7].view(np.uint32), rank[tris])

    order = []
    if b.root < 0:
        visit_leaf(b.root, None, None)
    else:
        stack = [(b.root, None, None)]
        while stack:
            node, lo, hi = stack.pop()
            order.append(node)
            kids = children(node)
            assert len(kids) >= 2
            for r, clo, chi in kids:
                if lo is not None:
                    assert np.all(clo >= lo) and np.all(chi <= hi), "child box outside its parent's"
            for r, clo, chi in reversed(kids):
                if r >= 0:
                    stack.append((r, clo, chi))
                else:
                    visit_leaf(r, clo, chi)
        assert order == list(range(len(b.nodes))), "nodes are not numbered in pre-order"
    assert np.all(seen == 1), "a triangle is missing from the leaves or repeated"
    assert b.nodes.shape[1] == per


@pytest.mark.parametrize("wide", [False, True])
@pytest.mark.parametrize("max_leaf", [1, 4, 16])
def test_host_tree_structure(wide, max_leaf):
    for scene in (random_soup(3000, 2), coincident_soup(300, 200), grid_soup(24)):
        b = R.traversal_bvh(scene, max_leaf, wide, -1)
        check_tree(scene, b, wide, max_leaf)


def test_host_tree_generated_scene():
    scene = P.SceneData.generate(A.PHX_SCENE_CAUSTIC, 1, 64, 64, detail=16)
    check_tree(scene, R.traversal_bvh(scene, 4, True, -1), True, 4)


def decode_qnodes(q: np.ndarray):
    """8-bit nodes -> (lo, hi) per child (float64, exact) and refs, for the containment check."""
    w = q.view(np.uint32)
    P = w[:, 0:3].view(np.float32).astype(np.float64)
    e = np.stack([(w[:, 3] >> (8 * a)) & 0xFF for a in range(3)], 1).astype(np.int64) - 127
    step = np.ldexp(1.0, e)
    lo = np.zeros((len(w), 4, 3))
    hi = np.zeros((len(w), 4, 3))
    for a in range(3):
        for k in range(4):
            lo[:, k, a] = P[:, a] + ((w[:, 4 + 2 * a] >> (8 * k)) & 0xFF) * step[:, a]
            hi[:, k, a] = P[:, a] + ((w[:, 5 + 2 * a] >> (8 * k)) & 0xFF) * step[:, a]
    return lo, hi, w[:, 12:16].view(np.int32), step


@pytest.mark.parametrize("scene_fn", [lambda: random_soup(4000, 9, scale=30.0, size=0.02),
                                      lambda: coincident_soup(300, 500),
                                      lambda: P.SceneData.generate(A.PHX_SCENE_ATRIUM, 1, 64, 64, detail=16)])
def test_quantized_nodes_contain_the_exact_boxes(scene_fn):
    """Every 8-bit child box contains its float box (rounded outward by less than one step), and
    the quantised tree has the 4-wide tree's topology."""
    scene = scene_fn()
    w = R.traversal_bvh(scene, 4, 1, -1)
    q = R.traversal_bvh(scene, 4, 2, -1)
    assert (q.root, q.depth, q.wdepth) == (w.root, w.depth, w.wdepth)
    assert np.array_equal(q.trirec.view(np.uint32), w.trirec.view(np.uint32))
    lo_q, hi_q, refs, step = decode_qnodes(q.nodes)
    refs_w = w.nodes[:, 24:28].view(np.int32)
    assert np.array_equal(refs, refs_w)
    valid = refs_w != EMPTY
    for a in range(3):
        lo_w = w.nodes[:, 8 * a:8 * a + 4].astype(np.float64)
        hi_w = w.nodes[:, 8 * a + 4:8 * a + 8].astype(np.float64)
        assert np.all(lo_q[:, :, a][valid] <= lo_w[valid])
        assert np.all(hi_q[:, :, a][valid] >= hi_w[valid])
        s = np.broadcast_to(step[:, a:a + 1], lo_w.shape)
        assert np.all(lo_w[valid] - lo_q[:, :, a][valid] < s[valid])
        assert np.all(hi_q[:, :, a][valid] - hi_w[valid] < s[valid])


def test_traversal_build_rejects_bad_input():
    scene = random_soup(10)
    with pytest.raises(A.PhxError):
        R.traversal_bvh(scene, 0, 1, -1)
    with pytest.raises(A.PhxError):
        R.traversal_bvh(scene, 17, 1, -1)


# ---- GPU: the device build --------------------------------------------------------------------

def gpu_cases():
    return {
        "one": lambda: random_soup(1, 3),
        "two": lambda: random_soup(2, 4),
        "soup_5k": lambda: random_soup(5000, 5),
        "soup_40k_thin": lambda: random_soup(40000, 6, scale=50.0, size=0.05),
        # > 2048 coincident centroids: the chunked (large-task) object-median path
        "coincident_big": lambda: coincident_soup(5000, 3000),
        "coincident_small": lambda: coincident_soup(70, 40),
        "grid": lambda: grid_soup(128),
        "cornell": lambda: P.SceneData.generate(A.PHX_SCENE_CORNELL, 1, 64, 64),
        "caustic": lambda: P.SceneData.generate(A.PHX_SCENE_CAUSTIC, 1, 1024, 1024),
        "atrium": lambda: P.SceneData.generate(A.PHX_SCENE_ATRIUM, 1, 1920, 1080),
    }


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(gpu_cases()))
def test_device_tree_equals_host(name):
    scene = gpu_cases()[name]()
    for wide, max_leaf in ((1, 4), (0, 4), (1, 1), (0, 16), (2, 4)):
        h = R.traversal_bvh(scene, max_leaf, wide, -1)
        d = R.traversal_bvh(scene, max_leaf, wide, 0)
        tag = f"{name} wide={wide} leaf={max_leaf}"
        assert (d.root, d.depth, d.wdepth) == (h.root, h.depth, h.wdepth), tag
        assert d.nodes.shape == h.nodes.shape, tag
        assert np.array_equal(d.nodes.view(np.uint32), h.nodes.view(np.uint32)), tag
        assert np.array_equal(d.trirec.view(np.uint32), h.trirec.view(np.uint32)), tag
        assert np.array_equal(d.leaf_tri, h.leaf_tri), tag
        if name in ("caustic", "atrium"):
            print(f"{tag}: {scene.n_triangles} triangles, host {h.build_ms:.1f} ms, device {d.build_ms:.1f} ms")


RENDER = {
    # name: (kind, detail, width, height, photons, bounces, grid)
    "cornell": (A.PHX_SCENE_CORNELL, 0, 64, 64, 1 << 14, 8, 50),
    "caustic": (A.PHX_SCENE_CAUSTIC, 0, 96, 80, 1 << 15, 12, 50),
    "atrium": (A.PHX_SCENE_ATRIUM, 16, 96, 54, 1 << 14, 16, 64),
}


def render(name, flags, rounds=3):
    kind, detail, w, h, ph, mb, g = RENDER[name]
    scene = P.SceneData.generate(kind, seed=1, width=w, height=h, detail=detail)
    args = P.ArgsList(width=w, height=h, photons_per_round=ph, max_photon_bounces=mb, grid_res=g, seed=3,
                      direct_samples=4, flags=flags)
    with P.Renderer(args) as r:
        r.set_scene(scene)
        r.iterate(rounds)
        info = r.info()
        return r.read("RADIANCE"), r.read("FLUX"), info


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(RENDER))
@pytest.mark.parametrize("extra", [0, A.PHX_F_BINARY_BVH, A.PHX_F_QUANT_BVH])
def test_device_tree_renders_identically(name, extra):
    rad_h, flux_h, ih = render(name, extra | A.PHX_F_HOST_BVH)
    rad_d, flux_d, idv = render(name, extra)
    assert (idv.trav_depth, idv.trav_inner_nodes) == (ih.trav_depth, ih.trav_inner_nodes)
    assert idv.stack_overflows == ih.stack_overflows == 0
    assert np.array_equal(rad_d.view(np.uint32), rad_h.view(np.uint32))
    assert np.array_equal(flux_d.view(np.uint32), flux_h.view(np.uint32))
    assert idv.bvh_build_ms > 0.0 and idv.setup_ms >= idv.bvh_build_ms


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(RENDER))
def test_quantized_nodes_render_identically(name):
    """8-bit child boxes only prune less tightly: every image equals the float-box render."""
    rad_h, flux_h, ih = render(name, 0)
    rad_q, flux_q, iq = render(name, A.PHX_F_QUANT_BVH | A.PHX_F_HOST_BVH)
    assert iq.stack_overflows == 0
    assert np.array_equal(rad_q.view(np.uint32), rad_h.view(np.uint32))
    assert np.array_equal(flux_q.view(np.uint32), flux_h.view(np.uint32))


@pytest.mark.gpu
def test_device_tree_in_a_batch():
    specs = [("cornell", 0), ("caustic", 0), ("atrium", 0)]
    out = {}
    for flags in (A.PHX_F_HOST_BVH, 0):
        scenes, args = [], []
        for name, _ in specs:
            kind, detail, w, h, ph, mb, g = RENDER[name]
            scenes.append(P.SceneData.generate(kind, seed=2, width=w, height=h, detail=detail))
            args.append(P.ArgsList(width=w, height=h, photons_per_round=ph, max_photon_bounces=mb, grid_res=g,
                                   seed=5, direct_samples=4, flags=flags))
        b = P.Batch(scenes, args)
        b.iterate(2)
        out[flags] = [b.read(i, "RADIANCE") for i in range(len(specs))]
        b.close()
    for a, d in zip(out[A.PHX_F_HOST_BVH], out[0]):
        assert np.array_equal(a.view(np.uint32), d.view(np.uint32))


def _slab_inv(d, o):
    """The kernels' inverse direction component: 1/d, with +-1e30 for a zero component while |o| < 1e4."""
    with np.errstate(divide="ignore"):
        r = np.float32(1.0) / d
    return np.where(np.isinf(r) & (np.abs(o) < 1e4), np.copysign(np.float32(1e30), r), r).astype(np.float32)


@pytest.mark.parametrize("scene_fn", [lambda: random_soup(3000, 2), lambda: grid_soup(24),
                                      lambda: P.SceneData.generate(A.PHX_SCENE_CAUSTIC, 1, 64, 64, detail=16)])
def test_empty_slots_are_never_entered(scene_fn):
    """The 4-wide traversal skips the reference check of an empty child slot in its slab test and
    checks the reference only where a child is stacked or entered.  That relies on every empty slot
    carrying the box (1e30, -1e30), which the sign-selected slab test (float32, fused multiply-add,
    NaN slabs ignored) never enters: checked for random, axis-aligned and far-away rays."""
    b = R.traversal_bvh(scene_fn(), 4, True, -1)
    nodes = b.nodes.reshape(-1, 7, 4)
    refs = nodes[:, 6, :].view(np.int32)
    empty = refs == EMPTY
    assert empty.any(), "the tree has no empty slot to check"
    lo, hi = nodes[:, 0:6:2, :], nodes[:, 1:6:2, :]  # rows minx, miny, minz / maxx, maxy, maxz
    assert np.all(lo[np.broadcast_to(empty[:, None, :], lo.shape)] == np.float32(1e30))
    assert np.all(hi[np.broadcast_to(empty[:, None, :], hi.shape)] == np.float32(-1e30))
    rng = np.random.default_rng(5)
    n = 20000
    for scale in (1.0, 1e3, 1e4, 1e5, 1e20):
        o = (rng.uniform(-1, 1, (n, 3)) * scale).astype(np.float32)
        d = rng.uniform(-1, 1, (n, 3)).astype(np.float32)
        d[0::5, 0] = 0.0
        d[1::5, :2] = 0.0
        d[2::5, 2] = -0.0
        d /= np.linalg.norm(d, axis=1, keepdims=True).astype(np.float32)
        inv = _slab_inv(d, o)
        oi = (o * inv).astype(np.float32)
        with np.errstate(invalid="ignore", over="ignore"):
            # an empty slot's entry plane is 1e30 for a positive inverse component and -1e30 for a
            # negative one, its exit plane the other; distances plane * inv - o * inv in float32
            near = np.where(inv >= 0, np.float32(1e30), np.float32(-1e30)).astype(np.float32)
            far = np.where(inv >= 0, np.float32(-1e30), np.float32(1e30)).astype(np.float32)
            tn = (near.astype(np.float64) * inv - oi).astype(np.float32)  # fma rounding: one rounding
            tf = (far.astype(np.float64) * inv - oi).astype(np.float32)
        tn = np.fmax(np.fmax(np.fmax(tn[:, 0], tn[:, 1]), tn[:, 2]), np.float32(1e-5))
        tf = np.fmin(np.fmin(np.fmin(tf[:, 0], tf[:, 1]), tf[:, 2]), np.float32(np.inf))
        assert not np.any(tn <= tf), f"an empty slot's box is entered (origin scale {scale})"
