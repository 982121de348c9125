"""Host-side logic and the C ABI, on CPU: library exports, struct layouts, the BVH builder, hash
grid, camera, light prefix sums, procedural scenes, and error reporting without a device."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle as O
import phosphor_b200 as P
from phosphor_b200 import _capi as A

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    text = (ROOT / "include" / "phx.h").read_text()
    return sorted(set(re.findall(r"PHX_API\s+[\w\s\*]+?\b(phx_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = A.load()
    names = declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the ctypes mirror declares exactly those entry points
    assert sorted(n for n, _, _ in A.PROTOTYPES) == names


def test_struct_sizes_match_reference_layouts():
    for t, size in A.SIZES.items():
        assert C.sizeof(t) == size, t.__name__
    assert A.Scene.camera.offset == 128
    assert A.Info.hash.offset == 64


@pytest.mark.parametrize("kind,tris", [(0, 12), (1, 149862), (2, 262898)])
def test_scene_generators(kind, tris):
    s = P.SceneData.generate(kind, seed=1, width=256, height=256)
    assert s.n_triangles == tris
    assert s.scene.n_lights >= 1
    m = s.materials()
    assert len(m) == s.scene.n_materials
    t = s.triangles()
    assert int(t["mat_index"].max()) < s.scene.n_materials


def test_scene_generation_is_deterministic():
    a = P.SceneData.generate(1, seed=7, width=64, height=64)
    b = P.SceneData.generate(1, seed=7, width=64, height=64)
    c = P.SceneData.generate(1, seed=8, width=64, height=64)
    assert a.triangles().tobytes() == b.triangles().tobytes()
    assert a.triangles().tobytes() != c.triangles().tobytes()


@pytest.mark.parametrize("kind", [0, 1])
def test_bvh_builder_matches_oracle(kind):
    s = P.SceneData.generate(kind, seed=1, width=64, height=64)
    nodes, depth = P.bvh_build(s)
    onodes, odepth = O.bvh_build(C.cast(s.scene.triangles, C.c_void_p).value, s.n_triangles)
    assert np.array_equal(nodes.view(np.uint32), onodes.view(np.uint32))
    assert depth == odepth
    assert depth < 22  # the reference's 24-entry stack never drops a subtree (hit.h:163-164)


def test_bvh_structure():
    s = P.SceneData.generate(1, seed=1, width=64, height=64)
    nodes, _ = P.bvh_build(s)
    u = nodes.view(np.uint32)
    n = s.n_triangles
    assert len(nodes) == 2 * n - 1
    leaves = u[:, 3] != 0xFFFFFFFF
    assert leaves.sum() == n
    assert sorted(u[leaves, 3].tolist()) == list(range(n))  # every triangle in exactly one leaf
    inner = np.nonzero(~leaves)[0]
    right = u[inner, 7]
    assert np.all(right > inner) and np.all(right < len(nodes))
    # children boxes are inside their parent
    for i in inner[:2000]:
        for c in (i + 1, right[np.searchsorted(inner, i)]):
            assert np.all(nodes[c, 0:3] >= nodes[i, 0:3]) and np.all(nodes[c, 4:7] <= nodes[i, 4:7])


def test_hash_info_matches_oracle():
    s = P.SceneData.generate(0, seed=1, width=64, height=64)
    nodes, _ = P.bvh_build(s)
    lib = A.load()
    hd = A.PhotonHashData()
    root = A.BvhNode.from_buffer_copy(nodes[0].tobytes())
    A.check(lib.phx_hash_info(C.byref(root), 50, C.byref(hd)))
    assert bytes(hd) == O.hash_info(nodes[0], 50)
    assert hd.grid_res == 50
    # 0.5/50 of the (1e-3 expanded) unit box: the initial radius is 0.01 of the scene diagonal
    assert hd.cell_sizes.x == pytest.approx(1.002 / 50, rel=1e-6)


def test_camera_basis():
    cam = P.camera_make([0.5, 0.5, 2.4], [0.5, 0.5, 0.0], [0, 1, 0], 40.0, 1.0)
    h = np.array([cam.horizontal.x, cam.horizontal.y, cam.horizontal.z])
    v = np.array([cam.vertical.x, cam.vertical.y, cam.vertical.z])
    assert np.dot(h, v) == pytest.approx(0.0, abs=1e-6)
    assert np.linalg.norm(h) == pytest.approx(2 * np.tan(np.radians(20.0)), rel=1e-5)  # focus distance 1
    ll = np.array([cam.lower_left_corner.x, cam.lower_left_corner.y, cam.lower_left_corner.z])
    centre = ll + 0.5 * h + 0.5 * v
    assert centre == pytest.approx([0.5, 0.5, 1.4], abs=1e-6)


def test_lum_pref_sum():
    lights = (A.Light * 3)()
    for i, p in enumerate([(1, 0, 0), (0, 2, 0), (-5, -5, -5)]):
        lights[i].power.x, lights[i].power.y, lights[i].power.z = p
    out = (C.c_float * 3)()
    A.check(A.load().phx_lum_pref_sum(lights, 3, out))
    assert list(out) == pytest.approx([0.2126, 0.2126 + 2 * 0.7152, 0.2126 + 2 * 0.7152], rel=1e-6)


def test_errors_are_status_codes():
    lib = A.load()
    assert lib.phx_destroy(None) == A.PHX_E_INVALID
    assert b"null" in lib.phx_last_error()
    assert lib.phx_round(None) == A.PHX_E_INVALID
    assert lib.phx_iterate(None, 1) == A.PHX_E_INVALID
    s = P.SceneData.generate(0, seed=1, width=8, height=8)
    ctx = C.c_void_p()
    bad = P.ArgsList(width=8, height=8, max_photon_bounces=0).params()
    assert lib.phx_create(C.byref(s.scene), C.byref(bad), 0, C.byref(ctx)) == A.PHX_E_INVALID
    assert b"max_photon_bounces" in lib.phx_last_error()
    bad = P.ArgsList(width=8, height=8, grid_res=256).params()
    assert lib.phx_create(C.byref(s.scene), C.byref(bad), 0, C.byref(ctx)) == A.PHX_E_INVALID
    bad = P.ArgsList(width=8, height=8, direct_samples=0).params()
    assert lib.phx_create(C.byref(s.scene), C.byref(bad), 0, C.byref(ctx)) == A.PHX_E_INVALID
    # degenerate triangle: all three vertices equal is fine (boxes are expanded); an infinity is not
    t = s.triangles().copy()
    t[0]["v0"]["x"] = np.inf
    sc = A.Scene.from_buffer_copy(s.scene)
    sc.triangles = t.ctypes.data_as(C.POINTER(A.Triangle))
    good = P.ArgsList(width=8, height=8).params()
    code = lib.phx_create(C.byref(sc), C.byref(good), 0, C.byref(ctx))
    assert code in (A.PHX_E_INVALID, A.PHX_E_CUDA)  # CUDA first when no device is present
    assert ctx.value is None


def test_png_writer(tmp_path):
    img = (np.arange(4 * 5 * 3) % 256).astype(np.uint8).reshape(4, 5, 3)
    p = tmp_path / "x.png"
    P.write_png(p, img)
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n" and b"IHDR" in data and data.endswith(b"IEND\xaeB`\x82")
