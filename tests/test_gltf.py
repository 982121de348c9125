"""glTF 2.0 scene ingest (phx_scene_load_gltf; the reference's read_gltf_scene, scene.cpp:206-233).

The reference's .glb assets are Git-LFS stubs here and assimp is absent, so the loader is checked
on documents written by tests/gltf_writer.py: a generated scene exported and read back gives the
same triangles, materials, emissive light and camera; node hierarchies transform positions,
normals, cameras and lights as glTF defines; the three punctual light kinds take the reference's
power (colour · intensity / 683) and directions; PNG textures of every colour type decode to the
8-bit RGB the reference's loader produces; strips and fans triangulate as glTF specifies; .glb,
.gltf with a .bin file and .gltf with a data URI read the same; malformed input is an error, not a
crash.  A GPU test renders a loaded scene and checks it against the oracle.
"""
import math

import numpy as np
import pytest

import oracle as O
import phosphor_b200 as P
from phosphor_b200 import _capi as A

from gltf_writer import Gltf, png_bytes


def f3(v):
    return np.array([v["x"], v["y"], v["z"]], np.float64)


def tris_array(scene) -> np.ndarray:
    t = scene.triangles()
    raw = np.frombuffer(t.tobytes(), np.float32).reshape(len(t), 44)
    return raw


def export_generated(scene, g: Gltf, hfov: float, aspect: float, cam_pos) -> None:
    """One primitive per material of a generated scene, the camera as a node looking along -z."""
    t = scene.triangles()
    mats = scene.materials()
    for mi in range(len(mats)):
        sel = np.flatnonzero(t["mat_index"] == mi)
        if len(sel) == 0:
            continue
        pos = np.stack([np.stack([t[v][c][sel] for c in "xyz"], 1) for v in ("v0", "v1", "v2")], 1).reshape(-1, 3)
        nrm = np.stack([np.stack([t[v][c][sel] for c in "xyz"], 1) for v in ("n0", "n1", "n2")], 1).reshape(-1, 3)
        m = mats[mi]
        mat = g.material(pbrMetallicRoughness={"baseColorFactor": [float(m["base_color"][c]) for c in "xyzw"],
                                               "metallicFactor": float(m["metallic"]),
                                               "roughnessFactor": float(m["roughness"])},
                         emissiveFactor=[float(m["emissive"][c]) for c in "xyz"] if m["emissive"]["x"] <= 1 else [1, 1, 1],
                         **({"extensions": {"KHR_materials_emissive_strength": {"emissiveStrength":
                                                                                float(m["emissive"]["x"])}}}
                            if m["emissive"]["x"] > 1 else {}))
        mesh = g.mesh([{"attributes": {"POSITION": g.accessor(pos), "NORMAL": g.accessor(nrm)}, "material": mat}])
        g.node(mesh=mesh)
    yfov = 2 * math.atan(math.tan(math.radians(hfov) / 2) / aspect)
    g.node(camera=g.camera(yfov, aspect), translation=list(cam_pos))


def test_generated_cornell_box_round_trip(tmp_path):
    w, h = 64, 48
    src = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=w, height=h)
    g = Gltf()
    export_generated(src, g, 40.0, w / h, (0.5, 0.5, 2.4))
    g.write_glb(tmp_path / "cornell.glb")
    got = P.SceneData.load_gltf(tmp_path / "cornell.glb", width=w, height=h)
    a, b = tris_array(src), tris_array(got)
    assert a.shape == b.shape
    # positions exactly, normals within rounding of the renormalisation
    order_src = np.lexsort(a[:, :12].T)
    order_got = np.lexsort(b[:, :12].T)
    assert np.array_equal(a[order_src, :12], b[order_got, :12])
    assert np.allclose(a[order_src, 12:24], b[order_got, 12:24], atol=1e-6)
    # tangents without UVs: the reference's face-tangent fallback, (1, 0, 0)
    assert np.allclose(b[:, 24:36].reshape(-1, 3, 4)[:, :, :3], [1, 0, 0])
    # one material per primitive with the exported factors; the light quad's emission and area light
    mats = got.materials()
    assert len(mats) == len(src.materials())
    assert np.allclose([m["base_color"]["x"] for m in mats], [m["base_color"]["x"] for m in src.materials()])
    lt_src, lt_got = src.lights(), got.lights()
    assert len(lt_got) == 1 and lt_got[0]["kind"] == A.PHX_LIGHT_TEXTURED
    assert np.allclose([lt_got[0]["power"][c] for c in "xyz"], [lt_src[0]["power"][c] for c in "xyz"], rtol=1e-6)
    assert got.scene.n_emissive_triangles == 2
    cam_src = np.frombuffer(bytes(src.scene.camera), np.float32)[:26]
    cam_got = np.frombuffer(bytes(got.scene.camera), np.float32)[:26]
    assert np.allclose(cam_src, cam_got, atol=2e-5)


def test_node_transforms_of_meshes_cameras_and_lights(tmp_path):
    g = Gltf()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    nrm = np.array([[0, 0, 1]] * 3, np.float32)
    mesh = g.mesh([{"attributes": {"POSITION": g.accessor(pos), "NORMAL": g.accessor(nrm)}}])
    ang = 0.7
    q = [0.0, math.sin(ang / 2), 0.0, math.cos(ang / 2)]  # rotation about +y
    child = g.node(root=False, mesh=mesh, translation=[0.0, 2.0, 0.0], scale=[2.0, 3.0, 1.0])
    g.node(children=[child], rotation=q, translation=[1.0, 0.0, -1.0])
    lt = g.light(type="spot", color=[1.0, 0.5, 0.25], intensity=683.0, spot={"innerConeAngle": 0.2,
                                                                              "outerConeAngle": 0.5})
    g.node(extensions={"KHR_lights_punctual": {"light": lt}}, rotation=q, translation=[0.0, 3.0, 0.0])
    g.node(camera=g.camera(0.8, 1.5), matrix=[1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0.0, 1.0, 5.0, 1])
    g.write_glb(tmp_path / "xf.glb")
    sc = P.SceneData.load_gltf(tmp_path / "xf.glb")
    # expected: parent (T R) * child (T S)
    c, s = math.cos(ang), math.sin(ang)
    R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]])
    world = [(R @ (np.array([2.0, 3.0, 1.0]) * p + [0, 2, 0])) + [1, 0, -1] for p in pos]
    t = sc.triangles()[0]
    for v, want in zip(("v0", "v1", "v2"), world):
        assert np.allclose(f3(t[v]), want, atol=1e-5)
    n_want = R @ np.linalg.inv(np.diag([2.0, 3.0, 1.0])).T @ [0, 0, 1]
    assert np.allclose(f3(t["n0"]), n_want / np.linalg.norm(n_want), atol=1e-6)
    l = sc.lights()[0]
    assert l["kind"] == A.PHX_LIGHT_SPOT
    assert np.allclose(f3(l["power"]), [1.0, 0.5, 0.25], rtol=1e-6)  # colour * intensity / 683
    assert np.allclose(f3(l["position"]), [0, 3, 0]) and np.allclose(f3(l["direction"]), R @ [0, 0, -1], atol=1e-6)
    assert l["aux"]["x"] == pytest.approx(0.2) and l["aux"]["y"] == pytest.approx(0.5)
    # the camera: position (0, 1, 5), looking along -z, hfov = 2 atan(aspect tan(yfov / 2))
    hfov = 2 * math.atan(1.5 * math.tan(0.4))
    want = np.frombuffer(O.camera_make((0, 1, 5), (0, 1, 4), (0, 1, 0), math.degrees(hfov), 1.5), np.float32)
    assert np.allclose(np.frombuffer(bytes(sc.scene.camera), np.float32)[:26], want[:26], atol=1e-5)


def test_point_and_directional_lights_and_defaults(tmp_path):
    g = Gltf()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    g.node(mesh=g.mesh([{"attributes": {"POSITION": g.accessor(pos)}}]))
    p = g.light(type="point", color=[0.2, 0.4, 0.8], intensity=100.0)
    d = g.light(type="directional")  # colour 1, intensity 1
    sp = g.light(type="spot")        # cone angles default to 0 and pi/4
    q = [math.sin(-math.pi / 4), 0.0, 0.0, math.cos(-math.pi / 4)]  # -90 deg about x: -z -> -y
    g.node(extensions={"KHR_lights_punctual": {"light": p}}, translation=[1, 2, 3])
    g.node(extensions={"KHR_lights_punctual": {"light": d}}, rotation=q)
    g.node(extensions={"KHR_lights_punctual": {"light": sp}})
    g.node(camera=g.camera(0.9, 1.0), translation=[0, 0, 3])
    g.write_glb(tmp_path / "lights.glb")
    sc = P.SceneData.load_gltf(tmp_path / "lights.glb", width=32, height=32)
    l = sc.lights()
    assert list(l["kind"]) == [A.PHX_LIGHT_POINT, A.PHX_LIGHT_DIRECTIONAL, A.PHX_LIGHT_SPOT]
    assert np.allclose(f3(l[0]["power"]), np.float32([0.2, 0.4, 0.8]) * np.float32(100.0) / np.float32(683.0))
    assert np.allclose(f3(l[0]["position"]), [1, 2, 3])
    assert np.allclose(f3(l[1]["direction"]), [0, -1, 0], atol=1e-6)
    # the directional light's disk frame (make_tbn, utils.h:45-55): orthonormal, perpendicular
    tt, bb = f3(l[1]["tangent"]), f3(l[1]["bitangent"])
    assert abs(np.dot(tt, [0, -1, 0])) < 1e-6 and abs(np.linalg.norm(tt) - 1) < 1e-6 and abs(np.dot(tt, bb)) < 1e-6
    assert l[2]["aux"]["x"] == 0.0 and l[2]["aux"]["y"] == pytest.approx(math.pi / 4)
    # materials: no material -> the reference's default (metallic 0, roughness 1, ior 1.5)
    m = sc.materials()[0]
    assert m["metallic"] == 0.0 and m["roughness"] == 1.0 and m["ior"] == pytest.approx(1.5)
    lum = np.ctypeslib.as_array(sc.scene.lum_pref_sum, shape=(3,))
    assert np.all(np.diff(lum) >= 0) and lum[-1] > 0


def test_materials_textures_and_uv_transforms(tmp_path):
    rng = np.random.default_rng(3)
    imgs = {
        "rgb": rng.integers(0, 256, (5, 7, 3)).astype(np.uint8),
        "rgba": rng.integers(0, 256, (4, 6, 4)).astype(np.uint8),
        "grey": rng.integers(0, 256, (3, 9)).astype(np.uint8),
        "grey_alpha": rng.integers(0, 256, (6, 2, 2)).astype(np.uint8),
        "rgb16": rng.integers(0, 65536, (4, 4, 3)).astype(np.uint16),
    }
    pal = rng.integers(0, 256, (16, 3)).astype(np.uint8)
    pidx = rng.integers(0, 16, (5, 5)).astype(np.uint8)
    g = Gltf()
    tex = {k: g.image_png(png_bytes(v), embed="view" if i % 2 else "uri") for i, (k, v) in enumerate(imgs.items())}
    tex["palette"] = g.image_png(png_bytes(pidx, palette=pal))
    g.doc["images"].append({"uri": "missing.jpg"})  # not loadable: skipped
    g.doc["textures"].append({"source": len(g.doc["images"]) - 1})
    tex["missing"] = len(g.doc["textures"]) - 1
    xf = {"KHR_texture_transform": {"offset": [0.25, -0.5], "scale": [2.0, 0.5], "rotation": 0.3}}
    mat = g.material(
        pbrMetallicRoughness={"baseColorFactor": [0.5, 0.6, 0.7, 1.0], "baseColorTexture": {"index": tex["rgb"],
                                                                                          "extensions": xf},
                              "metallicRoughnessTexture": {"index": tex["grey"]}, "metallicFactor": 0.25,
                              "roughnessFactor": 0.75},
        normalTexture={"index": tex["rgba"]}, occlusionTexture={"index": tex["grey_alpha"]},
        emissiveTexture={"index": tex["palette"]}, emissiveFactor=[0.0, 0.0, 0.0],
        extensions={"KHR_materials_transmission": {"transmissionFactor": 0.4,
                                                   "transmissionTexture": {"index": tex["rgb16"]}},
                    "KHR_materials_ior": {"ior": 1.33},
                    "KHR_materials_volume": {"thicknessFactor": 0.2, "attenuationDistance": 0.8,
                                             "attenuationColor": [0.9, 0.8, 0.7]}})
    mat2 = g.material(pbrMetallicRoughness={"baseColorTexture": {"index": tex["missing"]}})
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    uv = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]], np.float32)
    acc_p, acc_uv = g.accessor(pos), g.accessor(uv)
    g.node(mesh=g.mesh([{"attributes": {"POSITION": acc_p, "TEXCOORD_0": acc_uv}, "material": mat},
                        {"attributes": {"POSITION": acc_p}, "material": mat2}]))
    g.node(camera=g.camera(0.9, 1.0), translation=[0, 0, 3])
    g.write_glb(tmp_path / "tex.glb")
    sc = P.SceneData.load_gltf(tmp_path / "tex.glb")
    s = sc.scene
    # atlas order: per material base colour, emissive, normal, occlusion, metal-rough, transmission
    order = ["rgb", "palette", "rgba", "grey_alpha", "grey", "rgb16"]
    assert s.n_textures == len(order)
    meta = np.ctypeslib.as_array(s.tex_meta, shape=(s.n_textures,))
    atlas = np.ctypeslib.as_array(s.tex_atlas, shape=(s.tex_atlas_bytes,))

    def rgb8(k):
        im = pal[pidx] if k == "palette" else imgs[k]
        if im.ndim == 2:
            im = np.repeat(im[:, :, None], 3, axis=2)
        elif im.shape[2] == 2:
            im = np.repeat(im[:, :, :1], 3, axis=2)
        if im.dtype == np.uint16:
            im = (im >> 8).astype(np.uint8)
        return im[:, :, :3].reshape(-1)

    for i, k in enumerate(order):
        m = meta[i]
        want = rgb8(k)
        assert m["channels"] == 3 and m["width"] * m["height"] * 3 == len(want)
        assert np.array_equal(atlas[m["atlas_offset"]:m["atlas_offset"] + len(want)], want), k
    m0, m1 = sc.materials()
    assert (m0["diff_index"], m0["emis_index"], m0["norm_index"], m0["occlusion_index"], m0["metal_rough_index"],
            m0["transmission_index"]) == (0, 1, 2, 3, 4, 5)
    assert m0["metallic"] == pytest.approx(0.25) and m0["roughness"] == pytest.approx(0.75)
    assert m0["transmission"] == pytest.approx(0.4) and m0["ior"] == pytest.approx(1.33)
    assert m0["thickness"] == pytest.approx(0.2) and m0["att_dist"] == pytest.approx(0.8)
    assert m1["diff_index"] == A.PHX_NO_TEXTURE  # the image could not be loaded
    assert len(sc.lights()) == 0  # emission 0: no area light
    # UVs flipped to (u, 1 - v); the base-colour transform maps them so that the reference's
    # sampler (R(rot) S uv + offset, then v -> 1 - v) lands where KHR_texture_transform puts the
    # glTF coordinate
    t = sc.triangles()[0]
    assert (t["uv1"]["x"], t["uv1"]["y"], t["uv2"]["y"]) == (1.0, 1.0, 0.0)
    ut = np.frombuffer(bytes(s.uv_transforms[0].diff), np.float32)[:5]
    off, scl, rot = ut[0:2], ut[2:4], ut[4]
    for u, v in rng.uniform(-1, 2, (20, 2)):
        U, V = u, 1.0 - v
        sx, sy = U * scl[0], V * scl[1]
        ref = (math.cos(rot) * sx - math.sin(rot) * sy + off[0], math.sin(rot) * sx + math.cos(rot) * sy + off[1])
        r = 0.3
        gl = (math.cos(r) * 2.0 * u + math.sin(r) * 0.5 * v + 0.25, -math.sin(r) * 2.0 * u + math.cos(r) * 0.5 * v - 0.5)
        assert ref[0] == pytest.approx(gl[0], abs=1e-5) and 1.0 - ref[1] == pytest.approx(gl[1], abs=1e-5)


def test_strips_fans_and_containers_read_the_same(tmp_path):
    g = Gltf()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0], [0, 2, 0]], np.float32)
    ap = g.accessor(pos)
    strip = g.accessor(np.array([0, 1, 2, 3, 4], np.uint16), 5123)
    fan = g.accessor(np.array([0, 1, 3, 4], np.uint8), 5121)
    lines = g.accessor(np.array([0, 1], np.uint32), 5125)
    g.node(mesh=g.mesh([{"attributes": {"POSITION": ap}, "indices": strip, "mode": 5},
                        {"attributes": {"POSITION": ap}, "indices": fan, "mode": 6},
                        {"attributes": {"POSITION": ap}, "indices": lines, "mode": 1}]))
    g.node(camera=g.camera(0.9, 1.0), translation=[0, 0, 3])
    g.write_glb(tmp_path / "a.glb")
    g.write_gltf(tmp_path / "b.gltf")
    g.write_gltf(tmp_path / "c.gltf", data_uri=True)
    scenes = [P.SceneData.load_gltf(tmp_path / n) for n in ("a.glb", "b.gltf", "c.gltf")]
    t = scenes[0].triangles()
    idx = [[int(round(f3(tr[v])[0] + 2 * f3(tr[v])[1])) for v in ("v0", "v1", "v2")] for tr in t]
    code = {0: 0, 1: 1, 2: 2, 3: 3, 4: 4}
    # vertex i has x + 2y = (0, 1, 2, 3, 4)
    assert [[code[i] for i in tri] for tri in idx] == [[0, 1, 2], [2, 1, 3], [2, 3, 4], [1, 3, 0], [3, 4, 0]]
    for s in scenes[1:]:
        assert np.array_equal(s.triangles().view(np.uint8), scenes[0].triangles().view(np.uint8))


@pytest.mark.parametrize("case", ["missing", "not_json", "no_camera", "bad_index", "no_triangles", "truncated"])
def test_malformed_input_is_an_error(tmp_path, case):
    path = tmp_path / "x.glb"
    g = Gltf()
    pos = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    prim = {"attributes": {"POSITION": g.accessor(pos)}}
    if case == "bad_index":
        prim["indices"] = g.accessor(np.array([0, 1, 7], np.uint32), 5125)
    if case != "no_triangles":
        g.node(mesh=g.mesh([prim]))
    if case != "no_camera":
        g.node(camera=g.camera(0.9, 1.0), translation=[0, 0, 3])
    g.write_glb(path)
    if case == "missing":
        path = tmp_path / "nothing.glb"
    elif case == "not_json":
        path.write_text("{ this is not json")
    elif case == "truncated":
        path.write_bytes(path.read_bytes()[:40])
    with pytest.raises(P.PhxError) as e:
        P.SceneData.load_gltf(path)
    assert e.value.code == A.PHX_E_INVALID


@pytest.mark.gpu
def test_loaded_scene_renders_like_the_oracle(tmp_path):
    """A glTF-loaded scene goes through the same pipeline: one round bit-exact against the oracle."""
    w, h = 48, 40
    src = P.SceneData.generate(A.PHX_SCENE_CORNELL, seed=1, width=w, height=h)
    g = Gltf()
    export_generated(src, g, 40.0, w / h, (0.5, 0.5, 2.4))
    g.write_glb(tmp_path / "cornell.glb")
    sc = P.SceneData.load_gltf(tmp_path / "cornell.glb", width=w, height=h)
    args = P.ArgsList(width=w, height=h, photons_per_round=1 << 13, max_photon_bounces=8, grid_res=50, seed=3,
                      direct_samples=4)
    with P.Renderer(args) as r:
        r.set_scene(sc)
        r.round()
        flux, rad = r.read("FLUX"), r.read("RADIANCE")
    st = O.Oracle(sc).render(args.params(), 1, prec=0)
    assert np.array_equal(flux.view(np.uint32), st["flux"].view(np.uint32))
    assert np.array_equal(rad.view(np.uint32), st["radiance"].view(np.uint32))
    assert (st["weight"] > 0).mean() > 0.3
