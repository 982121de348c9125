"""Makes tests/golden/ref_sppm_golden.npz from the reference's own SPPM code.

oracle/build_ref_sppm.py compiles the reference's OpenCL kernels and host code for the CPU
(oracle/ref.py binds them); this script drives them the way Renderer::run does on small scenes and
stores what they compute, so that tests can check the CPU restatement (oracle/) and the CUDA
library against the reference itself without a reference checkout:

* the three procedural scenes (Cornell box, caustic box, atrium; reduced tessellation), stored as
  their generator spec plus a digest of the generated triangles;
* five scenes stored as arrays, built from those by changing lights and materials, for the code
  the procedural scenes never reach: a spot light and a directional light as the only light of
  a scene with a transmissive surface (with 2 and 16 direct samples), all four light kinds in one
  scene (5 samples), textured materials (base colour, emissive, metal-rough, transmission,
  occlusion and normal maps, non-identity UV transforms, an emissive texture on the area light,
  Beer-Lambert attenuation), three glass panes under a point light, and a box of rough mirrors
  whose camera paths outnumber the library's deferred specular-NEE slots.

The lights come from the reference's own constructors (light.cpp) and every light luminance
prefix sum from its SceneData::build_lum_pref_sum.

    python tests/golden/make_ref_sppm_golden.py path/to/reference   (or PHX_REFERENCE_DIR=...)
"""
from __future__ import annotations

import ctypes as C
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import oracle as O  # noqa: E402
from oracle import build_ref_sppm  # noqa: E402
from oracle import ref as R  # noqa: E402
from oracle.build_ref_filters import reference_dir  # noqa: E402
from phosphor_b200 import _capi as A  # noqa: E402
from phosphor_b200.renderer import ArgsList  # noqa: E402
from ref_fixture import FIXTURE, META, ArrayScene, digest, scene_arrays, triangle_bytes  # noqa: E402

ROUNDS = 3


def structs(raw: np.ndarray, st):
    n = len(raw) // C.sizeof(st)
    return (st * n).from_buffer_copy(raw.tobytes())


def to_raw(arr) -> np.ndarray:
    return np.frombuffer(bytes(arr), np.uint8).copy()


def lum_of(lights_raw: np.ndarray) -> np.ndarray:
    n = len(lights_raw) // C.sizeof(A.Light)
    return R.lum_pref_sum(lights_raw.ctypes.data, n) if n else np.zeros(0, np.float32)


def with_lights(arrays: dict, lights: list[bytes]) -> dict:
    out = dict(arrays)
    out["lights"] = np.frombuffer(b"".join(lights), np.uint8).copy()
    out["lum"] = lum_of(out["lights"])
    return out


def wall_of(t) -> str:
    n = (t.n0.x, t.n0.y, t.n0.z)
    ys = (t.v0.y, t.v1.y, t.v2.y)
    if n[1] > 0.5:
        return "floor"
    if n[1] < -0.5:
        return "light" if min(ys) > 0.99 and max(ys) < 0.9995 else "ceiling"
    if n[2] > 0.5:
        return "back"
    return "left" if n[0] > 0.5 else "right"


def spot_scene(base: dict) -> dict:
    light = R.make_light(R.LIGHT_SPOT, pos=(0.5, 0.95, 0.5), power=(2.0, 1.9, 1.7), direction=(0.05, -1.0, 0.1),
                         a=0.3, b=0.6)
    return with_lights(base, [light])


def directional_scene(base: dict) -> dict:
    d = np.array([0.25, -0.45, -1.0], np.float32)
    light = R.make_light(R.LIGHT_DIRECTIONAL, power=(1.2, 1.1, 1.0), direction=d / np.linalg.norm(d))
    return with_lights(base, [light])


def mixed_scene(base: dict) -> dict:
    area = base["lights"].tobytes()
    point = R.make_light(R.LIGHT_POINT, pos=(0.2, 0.8, 0.6), power=(0.5, 0.4, 0.3))
    spot = R.make_light(R.LIGHT_SPOT, pos=(0.8, 0.9, 0.3), power=(1.0, 1.0, 1.0), direction=(0.0, -1.0, 0.2),
                        a=0.2, b=0.5)
    d = np.array([0.2, -0.4, -1.0], np.float32)
    sun = R.make_light(R.LIGHT_DIRECTIONAL, power=(0.3, 0.3, 0.25), direction=d / np.linalg.norm(d))
    return with_lights(base, [area, point, spot, sun])


def textured_scene(base: dict) -> dict:
    rng = np.random.default_rng(2137)
    sizes = [(8, 8), (16, 4), (5, 7), (12, 12)]
    metas, atlas = [], []
    for i, (w, h) in enumerate(sizes):
        tex = rng.integers(0, 256, size=(h, w, 3)).astype(np.uint8)
        if i == 1:  # a normal map: tangent-space normals around +z
            tex[..., :2] = rng.integers(96, 160, size=(h, w, 2))
            tex[..., 2] = rng.integers(200, 256, size=(h, w))
        m = A.TextureMeta(atlas_offset=sum(len(a) for a in atlas), width=w, height=h, channels=3)
        metas.append(bytes(m))
        atlas.append(tex.reshape(-1))
    tris = structs(base["tris"], A.Triangle)
    mats = list(structs(base["mats"], A.Material))
    uvs = list(structs(base["uvs"], A.UvTransformBlock))

    def add_material(src: int, **kw) -> int:
        m = A.Material.from_buffer_copy(bytes(mats[src]))
        for k, v in kw.items():
            if isinstance(v, tuple):
                getattr(m, k).x, getattr(m, k).y, getattr(m, k).z = v
            else:
                setattr(m, k, v)
        mats.append(m)
        uvs.append(A.UvTransformBlock.from_buffer_copy(bytes(uvs[src])))
        return len(mats) - 1

    def set_uv(i, slot, off, scale, rot):
        t = getattr(uvs[i], slot)
        t.uv_offset.x, t.uv_offset.y = off
        t.uv_scale.x, t.uv_scale.y = scale
        t.uv_rotation = rot

    walls = {wall_of(t) for t in tris}
    assert walls == {"floor", "ceiling", "back", "left", "right", "light"}, walls
    m_floor = add_material(0, diff_index=0, occlusion_index=3)
    set_uv(m_floor, "diff", (0.1, -0.2), (1.5, 0.7), 0.3)
    set_uv(m_floor, "occlusion", (0.0, 0.5), (1.0, 1.0), 0.0)
    m_back = add_material(0, norm_index=1, metal_rough_index=2, metallic=0.5, roughness=0.8)
    set_uv(m_back, "norm", (0.3, 0.3), (2.0, 2.0), 1.1)
    set_uv(m_back, "metal_rough", (0.0, 0.0), (0.8, 1.3), -0.4)
    m_left = add_material(1, norm_index=1, transmission=0.5, transmission_index=2, diff_index=3, thickness=0.1,
                          att_dist=0.5, att_color=(0.8, 0.6, 0.5), roughness=0.3)
    set_uv(m_left, "transmission", (0.25, 0.0), (1.0, 1.0), 0.0)
    m_right = add_material(2, emissive=(0.5, 0.4, 0.3), emis_index=0)
    set_uv(m_right, "emis", (0.0, 0.0), (3.0, 3.0), 0.7)
    m_light = add_material(3, emis_index=3)
    assign = {"floor": m_floor, "back": m_back, "left": m_left, "right": m_right, "light": m_light}

    def uv_of(wall, v):
        if wall in ("floor", "ceiling"):
            return (v.x * 1.3, v.z * 1.3)
        if wall == "back":
            return (v.x, v.y)
        if wall == "light":
            return ((v.x - 0.375) / 0.25, (v.z - 0.375) / 0.25)
        return (v.z * 1.1, v.y * 0.9)

    for t in tris:
        wall = wall_of(t)
        if wall in assign:
            t.mat_index = assign[wall]
        for uv, v in ((t.uv0, t.v0), (t.uv1, t.v1), (t.uv2, t.v2)):
            uv.x, uv.y = uv_of(wall, v)
    etris = structs(base["etris"], A.Triangle)
    for t in etris:
        t.mat_index = m_light
        for uv, v in ((t.uv0, t.v0), (t.uv1, t.v1), (t.uv2, t.v2)):
            uv.x, uv.y = uv_of("light", v)
    old = A.Light.from_buffer_copy(base["lights"].tobytes())
    aux = np.frombuffer(bytes(old.aux), np.uint32)
    light = R.make_light(R.LIGHT_TEXTURED, power=(old.power.x, old.power.y, old.power.z), tex=3, start=int(aux[1]),
                         count=int(aux[2]), a=float(old.aux.w))
    out = dict(base)
    out.update(tris=to_raw(tris), etris=to_raw(etris), mats=np.frombuffer(b"".join(bytes(m) for m in mats), np.uint8),
               uvs=np.frombuffer(b"".join(bytes(u) for u in uvs), np.uint8),
               tex_meta=np.frombuffer(b"".join(metas), np.uint8), atlas=np.concatenate(atlas))
    return with_lights(out, [light])


def panes_scene(base: dict) -> dict:
    """Three horizontal transmissive panes between the floor and the ceiling under a point light."""
    tris = list(structs(base["tris"], A.Triangle))
    mats = list(structs(base["mats"], A.Material))
    uvs = list(structs(base["uvs"], A.UvTransformBlock))
    glass = A.Material.from_buffer_copy(bytes(mats[0]))
    glass.transmission, glass.roughness, glass.ior = 1.0, 0.1, 1.5
    glass.base_color.x, glass.base_color.y, glass.base_color.z = 0.9, 0.95, 0.9
    mats.append(glass)
    uvs.append(A.UvTransformBlock.from_buffer_copy(bytes(uvs[0])))
    for y in (0.25, 0.5, 0.75):
        c = [(0.1, 0.1), (0.9, 0.1), (0.9, 0.9), (0.1, 0.9)]
        for tri in ((0, 1, 2), (0, 2, 3)):
            t = A.Triangle.from_buffer_copy(bytes(tris[0]))
            for v, k in zip((t.v0, t.v1, t.v2), tri):
                v.x, v.y, v.z = c[k][0], y, c[k][1]
            for nrm in (t.n0, t.n1, t.n2):
                nrm.x, nrm.y, nrm.z = 0.0, 1.0, 0.0
            t.mat_index = len(mats) - 1
            tris.append(t)
    out = dict(base)
    out.update(tris=np.frombuffer(b"".join(bytes(t) for t in tris), np.uint8),
               mats=np.frombuffer(b"".join(bytes(m) for m in mats), np.uint8),
               uvs=np.frombuffer(b"".join(bytes(u) for u in uvs), np.uint8))
    return with_lights(out, [R.make_light(R.LIGHT_POINT, pos=(0.5, 0.9, 0.5), power=(1.0, 1.0, 1.0))])


def mirror_scene(base: dict) -> dict:
    """The back, left and right walls rough mirrors (floor and ceiling stay diffuse, so photons are
    stored): camera paths bounce between the mirrors with a specular event at nearly every bounce,
    more events than the library's deferred specular-NEE sample slots hold (one per pixel and
    sample), so many take its traced-in-place fallback."""
    tris = structs(base["tris"], A.Triangle)
    mats = list(structs(base["mats"], A.Material))
    uvs = list(structs(base["uvs"], A.UvTransformBlock))
    mirror = A.Material.from_buffer_copy(bytes(mats[0]))
    mirror.metallic, mirror.roughness = 1.0, 0.1
    mirror.base_color.x, mirror.base_color.y, mirror.base_color.z = 0.95, 0.93, 0.9
    mats.append(mirror)
    uvs.append(A.UvTransformBlock.from_buffer_copy(bytes(uvs[0])))
    for t in tris:
        if wall_of(t) in ("back", "left", "right"):
            t.mat_index = len(mats) - 1
    out = dict(base)
    out.update(tris=to_raw(tris), mats=np.frombuffer(b"".join(bytes(m) for m in mats), np.uint8),
               uvs=np.frombuffer(b"".join(bytes(u) for u in uvs), np.uint8))
    return out


PROCEDURAL = [
    # name, kind, detail, width, height, photons, bounces, grid, samples
    ("cornell", A.PHX_SCENE_CORNELL, 0, 32, 32, 4096, 8, 50, 4),
    ("caustic", A.PHX_SCENE_CAUSTIC, 24, 32, 32, 4096, 12, 50, 4),
    ("atrium", A.PHX_SCENE_ATRIUM, 8, 40, 24, 8192, 16, 64, 4),
]
CUSTOM = [
    # name, base kind, base detail, builder, photons, bounces, grid, samples
    ("caustic_spot", A.PHX_SCENE_CAUSTIC, 16, spot_scene, 4096, 12, 50, 2),
    ("caustic_directional", A.PHX_SCENE_CAUSTIC, 16, directional_scene, 4096, 12, 50, 16),
    ("cornell_mixed_lights", A.PHX_SCENE_CORNELL, 0, mixed_scene, 4096, 8, 50, 5),
    ("cornell_textured", A.PHX_SCENE_CORNELL, 0, textured_scene, 4096, 8, 50, 4),
    ("panes_point", A.PHX_SCENE_CORNELL, 0, panes_scene, 4096, 8, 50, 16),
    ("mirror_box", A.PHX_SCENE_CORNELL, 0, mirror_scene, 4096, 8, 50, 16),
]


def run_case(name: str, scene, meta: dict, alpha: float) -> dict:
    args = ArgsList(width=meta["width"], height=meta["height"], photons_per_round=meta["photons"],
                    max_photon_bounces=meta["bounces"], grid_res=meta["grid"], seed=meta["seed"],
                    direct_samples=meta["samples"], sppm_alpha=alpha)
    t0 = time.time()
    rr = R.RefRenderer(scene, args)
    first = rr.round(keep=True)
    out = {"r1_seed": np.array([first["seed"]], np.uint32), "r1_hp": first["hp"],
           "r1_photon_pos": first["photon_pos"], "r1_photon_power": first["photon_power"],
           "r1_photon_dir": first["photon_dir"], "r1_keys": first["grid_keys"], "r1_counts": first["grid_counts"],
           "r1_starts": first["grid_starts"], "r1_ends": first["grid_ends"],
           # the cell-sorted positions are a permutation of the photon positions: a digest suffices
           "r1_sorted_pos_digest": np.array(digest(first["grid_pos"])),
           "r1_sorted_power": first["grid_power"], "r1_sorted_dir": first["grid_dir"],
           "r1_flux": rr.flux.copy(), "r1_weight": rr.weight.copy(), "r1_radiance": rr.radiance.copy(),
           "bvh_digest": np.array(digest(rr.bvh)), "n_bvh_nodes": np.array([len(rr.bvh)], np.int64),
           "hash_data": np.frombuffer(rr.hash_data, np.uint8)}
    for _ in range(meta["rounds"] - 1):
        rr.round()
    out.update(flux=rr.flux, weight=rr.weight, radiance=rr.radiance, image=rr.image_u8(),
               total_emitted=np.array([rr.total_emitted], np.uint64))
    print(f"{name}: {len(first['photon_pos'])} photons in round 1, {time.time() - t0:.1f} s")
    return out


def main(reference: Path) -> None:
    build_ref_sppm.build(reference, verbose=True)
    arrays = {}
    cases = []
    for name, kind, detail, w, h, ph, mb, g, ds in PROCEDURAL:
        sc = O.GeneratedScene(kind, seed=1, width=w, height=h, detail=detail)
        meta = dict(kind=kind, detail=detail, gen_seed=1, width=w, height=h, photons=ph, bounces=mb, grid=g,
                    samples=ds, seed=1, rounds=ROUNDS)
        out = run_case(name, sc, meta, 0.7)
        out["tri_digest"] = np.array(digest(triangle_bytes(sc.scene)))
        cases.append((name, meta, out))
    for name, kind, detail, builder, ph, mb, g, ds in CUSTOM:
        base = O.GeneratedScene(kind, seed=1, width=32, height=32, detail=detail)
        arr = builder(scene_arrays(base.scene))
        sc = ArrayScene(arr)
        meta = dict(kind=-1, detail=0, gen_seed=0, width=32, height=32, photons=ph, bounces=mb, grid=g, samples=ds,
                    seed=7, rounds=ROUNDS)
        out = run_case(name, sc, meta, 0.75)
        out.update({f"arr_{k}": v for k, v in arr.items()})
        cases.append((name, meta, out))
    for i, (name, meta, out) in enumerate(cases):
        arrays[f"c{i}_name"] = np.array(name)
        arrays[f"c{i}_meta"] = np.array([meta[k] for k in META], np.int64)
        arrays[f"c{i}_alpha"] = np.array([0.7 if meta["kind"] >= 0 else 0.75], np.float32)
        for k, v in out.items():
            arrays[f"c{i}_{k}"] = v
    arrays["n_cases"] = np.array([len(cases)], np.int32)
    np.savez_compressed(FIXTURE, **arrays)
    print(f"wrote {FIXTURE} ({FIXTURE.stat().st_size / 1e6:.2f} MB, {len(cases)} cases)")


if __name__ == "__main__":
    ref = reference_dir(sys.argv[1] if len(sys.argv) > 1 else None)
    if ref is None:
        sys.exit("usage: make_ref_sppm_golden.py path/to/reference   (or set PHX_REFERENCE_DIR)")
    main(ref)
