"""Helpers for tests/golden/ref_sppm_golden.npz: the reference's own SPPM code (compiled for the
CPU by oracle/build_ref_sppm.py) run on small scenes, stored by tests/golden/make_ref_sppm_golden.py.

A case is either a procedural scene (kind >= 0, rebuilt from its generator spec; the stored digest
of its triangle bytes catches any change of the generator) or a scene stored as its arrays (kind
-1: triangles, materials, UV transforms, lights, luminance prefix sum, textures, camera).  For each
case the fixture holds the reference's round-1 stage outputs for the round's seed — hit points,
canonical photons, cell keys, counts, starts, ends, cell-sorted photons, the SPPM state after the
gather — and the SPPM state and 8-bit image after `rounds` rounds of Renderer::run.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from pathlib import Path

import numpy as np

from phosphor_b200 import _capi as A

FIXTURE = Path(__file__).resolve().parent / "golden" / "ref_sppm_golden.npz"

META = ["kind", "detail", "gen_seed", "width", "height", "photons", "bounces", "grid", "samples", "seed", "rounds"]
ARRAYS = {  # name -> (ctypes struct, Scene pointer field, Scene count field)
    "tris": (A.Triangle, "triangles", "n_triangles"),
    "etris": (A.Triangle, "emissive_triangles", "n_emissive_triangles"),
    "mats": (A.Material, "materials", "n_materials"),
    "uvs": (A.UvTransformBlock, "uv_transforms", None),
    "lights": (A.Light, "lights", "n_lights"),
    "tex_meta": (A.TextureMeta, "tex_meta", "n_textures"),
}


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def triangle_bytes(scene: A.Scene) -> np.ndarray:
    n = scene.n_triangles * C.sizeof(A.Triangle)
    return np.ctypeslib.as_array(C.cast(scene.triangles, C.POINTER(C.c_uint8)), shape=(n,)).copy()


def scene_arrays(scene: A.Scene) -> dict:
    """The raw bytes of every array of a phx_scene (for storing a scene in the fixture)."""
    out = {}
    for name, (st, ptr, cnt) in ARRAYS.items():
        n = getattr(scene, cnt) if cnt else scene.n_materials
        p = getattr(scene, ptr)
        size = n * C.sizeof(st)
        out[name] = (np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint8)), shape=(size,)).copy()
                     if size and p else np.zeros(0, np.uint8))
    nl = scene.n_lights
    out["lum"] = (np.ctypeslib.as_array(scene.lum_pref_sum, shape=(nl,)).copy() if nl else np.zeros(0, np.float32))
    nb = scene.tex_atlas_bytes
    out["atlas"] = (np.ctypeslib.as_array(scene.tex_atlas, shape=(nb,)).copy() if nb else np.zeros(0, np.uint8))
    out["camera"] = np.frombuffer(bytes(scene.camera), np.uint8).copy()
    return out


class ArrayScene:
    """A phx_scene over stored arrays (the `.scene` attribute, as SceneData / GeneratedScene have)."""

    def __init__(self, arrays: dict):
        self._keep = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        sc = A.Scene()
        for name, (st, ptr, cnt) in ARRAYS.items():
            a = self._keep[name]
            n = len(a) // C.sizeof(st)
            setattr(sc, ptr, C.cast(a.ctypes.data, C.POINTER(st)) if n else None)
            if cnt:
                setattr(sc, cnt, n)
        lum = self._keep["lum"] = np.ascontiguousarray(self._keep["lum"], np.float32)
        sc.lum_pref_sum = C.cast(lum.ctypes.data, C.POINTER(C.c_float)) if len(lum) else None
        atlas = self._keep["atlas"]
        sc.tex_atlas = C.cast(atlas.ctypes.data, C.POINTER(C.c_uint8)) if len(atlas) else None
        sc.tex_atlas_bytes = len(atlas)
        sc.camera = A.CameraParams.from_buffer_copy(self._keep["camera"].tobytes())
        self.scene = sc

    @property
    def n_triangles(self) -> int:
        return self.scene.n_triangles


def load_cases() -> list[dict]:
    z = np.load(FIXTURE)
    cases = []
    for i in range(int(z["n_cases"][0])):
        pre = f"c{i}_"
        c = {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}
        c["meta"] = dict(zip(META, (int(x) for x in c["meta"])))
        c["name"] = str(c["name"])
        c["alpha"] = float(c["alpha"][0])
        cases.append(c)
    return cases


def case_scene(case: dict, generate):
    """The case's scene: `generate(kind, seed, width, height, detail)` for a procedural one (its
    triangle digest is checked), the stored arrays otherwise."""
    m = case["meta"]
    if m["kind"] >= 0:
        sc = generate(m["kind"], m["gen_seed"], m["width"], m["height"], m["detail"])
        assert digest(triangle_bytes(sc.scene)) == str(case["tri_digest"]), "scene generator output changed"
        return sc
    return ArrayScene({k[len("arr_"):]: v for k, v in case.items() if k.startswith("arr_")})


def case_args(case: dict, ArgsList):
    m = case["meta"]
    return ArgsList(width=m["width"], height=m["height"], photons_per_round=m["photons"],
                    max_photon_bounces=m["bounces"], grid_res=m["grid"], seed=m["seed"], direct_samples=m["samples"],
                    sppm_alpha=case["alpha"])
