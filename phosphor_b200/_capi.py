"""ctypes mirror of include/phx.h (the C ABI of libphx.so).

Struct layouts are byte-compatible with the C header (checked by static_asserts on the C side and
by tests/test_capi_layout.py on this side).  This module only declares types and loads the
library; phosphor_b200.renderer builds the reference-style API on top of it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libphx.so"

# status codes
PHX_OK, PHX_E_INVALID, PHX_E_OOM, PHX_E_CUDA, PHX_E_TIMEOUT, PHX_E_NO_PHOTONS, PHX_E_STATE, PHX_E_OVERFLOW, \
    PHX_E_UNSUPPORTED = range(9)
STATUS_NAMES = {0: "PHX_OK", 1: "PHX_E_INVALID", 2: "PHX_E_OOM", 3: "PHX_E_CUDA", 4: "PHX_E_TIMEOUT",
                5: "PHX_E_NO_PHOTONS", 6: "PHX_E_STATE", 7: "PHX_E_OVERFLOW", 8: "PHX_E_UNSUPPORTED"}

PHX_NO_TEXTURE = 0xFFFFFFFF
PHX_LIGHT_POINT, PHX_LIGHT_SPOT, PHX_LIGHT_DIRECTIONAL, PHX_LIGHT_TEXTURED = range(4)
PHX_SCENE_CORNELL, PHX_SCENE_CAUSTIC, PHX_SCENE_ATRIUM = range(3)
PHX_F_DEFAULT, PHX_F_SIMPLE_TRAVERSAL, PHX_F_REFERENCE_BVH, PHX_F_BINARY_BVH, PHX_F_DEVICE_BVH = 0, 1, 2, 4, 8
PHX_F_QUANT_BVH, PHX_F_HOST_BVH = 16, 32

BUFFERS = ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT", "HP_EMISSION", "FLUX",
           "PHOTON_WEIGHT", "RADIANCE", "PHOTON_POS", "PHOTON_POWER", "PHOTON_DIR", "PHOTON_HASH", "CELL_COUNT",
           "CELL_START", "CELL_END", "SORTED_POS", "SORTED_POWER", "SORTED_DIR", "EMIT_COUNT", "BVH_NODES",
           "SORT_PERM", "ROUND_RNG"]
BUF = {name: i for i, name in enumerate(BUFFERS)}
# numpy element layout of each buffer (reference layout)
BUF_DTYPE = {name: (np.float32, 4) for name in ["HP_POS", "HP_NORMAL", "HP_THROUGHPUT", "HP_BASE_COLOR", "HP_DIRECT",
                                                 "HP_EMISSION", "FLUX", "RADIANCE", "PHOTON_POS", "SORTED_POS"]}
BUF_DTYPE.update({name: (np.uint32, 1) for name in ["PHOTON_POWER", "PHOTON_DIR", "PHOTON_HASH", "CELL_COUNT",
                                                     "CELL_START", "CELL_END", "SORTED_POWER", "SORTED_DIR",
                                                     "EMIT_COUNT", "SORT_PERM", "ROUND_RNG"]})
BUF_DTYPE["PHOTON_WEIGHT"] = (np.float32, 1)
BUF_DTYPE["BVH_NODES"] = (np.float32, 8)

STAGES = ["seeds", "trace", "shadow", "emit", "emit_scan", "hash", "cell_scan", "sort", "records", "gather"]


class f4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class f2(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float)]


class Triangle(C.Structure):
    _fields_ = [("v0", f4), ("v1", f4), ("v2", f4), ("n0", f4), ("n1", f4), ("n2", f4), ("t0", f4), ("t1", f4),
                ("t2", f4), ("uv0", f2), ("uv1", f2), ("uv2", f2), ("mat_index", C.c_uint32),
                ("_padding", C.c_uint8 * 4)]


class UvTransform(C.Structure):
    _fields_ = [("uv_offset", f2), ("uv_scale", f2), ("uv_rotation", C.c_float), ("_padding", C.c_uint8 * 12)]


class UvTransformBlock(C.Structure):
    _fields_ = [(n, UvTransform) for n in ("diff", "emis", "norm", "occlusion", "metal_rough", "transmission")]


class Material(C.Structure):
    _fields_ = [("base_color", f4), ("emissive", f4), ("att_color", f4)] + \
               [(n, C.c_float) for n in ("metallic", "roughness", "transmission", "ior", "att_dist", "thickness")] + \
               [(n, C.c_uint32) for n in ("diff_index", "emis_index", "norm_index", "occlusion_index",
                                          "metal_rough_index", "transmission_index")]


class Light(C.Structure):
    _fields_ = [(n, f4) for n in ("position", "power", "direction", "tangent", "bitangent", "origin", "aux")] + \
               [("kind", C.c_uint8), ("_padding", C.c_uint8 * 15)]


class TextureMeta(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("atlas_offset", "width", "height", "channels")]


class CameraParams(C.Structure):
    _fields_ = [(n, f4) for n in ("position", "lower_left_corner", "horizontal", "vertical", "defocus_disk_u",
                                  "defocus_disk_v")] + \
               [("defocus_angle", C.c_float), ("focus_distance", C.c_float), ("_padding", C.c_uint8 * 8)]


class BvhNode(C.Structure):
    _fields_ = [("min", f4), ("max", f4)]


class PhotonHashData(C.Structure):
    _fields_ = [("origin", f4), ("cell_sizes", f4), ("grid_res", C.c_uint32), ("_padding", C.c_uint8 * 12)]


class Scene(C.Structure):
    _fields_ = [("triangles", C.POINTER(Triangle)), ("n_triangles", C.c_uint32),
                ("emissive_triangles", C.POINTER(Triangle)), ("n_emissive_triangles", C.c_uint32),
                ("materials", C.POINTER(Material)), ("uv_transforms", C.POINTER(UvTransformBlock)),
                ("n_materials", C.c_uint32), ("lights", C.POINTER(Light)), ("n_lights", C.c_uint32),
                ("lum_pref_sum", C.POINTER(C.c_float)), ("tex_meta", C.POINTER(TextureMeta)),
                ("n_textures", C.c_uint32), ("tex_atlas", C.POINTER(C.c_uint8)), ("tex_atlas_bytes", C.c_uint64),
                ("envmap", C.POINTER(C.c_float)), ("envmap_width", C.c_uint32), ("envmap_height", C.c_uint32),
                ("camera", CameraParams)]


class Params(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("photons_per_round", C.c_uint32),
                ("max_photon_bounces", C.c_uint32), ("grid_res", C.c_uint32), ("sppm_alpha", C.c_float),
                ("direct_samples", C.c_uint32), ("seed", C.c_uint32), ("flags", C.c_uint32),
                ("bvh_leaf_size", C.c_uint32), ("reserved", C.c_uint32 * 6)]


class Info(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("n_pixels", "width", "height", "photons_per_round", "photon_buf_size",
                                          "bucket_count", "n_photons", "n_bvh_nodes", "bvh_depth", "rounds_done")] + \
               [("total_photons_emitted", C.c_uint64), ("stack_overflows", C.c_uint32), ("error_flags", C.c_uint32),
                ("_pad0", C.c_uint32 * 2), ("hash", PhotonHashData), ("kernels_per_round", C.c_uint32),
                ("sort_passes", C.c_uint32), ("trav_depth", C.c_uint32), ("trav_inner_nodes", C.c_uint32),
                ("spec_samples", C.c_uint32), ("setup_ms", C.c_float), ("bvh_build_ms", C.c_float),
                ("reserved", C.c_uint32 * 1)]


class GltfOptions(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("defocus_angle", C.c_float),
                ("focus_distance", C.c_float), ("camera", C.c_uint32), ("reserved", C.c_uint32 * 3)]


class SceneSpec(C.Structure):
    _fields_ = [("kind", C.c_int), ("seed", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("detail", C.c_uint32), ("reserved", C.c_uint32 * 5)]


class Tuning(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("trace_block", "emit_block", "gather_block", "trace_blocks_per_sm",
                                          "emit_blocks_per_sm", "persistent", "nee_wavefront",
                                          "concurrent_passes", "gather_sorted", "pipeline_rounds", "gather_coop")] + \
               [("reserved", C.c_uint32 * 1)]


class BvhPacked(C.Structure):
    _fields_ = [("nodes", C.POINTER(C.c_float)), ("trirec", C.POINTER(C.c_float)),
                ("leaf_tri", C.POINTER(C.c_uint32)), ("n_nodes", C.c_uint32), ("root", C.c_int32),
                ("depth", C.c_uint32), ("wdepth", C.c_uint32), ("build_ms", C.c_float),
                ("reserved", C.c_uint32 * 3)]


SIZES = {Triangle: 176, Material: 96, UvTransformBlock: 192, Light: 128, CameraParams: 112, BvhNode: 32,
         PhotonHashData: 48, TextureMeta: 16, Scene: 240, Info: 144, Params: 64, Tuning: 48, SceneSpec: 40, BvhPacked: 56}

# (name, restype, argtypes) of every entry point declared in include/phx.h
VP = C.c_void_p
PROTOTYPES = [
    ("phx_create", C.c_int, [C.POINTER(Scene), C.POINTER(Params), C.c_int, C.POINTER(VP)]),
    ("phx_destroy", C.c_int, [VP]),
    ("phx_get_info", C.c_int, [VP, C.POINTER(Info)]),
    ("phx_trace_rays", C.c_int, [VP, C.c_uint32]),
    ("phx_emit_photons", C.c_int, [VP, C.c_uint32]),
    ("phx_hash_sort", C.c_int, [VP]),
    ("phx_gather", C.c_int, [VP, C.c_float]),
    ("phx_round", C.c_int, [VP]),
    ("phx_iterate", C.c_int, [VP, C.c_uint32]),
    ("phx_round_seeded", C.c_int, [VP, C.c_uint32]),
    ("phx_sync", C.c_int, [VP]),
    ("phx_read_buffer", C.c_int, [VP, C.c_int, VP, C.c_uint64, C.c_uint64]),
    ("phx_write_buffer", C.c_int, [VP, C.c_int, VP, C.c_uint64, C.c_uint64]),
    ("phx_set_n_photons", C.c_int, [VP, C.c_uint32]),
    ("phx_image", C.c_int, [VP, C.c_float, C.c_int, C.c_uint64, C.c_uint32, VP, VP]),
    ("phx_bvh_build", C.c_int, [C.POINTER(Triangle), C.c_uint32, C.POINTER(BvhNode), C.POINTER(C.c_uint32)]),
    ("phx_traversal_bvh_build", C.c_int, [C.POINTER(Triangle), C.c_uint32, C.c_uint32, C.c_int, C.c_int,
                                          C.POINTER(BvhPacked)]),
    ("phx_hash_info", C.c_int, [C.POINTER(BvhNode), C.c_uint32, C.POINTER(PhotonHashData)]),
    ("phx_camera_make", C.c_int, [C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float,
                                  C.c_float, C.c_float, C.c_float, C.POINTER(CameraParams)]),
    ("phx_lum_pref_sum", C.c_int, [C.POINTER(Light), C.c_uint32, C.POINTER(C.c_float)]),
    ("phx_scene_generate", C.c_int, [C.POINTER(SceneSpec), C.POINTER(Scene), C.POINTER(VP)]),
    ("phx_scene_free", C.c_int, [VP]),
    ("phx_scene_load_gltf", C.c_int, [C.c_char_p, C.POINTER(GltfOptions), C.POINTER(Scene), C.POINTER(VP)]),
    ("phx_batch_create", C.c_int, [C.POINTER(Scene), C.POINTER(Params), C.c_uint32, C.c_int, C.POINTER(VP)]),
    ("phx_batch_destroy", C.c_int, [VP]),
    ("phx_batch_iterate", C.c_int, [VP, C.c_uint32, C.c_int]),
    ("phx_batch_read_buffer", C.c_int, [VP, C.c_uint32, C.c_int, VP, C.c_uint64, C.c_uint64]),
    ("phx_batch_get_info", C.c_int, [VP, C.c_uint32, C.POINTER(Info)]),
    ("phx_batch_image", C.c_int, [VP, C.c_uint32, C.c_float, C.c_int, VP]),
    ("phx_get_tuning", C.c_int, [VP, C.POINTER(Tuning)]),
    ("phx_set_tuning", C.c_int, [VP, C.POINTER(Tuning)]),
    ("phx_autotune", C.c_int, [VP, C.c_uint32, C.POINTER(Tuning)]),
    ("phx_profile", C.c_int, [VP, C.c_int]),
    ("phx_stage_ms", C.c_int, [VP, C.POINTER(C.c_float), C.c_uint32]),
    ("phx_get_stream", C.c_uint64, [VP]),
    ("phx_selftest_lookback_timeout", C.c_int, [C.c_int, C.c_uint32, C.POINTER(C.c_uint32)]),
    ("phx_scan_noalloc", C.c_int, [VP, VP, C.c_uint32, VP, C.c_uint64]),
    ("phx_mean_filter", C.c_int, [VP, VP, C.c_uint32, C.c_uint32, C.c_uint32, VP]),
    ("phx_median_filter", C.c_int, [VP, VP, C.c_uint32, C.c_uint32, C.c_uint32, VP]),
    ("phx_weighted_filter", C.c_int, [VP, VP, VP, C.c_uint32, C.c_uint32, C.c_uint32, VP]),
    ("phx_batch_set_active", C.c_int, [VP, C.c_uint32, C.c_int]),
    ("phx_shard", C.c_int, [VP, C.c_uint32, C.c_uint32]),
    ("phx_shard_begin", C.c_int, [VP, C.POINTER(C.c_uint32)]),
    ("phx_shard_get_photons", C.c_int, [VP, VP, VP, C.c_uint32]),
    ("phx_shard_put_photons", C.c_int, [VP, VP, VP, C.c_uint32]),
    ("phx_shard_end", C.c_int, [VP]),
    ("phx_nccl_unique_id", C.c_int, [VP, C.c_uint32]),
    ("phx_shard_nccl", C.c_int, [VP, VP]),
    ("phx_shard_round", C.c_int, [VP]),
    ("phx_set_materials", C.c_int, [VP, VP, C.c_uint32]),
    ("phx_set_lights", C.c_int, [VP, VP, C.c_uint32]),
    ("phx_adjoint_n_params", C.c_int, [VP, C.POINTER(C.c_uint32)]),
    ("phx_adjoint_forward", C.c_int, [VP, C.c_uint32, VP]),
    ("phx_adjoint_backward", C.c_int, [VP, VP, VP, C.c_uint32]),
    ("phx_last_error", C.c_char_p, []),
    ("phx_version", C.c_char_p, []),
]

_lib = None


class PhxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def load(path: Path | str | None = None) -> C.CDLL:
    """Loads libphx.so from the package directory.  Raises if it has not been built: there is no
    fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not built; run `python -m phosphor_b200.build`")
    lib = C.CDLL(str(p))
    for name, res, args in PROTOTYPES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(code: int) -> None:
    if code != PHX_OK:
        raise PhxError(code, load().phx_last_error().decode(errors="replace"))
