"""TEST INFRASTRUCTURE ONLY — Python binding of the CPU oracle (liboracle.so).

The oracle is a statement-by-statement C++ restatement of the reference SPPM kernels (see
oracle/phx_oracle.hpp for the file:line map and the fixed semantics).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg use it, as the checker; the library never
calls it.  Pinned to the reference itself: tests/test_ref_pin.py compares it stage by stage with
the reference's own kernels and host code compiled for the CPU (oracle/build_ref_sppm.py,
fixtures in tests/golden/ref_sppm_golden.npz).
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        from phosphor_b200.build import build_oracle
        build_oracle()
    lib = C.CDLL(str(LIB_PATH))
    vp = C.c_void_p
    sig = {
        "orc_scene_generate": (C.c_int, [vp, vp, vp]),
        "orc_scene_free": (None, [vp]),
        "orc_camera_make": (None, [vp, vp, vp, C.c_float, C.c_float, C.c_float, C.c_float, vp]),
        "orc_lum_pref_sum": (None, [vp, C.c_uint32, vp]),
        "orc_bvh_build": (C.c_int, [vp, C.c_uint32, vp, vp]),
        "orc_hash_info": (C.c_int, [vp, C.c_uint32, vp]),
        "orc_create": (vp, [vp]),
        "orc_destroy": (None, [vp]),
        "orc_bvh_depth": (C.c_uint32, [vp]),
        "orc_get_bvh": (C.c_int, [vp, vp, C.c_uint32]),
        "orc_trace": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, vp, C.c_uint32, C.c_int, vp,
                                C.c_int]),
        "orc_emit": (C.c_int, [vp, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, vp, vp, vp, vp,
                               C.c_uint64, vp, C.c_int]),
        "orc_hash": (C.c_int, [vp, C.c_uint32, vp, C.c_uint32, vp, vp]),
        "orc_scan": (C.c_int, [vp, C.c_uint32, vp]),
        "orc_scatter": (C.c_int, [vp, vp, vp, vp, C.c_uint32, vp, C.c_uint32, vp, vp, vp, vp, vp]),
        "orc_gather": (C.c_int, [vp, C.c_uint32, vp, vp, vp, vp, vp, vp, C.c_float, vp, vp, vp, C.c_int]),
        "orc_render": (C.c_int, [vp, vp, C.c_uint32, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]),
        "orc_image": (C.c_int, [vp, vp, C.c_uint32, C.c_int, C.c_float, C.c_int, C.c_uint64, C.c_uint32, vp]),
        "orc_pcg": (None, [C.c_uint32, C.c_uint32, vp, vp]),
        "orc_encode_rgbe": (None, [vp, C.c_uint32, vp]),
        "orc_decode_rgbe": (None, [vp, C.c_uint32, vp]),
        "orc_encode_oct": (None, [vp, C.c_uint32, vp]),
        "orc_decode_oct": (None, [vp, C.c_uint32, vp]),
        "orc_get_hash": (None, [vp, C.c_uint32, vp, vp]),
        "orc_math": (C.c_float, [C.c_int, C.c_float, C.c_float]),
        "orc_frozen_render": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32, C.c_int, vp, vp, vp]),
        "orc_frozen_grad": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_int, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a: np.ndarray):
    return a.ctypes.data if a is not None else None


def _chk(code: int) -> None:
    if code != 0:
        raise RuntimeError(f"oracle call failed with status {code}")


def default_threads() -> int:
    return max(1, os.cpu_count() or 1)


class GeneratedScene:
    """A procedural scene built by the oracle library's copy of the scene generators, in the same
    phx_scene layout as phosphor_b200.SceneData.generate (same generator source, same seeded output).
    CPU-only callers use it so that nothing maps the CUDA library."""

    def __init__(self, kind: int, seed: int = 1, width: int = 512, height: int = 512, detail: int = 0):
        from phosphor_b200 import _capi as A  # ctypes declarations only; loads no library
        self.lib = load()
        spec = A.SceneSpec(kind=kind, seed=seed, width=width, height=height, detail=detail)
        self.scene = A.Scene()
        self._h = C.c_void_p()
        _chk(self.lib.orc_scene_generate(C.byref(spec), C.byref(self.scene), C.byref(self._h)))

    @property
    def n_triangles(self) -> int:
        return self.scene.n_triangles

    def __del__(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.orc_scene_free(self._h)
            self._h = None


class Oracle:
    """Reference restatement bound to one scene (phx_scene from phosphor_b200.SceneData or
    GeneratedScene)."""

    def __init__(self, scene):
        self.lib = load()
        self._scene = scene
        self.h = self.lib.orc_create(C.addressof(scene.scene))
        if not self.h:
            raise RuntimeError("oracle could not build the scene BVH")
        self.n_nodes = 2 * scene.scene.n_triangles - 1

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.orc_destroy(self.h)
            self.h = None

    @property
    def depth(self) -> int:
        return int(self.lib.orc_bvh_depth(self.h))

    def bvh(self) -> np.ndarray:
        out = np.empty((self.n_nodes, 8), dtype=np.float32)
        _chk(self.lib.orc_get_bvh(self.h, _p(out), self.n_nodes))
        return out

    def trace(self, width: int, height: int, seed: int, direct_samples: int, ids=None, prec: int = 0,
              threads: int | None = None) -> np.ndarray:
        """Hit points (n, 6, 4): pos, normal, throughput, base_color, direct, emission."""
        n = width * height if ids is None else len(ids)
        ids_a = None if ids is None else np.ascontiguousarray(ids, dtype=np.uint32)
        out = np.empty((n, 6, 4), dtype=np.float64 if prec else np.float32)
        _chk(self.lib.orc_trace(self.h, width, height, seed, direct_samples, _p(ids_a), n, prec, _p(out),
                                threads or default_threads()))
        return out

    def emit(self, tid_begin: int, tid_end: int, max_bounces: int, seed: int, prec: int = 0,
             threads: int | None = None):
        """Canonical stored photons of paths [tid_begin, tid_end): counts, pos (n,4), power, dir."""
        npaths = tid_end - tid_begin
        cap = npaths * max_bounces
        counts = np.empty(npaths, dtype=np.uint32)
        pos = np.empty((cap, 4), dtype=np.float64 if prec else np.float32)
        power = np.empty(cap, dtype=np.uint32)
        dirs = np.empty(cap, dtype=np.uint32)
        n = C.c_uint64()
        _chk(self.lib.orc_emit(self.h, tid_begin, tid_end, max_bounces, seed, prec, _p(counts), _p(pos), _p(power),
                               _p(dirs), cap, C.byref(n), threads or default_threads()))
        k = n.value
        return counts, pos[:k].copy(), power[:k].copy(), dirs[:k].copy()

    def render(self, params, rounds: int, prec: int = 0, threads: int | None = None, state=None):
        """Renderer::run for `rounds` rounds; returns dict(flux, weight, radiance, total, n_last, seconds)."""
        npx = params.width * params.height
        dt = np.float64 if prec else np.float32
        if state is None:
            state = {"flux": np.zeros((npx, 4), dt), "weight": np.zeros(npx, dt), "radiance": np.zeros((npx, 4), dt),
                     "total": 0}
        total = C.c_uint64(state["total"])
        n_last = C.c_uint32()
        secs = np.zeros(4, dtype=np.float64)
        import phosphor_b200._capi as A
        code = self.lib.orc_render(self.h, C.addressof(params), rounds, prec, threads or default_threads(),
                                   _p(state["flux"]), _p(state["weight"]), _p(state["radiance"]), C.byref(total),
                                   C.byref(n_last), _p(secs))
        _chk(code)
        state["total"] = total.value
        state["n_last"] = n_last.value
        state["seconds"] = secs
        return state

    def frozen_render(self, params, rounds: int, materials: np.ndarray, lights: np.ndarray,
                      threads: int | None = None):
        """The frozen-path estimator F(θ') of phx_frozen.hpp: paths and all decisions from this
        scene's own materials and lights (θ0), weights from `materials` / `lights` (θ', arrays of
        phx_material / phx_light records in the scene's order).  Returns (image (npx, 3) float64
        linear radiance, θ0 flux (npx, 4) float32, θ0 radiance (npx, 4) float32)."""
        npx = params.width * params.height
        img = np.empty((npx, 3), dtype=np.float64)
        flux = np.empty((npx, 4), dtype=np.float32)
        rad = np.empty((npx, 4), dtype=np.float32)
        mats = np.ascontiguousarray(materials)
        lts = np.ascontiguousarray(lights)
        _chk(self.lib.orc_frozen_render(self.h, C.addressof(params), rounds, _p(mats), len(mats), _p(lts), len(lts),
                                        threads or default_threads(), _p(img), _p(flux), _p(rad)))
        return img, flux, rad


def _frozen_grad(self, params, rounds: int, materials: np.ndarray, lights: np.ndarray, g_img: np.ndarray,
                 threads: int | None = None):
    """The analytic FP64 gradient of L(θ) = Σ g·F(θ) (forward-mode dual numbers through the
    frozen-path estimator) at θ = (materials, lights): (gradient laid out like
    phosphor_b200.adjoint.ParamTable, L)."""
    mats = np.ascontiguousarray(materials)
    lts = np.ascontiguousarray(lights)
    g = np.ascontiguousarray(g_img, dtype=np.float64).reshape(-1)
    assert g.size == 3 * params.width * params.height
    grad = np.zeros(4 * len(mats) + 3 * len(lts), np.float64)
    loss = C.c_double()
    _chk(self.lib.orc_frozen_grad(self.h, C.addressof(params), rounds, _p(mats), len(mats), _p(lts), len(lts), _p(g),
                                  threads or default_threads(), _p(grad), C.byref(loss)))
    return grad, loss.value


Oracle.frozen_grad = _frozen_grad


def bvh_build(tris_ptr, n: int):
    out = np.empty((2 * n - 1, 8), dtype=np.float32)
    depth = C.c_uint32()
    _chk(load().orc_bvh_build(tris_ptr, n, _p(out), C.byref(depth)))
    return out, depth.value


def hash_info(root_node: np.ndarray, grid_res: int) -> bytes:
    out = (C.c_uint8 * 48)()
    r = np.ascontiguousarray(root_node, dtype=np.float32)
    _chk(load().orc_hash_info(_p(r), grid_res, out))
    return bytes(out)


def hash_photons(pos4: np.ndarray, hash_data: bytes, buckets: int):
    pos4 = np.ascontiguousarray(pos4, dtype=np.float32)
    keys = np.empty(len(pos4), dtype=np.uint32)
    counts = np.empty(buckets, dtype=np.uint32)
    hd = (C.c_uint8 * 48).from_buffer_copy(hash_data)
    _chk(load().orc_hash(_p(pos4), len(pos4), hd, buckets, _p(keys), _p(counts)))
    return keys, counts


def scan(counts: np.ndarray) -> np.ndarray:
    counts = np.ascontiguousarray(counts, dtype=np.uint32)
    out = np.empty_like(counts)
    _chk(load().orc_scan(_p(counts), len(counts), _p(out)))
    return out


def scatter(pos4, power, dirs, keys, start):
    n, buckets = len(keys), len(start)
    pos4 = np.ascontiguousarray(pos4, dtype=np.float32)
    args = [np.ascontiguousarray(a, dtype=np.uint32) for a in (power, dirs, keys, start)]
    spos = np.empty_like(pos4)
    spow = np.empty(n, np.uint32)
    sdir = np.empty(n, np.uint32)
    end = np.empty(buckets, np.uint32)
    perm = np.empty(n, np.uint32)
    _chk(load().orc_scatter(_p(pos4), _p(args[0]), _p(args[1]), _p(args[2]), n, _p(args[3]), buckets, _p(spos),
                            _p(spow), _p(sdir), _p(end), _p(perm)))
    return spos, spow, sdir, end, perm


def gather(hp6, spos, spower, sdir, start, end, hash_data: bytes, alpha: float, flux, weight, radiance,
           threads: int | None = None):
    """gather_flux over all pixels; flux/weight/radiance (float32) are updated in place."""
    hp6 = np.ascontiguousarray(hp6, dtype=np.float32)
    hd = (C.c_uint8 * 48).from_buffer_copy(hash_data)
    a = [np.ascontiguousarray(x) for x in (spos, spower, sdir, start, end)]
    _chk(load().orc_gather(_p(hp6), len(hp6), _p(a[0]), _p(a[1]), _p(a[2]), _p(a[3]), _p(a[4]), hd, alpha,
                           _p(flux), _p(weight), _p(radiance), threads or default_threads()))


def image(flux, radiance, prec: int, exposure: float, tonemap: bool, total_photons: int, rounds: int) -> np.ndarray:
    n = len(flux)
    out = np.empty((n, 3), dtype=np.float64)
    _chk(load().orc_image(_p(np.ascontiguousarray(flux)), _p(np.ascontiguousarray(radiance)), n, prec, exposure,
                          int(tonemap), total_photons, rounds, _p(out)))
    return out


def pcg(seed: int, n: int):
    out = np.empty(n, np.uint32)
    outf = np.empty(n, np.float32)
    load().orc_pcg(seed, n, _p(out), _p(outf))
    return out, outf


def encode_rgbe(p4):
    p4 = np.ascontiguousarray(p4, dtype=np.float32)
    out = np.empty(len(p4), np.uint32)
    load().orc_encode_rgbe(_p(p4), len(p4), _p(out))
    return out


def decode_rgbe(words):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.empty((len(words), 4), np.float32)
    load().orc_decode_rgbe(_p(words), len(words), _p(out))
    return out


def encode_oct(d4):
    d4 = np.ascontiguousarray(d4, dtype=np.float32)
    out = np.empty(len(d4), np.uint32)
    load().orc_encode_oct(_p(d4), len(d4), _p(out))
    return out


def decode_oct(words):
    words = np.ascontiguousarray(words, dtype=np.uint32)
    out = np.empty((len(words), 4), np.float32)
    load().orc_decode_oct(_p(words), len(words), _p(out))
    return out


def get_hash(p4, hash_data: bytes):
    p4 = np.ascontiguousarray(p4, dtype=np.float32)
    out = np.empty(len(p4), np.uint32)
    hd = (C.c_uint8 * 48).from_buffer_copy(hash_data)
    load().orc_get_hash(_p(p4), len(p4), hd, _p(out))
    return out


def math(fn: str, x: float, y: float = 0.0) -> float:
    code = {"sin": 0, "cos": 1, "exp": 2, "log": 3, "pow": 4, "acos": 5, "atan2": 6}[fn]
    return float(load().orc_math(code, x, y))


def camera_make(pos, at, up, hfov: float, aspect: float, defocus: float = 0.0, focus: float = 1.0) -> bytes:
    """The scene generators' camera (Camera + focus + to_params) as 112 bytes of CameraParams."""
    f = [np.ascontiguousarray(v, np.float32) for v in (pos, at, up)]
    out = (C.c_uint8 * 112)()
    load().orc_camera_make(_p(f[0]), _p(f[1]), _p(f[2]), hfov, aspect, defocus, focus, out)
    return bytes(out)


def lum_pref_sum(lights_ptr, n: int) -> np.ndarray:
    out = np.empty(n, np.float32)
    load().orc_lum_pref_sum(lights_ptr, n, _p(out))
    return out
