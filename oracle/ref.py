"""TEST INFRASTRUCTURE ONLY — the reference's own SPPM code, compiled for the CPU.

Binds oracle/_ref/libsppm_ref.so, which oracle/build_ref_sppm.py builds from a reference checkout:
the reference's eight OpenCL kernels (kernels/*.cl with include/{common,device}/*.h) run over
their NDRanges on the host, and its host-side BVH builder, camera, photon-grid set-up, scene
sphere, luminance prefix sum and image formation.  `RefRenderer` drives them the way
Renderer::set_scene / Renderer::run do (src/renderer/renderer.cpp:22-161), so its state after
each round is the reference's.  Used only by tests/ and tests/golden/make_ref_sppm_golden.py, as
the checker of the oracle and of the CUDA library; the library never loads it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "libsppm_ref.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(f"{LIB_PATH} is not built (python oracle/build_ref_sppm.py path/to/reference)")
    lib = C.CDLL(str(LIB_PATH))
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    sig = {
        "ref_bvh_build": (C.c_int, [vp, u32, vp]),
        "ref_hash_info": (None, [vp, u32, vp]),
        "ref_scene_sphere": (None, [vp, vp, vp]),
        "ref_camera": (None, [vp, vp, vp, f32, f32, f32, f32, f32, vp]),
        "ref_lum_pref_sum": (None, [vp, u32, vp]),
        "ref_make_light": (None, [C.c_int, vp, vp, vp, f32, f32, u32, u32, u32, vp]),
        "ref_tonemap": (None, [u32, u32, f32, C.c_int, vp, vp, C.c_uint64, u32, vp]),
        "ref_scene_create": (vp, [vp, vp, vp, f32]),
        "ref_scene_destroy": (None, [vp]),
        "ref_trace": (C.c_int, [vp, u32, u32, u32, u32, vp, C.c_int]),
        "ref_emit": (C.c_int, [vp, u32, u32, u32, u32, u32, vp, vp, vp, vp]),
        "ref_hash_sort": (C.c_int, [vp, vp, vp, u32, vp, u32, vp, vp, vp, vp, vp, vp, vp]),
        "ref_gather": (C.c_int, [vp, u32, vp, vp, vp, u32, vp, vp, vp, f32, vp, vp, vp, C.c_int]),
        "ref_codecs": (None, [vp, u32, vp, vp, vp, vp]),
        "ref_pcg": (None, [u32, u32, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


def _threads() -> int:
    return max(1, os.cpu_count() or 1)


def bvh_build(tris_ptr, n: int) -> np.ndarray:
    """Bvh::Bvh (bvh.cpp:74-84): (2n-1, 8) float32 nodes."""
    out = np.empty((2 * n - 1, 8), np.float32)
    if load().ref_bvh_build(tris_ptr, n, _p(out)) != 0:
        raise RuntimeError("the reference BVH builder stopped (degenerate triangle box)")
    return out


def hash_info(root: np.ndarray, grid_res: int) -> bytes:
    out = (C.c_uint8 * 48)()
    load().ref_hash_info(_p(np.ascontiguousarray(root, np.float32)), grid_res, out)
    return bytes(out)


def scene_sphere(root: np.ndarray):
    c = np.empty(3, np.float32)
    r = np.empty(1, np.float32)
    load().ref_scene_sphere(_p(np.ascontiguousarray(root, np.float32)), _p(c), _p(r))
    return c, float(r[0])


def camera(pos, at, up, hfov: float, aspect: float, render_aspect: float, defocus: float = 0.0,
           focus: float = 1.0) -> bytes:
    f = [np.ascontiguousarray(v, np.float32) for v in (pos, at, up)]
    out = (C.c_uint8 * 112)()
    load().ref_camera(_p(f[0]), _p(f[1]), _p(f[2]), hfov, aspect, render_aspect, defocus, focus, out)
    return bytes(out)


LIGHT_POINT, LIGHT_SPOT, LIGHT_DIRECTIONAL, LIGHT_TEXTURED = 0, 1, 2, 3


def make_light(kind: int, pos=None, power=(1.0, 1.0, 1.0), direction=None, a: float = 0.0, b: float = 0.0,
               tex: int = 0xFFFFFFFF, start: int = 0, count: int = 0) -> bytes:
    """A light record (128 bytes) from the reference's constructors (light.cpp:4-45)."""
    f = [None if v is None else np.ascontiguousarray(v, np.float32) for v in (pos, power, direction)]
    out = (C.c_uint8 * 128)()
    load().ref_make_light(kind, _p(f[0]), _p(f[1]), _p(f[2]), a, b, tex, start, count, out)
    return bytes(out)


def lum_pref_sum(lights_ptr, n: int) -> np.ndarray:
    out = np.empty(n, np.float32)
    load().ref_lum_pref_sum(lights_ptr, n, _p(out))
    return out


def tonemap(w: int, h: int, flux4, radiance4, total_photons: int, rounds: int, exposure: float = 0.66,
            tone: bool = False) -> np.ndarray:
    out = np.empty((h * w, 3), np.uint8)
    load().ref_tonemap(w, h, exposure, int(tone), _p(np.ascontiguousarray(flux4, np.float32)),
                       _p(np.ascontiguousarray(radiance4, np.float32)), total_photons, rounds, _p(out))
    return out


def codecs(v4: np.ndarray):
    v4 = np.ascontiguousarray(v4, np.float32)
    n = len(v4)
    rgbe, octw = np.empty(n, np.uint32), np.empty(n, np.uint32)
    rd, od = np.empty((n, 4), np.float32), np.empty((n, 4), np.float32)
    load().ref_codecs(_p(v4), n, _p(rgbe), _p(octw), _p(rd), _p(od))
    return rgbe, octw, rd, od


def pcg(seed: int, n: int):
    u = np.empty(n, np.uint32)
    f = np.empty(n, np.float32)
    load().ref_pcg(seed, n, _p(u), _p(f))
    return u, f


class RefRenderer:
    """Renderer::set_scene + Renderer::run over the reference's own code (renderer.cpp:22-161).

    `scene` is a phx_scene holder (phosphor_b200.SceneData or oracle.GeneratedScene); `params`
    the ArgsList fields used by the round (width, height, photons_per_round, max_photon_bounces,
    grid_res, sppm_alpha, direct_samples, seed, max_photons_per_batch)."""

    def __init__(self, scene, params, threads: int | None = None):
        lib = load()
        self.scene = scene
        self.p = params
        self.threads = threads or _threads()
        n = scene.scene.n_triangles
        self.bvh = bvh_build(scene.scene.triangles, n)
        self.hash_data = hash_info(self.bvh[0], params.grid_res)
        self.center, self.radius = scene_sphere(self.bvh[0])
        self.buckets = params.grid_res ** 3 + 1
        self.h = lib.ref_scene_create(C.addressof(scene.scene), _p(self.bvh), _p(self.center), self.radius)
        npx = params.width * params.height
        self.flux = np.zeros((npx, 4), np.float32)
        self.weight = np.zeros(npx, np.float32)
        self.radiance = np.zeros((npx, 4), np.float32)
        self.rng_state = self._pcg_seed(params.seed)
        self.total_emitted = 0
        self.rounds = 0

    def __del__(self):
        if getattr(self, "h", None):
            load().ref_scene_destroy(self.h)
            self.h = None

    @staticmethod
    def _pcg_seed(seed: int) -> int:  # random.h:16-24
        s = (0 * 747796405 + 2891336453) & 0xFFFFFFFF
        s = (s + seed) & 0xFFFFFFFF
        return (s * 747796405 + 2891336453) & 0xFFFFFFFF

    def next_seed(self) -> int:  # random.h:29-34, renderer.cpp:65
        old = self.rng_state
        self.rng_state = (old * 747796405 + 2891336453) & 0xFFFFFFFF
        return (((old >> ((old >> 28) + 4)) ^ old) * 277803737) & 0xFFFFFFFF

    def trace_rays(self, seed: int) -> np.ndarray:
        p = self.p
        out = np.empty((p.width * p.height, 6, 4), np.float32)
        load().ref_trace(self.h, p.width, p.height, seed, p.direct_samples, _p(out), self.threads)
        return out

    def emit_photons(self, seed: int):
        p = self.p
        cap = p.photons_per_round * p.max_photon_bounces  # renderer.cpp:40
        pos = np.empty((cap, 4), np.float32)
        power = np.empty(cap, np.uint32)
        dirs = np.empty(cap, np.uint32)
        n = C.c_uint32()
        batch = getattr(p, "max_photons_per_batch", 1 << 20)
        load().ref_emit(self.h, p.photons_per_round, batch, p.max_photon_bounces, seed, cap, _p(pos), _p(power),
                        _p(dirs), C.byref(n))
        k = n.value
        return pos[:k].copy(), power[:k].copy(), dirs[:k].copy()

    def hash_and_sort(self, pos, power, dirs):
        n = len(pos)
        keys = np.empty(n, np.uint32)
        counts = np.empty(self.buckets, np.uint32)
        starts = np.empty(self.buckets, np.uint32)
        ends = np.empty(self.buckets, np.uint32)
        spos = np.empty((n, 4), np.float32)
        spow = np.empty(n, np.uint32)
        sdir = np.empty(n, np.uint32)
        hd = (C.c_uint8 * 48).from_buffer_copy(self.hash_data)
        load().ref_hash_sort(_p(np.ascontiguousarray(pos)), _p(np.ascontiguousarray(power)),
                             _p(np.ascontiguousarray(dirs)), n, hd, self.buckets, _p(keys), _p(counts), _p(starts),
                             _p(ends), _p(spos), _p(spow), _p(sdir))
        return dict(keys=keys, counts=counts, starts=starts, ends=ends, pos=spos, power=spow, dir=sdir)

    def gather_flux(self, hp, grid):
        hd = (C.c_uint8 * 48).from_buffer_copy(self.hash_data)
        n = len(grid["pos"])
        load().ref_gather(_p(np.ascontiguousarray(hp)), len(hp), _p(grid["pos"]), _p(grid["power"]), _p(grid["dir"]),
                          n, _p(grid["starts"]), _p(grid["ends"]), hd, self.p.sppm_alpha, _p(self.flux),
                          _p(self.weight), _p(self.radiance), self.threads)

    def round(self, keep: bool = False) -> dict:
        """One SPPM round (renderer.cpp:64-73); returns that round's stage outputs if `keep`."""
        seed = self.next_seed()
        hp = self.trace_rays(seed)
        pos, power, dirs = self.emit_photons(seed)
        if len(pos) == 0:
            raise RuntimeError("no photon hit")  # renderer.cpp:117-118
        grid = self.hash_and_sort(pos, power, dirs)
        self.gather_flux(hp, grid)
        self.total_emitted += self.p.photons_per_round
        self.rounds += 1
        if not keep:
            return {"seed": seed}
        return dict(seed=seed, hp=hp, photon_pos=pos, photon_power=power, photon_dir=dirs, **{
            f"grid_{k}": v for k, v in grid.items()})

    def image_u8(self, exposure: float = 0.66, tone: bool = False) -> np.ndarray:
        return tonemap(self.p.width, self.p.height, self.flux, self.radiance, self.total_emitted, self.rounds,
                       exposure, tone)
