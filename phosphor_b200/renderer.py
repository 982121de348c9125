"""Reference-shaped host API over libphx.so.

Mirrors the reference renderer's host interface (include/host/renderer.hpp:16-72,
include/host/cmd_args.hpp:11-65): an ArgsList of the same flags and defaults, a Renderer with
set_scene(scene) and run(), and the per-stage methods trace_rays / emit_photons /
hash_and_sort_photons / gather_flux that the reference keeps private (exposed here so stage
parity can be checked).  Every call goes through the C ABI; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import dataclasses
import struct
import time
import zlib
from pathlib import Path

import numpy as np

from . import _capi as A


@dataclasses.dataclass
class ArgsList:
    """The flags of include/host/cmd_args.hpp:36-65 with the reference defaults (:11-34)."""
    width: int = 1024
    height: int = 1024
    exposure: float = 0.66
    tonemap: bool = False
    max_photons_per_batch: int = 1 << 20
    workgroup_size: int = 32
    seed: int = 2137
    photons_per_round: int = 1 << 20
    ray_step: float = 0.0001  # parsed but unused by the reference (cmd_args.hpp:48)
    max_photon_bounces: int = 16
    grid_res: int = 64
    defocus_angle: float = 0.0
    focus_distance: float = 1.0
    sppm_rounds: int = 64
    sppm_alpha: float = 0.7
    direct_samples: int = 16
    output_dir: str = ""
    save_snapshots: bool = False
    # B200 build knobs (no reference counterpart; results do not depend on them)
    flags: int = 0           # PHX_F_*
    bvh_leaf_size: int = 0   # 0 = library default

    def params(self) -> A.Params:
        p = A.Params()
        p.width, p.height = self.width, self.height
        p.photons_per_round = self.photons_per_round
        p.max_photon_bounces = self.max_photon_bounces
        p.grid_res = self.grid_res
        p.sppm_alpha = self.sppm_alpha
        p.direct_samples = self.direct_samples
        p.seed = self.seed
        p.flags = self.flags
        p.bvh_leaf_size = self.bvh_leaf_size
        return p


def _arr(ptr, n: int, ctype) -> np.ndarray:
    if n == 0 or not ptr:
        return np.zeros(0, dtype=np.uint8)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,))


class SceneData:
    """Host scene arrays (the reference's SceneData, include/host/scene_data.hpp:21-42) plus the
    resolved camera.  `generate` builds one of the procedural scenes in library-owned memory."""

    def __init__(self, scene: A.Scene, owner=None, keep=()):
        self.scene = scene
        self._owner = owner
        self._keep = keep

    @classmethod
    def generate(cls, kind: int, seed: int = 1, width: int = 512, height: int = 512, detail: int = 0) -> "SceneData":
        lib = A.load()
        spec = A.SceneSpec(kind=kind, seed=seed, width=width, height=height, detail=detail)
        sc = A.Scene()
        h = C.c_void_p()
        A.check(lib.phx_scene_generate(C.byref(spec), C.byref(sc), C.byref(h)))
        return cls(sc, owner=h)

    @classmethod
    def load_gltf(cls, path: str | os.PathLike, width: int = 0, height: int = 0, defocus_angle: float = 0.0,
                  focus_distance: float = 1.0, camera: int = 0) -> "SceneData":
        """read_gltf_scene (src/parsers/scene.cpp:206-233) for a .gltf or .glb file, with the
        render size's aspect and the focus settings applied to the chosen camera (renderer.cpp:24-28)."""
        lib = A.load()
        opt = A.GltfOptions(width=width, height=height, defocus_angle=defocus_angle, focus_distance=focus_distance,
                            camera=camera)
        sc = A.Scene()
        h = C.c_void_p()
        A.check(lib.phx_scene_load_gltf(os.fsencode(str(path)), C.byref(opt), C.byref(sc), C.byref(h)))
        return cls(sc, owner=h)

    def __del__(self):
        if getattr(self, "_owner", None) is not None and self._owner.value:
            try:
                A.load().phx_scene_free(self._owner)
            except Exception:
                pass
            self._owner = None

    # numpy views in the reference layouts
    @property
    def n_triangles(self) -> int:
        return self.scene.n_triangles

    def triangles(self) -> np.ndarray:
        return _arr(self.scene.triangles, self.scene.n_triangles, A.Triangle)

    def materials(self) -> np.ndarray:
        return _arr(self.scene.materials, self.scene.n_materials, A.Material)

    def lights(self) -> np.ndarray:
        return _arr(self.scene.lights, self.scene.n_lights, A.Light)

    def triangle_vertices(self) -> np.ndarray:
        """(n, 3, 3) float32 vertex positions."""
        t = self.triangles()
        raw = np.frombuffer(t.tobytes(), dtype=np.float32).reshape(len(t), 44)
        return raw[:, :12].reshape(len(t), 3, 4)[:, :, :3].copy()

    def with_camera(self, camera: A.CameraParams) -> "SceneData":
        sc = A.Scene.from_buffer_copy(self.scene)
        sc.camera = camera
        return SceneData(sc, owner=None, keep=(self,))


def _prefer_bundled_nccl() -> None:
    """Points PHX_NCCL_LIB at the NCCL that this Python environment bundles (the one torch links),
    so that the library and a framework in the same process share one NCCL."""
    if os.environ.get("PHX_NCCL_LIB"):
        return
    import importlib.util
    spec = importlib.util.find_spec("nvidia.nccl")
    for loc in (spec.submodule_search_locations or []) if spec else []:
        cand = Path(loc) / "lib" / "libnccl.so.2"
        if cand.exists():
            os.environ["PHX_NCCL_LIB"] = str(cand)
            return


def nccl_unique_id() -> bytes:
    """A fresh NCCL unique id (128 bytes) for phx_shard_nccl, made on one rank and sent to all."""
    _prefer_bundled_nccl()
    buf = (C.c_uint8 * 128)()
    A.check(A.load().phx_nccl_unique_id(buf, 128))
    return bytes(buf)


def bvh_build(scene: SceneData) -> tuple[np.ndarray, int]:
    """The reference's median-split BVH (src/renderer/bvh.cpp:74-84) as (2n-1, 8) float32 nodes."""
    lib = A.load()
    n = scene.scene.n_triangles
    out = (A.BvhNode * (2 * n - 1))()
    depth = C.c_uint32()
    A.check(lib.phx_bvh_build(scene.scene.triangles, n, out, C.byref(depth)))
    return np.frombuffer(bytes(out), dtype=np.float32).reshape(2 * n - 1, 8).copy(), depth.value


@dataclasses.dataclass
class TraversalBvh:
    nodes: np.ndarray      # (n_nodes, 16) child pairs or (n_nodes, 28) 4-wide, float32 (refs as int32 bits)
    trirec: np.ndarray     # (n, 12) float32, leaf order
    leaf_tri: np.ndarray   # (n,) uint32
    root: int
    depth: int
    wdepth: int
    build_ms: float


def traversal_bvh(scene: SceneData, max_leaf: int = 4, wide: int = 1, device: int = -1) -> TraversalBvh:
    """The SAH traversal tree the kernels walk, built on the host (device < 0) or on a GPU.
    wide: 0 child pairs (16 floats per node), 1 4-wide nodes (28 floats), 2 4-wide nodes with 8-bit
    child boxes (16 words)."""
    lib = A.load()
    n = scene.scene.n_triangles
    per = 28 if int(wide) == 1 else 16
    nodes = np.zeros((max(n, 1), 28), np.float32)
    trirec = np.zeros((n, 12), np.float32)
    leaf = np.zeros(n, np.uint32)
    out = A.BvhPacked()
    out.nodes = nodes.ctypes.data_as(C.POINTER(C.c_float))
    out.trirec = trirec.ctypes.data_as(C.POINTER(C.c_float))
    out.leaf_tri = leaf.ctypes.data_as(C.POINTER(C.c_uint32))
    A.check(lib.phx_traversal_bvh_build(scene.scene.triangles, n, max_leaf, int(wide), device, C.byref(out)))
    flat = nodes.reshape(-1)[:out.n_nodes * per].reshape(out.n_nodes, per).copy()
    return TraversalBvh(flat, trirec, leaf, out.root, out.depth, out.wdepth, out.build_ms)


def camera_make(position, look_at, up, hfov_deg, aspect, defocus_angle=0.0, focus_distance=1.0) -> A.CameraParams:
    lib = A.load()
    f3 = C.c_float * 3
    cam = A.CameraParams()
    A.check(lib.phx_camera_make(f3(*position), f3(*look_at), f3(*up), hfov_deg, aspect, defocus_angle,
                                focus_distance, C.byref(cam)))
    return cam


class Renderer:
    """Renderer(args) -> set_scene(scene) -> run(); the stage methods mirror renderer.cpp:90-161."""

    def __init__(self, args: ArgsList | None = None, output_dir: str | None = None, metadata: str = "",
                 device: int = 0):
        self.args = args or ArgsList()
        self.output_dir = Path(output_dir) if output_dir else None
        self.metadata = metadata
        self.device = device
        self.ctx = None
        self._lib = A.load()
        self._scene = None

    # Renderer::set_scene (renderer.cpp:22-57)
    def set_scene(self, scene: SceneData) -> None:
        self.close()
        p = self.args.params()
        ctx = C.c_void_p()
        A.check(self._lib.phx_create(C.byref(scene.scene), C.byref(p), self.device, C.byref(ctx)))
        self.ctx = ctx
        self._scene = scene

    def close(self) -> None:
        if self.ctx is not None and self.ctx.value:
            self._lib.phx_destroy(self.ctx)
        self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _need(self):
        if self.ctx is None:
            raise A.PhxError(A.PHX_E_STATE, "set_scene() first")
        return self.ctx

    # the reference's per-pass stages
    def trace_rays(self, seed: int) -> None:
        A.check(self._lib.phx_trace_rays(self._need(), seed))

    def emit_photons(self, seed: int) -> int:
        A.check(self._lib.phx_emit_photons(self._need(), seed))
        return self.info().n_photons

    def hash_and_sort_photons(self) -> None:
        A.check(self._lib.phx_hash_sort(self._need()))

    def gather_flux(self, alpha: float | None = None) -> None:
        A.check(self._lib.phx_gather(self._need(), self.args.sppm_alpha if alpha is None else alpha))

    def round(self) -> None:
        """One round in the plain per-pass form (renderer.cpp:64-78)."""
        A.check(self._lib.phx_round(self._need()))

    def iterate(self, rounds: int) -> None:
        """`rounds` rounds replayed from one captured CUDA graph."""
        A.check(self._lib.phx_iterate(self._need(), rounds))

    def round_seeded(self, seed: int) -> None:
        """One graph-replayed round whose seed comes from the host (asynchronous)."""
        A.check(self._lib.phx_round_seeded(self._need(), seed))

    def sync(self) -> None:
        A.check(self._lib.phx_sync(self._need()))

    # Renderer::run (renderer.cpp:59-88)
    def run(self, graph: bool = True) -> np.ndarray:
        rounds = self.args.sppm_rounds
        done = 0
        while done < rounds:
            step = rounds - done
            if self.args.save_snapshots:  # stop at power-of-two rounds for snapshots
                nxt = 1
                while nxt <= done:
                    nxt <<= 1
                step = min(step, nxt - done)
            if graph:
                self.iterate(step)
            else:
                for _ in range(step):
                    self.round()
            done += step
            if (self.args.save_snapshots and (done & (done - 1)) == 0) or done == rounds:
                self.save_snapshot(done)
        return self.image()

    def save_snapshot(self, round_: int) -> Path | None:
        if self.output_dir is None:
            return None
        self.output_dir.mkdir(parents=True, exist_ok=True)
        path = self.output_dir / f"{round_:06d}.png"
        write_png(path, self.image_u8())
        return path

    def info(self) -> A.Info:
        inf = A.Info()
        A.check(self._lib.phx_get_info(self._need(), C.byref(inf)))
        return inf

    def read(self, name: str) -> np.ndarray:
        """A device buffer in the reference layout (see PHX_BUF_* in include/phx.h)."""
        info = self.info()
        dt, width = A.BUF_DTYPE[name]
        count = {"CELL_COUNT": info.bucket_count, "CELL_START": info.bucket_count, "CELL_END": info.bucket_count,
                 "EMIT_COUNT": info.photons_per_round, "BVH_NODES": info.n_bvh_nodes, "ROUND_RNG": 1}.get(name)
        if count is None:
            count = info.n_pixels if name.startswith("HP_") or name in ("FLUX", "RADIANCE", "PHOTON_WEIGHT") \
                else info.n_photons
        out = np.empty((count, width) if width > 1 else (count,), dtype=dt)
        A.check(self._lib.phx_read_buffer(self._need(), A.BUF[name], out.ctypes.data, 0, out.nbytes))
        return out

    def write(self, name: str, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr)
        A.check(self._lib.phx_write_buffer(self._need(), A.BUF[name], a.ctypes.data, 0, a.nbytes))

    def set_n_photons(self, n: int) -> None:
        A.check(self._lib.phx_set_n_photons(self._need(), n))

    def image(self, exposure: float | None = None, tonemap: bool | None = None) -> np.ndarray:
        """Linear-to-display image of output.cpp:52-83 (before u8 quantisation), (H, W, 3) float32."""
        inf = self.info()
        out = np.empty((inf.height, inf.width, 3), dtype=np.float32)
        A.check(self._lib.phx_image(self._need(), self.args.exposure if exposure is None else exposure,
                                    int(self.args.tonemap if tonemap is None else tonemap), 0, 0,
                                    out.ctypes.data, None))
        return out

    def image_u8(self) -> np.ndarray:
        inf = self.info()
        out = np.empty((inf.height, inf.width, 3), dtype=np.uint8)
        A.check(self._lib.phx_image(self._need(), self.args.exposure, int(self.args.tonemap), 0, 0, None,
                                    out.ctypes.data))
        return out

    def tuning(self) -> A.Tuning:
        t = A.Tuning()
        A.check(self._lib.phx_get_tuning(self._need(), C.byref(t)))
        return t

    def set_tuning(self, t: A.Tuning) -> None:
        A.check(self._lib.phx_set_tuning(self._need(), C.byref(t)))

    def profile(self, on: bool) -> None:
        A.check(self._lib.phx_profile(self._need(), int(on)))

    def autotune(self, rounds_per_trial: int = 4) -> A.Tuning:
        """Times candidate launch tunings on graph-replayed rounds, keeps the fastest (results are
        bit-identical under all of them; the render state is restored)."""
        t = A.Tuning()
        A.check(self._lib.phx_autotune(self._need(), rounds_per_trial, C.byref(t)))
        return t

    def stage_ms(self) -> dict[str, float]:
        out = (C.c_float * len(A.STAGES))()
        A.check(self._lib.phx_stage_ms(self._need(), out, len(A.STAGES)))
        return dict(zip(A.STAGES, list(out)))

    def stream(self) -> int:
        return int(self._lib.phx_get_stream(self._need()))

    # one image over several GPUs (no reference counterpart; see include/phx.h)
    def shard(self, rank: int, world: int) -> None:
        A.check(self._lib.phx_shard(self._need(), rank, world))

    def shard_begin(self) -> int:
        """Seed, camera pass over this rank's pixels, photon pass over its paths; photons stored."""
        n = C.c_uint32()
        A.check(self._lib.phx_shard_begin(self._need(), C.byref(n)))
        return n.value

    def shard_get_photons(self, n: int) -> tuple[np.ndarray, np.ndarray]:
        pos = np.empty((n, 4), np.float32)
        pd = np.empty((n, 2), np.uint32)
        A.check(self._lib.phx_shard_get_photons(self._need(), pos.ctypes.data, pd.ctypes.data, n))
        return pos, pd

    def shard_put_photons(self, pos: np.ndarray, pd: np.ndarray) -> None:
        pos = np.ascontiguousarray(pos, np.float32)
        pd = np.ascontiguousarray(pd, np.uint32)
        A.check(self._lib.phx_shard_put_photons(self._need(), pos.ctypes.data, pd.ctypes.data, len(pos)))

    def shard_end(self) -> None:
        A.check(self._lib.phx_shard_end(self._need()))

    def shard_nccl(self, unique_id: bytes) -> None:
        _prefer_bundled_nccl()
        buf = (C.c_uint8 * 128).from_buffer_copy(unique_id)
        A.check(self._lib.phx_shard_nccl(self._need(), buf))

    def shard_round(self) -> None:
        A.check(self._lib.phx_shard_round(self._need()))

    # differentiation (no reference counterpart; see include/phx.h)
    def n_params(self) -> int:
        n = C.c_uint32()
        A.check(self._lib.phx_adjoint_n_params(self._need(), C.byref(n)))
        return n.value

    def set_materials(self, materials: np.ndarray) -> None:
        """Replaces the material table (phx_material records, the scene's count and order)."""
        m = np.ascontiguousarray(materials)
        A.check(self._lib.phx_set_materials(self._need(), m.ctypes.data, len(m)))

    def set_lights(self, lights: np.ndarray) -> None:
        lt = np.ascontiguousarray(lights)
        A.check(self._lib.phx_set_lights(self._need(), lt.ctypes.data, len(lt)))

    def adjoint_forward(self, rounds: int) -> np.ndarray:
        """Fresh render of `rounds` rounds recorded for the adjoint; linear image (H, W, 3)."""
        a = self.args
        img = np.empty((a.height, a.width, 3), dtype=np.float32)
        A.check(self._lib.phx_adjoint_forward(self._need(), rounds, img.ctypes.data))
        return img

    def adjoint_backward(self, dl_dimage: np.ndarray) -> np.ndarray:
        """dL/dθ (4 per material: base r, g, b, roughness; 3 per light: power r, g, b)."""
        g = np.ascontiguousarray(dl_dimage, dtype=np.float32)
        a = self.args
        if g.size != a.width * a.height * 3:
            raise ValueError("dL/dI must have width*height*3 entries")
        n = self.n_params()
        out = np.empty(n, dtype=np.float32)
        A.check(self._lib.phx_adjoint_backward(self._need(), g.ctypes.data, out.ctypes.data, n))
        return out


class Batch:
    """Many scenes advanced together: one launch per stage for all scenes (phx_batch_*)."""

    def __init__(self, scenes: list[SceneData], args: list[ArgsList], device: int = 0):
        self._lib = A.load()
        n = len(scenes)
        sc = (A.Scene * n)(*[s.scene for s in scenes])
        pr = (A.Params * n)(*[a.params() for a in args])
        h = C.c_void_p()
        A.check(self._lib.phx_batch_create(sc, pr, n, device, C.byref(h)))
        self.h = h
        self.n = n
        self.args = args
        self._scenes = scenes

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self._lib.phx_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, rounds: int, graph: bool = True) -> None:
        A.check(self._lib.phx_batch_iterate(self.h, rounds, 1 if graph else 0))

    def tuning(self) -> A.Tuning:
        t = A.Tuning()
        A.check(self._lib.phx_get_tuning(self.h, C.byref(t)))
        return t

    def set_tuning(self, t: A.Tuning) -> None:
        A.check(self._lib.phx_set_tuning(self.h, C.byref(t)))

    def set_active(self, s: int, active: bool) -> None:
        """Retire (False) or resume a scene: retired scenes cost no work in later rounds."""
        A.check(self._lib.phx_batch_set_active(self.h, s, int(active)))

    def info(self, s: int) -> A.Info:
        inf = A.Info()
        A.check(self._lib.phx_batch_get_info(self.h, s, C.byref(inf)))
        return inf

    def read(self, s: int, name: str) -> np.ndarray:
        info = self.info(s)
        dt, width = A.BUF_DTYPE[name]
        count = {"CELL_COUNT": info.bucket_count, "CELL_START": info.bucket_count, "CELL_END": info.bucket_count,
                 "EMIT_COUNT": info.photons_per_round, "BVH_NODES": info.n_bvh_nodes, "ROUND_RNG": 1}.get(name)
        if count is None:
            count = info.n_pixels if name.startswith("HP_") or name in ("FLUX", "RADIANCE", "PHOTON_WEIGHT") \
                else info.n_photons
        out = np.empty((count, width) if width > 1 else (count,), dtype=dt)
        A.check(self._lib.phx_batch_read_buffer(self.h, s, A.BUF[name], out.ctypes.data, 0, out.nbytes))
        return out

    def image(self, s: int, exposure: float = 0.66, tonemap: bool = False) -> np.ndarray:
        inf = self.info(s)
        out = np.empty((inf.height, inf.width, 3), dtype=np.float32)
        A.check(self._lib.phx_batch_image(self.h, s, exposure, int(tonemap), out.ctypes.data))
        return out

    def stream(self) -> int:
        return int(self._lib.phx_get_stream(self.h))

    def profile(self, on: bool) -> None:
        A.check(self._lib.phx_profile(self.h, int(on)))

    def autotune(self, rounds_per_trial: int = 4) -> A.Tuning:
        """phx_autotune over the whole batch (every stage launches all scenes at once)."""
        t = A.Tuning()
        A.check(self._lib.phx_autotune(self.h, rounds_per_trial, C.byref(t)))
        return t

    def stage_ms(self) -> dict[str, float]:
        out = (C.c_float * len(A.STAGES))()
        A.check(self._lib.phx_stage_ms(self.h, out, len(A.STAGES)))
        return dict(zip(A.STAGES, list(out)))


def write_png(path: Path | str, rgb: np.ndarray) -> None:
    """Minimal RGB8 PNG writer (the reference uses stb_image_write, output.cpp:86-87)."""
    h, w, _ = rgb.shape
    raw = b"".join(b"\x00" + rgb[y].astype(np.uint8).tobytes() for y in range(h))

    def chunk(tag: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 2, 0, 0, 0)) + \
        chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    Path(path).write_bytes(png)
