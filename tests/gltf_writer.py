"""A minimal glTF 2.0 writer for the scene-ingest tests: builds documents from numpy arrays and
writes them as .glb, or as .gltf with an external .bin or a data URI.  PNG images are encoded
here with zlib (colour types grey, grey+alpha, RGB, RGBA and palette; 8 or 16 bits)."""
from __future__ import annotations

import base64
import json
import struct
import zlib
from pathlib import Path

import numpy as np


def png_bytes(img: np.ndarray, palette: np.ndarray | None = None, filt: int = 4) -> bytes:
    """img: (h, w) grey, (h, w, 2|3|4) uint8 or uint16, or (h, w) palette indices with `palette`."""
    img = np.asarray(img)
    if palette is not None:
        ctype, depth = 3, 8
    else:
        ctype = {1: 0, 2: 4, 3: 2, 4: 6}[1 if img.ndim == 2 else img.shape[2]]
        depth = 16 if img.dtype == np.uint16 else 8
    h, w = img.shape[:2]
    arr = img.reshape(h, -1)
    if depth == 16:
        rows = arr.astype(">u2").view(np.uint8).reshape(h, -1)
    else:
        rows = arr.astype(np.uint8)
    bpp = max(1, (rows.shape[1] // w))
    out = bytearray()
    prev = np.zeros(rows.shape[1], np.int32)
    for y in range(h):
        cur = rows[y].astype(np.int32)
        f = filt if y % 2 == 0 else (y // 2) % 5  # mix the filter types
        a = np.concatenate([np.zeros(bpp, np.int32), cur[:-bpp]])
        c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]])
        if f == 0:
            enc = cur
        elif f == 1:
            enc = cur - a
        elif f == 2:
            enc = cur - prev
        elif f == 3:
            enc = cur - (a + prev) // 2
        else:
            p = a + prev - c
            pa, pb, pc = np.abs(p - a), np.abs(p - prev), np.abs(p - c)
            pred = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, prev, c))
            enc = cur - pred
        out.append(f)
        out += (enc & 0xFF).astype(np.uint8).tobytes()
        prev = cur

    def chunk(t: bytes, data: bytes) -> bytes:
        return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xFFFFFFFF)

    hdr = struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, 0)
    body = chunk(b"IHDR", hdr)
    if palette is not None:
        body += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    body += chunk(b"IDAT", zlib.compress(bytes(out)))
    return b"\x89PNG\r\n\x1a\n" + body + chunk(b"IEND", b"")


class Gltf:
    def __init__(self):
        self.doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": []}], "nodes": [], "meshes": [],
                    "materials": [], "accessors": [], "bufferViews": [], "buffers": [], "cameras": [],
                    "textures": [], "images": []}
        self.bin = bytearray()

    def _view(self, data: bytes) -> int:
        while len(self.bin) % 4:
            self.bin.append(0)
        self.doc["bufferViews"].append({"buffer": 0, "byteOffset": len(self.bin), "byteLength": len(data)})
        self.bin += data
        return len(self.doc["bufferViews"]) - 1

    def accessor(self, arr: np.ndarray, ctype: int = 5126, normalized: bool = False) -> int:
        arr = np.ascontiguousarray(arr)
        typ = {1: "SCALAR", 2: "VEC2", 3: "VEC3", 4: "VEC4"}[1 if arr.ndim == 1 else arr.shape[1]]
        dt = {5126: np.float32, 5125: np.uint32, 5123: np.uint16, 5121: np.uint8, 5122: np.int16, 5120: np.int8}[ctype]
        v = self._view(arr.astype(dt).tobytes())
        acc = {"bufferView": v, "componentType": ctype, "count": len(arr), "type": typ}
        if normalized:
            acc["normalized"] = True
        if ctype == 5126 and typ != "SCALAR":
            acc["min"] = arr.min(axis=0).tolist()
            acc["max"] = arr.max(axis=0).tolist()
        self.doc["accessors"].append(acc)
        return len(self.doc["accessors"]) - 1

    def material(self, **m) -> int:
        self.doc["materials"].append(m)
        return len(self.doc["materials"]) - 1

    def image_png(self, png: bytes, embed: str = "view") -> int:
        if embed == "view":
            self.doc["images"].append({"bufferView": self._view(png), "mimeType": "image/png"})
        else:
            self.doc["images"].append({"uri": "data:image/png;base64," + base64.b64encode(png).decode()})
        self.doc["textures"].append({"source": len(self.doc["images"]) - 1})
        return len(self.doc["textures"]) - 1

    def mesh(self, prims: list[dict]) -> int:
        self.doc["meshes"].append({"primitives": prims})
        return len(self.doc["meshes"]) - 1

    def node(self, root: bool = True, **n) -> int:
        self.doc["nodes"].append(n)
        i = len(self.doc["nodes"]) - 1
        if root:
            self.doc["scenes"][0]["nodes"].append(i)
        return i

    def camera(self, yfov: float, aspect: float) -> int:
        self.doc["cameras"].append({"type": "perspective",
                                    "perspective": {"yfov": yfov, "aspectRatio": aspect, "znear": 0.01}})
        return len(self.doc["cameras"]) - 1

    def light(self, **l) -> int:
        ext = self.doc.setdefault("extensions", {}).setdefault("KHR_lights_punctual", {"lights": []})
        ext["lights"].append(l)
        self.doc.setdefault("extensionsUsed", [])
        if "KHR_lights_punctual" not in self.doc["extensionsUsed"]:
            self.doc["extensionsUsed"].append("KHR_lights_punctual")
        return len(ext["lights"]) - 1

    def _clean(self) -> dict:
        return {k: v for k, v in self.doc.items() if v != []}

    def write_glb(self, path: Path) -> None:
        doc = self._clean()
        doc["buffers"] = [{"byteLength": len(self.bin)}]
        js = json.dumps(doc).encode()
        js += b" " * (-len(js) % 4)
        b = bytes(self.bin) + b"\0" * (-len(self.bin) % 4)
        total = 12 + 8 + len(js) + 8 + len(b)
        data = struct.pack("<III", 0x46546C67, 2, total) + struct.pack("<II", len(js), 0x4E4F534A) + js + \
            struct.pack("<II", len(b), 0x004E4942) + b
        Path(path).write_bytes(data)

    def write_gltf(self, path: Path, data_uri: bool = False) -> None:
        doc = self._clean()
        path = Path(path)
        if data_uri:
            doc["buffers"] = [{"byteLength": len(self.bin),
                               "uri": "data:application/octet-stream;base64," + base64.b64encode(self.bin).decode()}]
        else:
            name = path.stem + " data.bin"  # a space: written percent-encoded in the URI
            (path.parent / name).write_bytes(bytes(self.bin))
            doc["buffers"] = [{"byteLength": len(self.bin), "uri": name.replace(" ", "%20")}]
        path.write_text(json.dumps(doc, indent=1))
