"""TEST INFRASTRUCTURE ONLY — builds the reference's own SPPM code for the host CPU.

The reference's SPPM path is OpenCL C (kernels/*.cl and include/{common,device}/*.h) driven by a
C++ host that needs OpenCL, glm, assimp and stb, none of which exists here.  This recipe compiles
what it can of that code from where it lies in a reference checkout, with no copy entering the
repository (all output goes to the git-ignored oracle/_ref/):

1. Kernels.  The eight kernels are preprocessed together as OpenCL C (`__OPENCL_C_VERSION__`
   defined, the address-space qualifiers defined away, `__local` as `static`, which gives a work
   group's items one shared array) into one translation unit.  Two pieces of OpenCL C syntax that
   C++ cannot parse are rewritten: the vector literals `(float4)(...)` and `(float2)(...)` become
   calls of float4_ctor/float2_ctor, and the rvalue swizzle `.yx` becomes `.yx_()`; the recipe
   checks that no other vector literal or swizzle remains.  The result, oracle/_ref/
   sppm_kernels.inc, is compiled inside oracle/ref_kernels.cpp, which supplies the OpenCL types,
   builtins, work-item ids and barriers and launches each kernel over its NDRange.
2. Host code.  src/renderer/{bvh,camera,light}.cpp are compiled as they are, against
   the stand-in headers in oracle/ref_shim/ (OpenCL host vector types, glm 1.0.3's few functions,
   logging).  Three functions that live in classes tied to OpenCL buffers or image I/O are read
   out of their files by brace matching into oracle/_ref/host_extract.inc: output.cpp's tone_map
   and apply_tonemap, the scene-sphere part of ShadingBuffers::upload (shading.cpp) and
   SceneData::build_lum_pref_sum (scene_data.cpp).
3. g++ links everything into oracle/_ref/libsppm_ref.so with -ffp-contract=off, so every float
   operation is the one written.

    python oracle/build_ref_sppm.py path/to/reference     (or PHX_REFERENCE_DIR=path/to/reference)

oracle/ref.py binds the library; tests/golden/make_ref_sppm_golden.py runs it to make the
committed fixtures that pin the oracle (and, on the GPU, the CUDA library) to the reference.
"""
from __future__ import annotations

import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT_DIR = HERE / "_ref"
OUT = OUT_DIR / "libsppm_ref.so"
SHIM = HERE / "ref_shim"

KERNELS = ["trace_rays", "emit_photons", "hash_photons", "scan_small_chunks", "scan_big_chunks", "scan_add_offsets",
           "scatter_photons", "gather_flux"]
CXX = ["g++", "-O2", "-std=c++20", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-w"]


def _run(cmd: list[str], stdin: str | None = None) -> str:
    res = subprocess.run(cmd, input=stdin, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{res.stdout[-4000:]}\n{res.stderr[-4000:]}")
    return res.stdout


def preprocess_kernels(ref: Path) -> str:
    wrapper = "".join(f'#include "{k}.cl"\n' for k in KERNELS)
    wrapper += "constexpr uint SCAN_WG_SIZE_VALUE = SCAN_WG_SIZE;\nconstexpr uint SCAN_CHUNK_SIZE_VALUE = SCAN_CHUNK_SIZE;\n"
    cmd = ["g++", "-E", "-x", "c++", "-std=c++20", "-D__OPENCL_C_VERSION__=120", "-D__kernel=", "-D__global=",
           "-D__local=static", "-D__constant=const", "-D__private=", f"-I{ref / 'kernels'}", f"-I{ref / 'include'}", "-"]
    return _run(cmd, wrapper)


VEC_LITERAL = re.compile(r"\(\s*(float[24])\s*\)\s*\(")
SWIZZLE = re.compile(r"\.([xyzw]{2,4}|[rgba]{2,4})\b")


def rewrite_opencl(text: str) -> str:
    """The two OpenCL C constructs C++ cannot parse, rewritten; everything else is left as is."""
    text = VEC_LITERAL.sub(lambda m: f"{m.group(1)}_ctor(", text)
    text = re.sub(r"\.yx\b", ".yx_()", text)
    code = "\n".join(l for l in text.splitlines() if not l.startswith("#"))
    left = re.search(r"\(\s*float[234]\s*\)", code)
    if left:
        raise RuntimeError(f"unhandled vector literal or cast: {code[left.start() - 60:left.end() + 60]!r}")
    bad = sorted({m.group(1) for m in SWIZZLE.finditer(code)} - {"xy", "xyz"})
    if bad:
        raise RuntimeError(f"unhandled swizzles: {bad}")
    return text


def extract_function(src: str, signature: str) -> str:
    """The definition that starts at the first match of `signature` (a regex), through its
    matching closing brace."""
    m = re.search(signature, src)
    if not m:
        raise RuntimeError(f"not found: {signature}")
    i = src.index("{", m.end() - 1)
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[m.start():j + 1]
    raise RuntimeError(f"unbalanced braces after {signature}")


def extract_block(src: str, first: str, last: str) -> str:
    """The lines from the one containing `first` through the one containing `last`."""
    a = src.index(first)
    a = src.rfind("\n", 0, a) + 1
    b = src.index(last, a)
    b = src.index("\n", b)
    return src[a:b + 1]


def host_extract(ref: Path) -> str:
    out_cpp = (ref / "src" / "renderer" / "output.cpp").read_text()
    shading = (ref / "src" / "buffers" / "shading.cpp").read_text()
    scene_data = (ref / "src" / "renderer" / "scene_data.cpp").read_text()
    tone_map = extract_function(out_cpp, r"static inline f32 tone_map\(")
    apply_tonemap = extract_function(out_cpp, r"static std::vector<u8> apply_tonemap\(")
    sphere = extract_block(shading, "vec3 bbox_min(scene_bbox.min.x", "this->scene_radius = radius;")
    lum = extract_function(scene_data, r"void SceneData::build_lum_pref_sum\(\)")
    lum_body = lum[lum.index("{"):]
    return "\n".join([
        "// generated by oracle/build_ref_sppm.py from the reference's src/renderer/output.cpp,",
        "// src/buffers/shading.cpp and src/renderer/scene_data.cpp (functions read out verbatim)",
        "#pragma once",
        tone_map,
        apply_tonemap,
        "struct RefShadingSphere {",
        "    float4 scene_center{};",
        "    f32 scene_radius = 0.0f;",
        "    void compute(const BoundingBox &scene_bbox) {",
        sphere,
        "    }",
        "};",
        "struct RefSceneLum {",
        "    std::vector<Light> lights;",
        "    std::vector<f32> lum_pref_sum;",
        "    void build_lum_pref_sum() " + lum_body,
        "};",
        "",
    ])


def build(reference: Path | str | None = None, verbose: bool = False) -> Path:
    from oracle.build_ref_filters import reference_dir
    ref = reference_dir(reference)
    if ref is None or not (ref / "kernels" / "trace_rays.cl").is_file():
        raise RuntimeError("no reference checkout given (argument or PHX_REFERENCE_DIR)")
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    (OUT_DIR / "sppm_kernels.inc").write_text(rewrite_opencl(preprocess_kernels(ref)))
    (OUT_DIR / "host_extract.inc").write_text(host_extract(ref))
    objs = []
    host_inc = ["-I", str(SHIM), "-I", str(ref / "include"), "-I", str(OUT_DIR)]
    units = [
        (HERE / "ref_kernels.cpp", ["-I", str(OUT_DIR), "-I", str(ROOT / "include")]),
        (HERE / "ref_host.cpp", host_inc),
        (ref / "src" / "renderer" / "bvh.cpp", host_inc),
        (ref / "src" / "renderer" / "camera.cpp", host_inc),
        (ref / "src" / "renderer" / "light.cpp", host_inc),
    ]
    for src, inc in units:
        obj = OUT_DIR / (src.stem + ".o")
        _run([*CXX, *inc, "-c", str(src), "-o", str(obj)])
        objs.append(str(obj))
    tmp = OUT.with_suffix(".so.tmp")
    _run([*CXX, "-shared", "-o", str(tmp), *objs, "-lpthread"])
    tmp.replace(OUT)
    if verbose:
        print(f"built {OUT}")
    return OUT


if __name__ == "__main__":
    sys.path.insert(0, str(ROOT))
    build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
