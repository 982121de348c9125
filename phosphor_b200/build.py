"""Builds libphx.so (sm_100a CUDA kernels + C ABI) in-tree, and the CPU oracle used by the tests.

    python -m phosphor_b200.build            # library + oracle
    python -m phosphor_b200.build --force    # rebuild everything

The library is compiled for sm_100a only, with IEEE single-precision semantics (no fused
multiply-add contraction, correctly rounded division and square root, denormals kept) so that the
kernels reproduce the reference's float expression trees bit for bit.  The CUDA runtime is linked
statically, so the library loads on machines without a GPU.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"
LIB = PKG / "libphx.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liboracle.so"

CUDA_HOME = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda"))
NVCC = str(CUDA_HOME / "bin" / "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-Xcompiler", "-ffp-contract=off",
    "-I", str(INCLUDE), "-I", str(CSRC),
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-fvisibility=hidden", "-ffp-contract=off", "-Wall",
             "-Wno-unused-function", "-I", str(INCLUDE), "-I", str(CSRC), "-I", str(CUDA_HOME / "include")]


def _headers_mtime() -> float:
    hs = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(INCLUDE.glob("*.h"))
    return max((h.stat().st_mtime for h in hs), default=0.0)


def _tmp_path(target: Path) -> Path:
    """A file beside `target` private to this process: builds racing in parallel test workers
    each link into their own file and the last rename wins."""
    return target.with_name(f".{target.name}.{os.getpid()}.tmp")


def _compile(src: Path, force: bool, hdr_mtime: float) -> Path:
    obj = BUILD / (src.name + ".o")
    if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_mtime):
        return obj
    tmp = _tmp_path(obj)
    if src.suffix == ".cu":
        cmd = [NVCC, *NVCC_FLAGS, "-c", str(src), "-o", str(tmp)]
    else:
        cmd = ["g++", *CXX_FLAGS, "-c", str(src), "-o", str(tmp)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"compile failed: {src.name}\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, obj)
    return obj


def build_library(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    hm = _headers_mtime()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, hm), srcs))
    newest = max(o.stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        tmp = _tmp_path(LIB)
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs), "-lpthread", "-ldl", "-lrt", "-lz"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    if verbose:
        print(f"built {LIB}")
    return LIB


CLI = PKG / "phx_render"
HOST_DIR = PKG / "host"


def build_cli(force: bool = False, verbose: bool = False) -> Path:
    """phx_render: the reference's command line over libphx.so (C++ host, C ABI only)."""
    srcs = [HOST_DIR / "renderer.cpp", HOST_DIR / "main.cpp"]
    deps = srcs + [HOST_DIR / "renderer.hpp", INCLUDE / "phx.h", LIB]
    if not force and CLI.exists() and CLI.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return CLI
    tmp = _tmp_path(CLI)
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", str(INCLUDE), "-o", str(tmp), *map(str, srcs),
           f"-L{PKG}", "-lphx", "-Wl,-rpath,$ORIGIN", "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"phx_render build failed\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, CLI)
    if verbose:
        print(f"built {CLI}")
    return CLI


def build_oracle(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the CPU oracle (test infrastructure only; see oracle/phx_oracle.hpp)."""
    # the scene generators are host-only C++ shared with the library (synthetic inputs, not the
    # checked algorithm), so CPU-only callers of the oracle never map libphx.so
    srcs = [ORACLE_DIR / "oracle_capi.cpp", CSRC / "scenes.cpp"]
    deps = srcs + [ORACLE_DIR / "phx_oracle.hpp", ORACLE_DIR / "phx_frozen.hpp", INCLUDE / "phx.h",
                   INCLUDE / "phx_math.h", CSRC / "host.hpp"]
    if not force and ORACLE_LIB.exists() and ORACLE_LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return ORACLE_LIB
    tmp = _tmp_path(ORACLE_LIB)
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fvisibility=hidden", "-ffp-contract=off",
           "-I", str(INCLUDE), "-o", str(tmp), *map(str, srcs), "-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, ORACLE_LIB)
    if verbose:
        print(f"built {ORACLE_LIB}")
    return ORACLE_LIB


def ptxas_report() -> str:
    """Registers / spills / shared memory of every kernel (nvcc -Xptxas -v)."""
    out = []
    for src in sorted(CSRC.glob("*.cu")):
        cmd = [NVCC, *NVCC_FLAGS, "-Xptxas", "-v", "-c", str(src), "-o", os.devnull]
        res = subprocess.run(cmd, capture_output=True, text=True)
        out.append(f"== {src.name}\n{res.stderr}")
    return "\n".join(out)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print register/spill report")
    a = ap.parse_args(argv)
    build_library(a.force, verbose=True)
    build_cli(a.force, verbose=True)
    build_oracle(a.force, verbose=True)
    if a.ptxas:
        print(ptxas_report())
    return 0


if __name__ == "__main__":
    sys.exit(main())
