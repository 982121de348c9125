"""TEST INFRASTRUCTURE ONLY — builds the reference's own denoise filter kernels for the host CPU.

denoise/filters_gpu.py keeps its three OpenCL C kernels (mean_filter, median_filter,
weighted_filter; filters_gpu.py:8-86) in the string _KERNEL_SOURCE and runs them through pyopencl,
which is absent here.  The kernels only use int/float arithmetic, loops, `clamp` and
`get_global_id`, so this recipe reads that string out of the reference file where it lies (the
Python file is parsed, not executed), puts a C prelude in front of it that supplies those two
builtins and the address-space qualifiers, and a driver that runs each kernel once per pixel the
way an NDRange of (width, height) work items would.  gcc compiles it without contraction
(-ffp-contract=off), so every float operation is the one written.  The output goes to
oracle/_ref/ only (git-ignored); nothing from the reference enters the repository.

    python oracle/build_ref_filters.py path/to/reference     (or PHX_REFERENCE_DIR=path/to/reference)

tests/golden/make_denoise_golden.py runs the result to make the committed fixtures.
"""
from __future__ import annotations

import ast
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref" / "libfilters_ref.so"

PRELUDE = r"""
#include <stdint.h>
static int phx_gid[2];
static int get_global_id(int d) { return phx_gid[d]; }
static int clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
#define __kernel static
#define __global
"""

DRIVER = r"""
/* one work item per pixel, x fastest: the NDRange (width, height) of filters_gpu.py:_run_kernel */
int ref_filter(int which, const int *input, float *output, const float *weights, int width, int height, int k) {
    for (int y = 0; y < height; y++)
        for (int x = 0; x < width; x++) {
            phx_gid[0] = x;
            phx_gid[1] = y;
            if (which == 0)
                mean_filter(input, output, width, height, k);
            else if (which == 1)
                median_filter(input, output, width, height, k);
            else
                weighted_filter(input, output, weights, width, height, k);
        }
    return 0;
}
"""


def kernel_source(reference: Path) -> str:
    """The _KERNEL_SOURCE string of denoise/filters_gpu.py, read without executing the file."""
    tree = ast.parse((reference / "denoise" / "filters_gpu.py").read_text())
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id == "_KERNEL_SOURCE"
                                                for t in node.targets):
            return ast.literal_eval(node.value)
    raise RuntimeError("_KERNEL_SOURCE not found in denoise/filters_gpu.py")


def reference_dir(arg: str | os.PathLike | None = None) -> Path | None:
    """The reference checkout: the given path, else $PHX_REFERENCE_DIR, else None (no default)."""
    if arg:
        return Path(arg)
    env = os.environ.get("PHX_REFERENCE_DIR")
    return Path(env) if env else None


def reference_present(reference: Path | None = None) -> bool:
    reference = reference_dir(reference)
    return reference is not None and (reference / "denoise" / "filters_gpu.py").is_file()


def build(reference: Path | None = None, verbose: bool = False) -> Path:
    reference = reference_dir(reference)
    if reference is None:
        raise RuntimeError("no reference checkout given (argument or PHX_REFERENCE_DIR)")
    src = PRELUDE + kernel_source(reference) + DRIVER
    OUT.parent.mkdir(parents=True, exist_ok=True)
    cmd = ["gcc", "-O2", "-std=c99", "-fPIC", "-shared", "-ffp-contract=off", "-x", "c", "-o", str(OUT), "-"]
    res = subprocess.run(cmd, input=src, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"reference filter build failed\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(f"built {OUT}")
    return OUT


if __name__ == "__main__":
    build(sys.argv[1] if len(sys.argv) > 1 else None, verbose=True)
