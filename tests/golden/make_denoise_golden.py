"""Makes tests/golden/denoise_golden.npz from the reference's own denoise filter kernels.

oracle/build_ref_filters.py compiles the OpenCL kernels of denoise/filters_gpu.py (read from the
reference checkout) for the host CPU; this script runs them on seeded integer images — odd sizes,
a single pixel, a single column — for every filter and window the reference's denoiser offers
(Mean3/5, Median3/5, Gaussian3_1/3_2/5_1/5_2; denoise.py:60-78) plus a 7x7 mean, and stores inputs,
weights and outputs.  Needs the reference checkout; the fixture it writes is committed.

    python tests/golden/make_denoise_golden.py [path/to/reference]
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import build_ref_filters  # noqa: E402
from oracle.filters import gaussian_weights  # noqa: E402

FILTERS = {"mean": 0, "median": 1, "weighted": 2}


def main(reference: Path) -> None:
    lib = C.CDLL(str(build_ref_filters.build(reference)))
    rng = np.random.default_rng(20260)
    cases = []
    for (h, w) in [(1, 1), (5, 1), (9, 13), (20, 32)]:
        img = rng.integers(0, 256, size=(h, w, 3)).astype(np.int32)
        for name, k, sd in [("mean", 1, 0), ("mean", 2, 0), ("mean", 3, 0), ("median", 1, 0), ("median", 2, 0),
                            ("weighted", 1, 1), ("weighted", 1, 2), ("weighted", 2, 1), ("weighted", 2, 2)]:
            wt = gaussian_weights(k, sd) if name == "weighted" else np.zeros(0, np.float32)
            out = np.zeros((h, w, 3), np.float32)
            lib.ref_filter(FILTERS[name], img.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                           wt.ctypes.data_as(C.c_void_p) if len(wt) else None, w, h, k)
            cases.append((name, k, sd, img, wt, out))
    arrays = {}
    for i, (name, k, sd, img, wt, out) in enumerate(cases):
        arrays[f"c{i}_meta"] = np.array([FILTERS[name], k, sd], np.int32)
        arrays[f"c{i}_img"] = img
        arrays[f"c{i}_weights"] = wt
        arrays[f"c{i}_out"] = out
    arrays["n"] = np.array([len(cases)], np.int32)
    dst = Path(__file__).resolve().parent / "denoise_golden.npz"
    np.savez_compressed(dst, **arrays)
    print(f"wrote {dst} ({len(cases)} cases)")


if __name__ == "__main__":
    from oracle.build_ref_filters import reference_dir
    ref = reference_dir(sys.argv[1] if len(sys.argv) > 1 else None)
    if ref is None:
        sys.exit("usage: make_denoise_golden.py path/to/reference   (or set PHX_REFERENCE_DIR)")
    main(ref)
