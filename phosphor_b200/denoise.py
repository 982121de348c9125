"""The reference denoiser's GPU filters (denoise/filters_gpu.py) on the sm_100a kernels of libphx.so.

Same names, arguments, results and errors as filters_gpu.py, so denoise.py's menu entries
(Mean3/5, Median3/5, Gaussian3_1 ... 5_2) run unchanged against this module:

* mean_filter_gpu(arr, k=1), median_filter_gpu(arr, k=1), gaussian_filter_gpu(arr, k=1, sd=1):
  arr is an (H, W, 3) array, taken as int32 like filters_gpu.py:_run_kernel; the result is an
  (H, W, 3) float64 array of the kernel's float32 values (filters_gpu.py:128);
* ValueError for an array that is not (H, W, 3) and for a median with k > 2 (filters_gpu.py:116-117,
  138-139); other failures raise phosphor_b200's PhxError.

Windows are clamped to the image (border windows shrink), as in the reference's OpenCL kernels;
its CPU filters (filters_cpu.py) pad with edge pixels instead and differ at the borders.
`last_kernel_ms()` returns the CUDA-event time of the most recent filter kernel.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi as A

_last_ms = [0.0]


def last_kernel_ms() -> float:
    return _last_ms[0]


def _run(fn: str, arr, k: int, weights: np.ndarray | None = None) -> np.ndarray:
    a = np.asarray(arr)
    if a.ndim != 3 or a.shape[2] != 3:
        raise ValueError("expected an (H, W, 3) array")
    h, w, _ = a.shape
    src = np.ascontiguousarray(a.astype(np.int32))
    out = np.empty((h, w, 3), dtype=np.float32)
    ms = C.c_float(0.0)
    lib = A.load()
    if weights is None:
        rc = getattr(lib, fn)(src.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), w, h, int(k),
                              C.byref(ms))
    else:
        wt = np.ascontiguousarray(weights, np.float32)
        rc = getattr(lib, fn)(src.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p),
                              wt.ctypes.data_as(C.c_void_p), w, h, int(k), C.byref(ms))
    A.check(rc)
    _last_ms[0] = ms.value
    return out.astype(np.float64)


def mean_filter_gpu(arr, k=1):
    """filters_gpu.py:131-133 (kernel :9-27): the mean of each pixel's clamped window."""
    return _run("phx_mean_filter", arr, k)


def median_filter_gpu(arr, k=1):
    """filters_gpu.py:136-141 (kernel :29-67): the median of each pixel's clamped window, k <= 2."""
    if k > 2:
        raise ValueError("median filter k is > 3")
    return _run("phx_median_filter", arr, k)


def gaussian(x, y, sd):
    """filters_gpu.py:142-143."""
    return 1 / np.sqrt(2 * np.pi) / sd * np.exp(-(x ** 2 + y ** 2) / (2 * sd ** 2))


def gaussian_weights(k: int = 1, sd: float = 1) -> np.ndarray:
    """filters_gpu.py:148-154: the (2k+1)^2 Gaussian weights, float64 values stored as float32,
    normalised by their float32 sum, flattened row-major (row = dy + k, column = dx + k)."""
    size = 2 * k + 1
    weights = np.zeros((size, size), dtype=np.float32)
    for dy in range(-k, k + 1):
        for dx in range(-k, k + 1):
            weights[dy + k, dx + k] = gaussian(dx, dy, sd)
    weights /= weights.sum()
    return np.ascontiguousarray(weights.flatten())


def gaussian_filter_gpu(arr, k=1, sd=1):
    """filters_gpu.py:146-161 (kernel :69-86): the Gaussian-weighted sum of each clamped window
    (the weights are not renormalised where a border window shrinks, as in the reference)."""
    return _run("phx_weighted_filter", arr, k, gaussian_weights(k, sd))


def bench(width: int = 1920, height: int = 1080, reps: int = 5) -> list[dict]:
    """Kernel time and effective bandwidth of every filter of the reference's menu on a seeded
    8-bit image (the compulsory traffic of one filter: the int32 image in, the float32 image out)."""
    rng = np.random.default_rng(1)
    img = rng.integers(0, 256, size=(height, width, 3)).astype(np.int32)
    rows = []
    for name, fn, kw in [("Mean3", mean_filter_gpu, {"k": 1}), ("Mean5", mean_filter_gpu, {"k": 2}),
                         ("Median3", median_filter_gpu, {"k": 1}), ("Median5", median_filter_gpu, {"k": 2}),
                         ("Gaussian3_1", gaussian_filter_gpu, {"k": 1, "sd": 1}),
                         ("Gaussian5_2", gaussian_filter_gpu, {"k": 2, "sd": 2})]:
        times = []
        for _ in range(reps + 1):
            fn(img, **kw)
            times.append(last_kernel_ms())
        ms = min(times[1:])
        nbytes = img.size * 4 * 2
        rows.append({"filter": name, "kernel_ms": round(ms, 4), "gbs": round(nbytes / (ms * 1e-3) / 1e9, 1)})
    return rows


if __name__ == "__main__":
    import json
    import sys

    w, h = (int(sys.argv[1]), int(sys.argv[2])) if len(sys.argv) > 2 else (1920, 1080)
    for row in bench(w, h):
        print(json.dumps(row))
