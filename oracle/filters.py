"""TEST INFRASTRUCTURE ONLY — numpy restatement of the reference's denoise filter kernels.

The three OpenCL kernels of denoise/filters_gpu.py, one output per pixel and channel of an
(H, W, 3) int32 image, each over the window [clamp(x-k), clamp(x+k)] x [clamp(y-k), clamp(y+k)]
(clamped to the image, so windows shrink at the borders instead of replicating edge pixels):

* mean_filter (filters_gpu.py:9-27): float sum of the window in xx-major, yy-minor order, divided
  by the window's pixel count;
* median_filter (filters_gpu.py:29-67): the window's median; for an even count the mean of the
  two middle values, (a + b) / 2.0f with an integer sum;
* weighted_filter (filters_gpu.py:69-86): float sum of value * weight in the same order, with
  weight[(yy - y + k) * (2k + 1) + (xx - x + k)];

and the host-side Gaussian weights of gaussian_filter_gpu (filters_gpu.py:146-161).  The sums are
float32 additions in the kernels' order (numpy float32 arithmetic rounds every operation), so the
results are the kernels' bits.  Only the tests use this module, as the checker of
phosphor_b200's CUDA filters; it is pinned to the reference's own kernels, compiled for the CPU
by oracle/build_ref_filters.py, through the fixtures in tests/golden/denoise_golden.npz.
"""
from __future__ import annotations

import numpy as np


def _windows(h: int, w: int, k: int):
    """Per offset (dx outer, dy inner: the kernels' xx-major, yy-minor loop order) the source
    coordinates and the mask of pixels whose clamped window holds that offset."""
    ys, xs = np.mgrid[0:h, 0:w]
    for dx in range(-k, k + 1):
        for dy in range(-k, k + 1):
            sx, sy = xs + dx, ys + dy
            ok = (sx >= 0) & (sx < w) & (sy >= 0) & (sy < h)
            yield dx, dy, np.clip(sy, 0, h - 1), np.clip(sx, 0, w - 1), ok


def mean_filter(img: np.ndarray, k: int) -> np.ndarray:
    img = np.asarray(img, np.int32)
    h, w, _ = img.shape
    s = np.zeros((h, w, 3), np.float32)
    n = np.zeros((h, w), np.int32)
    for _, _, sy, sx, ok in _windows(h, w, k):
        v = img[sy, sx].astype(np.float32)
        s = np.where(ok[..., None], s + v, s)
        n += ok
    return s / n.astype(np.float32)[..., None]


def median_filter(img: np.ndarray, k: int) -> np.ndarray:
    img = np.asarray(img, np.int32)
    h, w, _ = img.shape
    big = np.iinfo(np.int32).max
    vals = []
    n = np.zeros((h, w), np.int32)
    for _, _, sy, sx, ok in _windows(h, w, k):
        vals.append(np.where(ok[..., None], img[sy, sx], big))
        n += ok
    win = np.sort(np.stack(vals, axis=-1), axis=-1)  # the window's values first, then padding
    nn = np.broadcast_to(n[..., None], (h, w, 3))
    lo = np.take_along_axis(win, ((nn - 1) // 2)[..., None], axis=-1)[..., 0]
    hi = np.take_along_axis(win, (nn // 2)[..., None], axis=-1)[..., 0]
    even = (nn % 2) == 0
    return np.where(even, (lo + hi).astype(np.float32) / np.float32(2.0), hi.astype(np.float32))


def weighted_filter(img: np.ndarray, weights: np.ndarray, k: int) -> np.ndarray:
    img = np.asarray(img, np.int32)
    wt = np.asarray(weights, np.float32).reshape(2 * k + 1, 2 * k + 1)
    h, w, _ = img.shape
    s = np.zeros((h, w, 3), np.float32)
    for dx, dy, sy, sx, ok in _windows(h, w, k):
        term = img[sy, sx].astype(np.float32) * wt[dy + k, dx + k]
        s = np.where(ok[..., None], s + term, s)
    return s


def gaussian_weights(k: int, sd: float) -> np.ndarray:
    """gaussian_filter_gpu's weights: the Gaussian of filters_gpu.py:142-143 evaluated in float64,
    stored as float32 and normalised by the float32 array's numpy sum."""
    size = 2 * k + 1
    wt = np.zeros((size, size), dtype=np.float32)
    for dy in range(-k, k + 1):
        for dx in range(-k, k + 1):
            wt[dy + k, dx + k] = 1 / np.sqrt(2 * np.pi) / sd * np.exp(-(dx ** 2 + dy ** 2) / (2 * sd ** 2))
    wt /= wt.sum()
    return np.ascontiguousarray(wt.flatten())
