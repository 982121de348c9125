"""The reference denoiser's filters (denoise/filters_gpu.py) on the GPU, against the reference's own
kernels (fixtures made by tests/golden/make_denoise_golden.py from the reference's OpenCL kernel
source compiled for the CPU) and against oracle/filters.py, the numpy restatement pinned to them.
Every comparison is bit-exact: the kernels sum integers converted to float in a fixed order."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest

from oracle import filters as F
from phosphor_b200 import _capi as A
from phosphor_b200 import denoise as D

GOLDEN = Path(__file__).resolve().parent / "golden" / "denoise_golden.npz"
NAMES = {0: "mean", 1: "median", 2: "weighted"}


def golden_cases():
    g = np.load(GOLDEN)
    for i in range(int(g["n"][0])):
        which, k, sd = (int(v) for v in g[f"c{i}_meta"])
        yield NAMES[which], k, sd, g[f"c{i}_img"], g[f"c{i}_weights"], g[f"c{i}_out"]


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def oracle(name, img, k, weights):
    if name == "mean":
        return F.mean_filter(img, k)
    if name == "median":
        return F.median_filter(img, k)
    return F.weighted_filter(img, weights, k)


def test_oracle_matches_the_reference_kernels():
    n = 0
    for name, k, sd, img, wt, out in golden_cases():
        assert np.array_equal(bits(oracle(name, img, k, wt)), bits(out)), (name, k, sd, img.shape)
        n += 1
    assert n == 36


def test_gaussian_weights_are_the_reference_host_weights():
    for name, k, sd, img, wt, out in golden_cases():
        if name == "weighted":
            assert np.array_equal(bits(D.gaussian_weights(k, sd)), bits(wt))
            assert np.array_equal(bits(F.gaussian_weights(k, sd)), bits(wt))


def test_argument_errors_before_the_device():
    with pytest.raises(ValueError):
        D.mean_filter_gpu(np.zeros((4, 4), np.int32))
    with pytest.raises(ValueError):
        D.median_filter_gpu(np.zeros((4, 4, 3), np.int32), k=3)  # filters_gpu.py:138-139


@pytest.mark.gpu
def test_filters_match_the_reference_kernels():
    for name, k, sd, img, wt, out in golden_cases():
        if name == "mean":
            got = D.mean_filter_gpu(img, k)
        elif name == "median":
            got = D.median_filter_gpu(img, k)
        else:
            got = D.gaussian_filter_gpu(img, k, sd)
        assert got.dtype == np.float64 and got.shape == img.shape
        assert np.array_equal(bits(got), bits(out)), (name, k, sd, img.shape)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1, 1), (1, 40), (33, 1), (131, 257), (64, 96)])
def test_filters_match_the_oracle(shape):
    """Sizes that are not multiples of the 32 x 8 blocks, single rows and columns; windows up to
    k = 12 (k > 8 reads the image without the shared-memory tile); values beyond 8 bits."""
    rng = np.random.default_rng(sum(shape))
    img = rng.integers(-300, 70000, size=shape + (3,)).astype(np.int32)
    for k in (0, 1, 2, 3, 9):
        assert np.array_equal(bits(D.mean_filter_gpu(img, k)), bits(F.mean_filter(img, k))), ("mean", k)
    for k in (0, 1, 2):
        assert np.array_equal(bits(D.median_filter_gpu(img, k)), bits(F.median_filter(img, k))), ("median", k)
    for k, sd in ((1, 1), (2, 2), (4, 3), (12, 5)):
        wt = D.gaussian_weights(k, sd)
        assert np.array_equal(bits(D.gaussian_filter_gpu(img, k, sd)), bits(F.weighted_filter(img, wt, k))), k


@pytest.mark.gpu
def test_filter_status_codes():
    lib = A.load()
    img = np.zeros((8, 8, 3), np.int32)
    out = np.zeros((8, 8, 3), np.float32)
    vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    assert lib.phx_median_filter(vp(img), vp(out), 8, 8, 3, None) == A.PHX_E_INVALID
    assert lib.phx_mean_filter(vp(img), vp(out), 8, 8, 33, None) == A.PHX_E_INVALID
    assert lib.phx_mean_filter(None, vp(out), 8, 8, 1, None) == A.PHX_E_INVALID
    assert lib.phx_mean_filter(vp(img), vp(out), 0, 8, 1, None) == A.PHX_E_INVALID
    assert lib.phx_weighted_filter(vp(img), vp(out), None, 8, 8, 1, None) == A.PHX_E_INVALID
    ms = C.c_float(-1.0)
    assert lib.phx_mean_filter(vp(img), vp(out), 8, 8, 1, C.byref(ms)) == A.PHX_OK
    assert ms.value >= 0.0
