"""Accuracy of the portable math in include/phx_math.h against double-precision libm (CPU only).

The kernels and the oracle share these implementations so their results agree bit for bit; here
we check they are accurate implementations of the OpenCL builtins the reference calls
(OpenCL C 3.0 s7.4 allows sin/cos 4 ulp, exp/log 3 ulp, pow 16 ulp).
"""
import math

import numpy as np
import pytest

import oracle as O


def ulp_err(got: float, want: float) -> float:
    g = np.float32(got)
    w = np.float64(want)
    if w == 0.0:
        return 0.0 if g == 0.0 else float("inf")
    ulp = np.spacing(np.float32(abs(w)))
    return abs(float(g) - w) / float(ulp)


def check(fn, xs, ref, limit, y=None):
    worst = 0.0
    for i, x in enumerate(xs):
        xf = float(np.float32(x))
        yf = float(np.float32(y[i])) if y is not None else 0.0
        got = O.math(fn, xf, yf)
        want = ref(xf, yf) if y is not None else ref(xf)
        worst = max(worst, ulp_err(got, want))
    assert worst <= limit, f"{fn}: {worst:.2f} ulp"


def test_sin_cos_render_range():
    xs = np.linspace(0.0, 2 * math.pi, 2001)
    check("sin", xs, math.sin, 4.0)
    check("cos", xs, math.cos, 4.0)


def test_sin_cos_wide_range():
    xs = np.linspace(-200.0, 200.0, 1001)
    check("sin", xs, math.sin, 4.0)
    check("cos", xs, math.cos, 4.0)


def test_exp():
    xs = np.concatenate([np.linspace(-1.0, 0.0, 1001), np.linspace(-80.0, 80.0, 801)])
    check("exp", xs, math.exp, 3.0)


def test_log():
    xs = np.concatenate([np.geomspace(1e-30, 1e30, 801), np.linspace(0.5, 2.0, 801)])
    check("log", xs, math.log, 3.0)


def test_pow():
    xs = np.linspace(0.0, 1.0, 501)[1:]
    check("pow", xs, lambda x, y: x ** y, 16.0, y=np.full(len(xs), 2.2))
    check("pow", xs, lambda x, y: x ** y, 4.0, y=np.full(len(xs), 5.0))
    check("pow", xs, lambda x, y: x ** y, 16.0, y=np.full(len(xs), 1 / 2.2))


def test_acos_atan2():
    xs = np.linspace(-1.0, 1.0, 1001)
    check("acos", xs, math.acos, 4.0)
    ang = np.linspace(-math.pi, math.pi, 1001)
    check("atan2", np.sin(ang), math.atan2, 4.0, y=np.cos(ang))


def test_special_values():
    assert O.math("exp", -200.0) == 0.0
    assert math.isinf(O.math("exp", 100.0))
    assert O.math("pow", 0.3, 0.0) == 1.0
    assert O.math("pow", 0.0, 5.0) == 0.0
    assert math.isnan(O.math("log", -1.0))
    assert O.math("atan2", 0.0, 0.0) == 0.0
