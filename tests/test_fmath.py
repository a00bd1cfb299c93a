"""Accuracy of the shared inverse-trigonometric functions (csrc/gq_fmath.h) used by
the SNCH cone test on the GPU and in the oracle: within a few ulp of the exact value."""
import ctypes as C

import numpy as np

import oracle


def _call(which, x, y=None):
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(np.zeros_like(x) if y is None else y, np.float32)
    out = np.empty_like(x)
    fn = oracle.lib().orc_fmath
    fn.restype = None
    fn(C.c_int(which), C.c_void_p(x.ctypes.data), C.c_void_p(y.ctypes.data), C.c_void_p(out.ctypes.data),
       C.c_int64(x.size))
    return out


def _ulp_err(got, exact):
    exact32 = exact.astype(np.float32)
    ulp = np.spacing(np.abs(exact32)).astype(np.float64)
    return np.abs(got.astype(np.float64) - exact) / ulp


def test_acos_asin_accuracy():
    x = np.linspace(-1.0, 1.0, 400001, dtype=np.float32)
    x = np.concatenate([x, np.float32([-1, -0.5, 0, 0.5, 1, 1e-8, -1e-8])])
    assert _ulp_err(_call(0, x), np.arccos(x.astype(np.float64))).max() <= 4
    assert _ulp_err(_call(1, x), np.arcsin(x.astype(np.float64))).max() <= 4
    assert np.isnan(_call(0, np.float32([1.5, np.nan]))).all()


def test_atan2_accuracy_all_quadrants():
    rng = np.random.default_rng(0)
    y = rng.uniform(-10, 10, 200000).astype(np.float32)
    x = rng.uniform(-10, 10, 200000).astype(np.float32)
    assert _ulp_err(_call(2, y, x), np.arctan2(y.astype(np.float64), x.astype(np.float64))).max() <= 4
    # the SNCH use: atan2(d >= 0, s >= 0), including s = 0
    d = np.float32([0, 1, 1, 0.5])
    s = np.float32([1, 0, 1, 2])
    ref = np.arctan2(d.astype(np.float64), s.astype(np.float64))
    assert _ulp_err(_call(2, d, s), ref).max() <= 4
