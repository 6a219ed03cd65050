"""Crash-pulse signal processing (include/crush.h crush_cfc_filter,
crush_resample): the SAE J211 channel-frequency-class filter and linear
resampling of src/signal.rs, for accelerometer histories."""
import ctypes as C

import numpy as np

from .native import check, lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def cfc_filter(x, dt, cfc=60.0):
    """Phaseless 2-pole Butterworth (forward and backward), CFC `cfc`."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    check(lib().crush_cfc_filter(_dp(x), len(x), dt, cfc, _dp(y)))
    return y


def resample(t, y, t0, dt, t_end):
    """(t, y) linearly onto t0 + k dt, k = 0 .. floor((t_end - t0) / dt)."""
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = C.c_int64()
    check(lib().crush_resample(_dp(t), _dp(y), len(t), t0, dt, t_end, None, None, 0, C.byref(n)))
    tu, yu = np.empty(n.value), np.empty(n.value)
    check(lib().crush_resample(_dp(t), _dp(y), len(t), t0, dt, t_end, _dp(tu), _dp(yu), n.value, C.byref(n)))
    return tu, yu
