"""Crash-pulse signal processing (crush_cfc_filter, crush_resample) against
the oracle's restatement of src/signal.rs and the reference's own tests
(src/signal.rs:310-345), restated. CPU only."""
import numpy as np

from crushrs_b200 import abi, pulse as G
from crushrs_b200.native import lib

from . import oracle_lib as O


def test_cfc_matches_oracle_bitwise():
    rng = np.random.default_rng(7)
    for n in (0, 1, 3, 4, 5, 17, 400, 5000):
        x = rng.normal(size=n) * 50.0 + 3.0
        for dt, cfc in ((1e-4, 60.0), (1e-5, 180.0), (2e-3, 60.0), (1e-6, 1000.0)):
            y = G.cfc_filter(x, dt, cfc)
            assert np.array_equal(y, O.cfc_filter(x, dt, cfc)), (n, dt, cfc)


def test_cfc60_passes_dc_and_kills_1khz():
    """src/signal.rs:311-324: DC passes, 1 kHz ripple removed, -3 dB near 100 Hz."""
    dt = 1e-4
    t = np.arange(5000) * dt
    x = 10.0 + 5.0 * np.sin(2 * np.pi * 1000.0 * t)
    y = G.cfc_filter(x, dt, 60.0)
    assert np.abs(y[1000:4000] - 10.0).max() < 0.05
    y100 = G.cfc_filter(np.sin(2 * np.pi * 100.0 * t), dt, 60.0)
    assert abs(np.abs(y100[1000:4000]).max() - 0.707) < 0.05


def test_cfc_short_signal_is_copied_and_bad_input_rejected():
    x = np.array([1.0, -2.0, 3.0])
    assert np.array_equal(G.cfc_filter(x, 1e-4, 60.0), x)
    y = np.zeros(8)
    import ctypes as C

    xp = np.ones(8)
    st = lib().crush_cfc_filter(xp.ctypes.data_as(C.POINTER(C.c_double)), 8, 0.0, 60.0, y.ctypes.data_as(C.POINTER(C.c_double)))
    assert st == abi.CRUSH_ERR_INVALID


def test_resample_is_linear():
    """src/signal.rs:339-345."""
    tu, yu = G.resample([0.0, 1.0, 3.0], [0.0, 2.0, 6.0], 0.0, 0.5, 3.0)
    assert len(tu) == 7
    assert abs(yu[1] - 1.0) < 1e-12 and abs(yu[3] - 3.0) < 1e-12 and abs(yu[6] - 6.0) < 1e-12


def test_resample_matches_oracle_bitwise():
    rng = np.random.default_rng(3)
    t = np.cumsum(rng.uniform(1e-5, 3e-5, size=300))
    y = rng.normal(size=300)
    for t0, dt, te in ((0.0, 1e-5, t[-1]), (t[5], 7e-6, t[-1] + 1e-4), (t[-1], 1e-5, t[0]), (-1e-4, 2e-5, t[40])):
        a = G.resample(t, y, t0, dt, te)
        b = O.resample(t, y, t0, dt, te)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
