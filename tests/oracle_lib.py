"""ctypes bindings of the oracle (oracle/liboracle.so): the CPU restatement of
the reference used as the checker. Only tests, smoke() and bench.py's CPU
baseline load it."""
import ctypes as C
import os
import subprocess

import numpy as np

from crushrs_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(ORACLE_SO):
        subprocess.run(["make", "-s", "-C", ORACLE_DIR, "CXX=g++"], check=True)
    lib = C.CDLL(ORACLE_SO)
    P = C.POINTER
    dp = P(C.c_double)
    fp = P(C.c_float)
    vp = C.c_void_p
    lib.oracle_last_error.restype = C.c_char_p
    lib.oracle_hardware_threads.restype = C.c_int
    lib.oracle_geometry.argtypes = [dp, C.c_double, C.c_double, C.c_double, C.c_double, dp, dp, dp, dp, dp]
    lib.oracle_char_length.argtypes = [dp, dp, dp]
    lib.oracle_honeycomb_update.argtypes = [P(abi.Material), dp, dp, dp, dp]
    lib.oracle_honeycomb_params.argtypes = [P(abi.Material), dp]
    lib.oracle_yield_at.argtypes = [P(abi.Material), C.c_double, dp, dp, dp, dp]
    lib.oracle_session_new.restype = vp
    lib.oracle_session_new.argtypes = [P(abi.ModelDesc), C.c_int, C.c_int]
    lib.oracle_session_free.argtypes = [vp]
    lib.oracle_session_forces.argtypes = [vp, dp, dp, P(C.c_int64)]
    lib.oracle_session_stable_dt.argtypes = [vp, dp, dp]
    lib.oracle_session_element_dts.argtypes = [vp, dp, dp]
    lib.oracle_session_mass_scaling.argtypes = [vp, dp, C.c_double, dp, dp, dp]
    lib.oracle_session_masses.argtypes = [vp, dp, dp]
    lib.oracle_session_geometry.argtypes = [vp, dp, dp, dp, dp]
    lib.oracle_session_set_lane_geometry.argtypes = [vp, fp, fp, fp, fp]
    lib.oracle_session_get_state.argtypes = [vp, fp, P(C.c_uint8)]
    lib.oracle_session_set_state.argtypes = [vp, fp, P(C.c_uint8)]
    lib.oracle_session_contact_apply.argtypes = [vp, C.c_int, dp, dp, dp, C.c_double, dp, P(C.c_int64), dp]
    lib.oracle_session_contact_nodes.argtypes = [vp, C.c_int, P(C.c_uint32), P(C.c_int64)]
    lib.oracle_run.argtypes = [P(abi.ModelDesc), C.c_int, C.c_int, P(abi.Results), dp, dp, dp, C.c_int64, dp]
    lib.oracle_run_window.argtypes = [P(abi.ModelDesc), C.c_int, C.c_int, C.c_int64, P(abi.Results), dp, dp, P(C.c_uint8), dp]
    lib.oracle_run_history.argtypes = [P(abi.ModelDesc), C.c_int, C.c_int, C.c_int, C.c_int, P(abi.Accelerometer), C.c_int64, dp,
                                       P(C.c_int64), dp, dp, P(C.c_int64), P(abi.Results)]
    lib.oracle_run_frames.argtypes = [P(abi.ModelDesc), C.c_int, C.c_int, C.c_int, C.c_int64, dp, P(C.c_int64), fp, fp, fp,
                                      P(C.c_uint8), P(C.c_int64)]
    lib.oracle_cfc_filter.argtypes = [dp, C.c_int64, C.c_double, C.c_double, dp]
    lib.oracle_resample.argtypes = [dp, dp, C.c_int64, C.c_double, C.c_double, C.c_double, dp, dp, C.c_int64]
    lib.oracle_resample.restype = C.c_int64
    lib.oracle_symmetric_eigen3.argtypes = [dp, dp, dp]
    lib.oracle_hencky_elastic.argtypes = [C.c_double, C.c_double, dp, dp]
    _lib = lib
    return lib


def ptr(a, ctype=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


def error():
    return load().oracle_last_error().decode()


def geometry(x, youngs, poisson, density, hourglass=0.1):
    lib = load()
    x = np.ascontiguousarray(x, np.float64).reshape(24)
    grad, vol, lumped, gamma, h = np.zeros(24), np.zeros(1), np.zeros(8), np.zeros(32), np.zeros(144)
    st = lib.oracle_geometry(ptr(x), youngs, poisson, density, hourglass, ptr(grad), ptr(vol), ptr(lumped), ptr(gamma), ptr(h))
    assert st == 0, error()
    return dict(grad=grad.reshape(8, 3), volume=vol[0], lumped=lumped, gamma=gamma.reshape(8, 4), h=h.reshape(12, 12))


def char_length(p):
    lib = load()
    p = np.ascontiguousarray(p, np.float64).reshape(24)
    l, v = C.c_double(), C.c_double()
    lib.oracle_char_length(ptr(p), C.byref(l), C.byref(v))
    return l.value, v.value


def default_state():
    s = np.zeros(25)
    s[[0, 4, 8]] = 1.0
    s[[9, 13, 17]] = 1.0
    return s


def honeycomb_update(mat, f, state):
    lib = load()
    f = np.ascontiguousarray(f, np.float64).reshape(9)
    state = np.ascontiguousarray(state, np.float64)
    tau, out = np.zeros(9), np.zeros(25)
    st = lib.oracle_honeycomb_update(C.byref(mat), ptr(f), ptr(state), ptr(tau), ptr(out))
    assert st == 0, error()
    return tau.reshape(3, 3), out


def yield_at(mat, c):
    lib = load()
    a, b, c2, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
    st = lib.oracle_yield_at(C.byref(mat), c, C.byref(a), C.byref(b), C.byref(c2), C.byref(d))
    assert st == 0, error()
    return (a.value, b.value), (c2.value, d.value)


class Session:
    """Elements + contact runtimes of one model (the drop-in calls)."""

    def __init__(self, desc, simd=True, threads=1):
        self.lib = load()
        self.desc = desc
        self.h = self.lib.oracle_session_new(C.byref(desc), int(simd), threads)
        assert self.h, error()
        self.n_nodes = desc.n_nodes
        self.n_hexes = desc.n_hexes

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.oracle_session_free(self.h)
            self.h = None

    def forces(self, u, out=None):
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        f = np.zeros(3 * self.n_nodes) if out is None else out
        n = C.c_int64()
        self.lib.oracle_session_forces(self.h, ptr(u), ptr(f), C.byref(n))
        return f, n.value

    def stable_dt(self, u):
        dt = C.c_double()
        st = self.lib.oracle_session_stable_dt(self.h, ptr(np.ascontiguousarray(u, np.float64)), C.byref(dt))
        return (dt.value if st == 0 else None)

    def element_dts(self, u):
        out = np.zeros(self.n_hexes)
        self.lib.oracle_session_element_dts(self.h, ptr(np.ascontiguousarray(u, np.float64)), ptr(out))
        return out

    def mass_scaling(self, u, dt_min, element_mass=None):
        added = np.zeros(self.n_nodes)
        total = C.c_double()
        self.lib.oracle_session_mass_scaling(self.h, ptr(np.ascontiguousarray(u, np.float64)), dt_min, ptr(element_mass), ptr(added), C.byref(total))
        return added, total.value

    def masses(self):
        lumped, em = np.zeros(self.n_nodes), np.zeros(self.n_hexes)
        self.lib.oracle_session_masses(self.h, ptr(lumped), ptr(em))
        return lumped, em

    def geometry(self):
        g, v, gm, hh = np.zeros((self.n_hexes, 24)), np.zeros(self.n_hexes), np.zeros((self.n_hexes, 32)), np.zeros((self.n_hexes, 144))
        self.lib.oracle_session_geometry(self.h, ptr(g), ptr(v), ptr(gm), ptr(hh))
        return g, v, gm, hh

    def set_lane_geometry(self, grad, volume, gamma, h):
        arrs = [np.ascontiguousarray(a, np.float32) for a in (grad, volume, gamma, h)]
        self.lib.oracle_session_set_lane_geometry(self.h, *[ptr(a, C.c_float) for a in arrs])

    def get_state(self):
        s, e = np.zeros((self.n_hexes, 25), np.float32), np.zeros(self.n_hexes, np.uint8)
        self.lib.oracle_session_get_state(self.h, ptr(s, C.c_float), ptr(e, C.c_uint8))
        return s, e

    def set_state(self, s, e):
        s = np.ascontiguousarray(s, np.float32)
        e = np.ascontiguousarray(e, np.uint8)
        self.lib.oracle_session_set_state(self.h, ptr(s, C.c_float), ptr(e, C.c_uint8))

    def contact_apply(self, c, u, v, masses, dt, force=None):
        f = np.zeros(3 * self.n_nodes) if force is None else force
        cnt, mp = C.c_int64(), C.c_double()
        st = self.lib.oracle_session_contact_apply(self.h, c, ptr(np.ascontiguousarray(u, np.float64)), ptr(v), ptr(masses), dt, ptr(f), C.byref(cnt), C.byref(mp))
        assert st == 0, error()
        return f, cnt.value, mp.value


def run(desc, simd=True, threads=1, want_state=False, want_dt=0):
    lib = load()
    r = abi.Results()
    n = desc.n_nodes
    u = np.zeros(3 * n) if want_state else None
    v = np.zeros(3 * n) if want_state else None
    dt = np.zeros(want_dt) if want_dt else None
    sec = np.zeros(4)  # wall, forces, contact, step loop (s)
    st = lib.oracle_run(C.byref(desc), int(simd), threads, C.byref(r), ptr(u), ptr(v), ptr(dt), want_dt, ptr(sec))
    assert st in (0, abi.CRUSH_ERR_NONFINITE), error()
    return r, u, v, dt, sec


def run_window(desc, time_from_step=0, simd=True, threads=1, want_state=False):
    """Whole run with the loop time of the steps from `time_from_step` on.
    Returns results, u, v, eroded flags (None unless want_state) and
    seconds (wall, forces, contact, step loop, window)."""
    lib = load()
    r = abi.Results()
    n, e = desc.n_nodes, desc.n_hexes
    u = np.zeros(3 * n) if want_state else None
    v = np.zeros(3 * n) if want_state else None
    er = np.zeros(e, np.uint8) if want_state else None
    sec = np.zeros(5)
    st = lib.oracle_run_window(C.byref(desc), int(simd), threads, int(time_from_step), C.byref(r), ptr(u), ptr(v),
                               None if er is None else er.ctypes.data_as(C.POINTER(C.c_uint8)), ptr(sec))
    assert st in (0, abi.CRUSH_ERR_NONFINITE), error()
    return r, u, v, er, sec


def run_history(desc, steps, accelerometers=(), cap=100000, simd=True, threads=1):
    """Whole run with time histories: dict time (R), step (R), parts (R, P, 11),
    nodes (R, J, 21), records, results. accelerometers: (nodes, frame|None)."""
    lib = load()
    arr = (abi.Accelerometer * max(len(accelerometers), 1))()
    keep = []
    n_nodes = 0
    for k, (nodes, frame) in enumerate(accelerometers):
        nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
        keep.append(nodes)
        n_nodes += len(nodes)
        arr[k].n_nodes = len(nodes)
        arr[k].nodes = nodes.ctypes.data_as(C.POINTER(C.c_uint32))
        arr[k].has_frame = 0 if frame is None else 1
        if frame is not None:
            arr[k].origin, arr[k].x_axis, arr[k].plane = (int(x) for x in frame)
    n_parts = desc.n_parts
    t = np.zeros(cap)
    st = (C.c_int64 * cap)()
    parts = np.zeros(cap * n_parts * 11)
    nodes = np.zeros(max(cap * n_nodes * 21, 1))
    nr = C.c_int64()
    r = abi.Results()
    status = lib.oracle_run_history(C.byref(desc), int(simd), threads, steps, len(accelerometers), arr, cap, ptr(t), st, ptr(parts),
                                    ptr(nodes), C.byref(nr), C.byref(r))
    assert status in (0, abi.CRUSH_ERR_NONFINITE), error()
    k = min(nr.value, cap)
    return {"records": nr.value, "time": t[:k], "step": np.array(st[:k], dtype=np.int64),
            "parts": parts[: k * n_parts * 11].reshape(k, n_parts, 11), "nodes": nodes[: k * n_nodes * 21].reshape(k, n_nodes, 21),
            "results": r}


def symmetric_eigen3(a):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(9)
    ev, vec = np.zeros(3), np.zeros(9)
    load().oracle_symmetric_eigen3(ptr(a), ptr(ev), ptr(vec))
    return ev, vec.reshape(3, 3)


def hencky_elastic(youngs, poisson, f):
    f = np.ascontiguousarray(f, dtype=np.float64).reshape(9)
    tau = np.zeros(9)
    load().oracle_hencky_elastic(C.c_double(youngs), C.c_double(poisson), ptr(f), ptr(tau))
    return tau.reshape(3, 3)


def cfc_filter(x, dt, cfc):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.empty_like(x)
    load().oracle_cfc_filter(ptr(x), len(x), dt, cfc, ptr(y))
    return y


def resample(t, y, t0, dt, t_end):
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    n = load().oracle_resample(ptr(t), ptr(y), len(t), t0, dt, t_end, None, None, 0)
    tu, yu = np.empty(n), np.empty(n)
    load().oracle_resample(ptr(t), ptr(y), len(t), t0, dt, t_end, ptr(tu), ptr(yu), n)
    return tu, yu


def run_frames(desc, steps, cap=64, simd=True, threads=1):
    """Whole run with frames: dict time, step, displacement (F, N, 3),
    plastic_strain (F, E), stress (F, E, 6), eroded (F, E), frames."""
    lib = load()
    n, e = desc.n_nodes, desc.n_hexes
    t = np.zeros(cap)
    st = (C.c_int64 * cap)()
    d = np.zeros(cap * 3 * n, np.float32)
    ps = np.zeros(cap * e, np.float32)
    sg = np.zeros(cap * 6 * e, np.float32)
    er = np.zeros(cap * e, np.uint8)
    nf = C.c_int64()
    fpp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    status = lib.oracle_run_frames(C.byref(desc), int(simd), threads, steps, cap, ptr(t), st, fpp(d), fpp(ps), fpp(sg),
                                   er.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(nf))
    assert status in (0, abi.CRUSH_ERR_NONFINITE), error()
    k = min(nf.value, cap)
    return {"frames": nf.value, "time": t[:k], "step": np.array(st[:k], dtype=np.int64), "displacement": d[: k * 3 * n].reshape(k, n, 3),
            "plastic_strain": ps[: k * e].reshape(k, e), "stress": sg[: k * 6 * e].reshape(k, e, 6), "eroded": er[: k * e].reshape(k, e)}
