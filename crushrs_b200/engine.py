"""Python face of the engine's C ABI, named after the reference's hot-path
calls (crushrs src/kernel.rs, src/contact.rs, src/solver.rs).

    ctx = Context(model_desc)               # Elements::build + lumped masses + ContactRuntime::new
    n = ctx.compute_forces(u, f_int)        # Elements::compute_forces (adds into f_int)
    ctx.contact_apply(c, u, v, m, dt, f)    # ContactRuntime::apply (adds into f)
    dt = ctx.stable_time_step(u)            # Elements::stable_time_step (None if no limit)
    total = ctx.mass_scaling(u, dt_min, element_mass, added)
    results = ctx.run()                     # crushrs::run

Every call goes to the CUDA library; there is no CPU path.
"""
import ctypes as C

import numpy as np

from . import abi
from .native import CrushError, check, lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One model, or a batch of models (a list of descriptors), resident on
    one GPU (crush_ctx)."""

    def __init__(self, desc, device=0, room=None):
        """desc: one model or a list (a batch). room: a dict of the
        crush_capacity fields (slots, contacts, nodes, hexes, faces,
        primary_nodes) to keep room for models appended later."""
        self._lib = lib()
        h = C.c_void_p()
        if room is not None:
            descs = list(desc) if isinstance(desc, (list, tuple)) else [desc]
            arr = (C.POINTER(abi.ModelDesc) * len(descs))(*[C.pointer(d) for d in descs])
            cap = abi.Capacity(**room)
            check(self._lib.crush_batch_create_reserved(arr, len(descs), device, C.byref(cap), C.byref(h)))
        elif isinstance(desc, (list, tuple)):
            arr = (C.POINTER(abi.ModelDesc) * len(desc))(*[C.pointer(d) for d in desc])
            check(self._lib.crush_batch_create(arr, len(desc), device, C.byref(h)))
        else:
            check(self._lib.crush_create(C.byref(desc), device, C.byref(h)))
        self.h = h
        self.n_slots = self._lib.crush_batch_size(self.h)
        nn, ne, na = C.c_int64(), C.c_int64(), C.c_int64()
        check(self._lib.crush_sizes(self.h, C.byref(nn), C.byref(ne), C.byref(na)))
        self.n_nodes, self.n_hexes, self.n_active = nn.value, ne.value, na.value

    def close(self):
        if getattr(self, "h", None):
            self._lib.crush_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- drop-in calls ----
    def compute_forces(self, u, global_forces):
        """Element forces at u, added into global_forces (3N f64); returns the newly eroded count."""
        assert global_forces.dtype == np.float64 and global_forces.flags.c_contiguous
        u = _f64(u)
        n = C.c_int64()
        check(self._lib.crush_compute_forces(self.h, _dp(u), _dp(global_forces), C.byref(n)))
        return n.value

    def compute_forces_device(self, u_ptr, f_ptr, want_count=False):
        """Device-pointer variant (ints are raw CUDA addresses)."""
        n = C.c_int64()
        check(self._lib.crush_compute_forces_device(self.h, C.c_void_p(u_ptr), C.c_void_p(f_ptr), C.byref(n) if want_count else None))
        return n.value

    def contact_apply(self, contact_id, u, v, masses, dt, force):
        assert force.dtype == np.float64 and force.flags.c_contiguous
        cnt, mp = C.c_int64(), C.c_double()
        check(self._lib.crush_contact_apply(self.h, contact_id, _dp(_f64(u)), None if v is None else _dp(_f64(v)),
                                            None if masses is None else _dp(_f64(masses)), dt, _dp(force), C.byref(cnt), C.byref(mp)))
        return cnt.value, mp.value

    def stable_time_step(self, u):
        dt = C.c_double()
        st = check(self._lib.crush_stable_dt(self.h, _dp(_f64(u)), C.byref(dt)), allow=(abi.CRUSH_OK, abi.CRUSH_NONE))
        return dt.value if st == abi.CRUSH_OK else None

    def mass_scaling(self, u, dt_min, element_mass=None, added=None):
        added = np.zeros(self.n_nodes) if added is None else added
        total = C.c_double()
        em = None if element_mass is None else _f64(element_mass)
        check(self._lib.crush_mass_scaling(self.h, _dp(_f64(u)), dt_min, _dp(em), _dp(added), C.byref(total)))
        return total.value, added

    def masses(self):
        lumped, em = np.zeros(self.n_nodes), np.zeros(self.n_hexes)
        check(self._lib.crush_masses(self.h, _dp(lumped), _dp(em)))
        return lumped, em

    def element_data(self):
        n = self.n_active
        g, v, gm, hh = (np.zeros((n, 24), np.float32), np.zeros(n, np.float32), np.zeros((n, 32), np.float32),
                        np.zeros((n, 144), np.float32))
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        check(self._lib.crush_element_data(self.h, fp(g), fp(v), fp(gm), fp(hh)))
        return g, v, gm, hh

    def get_state(self):
        s, e = np.zeros((self.n_active, 25), np.float32), np.zeros(self.n_active, np.uint8)
        check(self._lib.crush_get_state(self.h, s.ctypes.data_as(C.POINTER(C.c_float)), e.ctypes.data_as(C.POINTER(C.c_uint8))))
        return s, e

    def set_state(self, s, e):
        s = np.ascontiguousarray(s, np.float32)
        e = np.ascontiguousarray(e, np.uint8)
        check(self._lib.crush_set_state(self.h, s.ctypes.data_as(C.POINTER(C.c_float)), e.ctypes.data_as(C.POINTER(C.c_uint8))))

    # ---- whole runs ----
    def run(self):
        r = abi.Results()
        st = self._lib.crush_run(self.h, C.byref(r))
        if st not in (abi.CRUSH_OK, abi.CRUSH_ERR_NONFINITE):
            raise CrushError(st, self._lib.crush_last_error().decode())
        return r

    def run_begin(self):
        check(self._lib.crush_run_begin(self.h))

    def run_steps(self, n):
        done = C.c_int()
        check(self._lib.crush_run_steps(self.h, n, C.byref(done)))
        return bool(done.value)

    def set_profiling(self, level):
        """1: time only the element-force kernel inside the step graph; 2: every phase."""
        check(self._lib.crush_set_profiling(self.h, level))

    def run_steps_timed(self, n, phases=False):
        """Advance n steps; returns (done, device ms, phase ms array or None, phase steps)."""
        done, ms = C.c_int(), C.c_double()
        ph = np.zeros(6) if phases else None
        ps = C.c_int()
        check(self._lib.crush_run_steps_timed(self.h, n, C.byref(done), C.byref(ms), _dp(ph), C.byref(ps)))
        return bool(done.value), ms.value, ph, ps.value

    def results(self, slot=0):
        r = abi.Results()
        check(self._lib.crush_batch_results(self.h, slot, C.byref(r)))
        return r

    def batch_run(self):
        """Run every slot to its stop; list of per-slot Results."""
        rs = (abi.Results * self.n_slots)()
        check(self._lib.crush_batch_run(self.h, rs))
        return list(rs)

    def state(self):
        u, v = np.zeros(3 * self.n_nodes), np.zeros(3 * self.n_nodes)
        check(self._lib.crush_run_state(self.h, _dp(u), _dp(v)))
        return u, v

    def launches(self):
        return self._lib.crush_launch_count(self.h)

    def tuning(self):
        """The autotuned launch schedule: (slave lanes, contact ms per lane option 1/2/4/8/16/32)."""
        t = abi.Tuning()
        check(self._lib.crush_get_tuning(self.h, C.byref(t)))
        return t.slave_lanes, list(t.contact_ms)

    def schedule(self):
        """(element-kernel schedule, measured ms per step of each schedule)."""
        t = abi.Tuning()
        check(self._lib.crush_get_tuning(self.h, C.byref(t)))
        return t.forces_schedule, list(t.step_ms)

    def set_tuning(self, slave_lanes, forces_schedule, fused_contact_side=0, early_contact=0):
        """Fix the launch schedule (automatic tuning off)."""
        t = abi.Tuning()
        t.slave_lanes = slave_lanes
        t.forces_schedule = forces_schedule
        t.fused_contact_side = fused_contact_side
        t.early_contact = early_contact
        check(self._lib.crush_set_tuning(self.h, C.byref(t)))

    def fix_schedule(self):
        """Keep the schedule the trial chose (lanes, element-kernel schedule,
        fused or separate steps, early contact) for the rest of the run:
        automatic re-tuning off."""
        t = abi.Tuning()
        check(self._lib.crush_get_tuning(self.h, C.byref(t)))
        self.set_step_fusion(bool(t.step_fusion))
        self.set_tuning(t.slave_lanes, t.forces_schedule, t.fused_contact_side, t.early_contact)

    def autotune(self):
        """Re-tune at the open run's current state; returns tuning()."""
        t = abi.Tuning()
        check(self._lib.crush_autotune(self.h, C.byref(t)))
        return t.slave_lanes, list(t.contact_ms)

    def history_config(self, steps, max_records, accelerometers=(), slot=0):
        """Record slot's part states and accelerometer nodes every `steps`
        steps (include/crush.h crush_history_config). accelerometers: a list
        of (nodes, frame) with frame None or (origin, x_axis, plane)."""
        keep = []
        arr = (abi.Accelerometer * max(len(accelerometers), 1))()
        for k, (nodes, frame) in enumerate(accelerometers):
            nodes = np.ascontiguousarray(nodes, dtype=np.uint32)
            keep.append(nodes)
            a = arr[k]
            a.n_nodes = len(nodes)
            a.nodes = nodes.ctypes.data_as(C.POINTER(C.c_uint32))
            a.has_frame = 0 if frame is None else 1
            if frame is not None:
                a.origin, a.x_axis, a.plane = (int(x) for x in frame)
        check(self._lib.crush_history_config(self.h, slot, steps, max_records, len(accelerometers), arr))
        if not hasattr(self, "_hist_max"):
            self._hist_max = {}
        self._hist_max[slot] = max_records if steps > 0 else 0

    def history(self, slot=0):
        """The kept records: dict of numpy arrays time (R), step (R),
        parts (R, P, 11: mass, velocity 3, displacement 3, acceleration 3,
        kinetic energy) and nodes (R, J, 21: position, displacement,
        velocity, acceleration, local displacement, velocity, acceleration),
        plus the count of records taken."""
        n_rec, n_parts, n_nodes = C.c_int64(), C.c_int(), C.c_int64()
        check(self._lib.crush_history_counts(self.h, slot, C.byref(n_rec), C.byref(n_parts), C.byref(n_nodes)))
        kept = min(n_rec.value, getattr(self, "_hist_max", {}).get(slot, 0))
        t = np.zeros(max(kept, 1))
        st = (C.c_int64 * max(kept, 1))()
        ps = (abi.PartState * max(kept * n_parts.value, 1))()
        ns = (abi.NodeSample * max(kept * n_nodes.value, 1))()
        check(self._lib.crush_history_get(self.h, slot, _dp(t), st, ps, ns))
        parts = np.ctypeslib.as_array(C.cast(ps, C.POINTER(C.c_double)), (max(kept * n_parts.value, 1) * 11,))
        nodes = np.ctypeslib.as_array(C.cast(ns, C.POINTER(C.c_uint8)), (C.sizeof(abi.NodeSample) * max(kept * n_nodes.value, 1),))
        node_vals = nodes.view(np.uint8).reshape(-1, C.sizeof(abi.NodeSample))[:, 8:].copy().view(np.float64)
        return {"records": n_rec.value, "time": t[:kept].copy(), "step": np.array(st[:kept], dtype=np.int64),
                "parts": parts[: kept * n_parts.value * 11].reshape(kept, n_parts.value, 11).copy(),
                "nodes": node_vals[: kept * n_nodes.value].reshape(kept, n_nodes.value, 21),
                "node_ids": np.array([ns[j].node for j in range(n_nodes.value)], dtype=np.uint32) if kept else np.zeros(0, np.uint32)}

    def frames_config(self, steps, max_frames, slot=0):
        """Capture slot's frames every `steps` steps (crush_frames_config)."""
        check(self._lib.crush_frames_config(self.h, slot, steps, max_frames))
        if not hasattr(self, "_frame_max"):
            self._frame_max = {}
        self._frame_max[slot] = max_frames if steps > 0 else 0

    def frames_count(self, slot=0):
        n = C.c_int64()
        check(self._lib.crush_frames_count(self.h, slot, C.byref(n)))
        return n.value

    def frame(self, k, slot=0, n_nodes=None, n_hexes=None):
        """Kept frame k: time, step, displacement (N, 3), plastic_strain (E),
        stress (E, 6: xx yy zz xy yz xz), eroded (E); sizes default to the
        context's (a single-model context)."""
        nn = self.n_nodes if n_nodes is None else n_nodes
        ne = self.n_hexes if n_hexes is None else n_hexes
        t, st = C.c_double(), C.c_int64()
        d = np.zeros(3 * nn, np.float32)
        ps = np.zeros(ne, np.float32)
        sg = np.zeros(6 * ne, np.float32)
        er = np.zeros(ne, np.uint8)
        fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        check(self._lib.crush_frame_get(self.h, slot, k, C.byref(t), C.byref(st), fp(d), fp(ps), fp(sg),
                                        er.ctypes.data_as(C.POINTER(C.c_uint8))))
        return {"time": t.value, "step": st.value, "displacement": d.reshape(nn, 3), "plastic_strain": ps,
                "stress": sg.reshape(ne, 6), "eroded": er}

    def set_contact_search(self, exhaustive):
        """True: every contact search tests every face (no broad phase)."""
        check(self._lib.crush_set_contact_search(self.h, int(bool(exhaustive))))

    def append(self, descs):
        """Add models as new slots (crush_batch_append); returns the first
        new slot's index. With a run open, call on a multiple of 20 steps."""
        descs = list(descs)
        arr = (C.POINTER(abi.ModelDesc) * len(descs))(*[C.pointer(d) for d in descs])
        first = C.c_int()
        check(self._lib.crush_batch_append(self.h, arr, len(descs), C.byref(first)))
        self.n_slots = self._lib.crush_batch_size(self.h)
        nn, ne, na = C.c_int64(), C.c_int64(), C.c_int64()
        check(self._lib.crush_sizes(self.h, C.byref(nn), C.byref(ne), C.byref(na)))
        self.n_nodes, self.n_hexes, self.n_active = nn.value, ne.value, na.value
        return first.value

    def batch_done(self):
        """(done flag per slot, all done) of the open run."""
        flags = (C.c_int * self.n_slots)()
        all_ = C.c_int()
        check(self._lib.crush_batch_done(self.h, flags, C.byref(all_)))
        return [bool(x) for x in flags], bool(all_.value)

    def set_step_fusion(self, fused):
        """True (default): fuse a step's full update with the next step's half
        step where nothing falls between them; False: separate passes."""
        check(self._lib.crush_set_step_fusion(self.h, int(bool(fused))))

    def contact_search_stats(self, contact_id, reset=False):
        """(exhaustive fallback searches, overflow faces, walked gather roles) of a contact."""
        out = (C.c_uint64 * 3)()
        check(self._lib.crush_contact_search_stats(self.h, contact_id, out, int(reset)))
        return tuple(out)


def contact_apply_static(n_model_nodes, positions, u, masses, nodes, node_scale, faces, stiffness, max_distance, dt,
                         f_accum, stats=None, stream=0):
    """crush_contact_apply_static: one contact's penalty forces added into
    f_accum, with no allocation and no context. Every array argument is a raw
    device address (int) on the current device — nodes / faces as
    (address, count) pairs, node_scale and stats may be None; `stream` is a
    cudaStream_t address (0 = legacy default stream). Asynchronous."""
    (nodes_ptr, n_nodes), (faces_ptr, n_faces) = nodes, faces
    vp = C.c_void_p
    check(lib().crush_contact_apply_static(n_model_nodes, vp(positions), vp(u), vp(masses), n_nodes, vp(nodes_ptr),
                                           vp(node_scale), n_faces, vp(faces_ptr), stiffness, max_distance, dt,
                                           vp(f_accum), vp(stats), vp(stream)))


def run(desc, device=0):
    """crushrs::run on the GPU: results of a whole run of `desc`."""
    ctx = Context(desc, device)
    try:
        return ctx.run()
    finally:
        ctx.close()


def solve_batch(descs, device=0):
    """crush_batch_solve: every model of `descs` run as one batch, set-up
    pipelined with the run (later groups of models join the open run);
    per-model Results, each equal to the model run alone."""
    descs = list(descs)
    arr = (C.POINTER(abi.ModelDesc) * len(descs))(*[C.pointer(d) for d in descs])
    rs = (abi.Results * len(descs))()
    check(lib().crush_batch_solve(arr, len(descs), device, rs))
    return list(rs)
