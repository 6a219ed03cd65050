#!/usr/bin/env python
"""Headline benchmark of the B200 crash engine.

Main line (the workload the metric is quoted on when it fits one GPU): the
refined head-on, 278,640 one-point honeycomb hexahedra, 299,666 nodes, run to
separation (<= 5000 steps). One step = the whole explicit time step: stable-dt
check and mass scaling (every 5 steps), node-to-face contact, the half step,
the element forces, the ordered force gather with the full step.

  value      element-updates/s of the whole job over exactly K steps after W
             warm-up steps, device-timed (CUDA events on the engine's stream),
             inputs resident in HBM; the per-step working set (~0.33 GB) is
             larger than L2, so no flush is needed.
  e2e        the same metric end to end through the reference-facing C ABI
             with host buffers: crush_create from the host model (the upload
             inside the timed region) + crush_run to separation + the FP64
             delta-v results read back, host-clock timed.
  e2e_dropin the drop-in loop a reference caller would write (src/solver.rs:
             287-342 on the host, crush_contact_apply + crush_compute_forces
             per step, u in and forces out through host buffers).
  roofline   HBM roofline of the element-force kernel: algorithmic bytes per
             launch (870 B per element + 24 B per node) over its average
             device time inside the timed region.
  cpu_baseline  the oracle's f32 8-lane restatement of the reference step on
             all host threads, a bounded number of steps of the same mesh.
  batched    4096 seeded uneven head-on crashes (300-6000 elements) in one
             batched context, crashes/s (host clock, set-up included) against
             the plain one-crash-per-launch path (crush_create + crush_run per
             crash) on a sample, and the FP64 delta-v error of a sample against
             the reference's f64 scalar restatement.
  serving    the crash server (continuous batching: requests join running
             serving contexts between chunks of steps) under open-loop
             Poisson streams of seeded head-on / T-bone / rear-end queries
             (300-20000 elements) at 200, 500, 1000 and 2000 req/s:
             crashes/s and p50/p99 submit-to-result latency, beside the
             median time of one query run alone.
--impl reference runs the CPU restatement of the reference as the reference arm.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_ELEM_KERNEL = 870  # per element: conn 32, grad 96, volume 4, gamma 128, H 312, state r+w 200, eroded r+w 2, corner forces 96
BYTES_NODE_KERNEL = 24   # per node: positions + displacements read by the element kernel
BYTES_STEP_ELEM = 998    # whole step, per element
BYTES_STEP_NODE = 92     # whole step, per node
METRIC = "crashes/sec + p50/p99 latency vs plain GPU path at <=0.5% delta-v err; elem-upd/s"


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def read_traffic(n_elem):
    """dram bytes per element-kernel launch from the committed ncu summary,
    scaled from the captured case by elements."""
    path = os.path.join(ROOT, "profiles", "k_forces_refined_headon.txt")
    try:
        vals = {}
        with open(path) as f:
            for line in f:
                if ":" in line:
                    k, v = line.split(":", 1)
                    vals[k.strip()] = v.strip()
        per_elem = float(vals["dram_bytes_per_element"])
        return per_elem * n_elem
    except Exception:
        return None


class ClockSampler:
    """SM clocks and throttle reasons sampled from NVML every ~2 ms on a
    thread started before the warm-up, so the few milliseconds of a short
    timed region still get samples. mark_start()/mark_end() bracket the
    timed region; summary() reports the samples inside it ("timed region")
    and, when it holds none, the samples from warm-up to its end."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, device, period_s=0.002):
        self.device = device
        self.period_s = period_s
        self.samples = []  # (host time, sm MHz, max sm MHz, reasons bitmask)
        self.t_start = self.t_end = None
        self._stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nv = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self._max = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def _run(self):
        nv, h = self._nv, self._h
        while not self._stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = self._reasons(h)
                self.samples.append((time.perf_counter(), float(sm), float(self._max), int(rs)))
            except Exception:
                return
            self._stop.wait(self.period_s)

    def mark_start(self):
        self.t_start = time.perf_counter()

    def mark_end(self):
        self.t_end = time.perf_counter()

    def __exit__(self, *a):
        self._stop.set()
        if self.thread:
            self.thread.join(timeout=2)
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        inside = [x for x in self.samples if self.t_start is not None and self.t_end is not None and self.t_start <= x[0] <= self.t_end]
        window = "timed region"
        if not inside:
            inside = [x for x in self.samples if self.t_end is None or x[0] <= self.t_end]
            window = "warm-up through timed region"
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "window": None, "source": "nvml"}
        reasons = sorted(name for name, bit in self.REASONS.items() if any(x[3] & bit for x in inside))
        return {"sm_mhz": statistics.median(x[1] for x in inside), "sm_max_mhz": inside[-1][2], "reasons": reasons,
                "samples": len(inside), "window": window, "source": "nvml, every 2 ms"}


def dist_setup(backend=None):
    """One process per GPU (torchrun's env): the process group for the
    barrier and the max-over-ranks timing. The single-mesh workload does not
    shard, so ranks run replicas and exchange nothing else. backend: "nccl"
    (default) or "gloo" (the CPU tests of this path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = backend or "nccl"
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    return world, rank, local


def all_sum(x, world):
    """Sum of x over the ranks."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def all_max(x, world):
    """Max of x over the ranks (the job's time is its slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def cpu_reference(desc, steps, threads):
    """The oracle's restatement of the reference step loop, bounded to `steps`."""
    from tests import oracle_lib as O

    s = desc.settings
    saved = (s.max_steps, s.stop_rule)
    desc.settings.max_steps = steps
    desc.settings.stop_rule = 0
    try:
        r, _, _, _, sec = O.run(desc, simd=True, threads=threads)
    finally:
        desc.settings.max_steps, desc.settings.stop_rule = saved
    loop = sec[3]
    return r.steps, loop, sec


def e2e_dropin(ctx, desc, steps, n_hc):
    """Reference-facing drop-in loop (src/solver.rs:287-342 as the caller):
    host f64 state, GPU contact + element forces through the C ABI each step."""
    import torch

    n = desc.n_nodes
    pin = lambda: torch.zeros(3 * n, dtype=torch.float64).pin_memory().numpy()
    u, v, vh, f_int, f_ext = pin(), pin(), pin(), pin(), pin()
    v[:] = np.ctypeslib.as_array(desc.initial_velocity, (3 * n,))
    lumped, _ = ctx.masses()
    inv_m = np.repeat(np.where(lumped > 0, 1.0 / np.where(lumped > 0, lumped, 1.0), 0.0), 3)
    fixed = np.zeros(n, bool)
    if desc.n_fixed:
        fixed[np.ctypeslib.as_array(desc.fixed_nodes, (desc.n_fixed,))] = True
    fixed3 = np.repeat(fixed, 3)
    dt = 1e-5
    ctx.compute_forces(u, f_int)
    t0 = time.perf_counter()
    for _ in range(steps):
        f_ext[:] = 0.0
        for c in range(desc.n_contacts):
            ctx.contact_apply(c, u, None, None, dt, f_ext)
        a = (f_ext - f_int) * inv_m
        vh[:] = v + 0.5 * dt * a
        u += dt * vh
        u[fixed3] = 0.0
        f_int[:] = 0.0
        ctx.compute_forces(u, f_int)
        a = (f_ext - f_int) * inv_m
        v[:] = vh + 0.5 * dt * a
        v[fixed3] = 0.0
    wall = time.perf_counter() - t0
    h2d = 8 * 3 * n * (desc.n_contacts + 1)
    d2h = 8 * 3 * n * (desc.n_contacts + 1)
    return n_hc * steps / wall, h2d, d2h


def e2e_run(desc, device, n_hc, n_nodes):
    """crush_create from the host model + crush_run + results: host-clock elem-upd/s."""
    from crushrs_b200.engine import Context

    t0 = time.perf_counter()
    ctx = Context(desc, device=device)
    r = ctx.run()
    wall = time.perf_counter() - t0
    ctx.close()
    steps = max(int(r.steps), 1)
    h2d = 8 * 6 * n_nodes + 36 * desc.n_hexes  # positions, velocities, hexes, parts, incidence
    return {"value": n_hc * r.steps / wall, "unit": "elem-upd/s", "steps": int(r.steps), "wall_s": wall,
            "h2d_bytes_per_step": int(h2d / steps), "d2h_bytes_per_step": int((8 * 7 * 2 + 4 * 4096) / steps),
            "path": "crush_create (host model) + crush_run to separation + FP64 delta-v read back",
            "delta_v": [r.vehicle[k].delta_v[0] for k in range(r.n_vehicles)]}


def batched_section(n, plain_sample, oracle_sample, device, world=1):
    """4096 seeded uneven head-on crashes as one batch vs the plain
    one-crash-per-launch path. The batch runs through crush_batch_solve (the
    set-up pipelined with the run: later groups of crashes join the open
    run) and, beside it, as one context created from all crashes before its
    run (crush_batch_create + crush_batch_run, "one_shot"). With several
    ranks the crashes are split by estimated device bytes
    (serve.partition_by_footprint, the same on every rank) and each rank
    solves its share; the time is the slowest rank's, with no collective on
    the data path."""
    from crushrs_b200 import scenarios as S
    from crushrs_b200.engine import Context, solve_batch
    from crushrs_b200.serve import partition_by_footprint

    all_models = [S.Model.build(S.batch_headon(i)) for i in range(n)]
    if world > 1:
        import torch.distributed as dist

        mine = partition_by_footprint([m.desc for m in all_models], world)[dist.get_rank()]
        models = [all_models[i] for i in mine]
    else:
        models = all_models
    elems = sum(m.n_hexes for m in models)
    w = Context(models[0].desc, device=device)  # CUDA and module warm-up
    w.run()
    w.close()
    barrier(world)
    t0 = time.perf_counter()
    rs = solve_batch([m.desc for m in models], device=device)
    t1 = time.perf_counter()
    steps = [int(r.steps) for r in rs]
    eu = sum(m.n_hexes * st for m, st in zip(models, steps))
    if world > 1:
        wall = all_max(t1 - t0, world)
        total_eu = all_sum(eu, world)
        return {"crashes": n, "ranks": world, "crashes_this_rank": len(models), "crashes_per_s": n / wall, "wall_s": wall,
                "elem_upd_per_s": total_eu / wall, "split": "by estimated device bytes, largest first to the least-loaded rank",
                "scaling": "strong: the same crashes shared by the ranks", "path": "crush_batch_solve per rank"}
    # the same crashes as one context created from all of them, then run
    t2 = time.perf_counter()
    ctx = Context([m.desc for m in models], device=device)
    t3 = time.perf_counter()
    rs1 = ctx.batch_run()
    t4 = time.perf_counter()
    lanes, _ = ctx.tuning()
    launches = ctx.launches()
    ctx.close()
    fields = lambda r: (r.status, r.steps, r.time, r.dt_min, r.eroded_elements,
                        [tuple(r.vehicle[k].delta_v) + (r.vehicle[k].crush,) for k in range(r.n_vehicles)])
    solve_equals_one_shot = all(fields(a) == fields(b) for a, b in zip(rs, rs1))
    # plain path: one context and one run per crash, a sample, after its own warm-up
    times = []
    same = True
    for i in range(plain_sample):
        t = time.perf_counter()
        c = Context(models[i].desc, device=device)
        r = c.run()
        c.close()
        times.append(time.perf_counter() - t)
        same &= r.steps == rs[i].steps and list(r.vehicle[0].delta_v) == list(rs[i].vehicle[0].delta_v)
    batched_cps = n / (t1 - t0)
    out = {"crashes": n, "elements": elems, "wall_s": t1 - t0, "crashes_per_s": batched_cps,
           "elem_upd_per_s": eu / (t1 - t0), "steps_mean": statistics.mean(steps), "steps_max": max(steps),
           "path": "crush_batch_solve: a context from the first eighth of the elements starts the run, the rest join it "
                   "group by group at step-graph boundaries (set-up overlapping the run)",
           "one_shot": {"create_s": t3 - t2, "run_s": t4 - t3, "crashes_per_s": n / (t4 - t2), "gpu_launches": int(launches),
                        "slave_lanes": lanes, "path": "crush_batch_create of all crashes, then crush_batch_run"},
           "solve_equals_one_shot": bool(solve_equals_one_shot)}
    if times:
        plain_s = statistics.median(times)
        out["plain"] = {"crashes_per_s": 1.0 / plain_s, "median_s_per_crash": plain_s, "sample": plain_sample,
                        "path": "crush_create + crush_run per crash (CUDA graphs of 20 steps)"}
        out["speedup_vs_plain"] = batched_cps * plain_s
        out["one_shot"]["speedup_vs_plain"] = n / (t4 - t2) * plain_s
        out["batched_equals_plain"] = bool(same)
    if oracle_sample:
        from tests import oracle_lib as O

        errs = []
        for i in range(oracle_sample):
            ro, _, _, _, _ = O.run(models[i].desc, simd=False, threads=os.cpu_count() or 1)
            for k in range(rs[i].n_vehicles):
                ref = ro.vehicle[k].delta_v[0]
                errs.append(abs(rs[i].vehicle[k].delta_v[0] - ref) / max(abs(ref), 1e-9))
        out["delta_v_max_rel_err_vs_f64_oracle"] = max(errs)
        out["delta_v_oracle_sample"] = oracle_sample
    return out


def two_part_section(n, device):
    """Two-part vehicles (crush zone, rail box, bumper, elastic Hencky body):
    the Navigator into the pulse-fitted Neon at 30.14 mph each to 150 ms,
    alone and as a batch of n with seeded rail boxes (the calibration's
    workload, src/headon.rs:147-250)."""
    from crushrs_b200 import calibrate as K, scenarios as S
    from crushrs_b200.engine import Context

    setup = K.HeadOn(30.14 * S.MPH, 30.14 * S.MPH)
    a, b = S.lincoln_navigator_1999(), S.neon_1996_pulse()
    m = setup.build(a, b)
    elastic = sum(1 for p in m.hex_part() if m.material(p).model == 1)
    w = Context(m.desc, device=device)
    w.run()
    w.close()
    t0 = time.perf_counter()
    c = Context(m.desc, device=device)
    r = c.run()
    c.close()
    single = time.perf_counter() - t0
    rng = K.Rng(0x5EED)
    pairs = []
    for _ in range(n):
        u = [rng.uniform() for _ in range(8)]
        pairs.append((K.with_rail_box(a, K.rail_box_from_unit(tuple(a.size), u[:4])),
                      K.with_rail_box(b, K.rail_box_from_unit(tuple(b.size), u[4:]))))
    models = [setup.build(x, y) for x, y in pairs]
    t0 = time.perf_counter()
    ctx = Context([x.desc for x in models], device=device)
    rs = ctx.batch_run()
    ctx.close()
    batch = time.perf_counter() - t0
    eu = sum(x.n_hexes * int(q.steps) for x, q in zip(models, rs))
    return {"elements": m.n_hexes, "elastic_elements": elastic, "steps": int(r.steps), "single_s": single,
            "single_elem_upd_per_s": m.n_hexes * r.steps / single, "batch": n, "batch_s": batch,
            "batch_crashes_per_s": n / batch, "batch_elem_upd_per_s": eu / batch,
            "path": "crush_create + crush_run (single); crush_batch_create + crush_batch_run (batch), set-up included"}


def serving_pool(n):
    """n distinct seeded serving queries (head-on, T-bone, rear-end; 300-20000
    hexahedra), built once; the arrival stream cycles through them."""
    from crushrs_b200 import scenarios as S

    return [S.Model.build(S.serve_query(i)[1]) for i in range(n)]


SERVE_QUEUE = 1024
TRIAL_STEPS = 240  # the engine's schedule trial: 2 rounds x 6 candidate schedules x a 20-step graph


def serving_section(rate, seconds, device, pool):
    """The crash server under an open-loop Poisson stream at `rate` req/s
    for `seconds` of arrivals (continuous batching: requests join running
    serving contexts between chunks of steps)."""
    from crushrs_b200.serve import Server, open_loop

    n = max(1, int(rate * seconds))
    models = [pool[i % len(pool)] for i in range(n)]
    # admission control: at most SERVE_QUEUE requests wait; arrivals beyond
    # are refused (counted), as a service under overload sheds load
    with Server(device=device, max_queue=SERVE_QUEUE) as srv:
        res, wall, tickets = open_loop(srv, models, rate=rate)
        st = srv.stats()
    refused = sum(1 for t in tickets if t < 0)
    lat = sorted(r.finish_s - r.submit_s for r in res.values())
    wait = sorted(r.start_s - r.submit_s for r in res.values())
    pick = lambda xs, q: xs[min(len(xs) - 1, int(q * len(xs)))]
    return {"rate_req_per_s": rate, "seconds": seconds, "arrivals": n, "refused": refused, "queue_limit": SERVE_QUEUE,
            "crashes": len(res), "crashes_per_s": len(res) / wall, "wall_s": wall,
            "p50_ms": 1e3 * pick(lat, 0.5), "p99_ms": 1e3 * pick(lat, 0.99), "admission_wait_p50_ms": 1e3 * pick(wait, 0.5),
            "contexts": int(st.waves), "peak_gb": st.peak_bytes_in_use / 1e9,
            "elements_mean": sum(m.n_hexes for m in models) / n, "ok": all(r.status == 0 for r in res.values())}


def serving_standalone(pool, device, sample=16):
    """Median seconds of one query alone (crush_create + crush_run), the
    reference point of the served latencies."""
    from crushrs_b200.engine import Context

    times = []
    for m in pool[:sample]:
        t = time.perf_counter()
        c = Context(m.desc, device=device)
        c.run()
        c.close()
        times.append(time.perf_counter() - t)
    return statistics.median(times)


def serving_all(args, device):
    pool = serving_pool(args.serve_pool)
    alone = serving_standalone(pool, device)
    return {"standalone_median_ms": 1e3 * alone, "pool": len(pool),
            "rates": [serving_section(float(r), args.serve_seconds, device, pool) for r in args.serve_rates.split(",") if r]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--batch", type=int, default=4096, help="crashes of the batched section (0: skip)")
    ap.add_argument("--plain-sample", type=int, default=64)
    ap.add_argument("--oracle-sample", type=int, default=4)
    ap.add_argument("--serve-rates", default="100,200,500,1000,2000", help="req/s of the serving section ('' : skip)")
    ap.add_argument("--serve-seconds", type=float, default=10.0, help="seconds of arrivals per rate")
    ap.add_argument("--serve-pool", type=int, default=1024, help="distinct seeded queries the arrival stream cycles through")
    ap.add_argument("--schedule-steps", type=int, default=200, help="steps timed under each step schedule after the main region")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sections", default="refined,e2e,batched,serving,cpu",
                    help="which parts to run (profiling runs pick one; the refined part gives the main line's value)")
    args = ap.parse_args()
    sections = set(args.sections.split(","))
    if "e2e" not in sections:
        args.no_e2e = True
    if "cpu" not in sections:
        args.no_cpu = True
    if "batched" not in sections:
        args.batch = 0
    if "serving" not in sections:
        args.serve_rates = ""
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")

    world, rank, local = dist_setup()
    config = {"workload": "refined head-on, 0.05 m hexahedra (36x30x138 + 36x24x150), run to separation (<= 5000 steps)",
              "elements": None, "nodes": None, "timed_steps": None,
              "l2": "per-step working set > L2 (126 MB), no flush",
              "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}

    if args.impl == "reference":
        # The reference's step loop as the oracle restates it (f32 8-lane
        # element kernel on all host threads, serial scatter, contact and
        # update), on the same refined head-on built by the checker's numpy
        # builder: this arm never loads the engine library. Exactly K steps
        # after W warm-up steps are timed.
        if rank != 0:
            return
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import headon as H
        from tests import oracle_lib as O

        threads = os.cpu_count() or 1
        model = H.refined_headon(max_steps=args.warmup + args.steps)
        n_hc = int((model.hex_part < 2).sum())
        config["elements"] = n_hc
        config["nodes"] = int(model.n_nodes)
        config["timed_steps"] = f"steps {args.warmup}..{args.warmup + args.steps}"
        r, _, _, _, sec = O.run_window(model.desc, time_from_step=args.warmup, simd=True, threads=threads)
        steps = int(r.steps) - args.warmup
        value = n_hc * steps / sec[4]
        line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "elem-upd/s", "n_gpus": args.gpus, "steps": steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * sec[4] / steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32 element / f64 nodal", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": value, "unit": "elem-upd/s", "cores": threads, "kind": "port",
                                 "sample": f"steps {args.warmup}..{args.warmup + args.steps} of the refined head-on (whole step: contact, "
                                           "forces, update, dt), oracle f32 8-lane AVX2 restatement, model from the numpy builder"},
                "e2e": {"value": value, "unit": "elem-upd/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    from crushrs_b200 import scenarios as S

    model = S.Model.build(S.refined_headon())
    desc = model.desc
    n_nodes = desc.n_nodes
    config["nodes"] = n_nodes

    from crushrs_b200.engine import Context

    if "refined" not in sections:
        line = {"metric": METRIC, "sections": sorted(sections)}
        if args.batch > 0:
            b = batched_section(args.batch, args.plain_sample, args.oracle_sample, local, world)
            if rank == 0:
                line["batched"] = b
        if rank == 0 and world == 1 and args.serve_rates:
            line["serving"] = serving_all(args, local)
        if rank == 0 and "twopart" in sections:
            line["two_part"] = two_part_section(64, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return

    ctx = Context(desc, device=local)
    n_hc = ctx.n_active
    config["elements"] = n_hc
    clocks = ClockSampler(local).__enter__()
    ctx.run_begin()
    # Inside the timed region the step graph records CUDA events around the
    # element-force kernel only (two per step); the per-phase breakdown comes
    # from a short profiled region after it.
    ctx.set_profiling(1)
    ctx.run_steps_timed(args.warmup, phases=True)
    # Untimed: steps up to a step-graph boundary (the engine replays one
    # captured graph per 20 steps), TRIAL_STEPS more (where a context large
    # enough holds the schedule trial: two rounds of its six candidate
    # schedules, a graph period each), then the schedule is kept for the rest
    # of the run (no re-tuning, so no graph is captured inside the timed
    # region) and its graph built over two periods.
    align = (-args.warmup) % 20
    ctx.run_steps_timed(align + TRIAL_STEPS, phases=True)
    ctx.fix_schedule()
    ctx.run_steps_timed(40, phases=True)
    first = args.warmup + align + TRIAL_STEPS + 40
    config["timed_steps"] = (f"steps {first}..{first + args.steps} (warm-up: {args.warmup} steps, {align} to a step-graph boundary, "
                             f"{TRIAL_STEPS} more (a context of 2M+ elements holds its schedule trial there), 40 on the kept "
                             f"schedule's graph)")
    barrier(world)
    launches0 = ctx.launches()
    # phase events of the last graph only; the force kernel's average comes
    # from a separate profiled window of the same length inside the run
    clocks.mark_start()
    done, ms, phases, psteps = ctx.run_steps_timed(args.steps, phases=True)
    clocks.mark_end()
    clocks.__exit__(None, None, None)
    launches = ctx.launches() - launches0
    ms_max = all_max(ms, world)
    barrier(world)
    ctx.set_profiling(2)
    _, _, all_phases, all_psteps = ctx.run_steps_timed(40, phases=True)
    lanes, tune_ms = ctx.tuning()
    # The same run continued under each step schedule (bit-identical
    # results): separate half and full passes, then the fused one.
    # The element kernel's schedule the run chose (and the trial's timings).
    chosen, trial_ms = ctx.schedule()
    schedules = {"chosen_forces_schedule": chosen, "trial_ms_per_step": trial_ms}
    for name, fused, fs in (("separate, persistent forces", False, 0), ("fused, persistent forces", True, 0),
                            ("fused, block-per-chunk forces", True, 1)):
        ctx.set_step_fusion(fused)
        ctx.set_tuning(lanes, fs)
        ctx.run_steps_timed(40)
        _, ms_s, _, _ = ctx.run_steps_timed(args.schedule_steps)
        schedules[name] = {"ms_per_step": ms_s / args.schedule_steps, "steps": args.schedule_steps}
    value = world * n_hc * args.steps / (ms_max / 1e3)
    peak, peak_kind = measured_peak()
    forces_ms = phases[3] / psteps
    bytes_launch = BYTES_ELEM_KERNEL * n_hc + BYTES_NODE_KERNEL * n_nodes
    achieved = bytes_launch / (forces_ms / 1e3) / 1e9
    step_bytes = BYTES_STEP_ELEM * n_hc + BYTES_STEP_NODE * n_nodes
    step_gbs = step_bytes / (ms / args.steps / 1e3) / 1e9
    traffic = read_traffic(n_hc)
    line = {"metric": METRIC, "value": value, "unit": "elem-upd/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 element / f64 nodal", "data": "synthetic", "config": config, "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "k_forces", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": traffic, "bytes_per_launch": bytes_launch, "avg_launch_ms": forces_ms},
            "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_gbs, "frac": step_gbs / peak},
            "phase_ms_per_step": {k: v / all_psteps for k, v in zip(["dt", "contact", "half", "forces", "gather_full", "checks"], all_phases)},
            "clocks": clocks.summary(), "run_done_early": done, "slave_lanes": lanes, "schedules": schedules}
    ctx.close()
    if rank == 0 and world == 1 and not args.no_e2e:
        line["e2e"] = e2e_run(desc, local, n_hc, n_nodes)
        c3 = Context(desc, device=local)
        e, h2d, d2h = e2e_dropin(c3, desc, args.e2e_steps, n_hc)
        c3.close()
        line["e2e_dropin"] = {"value": e, "unit": "elem-upd/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                              "path": "crush_contact_apply x contacts + crush_compute_forces per step, host f64 state, pinned buffers"}
    if args.batch > 0:
        b = batched_section(args.batch, args.plain_sample, args.oracle_sample, local, world)
        if rank == 0:
            line["batched"] = b
    if rank == 0 and world == 1 and args.serve_rates:
        line["serving"] = serving_all(args, local)
    if rank == 0 and world == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        steps, loop, sec = cpu_reference(desc, args.cpu_steps, threads)
        line["cpu_baseline"] = {"value": n_hc * steps / loop, "unit": "elem-upd/s", "cores": threads, "kind": "port",
                                "sample": f"{steps} steps of the same mesh (contact, forces, update, dt), oracle f32 8-lane AVX2 restatement"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
