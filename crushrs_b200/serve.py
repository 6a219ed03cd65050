"""Python face of the continuous-batching crash server (include/crush_server.h).

    with Server(max_waves=4) as srv:
        t = srv.submit(model.desc)          # copies the model, returns a ticket
        for r in srv.poll(wait_ms=100):     # finished crashes, as they finish
            print(r.ticket, r.results.vehicle[0].delta_v[0], r.finish_s - r.submit_s)

Also an open-loop Poisson load driver for latency and throughput figures.
"""
import ctypes as C
import math
import time

from . import abi
from .native import check, lib


class Server:
    """crush_server: waves of batched contexts on one GPU."""

    def __init__(self, device=0, max_waves=4, max_wave_slots=1024, chunk_steps=100, max_wave_elements=2_000_000,
                 hbm_budget_bytes=0.0, gather_ms=2.0, idle_ms=200.0, max_queue=0, max_running=0):
        self._lib = lib()
        cfg = abi.ServerConfig(device, max_waves, max_wave_slots, chunk_steps, max_wave_elements, hbm_budget_bytes, gather_ms, idle_ms,
                               max_queue, max_running)
        h = C.c_void_p()
        check(self._lib.crush_server_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def submit(self, desc):
        """Queue a model; its ticket, or None when the server's max_queue
        requests already wait (the request is refused)."""
        t = C.c_uint64()
        st = check(self._lib.crush_server_submit(self.h, C.byref(desc), C.byref(t)), allow=(abi.CRUSH_OK, abi.CRUSH_ERR_BUSY))
        return t.value if st == abi.CRUSH_OK else None

    def poll(self, max_results=256, wait_ms=0):
        out = (abi.ServerResult * max_results)()
        n = C.c_int()
        check(self._lib.crush_server_poll(self.h, out, max_results, C.byref(n), wait_ms))
        return [out[k] for k in range(n.value)]

    def stats(self):
        s = abi.ServerStats()
        check(self._lib.crush_server_stats_get(self.h, C.byref(s)))
        return s

    def close(self):
        if getattr(self, "h", None):
            self._lib.crush_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def footprint(desc):
    """The server's admission estimate of a model's device bytes."""
    return lib().crush_model_footprint(C.byref(desc))


def partition_by_footprint(descs, parts):
    """Split crashes across `parts` GPUs by estimated device bytes: largest
    first onto the least-loaded GPU (ties: the lower index), so every rank
    computes the same split. Returns one list of crash indices per part,
    each ascending."""
    sizes = [footprint(d) for d in descs]
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(descs)), key=lambda k: (-sizes[k], k)):
        g = min(range(parts), key=lambda q: (load[q], q))
        out[g].append(i)
        load[g] += sizes[i]
    return [sorted(x) for x in out]


def route_online(sizes, parts):
    """Placement of a stream of crashes across `parts` GPUs as they arrive:
    each goes to the GPU with the fewest estimated device bytes placed so far
    (ties: the lower index). Every rank computes the same placement from the
    same seeded stream, so each serves its share with no exchange of
    requests. Returns the GPU of every crash, in arrival order."""
    load = [0.0] * parts
    out = []
    for x in sizes:
        g = min(range(parts), key=lambda q: (load[q], q))
        out.append(g)
        load[g] += x
    return out


def serve_share(server, models, rate, rank, parts, seed=1):
    """This rank's share of an open-loop stream served across `parts` GPUs:
    the full stream's arrival times are drawn on every rank (same seed), and
    the rank submits the crashes route_online places on it at their arrival
    times. Returns (results by stream index, wall seconds)."""
    sizes = [footprint(m.desc) for m in models]
    mine = [i for i, g in enumerate(route_online(sizes, parts)) if g == rank]
    rng = _Rng(seed)
    times, t = [], 0.0
    for _ in models:
        times.append(t)
        t += -math.log(1.0 - rng.uniform()) / rate
    t0 = time.perf_counter()
    tickets, results, i = {}, {}, 0
    while i < len(mine) or len(results) < len(mine):
        now = time.perf_counter() - t0
        while i < len(mine) and times[mine[i]] <= now:
            tickets[server.submit(models[mine[i]].desc)] = mine[i]
            i += 1
        for r in server.poll(wait_ms=0 if i < len(mine) else 20):
            results[tickets[r.ticket]] = r
        if i < len(mine):
            sleep = times[mine[i]] - (time.perf_counter() - t0)
            if sleep > 0:
                time.sleep(min(sleep, 0.002))
    return results, time.perf_counter() - t0


def open_loop(server, models, rate, seed=1):
    """Submit `models` (objects with .desc) at Poisson arrival times of the
    given rate (req/s), open loop; returns (results by ticket, wall seconds,
    ticket -> model index). Requests the server refuses (its queue full) are
    counted in the returned map under negative keys, without results."""
    rng = _Rng(seed)
    t0 = time.perf_counter()
    t_next = 0.0
    tickets = {}
    results = {}
    refused = 0
    i = 0
    while i < len(models) or len(results) < len(models) - refused:
        now = time.perf_counter() - t0
        while i < len(models) and t_next <= now:
            t = server.submit(models[i].desc)
            if t is None:
                refused += 1
                tickets[-refused] = i
            else:
                tickets[t] = i
            i += 1
            t_next += -math.log(1.0 - rng.uniform()) / rate
        wait = 0 if i < len(models) else 20
        for r in server.poll(wait_ms=wait):
            results[r.ticket] = r
        if i < len(models):
            sleep = t_next - (time.perf_counter() - t0)
            if sleep > 0:
                time.sleep(min(sleep, 0.002))
    return results, time.perf_counter() - t0, tickets


class _Rng:
    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF or 1

    def uniform(self):
        x = self.s
        x ^= x >> 12
        x ^= (x << 25) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 27
        self.s = x
        return (((x * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF) >> 11) / float(1 << 53)
