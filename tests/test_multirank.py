"""The multi-rank path of bench.py on CPU: two gloo ranks (one process each)
set up the process group as bench.py does, take the max of their timings and
meet at the barriers. On GPUs the same code runs over NCCL, one rank per GPU,
each running a replica of the single-mesh workload and a share of the
batched crashes."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import bench
    import torch.distributed as dist

    w, r, _ = bench.dist_setup(backend="gloo")
    bench.barrier(w)
    m = bench.all_max(1.5 + r, w)
    total = bench.all_sum(10 * (r + 1), w)
    # the batched section's split: every rank computes the same one
    from crushrs_b200 import scenarios as S
    from crushrs_b200.serve import partition_by_footprint

    descs = [S.Model.build(S.batch_headon(i)).desc for i in range(24)]
    split = partition_by_footprint(descs, w)
    bench.barrier(w)
    out[r] = (w, r, m, total, split)
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(out.values(), key=lambda x: x[1])
    assert [g[:4] for g in got] == [(2, 0, 2.5, 30.0), (2, 1, 2.5, 30.0)]
    assert got[0][4] == got[1][4]  # the same split on both ranks
    assert sorted(got[0][4][0] + got[0][4][1]) == list(range(24))


def test_footprint_split_is_balanced_and_complete():
    from crushrs_b200 import scenarios as S
    from crushrs_b200.serve import footprint, partition_by_footprint

    descs = [S.Model.build(S.batch_headon(i)).desc for i in range(64)]
    sizes = [footprint(d) for d in descs]
    for parts in (1, 2, 3, 8):
        split = partition_by_footprint(descs, parts)
        assert len(split) == parts
        assert sorted(i for p in split for i in p) == list(range(64))
        loads = [sum(sizes[i] for i in p) for p in split]
        assert max(loads) - min(loads) <= max(sizes)  # largest first onto the least loaded
        assert split == partition_by_footprint(descs, parts)


class _FakeServer:
    """Stands in for a crush_server on CPU: every submitted crash finishes at
    once with its ticket as the result."""

    def __init__(self):
        self.pending = []
        self.next = 1

    def submit(self, desc):
        t = self.next
        self.next += 1
        self.pending.append(t)
        return t

    def poll(self, wait_ms=0):
        class R:
            pass

        out = []
        for t in self.pending:
            r = R()
            r.ticket = t
            r.submit_s = r.start_s = r.finish_s = 0.0
            out.append(r)
        self.pending = []
        return out


def _serve_rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    import bench
    import torch
    import torch.distributed as dist

    w, r, _ = bench.dist_setup(backend="gloo")
    from crushrs_b200 import scenarios as S
    from crushrs_b200.serve import serve_share

    models = [S.Model.build(S.serve_query(i, e_range=(300, 2000))[1]) for i in range(40)]
    res, _ = serve_share(_FakeServer(), models, rate=4000.0, rank=r, parts=w, seed=5)
    # the only exchange: which stream indices each rank served, gathered on the host
    mine = torch.zeros(len(models), dtype=torch.int64)
    for i in res:
        mine[i] = r + 1
    dist.all_reduce(mine)
    out[r] = (sorted(res), mine.tolist())
    dist.destroy_process_group()


def test_two_gloo_ranks_serve_disjoint_shares_of_one_stream():
    """Multi-GPU serving: two ranks draw the same seeded stream, each serves
    the crashes the online router places on it, and together they serve
    every crash exactly once."""
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = out[0], out[1]
    assert a[1] == b[1]  # both ranks see the same ownership after the gather
    assert set(a[0]).isdisjoint(b[0]) and sorted(a[0] + b[0]) == list(range(40))
    assert all(x in (1, 2) for x in a[1])
    assert abs(len(a[0]) - len(b[0])) <= 8  # balanced by estimated bytes


def test_online_router_is_least_loaded_and_deterministic():
    from crushrs_b200.serve import route_online

    sizes = [5.0, 1.0, 1.0, 3.0, 2.0, 2.0]
    assert route_online(sizes, 2) == [0, 1, 1, 1, 0, 1]
    assert route_online(sizes, 2) == route_online(list(sizes), 2)
    assert route_online(sizes, 1) == [0] * 6
