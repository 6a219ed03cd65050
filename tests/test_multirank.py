"""The multi-rank path of bench.py on CPU: two gloo ranks (one process each)
set up the process group as bench.py does, take the max of their timings and
meet at the barriers. On GPUs the same code runs over NCCL, one rank per GPU,
each running a replica of the single-mesh workload."""
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
    bench.barrier(w)
    out[r] = (w, r, m)
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
    assert sorted(out.values()) == [(2, 0, 2.5), (2, 1, 2.5)]
