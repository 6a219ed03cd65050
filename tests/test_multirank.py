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
