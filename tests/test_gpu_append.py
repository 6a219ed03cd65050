"""Continuous batching: models added to a context as new slots
(crush_batch_append), before its run or while it runs. Every slot's
results are bit-identical to the same model run alone, whether it was
created with the context or joined a running one, next to slots that stop
earlier or later; a context refuses models beyond its room and runs on."""
import numpy as np
import pytest

from crushrs_b200 import abi, scenarios as S
from crushrs_b200.engine import Context
from crushrs_b200.native import CrushError

from .test_gpu_batch import _same

pytestmark = pytest.mark.gpu

ROOM = dict(slots=64, contacts=256, nodes=400_000, hexes=300_000, faces=80_000, primary_nodes=120_000)


@pytest.fixture(scope="module")
def models():
    ms = [S.Model.build(S.batch_headon(i)) for i in range(6)]
    ms.append(S.Model.build(S.plain_headon(end_time=0.0301)))
    ms.append(S.Model.build(S.serve_query(3)[1]))
    ms.append(S.Model.build(S.serve_query(11)[1]))
    return ms


@pytest.fixture(scope="module")
def alone(models):
    out = []
    for m in models:
        ctx = Context(m.desc)
        out.append(ctx.run())
        ctx.close()
    return out


def _run_to_end(ctx, chunk=100):
    done = False
    while not done:
        done = ctx.run_steps(chunk)


def test_append_before_the_run_equals_alone(models, alone):
    ctx = Context([m.desc for m in models[:2]], room=ROOM)
    assert ctx.append([m.desc for m in models[2:5]]) == 2
    assert ctx.append([m.desc for m in models[5:]]) == 5
    rs = ctx.batch_run()
    for r, a in zip(rs, alone):
        _same(r, a)


def test_append_into_a_running_context_equals_alone(models, alone):
    """Slots join an open run at steps 40, 200 and 500 (graph boundaries)
    and each gives exactly its alone results, as do the slots already
    running."""
    ctx = Context([m.desc for m in models[:2]], room=ROOM)
    ctx.run_begin()
    ctx.run_steps(40)
    first = ctx.append([m.desc for m in models[2:4]])
    assert first == 2
    ctx.run_steps(160)
    ctx.append([models[4].desc, models[7].desc])
    ctx.run_steps(300)
    ctx.append([models[5].desc, models[6].desc, models[8].desc])
    _run_to_end(ctx)
    order = [0, 1, 2, 3, 4, 7, 5, 6, 8]
    for slot, k in enumerate(order):
        _same(ctx.results(slot), alone[k])


def test_append_every_period_equals_alone(models, alone):
    """The serving pattern: one graph period issued at a time with slots
    joining at most boundaries (each set up beside the period in flight,
    the period after a join launched step by step), then periods without
    joins (graphs again); every slot gives its alone results."""
    ctx = Context([models[0].desc], room=ROOM)
    ctx.run_begin()
    order = [0]
    for k in range(1, len(models)):
        ctx.run_steps(20)
        ctx.append([models[k].desc])
        order.append(k)
        if k % 3 == 0:
            ctx.run_steps(40)
    _run_to_end(ctx, chunk=20)
    for slot, k in enumerate(order):
        _same(ctx.results(slot), alone[k])


def test_append_refuses_beyond_room_and_runs_on(models, alone):
    small = dict(slots=3, contacts=12, nodes=10_000, hexes=8_000, faces=3_000, primary_nodes=4_000)
    ctx = Context([models[0].desc], room=small)
    ctx.run_begin()
    ctx.run_steps(20)
    big = S.Model.build(S.serve_query(7, e_range=(15_000, 20_000))[1])
    with pytest.raises(CrushError) as e:
        ctx.append([big.desc])
    assert e.value.status == abi.CRUSH_ERR_BUSY
    assert ctx.n_slots == 1
    with pytest.raises(CrushError) as e:  # off a step-graph boundary
        ctx.run_steps(7)
        ctx.append([models[1].desc])
    assert e.value.status == abi.CRUSH_ERR_INVALID
    ctx.run_steps(13)
    ctx.append([models[1].desc])
    _run_to_end(ctx)
    _same(ctx.results(0), alone[0])
    _same(ctx.results(1), alone[1])
