"""The fused step schedule (a step's full update and the next step's half
step as one pass over the nodes, the next step's contact forces computed
beside the element forces) against separate passes: bit-identical states and
results, for a whole run, for runs issued in odd-sized pieces, for batches
whose crashes stop at different steps, and with time histories recorded."""
import numpy as np
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context

from .test_gpu_batch import _same

pytestmark = pytest.mark.gpu


def _run(desc, fused, steps=None):
    ctx = Context(desc)
    ctx.set_step_fusion(fused)
    if steps is None:
        r = ctx.run()
    else:
        ctx.run_begin()
        for n in steps:  # odd-sized issues: the state between calls is a whole step's
            ctx.run_steps(n)
        r = ctx.results()
    u, v = ctx.state()
    ctx.close()
    return r, u, v


def test_fused_run_equals_separate_passes():
    m = S.Model.build(S.plain_headon())
    a, ua, va = _run(m.desc, True)
    b, ub, vb = _run(m.desc, False)
    _same(a, b)
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)


def test_fused_steps_in_odd_issues_equal_separate_passes():
    m = S.Model.build(S.refined_headon(max_steps=400))
    a, ua, va = _run(m.desc, True, steps=[3, 7, 1, 29, 60, 13])
    b, ub, vb = _run(m.desc, False, steps=[113])
    _same(a, b)
    assert a.steps == 113
    assert np.array_equal(ua, ub) and np.array_equal(va, vb)


def test_fused_batch_equals_separate_passes():
    models = [S.Model.build(S.batch_headon(i)) for i in range(6)]
    models.append(S.Model.build(S.plain_headon(end_time=0.0301)))  # stops on a step that is not a multiple of 5
    ref = None
    for fused in (True, False):
        ctx = Context([m.desc for m in models])
        ctx.set_step_fusion(fused)
        rs = ctx.batch_run()
        ctx.close()
        if ref is None:
            ref = rs
        else:
            for x, y in zip(ref, rs):
                _same(x, y)


def test_fused_histories_equal_separate_passes():
    m = S.Model.build(S.plain_headon(end_time=0.05))
    recs = []
    for fused in (True, False):
        ctx = Context(m.desc)
        ctx.set_step_fusion(fused)
        ctx.history_config(7, 4096, [m.accelerometer(0), m.accelerometer(1)])
        ctx.run()
        recs.append(ctx.history())
        ctx.close()
    a, b = recs
    assert a["records"] == b["records"] > 10
    for k in ("time", "step", "parts", "nodes"):
        assert np.array_equal(a[k], b[k]), k


def test_every_launch_schedule_gives_the_same_bits():
    """Element-kernel schedules (persistent wave, block per chunk, wave on
    fewer SMs), the place of a fused step's next contact forces and contact
    lane counts, fixed by crush_set_tuning, all compute the same run; the
    automatic schedule trial (a context of 2,000,000+ hexahedra times the
    schedules on its first step graphs: eight copies of the mesh) does too."""
    m = S.Model.build(S.refined_headon(max_steps=240))
    out = []
    for tuning in ((32, 0, 0, 0), (8, 1, 1, 1), (4, 2, 0, 1), (16, 3, 0, 0)):
        ctx = Context(m.desc)
        ctx.set_tuning(*tuning)
        ctx.run_begin()
        ctx.run_steps(240)
        out.append((ctx.results(), ctx.state()))
        ctx.close()
    for r, (u, v) in out[1:]:
        _same(out[0][0], r)
        assert np.array_equal(out[0][1][0], u) and np.array_equal(out[0][1][1], v)
    ctx = Context([m.desc] * 8)
    ctx.run_begin()
    ctx.run_steps(240)  # the trial: 2 rounds x 6 candidates x 20 steps
    for k in range(8):
        _same(out[0][0], ctx.results(k))
    sched, step_ms = ctx.schedule()
    ctx.close()
    assert sched in (0, 1, 2, 3) and len(step_ms) == 6 and all(x > 0.0 for x in step_ms)
