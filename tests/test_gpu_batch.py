"""Batched contexts: many crash models advanced by one launch sequence per
step. Every slot must give exactly what the same model gives alone
(bit-identical f64 results), in any batch order and next to slots that stop
earlier or later; the only exception is added_mass_max, a diagnostic summed
with atomics, compared to 1e-12 relative."""
import numpy as np
import pytest

from crushrs_b200 import abi, scenarios as S
from crushrs_b200.engine import Context
from crushrs_b200.native import CrushError

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status
    assert a.steps == b.steps
    assert a.time == b.time
    assert a.eroded_elements == b.eroded_elements
    assert a.dt_min == b.dt_min
    assert a.added_mass_max == pytest.approx(b.added_mass_max, rel=1e-12, abs=0.0)
    assert a.n_vehicles == b.n_vehicles
    for k in range(a.n_vehicles):
        va, vb = a.vehicle[k], b.vehicle[k]
        assert va.mass == vb.mass
        assert list(va.delta_v) == list(vb.delta_v)
        assert list(va.velocity) == list(vb.velocity)
        assert va.crush == vb.crush


@pytest.fixture(scope="module")
def models():
    ms = [S.Model.build(S.batch_headon(i)) for i in range(4)]
    short = S.plain_headon(end_time=0.03)
    ms.append(S.Model.build(short))
    return ms


@pytest.fixture(scope="module")
def alone(models):
    out = []
    for m in models:
        ctx = Context(m.desc)
        out.append(ctx.run())
        ctx.close()
    return out


def test_batch_equals_alone(models, alone):
    ctx = Context([m.desc for m in models])
    assert ctx.n_slots == len(models)
    rs = ctx.batch_run()
    for r, a in zip(rs, alone):
        _same(r, a)


def test_batch_order_does_not_matter(models, alone):
    order = [4, 2, 0, 3, 1]
    ctx = Context([models[i].desc for i in order])
    rs = ctx.batch_run()
    for r, i in zip(rs, order):
        _same(r, alone[i])


def test_batch_stepwise_results(models, alone):
    """Driving the batch in chunks gives the same per-slot results, and a slot
    that has stopped stays frozen while others run on."""
    ctx = Context([models[4].desc, models[0].desc])
    ctx.run_begin()
    done = False
    frozen = None
    while not done:
        done = ctx.run_steps(200)
        r0 = ctx.results(0)
        if r0.steps == alone[4].steps:
            if frozen is None:
                frozen = r0
            else:
                _same(r0, frozen)
    _same(ctx.results(0), alone[4])
    _same(ctx.results(1), alone[0])


def test_batch_drop_in_forces_are_concatenated(models):
    """crush_compute_forces on a batch context: each slot's nodal forces equal
    the forces of its model alone."""
    rng = np.random.default_rng(7)
    ds = [models[1].desc, models[2].desc]
    us = [rng.normal(scale=1e-3, size=3 * d.n_nodes) for d in ds]
    ctx = Context(ds)
    f = np.zeros(3 * ctx.n_nodes)
    ctx.compute_forces(np.concatenate(us), f)
    off = 0
    for d, u in zip(ds, us):
        c1 = Context(d)
        f1 = np.zeros(3 * d.n_nodes)
        c1.compute_forces(u, f1)
        assert np.array_equal(f[off:off + 3 * d.n_nodes], f1)
        off += 3 * d.n_nodes


def test_batch_rejects_mixed_check_cadence(models):
    m = S.Model.build(S.batch_headon(5))
    m.settings.adaptive_check_steps = 7
    m.refresh()
    with pytest.raises(CrushError) as e:
        Context([models[0].desc, m.desc])
    assert e.value.status == abi.CRUSH_ERR_UNSUPPORTED


def test_large_batch_equals_alone():
    """1024 uneven crashes (about 3 M nodes) in one context: the contact
    gathers of heavy nodes (more than 16 reaction events) run beside the
    ordinary gather on a second stream and the step's kernels loop over
    their grids, so this covers the ordering between them that a handful of
    slots never stresses. Sampled slots must equal the same crash alone."""
    ms = [S.Model.build(S.batch_headon(i)) for i in range(1024)]
    ctx = Context([m.desc for m in ms])
    rs = ctx.batch_run()
    ctx.close()
    for i in (0, 85, 266, 363, 402, 1023):
        a = Context(ms[i].desc)
        r = a.run()
        a.close()
        _same(rs[i], r)


def test_solve_equals_alone(models, alone):
    """crush_batch_solve (set-up pipelined with the run: later groups join
    the open run) gives every model its alone results; 40 models so that
    several groups join, in an order that mixes long and short crashes."""
    from crushrs_b200.engine import solve_batch

    extra = [S.Model.build(S.batch_headon(i)) for i in range(4, 40)]
    order = list(models) + extra
    rs = solve_batch([m.desc for m in order])
    assert len(rs) == len(order)
    for r, a in zip(rs, alone):
        _same(r, a)
    for m, r in zip(extra[::7], rs[len(models)::7]):
        ctx = Context(m.desc)
        _same(r, ctx.run())
        ctx.close()
