"""The calibration client on the GPU (crushrs_b200/calibrate.py).

* The device's rear-seat pulse of the pulse-fitted Neon into the rigid
  barrier at 35 mph (histories recorded every step on the device, body
  frame) against the oracle's (delta-v within 0.5 %, velocity history within
  1 % of the impact speed) and the reference's documented 17.64 m/s
  (src/vehicle.rs:536-540, within 1 %).
* calibrate_rail_boxes (src/headon.rs:147-250) against pulses simulated with
  the presets' own rail boxes: every generation runs as one batched context,
  the best objective never rises, and the fitted pair run alone gives the
  recorded objective exactly (batched slots are bit-identical to single
  runs)."""
import pytest

from crushrs_b200 import calibrate as K, scenarios as S
from crushrs_b200.engine import Context

from . import oracle_lib as O

pytestmark = pytest.mark.gpu


def test_device_pulse_matches_oracle_and_reference():
    m = S.Model.build(S.barrier(S.neon_1996_pulse(), 35 * S.MPH))
    ctx = Context(m.desc)
    ctx.history_config(1, 20000, [m.accelerometer(0)])
    r = ctx.run()
    h = ctx.history()
    ctx.close()
    assert h["records"] == r.steps + 1
    p = K.Pulse.from_history(h["time"], h["nodes"][:, 0, 18]).filtered(60.0)
    ho = O.run_history(m.desc, 1, [m.accelerometer(0)], cap=20000, threads=8)
    po = K.Pulse.from_history(ho["time"], ho["nodes"][:, 0, 18]).filtered(60.0)
    speed = 35 * S.MPH
    dv, dvo = p.velocity(0.0)[-1], po.velocity(0.0)[-1]
    assert abs(dv - dvo) <= 5e-3 * abs(dvo), (dv, dvo)
    n = min(len(p.time), len(po.time))
    assert abs(p.velocity(speed)[:n] - po.velocity(speed)[:n]).max() <= 0.01 * speed
    assert abs(-dv - 17.64) <= 0.01 * 17.64


def _without_rail_box(v):
    w = type(v).from_buffer_copy(v)
    w.has_rail_box = 0
    return w


def test_rail_box_calibration_batches():
    setup = K.HeadOn(30.14 * S.MPH, 30.14 * S.MPH)
    a, b = S.lincoln_navigator_1999(), S.neon_1996_pulse()
    (pa, pb), = setup.run_batch([(a, b)])
    fit = K.calibrate_rail_boxes(_without_rail_box(a), _without_rail_box(b), setup, pa, pb, population=6, generations=2)
    assert fit.evaluations == 18
    bests = [x[0] for x in fit.history]
    assert all(b1 <= b0 for b0, b1 in zip(bests, bests[1:]))
    assert fit.objective == bests[-1] and fit.objective > 0.0
    (qa, qb), = setup.run_batch([(fit.a, fit.b)])
    meas_a = pa.filtered(60.0).resampled(K.PULSE_DT).truncated(setup.end_time)
    meas_b = pb.filtered(60.0).resampled(K.PULSE_DT).truncated(setup.end_time)
    j = K.pulse_objective(K.PulseComparison(meas_a, qa, a.mass, setup.speed_a)) + \
        K.pulse_objective(K.PulseComparison(meas_b, qb, b.mass, setup.speed_b))
    assert j == fit.objective


def test_pulse_calibration_batches_each_round():
    """calibrate_pulse (src/vehicle.rs:1144-1256) against the preset Neon's
    own barrier pulse, starting from a softer, weaker vehicle: each round's
    18 probes run as one batched context, the best objective never rises and
    improves on the start, and the fitted vehicle run alone reproduces the
    recorded objective exactly."""
    speed = 35 * S.MPH
    target = S.neon_1996_pulse(table=True)
    (measured,) = K.run_barrier_pulses([target.spec()], speed)
    start = target.copy()
    start.modulus *= 1.3
    start.table = [(x, f * 0.8) for x, f in start.table]
    tuned, cmp, history = K.calibrate_pulse(start, measured, speed, rounds=2)
    assert len(history) == 3
    assert all(b <= a for a, b in zip(history, history[1:]))
    assert history[-1] < history[0]
    (again,) = K.run_barrier_pulses([tuned.spec()], speed)
    meas = measured.filtered(60.0).resampled(K.PULSE_DT).truncated(K.PULSE_END)
    assert K.pulse_objective(K.PulseComparison(meas, again, target.mass, speed)) == history[-1]


def test_barrier_metrics_and_calibration_batches():
    """The barrier runs of the tuned Neon and Silverado as one batched
    context: their metrics from device part histories against the oracle's
    (KW 1 %, crush 0.5 %, restitution 0.005); then calibrate (src/vehicle.rs:1013)
    both at once towards the NHTSA targets the reference tuned them to
    (src/vehicle.rs:614-644): each iteration is one batch whose metrics are
    exactly those of the same vehicles run as a batch by hand."""
    from .test_calibrate import TUNED

    vs = [TUNED["neon"][0], TUNED["silverado"][0]]
    targets = [K.BarrierTargets(1251e3, 0.527, 0.112, 35 * S.MPH), K.BarrierTargets(2550e3, 0.513, 0.119, 35 * S.MPH)]
    mets = K.run_barrier_metrics(vs, targets, S.TUNED_ELEMENT_SIZE)
    for v, met in zip(vs, mets):
        m = S.Model.build(S.barrier(v.spec(), 35 * S.MPH, end_time=0.14))
        h = O.run_history(m.desc, 2, [], cap=20000, threads=8)
        ref = K.BarrierMetrics(K.part_series(h["time"], h["parts"], K.vehicle_parts(m)))
        assert abs(met.kw400 - ref.kw400) <= 0.01 * ref.kw400
        assert abs(met.max_crush - ref.max_crush) <= 0.005 * ref.max_crush
        assert abs(met.restitution - ref.restitution) <= 0.005
    first = K.calibrate(vs, targets, iterations=1)  # the same batch as above, then one curve update
    for (tuned, met), before, v in zip(first, mets, vs):
        assert (met.kw400, met.max_crush, met.restitution) == (before.kw400, before.max_crush, before.restitution)
        assert (tuned.yield_force, tuned.stiffness) != (v.yield_force, v.stiffness)
    out = K.calibrate(vs, targets, iterations=2)
    assert len(out) == 2 and all(m is not None and m.max_crush > 0.0 for _, m in out)
