"""The calibration client's host pieces (crushrs_b200/calibrate.py) and
the two-part vehicle chain pinned by the reference's documented numbers.

* The oracle's rigid-barrier run of the pulse-fitted Neon
  (Vehicle::dodge_neon_1996_pulse and barrier_model at 35 mph,
  src/vehicle.rs:541-566, :951) reproduces what the reference documents for
  its own simulation (src/vehicle.rs:536-540): rear-seat pulse delta-v
  17.64 m/s at 150 ms, peak -32.9 g, maximum crush 800 mm at 83 ms,
  restitution 0.13 - within 1 %, 5 %, 6 % / 3 ms and 0.01.
* Pulse integrals, the comparison and the objective (src/signal.rs:68-210,
  src/vehicle.rs:1047-1125), the rail-box unit cube (src/headon.rs:88-104)
  and the differential evolution (src/headon.rs:196-243) on CPU."""
import math

import numpy as np

from crushrs_b200 import calibrate as K, scenarios as S

from . import oracle_lib as O


def test_oracle_neon_pulse_barrier_known_answer():
    m = S.Model.build(S.barrier(S.neon_1996_pulse(), 35 * S.MPH))
    h = O.run_history(m.desc, 1, [m.accelerometer(0)], cap=20000, threads=8)
    assert h["records"] == h["results"].steps + 1
    p = K.Pulse.from_history(h["time"], h["nodes"][:, 0, 18]).filtered(60.0)
    speed = 35 * S.MPH
    dv = p.velocity(0.0)[-1]
    assert abs(p.time[-1] - 0.15) < 2e-4
    assert abs(-dv - 17.64) <= 0.01 * 17.64, dv
    assert abs(p.accel.min() / 9.81 - (-32.9)) <= 0.05 * 32.9
    x = p.displacement(speed)
    assert abs(x.max() - 0.800) <= 0.06 * 0.800
    assert abs(p.time[x.argmax()] - 0.083) <= 0.003
    v = p.velocity(speed)
    assert abs(max(-v.min() / speed, 0.0) - 0.13) <= 0.01


def test_pulse_integrals_and_objective():
    t = np.arange(0.0, 0.1 + 1e-12, 1e-4)
    a = -200.0 * np.sin(np.pi * t / 0.1)
    p = K.Pulse(t, a)
    v = p.velocity(10.0)
    assert abs(v[-1] - (10.0 - 400.0 * 0.1 / np.pi)) < 1e-4
    assert abs(p.displacement(10.0)[-1] - (1.0 - 200.0 * 0.01 / np.pi)) < 1e-4
    same = K.PulseComparison(p, p, 1000.0, 10.0)
    assert K.pulse_objective(same) == 0.0
    shifted = K.PulseComparison(p, K.Pulse(t, a - 9.81), 1000.0, 10.0)
    j = K.pulse_objective(shifted)
    # v error grows linearly to 9.81 x 0.1 s: RMS ~ 0.98 / sqrt(3), end 0.981, accel RMS 1 g
    expect = 0.981 / math.sqrt(3.0) + 0.5 * 0.981 + 0.1
    assert abs(j - expect) < 2e-3 * expect
    assert len(p.truncated(0.05).time) == 501


def test_rail_box_unit_cube_round_trip():
    size = (4.36, 1.71, 1.35)
    for u in ([0.0, 0.0, 0.0, 0.0], [1.0, 1.0, 0.2, 1.0], [0.3, 0.6, 0.4, 0.7]):
        rb = K.rail_box_from_unit(size, u)
        back = K.unit_from_rail_box(size, rb)
        assert np.allclose(back, u, atol=1e-12)
    width, (z0, z1), f = K.rail_box_from_unit(size, [0.5, 0.5, 0.5, 0.5])
    assert abs(width - 0.6 * 1.71) < 1e-12 and abs(f - 0.725) < 1e-12 and 0.0 <= z0 < z1 <= 1.35


def test_rng_is_the_reference_generator():
    r, x = K.Rng(), S.XorShift64Star(0x9E3779B97F4A7C15)
    assert [r.next_u64() for _ in range(5)] == [x.next_u64() for _ in range(5)]
    assert all(0 <= K.Rng(7).below(6) < 6 for _ in range(10))


def test_differential_evolution_descends():
    target = np.linspace(0.2, 0.8, 8)
    calls = []

    def evaluate_all(us):
        calls.append(len(us))
        return [(float(np.sum((np.asarray(u) - target) ** 2)),) for u in us]

    pop, scored, best, history = K.differential_evolution([0.5] * 8, 8, 10, 25, evaluate_all)
    assert calls == [10] * 26
    bests = [h[0] for h in history]
    assert all(b1 <= b0 for b0, b1 in zip(bests, bests[1:]))
    assert bests[-1] < 0.05 * bests[0]
    assert all(0.0 <= c <= 1.0 for u in pop for c in u)
    again = K.differential_evolution([0.5] * 8, 8, 10, 25, evaluate_all)
    assert again[0] == pop  # repeatable: the same generator and seed


def test_pulse_metrics_of_a_half_sine():
    # 10 m/s into a wall, a 100 ms half-sine deceleration of 200 m/s^2 peak:
    # v = 10 - (20/pi)(1 - cos(pi t / 0.1)), rebounding at 2.73 m/s
    t = np.arange(0.0, 0.1 + 1e-12, 1e-4)
    a = -200.0 * np.sin(np.pi * t / 0.1)
    m = K.PulseMetrics(K.Pulse(t, a), 1000.0, 10.0)
    v_end = 10.0 - 40.0 / np.pi
    assert abs(m.v_end - v_end) < 1e-4
    assert abs(m.restitution + v_end / 10.0) < 1e-5
    assert abs(m.peak_accel + 200.0) < 1e-3
    t_stop = 0.1 / np.pi * np.arccos(1.0 - np.pi / 2.0)
    crush = 10.0 * t_stop - (20.0 / np.pi) * (t_stop - 0.1 / np.pi * np.sin(np.pi * t_stop / 0.1))
    assert abs(m.t_max_crush - t_stop) <= 1e-4 and abs(m.max_crush - crush) < 1e-5
    # mean force over the loading phase = the initial kinetic energy / max crush
    e = 0.5 * 1000.0 * 10.0 ** 2
    assert abs(m.mean_force(0.0, m.max_crush) - e / m.max_crush) < 2e-3 * e / m.max_crush
    assert m.mean_force(5.0, 6.0) is None


def test_table_vehicle_is_the_preset():
    assert bytes(S.neon_1996_pulse()) == bytes(S.neon_1996_pulse(table=True).spec())
    tv = S.neon_1996_pulse(table=True)
    mat = tv.spec().material
    assert mat.n_curve == 7 and mat.has_densification  # 7 table knots, the lock-up knot added by the material
    assert abs(mat.curve[1][1] - 135e3 / (1.71 * 1.35)) < 1e-9 * mat.curve[1][1]


TUNED = {  # src/vehicle.rs:614-644: tuned curves and what the reference reports for them at 35 mph, 0.3 m elements
    "neon": (K.CurveVehicle(1354.0, (4.36, 1.71, 1.35), 16.73e3, 2.930e5, 23.1e6), 1269e3, 0.538, 0.112),
    "silverado": (K.CurveVehicle(2622.0, (5.85, 2.03, 1.87), 51.21e3, 5.592e5, 27.8e6), 2563e3, 0.540, 0.119),
}


def test_oracle_barrier_metrics_known_answers():
    """The oracle's rigid-barrier runs of the tuned Neon and Silverado
    reproduce the reference's documented calibration results
    (src/vehicle.rs:614-644: KW400 1269 and 2563 N/mm, maximum crush 538
    and 540 mm, restitution 0.112 and 0.119) within 4 %, 1 % and 0.01."""
    for name, (v, kw, crush, e) in TUNED.items():
        m = S.Model.build(S.barrier(v.spec(), 35 * S.MPH, end_time=0.14))
        h = O.run_history(m.desc, 2, [], cap=20000, threads=8)
        met = K.BarrierMetrics(K.part_series(h["time"], h["parts"], K.vehicle_parts(m)))
        assert abs(met.kw400 - kw) <= 0.04 * kw, (name, met.kw400)
        assert abs(met.max_crush - crush) <= 0.01 * crush, (name, met.max_crush)
        assert abs(met.restitution - e) <= 0.01, (name, met.restitution)


def test_barrier_targets_from_the_curve():
    v = TUNED["neon"][0]
    t = K.BarrierTargets.from_vehicle(v, 0.12)
    # KW400 = k + 2 (0.375) / (0.16 - 0.000625) F_y; 0.5 k C^2 + F_y C = 0.5 m v^2
    assert abs(t.kw400 - (2.930e5 + 2 * 0.375 / (0.16 - 0.000625) * 16.73e3)) < 1e-6 * t.kw400
    e = 0.5 * 1354.0 * (35 * S.MPH) ** 2
    assert abs(0.5 * 2.930e5 * t.max_crush ** 2 + 16.73e3 * t.max_crush - e) < 1e-6 * e
