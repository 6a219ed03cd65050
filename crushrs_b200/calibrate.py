"""Calibration drivers as clients of the batched engine.

The reference fits vehicles to measured crash pulses by running many
independent impacts (src/headon.rs:147-250 calibrate_rail_boxes: a
differential evolution whose generations are independent runs). Here every
generation's trials run as ONE batched context on the GPU, each trial a crash
slot recording its two rear-seat accelerometers every step on the device;
the pulses are then taken from the device histories (src/signal.rs:129-146
Pulse::from_history: local-x acceleration resampled to 0.1 ms, CFC 60).

Pieces restated from the reference: Pulse and its integrals
(src/signal.rs:68-210), PulseComparison and pulse_objective
(src/vehicle.rs:1047-1135), the rail-box unit-cube parameterisation and the
xorshift64* generator (src/headon.rs:88-131), and the synchronous
rand/1/bin differential evolution of calibrate_rail_boxes
(src/headon.rs:147-250).
"""
import math

import numpy as np

from . import scenarios as S
from .engine import Context
from .pulse import cfc_filter, resample

PULSE_DT = S.PULSE_DT
PULSE_END = S.PULSE_END
G = 9.81


def integrate(t, y, y0):
    """Cumulative trapezoidal integral from y0 (src/signal.rs:68-78)."""
    out = np.empty(len(y))
    acc = y0
    out[0] = acc
    for i in range(1, len(y)):
        acc += 0.5 * (y[i] + y[i - 1]) * (t[i] - t[i - 1])
        out[i] = acc
    return out


class Pulse:
    """A uniformly sampled acceleration history (m/s^2), t = 0 at first contact."""

    def __init__(self, time, accel):
        self.time = np.asarray(time, dtype=np.float64)
        self.accel = np.asarray(accel, dtype=np.float64)

    def dt(self):
        n = len(self.time)
        return (self.time[-1] - self.time[0]) / (n - 1) if n > 1 else 0.0

    @classmethod
    def from_history(cls, time, local_ax, dt=PULSE_DT):
        """Pulse::from_history: the accelerometer's local-x acceleration
        resampled onto 0, dt, ... up to the last record."""
        if len(time) < 4:
            raise ValueError("accelerometer history is empty")
        t, a = resample(time, local_ax, 0.0, dt, time[-1])
        return cls(t, a)

    def filtered(self, cfc=60.0):
        return Pulse(self.time, cfc_filter(self.accel, self.dt(), cfc))

    def resampled(self, dt):
        t, a = resample(self.time, self.accel, self.time[0], dt, self.time[-1])
        return Pulse(t, a)

    def truncated(self, t_end):
        n = int(np.count_nonzero(self.time <= t_end + 1e-12)) if len(self.time) else 0
        # take_while semantics on an ascending grid
        return Pulse(self.time[:n], self.accel[:n])

    def negated(self):
        return Pulse(self.time, -self.accel)

    def velocity(self, v0):
        return integrate(self.time, self.accel, v0)

    def displacement(self, v0):
        return integrate(self.time, self.velocity(v0), 0.0)


class PulseMetrics:
    """Barrier-test summary of a pulse (PulseMetrics::new,
    src/signal.rs:212-236): maximum dynamic crush and its time, end
    velocity, restitution, peak deceleration, and the loading phase's
    force-crush samples F = -m a."""

    def __init__(self, p, mass, v0):
        v = p.velocity(v0)
        x = p.displacement(v0)
        i_max, max_crush = 0, 0.0
        for i, xi in enumerate(x):
            if xi > max_crush:
                i_max, max_crush = i, xi
        self.t_max_crush = p.time[i_max]
        self.max_crush = max_crush
        self.v_end = v[-1]
        self.restitution = max(-min(v.min(), np.inf) / v0, 0.0)
        self.peak_accel = min(0.0, float(p.accel.min()))
        self.force_crush = [(x[i], -mass * p.accel[i]) for i in range(i_max + 1)]

    def mean_force(self, x0, x1):
        """Mean force over the crush window [x0, x1] of the loading phase
        (src/signal.rs:275-290), None when fewer than two samples span it."""
        pts = [q for q in self.force_crush if x0 <= q[0] <= x1]
        if len(pts) < 2:
            return None
        e = 0.0
        for (c0, f0), (c1, f1) in zip(pts, pts[1:]):
            e += 0.5 * (f0 + f1) * (c1 - c0)
        span = pts[-1][0] - pts[0][0]
        return e / span if span > 0.0 else None


class PulseComparison:
    """Measured vs simulated pulse on the measured grid
    (PulseComparison::new, src/vehicle.rs:1059-1078)."""

    def __init__(self, meas, sim, mass, speed):
        t_end = min(meas.time[-1], sim.time[-1])
        m = meas.truncated(t_end)
        s = sim.resampled(m.dt()).truncated(t_end) if abs(sim.dt() - m.dt()) > 1e-9 * m.dt() else sim.truncated(t_end)
        n = min(len(m.time), len(s.time))
        self.mass, self.speed = mass, speed
        self.time = m.time[:n]
        self.a_meas, self.a_sim = m.accel[:n], s.accel[:n]
        self.v_meas, self.v_sim = m.velocity(speed)[:n], s.velocity(speed)[:n]
        self.x_meas, self.x_sim = m.displacement(speed)[:n], s.displacement(speed)[:n]

    def rms_accel_error(self):
        return math.sqrt(float(np.sum((self.a_meas - self.a_sim) ** 2)) / len(self.a_meas))


def pulse_objective(cmp):
    """Velocity-history RMS error + 0.5 end-velocity error + 0.1 x CFC 60
    acceleration RMS error in g (src/vehicle.rs:1120-1125)."""
    n = len(cmp.time)
    v_rms = math.sqrt(float(np.sum((cmp.v_meas - cmp.v_sim) ** 2)) / n)
    v_end = abs(cmp.v_sim[-1] - cmp.v_meas[-1])
    return v_rms + 0.5 * v_end + 0.1 * cmp.rms_accel_error() / G


class Rng(S.XorShift64Star):
    """The calibrations' xorshift64* (src/headon.rs:112-131), so they are
    repeatable; below(n) draws an index in [0, n)."""

    def __init__(self, seed=0x9E3779B97F4A7C15):
        super().__init__(seed)

    def below(self, n):
        return int(self.uniform() * n) % n


def rail_box_from_unit(size, u):
    """src/headon.rs:88-97: [width / vehicle width, z-centre / height,
    z-extent / height, force fraction] in the unit cube -> (width, (z0, z1),
    force fraction): 25-95 % of the width, centred at 15-50 % of the height,
    15-60 % of the height tall, 50-95 % of the force."""
    w, hgt = size[1], size[2]
    width = (0.25 + 0.7 * u[0]) * w
    zc = (0.15 + 0.35 * u[1]) * hgt
    dz = (0.15 + 0.45 * u[2]) * hgt
    return (width, (max(zc - 0.5 * dz, 0.0), min(zc + 0.5 * dz, hgt)), 0.5 + 0.45 * u[3])


def unit_from_rail_box(size, rb):
    """src/headon.rs:99-104, the inverse, clamped to the unit cube."""
    w, hgt = size[1], size[2]
    width, (z0, z1), f = rb
    zc = 0.5 * (z0 + z1) / hgt
    dz = (z1 - z0) / hgt
    clamp = lambda x: min(max(x, 0.0), 1.0)
    return [clamp((width / w - 0.25) / 0.7), clamp((zc - 0.15) / 0.35), clamp((dz - 0.15) / 0.45), clamp((f - 0.5) / 0.45)]


def _rail_box_of(spec):
    if not spec.has_rail_box:
        return None
    return (spec.rail_box_width, (spec.rail_box_z[0], spec.rail_box_z[1]), spec.rail_box_force_fraction)


def with_rail_box(spec, rb):
    v = type(spec).from_buffer_copy(spec)
    v.has_rail_box = 1
    v.rail_box_width = rb[0]
    v.rail_box_z[0], v.rail_box_z[1] = rb[1]
    v.rail_box_force_fraction = rb[2]
    return v


class HeadOn:
    """HeadOn (src/headon.rs:17-86): A heads +x at speed_a, B heads -x at
    speed_b (the struct's own speeds; B's pulse is negated so each vehicle's
    forward direction is positive)."""

    def __init__(self, speed_a, speed_b, offset=0.0, clearance=0.15, element_size=S.TUNED_ELEMENT_SIZE, end_time=PULSE_END,
                 max_records=20000):
        self.max_records = max_records  # history records kept per crash (every step up to end_time)
        self.speed_a, self.speed_b = speed_a, speed_b
        self.offset, self.clearance = offset, clearance
        self.element_size, self.end_time = element_size, end_time

    def build(self, a, b):
        return S.Model.build(S.scenario(a, b, self.speed_a, self.speed_b, offset=self.offset, clearance=self.clearance,
                                        element_size=self.element_size, end_time=self.end_time))

    def run_batch(self, pairs, device=0):
        """Run every (a, b) pair as one slot of one batched context,
        recording both rear-seat accelerometers every step on the device;
        returns per pair (pulse A, pulse B), CFC 60, forward positive."""
        models = [self.build(a, b) for a, b in pairs]
        ctx = Context([m.desc for m in models], device=device)
        for k, m in enumerate(models):
            ctx.history_config(1, self.max_records, [m.accelerometer(0), m.accelerometer(1)], slot=k)
        ctx.batch_run()
        out = []
        for k in range(len(models)):
            h = ctx.history(slot=k)
            if h["records"] > self.max_records:
                raise RuntimeError(f"slot {k}: {h['records']} history records, more than max_records {self.max_records}")
            pa = Pulse.from_history(h["time"], h["nodes"][:, 0, 18]).filtered(60.0)
            pb = Pulse.from_history(h["time"], h["nodes"][:, 1, 18]).negated().filtered(60.0)
            out.append((pa, pb))
        ctx.close()
        return out


def differential_evolution(seed, dims, population, generations, evaluate_all, rng=None, log=None):
    """The synchronous rand/1/bin differential evolution of
    calibrate_rail_boxes (src/headon.rs:196-243) in the unit cube:
    population max(population, 4) seeded with `seed` and uniform draws of the
    xorshift64* generator (seed 0x9E3779B97F4A7C15), F 0.7, CR 0.9, trial
    coordinates reflected into [0, 1], a trial replacing its parent when its
    score is not worse. evaluate_all(list of members) -> list of tuples whose
    first item is the score; a generation's members are evaluated together.
    Returns (population, scores, index of the best, per generation (best,
    mean) score)."""
    rng = rng or Rng(0x9E3779B97F4A7C15)
    npop = max(population, 4)
    pop = [list(seed)]
    while len(pop) < npop:
        pop.append([rng.uniform() for _ in range(dims)])
    scored = evaluate_all(pop)
    best_index = lambda sc: min(range(len(sc)), key=lambda i: sc[i][0])
    best = best_index(scored)
    history = [(scored[best][0], sum(x[0] for x in scored) / npop)]
    if log:
        log(f"initial population of {npop}: best J {scored[best][0]:.3f}")
    f_weight, cr = 0.7, 0.9
    for gen in range(generations):
        trials = []
        for i in range(npop):
            while True:
                r = [rng.below(npop), rng.below(npop), rng.below(npop)]
                if r[0] != i and r[1] != i and r[2] != i and r[0] != r[1] and r[0] != r[2] and r[1] != r[2]:
                    break
            r1, r2, r3 = r
            j_rand = rng.below(dims)
            trial = []
            for j in range(dims):
                if j == j_rand or rng.uniform() < cr:
                    v = pop[r1][j] + f_weight * (pop[r2][j] - pop[r3][j])
                    v = -v if v < 0.0 else (2.0 - v if v > 1.0 else v)  # reflect into the unit cube
                    trial.append(min(max(v, 0.0), 1.0))
                else:
                    trial.append(pop[i][j])
            trials.append(trial)
        results = evaluate_all(trials)
        for i, (trial, sc) in enumerate(zip(trials, results)):
            if sc[0] <= scored[i][0]:
                pop[i] = trial
                scored[i] = sc
        best = best_index(scored)
        history.append((scored[best][0], sum(x[0] for x in scored) / npop))
        if log:
            log(f"generation {gen}: best J {scored[best][0]:.3f}, mean {history[-1][1]:.3f}")
    return pop, scored, best, history


class RailBoxFit:
    def __init__(self, a, b, objective, cmp_a, cmp_b, evaluations, history):
        self.a, self.b, self.objective = a, b, objective
        self.cmp_a, self.cmp_b = cmp_a, cmp_b
        self.evaluations = evaluations
        self.history = history  # per generation: (best J, mean J)


def calibrate_rail_boxes(a, b, setup, measured_a, measured_b, population, generations, device=0, log=None):
    """calibrate_rail_boxes (src/headon.rs:147-250): fit the rail boxes of
    both vehicles (width, height band, force fraction each: 8 parameters in
    the unit cube, seeded with the current boxes) so the two rear-seat
    pulses of `setup` match the measured ones, by synchronous rand/1/bin
    differential evolution (F 0.7, CR 0.9, reflection into the cube). Each
    generation's trials run together as one batched GPU context."""
    meas_a = measured_a.filtered(60.0).resampled(PULSE_DT).truncated(setup.end_time)
    meas_b = measured_b.filtered(60.0).resampled(PULSE_DT).truncated(setup.end_time)

    def base(v):
        if _rail_box_of(v) is None:
            return with_rail_box(v, (0.5 * v.size[1], (0.2 * v.size[2], 0.6 * v.size[2]), 0.7))
        return v

    a0, b0 = base(a), base(b)
    size_a, size_b = tuple(a0.size), tuple(b0.size)
    dims = 8

    def with_(u):
        return with_rail_box(a0, rail_box_from_unit(size_a, u[:4])), with_rail_box(b0, rail_box_from_unit(size_b, u[4:]))

    evaluations = [0]

    def evaluate_all(us):
        pulses = setup.run_batch([with_(u) for u in us], device=device)
        res = []
        for pa, pb in pulses:
            ca = PulseComparison(meas_a, pa, a.mass, setup.speed_a)
            cb = PulseComparison(meas_b, pb, b.mass, setup.speed_b)
            res.append((pulse_objective(ca) + pulse_objective(cb), ca, cb))
        evaluations[0] += len(us)
        return res

    seed = unit_from_rail_box(size_a, _rail_box_of(a0)) + unit_from_rail_box(size_b, _rail_box_of(b0))
    pop, scored, best, history = differential_evolution(seed, dims, population, generations, evaluate_all, log=log)
    va, vb = with_(pop[best])
    objective, ca, cb = scored[best]
    return RailBoxFit(va, vb, objective, ca, cb, evaluations[0], history)


def run_barrier_pulses(vehicles, speed, element_size=S.TUNED_ELEMENT_SIZE, end_time=PULSE_END, max_records=20000, device=0):
    """run_barrier_pulse (src/vehicle.rs:1106-1115) for every vehicle spec,
    all as one batched context: the barrier at `speed`, the rear-seat
    accelerometer recorded every step on the device; returns the CFC 60
    pulses."""
    models = [S.Model.build(S.barrier(v, speed, element_size=element_size, end_time=end_time)) for v in vehicles]
    ctx = Context([m.desc for m in models], device=device)
    for k, m in enumerate(models):
        ctx.history_config(1, max_records, [m.accelerometer(0)], slot=k)
    ctx.batch_run()
    out = []
    for k in range(len(models)):
        h = ctx.history(slot=k)
        if h["records"] > max_records:
            raise RuntimeError(f"slot {k}: {h['records']} history records, more than max_records {max_records}")
        out.append(Pulse.from_history(h["time"], h["nodes"][:, 0, 18]).filtered(60.0))
    ctx.close()
    return out


N_KNOTS = 7  # MAX_KNOTS - 1: one knot is the densification


def calibrate_pulse(v, measured, speed, element_size=S.TUNED_ELEMENT_SIZE, rounds=8, device=0, log=None):
    """calibrate_pulse (src/vehicle.rs:1144-1256): fit a TableVehicle's
    force-crush table (7 knots over the measured dynamic crush, initialised
    from the measured force-crush curve when the vehicle's table has another
    length), the crush zone's modulus and the body's modulus so its
    rigid-barrier rear-seat pulse matches `measured`: a pattern search on the
    logs of the 9 parameters, each round's up-and-down probes (the table kept
    non-decreasing from its second knot) run as ONE batched context, the best
    probe taken when it improves, the step halved when none does, stopping
    below 0.04. Returns (vehicle, comparison, per-round best objective)."""
    meas = measured.filtered(60.0).resampled(PULSE_DT).truncated(PULSE_END)
    mm = PulseMetrics(meas, v.mass, speed)
    x_max = mm.max_crush
    spacing = x_max * 0.95 / (N_KNOTS - 1)
    knots = [i * spacing for i in range(N_KNOTS)]
    w = 0.5 * spacing
    tuned = v.copy()
    if len(tuned.table) != N_KNOTS:
        targets = []
        for x in knots:
            f = mm.mean_force(max(x - w, 0.0), min(x + w, x_max))
            targets.append(max(f if f is not None else 0.0, 1e3))
        for i in range(2, len(targets)):
            targets[i] = max(targets[i], targets[i - 1])
        tuned.table = list(zip(knots, targets))

    def evaluate_all(cands):
        pulses = run_barrier_pulses([c.spec() for c in cands], speed, element_size, device=device)
        return [PulseComparison(meas, p, v.mass, speed) for p in pulses]

    def candidate(base, param, factor):
        cand = base.copy()
        if param < N_KNOTS:
            t = [list(k) for k in cand.table]
            t[param][1] *= factor
            for i in range(2, len(t)):
                t[i][1] = max(t[i][1], t[i - 1][1])
            t = [tuple(k) for k in t]
            if t == base.table:
                return None
            cand.table = t
        elif param == N_KNOTS:
            cand.modulus = min(max(cand.modulus * factor, 2e6), 500e6)
        else:
            cand.body_modulus = min(max(cand.body_modulus * factor, 2e7), 5e9)
        return cand

    best_cmp = evaluate_all([tuned])[0]
    best_j = pulse_objective(best_cmp)
    history = [best_j]
    if log:
        log(f"start: J {best_j:.3f}")
    step = 0.3
    for rnd in range(rounds):
        probes = []
        for param in range(N_KNOTS + 2):
            for d in (1.0, -1.0):
                c = candidate(tuned, param, math.exp(d * step))
                if c is not None:
                    probes.append((param, d, c))
        cmps = evaluate_all([c for _, _, c in probes])
        js = [pulse_objective(c) for c in cmps]
        i = min(range(len(js)), key=lambda k: js[k])
        if js[i] < best_j:
            best_j, tuned, best_cmp = js[i], probes[i][2], cmps[i]
            if log:
                log(f"round {rnd} p{probes[i][0]}{'+' if probes[i][1] > 0 else '-'}: J {best_j:.3f}")
        else:
            step *= 0.5
            if log:
                log(f"round {rnd}: no improvement, step {step:.3f}")
            if step < 0.04:
                history.append(best_j)
                break
        history.append(best_j)
    return tuned, best_cmp, history


# ---------------- rigid-barrier calibration (src/vehicle.rs:985-1041) ----------------

def kw_window(yield_force, stiffness, window):
    """CrushCurve::kw_window (src/vehicle.rs:61-64): energy-equivalent
    stiffness of the bilinear curve F = F_y + k C over a crush window."""
    w0, w1 = window
    return stiffness + 2.0 * (w1 - w0) / (w1 * w1 - w0 * w0) * yield_force


def crush_for_energy(yield_force, stiffness, energy):
    """CrushCurve::crush_for_energy (src/vehicle.rs:67-72)."""
    a, b = 0.5 * stiffness, yield_force
    return (-b + math.sqrt(b * b + 4.0 * a * energy)) / (2.0 * a)


class CurveVehicle:
    """A homogeneous honeycomb block with the bilinear frontal curve
    F = F_y + k C (Vehicle::crush_material with the whole block as crush
    zone, src/vehicle.rs:478-490): what the barrier calibration moves."""

    def __init__(self, mass, size, yield_force, stiffness, modulus, transverse=S.TRANSVERSE_FACTOR):
        self.mass, self.size = mass, tuple(size)
        self.yield_force, self.stiffness, self.modulus = yield_force, stiffness, modulus
        self.transverse = transverse

    def copy(self):
        return CurveVehicle(self.mass, self.size, self.yield_force, self.stiffness, self.modulus, self.transverse)

    def spec(self):
        area = self.size[1] * self.size[2]
        density = self.mass / (self.size[0] * self.size[1] * self.size[2])
        mat = S.honeycomb(self.modulus, density, self.yield_force / area, self.stiffness * self.size[0] / area,
                          transverse=self.transverse)
        return S.vehicle(self.mass, self.size, mat, contact_modulus=self.modulus)


class BarrierTargets:
    """BarrierTargets (src/vehicle.rs:985-1004): KW over the window, the
    crush that absorbs the impact energy on the curve, restitution."""

    def __init__(self, kw400, max_crush, restitution, speed, window=(0.025, 0.4)):
        self.kw400, self.max_crush, self.restitution, self.speed, self.window = kw400, max_crush, restitution, speed, window

    @classmethod
    def from_curve(cls, v, speed, window, restitution):
        crush = crush_for_energy(v.yield_force, v.stiffness, 0.5 * v.mass * speed * speed)
        return cls(kw_window(v.yield_force, v.stiffness, window), crush, restitution, speed, window)

    @classmethod
    def from_vehicle(cls, v, restitution):
        return cls.from_curve(v, 35.0 * S.MPH, (0.025, 0.4), restitution)


class BarrierMetrics:
    """barrier_metrics_window (src/vehicle.rs:887-948) from a series of
    (t, mass, mean velocity, mean displacement) along the impact axis of the
    vehicle's parts: force -m dv/dt (central differences, smoothed 1-2-1),
    contact at 2 % of the peak, crush from there, KW over the window from
    the loading curve's energy, mean force, restitution and delta-v."""

    def __init__(self, series, window=(0.025, 0.4)):
        n = len(series)
        if n <= 3:
            raise ValueError("no history")
        v0 = series[0][2]
        sign = math.copysign(1.0, v0)
        force = [0.0] * n
        for i in range(1, n - 1):
            t0, m, v_prev, _ = series[i - 1]
            t2, _, v_next, _ = series[i + 1]
            force[i] = -sign * m * (v_next - v_prev) / (t2 - t0)
        force = [force[i] if i == 0 or i == n - 1 else (force[i - 1] + 2.0 * force[i] + force[i + 1]) / 4.0 for i in range(n)]
        peak = max([0.0] + force)
        contact = next((i for i, f in enumerate(force) if f > 0.02 * peak), 0)
        x_contact = series[contact][3]
        crush = [sign * (s[3] - x_contact) for s in series]
        i_max = max(range(n), key=lambda i: (crush[i], i))  # the last maximum
        self.max_crush = crush[i_max]
        self.curve = [(crush[i], force[i]) for i in range(contact, i_max + 1)]

        def energy_at(d):
            e = 0.0
            for (c0, f0), (c1, f1) in zip(self.curve, self.curve[1:]):
                if c1 <= c0:
                    continue
                if c1 <= d:
                    e += 0.5 * (f0 + f1) * (c1 - c0)
                elif c0 < d:
                    f_d = f0 + (f1 - f0) * (d - c0) / (c1 - c0)
                    e += 0.5 * (f0 + f_d) * (d - c0)
                    break
                else:
                    break
            return e

        w0, w1 = window
        self.kw400 = 2.0 * (energy_at(w1) - energy_at(w0)) / (w1 * w1 - w0 * w0)
        self.mean_force = energy_at(self.max_crush) / self.max_crush if self.max_crush > 0.0 else 0.0
        self.peak_force = peak
        v_end = series[-1][2]
        self.restitution = -v_end / v0
        self.delta_v = v_end - v0


def part_series(time, parts, vehicle_parts, axis=0):
    """(t, m, mean v, mean u) of the vehicle's parts from device part-state
    records (values mass, v 3, u 3, ...; the parts of a two-part vehicle
    combined, src/vehicle.rs:892-907)."""
    out = []
    for r, t in enumerate(time):
        m = mv = mu = 0.0
        for q in vehicle_parts:
            s = parts[r, q]
            m += s[0]
            mv += s[0] * s[1 + axis]
            mu += s[0] * s[4 + axis]
        out.append((t, m, mv / m, mu / m))
    return out


def vehicle_parts(model, vehicle=0):
    """Parts whose elements all lie on the vehicle's nodes."""
    nodes, _, _ = model.vehicle(vehicle)
    inside = np.zeros(model.n_nodes, bool)
    inside[nodes] = True
    part = model.hex_part()
    mine = inside[model.hexes()].all(axis=1)
    return sorted(int(p) for p in np.unique(part[mine]) if np.all(mine[part == p]))


def run_barrier_metrics(vehicles, targets, element_size, end_time=0.14, history_steps=2, max_records=20000, device=0):
    """The barrier run of every vehicle at its target speed as one batched
    context, part states recorded every `history_steps` steps on the
    device (barrier_model's history_steps 2); returns BarrierMetrics each."""
    models = [S.Model.build(S.barrier(v.spec(), t.speed, element_size=element_size, end_time=end_time)) for v, t in zip(vehicles, targets)]
    ctx = Context([m.desc for m in models], device=device)
    for k in range(len(models)):
        ctx.history_config(history_steps, max_records, [], slot=k)
    ctx.batch_run()
    out = []
    for k, (m, t) in enumerate(zip(models, targets)):
        h = ctx.history(slot=k)
        if h["records"] > max_records:
            raise RuntimeError(f"slot {k}: {h['records']} history records, more than max_records {max_records}")
        out.append(BarrierMetrics(part_series(h["time"], h["parts"], vehicle_parts(m)), t.window))
    ctx.close()
    return out


def calibrate(vehicles, targets, element_size=S.TUNED_ELEMENT_SIZE, iterations=8, device=0, log=None):
    """calibrate (src/vehicle.rs:1013-1041) for several vehicles at once:
    each iteration runs every vehicle still unconverged as one batched
    context, then moves its curve by the damped log-space secant on the KW,
    crush and restitution ratios (yield force and stiffness; the modulus once
    KW and crush are within 15 %), until all three are within 2 %, 2 % and
    10 %. Returns [(vehicle, metrics)]."""
    tuned = [v.copy() for v in vehicles]
    last = [None] * len(tuned)
    active = list(range(len(tuned)))
    for it in range(iterations):
        if not active:
            break
        ms = run_barrier_metrics([tuned[i] for i in active], [targets[i] for i in active], element_size, device=device)
        still = []
        for i, m in zip(active, ms):
            tg, v = targets[i], tuned[i]
            if log:
                log(f"vehicle {i} it {it}: KW {m.kw400 / 1e3:.0f}/{tg.kw400 / 1e3:.0f} N/mm, crush {m.max_crush * 1e3:.0f}/"
                    f"{tg.max_crush * 1e3:.0f} mm, e {m.restitution:.3f}/{tg.restitution:.3f}")
            r_c = tg.max_crush / m.max_crush
            r_k = tg.kw400 / m.kw400 if m.max_crush >= tg.window[1] else 1.0 / max(r_c, 1.0)
            r_e = tg.restitution / max(m.restitution, 1e-3)
            last[i] = m
            if abs(r_k - 1.0) < 0.02 and abs(r_c - 1.0) < 0.02 and abs(r_e - 1.0) < 0.1:
                continue
            damp = 0.7
            v.stiffness *= r_k ** damp
            v.yield_force *= (1.0 / r_c) ** damp * r_k ** (0.3 * damp)
            if abs(r_k - 1.0) < 0.15 and abs(r_c - 1.0) < 0.15:
                v.modulus *= min(max((1.0 / r_e) ** (2.0 * damp), 0.5), 2.0)
            still.append(i)
        active = still
    return list(zip(tuned, last))
