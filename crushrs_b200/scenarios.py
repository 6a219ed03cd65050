"""Crash scenarios: material and vehicle specs, the reference's presets and
the synthetic workloads the engine is measured on.

Reference presets follow crushrs's src/vehicle.rs:
  Vehicle::from_ncap              :230   (curve, modulus)
  Vehicle::crush_material_axial   :478   (sigma_y = F_y / A, H = k L_c / A)
  TRANSVERSE_FACTOR = 4.0         :493
  chevrolet_silverado_2007_tuned  :638
  dodge_neon_1996_tuned           :621
The synthetic workloads are the seeded block head-ons, T-bones and rear-ends
of the engine's benchmark configurations (sizes in each function).
"""
import ctypes as C
import math

import numpy as np

from . import abi
from .native import check, lib

MPH = 0.44704  # src/lib.rs:28
TUNED_ELEMENT_SIZE = 0.3  # src/vehicle.rs:647
TRANSVERSE_FACTOR = 4.0  # src/vehicle.rs:493


def honeycomb(youngs, density, yield_stress=0.0, hardening=0.0, curve=None, densification=None, transverse=1.0):
    """Material::honeycomb / honeycomb_curve (src/material.rs:179, :186)."""
    m = abi.Material()
    m.model = abi.MAT_HONEYCOMB
    m.youngs_modulus = youngs
    m.poisson_ratio = 0.0
    m.density = density
    m.transverse_factor = transverse
    if curve:
        assert 2 <= len(curve) <= abi.MAX_KNOTS
        m.n_curve = len(curve)
        for i, (c, s) in enumerate(curve):
            m.curve[i][0] = c
            m.curve[i][1] = s
        m.yield_stress = curve[0][1]
        m.hardening = (curve[1][1] - curve[0][1]) / (curve[1][0] - curve[0][0])
    else:
        m.yield_stress = yield_stress
        m.hardening = hardening
    if densification is not None:
        m.has_densification = 1
        m.densification[0] = densification[0]
        m.densification[1] = densification[1]
    return m


def elastic(youngs, poisson, density):
    m = abi.Material()
    m.model = abi.MAT_ELASTIC
    m.youngs_modulus = youngs
    m.poisson_ratio = poisson
    m.density = density
    m.transverse_factor = 1.0
    return m


def vehicle(mass, size, material, contact_modulus=0.0, rail_box=None, crush_zone_length=0.0, body_modulus=0.0,
            crush_zone_mass=0.0, bumper=None, crush_element_size=0.0):
    """A crushable vehicle (crush_vehicle_spec). rail_box = (width, (z0, z1),
    force_fraction). With 0 < crush_zone_length < length it is the
    reference's two-part vehicle (src/vehicle.rs:663-790): a honeycomb crush
    zone of that length (with `crush_zone_mass` kg, elements of
    `crush_element_size` along x) in front of an elastic body of modulus
    `body_modulus`, and bumper = (thickness, mass, modulus) an elastic front
    layer."""
    v = abi.VehicleSpec()
    v.mass = mass
    for i in range(3):
        v.size[i] = size[i]
    v.material = material
    v.contact_modulus = contact_modulus
    if rail_box is not None:
        v.has_rail_box = 1
        v.rail_box_width = rail_box[0]
        v.rail_box_z[0], v.rail_box_z[1] = rail_box[1]
        v.rail_box_force_fraction = rail_box[2]
    v.crush_zone_length = crush_zone_length
    v.body_modulus = body_modulus
    v.crush_zone_mass = crush_zone_mass
    if bumper is not None:
        for i in range(3):
            v.bumper[i] = bumper[i]
    v.crush_element_size = crush_element_size
    return v


LOCK_COMPACTION = 1.4    # src/vehicle.rs:503
LOCK_SLOPE_FACTOR = 1.0  # src/vehicle.rs:504


def force_table_material(modulus, density, table, honeycomb_length, area, transverse=TRANSVERSE_FACTOR):
    """Vehicle::crush_material_axial with a force-crush table
    (src/vehicle.rs:478-488, yield_curve :509): compaction c = -ln(1 - x/L_c)
    (x/L_c capped at 0.95), yield stress F/A, locking up at c = 1.4 with slope
    1.0 E."""
    curve = [(-math.log(1.0 - min(x / honeycomb_length, 0.95)), f / area) for x, f in table]
    return honeycomb(modulus, density, curve=curve, densification=(LOCK_COMPACTION, LOCK_SLOPE_FACTOR * modulus), transverse=transverse)


class TableVehicle:
    """A two-part vehicle whose crush zone follows a tabulated force-crush
    curve (the reference's Vehicle with `force_table`, src/vehicle.rs:137-147,
    478-488): the parameters a pulse calibration moves (the table, the crush
    zone's and the body's moduli) and the rest of the vehicle. spec() builds
    the crush_vehicle_spec."""

    def __init__(self, mass, size, crush_zone, crush_zone_mass, bumper, rail_box, modulus, body_modulus, table,
                 crush_element_size=0.1, transverse=TRANSVERSE_FACTOR):
        self.mass, self.size = mass, tuple(size)
        self.crush_zone, self.crush_zone_mass = crush_zone, crush_zone_mass
        self.bumper, self.rail_box = tuple(bumper), rail_box
        self.modulus, self.body_modulus = modulus, body_modulus
        self.table = [tuple(k) for k in table]  # (crush m, force N)
        self.crush_element_size, self.transverse = crush_element_size, transverse

    def copy(self):
        return TableVehicle(self.mass, self.size, self.crush_zone, self.crush_zone_mass, self.bumper, self.rail_box, self.modulus,
                            self.body_modulus, list(self.table), self.crush_element_size, self.transverse)

    def spec(self):
        area = self.size[1] * self.size[2]
        l_c = self.crush_zone - self.bumper[0]
        density = (self.crush_zone_mass - self.bumper[1]) / (l_c * area)  # Vehicle::crush_density
        mat = force_table_material(self.modulus, density, self.table, l_c, area, self.transverse)
        return vehicle(self.mass, self.size, mat, contact_modulus=self.modulus, rail_box=self.rail_box,
                       crush_zone_length=self.crush_zone, body_modulus=self.body_modulus, crush_zone_mass=self.crush_zone_mass,
                       bumper=self.bumper, crush_element_size=self.crush_element_size)


def _pulse_vehicle(mass, size, crush_zone, crush_zone_mass, bumper, rail_box, modulus, body_modulus, knots, force_kn, table=False):
    tv = TableVehicle(mass, size, crush_zone, crush_zone_mass, bumper, rail_box, modulus, body_modulus,
                      [(x, f * 1e3) for x, f in zip(knots, force_kn)])
    return tv if table else tv.spec()


def neon_1996_pulse(table=False):
    """Vehicle::dodge_neon_1996_pulse (src/vehicle.rs:541-566): the Neon
    fitted to a rear-seat barrier pulse, a 1.5 m crush zone of 0.1 m
    elements and 190 kg with a 0.1 m bumper, ahead of an elastic body, and a
    rail box carrying 80 % of the force (table=True: as a TableVehicle)."""
    return _pulse_vehicle(1354.0, (4.36, 1.71, 1.35), 1.5, 190.0, (0.1, 25.0, 3.0e8), (0.45, (0.06, 0.41), 0.8), 4e6, 2.7e8,
                          [0.0, 0.1165, 0.2330, 0.3496, 0.4661, 0.5826, 0.6991], [13.0, 135.0, 135.0, 146.0, 361.0, 364.0, 364.0],
                          table)


def ford_expedition_1999(mass=2460.0, size=(5.2, 2.0, 1.9), table=False):
    """Vehicle::ford_expedition_1999 (src/vehicle.rs:568-593): a 1.7 m crush
    zone with 320 kg and a bumper, the rail box carrying 75 % of the force."""
    return _pulse_vehicle(mass, size, 1.7, 320.0, (0.1, 35.0, 3.0e8), (1.25, (0.15, 0.72), 0.75), 7.3e6, 3.93e8,
                          [0.0, 0.1064, 0.2128, 0.3192, 0.4256, 0.5320, 0.6384], [29.0, 183.0, 259.0, 417.0, 457.0, 457.0, 457.0],
                          table)


def lincoln_navigator_1999(table=False):
    """Vehicle::lincoln_navigator_1999 (src/vehicle.rs:595-603): the
    Expedition structure with 2873 kg and 5.175 x 2.049 x 1.9 m."""
    return ford_expedition_1999(2873.0, (5.175, 2.049, 1.9), table)


def _preset(mass, size, yield_force, stiffness, modulus):
    # crush_material_axial with the whole block as crush zone (src/vehicle.rs:488).
    area = size[1] * size[2]
    density = mass / (size[0] * size[1] * size[2])
    mat = honeycomb(modulus, density, yield_force / area, stiffness * size[0] / area, transverse=TRANSVERSE_FACTOR)
    return vehicle(mass, size, mat, contact_modulus=modulus)


def silverado_2007_tuned():
    """src/vehicle.rs:611-613, :638-644."""
    return _preset(2622.0, (5.85, 2.03, 1.87), 51.21e3, 5.592e5, 27.8e6)


def neon_1996_tuned():
    """src/vehicle.rs:528-531, :621-633 (frontal profile)."""
    return _preset(1354.0, (4.36, 1.71, 1.35), 16.73e3, 2.930e5, 23.1e6)


def settings(end_time=0.15, **kw):
    s = lib().crush_settings_default(end_time)
    for k, v in kw.items():
        setattr(s, k, v)
    return s


def scenario(a, b, speed_a, speed_b, offset=0.0, clearance=0.15, element_size=0.3, layout=abi.LAYOUT_HEADON, end_time=0.15, **settings_kw):
    s = abi.Scenario()
    s.layout = layout
    s.a = a
    s.b = b
    s.speed_a = speed_a
    s.speed_b = speed_b
    s.offset = offset
    s.clearance = -1.0 if clearance is None else clearance
    s.element_size = element_size
    s.settings = settings(end_time, **settings_kw)
    return s


class Model:
    """A model built by the engine's host builder (owns the C crush_model)."""

    def __init__(self, handle):
        self._h = C.c_void_p(handle)
        self.desc = abi.ModelDesc()
        check(lib().crush_model_desc_get(self._h, C.byref(self.desc)))

    @classmethod
    def build(cls, scen):
        h = C.c_void_p()
        check(lib().crush_scenario_build(C.byref(scen), C.byref(h)))
        return cls(h.value)

    def __del__(self):
        try:
            if self._h:
                lib().crush_model_free(self._h)
                self._h = None
        except Exception:
            pass

    def refresh(self):
        check(lib().crush_model_desc_get(self._h, C.byref(self.desc)))

    @property
    def settings(self):
        return lib().crush_model_settings(self._h).contents

    # numpy views (valid while the model lives)
    @property
    def n_nodes(self):
        return self.desc.n_nodes

    @property
    def n_hexes(self):
        return self.desc.n_hexes

    def positions(self):
        return np.ctypeslib.as_array(self.desc.positions, (self.desc.n_nodes, 3))

    def hexes(self):
        return np.ctypeslib.as_array(self.desc.hexes, (self.desc.n_hexes, 8))

    def hex_part(self):
        return np.ctypeslib.as_array(self.desc.hex_part, (self.desc.n_hexes,))

    def initial_velocity(self):
        return np.ctypeslib.as_array(self.desc.initial_velocity, (self.desc.n_nodes, 3))

    def fixed_nodes(self):
        if self.desc.n_fixed == 0:
            return np.zeros(0, np.uint32)
        return np.ctypeslib.as_array(self.desc.fixed_nodes, (self.desc.n_fixed,))

    def material(self, p):
        return self.desc.materials[p]

    def contact(self, c):
        k = self.desc.contacts[c]
        nodes = np.ctypeslib.as_array(k.nodes, (k.n_nodes,))
        faces = np.ctypeslib.as_array(k.faces, (k.n_faces, 4))
        scale = np.ctypeslib.as_array(k.node_scale, (k.n_nodes,)) if k.node_scale else None
        return nodes, faces, scale, k.stiffness, k.max_distance

    def vehicle(self, v):
        w = self.desc.vehicles[v]
        return (np.ctypeslib.as_array(w.nodes, (w.n_nodes,)), int(w.accel_node),
                np.ctypeslib.as_array(w.front_nodes, (w.n_front,)))

    def vehicle_frame(self, v):
        """(origin, x axis, plane) nodes of vehicle v's accelerometer frame
        (Model::add_accelerometer_at, src/model.rs:185-214)."""
        f = (C.c_uint32 * 3)()
        check(lib().crush_model_vehicle_frame(self._h, v, f))
        return tuple(int(x) for x in f)

    def accelerometer(self, v):
        """Vehicle v's rear-seat accelerometer with its body frame, as
        history_config takes it."""
        return ([self.vehicle(v)[1]], self.vehicle_frame(v))


PULSE_END = 0.15  # src/vehicle.rs:1104
PULSE_DT = 1e-4   # src/vehicle.rs:1102


def barrier(v, speed, element_size=TUNED_ELEMENT_SIZE, end_time=PULSE_END, clearance=0.15, **settings_kw):
    """barrier_model (src/vehicle.rs:951): vehicle v at `speed` into a fixed
    rigid wall at x = 0, on the road."""
    dummy = vehicle(1.0, (1.0, 1.0, 1.0), honeycomb(1.0, 1.0))
    return scenario(v, dummy, speed, 0.0, clearance=clearance, element_size=element_size, layout=abi.LAYOUT_BARRIER,
                    end_time=end_time, **settings_kw)


def crash_30_30():
    """`crushrs crash 30 30` (src/bin/crushrs.rs:403-416): Silverado vs Neon,
    head-on at 30 mph each, 0.3 m elements, no road, 0.15 s."""
    return scenario(silverado_2007_tuned(), neon_1996_tuned(), 30 * MPH, 30 * MPH, clearance=None, element_size=TUNED_ELEMENT_SIZE, end_time=0.15)


# ---------------- synthetic workloads ----------------

def _block_material(E, density, sigma_y, hardening=0.2e6, lock=0.8, curve=None):
    dens = None if curve is not None and len(curve) >= abi.MAX_KNOTS else (lock, E)
    return honeycomb(E, density, sigma_y, hardening, curve=curve, densification=dens)


def plain_headon(end_time=0.1275):
    """Plain head-on, 1290 hexahedra: A 6x5x23 (y, z, x) cubes of 0.3 m, 2622 kg,
    +13.41 m/s; B 6x4x25, 1354 kg, -13.41 m/s; E 5 MPa, sigma_y 0.30 MPa
    (A 0.55 MPa), H 0.2 MPa, lock-up at c = 0.8 with k_lock = E; road 0.15 m
    below; about 650 steps (end time 0.1275 s)."""
    sa, sb = (6.9, 1.8, 1.5), (7.5, 1.8, 1.2)
    ma, mb = 2622.0, 1354.0
    E = 5e6
    a = vehicle(ma, sa, _block_material(E, ma / np.prod(sa), 0.55e6))
    b = vehicle(mb, sb, _block_material(E, mb / np.prod(sb), 0.30e6))
    return scenario(a, b, 13.41, 13.41, clearance=0.15, element_size=0.3, end_time=end_time)


def refined_headon(max_steps=5000):
    """Refined head-on for the bandwidth roofline: the same blocks at 0.05 m
    (36x30x138 and 36x24x150 = 278,640 hexahedra), an 8-knot yield curve
    (c = k 0.8/7, sigma 0.3 -> 1.2 MPa), lateral offset 0.45 m, +-15.6 m/s,
    run to separation (CRUSH_STOP_SEPARATION), capped at 5000 steps."""
    sa, sb = (6.9, 1.8, 1.5), (7.5, 1.8, 1.2)
    ma, mb = 2622.0, 1354.0
    E = 5e6
    curve = [(k * 0.8 / 7.0, 0.3e6 + k * (0.9e6 / 7.0)) for k in range(8)]
    a = vehicle(ma, sa, _block_material(E, ma / np.prod(sa), 0.3e6, curve=curve))
    b = vehicle(mb, sb, _block_material(E, mb / np.prod(sb), 0.3e6, curve=curve))
    return scenario(a, b, 15.6, 15.6, offset=0.45, clearance=0.15, element_size=0.05, end_time=1.0,
                    stop_rule=abi.STOP_SEPARATION, max_steps=max_steps)


class XorShift64Star:
    """xorshift64* (the generator of src/headon.rs:105-122)."""

    def __init__(self, seed):
        self.s = seed & 0xFFFFFFFFFFFFFFFF or 1

    def next_u64(self):
        x = self.s
        x ^= x >> 12
        x ^= (x << 25) & 0xFFFFFFFFFFFFFFFF
        x ^= x >> 27
        self.s = x
        return (x * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF

    def uniform(self, lo=0.0, hi=1.0):
        return lo + (hi - lo) * ((self.next_u64() >> 11) / float(1 << 53))


BATCH_SEED = 0x9E3779B97F4A7C15


def _seeded_pair(rng, e_lo, e_hi, h_choices=None, h_range=(0.15, 0.3)):
    """Two blocks whose total element count is drawn log-uniform in [e_lo, e_hi]."""
    h = rng.uniform(*h_range) if h_choices is None else h_choices[int(rng.uniform(0, len(h_choices))) % len(h_choices)]
    e_target = math.exp(rng.uniform(math.log(e_lo), math.log(e_hi)))
    # Car-like proportions: length 3.8 x height; width 1.2 x height.
    per = e_target / 2.0
    blocks = []
    for _ in range(2):
        scale_len = rng.uniform(0.8, 1.2)
        nz = max(2, round((per / (3.8 * 1.2 * scale_len)) ** (1.0 / 3.0)))
        ny = max(2, round(1.2 * nz))
        nx = max(2, round(per / (ny * nz)))
        blocks.append((nx * h, ny * h, nz * h))
    return h, blocks[0], blocks[1]


def batch_headon(i, seed=BATCH_SEED):
    """Crash i of the batched workload: 300-6000 hexahedra (log-uniform),
    element size 0.15-0.3 m, masses 1000-3000 kg, speeds 5-25 m/s each,
    offset 0-0.9 m, bilinear sigma_y 0.2-0.6 MPa. Deterministic in (seed, i)."""
    rng = XorShift64Star(seed ^ ((i + 1) * 0x9E3779B97F4A7C15 & 0xFFFFFFFFFFFFFFFF))
    for _ in range(4):
        rng.next_u64()
    h, sa, sb = _seeded_pair(rng, 300, 6000)
    ma, mb = rng.uniform(1000, 3000), rng.uniform(1000, 3000)
    va, vb = rng.uniform(5, 25), rng.uniform(5, 25)
    off = rng.uniform(0.0, 0.9)
    sya, syb = rng.uniform(0.2e6, 0.6e6), rng.uniform(0.2e6, 0.6e6)
    E = 5e6
    a = vehicle(ma, sa, _block_material(E, ma / np.prod(sa), sya))
    b = vehicle(mb, sb, _block_material(E, mb / np.prod(sb), syb))
    return scenario(a, b, va, vb, offset=off, clearance=0.15, element_size=h, end_time=0.12)


SERVE_SEED = 0xD1B54A32D192ED03
SERVE_KINDS = ("head-on", "t-bone", "rear-end")


def serve_query(i, seed=SERVE_SEED, e_range=(300, 20000)):
    """Delta-v query i of the serving workload: a head-on, T-bone or rear-end
    (one third each), 300-20000 hexahedra (log-uniform), element size from
    {0.1, 0.15, 0.2, 0.25, 0.3} m, speeds 5-30 m/s, masses 1000-3000 kg,
    bilinear sigma_y 0.2-0.6 MPa. Deterministic in (seed, i). Returns
    (kind, scenario)."""
    rng = XorShift64Star(seed ^ ((i + 1) * 0xBF58476D1CE4E5B9 & 0xFFFFFFFFFFFFFFFF))
    for _ in range(4):
        rng.next_u64()
    kind = SERVE_KINDS[int(rng.uniform(0, 3)) % 3]
    h, sa, sb = _seeded_pair(rng, e_range[0], e_range[1], h_choices=(0.1, 0.15, 0.2, 0.25, 0.3))
    ma, mb = rng.uniform(1000, 3000), rng.uniform(1000, 3000)
    sya, syb = rng.uniform(0.2e6, 0.6e6), rng.uniform(0.2e6, 0.6e6)
    E = 5e6
    a = vehicle(ma, sa, _block_material(E, ma / np.prod(sa), sya))
    b = vehicle(mb, sb, _block_material(E, mb / np.prod(sb), syb))
    if kind == "head-on":
        va, vb = rng.uniform(5, 30), rng.uniform(5, 30)
        return kind, scenario(a, b, va, vb, offset=rng.uniform(0.0, 0.9), clearance=0.15, element_size=h, end_time=0.12)
    if kind == "t-bone":
        # B turned 90 degrees: its length along y, its side facing A's front
        va = rng.uniform(5, 30)
        bt = vehicle(mb, (sb[1], sb[0], sb[2]), _block_material(E, mb / np.prod(sb), syb))
        return kind, scenario(a, bt, va, 0.0, offset=rng.uniform(0.0, 0.3) * sb[0], clearance=0.15, element_size=h,
                              layout=abi.LAYOUT_TBONE, end_time=0.12)
    va = rng.uniform(10, 30)  # rear-end: B moves the same way, slower
    vb = va * rng.uniform(0.1, 0.6)
    return kind, scenario(a, b, va, -vb, offset=rng.uniform(0.0, 0.5), clearance=0.15, element_size=h, end_time=0.12)


def tbone_coverage():
    """T-bone coverage case (about 2000 hexahedra): A's front into the side of
    B turned 90 degrees (B's length along y), B's side sigma_y 0.15 MPa,
    A at 13.41 m/s (30 mph), B at rest, element size 0.2 m."""
    h = 0.2
    sa, sb = (3.4, 1.6, 1.2), (1.6, 4.6, 1.2)
    ma, mb = 1600.0, 1400.0
    E = 5e6
    a = vehicle(ma, sa, _block_material(E, ma / np.prod(sa), 0.4e6))
    b = vehicle(mb, sb, _block_material(E, mb / np.prod(sb), 0.15e6))
    return scenario(a, b, 30 * MPH, 0.0, offset=0.3, clearance=0.15, element_size=h, layout=abi.LAYOUT_TBONE, end_time=0.1)


def railbox_coverage(densify=False, speed=9.0):
    """Rail-box coverage case (about 2000 hexahedra): head-on where A's front
    has a central rail box 0.9 m wide over z 0.3-0.9 m carrying 0.7 of the
    crush force (modulus, yield and density scaled alike), element size 0.2 m,
    both at `speed` m/s. densify=True adds the lock-up knot [0.75, 50 MPa] to
    both materials. With densification at 15 m/s elements invert and erode."""
    h = 0.2
    sa, sb = (3.6, 1.8, 1.2), (3.6, 1.8, 1.2)
    ma, mb = 1800.0, 1500.0
    E = 5e6
    dens = (0.75, 50e6) if densify else None
    ha = honeycomb(E, ma / np.prod(sa), 0.45e6, 0.2e6, densification=dens)
    hb = honeycomb(E, mb / np.prod(sb), 0.35e6, 0.2e6, densification=dens)
    a = vehicle(ma, sa, ha, rail_box=(0.9, (0.3, 0.9), 0.7))
    b = vehicle(mb, sb, hb)
    return scenario(a, b, speed, speed, offset=0.0, clearance=0.15, element_size=h, end_time=0.1)
