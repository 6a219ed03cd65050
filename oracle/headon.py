"""Head-on crash models built in numpy, for the CPU checker and the reference
arm of the benchmark. Test infrastructure: nothing in the engine library
imports it.

Restates, for vehicles that are one homogeneous honeycomb block (no crush
zone, bumper or rail box), the reference's scenario construction:

* ``Mesh::add_hex_block`` / ``add_hex_block_n`` (src/mesh.rs:111-171): node
  numbering i + (nx+1)(j + (ny+1)k), C3D8 corner order, face sets with the
  max-side faces (p0, p1, p2, p3) and min-side faces (p0, p3, p2, p1);
* ``HeadOn::build`` (src/headon.rs:40-66): A's front at x = -5 mm moving +x,
  B's front at +5 mm moving -x with its centre at y = offset, the road slab
  under both (``add_ground`` src/vehicle.rs:829, fixed, elastic 1 GPa), the
  underbody contacts (``add_ground_contact`` :838) and the front pair
  (``Model::add_contact_pair_scaled`` src/model.rs:257, half the smaller
  ``contact_stiffness_per_node`` src/vehicle.rs:384 per side);
* the vehicle outputs: node set, accelerometer node
  (``add_vehicle_accelerometer`` src/vehicle.rs:792-822 via
  ``Mesh::nearest_node``) and front face nodes (``Mesh::face_set_nodes``
  src/mesh.rs:97).

The descriptor it returns is array-for-array the one the engine's own
scenario builder makes for the same scenario (tests/test_oracle_headon.py),
so a CPU run of this model is a run of the same crash without loading the
engine library.
"""
import ctypes as C
import math

import numpy as np

from crushrs_b200 import abi
from crushrs_b200.model import ArrayModel

GAP = 0.005  # src/headon.rs:42
XMIN, XMAX, YMIN, YMAX, ZMIN, ZMAX = range(6)


def _count(length, h):
    """max(round(length / h), 1) with f64::round (half away from zero)."""
    return max(int(math.floor(length / h + 0.5)), 1)


class _Mesh:
    def __init__(self):
        self.pos = []      # arrays of (n, 3)
        self.hexes = []    # arrays of (e, 8)
        self.parts = []    # part id per element, arrays
        self.n_nodes = 0
        self.n_parts = 0
        self.face_sets = {}
        self.node_sets = {}

    def add_block(self, name, origin, size, n, surfaces):
        """Mesh::add_hex_block_n (src/mesh.rs:117-171)."""
        n = [max(int(x), 1) for x in n]
        d = [size[a] / n[a] for a in range(3)]
        node0 = self.n_nodes
        k, j, i = np.meshgrid(np.arange(n[2] + 1), np.arange(n[1] + 1), np.arange(n[0] + 1), indexing="ij")
        x = np.stack([origin[0] + i.ravel() * d[0], origin[1] + j.ravel() * d[1], origin[2] + k.ravel() * d[2]], axis=1)
        self.pos.append(x)

        def nid(i, j, k):
            return node0 + i + (n[0] + 1) * (j + (n[1] + 1) * k)

        k, j, i = np.meshgrid(np.arange(n[2]), np.arange(n[1]), np.arange(n[0]), indexing="ij")
        i, j, k = i.ravel(), j.ravel(), k.ravel()
        h = np.stack([nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                      nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)], axis=1)
        self.hexes.append(h.astype(np.uint32))
        part = self.n_parts
        self.n_parts += 1
        self.parts.append(np.full(h.shape[0], part, np.int32))
        for face, set_name in surfaces:
            a, max_side = face // 2, face % 2 == 1
            b, c = (a + 1) % 3, (a + 2) % 3
            fixed = n[a] if max_side else 0
            ic, ib = np.meshgrid(np.arange(n[c]), np.arange(n[b]), indexing="ij")
            ic, ib = ic.ravel(), ib.ravel()

            def at(ib, ic):
                ijk = [None, None, None]
                ijk[a], ijk[b], ijk[c] = fixed, ib, ic
                return nid(*ijk)

            p0, p1, p2, p3 = at(ib, ic), at(ib + 1, ic), at(ib + 1, ic + 1), at(ib, ic + 1)
            q = np.stack([p0, p1, p2, p3] if max_side else [p0, p3, p2, p1], axis=1)
            self.face_sets[set_name] = np.asarray(q, np.uint32).reshape(-1, 4)
        self.n_nodes += x.shape[0]
        self.node_sets[name] = np.arange(node0, self.n_nodes, dtype=np.uint32)
        return part

    def add_block_h(self, name, origin, size, h, surfaces):
        """Mesh::add_hex_block (src/mesh.rs:111)."""
        return self.add_block(name, origin, size, [_count(size[a], h) for a in range(3)], surfaces)

    def positions(self):
        return np.concatenate(self.pos)

    def face_nodes(self, name):
        return np.unique(self.face_sets[name]).astype(np.uint32)


def honeycomb(youngs, density, yield_stress=0.0, hardening=0.0, curve=None, densification=None):
    """Material::honeycomb / honeycomb_curve (src/material.rs:179, :186)."""
    m = abi.Material()
    m.model = abi.MAT_HONEYCOMB
    m.youngs_modulus = youngs
    m.poisson_ratio = 0.0
    m.density = density
    m.transverse_factor = 1.0
    if curve:
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
        m.densification[0], m.densification[1] = densification
    return m


def _elastic(youngs, poisson, density):
    m = abi.Material()
    m.model = abi.MAT_ELASTIC
    m.youngs_modulus = youngs
    m.poisson_ratio = poisson
    m.density = density
    m.transverse_factor = 1.0
    return m


def _accelerometer_node(pos, nodes, front):
    """add_vehicle_accelerometer (src/vehicle.rs:792-822): the part node
    nearest the point at mid-length, mid-width and 35 % height, moved a
    quarter length away from a front at a bounding-box side (first minimum)."""
    p = pos[nodes]
    lo, hi = p.min(axis=0), p.max(axis=0)
    c = np.zeros(3)
    for nd in front:
        c += pos[nd] / len(front)
    at = np.array([0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]), lo[2] + 0.35 * (hi[2] - lo[2])])
    for d in range(2):
        length = hi[d] - lo[d]
        if c[d] <= lo[d] + 1e-6 * length:
            at[d] = hi[d] - 0.25 * length
        elif c[d] >= hi[d] - 1e-6 * length:
            at[d] = lo[d] + 0.25 * length
    d2 = (p[:, 0] - at[0]) * (p[:, 0] - at[0]) + (p[:, 1] - at[1]) * (p[:, 1] - at[1])
    d2 = d2 + (p[:, 2] - at[2]) * (p[:, 2] - at[2])
    return int(nodes[int(np.argmin(d2))])


def headon(mass_a, size_a, mat_a, mass_b, size_b, mat_b, speed_a, speed_b, offset=0.0, clearance=0.15, element_size=0.3,
           end_time=0.15, stop_rule=abi.STOP_END_TIME, max_steps=0):
    """Two homogeneous honeycomb blocks head-on (HeadOn::build,
    src/headon.rs:40-66); clearance None: no road. Returns an ArrayModel."""
    h = element_size
    m = _Mesh()
    m.add_block_h("a", (-GAP - size_a[0], 0.0 - size_a[1] / 2.0, 0.0), size_a, h, [(XMAX, "a_front"), (ZMIN, "a_bottom")])
    m.add_block_h("b", (GAP, offset - size_b[1] / 2.0, 0.0), size_b, h, [(XMIN, "b_front"), (ZMIN, "b_bottom")])
    road = clearance is not None and clearance >= 0.0
    mats = [mat_a, mat_b]
    if road:
        w = max(size_a[1], size_b[1]) + 2.0 * abs(offset)
        xr, yr, th = (-size_a[0] - 3.0, size_b[0] + 3.0), (-w, w), 0.3
        hg = max(min(xr[1] - xr[0], yr[1] - yr[0]) / 8.0, th)
        m.add_block_h("ground", (xr[0], yr[0], -clearance - th), (xr[1] - xr[0], yr[1] - yr[0], th), hg, [(ZMAX, "ground_face")])
        mats.append(_elastic(1e9, 0.3, 1000.0))
    pos = m.positions()
    vel = np.zeros_like(pos)
    vel[m.node_sets["a"], 0] = speed_a
    vel[m.node_sets["b"], 0] = -speed_b

    def k_per_node(size, mat, n_face):  # Vehicle::contact_stiffness_per_node, src/vehicle.rs:384
        return mat.youngs_modulus * (size[1] * size[2]) / (n_face * h)

    fa, fb = m.face_nodes("a_front"), m.face_nodes("b_front")
    contacts, fixed = [], np.zeros(0, np.uint32)
    if road:
        ground = m.face_sets["ground_face"]
        for name, size, mat, front in (("a", size_a, mat_a, fa), ("b", size_b, mat_b, fb)):
            fixed = np.concatenate([fixed, m.node_sets["ground"]])  # once per underbody contact, as add_ground_contact does
            contacts.append({"nodes": m.face_nodes(name + "_bottom"), "faces": ground,
                             "stiffness": k_per_node(size, mat, len(front)), "max_distance": clearance + 0.3})
    n_face = min(len(fa), len(fb))
    k = min(k_per_node(size_a, mat_a, n_face), k_per_node(size_b, mat_b, n_face))
    contacts.append({"nodes": fa, "faces": m.face_sets["b_front"], "stiffness": 0.5 * k, "max_distance": 0.3})
    contacts.append({"nodes": fb, "faces": m.face_sets["a_front"], "stiffness": 0.5 * k, "max_distance": 0.3})
    vehicles = []
    for name, front in (("a", fa), ("b", fb)):
        nodes = m.node_sets[name]
        vehicles.append({"nodes": nodes, "accel": _accelerometer_node(pos, nodes, front), "front": front})
    settings = abi.Settings(end_time=end_time, dt_scale=0.85, time_step=0.0, adaptive_check_steps=5, hourglass=0.1,
                            velocity_damping=1.0, mass_scaling=0.25, stop_rule=stop_rule, max_steps=max_steps)
    return ArrayModel(pos, np.concatenate(m.hexes), np.concatenate(m.parts), mats, initial_velocity=vel, fixed_nodes=fixed,
                      contacts=contacts, vehicles=vehicles, settings=settings)


BLOCK_A = (2622.0, (6.9, 1.8, 1.5), 0.55e6)
BLOCK_B = (1354.0, (7.5, 1.8, 1.2), 0.30e6)


def refined_headon(max_steps=5000):
    """The refined head-on: both blocks at 0.05 m (36x30x138 and 36x24x150
    = 278,640 hexahedra), an 8-knot yield curve (c = k 0.8/7, sigma 0.3 ->
    1.2 MPa), B offset 0.45 m laterally, +-15.6 m/s, road 0.15 m below, run
    to separation capped at max_steps."""
    curve = [(k * 0.8 / 7.0, 0.3e6 + k * (0.9e6 / 7.0)) for k in range(8)]
    (ma, sa, _), (mb, sb, _) = BLOCK_A, BLOCK_B
    E = 5e6
    mat_a = honeycomb(E, ma / np.prod(sa), curve=curve)
    mat_b = honeycomb(E, mb / np.prod(sb), curve=curve)
    return headon(ma, sa, mat_a, mb, sb, mat_b, 15.6, 15.6, offset=0.45, clearance=0.15, element_size=0.05, end_time=1.0,
                  stop_rule=abi.STOP_SEPARATION, max_steps=max_steps)


def plain_headon(end_time=0.1275):
    """The plain head-on, 1290 hexahedra of 0.3 m: bilinear honeycomb (E 5 MPa,
    sigma_y 0.55 / 0.30 MPa, H 0.2 MPa, lock-up at c = 0.8 with slope E),
    +-13.41 m/s, road 0.15 m below."""
    (ma, sa, ya), (mb, sb, yb) = BLOCK_A, BLOCK_B
    E = 5e6
    mat_a = honeycomb(E, ma / np.prod(sa), ya, 0.2e6, densification=(0.8, E))
    mat_b = honeycomb(E, mb / np.prod(sb), yb, 0.2e6, densification=(0.8, E))
    return headon(ma, sa, mat_a, mb, sb, mat_b, 13.41, 13.41, clearance=0.15, element_size=0.3, end_time=end_time)


def desc_arrays(desc):
    """The descriptor's arrays, for comparisons."""
    out = {"positions": np.ctypeslib.as_array(desc.positions, (desc.n_nodes * 3,)).copy(),
           "hexes": np.ctypeslib.as_array(desc.hexes, (desc.n_hexes * 8,)).copy(),
           "hex_part": np.ctypeslib.as_array(desc.hex_part, (desc.n_hexes,)).copy(),
           "velocity": np.ctypeslib.as_array(desc.initial_velocity, (desc.n_nodes * 3,)).copy(),
           "fixed": np.ctypeslib.as_array(desc.fixed_nodes, (desc.n_fixed,)).copy() if desc.n_fixed else np.zeros(0, np.uint32)}
    for p in range(desc.n_parts):
        mt = desc.materials[p]
        out[f"mat{p}"] = np.array([mt.model, mt.youngs_modulus, mt.poisson_ratio, mt.density, mt.yield_stress, mt.hardening, mt.n_curve,
                                   mt.has_densification, mt.densification[0], mt.densification[1], mt.transverse_factor]
                                  + [mt.curve[i][j] for i in range(abi.MAX_KNOTS) for j in range(2)])
    for c in range(desc.n_contacts):
        k = desc.contacts[c]
        out[f"c{c}_nodes"] = np.ctypeslib.as_array(k.nodes, (k.n_nodes,)).copy()
        out[f"c{c}_faces"] = np.ctypeslib.as_array(k.faces, (k.n_faces * 4,)).copy()
        out[f"c{c}_scale"] = np.ctypeslib.as_array(k.node_scale, (k.n_nodes,)).copy() if k.node_scale else None
        out[f"c{c}_k"] = np.array([k.stiffness, k.max_distance])
    for v in range(desc.n_vehicles):
        w = desc.vehicles[v]
        out[f"v{v}_nodes"] = np.ctypeslib.as_array(w.nodes, (w.n_nodes,)).copy()
        out[f"v{v}_accel"] = np.array([w.accel_node])
        out[f"v{v}_front"] = np.ctypeslib.as_array(w.front_nodes, (w.n_front,)).copy()
    s = desc.settings
    out["settings"] = np.array([s.end_time, s.dt_scale, s.time_step, s.adaptive_check_steps, s.hourglass, s.velocity_damping,
                                s.mass_scaling, s.stop_rule, s.max_steps])
    return out
