"""Model descriptors from numpy arrays (any hexahedral mesh), mirroring the
reference's Model (src/model.rs:153): nodes, C3D8 hexahedra with a part per
element, one material per part, initial velocities, fixed nodes, one-way
contacts and the vehicles whose delta-v and crush are reported."""
import ctypes as C

import numpy as np

from . import abi


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class ArrayModel:
    """Owns the arrays behind a crush_model_desc (keep it alive while the
    descriptor is in use)."""

    def __init__(self, positions, hexes, hex_part, materials, initial_velocity=None, fixed_nodes=(),
                 contacts=(), vehicles=(), settings=None):
        self.positions = _f64(positions).reshape(-1, 3)
        self.hexes = _u32(hexes).reshape(-1, 8)
        self.hex_part = np.ascontiguousarray(hex_part, dtype=np.int32).reshape(-1)
        n = self.positions.shape[0]
        self.initial_velocity = _f64(np.zeros((n, 3)) if initial_velocity is None else initial_velocity).reshape(-1, 3)
        self.fixed_nodes = _u32(fixed_nodes).reshape(-1)
        self.materials = (abi.Material * len(materials))(*materials)
        self._contacts = []
        for c in contacts:
            nodes = _u32(c["nodes"])
            faces = _u32(c["faces"]).reshape(-1, 4)
            scale = None if c.get("scale") is None else _f64(c["scale"])
            self._contacts.append((nodes, faces, scale, float(c["stiffness"]), float(c["max_distance"])))
        self._vehicles = [(_u32(v["nodes"]), int(v["accel"]), _u32(v["front"])) for v in vehicles]
        if settings is None:
            settings = abi.Settings(end_time=0.15, dt_scale=0.85, time_step=0.0, adaptive_check_steps=5, hourglass=0.1,
                                    velocity_damping=1.0, mass_scaling=0.25, stop_rule=0, max_steps=0)
        self.settings = settings
        self.desc = self._make_desc()

    def _make_desc(self):
        d = abi.ModelDesc()
        d.n_nodes = self.positions.shape[0]
        d.positions = self.positions.ctypes.data_as(C.POINTER(C.c_double))
        d.n_hexes = self.hexes.shape[0]
        d.hexes = self.hexes.ctypes.data_as(C.POINTER(C.c_uint32))
        d.hex_part = self.hex_part.ctypes.data_as(C.POINTER(C.c_int32))
        d.n_parts = len(self.materials)
        d.materials = C.cast(self.materials, C.POINTER(abi.Material))
        d.initial_velocity = self.initial_velocity.ctypes.data_as(C.POINTER(C.c_double))
        d.n_fixed = self.fixed_nodes.shape[0]
        d.fixed_nodes = self.fixed_nodes.ctypes.data_as(C.POINTER(C.c_uint32))
        self._cd = (abi.Contact * max(1, len(self._contacts)))()
        for i, (nodes, faces, scale, k, md) in enumerate(self._contacts):
            c = self._cd[i]
            c.n_nodes = nodes.shape[0]
            c.nodes = nodes.ctypes.data_as(C.POINTER(C.c_uint32))
            c.node_scale = scale.ctypes.data_as(C.POINTER(C.c_double)) if scale is not None else None
            c.n_faces = faces.shape[0]
            c.faces = faces.ctypes.data_as(C.POINTER(C.c_uint32))
            c.stiffness = k
            c.max_distance = md
        d.n_contacts = len(self._contacts)
        d.contacts = C.cast(self._cd, C.POINTER(abi.Contact))
        self._vd = (abi.Vehicle * max(1, len(self._vehicles)))()
        for i, (nodes, accel, front) in enumerate(self._vehicles):
            v = self._vd[i]
            v.n_nodes = nodes.shape[0]
            v.nodes = nodes.ctypes.data_as(C.POINTER(C.c_uint32))
            v.accel_node = accel
            v.n_front = front.shape[0]
            v.front_nodes = front.ctypes.data_as(C.POINTER(C.c_uint32))
        d.n_vehicles = len(self._vehicles)
        d.vehicles = C.cast(self._vd, C.POINTER(abi.Vehicle))
        d.settings = self.settings
        return d

    @property
    def n_nodes(self):
        return self.positions.shape[0]

    @property
    def n_hexes(self):
        return self.hexes.shape[0]


# C3D8 parametric corners (src/element.rs:9).
XI = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
               [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], dtype=np.float64)


def single_hex(material, nodes=None, side=1.0, settings=None):
    """One hexahedron (default: the cube [0, side]^3 in C3D8 order)."""
    x = 0.5 * side * (XI + 1.0) if nodes is None else np.asarray(nodes, np.float64)
    return ArrayModel(x, np.arange(8), [0], [material], settings=settings)
