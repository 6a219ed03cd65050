"""Abaqus `.inp` meshes (as Gmsh exports them) into engine models: the
reference's minimal reader (src/input/inp.rs:8-78) and the Model calls a
configuration makes on the mesh (src/model.rs:222-270: materials per part,
initial velocity and fixed nodes per node set or part, one-way and paired
contacts between face sets).

    mesh = read_inp(text)                       # *NODE, *ELEMENT C3D8 / CPS4, *NSET
    b = InpModel(mesh)
    b.set_material("block", S.honeycomb(...)); b.set_initial_velocity("block", (10, 0, 0))
    b.fix("wall"); b.add_contact_pair("front", "wall_face", k, 0.3)
    model = b.build(settings)                   # an ArrayModel: model.desc for Context
"""
import numpy as np

from .model import ArrayModel
from .scenarios import elastic


class InpMesh:
    """Nodes, C3D8 hexahedra with a part per element set, CPS4 quads in face
    sets, node sets (part names also name their element nodes)."""

    def __init__(self):
        self.nodes = []
        self.hexes = []
        self.hex_part = []
        self.parts = []
        self.faces = []
        self.face_sets = {}
        self.node_sets = {}

    def part_index(self, name):
        return self.parts.index(name) if name in self.parts else None

    def part_nodes(self, p):
        return sorted({n for h, q in zip(self.hexes, self.hex_part) if q == p for n in h})

    def nodes_of(self, name):
        """Mesh::nodes_of (src/mesh.rs:85): a node set, else a part's nodes."""
        if name in self.node_sets:
            return list(self.node_sets[name])
        p = self.part_index(name)
        return None if p is None else self.part_nodes(p)

    def face_set_nodes(self, name):
        """Mesh::face_set_nodes (src/mesh.rs:97): sorted, unique."""
        if name not in self.face_sets:
            return None
        return sorted({n for f in self.face_sets[name] for n in self.faces[f]})


def read_inp(text):
    """read_inp (src/input/inp.rs:8-78) on the file's text: `*NODE` lines
    `id, x, y, z`; `*ELEMENT, type=C3D8` (one part per ELSET, in order of
    first appearance) and `type=CPS4` (quads into the ELSET's face set);
    `*NSET` ids; `**` comments; ids renumbered in order of appearance; every
    part also becomes a node set of its nodes unless one of that name exists."""
    mesh = InpMesh()
    index = {}
    section, params, set_name = "", {}, ""
    for raw in text.splitlines():
        line = raw.strip()
        if not line or line.startswith("**"):
            continue
        if line.startswith("*"):
            parts = [s.strip() for s in line[1:].split(",")]
            section = parts[0].upper()
            params = {}
            for p in parts[1:]:
                if "=" in p:
                    k, v = p.split("=", 1)
                    params[k.strip().upper()] = v.strip()
            set_name = params.get("ELSET", params.get("NSET", ""))
            continue
        fields = [s.strip() for s in line.split(",") if s.strip()]
        if section == "NODE":
            if len(fields) < 4:
                continue
            try:
                nid = int(fields[0])
            except ValueError:
                raise ValueError(f"bad node line: {line}")

            def num(s):
                try:
                    return float(s)
                except ValueError:
                    return 0.0

            index[nid] = len(mesh.nodes)
            mesh.nodes.append([num(fields[1]), num(fields[2]), num(fields[3])])
        elif section == "ELEMENT":
            ty = params.get("TYPE", "").upper()
            try:
                ids = [index[int(f)] for f in fields[1:]]
            except (KeyError, ValueError):
                raise ValueError(f"unknown node in element line: {line}")
            if ty == "C3D8" and len(ids) == 8:
                p = mesh.part_index(set_name)
                if p is None:
                    mesh.parts.append(set_name)
                    p = len(mesh.parts) - 1
                mesh.hexes.append(ids)
                mesh.hex_part.append(p)
            elif ty == "CPS4" and len(ids) == 4:
                mesh.faces.append(ids)
                mesh.face_sets.setdefault(set_name, []).append(len(mesh.faces) - 1)
        elif section == "NSET":
            s = mesh.node_sets.setdefault(set_name, [])
            for f in fields:
                try:
                    s.append(index[int(f)])
                except (KeyError, ValueError):
                    pass
    for p, name in enumerate(mesh.parts):
        mesh.node_sets.setdefault(name, mesh.part_nodes(p))
    return mesh


class InpModel:
    """The Model calls of a configuration on a read mesh
    (src/model.rs:216-270), then build() -> ArrayModel."""

    def __init__(self, mesh):
        self.mesh = mesh
        self.materials = [None] * len(mesh.parts)
        self.velocity = np.zeros((len(mesh.nodes), 3))
        self.fixed = []
        self.contacts = []
        self.vehicles = []

    def _nodes(self, name):
        nodes = self.mesh.nodes_of(name)
        if nodes is None:
            raise KeyError(f"no node set or part '{name}'")
        return nodes

    def set_material(self, part, material):
        p = self.mesh.part_index(part)
        if p is None:
            raise KeyError(f"no part '{part}'")
        self.materials[p] = material
        return self

    def set_initial_velocity(self, name, v):
        self.velocity[self._nodes(name)] = v
        return self

    def fix(self, name):
        self.fixed.extend(self._nodes(name))
        return self

    def _faces(self, name):
        if name not in self.mesh.face_sets:
            raise KeyError(f"no face set '{name}'")
        return [self.mesh.faces[f] for f in self.mesh.face_sets[name]]

    def add_contact_one_way(self, nodes, faces, stiffness, max_distance):
        """The nodes of face set `nodes` against the faces of `faces` at the full stiffness (src/model.rs:240)."""
        n = self.mesh.face_set_nodes(nodes)
        if n is None:
            raise KeyError(f"no face set '{nodes}'")
        self.contacts.append({"nodes": n, "faces": self._faces(faces), "stiffness": stiffness, "max_distance": max_distance})
        return self

    def add_contact_pair(self, a, b, stiffness, max_distance, scale_a=None, scale_b=None):
        """Each side's nodes against the other's faces at half the stiffness (src/model.rs:252-265)."""
        for p, s, scale in ((a, b, scale_a), (b, a, scale_b)):
            n = self.mesh.face_set_nodes(p)
            if n is None:
                raise KeyError(f"no face set '{p}'")
            self.contacts.append({"nodes": n, "faces": self._faces(s), "stiffness": 0.5 * stiffness, "max_distance": max_distance,
                                  "scale": scale})
        return self

    def add_vehicle(self, nodes, accel_node, front_faces):
        """Delta-v and crush outputs of a node set: its accelerometer node and front face set."""
        self.vehicles.append({"nodes": self._nodes(nodes), "accel": accel_node, "front": self.mesh.face_set_nodes(front_faces)})
        return self

    def build(self, settings=None):
        """Parts given no material keep Model::new's default, elastic
        E = 1, nu = 0, density 1 (src/model.rs:170)."""
        mats = [m if m is not None else elastic(1.0, 0.0, 1.0) for m in self.materials]
        return ArrayModel(np.asarray(self.mesh.nodes, np.float64), np.asarray(self.mesh.hexes, np.uint32),
                          np.asarray(self.mesh.hex_part, np.int32), mats, initial_velocity=self.velocity,
                          fixed_nodes=sorted(set(self.fixed)), contacts=self.contacts, vehicles=self.vehicles, settings=settings)
