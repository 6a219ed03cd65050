"""The Abaqus .inp reader (src/input/inp.rs:8-78) and the model calls on its
mesh (src/model.rs:216-270), on a small Gmsh-style file: a honeycomb block
of two hexahedra moving into a fixed elastic wall block, a CPS4 face set on
each side and a node set. The model runs through the oracle."""
import numpy as np
import pytest

from crushrs_b200 import inp, scenarios as S

from . import oracle_lib as O


def _block_lines(first_node, first_elem, x0, nx, name, face_name, face_side):
    """A 1 x 1 x nx column of unit-ish hexahedra along x as .inp text."""
    lines, ids = ["*NODE"], {}
    nid = first_node
    for k in range(2):
        for j in range(2):
            for i in range(nx + 1):
                ids[i, j, k] = nid
                lines.append(f"{nid}, {x0 + 0.3 * i:.6f}, {0.3 * j:.6f}, {0.3 * k:.6f}")
                nid += 1
    lines.append(f"*ELEMENT, type=C3D8, ELSET={name}")
    eid = first_elem
    for i in range(nx):
        h = [ids[i, 0, 0], ids[i + 1, 0, 0], ids[i + 1, 1, 0], ids[i, 1, 0], ids[i, 0, 1], ids[i + 1, 0, 1], ids[i + 1, 1, 1], ids[i, 1, 1]]
        lines.append(f"{eid}, " + ", ".join(str(n) for n in h))
        eid += 1
    i = nx if face_side > 0 else 0
    q = [ids[i, 0, 0], ids[i, 1, 0], ids[i, 1, 1], ids[i, 0, 1]]
    if face_side < 0:
        q = q[::-1]
    lines.append(f"*ELEMENT, type=CPS4, ELSET={face_name}")
    lines.append(f"{eid}, " + ", ".join(str(n) for n in q))
    return lines, nid, eid + 1


def _text():
    a, n, e = _block_lines(1, 1, -0.605, 2, "block", "front", +1)
    b, _, _ = _block_lines(101, 50, 0.0, 1, "wall", "wall_face", -1)
    return "\n".join(["** a Gmsh-style test file", *a, *b, "*NSET, NSET=rear", "1, 4, 7, 10"]) + "\n"


def test_read_inp():
    mesh = inp.read_inp(_text())
    assert len(mesh.nodes) == 12 + 8 and len(mesh.hexes) == 3
    assert mesh.parts == ["block", "wall"] and mesh.hex_part == [0, 0, 1]
    assert sorted(mesh.face_sets) == ["front", "wall_face"] and len(mesh.faces) == 2
    assert mesh.node_sets["rear"] == [0, 3, 6, 9]  # ids renumbered in order of appearance
    assert mesh.node_sets["block"] == list(range(12)) and mesh.nodes_of("wall") == list(range(12, 20))
    assert mesh.face_set_nodes("front") == [2, 5, 8, 11]
    with pytest.raises(ValueError):
        inp.read_inp("*NODE\n1, 0, 0, 0\n*ELEMENT, type=C3D8, ELSET=x\n1, 1, 2, 3, 4, 5, 6, 7, 8\n")


def test_inp_model_runs():
    mesh = inp.read_inp(_text())
    b = inp.InpModel(mesh)
    b.set_material("block", S.honeycomb(5e6, 140.0, 0.3e6, 0.2e6))
    b.set_material("wall", S.elastic(1e9, 0.3, 1000.0))
    b.set_initial_velocity("block", (10.0, 0.0, 0.0)).fix("wall")
    b.add_contact_pair("front", "wall_face", 5e6 * 0.09 / 0.3, 0.3)
    b.add_vehicle("block", 0, "front")
    m = b.build(S.settings(0.02))
    assert m.desc.n_contacts == 2 and m.desc.n_fixed == 8
    r, *_ = O.run(m.desc, simd=True)
    assert r.status == 0 and r.steps > 10
    assert r.vehicle[0].delta_v[0] < -1.0  # the wall stops the block
    assert np.isfinite(r.vehicle[0].crush)
