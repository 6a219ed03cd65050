"""The scenario builder (crush_scenario.h) builds the configurations the
engine is measured on: element counts, outward contact normals, the contact
pair at half stiffness per side (src/model.rs:257-265), the road, and seeded
workloads that are deterministic in their seed."""
import numpy as np

from crushrs_b200 import abi, scenarios as S


def _honeycomb_count(m):
    return sum(1 for p in m.hex_part() if m.material(p).model == abi.MAT_HONEYCOMB)


def test_plain_headon_sizes():
    m = S.Model.build(S.plain_headon())
    assert _honeycomb_count(m) == 6 * 5 * 23 + 6 * 4 * 25 == 1290
    assert m.desc.n_contacts == 4 and m.desc.n_vehicles == 2


def test_refined_headon_sizes():
    m = S.Model.build(S.refined_headon())
    assert _honeycomb_count(m) == 36 * 30 * 138 + 36 * 24 * 150 == 278640
    assert m.desc.settings.stop_rule == abi.STOP_SEPARATION


def test_contact_faces_point_out_of_their_block():
    m = S.Model.build(S.plain_headon())
    x = m.positions()
    hexes = m.hexes()
    centroid = {}
    for c in range(m.desc.n_contacts):
        nodes, faces, _, _, _ = m.contact(c)
        for f in faces[:: max(1, len(faces) // 20)]:
            p = x[f]
            n = np.cross(p[1] - p[0], p[2] - p[0])
            # the element that owns the face lies on the inner side
            owner = next(h for h in hexes if set(f) <= set(h))
            inside = x[owner].mean(axis=0)
            assert np.dot(n, p.mean(axis=0) - inside) > 0


def test_pair_contacts_split_the_stiffness():
    m = S.Model.build(S.plain_headon())
    ks = [m.contact(c)[3] for c in range(4)]
    assert ks[2] == ks[3] > 0
    assert m.contact(2)[4] == m.contact(3)[4] == 0.3


def test_seeded_workloads_are_deterministic():
    a = S.Model.build(S.batch_headon(17))
    b = S.Model.build(S.batch_headon(17))
    assert np.array_equal(a.positions(), b.positions()) and np.array_equal(a.hexes(), b.hexes())
    sizes = [_honeycomb_count(S.Model.build(S.batch_headon(i))) for i in range(40)]
    assert 250 <= min(sizes) and max(sizes) <= 7000
    kinds = [S.serve_query(i)[0] for i in range(60)]
    assert set(kinds) == set(S.SERVE_KINDS)
