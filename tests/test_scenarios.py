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


def test_two_part_vehicle_parts_and_mass():
    """The reference's two-part vehicle (add_vehicle / assign_vehicle,
    src/vehicle.rs:663-790) for the pulse-fitted Neon in the barrier model
    (src/vehicle.rs:951): body, crush zone, bumper, rail box and bumper rails
    with the rail-box factors over the element counts; coincident interface
    nodes merged; every part's mass adds up to the test mass."""
    from . import oracle_lib as O

    v = S.neon_1996_pulse()
    m = S.Model.build(S.barrier(v, 35 * S.MPH))
    part = m.hex_part()
    counts = np.bincount(part, minlength=m.desc.n_parts)
    # body 10x6x5, crush zone 14x6x5 (0.1 m along x) minus the rail box, bumper 1x6x5 minus its rails
    assert list(counts[:5]) == [300, 364, 26, 56, 4]
    assert m.desc.n_vehicles == 1 and m.desc.n_contacts == 3
    # nodes: blocks 11x7x6 + 15x7x6 + 2x7x6 with two interfaces of 7x6 merged, wall 2x6x5, road 13x9x2
    assert m.n_nodes == (462 + 630 + 84 - 2 * 42) + 60 + 234
    mats = [m.material(p) for p in range(m.desc.n_parts)]
    assert mats[0].model == abi.MAT_ELASTIC and mats[0].youngs_modulus == 2.7e8 and mats[0].poisson_ratio == 0.3
    assert mats[1].model == abi.MAT_HONEYCOMB and mats[3].model == abi.MAT_HONEYCOMB
    f_rails, f_skin = 0.8 / (56 / 420), 0.2 / (1 - 56 / 420)  # Vehicle::rail_box_factors
    assert abs(mats[3].youngs_modulus / mats[1].youngs_modulus - f_rails / f_skin) < 1e-9 * f_rails / f_skin
    assert abs(mats[4].youngs_modulus / mats[2].youngs_modulus - f_rails / f_skin) < 1e-9 * f_rails / f_skin
    lumped, _ = O.Session(m.desc).masses()
    nodes, _, front = m.vehicle(0)
    assert abs(lumped[nodes].sum() - 1354.0) < 1e-9 * 1354.0
    x = m.positions()
    assert np.all(x[front, 0] == x[front, 0].max())  # the bumper's front face, heading +x
    assert len(np.unique(x[nodes].round(9), axis=0)) == len(nodes)  # no coincident nodes left


def test_two_part_headon_builds_both_headings():
    a, b = S.neon_1996_pulse(), S.lincoln_navigator_1999()
    m = S.Model.build(S.scenario(a, b, 13.4, 13.4, element_size=0.3))
    x = m.positions()
    for k, sign in ((0, 1.0), (1, -1.0)):
        nodes, accel, front = m.vehicle(k)
        # the front face is the vehicle's extreme along its heading, the accelerometer in its body
        ext = x[nodes, 0].max() if sign > 0 else x[nodes, 0].min()
        assert np.all(x[front, 0] == ext)
        assert sign * (x[accel, 0] - x[front, 0].mean()) < -1.0
    assert m.desc.n_contacts == 4


def test_two_part_variants_and_errors():
    """A crush zone without a bumper or rail box, a T-bone with a two-part
    striking vehicle, and the spec checks of the two-part fields."""
    from crushrs_b200.native import CrushError
    import pytest

    mat = S.honeycomb(5e6, 0.0, 0.3e6, 0.2e6)  # density from the crush zone's mass
    plain_two = S.vehicle(1500.0, (4.2, 1.8, 1.4), mat, crush_zone_length=1.2, body_modulus=2e8, crush_zone_mass=300.0)
    m = S.Model.build(S.barrier(plain_two, 15.0))
    counts = np.bincount(m.hex_part(), minlength=m.desc.n_parts)
    mats = [m.material(p) for p in range(m.desc.n_parts)]
    assert mats[0].model == abi.MAT_ELASTIC and mats[1].model == abi.MAT_HONEYCOMB and m.desc.n_parts == 4  # body, crush, wall, road
    assert counts[0] == 10 * 6 * 5 and counts[1] == 4 * 6 * 5  # 3.0 m and 1.2 m at 0.3 m
    assert abs(mats[1].density - 300.0 / (1.2 * 1.8 * 1.4)) < 1e-9 * mats[1].density
    assert abs(mats[0].density - 1200.0 / (3.0 * 1.8 * 1.4)) < 1e-9 * mats[0].density
    tb = S.Model.build(S.scenario(plain_two, S.neon_1996_tuned(), 15.0, 0.0, layout=abi.LAYOUT_TBONE))
    assert tb.desc.n_vehicles == 2 and tb.desc.n_contacts >= 2
    for bad in (dict(body_modulus=0.0), dict(crush_zone_mass=1500.0), dict(bumper=(1.5, 10.0, 1e8))):
        kw = dict(crush_zone_length=1.2, body_modulus=2e8, crush_zone_mass=300.0)
        kw.update(bad)
        with pytest.raises(CrushError):
            S.Model.build(S.barrier(S.vehicle(1500.0, (4.2, 1.8, 1.4), mat, **kw), 15.0))
