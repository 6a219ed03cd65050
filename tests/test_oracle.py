"""Pins the oracle (the CPU restatement used as checker) against the
reference's own unit tests, restated with their tolerances:
  src/element.rs:203  cube_geometry
  src/element.rs:215  rank12_equals_dense_on_distorted_hex
  src/kernel.rs:356   rigid_motion_gives_zero_force (honeycomb)
  src/kernel.rs:369   uniform_crush_matches_material_law
  src/kernel.rs:389   hourglass_mode_is_resisted
  src/kernel_simd.rs:613-685 check_lane_vs_scalar (3 parameter sets, yield_at known answers)
  src/material.rs:961 honeycomb_matches_foam_in_uniaxial_crush (honeycomb assertions)
  src/material.rs:998 honeycomb_is_objective_under_superposed_rotation
No GPU is used here."""
import math

import numpy as np
import pytest

from crushrs_b200 import abi
from crushrs_b200.model import XI, single_hex
from crushrs_b200.scenarios import honeycomb

from . import oracle_lib as O

GAUSS = 0.5773502691896258


def rot_euler(roll, pitch, yaw):
    """nalgebra Rotation3::from_euler_angles: Rz(yaw) Ry(pitch) Rx(roll)."""
    cr, sr, cp, sp, cy, sy = math.cos(roll), math.sin(roll), math.cos(pitch), math.sin(pitch), math.cos(yaw), math.sin(yaw)
    rx = np.array([[1, 0, 0], [0, cr, -sr], [0, sr, cr]])
    ry = np.array([[cp, 0, sp], [0, 1, 0], [-sp, 0, cp]])
    rz = np.array([[cy, -sy, 0], [sy, cy, 0], [0, 0, 1]])
    return rz @ ry @ rx


def rot_axis(axis, angle):
    a = np.asarray(axis, float)
    a = a / np.linalg.norm(a)
    k = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * k + (1 - math.cos(angle)) * k @ k


def test_cube_geometry():
    g = O.geometry(0.5 * 0.3 * (XI + 1.0), 1e6, 0.0, 100.0, 0.1)
    assert abs(g["volume"] - 0.027) < 1e-12
    assert np.all(np.abs(g["lumped"] - 100.0 * 0.027 / 8.0) < 1e-12)
    assert abs(g["grad"][0, 0] + 1.0 / 1.2) < 1e-12


def _dense_k(x, e_hg, nu):
    """K = sum_gp (B_gp - B_c)^T C (B_gp - B_c) det J, restating the test's own K."""
    def dn(xi, eta, zeta):
        s = XI
        return np.stack([0.125 * s[:, 0] * (1 + s[:, 1] * eta) * (1 + s[:, 2] * zeta),
                         0.125 * s[:, 1] * (1 + s[:, 0] * xi) * (1 + s[:, 2] * zeta),
                         0.125 * s[:, 2] * (1 + s[:, 0] * xi) * (1 + s[:, 1] * eta)], axis=1)

    def grads(d):
        j = d.T @ x
        return d @ np.linalg.inv(j).T, np.linalg.det(j)

    def bmat(g):
        b = np.zeros((6, 24))
        for i in range(8):
            n0, n1, n2 = g[i]
            b[0, 3 * i], b[1, 3 * i + 1], b[2, 3 * i + 2] = n0, n1, n2
            b[3, 3 * i], b[3, 3 * i + 1] = n1, n0
            b[4, 3 * i + 1], b[4, 3 * i + 2] = n2, n1
            b[5, 3 * i], b[5, 3 * i + 2] = n2, n0
        return b

    lam = e_hg * nu / ((1 + nu) * (1 - 2 * nu))
    mu = e_hg / (2 * (1 + nu))
    c = np.zeros((6, 6))
    c[:3, :3] = lam
    for i in range(3):
        c[i, i] = lam + 2 * mu
        c[i + 3, i + 3] = mu
    gc, _ = grads(dn(0, 0, 0))
    bc = bmat(gc)
    k = np.zeros((24, 24))
    for s in XI:
        g, dj = grads(dn(*(s * GAUSS)))
        db = bmat(g) - bc
        k += db.T @ c @ db * dj
    return k


def _hg_force(gamma, h, u):
    u_mat = u.reshape(8, 3).T  # 3 x 8
    q = u_mat @ gamma  # 3 x 4
    r = h @ q.T.reshape(12)  # q[3 a + d]
    return (r.reshape(4, 3).T @ gamma.T).T.reshape(24)


def test_rank12_equals_dense_on_distorted_hex():
    x = np.array([0.0, 0.0, 0.0, 1.2, 0.1, 0.0, 1.1, 0.9, 0.1, -0.1, 1.0, 0.0, 0.1, 0.0, 1.0, 1.0, 0.2, 1.1, 1.3, 1.1, 0.9, 0.0, 0.8, 1.2]).reshape(8, 3)
    g = O.geometry(x, 20e6, 0.0, 200.0, 0.1)
    k = _dense_k(x, 0.1 * 20e6, 0.0)
    u = np.array([((i * 7 % 11) - 5.0) * 1e-3 for i in range(24)])
    f = _hg_force(g["gamma"], g["h"], u)
    dense = k @ u
    assert np.linalg.norm(f - dense) < 1e-9 * np.linalg.norm(dense)
    a = rot_euler(0.3, -0.7, 1.1) @ np.array([[1.1, 0.05, 0.0], [0.0, 0.9, 0.02], [0.0, 0.0, 1.05]])
    u2 = (x @ a.T - x).reshape(24)
    f2 = _hg_force(g["gamma"], g["h"], u2)
    assert np.linalg.norm(f2) < 1e-8 * np.linalg.norm(dense)


def _displacement(nodes, a, c):
    return (nodes @ a.T + c - nodes).reshape(24)


def test_rigid_motion_gives_zero_force():
    m = single_hex(honeycomb(20e6, 200.0, 0.2e6, 0.5e6))
    s = O.Session(m.desc, simd=False)
    r = rot_euler(0.4, 1.2, -0.8)
    u = _displacement(m.positions, r, np.array([3.0, -1.0, 2.0]))
    g, _ = s.forces(u)
    assert np.linalg.norm(g) < 1e-3


def test_uniform_crush_matches_material_law():
    m = single_hex(honeycomb(20e6, 200.0, 0.2e6, 0.5e6))
    s = O.Session(m.desc, simd=False)
    for k in range(1, 101):
        a = np.diag([1.0 - 0.4 * k / 100.0, 1.0, 1.0])
        g, _ = s.forces(_displacement(m.positions, a, np.zeros(3)))
    fx_face = sum(g[3 * i] for i in (1, 2, 5, 6))
    st, _ = s.get_state()
    c = float(st[0, 24])
    sigma_y = 0.2e6 + 0.5e6 * c
    assert abs(fx_face + sigma_y) < 1e-6 * sigma_y + 0.05  # compaction read back as f32
    expected = -math.log(0.6) - sigma_y / 20e6
    assert abs(c - expected) < 2e-3


def test_hourglass_mode_is_resisted():
    m = single_hex(honeycomb(20e6, 200.0, 0.2e6, 0.5e6))
    s = O.Session(m.desc, simd=False)
    hmode = [1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0]
    u = np.zeros(24)
    for i in range(8):
        u[3 * i] = 1e-3 * hmode[i]
    g, _ = s.forces(u)
    assert np.linalg.norm(g) > 1.0
    st, _ = s.get_state()
    assert st[0, 24] == 0.0


def _check_lane_vs_scalar(mat):
    """src/kernel_simd.rs:613-662: a 0.3 m cube crushed over 200 steps through
    the f32 lane kernel and the f64 rate update."""
    cube = 0.15 * (XI + 1.0)
    m = single_hex(mat, nodes=cube)
    s = O.Session(m.desc, simd=True)
    grad = XI / (4.0 * 0.3)
    s.set_lane_geometry(grad.reshape(1, 24), np.array([0.027]), np.zeros((1, 32)), np.zeros((1, 144)))
    knots_yield = lambda c: O.yield_at(mat, c)[0][0]
    state = O.default_state()
    for step in range(1, 201):
        c = 0.5 * step / 200.0
        u = np.zeros(24)
        for i in (1, 2, 5, 6):
            u[3 * i] = -c * 0.3
            u[3 * i + 1] = 0.02 * c * 0.3
        out, _ = s.forces(u)
        f = np.zeros((3, 3))
        for i in range(8):
            xi = cube[i] + u[3 * i:3 * i + 3]
            f += np.outer(xi, grad[i])
        tau, state = O.honeycomb_update(mat, f, state)
        mm = tau @ np.linalg.inv(f).T * 0.027
        lane, _ = s.get_state()
        floor = 1e-6 * mat.youngs_modulus + 2e-3 * knots_yield(state[24])
        assert abs(lane[0, 24] - state[24]) < 1e-3 * max(state[24], 1e-6) + 1e-6, step
        assert np.all(np.abs(lane[0, 18:24] - state[18:24]) < floor), step
        for i in range(8):
            fi = mm @ grad[i]
            assert np.all(np.abs(out[3 * i:3 * i + 3] - fi) < floor * 0.027 / 0.3), (step, i)
    assert state[24] > 0.3


def test_lane_kernel_matches_scalar_reference():
    mat = honeycomb(125.8e6, 100.0, 1234.0, 800339.0)  # HoneycombParams::new(E, sigma_y, H)
    _check_lane_vs_scalar(mat)


def test_lane_kernel_matches_scalar_with_tabulated_curve():
    mat = honeycomb(23.1e6, 100.0, curve=[(0.0, 7000.0), (0.05, 10000.0), (0.15, 6000.0), (0.3, 30000.0), (0.45, 30000.0)],
                    densification=(1.0, 2.0e6))
    close = lambda a, b: abs(a[0] - b[0]) < 1e-9 * max(abs(b[0]), 1.0) and abs(a[1] - b[1]) < 1e-9 * max(abs(b[1]), 1.0)
    for c, want in [(0.0, (7000.0, 60000.0)), (0.1, (8000.0, -40000.0)), (0.6, (30000.0, 0.0)), (1.5, (30000.0 + 1.0e6, 2.0e6))]:
        knots, curve = O.yield_at(mat, c)
        assert close(knots, want), (c, knots)
    for c in (1.5, 0.1):
        knots, curve = O.yield_at(mat, c)
        assert close(curve, knots)
    _check_lane_vs_scalar(mat)
    mat.transverse_factor = 4.0
    _check_lane_vs_scalar(mat)


def test_honeycomb_uniaxial_crush():
    mat = honeycomb(20e6, 200.0, 0.2e6, 0.5e6)
    st = O.default_state()
    f = np.eye(3)
    tau = None
    for k in range(1, 201):
        f[0, 0] = 1.0 - 0.6 * k / 200.0
        tau, st = O.honeycomb_update(mat, f, st)
    # Hencky foam compaction in closed form: c = -ln(0.4) - sigma_y(c) / E.
    c_foam = -math.log(0.4)
    for _ in range(100):
        c_foam = -math.log(0.4) - (0.2e6 + 0.5e6 * c_foam) / 20e6
    assert abs(st[24] - c_foam) < 2e-2 * c_foam
    j = np.linalg.det(f)
    sigma_y = 0.2e6 + 0.5e6 * st[24]
    assert abs(tau[0, 0] / j + sigma_y) < 1e-6 * sigma_y
    assert abs(tau[1, 1]) < 1e-6 * abs(tau[0, 0])
    tau2, st2 = O.honeycomb_update(mat, f, st)
    assert np.linalg.norm(tau2 - tau) < 1e-9 * np.linalg.norm(tau)
    assert st2[24] == st[24]
    f2 = f.copy()
    f2[0, 0] += 0.01
    tau3, st3 = O.honeycomb_update(mat, f2, st)
    assert tau3[0, 0] > tau[0, 0]
    assert st3[24] == st[24]


def test_honeycomb_is_objective_under_superposed_rotation():
    mat = honeycomb(20e6, 200.0, 0.2e6, 0.5e6)
    st = O.default_state()
    f0 = np.diag([0.7, 1.0, 1.0])
    f = np.eye(3)
    for k in range(1, 101):
        f = np.eye(3) + (f0 - np.eye(3)) * (k / 100.0)
        _, st = O.honeycomb_update(mat, f, st)
    tau0, _ = O.honeycomb_update(mat, f, st)
    c0 = st[24]
    axis = (0.3, -0.5, 0.8)
    tau = tau0
    for k in range(1, 201):
        r = rot_axis(axis, 1.2 * k / 200.0)
        tau, st = O.honeycomb_update(mat, r @ f, st)
    r = rot_axis(axis, 1.2)
    assert np.linalg.norm(tau - r @ tau0 @ r.T) < 1e-4 * np.linalg.norm(tau0)
    assert abs(st[24] - c0) < 1e-6


def test_characteristic_length_of_box():
    p = 0.5 * (XI + 1.0) * np.array([0.4, 0.3, 0.2])
    l, v = O.char_length(p)
    assert abs(v - 0.024) < 1e-15 and abs(l - 0.2) < 1e-15
    inverted = p.copy()
    inverted[4:, 2] = -0.1
    l, v = O.char_length(inverted)
    assert math.isinf(l) and v < 0
