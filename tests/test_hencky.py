"""The oracle's restatement of the reference's Hencky elasticity and its
closed-form symmetric eigensolver, pinned by the reference's own unit tests
restated here (src/material.rs:840-931): eigen reconstruction, orthonormal
vectors, ascending values against a library eigensolver over 13 decades and
near-repeated roots; objectivity of the Hencky stress; K ln J pressure under
pure volume change; agreement with linear elasticity at small strain."""
import numpy as np

from . import oracle_lib as O


def _lcg(seed=12345):
    """The reference test's generator: 64-bit LCG, uniform in [-1, 1)."""
    s = seed
    while True:
        s = (s * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        yield ((s >> 11) / float(1 << 53)) * 2.0 - 1.0


def _rot(a, b, c):
    """Rotation from Euler angles (roll a about x, pitch b about y, yaw c about z), R = Rz Ry Rx."""
    ca, sa, cb, sb, cc, sc = np.cos(a), np.sin(a), np.cos(b), np.sin(b), np.cos(c), np.sin(c)
    rx = np.array([[1, 0, 0], [0, ca, -sa], [0, sa, ca]])
    ry = np.array([[cb, 0, sb], [0, 1, 0], [-sb, 0, cb]])
    rz = np.array([[cc, -sc, 0], [sc, cc, 0], [0, 0, 1]])
    return rz @ ry @ rx


def _check_eigen(a):
    vals, vecs = O.symmetric_eigen3(a)
    scale = max(np.linalg.norm(a), 1e-300)
    recon = vecs @ np.diag(vals) @ vecs.T
    assert np.linalg.norm(recon - a) <= 1e-12 * scale
    assert np.linalg.norm(vecs.T @ vecs - np.eye(3)) < 1e-12
    assert vals[0] <= vals[1] <= vals[2]
    ref = np.sort(np.linalg.eigvalsh(a))
    assert np.all(np.abs(vals - ref) <= 1e-12 * scale)


def test_closed_form_eigen():
    r = _lcg()
    nxt = lambda: next(r)
    for k in range(4000):
        s = 10.0 ** ((k % 13) - 6)
        m = np.array([nxt() for _ in range(9)]).reshape(3, 3)
        _check_eigen((m + m.T) * s)
    for k in range(400):
        e = 10.0 ** (-(k % 12))
        m = np.array([nxt() for _ in range(9)]).reshape(3, 3)
        _check_eigen(np.eye(3) + (m + m.T) * e)
        rot = _rot(nxt(), nxt(), nxt())
        _check_eigen(rot @ np.diag([2.0, 2.0 + e * nxt(), 0.5]) @ rot.T)
        _check_eigen(rot @ np.diag([0.3, 1.0, 1.0]) @ rot.T)
    _check_eigen(np.eye(3))
    _check_eigen(np.zeros((3, 3)))
    _check_eigen(np.diag([3.0, -1.0, 2.0]))


def test_hencky_is_objective():
    f = np.array([[0.7, 0.2, 0.0], [0.1, 1.2, 0.05], [0.0, 0.0, 1.15]])
    r = _rot(0.4, -1.1, 2.0)
    t1 = O.hencky_elastic(1e9, 0.3, f)
    t2 = O.hencky_elastic(1e9, 0.3, r @ f)
    assert np.linalg.norm(r @ t1 @ r.T - t2) / np.linalg.norm(t1) < 1e-9


def test_hencky_pressure_under_volume_change():
    k = 20e6 / (3.0 * 0.4)
    tau = O.hencky_elastic(20e6, 0.3, np.eye(3) * 0.5 ** (1.0 / 3.0))
    assert abs(np.trace(tau) / 3.0 - k * np.log(0.5)) < 1e-6 * k
    assert np.linalg.norm(tau - np.eye(3) * tau[0, 0]) < 1e-9 * abs(tau[0, 0])


def test_hencky_small_strain_is_linear_elastic():
    e, nu = 1e9, 0.3
    h = np.array([[2e-6, 3e-7, 0.0], [3e-7, -1e-6, 1e-7], [0.0, 1e-7, -5e-7]])
    tau = O.hencky_elastic(e, nu, np.eye(3) + h)
    lam = e * nu / ((1 + nu) * (1 - 2 * nu))
    mu = e / (2 * (1 + nu))
    eps = 0.5 * (h + h.T)
    lin = lam * np.trace(eps) * np.eye(3) + 2 * mu * eps
    assert np.linalg.norm(tau - lin) / np.linalg.norm(lin) < 1e-5
    assert np.all(O.hencky_elastic(e, nu, np.eye(3)) == 0.0)
