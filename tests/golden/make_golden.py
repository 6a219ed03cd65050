"""Generates the golden fixtures of tests/golden/ from the oracle (the CPU
restatement of the reference's kernels): nodal force vectors of the f32 lane
kernel and of the f64 scalar kernel on seeded states, and end-of-run results.

    python tests/golden/make_golden.py

Cases:
  hex1      one distorted honeycomb hexahedron, seeded displacement (three
            successive calls, so committed material state is exercised);
  block8    a 2x2x2 block of honeycomb hexahedra, seeded displacement;
  plain     the plain head-on model (1290 hexahedra), both noses pushed into
            each other plus seeded noise;
  runs      end-of-run delta-v, crush, steps and eroded count of the plain
            head-on (f32 lane and f64 scalar paths).
The fixtures pin the oracle against later changes (tests/test_golden.py) and
give the GPU tests fixed expected forces without running the oracle."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from crushrs_b200 import scenarios as S  # noqa: E402
from crushrs_b200.model import ArrayModel  # noqa: E402
from tests import oracle_lib as O  # noqa: E402

SEED = 20261203


def hex1_model():
    x = np.array([[0, 0, 0], [1.1, 0.05, 0], [1.0, 0.9, 0.1], [-0.05, 1.0, 0], [0.02, 0, 1.0], [1.0, -0.05, 1.1], [1.05, 1.0, 0.95],
                  [0, 1.1, 1.0]], float) * 0.3
    mat = S.honeycomb(5e6, 120.0, 0.3e6, 0.2e6, densification=(0.8, 5e6))
    return ArrayModel(x, np.arange(8)[None, :], [0], [mat])


def block8_model():
    h = 0.25
    idx = {}
    pts = []
    for k in range(3):
        for j in range(3):
            for i in range(3):
                idx[(i, j, k)] = len(pts)
                pts.append((i * h, j * h, k * h))
    hexes = []
    for k in range(2):
        for j in range(2):
            for i in range(2):
                c = [(i, j, k), (i + 1, j, k), (i + 1, j + 1, k), (i, j + 1, k), (i, j, k + 1), (i + 1, j, k + 1), (i + 1, j + 1, k + 1),
                     (i, j + 1, k + 1)]
                hexes.append([idx[q] for q in c])
    curve = [(k * 0.8 / 7.0, 0.3e6 + k * (0.9e6 / 7.0)) for k in range(8)]
    mat = S.honeycomb(5e6, 140.0, curve=curve, transverse=4.0)
    return ArrayModel(np.array(pts), hexes, [0] * 8, [mat])


def crush_field(desc, rng, amp):
    x = np.ctypeslib.as_array(desc.positions, (desc.n_nodes, 3))
    near = np.exp(-np.abs(x[:, 0]) / 0.6)
    u = np.zeros((desc.n_nodes, 3))
    u[:, 0] = -np.sign(x[:, 0]) * amp * near
    u += rng.normal(scale=amp * 0.02, size=u.shape) * near[:, None]
    if desc.n_fixed:
        u[np.ctypeslib.as_array(desc.fixed_nodes, (desc.n_fixed,))] = 0.0
    return u.reshape(-1)


def forces_sequence(desc, us, simd):
    s = O.Session(desc, simd=simd)
    out = []
    for u in us:
        f, _ = s.forces(u)
        out.append(f)
    return np.array(out)


def main():
    rng = np.random.default_rng(SEED)
    data = {}
    m1 = hex1_model()
    us = [rng.normal(scale=s, size=24) for s in (0.002, 0.01, 0.02)]
    data["hex1_u"] = np.array(us)
    data["hex1_f32"] = forces_sequence(m1.desc, us, True)
    data["hex1_f64"] = forces_sequence(m1.desc, us, False)
    m8 = block8_model()
    us = [rng.normal(scale=0.01, size=3 * m8.desc.n_nodes), rng.normal(scale=0.03, size=3 * m8.desc.n_nodes)]
    data["block8_u"] = np.array(us)
    data["block8_f32"] = forces_sequence(m8.desc, us, True)
    data["block8_f64"] = forces_sequence(m8.desc, us, False)
    plain = S.Model.build(S.plain_headon())
    us = [crush_field(plain.desc, rng, 0.2), crush_field(plain.desc, rng, 0.35)]
    data["plain_u"] = np.array(us)
    data["plain_f32"] = forces_sequence(plain.desc, us, True)
    data["plain_f64"] = forces_sequence(plain.desc, us, False)
    for tag, simd in (("f32", True), ("f64", False)):
        r, _, _, _, _ = O.run(plain.desc, simd=simd, threads=8)
        data[f"run_{tag}"] = np.array([r.steps, r.eroded_elements] + [r.vehicle[k].delta_v[0] for k in range(2)] +
                                      [r.vehicle[k].crush for k in range(2)])
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **data)
    print({k: v.shape for k, v in data.items()})


if __name__ == "__main__":
    main()
