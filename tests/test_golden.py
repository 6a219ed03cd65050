"""Golden fixtures (tests/golden/golden.npz, made by tests/golden/make_golden.py
from the oracle): the oracle must keep reproducing them exactly (CPU), and
the CUDA engine must reproduce the f32 lane forces bit for bit, stay within
1e-5 norm-relative of them and within 1e-4 of the f64 scalar forces, and end
the plain head-on within 0.5 % of the recorded delta-v and crush (GPU)."""
import os

import numpy as np
import pytest

from crushrs_b200 import abi, scenarios as S

from . import oracle_lib as O
from .golden.make_golden import block8_model, hex1_model

GOLDEN = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))


def _models():
    return {"hex1": hex1_model(), "block8": block8_model(), "plain": S.Model.build(S.plain_headon())}


@pytest.mark.parametrize("case", ["hex1", "block8", "plain"])
def test_oracle_reproduces_golden_forces(case):
    m = _models()[case]
    for tag, simd in (("f32", True), ("f64", False)):
        s = O.Session(m.desc, simd=simd)
        for u, f_ref in zip(GOLDEN[f"{case}_u"], GOLDEN[f"{case}_{tag}"]):
            f, _ = s.forces(u)
            assert np.array_equal(f, f_ref), (case, tag)


def test_oracle_reproduces_golden_run():
    m = S.Model.build(S.plain_headon())
    r, _, _, _, _ = O.run(m.desc, simd=True, threads=8)
    got = np.array([r.steps, r.eroded_elements] + [r.vehicle[k].delta_v[0] for k in range(2)] + [r.vehicle[k].crush for k in range(2)])
    assert np.array_equal(got, GOLDEN["run_f32"])


def _elastic_dofs(d):
    """Degrees of freedom of the nodes of elastic elements."""
    hexes = np.ctypeslib.as_array(d.hexes, (d.n_hexes, 8))
    part = np.ctypeslib.as_array(d.hex_part, (d.n_hexes,))
    elastic = np.array([d.materials[p].model == abi.MAT_ELASTIC for p in part])
    mask = np.zeros(d.n_nodes, bool)
    mask[hexes[elastic].ravel()] = True
    return np.repeat(mask, 3)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["hex1", "block8", "plain"])
def test_device_forces_match_golden(case):
    from crushrs_b200.engine import Context

    m = _models()[case]
    ctx = Context(m.desc)
    el = _elastic_dofs(m.desc)
    for u, f32, f64 in zip(GOLDEN[f"{case}_u"], GOLDEN[f"{case}_f32"], GOLDEN[f"{case}_f64"]):
        f = np.zeros_like(f32)
        ctx.compute_forces(u, f)
        # bit-equal where only honeycomb elements act; the elastic road's
        # f64 forces (round-off of F = I here) to 1e-9 of the largest force
        assert np.array_equal(f[~el], f32[~el]), case
        assert np.abs(f[el] - f32[el]).max(initial=0.0) <= 1e-9 * np.abs(f32).max(), case
        assert np.linalg.norm(f - f32) <= 1e-5 * np.linalg.norm(f32)
        assert np.linalg.norm(f - f64) <= 1e-4 * np.linalg.norm(f64)


@pytest.mark.gpu
def test_device_run_matches_golden():
    from crushrs_b200.engine import Context

    m = S.Model.build(S.plain_headon())
    r = Context(m.desc).run()
    for tag in ("run_f32", "run_f64"):
        g = GOLDEN[tag]
        for k in range(2):
            assert abs(r.vehicle[k].delta_v[0] - g[2 + k]) <= 5e-3 * abs(g[2 + k])
            assert abs(r.vehicle[k].crush - g[4 + k]) <= 5e-3 * max(abs(g[4 + k]), 1e-3)
