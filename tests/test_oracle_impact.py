"""The reference's own end-to-end assertions (tests/impact.rs:33-47,
`head_on_conserves_momentum_with_plausible_delta_v`) restated on the oracle:
the tuned Silverado and Neon head-on at 30 mph each (0.3 m elements, no
road, 0.15 s) conserves momentum to round-off, the car's delta-v lies
between the perfectly plastic limit and 1.3 times it, the restitution is in
(0, 0.3) and no element erodes. Both oracle paths (f32 lane, f64 scalar)."""
import pytest

from crushrs_b200 import scenarios as S

from . import oracle_lib as O


def impact_checks(r):
    mt, dvt = r.vehicle[0].mass, r.vehicle[0].delta_v[0]
    mc, dvc = r.vehicle[1].mass, r.vehicle[1].delta_v[0]
    v0 = 30.0 * S.MPH
    assert abs(mt * dvt + mc * dvc) < 1e-6 * mt * v0, (mt * dvt + mc * dvc)
    v_common = (mt * v0 - mc * v0) / (mt + mc)
    plastic = v_common + v0
    assert plastic < dvc < 1.3 * plastic, (dvc, plastic)
    e = ((dvc - v0) - (v0 + dvt)) / (2.0 * v0)
    assert 0.0 < e < 0.3, e
    assert r.eroded_elements == 0


@pytest.mark.parametrize("simd", [True, False])
def test_head_on_conserves_momentum_with_plausible_delta_v(simd):
    m = S.Model.build(S.crash_30_30())
    r, _, _, _, _ = O.run(m.desc, simd=simd, threads=8)
    assert r.status == 0
    impact_checks(r)
