"""Feature coverage against the oracle (FP32 element kernels, FP64 momentum,
delta-v and crush): a T-bone (B turned 90 degrees, side sigma_y 0.15 MPa), a
rail-box front (central box 0.9 m wide over z 0.3-0.9 m, force fraction 0.7),
the rail box with densification lock-up [0.75, 50 MPa], and a case where
elements invert and erode.

Bars: without erosion, delta-v and crush within 0.5 % of both the f32 lane
restatement and the f64 scalar restatement of the reference. With erosion the
outcome depends on which elements invert first, which the f32 and f64 paths
of the reference itself decide differently (delta-v 3.9 % apart, crush by a
factor 1.3 in this case); there the device must match the f32 lane path (the
reference's production path) within 0.5 % with the same eroded count, and lie
within the f32/f64 spread of the f64 path."""
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context

from . import oracle_lib as O

pytestmark = pytest.mark.gpu

REL = 5e-3


def _runs(scen):
    m = S.Model.build(scen)
    r = Context(m.desc).run()
    r32, _, _, _, _ = O.run(m.desc, simd=True, threads=8)
    r64, _, _, _, _ = O.run(m.desc, simd=False, threads=8)
    assert r.status == 0
    return r, r32, r64


def _close(a, b, rel=REL, floor=1e-3):
    return abs(a - b) <= rel * max(abs(b), floor)


@pytest.mark.parametrize("name,scen", [
    ("t-bone", S.tbone_coverage),
    ("rail-box", lambda: S.railbox_coverage(False, 9.0)),
    ("rail-box densification", lambda: S.railbox_coverage(True, 12.0)),
])
def test_coverage_matches_oracles(name, scen):
    r, r32, r64 = _runs(scen())
    assert r.eroded_elements == 0
    for ref in (r32, r64):
        for k in range(r.n_vehicles):
            assert _close(r.vehicle[k].delta_v[0], ref.vehicle[k].delta_v[0]), (name, k, r.vehicle[k].delta_v[0], ref.vehicle[k].delta_v[0])
            assert _close(r.vehicle[k].crush, ref.vehicle[k].crush), (name, k, r.vehicle[k].crush, ref.vehicle[k].crush)


def test_erosion_case_matches_lane_path():
    r, r32, r64 = _runs(S.railbox_coverage(True, 15.0))
    assert r.eroded_elements > 0
    assert r.eroded_elements == r32.eroded_elements
    for k in range(r.n_vehicles):
        d, d32, d64 = r.vehicle[k].delta_v[0], r32.vehicle[k].delta_v[0], r64.vehicle[k].delta_v[0]
        assert _close(d, d32)
        assert abs(d - d64) <= abs(d32 - d64) + REL * abs(d64)
