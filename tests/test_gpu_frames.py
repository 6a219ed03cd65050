"""Frames captured on the device (crush_frames_config / crush_frame_get)
against the oracle's restatement of the frame capture of crushrs::run
(src/solver.rs:265-281; plastic_strain and cauchy_stress,
src/kernel.rs:269-321) on the plain head-on, through the C ABI.

Bars: frame steps and erosion flags identical; times to 1e-12 relative;
displacements (f32) to 1e-6 and stresses (f32 of an f64 R sigma R^T) to 1e-5
of the field's largest magnitude; plastic strain to 1e-6; the last frame's
displacement is the f32 of the run's final u exactly."""
import numpy as np
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context

from . import oracle_lib as O

pytestmark = pytest.mark.gpu


def _model(max_steps):
    m = S.Model.build(S.plain_headon())
    m.settings.max_steps = max_steps
    m.refresh()
    return m


@pytest.mark.parametrize("steps,expected", [(20, [0, 20, 40, 60]), (25, [0, 25, 50, 60])])
def test_frames_match_oracle(steps, expected):
    m = _model(60)
    ctx = Context(m.desc)
    ctx.frames_config(steps, 16)
    ctx.run()
    n = ctx.frames_count()
    o = O.run_frames(m.desc, steps)
    assert n == o["frames"] == len(expected)
    assert list(o["step"]) == expected
    for k in range(n):
        f = ctx.frame(k)
        assert f["step"] == expected[k]
        assert abs(f["time"] - o["time"][k]) <= 1e-12 * max(o["time"][k], 1e-30)
        assert np.array_equal(f["eroded"], o["eroded"][k])
        for key, rel in (("displacement", 1e-6), ("stress", 1e-5)):
            ref = o[key][k]
            scale = max(np.abs(ref).max(), 1e-30)
            assert np.abs(f[key] - ref).max() <= rel * scale, (key, k)
        assert np.abs(f["plastic_strain"] - o["plastic_strain"][k]).max() <= 1e-6
    stress = ctx.frame(n - 1)["stress"]
    assert np.abs(stress).max() > 0.0  # the noses are crushing by step 60
    u, _ = ctx.state()
    assert np.array_equal(ctx.frame(n - 1)["displacement"].reshape(-1), u.astype(np.float32))


def test_frames_keep_max_and_count_the_rest():
    m = _model(60)
    ctx = Context(m.desc)
    ctx.frames_config(10, 2)
    ctx.run()
    assert ctx.frames_count() == 7
    assert ctx.frame(1)["step"] == 10
    with pytest.raises(Exception):
        ctx.frame(2)
