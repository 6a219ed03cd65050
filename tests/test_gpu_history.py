"""Time histories recorded on the device (crush_history_config / _get)
against the oracle's restatement of part_states and sample_accelerometers
(src/solver.rs:114-187) on the plain head-on, through the C ABI.

Bars: record steps identical; times to 1e-12 relative; part values and
accelerometer samples to 1e-9 of each column's largest magnitude (the part
sums are reduced in a fixed tree order on the device, serially in the
oracle); the last record equals the run's final state exactly where it is a
copy (positions, displacements, velocities); a crash's history in a batch is
bit-identical to its history alone."""
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


def _accelerometers(m):
    """A body-frame accelerometer on vehicle A (its accel node, frame axes to
    nodes 0.6 m along x and y) and a global one on vehicle B."""
    x = m.positions()
    d = m.desc
    va, vb = d.vehicles[0], d.vehicles[1]
    an = np.ctypeslib.as_array(va.nodes, (va.n_nodes,))
    bn = np.ctypeslib.as_array(vb.nodes, (vb.n_nodes,))
    a0 = int(va.accel_node)

    def nearest(nodes, p):
        return int(nodes[np.argmin(np.linalg.norm(x[nodes] - p, axis=1))])

    frame = (a0, nearest(an, x[a0] + [0.6, 0.0, 0.0]), nearest(an, x[a0] + [0.0, 0.6, 0.0]))
    return [([a0, frame[1]], frame), ([int(vb.accel_node), int(bn[0]), int(bn[-1])], None)]


def _close(dev, ref, rel):
    scale = np.abs(ref).reshape(-1, ref.shape[-1]).max(axis=0)
    err = np.abs(dev - ref).reshape(-1, ref.shape[-1]).max(axis=0)
    assert np.all(err <= rel * np.maximum(scale, 1e-300) + 1e-300), (err, scale)


@pytest.mark.parametrize("steps,expected", [(1, 61), (7, 10)])
def test_history_matches_oracle(steps, expected):
    m = _model(60)
    acc = _accelerometers(m)
    ctx = Context(m.desc)
    ctx.history_config(steps, 1000, acc)
    r = ctx.run()
    assert r.steps == 60
    h = ctx.history()
    o = O.run_history(m.desc, steps, acc, simd=True)
    assert h["records"] == o["records"] == expected
    assert np.array_equal(h["step"], o["step"])
    assert h["step"][0] == 0 and h["step"][-1] == 60
    np.testing.assert_allclose(h["time"], o["time"], rtol=1e-12, atol=0.0)
    assert h["parts"].shape == o["parts"].shape and h["nodes"].shape == o["nodes"].shape
    _close(h["parts"], o["parts"], 1e-9)
    _close(h["nodes"], o["nodes"], 1e-9)
    # the last record is the final state
    u, v = ctx.state()
    x = m.positions().reshape(-1)
    ids = h["node_ids"]
    last = h["nodes"][-1]
    for j, n in enumerate(ids):
        assert np.array_equal(last[j, 0:3], x[3 * n:3 * n + 3] + u[3 * n:3 * n + 3])
        assert np.array_equal(last[j, 3:6], u[3 * n:3 * n + 3])
        assert np.array_equal(last[j, 6:9], v[3 * n:3 * n + 3])
    # parts: masses are the lumped masses of the part's nodes
    mass, _ = ctx.masses()
    hexes, part = m.hexes(), m.hex_part()
    for p in range(m.desc.n_parts):
        nodes = np.unique(hexes[part == p])
        assert abs(h["parts"][-1, p, 0] - mass[nodes].sum()) <= 1e-12 * mass[nodes].sum()


def test_history_keeps_max_records_and_reruns_fresh():
    m = _model(30)
    ctx = Context(m.desc)
    ctx.history_config(1, 5, _accelerometers(m))
    ctx.run()
    h = ctx.history()
    assert h["records"] == 31 and len(h["time"]) == 5 and list(h["step"]) == [0, 1, 2, 3, 4]
    first = h["parts"].copy()
    ctx.run()  # a second run starts its history again, identically
    h2 = ctx.history()
    assert h2["records"] == 31 and np.array_equal(h2["parts"], first)


def test_history_in_a_batch_equals_alone():
    m = _model(40)
    other = S.Model.build(S.batch_headon(3))
    acc = _accelerometers(m)
    alone = Context(m.desc)
    alone.history_config(3, 100, acc)
    alone.run()
    ha = alone.history()
    b = Context([other.desc, m.desc])
    b.history_config(3, 100, acc, slot=1)
    b.batch_run()
    hb = b.history(slot=1)
    assert hb["records"] == ha["records"]
    for k in ("time", "step", "parts", "nodes"):
        assert np.array_equal(hb[k], ha[k]), k
    assert b.history(slot=0)["records"] == 0
