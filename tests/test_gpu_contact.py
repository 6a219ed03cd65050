"""The contact broad phase is exact: runs with the grids (static grids for
fixed faces, hierarchical hashed grids for moving ones) give bit-identical
results to runs where every search tests every face of its contact, as the
reference's ContactRuntime::apply does (src/contact.rs:115). Covers the
refined head-on through erosion and the crushed late phase, where faces get
large, warped and tangled."""
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context

pytestmark = pytest.mark.gpu


def _run(desc, exhaustive):
    ctx = Context(desc)
    ctx.set_contact_search(exhaustive)
    r = ctx.run()
    stats = [ctx.contact_search_stats(c) for c in range(desc.n_contacts)]
    ctx.close()
    return r, stats


def _same(a, b):
    assert (a.steps, a.time, a.eroded_elements, a.status) == (b.steps, b.time, b.eroded_elements, b.status)
    for k in range(a.n_vehicles):
        assert list(a.vehicle[k].delta_v) == list(b.vehicle[k].delta_v)
        assert a.vehicle[k].crush == b.vehicle[k].crush


@pytest.mark.parametrize("scenario", [S.plain_headon, S.crash_30_30, lambda: S.batch_headon(3)])
def test_grid_equals_exhaustive_small(scenario):
    m = S.Model.build(scenario())
    g, stats = _run(m.desc, False)
    e, _ = _run(m.desc, True)
    _same(g, e)
    assert all(s[0] == 0 for s in stats)  # no search fell back to every face


def test_grid_equals_exhaustive_refined_headon():
    m = S.Model.build(S.refined_headon(max_steps=3000))
    g, stats = _run(m.desc, False)
    e, _ = _run(m.desc, True)
    assert g.eroded_elements > 0  # the crushed phase is covered
    _same(g, e)
