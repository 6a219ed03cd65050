"""The contact broad phase is exact: runs with the grids (static grids for
fixed faces, hierarchical hashed grids for moving ones) give bit-identical
results to runs where every search tests every face of its contact, as the
reference's ContactRuntime::apply does (src/contact.rs:115). Covers the
refined head-on through erosion and the crushed late phase, where faces get
large, warped and tangled."""
import numpy as np
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context
from crushrs_b200.model import XI, ArrayModel

from . import oracle_lib as O

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


def _heavy_contact_model(sides=(5, 55), seed=11):
    """One honeycomb cube whose top face (nodes 4-7) is the only face of two
    contacts, with k x k free primary nodes just under it at seeded depths:
    every node hits, so each face corner takes k^2 reaction events, above
    the 16 a contact node's own list holds (5 x 5: the block-sorted heavy
    gather) and above 2048 (55 x 55: the walk over the contact's entries)."""
    rng = np.random.default_rng(seed)
    pts = [0.5 * (XI + 1.0)]
    contacts = []
    base = 8
    for k in sides:
        g = (np.arange(k) + 0.5) / k
        X, Y = np.meshgrid(g, g, indexing="ij")
        z = 1.0 - rng.uniform(0.002, 0.05, k * k)
        pts.append(np.stack([X.ravel(), Y.ravel(), z], 1))
        contacts.append({"nodes": np.arange(base, base + k * k), "faces": [[4, 5, 6, 7]], "stiffness": 1e7,
                         "max_distance": 0.1})
        base += k * k
    return ArrayModel(np.concatenate(pts), np.arange(8), [0], [S.honeycomb(1e8, 100.0, yield_stress=1e6)],
                      contacts=contacts)


def test_heavy_nodes_match_oracle():
    """Drop-in contact on one stream with face corners that take 25 and
    3025 reaction events: forces equal to the oracle's ordered sums."""
    m = _heavy_contact_model()
    n = m.n_nodes
    masses = np.random.default_rng(3).uniform(0.005, 0.02, n)
    u = np.zeros(3 * n)
    ctx = Context(m.desc)
    s = O.Session(m.desc)
    for c in range(2):
        fd = np.zeros(3 * n)
        cnt_d, mp_d = ctx.contact_apply(c, u, None, masses, 1e-5, fd)
        fo, cnt_o, mp_o = s.contact_apply(c, u, np.zeros(3 * n), masses, 1e-5, np.zeros(3 * n))
        assert cnt_d == cnt_o == m._contacts[c][0].shape[0]
        assert mp_d == mp_o
        assert np.all(fo[3 * 4 + 2:3 * 8:3] != 0.0)  # the corners' normal (z) reactions
        assert np.allclose(fd, fo, rtol=1e-12, atol=1e-12 * np.abs(fo).max())
    ctx.close()
