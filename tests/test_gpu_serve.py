"""The crash server on the GPU: crashes submitted at random times are
admitted into running serving contexts (continuous batching) and into
contexts that overlap on the device, and each result equals the same model
run alone (bit-identical f64 results; added_mass_max to 1e-12 relative, as
in test_gpu_batch.py)."""
import pytest

from crushrs_b200 import scenarios as S
from crushrs_b200.engine import Context
from crushrs_b200.serve import Server, footprint, open_loop

from .test_gpu_batch import _same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def queries():
    return [S.Model.build(S.serve_query(i, e_range=(300, 3000))[1]) for i in range(24)]


@pytest.fixture(scope="module")
def alone(queries):
    out = []
    for m in queries:
        ctx = Context(m.desc)
        out.append(ctx.run())
        ctx.close()
    return out


def test_served_results_equal_alone(queries, alone):
    with Server(max_waves=3, max_wave_slots=5, gather_ms=1.0) as srv:
        results, wall, tickets = open_loop(srv, queries, rate=400.0, seed=3)
        st = srv.stats()
    assert len(results) == len(queries)
    assert st.waves >= 5
    for t, r in results.items():
        assert r.status == 0
        _same(r.results, alone[tickets[t]])
    waves = {}
    for r in results.values():
        waves.setdefault(r.wave, []).append(r)
    # contexts overlapped in time
    spans = sorted((min(x.start_s for x in v), max(x.finish_s for x in v)) for v in waves.values())
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    # crashes joined a context while others of it were running
    assert any(b.start_s > a.start_s and b.start_s < a.finish_s for v in waves.values() for a in v for b in v)


def test_admission_respects_the_memory_budget(queries, alone):
    budget = 2.5 * max(footprint(m.desc) for m in queries[:8])
    with Server(max_waves=4, hbm_budget_bytes=budget, gather_ms=0.0) as srv:
        tickets = {srv.submit(m.desc): i for i, m in enumerate(queries[:8])}
        got = {}
        while len(got) < len(tickets):
            for r in srv.poll(wait_ms=50):
                got[r.ticket] = r
        st = srv.stats()
    assert st.peak_bytes_in_use <= budget
    for t, r in got.items():
        _same(r.results, alone[tickets[t]])


def test_queue_limit_refuses_and_serves_the_rest(queries, alone):
    """Admission control: with max_queue requests waiting, a submit is
    refused (None) and copies nothing; every accepted request is answered
    once, with its alone results, and refusals stop once the queue drains."""
    with Server(max_waves=2, max_wave_slots=4, gather_ms=0.0, max_queue=2) as srv:
        tickets = {}
        refused = 0
        for i, m in enumerate(queries):
            t = srv.submit(m.desc)
            if t is None:
                refused += 1
            else:
                tickets[t] = i
        got = {}
        while len(got) < len(tickets):
            for r in srv.poll(wait_ms=50):
                assert r.ticket not in got
                got[r.ticket] = r
        late = srv.submit(queries[0].desc)  # the queue has drained
        assert late is not None
        while late not in got:
            for r in srv.poll(wait_ms=50):
                got[r.ticket] = r
    assert refused + len(tickets) == len(queries) and len(tickets) >= 2
    for t, i in tickets.items():
        _same(got[t].results, alone[i])
    _same(got[late].results, alone[0])
