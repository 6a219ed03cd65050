"""Host logic of the crash server, without a GPU: every submitted request is
answered exactly once, waves respect their slot limit, and shutdown drains
the queue. (With no CUDA device every wave fails at context creation, so the
answers carry that error status; test_gpu_serve.py checks real runs.)"""
import pytest
import torch

from crushrs_b200 import abi, scenarios as S
from crushrs_b200.serve import Server, footprint

pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="exercises the no-device path")


def test_every_request_answered_once_without_a_device():
    models = [S.Model.build(S.batch_headon(i)) for i in range(10)]
    srv = Server(max_waves=2, max_wave_slots=3, hbm_budget_bytes=1e12, gather_ms=0.0)
    tickets = [srv.submit(m.desc) for m in models]
    assert len(set(tickets)) == len(tickets)
    got = {}
    for _ in range(200):
        for r in srv.poll(wait_ms=50):
            assert r.ticket not in got
            got[r.ticket] = r
        if len(got) == len(tickets):
            break
    assert set(got) == set(tickets)
    assert all(r.status == abi.CRUSH_ERR_CUDA for r in got.values())
    waves = {}
    for r in got.values():
        waves.setdefault(r.wave, []).append(r.ticket)
    assert all(len(v) <= 3 for v in waves.values())
    assert len(waves) >= 4
    st = srv.stats()
    assert st.submitted == 10 and st.completed == 10 and st.queued == 0
    srv.close()


def test_footprint_grows_with_the_model():
    plain = S.Model.build(S.plain_headon())
    refined = S.Model.build(S.refined_headon())
    assert 0 < footprint(plain.desc) < footprint(refined.desc)
    # about a kilobyte per element
    assert 1000 * refined.n_hexes < footprint(refined.desc) < 3000 * refined.n_hexes
