"""The contact cap on the time step (src/solver.rs:217-225 and :297): the
stable step is the smaller of the elements' limit and 2*sqrt(m/k) over every
node a contact lists (nodes with mass and contacts with stiffness only),
and each adaptive re-evaluation caps the step the same way. Cases where the
penalty springs bind (stiffness raised 100x), where one contact alone binds,
where a contact of zero stiffness is skipped and where the elements bind;
the oracle's first steps against the formula on its own lumped masses, and
(GPU) the engine's steps against the oracle's, alone and in one batch."""
import numpy as np
import pytest

from crushrs_b200 import scenarios as S

from . import oracle_lib as O

STEPS = 12


def _model(scale):
    """Small seeded head-on; `scale` multiplies each contact's stiffness
    (a number for all, or one per contact)."""
    m = S.Model.build(S.batch_headon(0))
    d = m.desc
    scales = scale if isinstance(scale, (list, tuple)) else [scale] * d.n_contacts
    for c in range(d.n_contacts):
        d.contacts[c].stiffness *= scales[c]
    d.settings.max_steps = STEPS
    return m


def _caps(d):
    """(element limit, contact limit) on the undeformed mesh, from the
    oracle's elements and lumped masses."""
    s = O.Session(d)
    lumped, _ = s.masses()
    element = s.stable_dt(np.zeros(3 * d.n_nodes))
    contact = np.inf
    for c in range(d.n_contacts):
        k = d.contacts[c].stiffness
        nodes = np.ctypeslib.as_array(d.contacts[c].nodes, (d.contacts[c].n_nodes,))
        m = lumped[nodes]
        m = m[m > 0.0]
        if k > 0.0 and m.size:
            contact = min(contact, 2.0 * float(np.sqrt(m.min() / k)))
    return element, contact


CASES = {
    "contact binds": 100.0,
    "one contact binds": [1.0, 1.0, 400.0, 1.0],
    "zero stiffness skipped": [0.0, 0.0, 400.0, 400.0],
    "elements bind": 1.0,
}


@pytest.mark.parametrize("case", list(CASES))
def test_oracle_step_is_the_capped_stable_step(case):
    m = _model(CASES[case])
    d = m.desc
    element, contact = _caps(d)
    if case == "elements bind":
        assert element < contact
    else:
        assert contact < 0.9 * element
    r, _, _, dts, _ = O.run(d, want_dt=STEPS)
    assert r.steps == STEPS
    want = d.settings.dt_scale * min(element, contact)
    # every step of the window: the first, and the adaptive re-evaluations
    # at steps 5 and 10 cap it the same way
    assert np.all(dts == want), (dts, want)
    assert r.dt_min == want


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_engine_step_equals_the_oracle(case):
    from crushrs_b200.engine import Context

    m = _model(CASES[case])
    d = m.desc
    ro, _, _, dts, _ = O.run(d, want_dt=STEPS)
    ctx = Context(d)
    r = ctx.run()
    ctx.close()
    assert r.steps == ro.steps == STEPS
    assert r.dt_min == ro.dt_min == dts[0]
    assert r.time == ro.time


@pytest.mark.gpu
def test_batch_slots_keep_their_own_contact_cap():
    """Slots of one batch take each its own cap: a binding slot's step
    does not leak into its neighbours."""
    from crushrs_b200.engine import Context

    ms = [_model(CASES[c]) for c in CASES]
    want = [O.run(m.desc)[0] for m in ms]
    ctx = Context([m.desc for m in ms])
    rs = ctx.batch_run()
    ctx.close()
    for r, ro in zip(rs, want):
        assert r.steps == ro.steps
        assert r.dt_min == ro.dt_min
        assert r.time == ro.time
