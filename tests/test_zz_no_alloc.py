"""crush_contact_apply_static (the allocation-free contact call) against
crush_contact_apply on the same contacts and displacements: forces, the
penetration count and the largest penetration bit-identical, on two calls in
a row with different displacement fields (the second call must not see the
first one's scratch). The file name sorts last so these run after every
other GPU test, in the same process, as well as alone."""
import ctypes as C

import numpy as np
import pytest

from crushrs_b200 import abi, scenarios as S
from crushrs_b200.engine import Context, contact_apply_static
from crushrs_b200.native import CrushError

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _field(desc, seed, amp):
    """Both blocks pushed nose-first into each other plus small noise, so
    nodes near the interface and the road penetrate faces."""
    rng = np.random.default_rng(seed)
    x = np.ctypeslib.as_array(desc.positions, (desc.n_nodes, 3))
    near = np.exp(-np.abs(x[:, 0]) / 0.6)
    u = np.zeros((desc.n_nodes, 3))
    u[:, 0] = -np.sign(x[:, 0]) * amp * near
    u[:, 2] = -0.5 * amp * near
    u += rng.normal(scale=amp * 0.02, size=u.shape) * near[:, None]
    if desc.n_fixed:
        u[np.ctypeslib.as_array(desc.fixed_nodes, (desc.n_fixed,))] = 0.0
    return u.reshape(-1)


def _dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype=dtype, device="cuda")


class _Static:
    """Device copies of one model's arrays for the static call."""

    def __init__(self, model, masses):
        self.model = model
        self.n = model.n_nodes
        self.pos = _dev(model.positions().reshape(-1), torch.float64)
        self.masses = _dev(masses, torch.float64)
        self.stats = torch.zeros(3, dtype=torch.int64, device="cuda")  # sizeof(crush_contact_stats) == 24

    def apply(self, c, u, dt):
        nodes, faces, scale, stiffness, md = self.model.contact(c)
        nd = _dev(nodes.view(np.int32), torch.int32)
        fc = _dev(faces.reshape(-1).view(np.int32), torch.int32)
        sc = _dev(scale, torch.float64) if scale is not None else None
        ud = _dev(u, torch.float64)
        f = torch.zeros(3 * self.n, dtype=torch.float64, device="cuda")
        contact_apply_static(self.n, self.pos.data_ptr(), ud.data_ptr(), self.masses.data_ptr(), (nd.data_ptr(), len(nodes)),
                             None if sc is None else sc.data_ptr(), (fc.data_ptr(), len(faces)), stiffness, md, dt,
                             f.data_ptr(), self.stats.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        st = abi.ContactStats.from_buffer_copy(self.stats.cpu().numpy().tobytes())
        return f.cpu().numpy(), st


def _check_model(model, amps, dt):
    ctx = Context(model.desc)
    lumped, _ = ctx.masses()
    static = _Static(model, lumped)
    hits = 0
    for call, amp in enumerate(amps):
        u = _field(model.desc, 100 + call, amp)
        for c in range(model.desc.n_contacts):
            f_ref = np.zeros(3 * model.n_nodes)
            cnt, mp = ctx.contact_apply(c, u, None, None, dt, f_ref)
            f, st = static.apply(c, u, dt)
            assert st.status == abi.CRUSH_OK
            assert st.penetration_count == cnt
            assert st.max_penetration == mp
            assert np.array_equal(f, f_ref), f"contact {c}, call {call}: forces differ"
            hits += cnt
    assert hits > 0
    return ctx, static


@pytest.fixture(scope="module")
def plain():
    return S.Model.build(S.plain_headon())


def test_static_contact_matches_context_call_twice(plain):
    _check_model(plain, amps=(0.25, 0.4), dt=1.0e-4)


def test_static_contact_matches_on_refined_mesh():
    model = S.Model.build(S.refined_headon())
    for c in range(model.desc.n_contacts):
        nodes, faces, _, _, _ = model.contact(c)
        assert len(nodes) <= abi.STATIC_MAX_NODES and len(faces) <= abi.STATIC_MAX_FACES
    _check_model(model, amps=(0.12, 0.2), dt=2.0e-5)


def test_static_contact_adds_in_reference_order(plain):
    """Into a non-zero f_accum, the call adds each node's contributions in
    sequence; a second call then adds the same forces again."""
    ctx = Context(plain.desc)
    lumped, _ = ctx.masses()
    static = _Static(plain, lumped)
    u = _field(plain.desc, 5, 0.3)
    for c in range(plain.desc.n_contacts):  # the first contact with a penetration
        once, st = static.apply(c, u, 1.0e-4)
        if st.penetration_count > 0:
            break
    nodes, faces, scale, stiffness, md = plain.contact(c)
    nd = _dev(nodes.view(np.int32), torch.int32)
    fc = _dev(faces.reshape(-1).view(np.int32), torch.int32)
    ud = _dev(u, torch.float64)
    f = torch.zeros(3 * plain.n_nodes, dtype=torch.float64, device="cuda")
    for _ in range(2):
        contact_apply_static(plain.n_nodes, static.pos.data_ptr(), ud.data_ptr(), static.masses.data_ptr(),
                             (nd.data_ptr(), len(nodes)), None, (fc.data_ptr(), len(faces)), stiffness, md, 1.0e-4,
                             f.data_ptr(), None, 0)
    torch.cuda.synchronize()
    twice = f.cpu().numpy()
    assert np.any(once != 0.0)
    np.testing.assert_allclose(twice, 2.0 * once, rtol=1e-12, atol=1e-9)


def test_static_contact_rejects_oversized_and_bad_ids(plain):
    ctx = Context(plain.desc)
    lumped, _ = ctx.masses()
    static = _Static(plain, lumped)
    nodes, faces, _, stiffness, md = plain.contact(0)
    big = np.zeros((abi.STATIC_MAX_FACES + 1, 4), np.uint32)
    fc = _dev(big.reshape(-1).view(np.int32), torch.int32)
    nd = _dev(nodes.view(np.int32), torch.int32)
    u = torch.zeros(3 * plain.n_nodes, dtype=torch.float64, device="cuda")
    f = torch.zeros(3 * plain.n_nodes, dtype=torch.float64, device="cuda")
    with pytest.raises(CrushError) as e:
        contact_apply_static(plain.n_nodes, static.pos.data_ptr(), u.data_ptr(), static.masses.data_ptr(),
                             (nd.data_ptr(), len(nodes)), None, (fc.data_ptr(), len(big)), stiffness, md, 1e-4,
                             f.data_ptr(), None, 0)
    assert e.value.status == abi.CRUSH_ERR_INVALID and "CRUSH_STATIC_MAX_FACES" in str(e.value)
    # A node id past the model: checked on the device before any access;
    # nothing is written and the stats carry the error.
    bad = nodes.copy()
    bad[len(bad) // 2] = plain.n_nodes
    bd = _dev(bad.view(np.int32), torch.int32)
    fc = _dev(faces.reshape(-1).view(np.int32), torch.int32)
    f.fill_(1.5)
    contact_apply_static(plain.n_nodes, static.pos.data_ptr(), u.data_ptr(), static.masses.data_ptr(),
                         (bd.data_ptr(), len(bad)), None, (fc.data_ptr(), len(faces)), stiffness, md, 1e-4,
                         f.data_ptr(), static.stats.data_ptr(), 0)
    torch.cuda.synchronize()
    st = abi.ContactStats.from_buffer_copy(static.stats.cpu().numpy().tobytes())
    assert st.status == abi.CRUSH_ERR_INVALID
    assert bool(torch.all(f == 1.5))


def test_static_contact_leaves_device_memory_unchanged(plain):
    """After the first call in this process's context, further calls change
    neither the device's free memory nor torch's allocator: the call takes
    all its scratch from the library's static record."""
    ctx = Context(plain.desc)
    lumped, _ = ctx.masses()
    static = _Static(plain, lumped)
    nodes, faces, _, stiffness, md = plain.contact(plain.desc.n_contacts - 1)
    nd = _dev(nodes.view(np.int32), torch.int32)
    fc = _dev(faces.reshape(-1).view(np.int32), torch.int32)
    ud = _dev(_field(plain.desc, 9, 0.3), torch.float64)
    f = torch.zeros(3 * plain.n_nodes, dtype=torch.float64, device="cuda")

    def call():
        contact_apply_static(plain.n_nodes, static.pos.data_ptr(), ud.data_ptr(), static.masses.data_ptr(),
                             (nd.data_ptr(), len(nodes)), None, (fc.data_ptr(), len(faces)), stiffness, md, 1.0e-4,
                             f.data_ptr(), static.stats.data_ptr(), 0)

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(16):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0
