"""The JAX/XLA custom-call handlers (fct_xla_forward / fct_xla_adjoint), invoked the way
XLA invokes a legacy GPU custom call: a stream, a fixed list of device buffers, the
opaque bytes; the status comes back in an int32 device result. Their results equal the
direct C-ABI calls bit for bit, and the golden vectors of the reference's own
advect_one_fct (with Z3d/zbar3 and w_i) through the handler."""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from tests.golden_cases import DT, cases, check_against_golden, load_golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _d(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_forward_handler_equals_fct_forward(torch, pi):
    from fesom_jax_b200 import xla
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=21, ab2=True, n_passive=1)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers), _d(torch, f.tracers_old)
    plan = get_plan(pi, 0)
    plan.reserve(3)
    ref = plan.forward(*args, T, To, DT)
    got, st = xla.forward(plan, *args, T, To, DT)
    assert int(st.item()) == 0
    assert torch.equal(got, ref)


def test_forward_handler_optional_operands_match_golden(torch, pi):
    """w_split + z* (Z3d, zbar3, w_i) through the handler equals the reference golden."""
    from fesom_jax_b200 import xla
    from fesom_jax_b200.tracer_adv import get_plan
    c = cases(pi)["T_wsplit_zstar"]
    args = [_d(torch, c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new", "T", "T_old")]
    kw = {k: _d(torch, v) for k, v in c["kw"].items()}
    got, st = xla.forward(get_plan(pi, 0), *args, DT, **kw)
    assert int(st.item()) == 0
    check_against_golden(pi, load_golden(), "T_wsplit_zstar", c, got.cpu().numpy())


def test_adjoint_handler_equals_fct_adjoint(torch, pi):
    from fesom_jax_b200 import xla
    from fesom_jax_b200.adjoint import advect_one_fct_vjp
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=22, ab2=True, kind="white", sigma=0.02)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    gTn = _d(torch, np.random.default_rng(5).normal(size=T.shape))
    ref = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT)   # also reserves the adjoint
    *got, st = xla.adjoint(get_plan(pi, 0), *args, T, To, gTn, DT)
    assert int(st.item()) == 0
    for a, b in zip(got, ref):
        assert torch.equal(a, b)


def test_handlers_report_errors_in_the_status_result(torch, pi):
    from fesom_jax_b200 import xla
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=23)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    plan = get_plan(pi, 0)
    good = xla.opaque(plan, DT, 1)
    _, st = xla.forward(plan, *args, T, To, DT, op=good[:-4])           # malformed opaque
    assert int(st.item()) == -1
    bogus = bytes(memoryview(xla.FctXlaOpaque(0x1234560, DT, 1, 0)))
    _, st = xla.forward(plan, *args, T, To, DT, op=bogus)               # no such plan
    assert int(st.item()) == -1
    _, st = xla.forward(plan, *args, T, To, DT, op=xla.opaque(plan, DT, 64))
    assert int(st.item()) == -3                                         # over the reservation
    _, st = xla.forward(plan, *args, T, To, -DT, op=xla.opaque(plan, -DT, 1))
    assert int(st.item()) == -1                                         # dt <= 0
    *_, st = xla.adjoint(plan, *args, T, To, T, DT, op=xla.opaque(plan, DT, 1, w_i=True))
    assert int(st.item()) == -4                                         # w_i not differentiated
    _, st = xla.forward(plan, *args, T, To, DT, op=good)
    assert int(st.item()) == 0
