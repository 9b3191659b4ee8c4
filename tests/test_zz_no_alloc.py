"""fct_forward_noalloc: the forward step whose scratch is a static device array.

An XLA custom-call handler runs inside a runtime that owns the GPU's memory, and a
latency-bound serving loop must not wait on the allocator: such callers cannot allocate at
call time, and this entry point gives them the same step with no allocation. Checked
through the C ABI against fct_forward on two calls in a row with different inputs and
tracer counts (the static array keeps the previous call's contents, which must not leak
into the next result), and for its size limit.
"""

import ctypes as C

import numpy as np
import pytest

from tests.golden_cases import DT, RTOL, cases

pytestmark = pytest.mark.gpu


def _fn():
    from fesom_jax_b200 import _lib
    f = _lib.lib().fct_forward_noalloc
    f.argtypes = [C.c_void_p, C.POINTER(_lib.FctFields), C.c_double, C.c_int, C.c_void_p]
    f.restype = C.c_int
    return f


def _fields(torch, c, ntr, shift=0.0):
    from fesom_jax_b200 import _lib
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    t = {k: d(c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new")}
    t["T"] = d(np.stack([c["T"] + i + shift for i in range(ntr)]))
    t["T_old"] = d(np.stack([c["T_old"] + i + shift for i in range(ntr)]))
    f = _lib.FctFields()
    for k in ("uv", "w_e", "helem", "hnode", "hnode_new", "T", "T_old"):
        setattr(f, k, t[k].data_ptr())
    f.tracer_stride = 0
    return f, t


def test_noalloc_matches_forward_on_two_calls(pi):
    import torch
    from fesom_jax_b200.tracer_adv import get_plan
    plan = get_plan(pi, 0)
    fn = _fn()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    # call 1 fills the static array with a 3-tracer step of one case, call 2 must give the
    # 2-tracer step of another case exactly as fct_forward does
    for call, (name, ntr, shift) in enumerate((("sharp_x5", 3, 5.0), ("T_ab2", 2, 0.0))):
        c = cases(pi)[name]
        f, t = _fields(torch, c, ntr, shift)
        ref = plan.forward(t["uv"], t["w_e"], t["helem"], t["hnode"], t["hnode_new"],
                           t["T"], t["T_old"], DT)
        out = torch.full_like(t["T"], 1.0e30 + call)
        f.T_new = out.data_ptr()
        assert fn(plan.handle, C.byref(f), DT, ntr, stream) == 0
        torch.cuda.synchronize()
        err = (out - ref).abs().max().item() / ref.abs().max().item()
        assert err <= RTOL, (call, name, err)


def test_noalloc_rejects_sizes_beyond_the_static_array(pi):
    import torch
    from fesom_jax_b200 import _lib
    from fesom_jax_b200.tracer_adv import get_plan
    c = cases(pi)["T_ab2"]
    f, t = _fields(torch, c, 1)
    out = torch.empty_like(t["T"])
    f.T_new = out.data_ptr()
    st = _fn()(get_plan(pi, 0).handle, C.byref(f), DT, 64, None)
    assert st == -3
    assert b"static array" in _lib.lib().fct_last_error()
