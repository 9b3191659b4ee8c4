"""Health counters, cross-stream ordering on one plan, and long runs from poisoned memory.

* The finiteness gate of the reference's diagnostics (fesom_jax/diagnostics.py:31-101)
  on the GPU path: a non-finite input lane gives non-finite outputs, which the final
  stage counts (fct_plan_health / fct_batch_health / the serving engine's per-request
  counters report FCT_ERR_NONFINITE or the count); healthy steps count nothing.
* Calls on one plan from two streams are ordered on the GPU (the plan's workspace is
  shared): the results equal those of the same calls made one after another.
* 900 FCT steps on pi and on a 600-node coastline mesh from a workspace arena, a plan
  workspace and unwritten state buffers filled with NaN bytes stay finite, stay inside
  the limiter window and match the oracle step for step every 30 steps: no stage reads
  an entry it did not write in the same step. The velocities are closed-basin flows
  (inputs.basin_velocities), whose low-order CFL is below 1, so the steps are stable.
"""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from fesom_jax_b200 import meshgen
from oracle import fct_c, fct_np, gates

pytestmark = pytest.mark.gpu
RTOL = 1e-12


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _dev(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def test_plan_health_counts_nonfinite_outputs(torch, pi):
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=41, ab2=True)
    plan = get_plan(pi, 0)
    args = [_dev(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _dev(torch, f.tracers), _dev(torch, f.tracers_old)
    plan.health()                       # start from a clean counter
    out = plan.forward(*args, T, To, 3600.0)
    assert plan.health() == 0 and bool(torch.isfinite(out).all())
    n, k = np.argwhere(pi.node_layer_mask)[777]
    T[0, n, k] = float("nan")
    out = plan.forward(*args, T, To, 3600.0)
    bad = int((~torch.isfinite(out)).sum())
    assert bad > 0
    assert plan.health() == bad          # counted exactly, then reset
    assert plan.health() == 0


def test_batch_health_names_the_member(torch, pi):
    from fesom_jax_b200.ensemble import Ensemble
    ens = Ensemble(device=0)
    for i in range(3):
        f = I.make_fields(pi, seed=50 + i, ab2=True, kind="basin")
        T = f.tracers.copy()
        if i == 1:
            n, k = np.argwhere(pi.node_layer_mask)[999]
            T[1, n, k] = np.inf
        ens.add_member(pi, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, T, f.tracers_old,
                       1800.0)
    ens.build()
    ens.run(2)
    counts = ens.health()
    assert counts[0] == 0 and counts[2] == 0 and counts[1] > 0
    assert ens.health() == [0, 0, 0]
    ens.close()


def test_two_streams_on_one_plan_equal_serial_calls(torch, pi):
    from fesom_jax_b200.tracer_adv import FctPlan
    plan = FctPlan(pi, 0, max_tracers=2)
    cases = []
    for s in range(6):
        f = I.make_fields(pi, seed=60 + s, ab2=True)
        cases.append([_dev(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                               f.tracers, f.tracers_old)])
    serial = []
    for c in cases:
        serial.append(plan.forward(*c[:7], 3600.0).clone())
    torch.cuda.synchronize()
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    outs = [torch.empty_like(c[5]) for c in cases]
    for rep in range(3):
        for i, c in enumerate(cases):
            st = streams[i % 2]
            with torch.cuda.stream(st):
                plan.forward(*c[:7], 3600.0, out=outs[i], stream=st.cuda_stream)
        torch.cuda.synchronize()
        for i in range(len(cases)):
            assert torch.equal(outs[i], serial[i]), (rep, i)
    plan.close()


def _basin_member(m, seed, npass):
    return I.make_fields(m, seed=seed, n_passive=npass, ab2=True, kind="basin")


@pytest.mark.parametrize("mesh_name", ["pi", "small600"])
def test_900_steps_from_poisoned_memory(torch, pi, mesh_name):
    from fesom_jax_b200.ensemble import Ensemble
    from fesom_jax_b200.tracer_adv import get_plan
    m = pi if mesh_name == "pi" else meshgen.make_mesh(600, seed=3, name="small600")
    dt = 1800.0
    f = _basin_member(m, 70, 2)
    assert I.lo_outflow_cfl(m, f.uv, f.w_e, f.hnode, dt) < 1.0
    plan = get_plan(m, 0)
    plan.reserve(f.tracers.shape[0])
    plan.fill_workspace(0xFF)
    ens = Ensemble(device=0)
    ens.add_member(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, f.tracers, f.tracers_old,
                   dt)
    ens.build()
    # poison what the steps must not read: the arena, T_new's buffer and T_old's dry levels
    buf = ens.members[0].buf
    lm = torch.from_numpy(m.node_layer_mask).cuda()[:, :, None]
    nan = float("nan")
    buf[2].fill_(nan)
    buf[0].copy_(torch.where(lm, buf[0], nan))
    ens.prepare()
    ens.fill_workspace(0xFF)
    ens.set_chunk(2)
    lmn = m.node_layer_mask
    keep = []
    from fesom_jax_b200 import _lib as fl
    desc = fl.mesh_desc(m, keep)
    for block in range(30):
        ens.run(30)
        T, To = (x.cpu().numpy() for x in ens.state(0))
        assert np.isfinite(T).all(), block
        # one step of the resident state on the GPU (plain fused call, poisoned plan
        # workspace) against the oracle from the same state
        g = plan.forward(*[_dev(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode,
                                                    f.hnode_new)],
                         _dev(torch, T), _dev(torch, To), dt).cpu().numpy()
        for t in range(T.shape[0]):
            ref, _ = fct_c.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                          T[t], To[t], dt=dt, desc=desc)
            err = np.max(np.abs(g[t][lmn] - ref[lmn])) / np.max(np.abs(ref[lmn]))
            assert err <= RTOL, (block, t, err)
        if block % 10 == 9:   # the limiter window of tracer 0 (numpy oracle intermediates)
            inter = {}
            fct_np.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, T[0], To[0],
                                  dt=dt, intermediates=inter)
            assert len(gates.window_violations(m, T[0], f.hnode_new, g[0], inter,
                                              gates.GPU_WINDOW_ULPS)) == 0
    # passive tracers started in [0, 1]: a bounded scheme keeps them there
    T = ens.state(0)[0].cpu().numpy()
    assert T[2][lmn].min() >= -1e-12 and T[2][lmn].max() <= 1.0 + 1e-12
    assert ens.health() == [0]
    assert plan.health() == 0
    ens.close()


def test_serving_counts_nonfinite_requests(torch, pi):
    from fesom_jax_b200.serve import Request, ServingEngine
    eng = ServingEngine({"pi": pi}, {"pi": 1800.0}, budget_bytes=4e9, ntr=2,
                        workspace_bytes=1e9, adjoint_meshes=())
    reqs = [Request(rid=i, arrival=0.0, mesh="pi", K=3, adjoint=False, seed=100 + i)
            for i in range(3)]
    st = eng.run(reqs)
    assert st["completed"] == 3 and st["nonfinite_requests"] == 0
    eng.close()


@pytest.mark.parametrize("fused", [True, False])
def test_every_option_ignores_a_poisoned_workspace(torch, pi, fused):
    """The step with every option (w_split w_i, zstar Z3d/zbar3), fused and one kernel per
    stage, gives the same bits on a plan whose workspace was filled with NaN bytes as on a
    fresh plan: no stage reads a workspace entry it did not write in the same call."""
    from fesom_jax_b200.tracer_adv import FctPlan
    from tests.golden_cases import cases
    c = cases(pi)["T_wsplit_zstar"]
    d = lambda x: _dev(torch, x)  # noqa: E731
    args = [d(c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new", "T", "T_old")]
    kw = {k: d(v) for k, v in c["kw"].items()}
    outs = []
    for poison in (False, True):
        plan = FctPlan(pi, 0, max_tracers=1)
        plan.set_fused(fused)
        if poison:
            plan.fill_workspace(0xFF)
        outs.append(plan.forward(*args, 3600.0, **kw).cpu().numpy())
        assert plan.health() == 0
        plan.close()
    assert np.array_equal(outs[0], outs[1])
