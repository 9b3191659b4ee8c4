"""Continuous-batching serving (fct_serve_step): each request's result is the same alone
and in the mix, the batch really mixes requests, and admission respects the budget."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine(pi):
    from fesom_jax_b200 import meshgen
    from fesom_jax_b200.serve import ServingEngine
    small = meshgen.make_mesh(600, seed=3, name="small600")
    eng = ServingEngine({"pi": pi, "small": small}, {"pi": 3600.0, "small": 1800.0},
                        budget_bytes=8e9, workspace_bytes=2e9, velocity_pool=2)
    yield eng
    eng.close()


def _alone(eng, r):
    """The request run by itself through the single-instance path (fct_forward)."""
    import torch
    e = eng.meshes[r.mesh]
    uv, w = e.vel[r.seed % len(e.vel)]
    st = eng.init_state(r)
    T = st[1].permute(2, 0, 1).contiguous()
    To = T.clone()
    for _ in range(r.K):
        Tn = e.plan.forward(uv, w, e.thick.helem, e.thick.hnode, e.thick.hnode_new, T, To, e.dt)
        To, T = T, Tn
    torch.cuda.synchronize()
    return T.cpu().numpy()


def test_results_same_alone_and_in_the_mix(engine):
    from fesom_jax_b200.serve import poisson_requests
    reqs = poisson_requests(rate=2000.0, duration=0.02, mix=(("pi", 0.5), ("small", 0.5)),
                            kmax=6, p_adjoint=0.3, seed=11, max_requests=24)
    assert len(reqs) >= 8
    stats = engine.run(reqs, keep_results=True)
    assert stats["completed"] == len(reqs)
    assert stats["mean_batch"] > 1.5          # requests really shared iterations
    # the 600-node requests took extra steps in iterations led by a pi-size request
    assert stats["multi_round_iterations"] > 0
    for r in reqs:
        alone = _alone(engine, r)
        err = np.max(np.abs(r.result - alone)) / np.max(np.abs(alone))
        assert err <= 1e-12, (r.rid, r.mesh, r.K, err)
        assert r.done >= r.arrival
        if r.adjoint:
            assert r.grad is not None and bool(np.isfinite(r.grad[0].cpu().numpy()).all())


def test_admission_respects_budget(engine, pi):
    """With room for a single pi member beyond the static pools, requests queue and run
    one after another; all still complete with the same results."""
    from fesom_jax_b200.serve import poisson_requests
    reqs = poisson_requests(rate=5000.0, duration=0.01, mix=(("pi", 1.0),), kmax=3,
                            p_adjoint=0.0, seed=5, max_requests=4)
    one = engine.state_bytes(reqs[0])
    budget, engine.budget = engine.budget, engine.static_bytes + one
    try:
        stats = engine.run(reqs, keep_results=True)
    finally:
        engine.budget = budget
    assert stats["completed"] == len(reqs) and stats["mean_batch"] == 1.0
    for r in reqs:
        assert np.max(np.abs(r.result - _alone(engine, r))) / np.max(np.abs(r.result)) <= 1e-12
