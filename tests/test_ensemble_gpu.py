"""Batched ensemble stepping on the GPU (fct_batch_*): mixed meshes, several workspace
groups, CUDA-graph runs; results equal the single-instance C-ABI path bit for bit and
the oracle within tolerance."""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from fesom_jax_b200 import meshgen
from oracle import fct_np

pytestmark = pytest.mark.gpu
DT = 1800.0
STEPS = 4


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def members(pi):
    small = meshgen.make_mesh(600, seed=3, name="small600")
    out = []
    for i, (m, npass) in enumerate([(pi, 1), (small, 2), (pi, 0), (small, 0)]):
        out.append((m, I.make_fields(m, seed=10 + i, n_passive=npass, ab2=True)))
    return out


def _ensemble(torch, members, budget):
    from fesom_jax_b200.ensemble import Ensemble
    ens = Ensemble(device=0, workspace_budget=budget)
    for m, f in members:
        ens.add_member(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, f.tracers,
                       f.tracers_old, DT)
    ens.build()
    return ens


def _plain(torch, m, f, steps):
    from fesom_jax_b200.tracer_adv import advect_one_fct
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    args = [d(x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = d(f.tracers), d(f.tracers_old)
    for _ in range(steps):
        Tn, To = advect_one_fct(m, *args, T, To, dt=DT)
        T = Tn
    return T.cpu().numpy(), To.cpu().numpy()


@pytest.mark.parametrize("budget,graph", [(24 << 30, True), (1, True), (1, False)])
def test_ensemble_equals_plain_calls(torch, members, budget, graph):
    ens = _ensemble(torch, members, budget)
    if budget == 1:
        assert ens.info()["groups"] == len(members)
    if graph:
        ens.run(STEPS)
    else:
        for _ in range(STEPS):
            ens.step()
    torch.cuda.synchronize()
    for i, (m, f) in enumerate(members):
        T, To = ens.state(i)
        Tp, Top = _plain(torch, m, f, STEPS)
        assert np.array_equal(T.cpu().numpy(), Tp), f"member {i}"
        assert np.array_equal(To.cpu().numpy(), Top), f"member {i} T_old"
    ens.close()


def test_ensemble_matches_oracle_multistep(torch, members):
    ens = _ensemble(torch, members, 24 << 30)
    ens.run(3)
    torch.cuda.synchronize()
    for i, (m, f) in enumerate(members):
        T_gpu = ens.state(i)[0].cpu().numpy()
        for t in range(f.tracers.shape[0]):
            T, To = f.tracers[t], f.tracers_old[t]
            for _ in range(3):
                Tn, To = fct_np.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                               T, To, dt=DT)
                T = Tn
            lm = m.node_layer_mask
            err = np.max(np.abs(T_gpu[t][lm] - T[lm])) / np.max(np.abs(T[lm]))
            assert err <= 1e-12, (i, t, err)
            assert np.array_equal(T_gpu[t][~lm], f.tracers[t][~lm])
    ens.close()


def test_profile_step_reports_every_stage(torch, members):
    ens = _ensemble(torch, members, 24 << 30)
    prof = ens.profile_step()
    assert {"node_lo", "edge_adf", "node_final"} <= set(prof)
    assert all(v >= 0.0 for v in prof.values()) and prof["node_final"] > 0.0
    ens.close()


def _ws_bytes(m, ntr):
    L = m.nl
    pad = lambda n: (n + 31) // 32 * 32  # noqa: E731  (fields on 256-byte boundaries)
    return 8 * (pad(m.edge2D * L) + 4 * pad(ntr * m.nod2D * L) + pad(ntr * m.edge2D * L))


@pytest.mark.parametrize("per_thread", [8, 2, 1])
def test_chunked_workspace_equals_plain(torch, pi, per_thread):
    """A budget that holds the workspace of 4 of a member's 10 tracers: the stages run
    chunk by chunk (4, 4, 2 tracers) through one small workspace; results equal the
    plain path bit for bit whatever the tracers per thread."""
    f = I.make_fields(pi, seed=21, n_passive=8, ab2=True)
    assert f.tracers.shape[0] == 10
    ens = _ensemble(torch, [(pi, f)], _ws_bytes(pi, 4) + 1024)
    info = ens.info()
    assert info["workspace_tracers"] == 4 and info["groups"] == 1
    ens.set_chunk(per_thread)
    ens.run(STEPS)
    torch.cuda.synchronize()
    launches = ens.info()["launches_per_step"]
    # one launch per stage per chunk: S slices x per_thread tracers cover each chunk
    assert launches == 1 + 5 * 3   # vflux + 5 fused stages per chunk
    T, To = ens.state(0)
    Tp, Top = _plain(torch, pi, f, STEPS)
    assert np.array_equal(T.cpu().numpy(), Tp)
    assert np.array_equal(To.cpu().numpy(), Top)
    prof = ens.profile_step()
    assert prof["node_final"] > 0.0
    ens.close()


def test_derived_w_equals_compute_w_then_fct(torch, pi):
    """A member with derive_w runs compute_w(uv, helem) inside every step's graph; it
    equals the plain compute_w call followed by the plain FCT calls, bit for bit."""
    from fesom_jax_b200.ale import compute_w
    from fesom_jax_b200.ensemble import Ensemble
    f = I.make_fields(pi, seed=31, n_passive=1, ab2=True)
    ens = Ensemble(device=0)
    ens.add_member(pi, f.uv, None, f.helem, f.hnode, f.hnode_new, f.tracers, f.tracers_old,
                   DT, derive_w=True)
    ens.build()
    # compute_w + vflux + 5 fused stages x 2 launches (3 tracers: a 2-tracer and a 1-tracer split)
    assert ens.info()["launches_per_step"] == 1 + 1 + 5 * 2
    ens.run(STEPS)
    torch.cuda.synchronize()
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    w = compute_w(pi, d(f.uv), d(f.helem))
    T, To = _plain(torch, pi, I.Fields(**{**f.__dict__, "w_e": w.cpu().numpy()}), STEPS)
    Tb, Tob = ens.state(0)
    assert np.array_equal(Tb.cpu().numpy(), T) and np.array_equal(Tob.cpu().numpy(), To)
    ens.close()


def test_batch_rejects_interleaved_arrays_beyond_2_32(torch, pi):
    """The kernels index interleaved [entity, nl, tracers] arrays in 32 bits: a batch whose
    instance would need 2^32 or more elements in one is refused while validating (the
    placeholder field pointers are never dereferenced)."""
    import ctypes as C
    from fesom_jax_b200 import _lib
    from fesom_jax_b200.ensemble import FctInstance, _bind_batch
    from fesom_jax_b200.tracer_adv import get_plan
    L = _bind_batch(_lib.lib())
    plan = get_plan(pi, 0)
    p = 1 << 20
    ntr = 10000   # 8986 edges x 48 levels x 10000 tracers > 2^32
    arr = (FctInstance * 1)(FctInstance(plan.handle.value, p, p, p, p, p,
                                        (C.c_void_p * 3)(p, p, p), ntr, 1800.0, None, None))
    h = C.c_void_p()
    st = L.fct_batch_create(arr, 1, 1 << 34, C.byref(h))
    assert st == -3 and not h.value
    assert "2^32" in L.fct_last_error().decode()


def test_autotune_cache_applies_the_stored_mapping(torch, members, tmp_path):
    """The first tuning of a batch shape stores its per-stage mapping; a second ensemble of
    the same meshes and shape applies it without timing, and steps to the same bits."""
    from fesom_jax_b200.tuning import TuningCache
    cache = TuningCache(tmp_path / "tuning.json")
    a = _ensemble(torch, members, 24 << 30)
    first = a.autotune(steps=1, reps=1, cache=cache)
    assert "cached" not in first
    b = _ensemble(torch, members, 24 << 30)
    second = b.autotune(steps=1, reps=1, cache=cache)
    assert second["cached"] and [tuple(m) for m in second["stage_map"]] == list(a.stage_map)
    assert b.stage_map == a.stage_map
    a.close()
    b.close()
