"""CUDA FCT forward vs the oracle and the reference-generated golden vectors (GPU)."""

import numpy as np
import pytest

from oracle import fct_np
from tests.golden_cases import DT, RTOL, cases, check_against_golden, load_golden

pytestmark = pytest.mark.gpu
# fused stages against the one-kernel-per-stage path: max|difference| / max|T| per step
FUSED_RTOL = 1e-13

NAMES = ["T_step1", "S_step1", "T_ab2", "sharp_x5", "const", "T_wsplit_zstar"]


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def golden():
    return load_golden()


@pytest.fixture(scope="module")
def pi_cases(pi):
    return cases(pi)


def _dev(torch, x):
    return None if x is None else torch.from_numpy(np.ascontiguousarray(x)).cuda()


def run_gpu(torch, mesh, c):
    from fesom_jax_b200.tracer_adv import advect_one_fct
    args = [_dev(torch, c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new", "T", "T_old")]
    kw = {k: _dev(torch, v) for k, v in c["kw"].items()}
    T_new, T_old_new = advect_one_fct(mesh, *args, dt=DT, **kw)
    assert T_old_new is args[5]
    return T_new.cpu().numpy()


@pytest.mark.parametrize("name", NAMES)
def test_forward_matches_golden(torch, pi, golden, pi_cases, name):
    T_new = run_gpu(torch, pi, pi_cases[name])
    check_against_golden(pi, golden, name, pi_cases[name], T_new)


@pytest.mark.parametrize("name", NAMES)
def test_forward_matches_oracle_full_field(torch, pi, pi_cases, name):
    c = pi_cases[name]
    ref, _ = fct_np.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                   c["hnode_new"], c["T"], c["T_old"], dt=DT, **c["kw"])
    got = run_gpu(torch, pi, c)
    lm = pi.node_layer_mask
    err = np.max(np.abs(got[lm] - ref[lm])) / np.max(np.abs(ref[lm]))
    assert err <= RTOL, err
    # dry lanes keep T exactly (ale_reconstruct, tracer_adv.py:147-151)
    assert np.array_equal(got[~lm], c["T"][~lm])


def test_two_tracers_one_call_equal_separate(torch, pi, pi_cases):
    """T and S advanced together (ntr=2) equal two single-tracer calls bit for bit."""
    from fesom_jax_b200.tracer_adv import advect_one_fct
    cT, cS = pi_cases["T_ab2"], pi_cases["S_step1"]
    # S with T_ab2's velocities so both tracers share them
    common = [_dev(torch, cT[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new")]
    TT = _dev(torch, np.stack([cT["T"], cS["T"]]))
    TO = _dev(torch, np.stack([cT["T_old"], cS["T_old"]]))
    both, _ = advect_one_fct(pi, *common, TT, TO, dt=DT)
    one, _ = advect_one_fct(pi, *common, TT[0].contiguous(), TO[0].contiguous(), dt=DT)
    two, _ = advect_one_fct(pi, *common, TT[1].contiguous(), TO[1].contiguous(), dt=DT)
    assert torch.equal(both[0], one) and torch.equal(both[1], two)


def test_bitwise_deterministic(torch, pi, pi_cases):
    a = run_gpu(torch, pi, pi_cases["sharp_x5"])
    b = run_gpu(torch, pi, pi_cases["sharp_x5"])
    assert np.array_equal(a, b)


def test_host_arrays_round_trip(torch, pi, pi_cases):
    """numpy in -> numpy out through the same CUDA path."""
    from fesom_jax_b200.tracer_adv import advect_one_fct
    c = pi_cases["T_step1"]
    T_new, T_alias = advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                    c["hnode_new"], c["T"], c["T_old"], dt=DT)
    assert isinstance(T_new, np.ndarray) and T_alias is c["T"]
    assert np.array_equal(T_new, run_gpu(torch, pi, c))


def test_exch_rejected(pi, pi_cases):
    from fesom_jax_b200.tracer_adv import advect_one_fct
    c = pi_cases["T_step1"]
    with pytest.raises(NotImplementedError):
        advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"], c["hnode_new"],
                       c["T"], c["T_old"], dt=DT, exch=lambda f, kind: f)


def test_compute_w_gpu_matches_reference_digest(torch, pi, golden, pi_cases):
    """The CUDA w producer (ale.py:309-365) against the reference-generated digest."""
    from fesom_jax_b200.ale import compute_w
    from tests.golden_cases import field_digest
    c = pi_cases["T_step1"]
    w = compute_w(pi, _dev(torch, c["uv"]), _dev(torch, c["helem"])).cpu().numpy()
    d, r = field_digest(pi, w, pi.node_iface_mask), golden["w_e__digest"]
    assert abs(d[1] - r[1]) <= 1e-12 * r[2]
    assert abs(d[3] - r[3]) <= 1e-12 * r[3]
    ref = c["w_e"]
    assert np.max(np.abs(w - ref)) <= 1e-12 * np.max(np.abs(ref))
    assert np.all(w[~pi.node_iface_mask] == 0.0)


def test_dry_levels_keep_T_exactly(torch, pi, pi_cases):
    """Invalid lanes keep T (tracer_adv.py:147-151) even when T is nonzero there and the
    output buffer holds stale data."""
    from fesom_jax_b200.tracer_adv import get_plan
    c = pi_cases["T_ab2"]
    lm = pi.node_layer_mask
    T = np.where(lm, c["T"], 99.0)
    To = np.where(lm, c["T_old"], -7.0)
    args = [_dev(torch, c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new")]
    out = torch.full((2, pi.nod2D, pi.nl), 12345.0, dtype=torch.float64, device="cuda")
    TT, TO = _dev(torch, np.stack([T, T])), _dev(torch, np.stack([To, To]))
    get_plan(pi, 0).forward(*args, TT, TO, DT, out=out)
    got = out.cpu().numpy()
    assert np.all(got[:, ~lm] == 99.0)
    ref, _ = fct_np.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                   c["hnode_new"], T, To, dt=DT)
    assert np.max(np.abs(got[0][lm] - ref[lm])) / np.max(np.abs(ref[lm])) <= RTOL


@pytest.mark.parametrize("name", NAMES)
def test_fused_equals_unfused(torch, pi, pi_cases, name):
    """The fused stage kernels (the default) and one kernel per reference stage give the
    same T_new to rounding (the fused stages multiply by reciprocals and fuse
    multiply-adds; the stage-by-stage path rounds every quotient correctly)."""
    from fesom_jax_b200.tracer_adv import get_plan
    plan = get_plan(pi, 0)
    c = pi_cases[name]
    try:
        plan.set_fused(False)
        ref = run_gpu(torch, pi, c)
    finally:
        plan.set_fused(True)
    got = run_gpu(torch, pi, c)
    assert np.max(np.abs(got - ref)) <= FUSED_RTOL * np.max(np.abs(ref))
    assert np.array_equal(got[~pi.node_layer_mask], ref[~pi.node_layer_mask])


def test_fused_equals_unfused_generated_mesh(torch):
    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200 import meshgen
    from fesom_jax_b200.tracer_adv import advect_one_fct, get_plan
    m = meshgen.make_mesh(2000, seed=11, name="gen2000")
    f = I.make_fields(m, seed=4, n_passive=3, ab2=True)
    args = [_dev(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                     f.tracers, f.tracers_old)]
    plan = get_plan(m, 0)
    try:
        plan.set_fused(False)
        ref = advect_one_fct(m, *args, dt=DT)[0].cpu().numpy()
    finally:
        plan.set_fused(True)
    got = advect_one_fct(m, *args, dt=DT)[0].cpu().numpy()
    assert np.max(np.abs(got - ref)) <= FUSED_RTOL * np.max(np.abs(ref))
