"""Implicit vertical tracer diffusion (fesom_jax/tracer_diff.py:68-141): the oracle and the
CUDA kernel against the reference-generated golden vectors
(tests/golden/make_vdiff_golden.py), the reference test's own properties (a constant
tracer stays put, column integrals are conserved, diffusion smooths;
fesom_jax/tests/test_tracers.py:214-235), and the batched epilogue."""

import numpy as np
import pytest

from oracle import vdiff_np
from tests.golden_cases import RTOL, SAMPLE, VDIFF_GOLDEN, _sha, field_digest, vdiff_cases

DT = 3600.0
NAMES = ["T", "S_bc", "T_sw", "T_zstar", "const", "grad"]


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(VDIFF_GOLDEN))


@pytest.fixture(scope="module")
def vcases(pi):
    return vdiff_cases(pi)


def _check(m, g, name, c, T_new, rtol=RTOL):
    assert _sha(c["T"], c["Kv"], c["hnode_new"], *c["kw"].values()) == \
        g[f"{name}__in_digest"].tobytes(), f"{name}: input generation drifted"
    lm = m.node_layer_mask
    ref = g[f"{name}__T_new"]
    got = T_new[SAMPLE][lm[SAMPLE]]
    scale = max(np.max(np.abs(ref)), 1e-300)
    err = np.max(np.abs(got - ref[lm[SAMPLE]])) / scale
    assert err <= rtol, (name, err)
    d = field_digest(m, T_new)
    gd = g[f"{name}__digest"]
    assert np.all(np.abs(d - gd) <= 1e-11 * np.maximum(np.abs(gd), 1.0)), (name, d, gd)
    assert np.array_equal(T_new[~lm], c["T"][~lm])   # dry levels keep T
    return err


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_golden(pi, golden, vcases, name):
    c = vcases[name]
    T_new = vdiff_np.impl_vert_diff_one(pi, c["T"], c["Kv"], c["hnode_new"], dt=DT, **c["kw"])
    _check(pi, golden, name, c, T_new, rtol=1e-13)


def test_oracle_pair_matches_reference(pi, golden, vcases):
    c = vcases
    Tn, Sn = vdiff_np.impl_vert_diff(pi, c["T"]["T"], c["S_bc"]["T"], c["T"]["Kv"],
                                     c["T"]["hnode_new"], dt=DT,
                                     bc_T=c["S_bc"]["kw"]["bc_surf"] * 2.0,
                                     bc_S=c["S_bc"]["kw"]["bc_surf"],
                                     sw_3d=c["T_sw"]["kw"]["sw_3d"])
    lm = pi.node_layer_mask[SAMPLE]
    for x, key in ((Tn, "pair__T_new"), (Sn, "pair__S_new")):
        ref = golden[key]
        assert np.max(np.abs(x[SAMPLE][lm] - ref[lm])) <= 1e-13 * np.max(np.abs(ref))


def column_properties(m, c, T_new):
    """(max constant drift, max relative column-integral change, smoothing ok)."""
    lm = m.node_layer_mask
    av, hn = m.areasvol, c["hnode_new"]
    i0 = np.sum(av * hn * np.where(lm, c["T"], 0.0), axis=1)
    i1 = np.sum(av * hn * np.where(lm, T_new, 0.0), axis=1)
    cons = np.max(np.abs(i1 - i0) / np.maximum(np.abs(i0), 1e-30))
    r0 = np.where(lm, c["T"], -1e30).max(1) - np.where(lm, c["T"], 1e30).min(1)
    r1 = np.where(lm, T_new, -1e30).max(1) - np.where(lm, T_new, 1e30).min(1)
    return cons, r1.mean() < r0.mean()


def test_oracle_reference_properties(pi, vcases):
    c = vcases["const"]
    Tc = vdiff_np.impl_vert_diff_one(pi, c["T"], c["Kv"], c["hnode_new"], dt=DT)
    assert np.max(np.abs(Tc[pi.node_layer_mask] - 20.0)) < 1e-12
    c = vcases["grad"]
    Tg = vdiff_np.impl_vert_diff_one(pi, c["T"], c["Kv"], c["hnode_new"], dt=DT)
    cons, smooth = column_properties(pi, c, Tg)
    assert cons < 1e-12 and smooth


# ----------------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    return torch


def _gpu(torch, m, c, ntr_stack=None):
    from fesom_jax_b200.tracer_diff import impl_vert_diff_one
    d = lambda x: None if x is None else torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa
    kw = {k: d(v) for k, v in c["kw"].items()}
    T = d(c["T"] if ntr_stack is None else ntr_stack)
    return impl_vert_diff_one(m, T, d(c["Kv"]), d(c["hnode_new"]), dt=DT, **kw).cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_reference_golden_and_oracle(torch, pi, golden, vcases, name):
    c = vcases[name]
    got = _gpu(torch, pi, c)
    _check(pi, golden, name, c, got)
    ref = vdiff_np.impl_vert_diff_one(pi, c["T"], c["Kv"], c["hnode_new"], dt=DT, **c["kw"])
    lm = pi.node_layer_mask
    assert np.max(np.abs(got[lm] - ref[lm])) <= RTOL * np.max(np.abs(ref[lm]))


@pytest.mark.gpu
def test_gpu_reference_properties_and_determinism(torch, pi, vcases):
    c = vcases["const"]
    Tc = _gpu(torch, pi, c)
    assert np.max(np.abs(Tc[pi.node_layer_mask] - 20.0)) < 1e-12
    c = vcases["grad"]
    Tg = _gpu(torch, pi, c)
    cons, smooth = column_properties(pi, c, Tg)
    assert cons < 1e-12 and smooth
    c = vcases["T"]
    assert np.array_equal(_gpu(torch, pi, c), _gpu(torch, pi, c))


@pytest.mark.gpu
def test_gpu_pair_and_stacked_tracers(torch, pi, golden, vcases):
    """impl_vert_diff (T with bc and shortwave, S with bc) equals the reference; a
    stacked [ntr, N, nl] call equals separate calls bit for bit."""
    from fesom_jax_b200.tracer_diff import impl_vert_diff, impl_vert_diff_one
    c = vcases
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    Tn, Sn = impl_vert_diff(pi, d(c["T"]["T"]), d(c["S_bc"]["T"]), d(c["T"]["Kv"]),
                            d(c["T"]["hnode_new"]), dt=DT,
                            bc_T=d(c["S_bc"]["kw"]["bc_surf"] * 2.0),
                            bc_S=d(c["S_bc"]["kw"]["bc_surf"]), sw_3d=d(c["T_sw"]["kw"]["sw_3d"]))
    lm = pi.node_layer_mask[SAMPLE]
    for x, key in ((Tn, "pair__T_new"), (Sn, "pair__S_new")):
        ref = golden[key]
        assert np.max(np.abs(x.cpu().numpy()[SAMPLE][lm] - ref[lm])) <= RTOL * np.max(np.abs(ref))
    stack = np.stack([c["T"]["T"], c["S_bc"]["T"], c["grad"]["T"]])
    both = impl_vert_diff_one(pi, d(stack), d(c["T"]["Kv"]), d(c["T"]["hnode_new"]), dt=DT)
    for i in range(3):
        one = impl_vert_diff_one(pi, d(stack[i]), d(c["T"]["Kv"]), d(c["T"]["hnode_new"]), dt=DT)
        assert torch.equal(both[i], one)


@pytest.mark.gpu
def test_batched_epilogue_equals_fct_then_diffusion(torch, pi, vcases):
    """An ensemble member with Kv runs FCT + implicit vertical diffusion each step; it
    equals the plain FCT call followed by the plain diffusion call, bit for bit."""
    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200.ensemble import Ensemble
    from fesom_jax_b200.tracer_adv import advect_one_fct
    from fesom_jax_b200.tracer_diff import impl_vert_diff_one
    f = I.make_fields(pi, seed=12, n_passive=1, ab2=True)
    Kv = vcases["T"]["Kv"]
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    ens = Ensemble(device=0)
    ens.add_member(pi, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, f.tracers, f.tracers_old,
                   1800.0, Kv=Kv)
    ens.build()
    ens.run(3)
    torch.cuda.synchronize()
    T, To = d(f.tracers), d(f.tracers_old)
    args = [d(x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    for _ in range(3):
        Tn, _ = advect_one_fct(pi, *args, T, To, dt=1800.0)
        Tn = impl_vert_diff_one(pi, Tn, d(Kv), args[4], dt=1800.0)
        To, T = T, Tn
    Tb, Tob = ens.state(0)
    assert torch.equal(Tb, T) and torch.equal(Tob, To)
    ens.close()
