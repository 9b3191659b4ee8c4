"""Edge case: an ice-shelf cavity (nodes and cells whose top layers are dry, nzmin > 0),
against golden vectors of the reference's own advect_one_fct / compute_w /
impl_vert_diff_one on the same cavity mesh (tests/golden/make_cavity_golden.py): the
oracle on CPU; the fused and one-kernel-per-stage CUDA paths, the batched engine, the
vertical diffusion and the reverse pass on the GPU."""

import numpy as np
import pytest

from oracle import fct_np, vdiff_np
from tests.golden_cases import (CAVITY_GOLDEN, RTOL, SAMPLE, cases, cavity_mesh, field_digest,
                                vdiff_cases)

DT = 3600.0
NAMES = ["T_step1", "T_ab2", "sharp_x5"]


@pytest.fixture(scope="module")
def cav(pi):
    return cavity_mesh(pi)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(CAVITY_GOLDEN))


def _check(m, g, key, x, mask=None, rtol=RTOL):
    mask = m.node_layer_mask if mask is None else mask
    ref = g[f"{key}"]
    ms = mask[SAMPLE]
    scale = np.max(np.abs(ref[ms]))
    assert np.max(np.abs(x[SAMPLE][ms] - ref[ms])) <= rtol * scale, key
    d, gd = field_digest(m, x, mask), g[f"{key.split('__')[0]}__digest"]
    assert np.all(np.abs(d - gd) <= 1e-11 * np.maximum(np.abs(gd), 1.0)), (key, d, gd)


def test_cavity_mesh_has_dry_tops(cav):
    assert (cav.ulevels_nod2D > 1).sum() > 100 and (cav.ulevels > 1).sum() > 100


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_on_cavity(cav, golden, name):
    c = cases(cav)[name]
    Tn, _ = fct_np.advect_one_fct(cav, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                  c["hnode_new"], c["T"], c["T_old"], dt=DT)
    _check(cav, golden, f"{name}__T_new", Tn, rtol=1e-13)
    assert np.array_equal(Tn[~cav.node_layer_mask], c["T"][~cav.node_layer_mask])


def test_oracle_compute_w_and_vdiff_on_cavity(cav, golden):
    from fesom_jax_b200 import inputs as I
    c = cases(cav)["T_step1"]
    w = I.compute_w(cav, c["uv"], c["helem"])
    _check(cav, golden, "w_e", w, mask=cav.node_iface_mask, rtol=1e-13)
    v = vdiff_cases(cav)["T"]
    _check(cav, golden, "vdiff__T_new",
           vdiff_np.impl_vert_diff_one(cav, v["T"], v["Kv"], v["hnode_new"], dt=DT), rtol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_fused_and_unfused_on_cavity(cav, golden, name):
    import torch
    from fesom_jax_b200.tracer_adv import advect_one_fct, get_plan
    c = cases(cav)[name]
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    args = [d(c[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new", "T", "T_old")]
    got = advect_one_fct(cav, *args, dt=DT)[0].cpu().numpy()
    _check(cav, golden, f"{name}__T_new", got)
    assert np.array_equal(got[~cav.node_layer_mask], c["T"][~cav.node_layer_mask])
    plan = get_plan(cav, 0)
    try:
        plan.set_fused(False)
        ref = advect_one_fct(cav, *args, dt=DT)[0].cpu().numpy()
    finally:
        plan.set_fused(True)
    # the fused stages divide by reciprocals and fuse multiply-adds: equal to rounding
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    assert np.array_equal(got[~cav.node_layer_mask], ref[~cav.node_layer_mask])


@pytest.mark.gpu
def test_gpu_producers_batched_and_reverse_on_cavity(cav, golden):
    import torch
    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200.adjoint import advect_one_fct_vjp
    from fesom_jax_b200.ale import compute_w
    from fesom_jax_b200.ensemble import Ensemble
    from fesom_jax_b200.tracer_adv import advect_one_fct
    from fesom_jax_b200.tracer_diff import impl_vert_diff_one
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    c = cases(cav)["T_step1"]
    w = compute_w(cav, d(c["uv"]), d(c["helem"])).cpu().numpy()
    _check(cav, golden, "w_e", w, mask=cav.node_iface_mask)
    v = vdiff_cases(cav)["T"]
    Tv = impl_vert_diff_one(cav, d(v["T"]), d(v["Kv"]), d(v["hnode_new"]), dt=DT).cpu().numpy()
    _check(cav, golden, "vdiff__T_new", Tv)
    # batched (interleaved, derived w, diffusion epilogue) == plain calls, bit for bit
    f = I.make_fields(cav, seed=8, n_passive=1, ab2=True)
    ens = Ensemble(device=0)
    ens.add_member(cav, f.uv, None, f.helem, f.hnode, f.hnode_new, f.tracers, f.tracers_old,
                   DT, Kv=v["Kv"], derive_w=True)
    ens.build()
    ens.run(2)
    torch.cuda.synchronize()
    args = [d(x) for x in (f.uv, f.helem, f.hnode, f.hnode_new)]
    wd = compute_w(cav, args[0], args[1])
    T, To = d(f.tracers), d(f.tracers_old)
    for _ in range(2):
        Tn = advect_one_fct(cav, args[0], wd, args[1], args[2], args[3], T, To, dt=DT)[0]
        T, To = impl_vert_diff_one(cav, Tn, d(v["Kv"]), args[3], dt=DT), T
    assert torch.equal(ens.state(0)[0], T)
    ens.close()
    # the reverse pass runs on the cavity mesh and its cotangents are finite
    g = advect_one_fct_vjp(cav, d(f.uv), d(f.w_e), d(f.helem), d(f.hnode), d(f.hnode_new),
                           d(f.tracers), d(f.tracers_old),
                           d(np.where(cav.node_layer_mask, 1.0, 0.0) * np.ones_like(f.tracers)),
                           dt=DT)
    assert all(bool(torch.isfinite(x).all()) for x in g)


@pytest.mark.gpu
def test_gpu_vjp_matches_reference_autodiff_on_cavity(cav):
    """The reverse pass on the cavity mesh (its dry-top levels, nzmin > 0) against the
    reference's own autodiff (tests/golden/make_cavity_grad_golden.py)."""
    import torch
    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200.adjoint import advect_one_fct_vjp
    from tests.test_adjoint_gpu import GRTOL, _check
    g = dict(np.load("tests/golden/fct_cavity_grad_golden.npz"))
    f = I.make_fields(cav, seed=0, ab2=True)
    lm = cav.node_layer_mask
    wts = np.where(lm, np.random.default_rng(99).normal(size=lm.shape), 0.0)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    res = advect_one_fct_vjp(cav, d(f.uv), d(f.w_e), d(f.helem), d(f.hnode), d(f.hnode_new),
                             d(f.tracers[0]), d(f.tracers_old[0]), d(wts), dt=DT)
    for name, x in zip(("T", "T_old", "uv", "w_e"), res):
        err = _check(name, x.cpu().numpy(), g[f"step__g_{name}"], g[f"step__g_{name}_digest"], cav)
        assert err <= GRTOL
