"""Reverse mode on the GPU (fct_adjoint, fct_compute_w_adjoint) against the reference's
own autodiff (tests/golden/make_grad_golden.py: torch autograd through the unmodified
reference tracer_adv) and against central finite differences."""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I

pytestmark = pytest.mark.gpu
GOLDEN = "tests/golden/fct_pi_grad_golden.npz"
DT = 3600.0
# cotangents: max-norm relative error vs the reference's autodiff
GRTOL = 1e-10


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def _d(torch, x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _check(name, got, ref_sample, ref_digest, pi):
    sl = slice(0, None, 4) if got.shape[0] == pi.nod2D else slice(0, None, 16)
    s = got[sl]
    err = np.max(np.abs(s - ref_sample)) / max(np.max(np.abs(ref_sample)), 1e-300)
    assert err <= GRTOL, f"{name}: sampled rel err {err:.3e}"
    wts = np.random.default_rng(4321).normal(size=got.shape)
    assert abs(got.sum() - ref_digest[0]) <= 1e-9 * ref_digest[1], f"{name}: sum"
    assert abs((got * wts).sum() - ref_digest[2]) <= 1e-9 * ref_digest[1], f"{name}: wsum"
    return err


def test_step_vjp_matches_reference_autodiff(torch, pi, golden):
    from fesom_jax_b200.adjoint import advect_one_fct_vjp
    f = I.make_fields(pi, seed=0, ab2=True)
    lm = pi.node_layer_mask
    wts = np.where(lm, np.random.default_rng(99).normal(size=lm.shape), 0.0)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                   f.tracers[0], f.tracers_old[0])]
    gT, gTo, guv, gw = advect_one_fct_vjp(pi, *args, _d(torch, wts), dt=DT)
    for name, g in (("T", gT), ("T_old", gTo), ("uv", guv), ("w_e", gw)):
        _check(name, g.cpu().numpy(), golden[f"step__g_{name}"], golden[f"step__g_{name}_digest"], pi)


def test_chain_grad_matches_reference_autodiff(torch, pi, golden):
    from fesom_jax_b200.adjoint import chain_loss_and_grad
    f = I.make_fields(pi, seed=0, ab2=True)
    target = np.random.default_rng(7).normal(20.0, 2.0, pi.nod2D)
    K = int(golden["chain__K"])
    loss, gT0, guv = chain_loss_and_grad(
        pi, _d(torch, f.tracers[0]), _d(torch, f.uv), _d(torch, f.helem), _d(torch, f.hnode),
        _d(torch, f.hnode_new), torch.from_numpy(target), K, dt=DT)
    assert abs(loss - float(golden["chain__loss"])) <= 1e-12 * abs(float(golden["chain__loss"]))
    _check("T0", gT0.cpu().numpy(), golden["chain__g_T"], golden["chain__g_T_digest"], pi)
    _check("uv", guv.cpu().numpy(), golden["chain__g_uv"], golden["chain__g_uv_digest"], pi)


def test_chain_grad_central_fd(torch, pi):
    """Central FD (eps = 1e-7 along N(0,1) directions) on 20 seeded random directions
    (10 for T0, 10 for uv) of the 3-step chain loss with w = compute_w(uv).

    The point must be one where the step is differentiable, which two structural cases
    are not: (1) a streamfunction velocity is discretely divergence-free, so
    w = compute_w(uv) is roundoff (~1e-20) at interior nodes and the upwind |w| sits at its
    kink (autodiff, the reference's and this one, takes sign(w) of the roundoff, central FD
    averages both sides); (2) with T_old == T the surface antidiffusive flux is exactly 0,
    the kink of the limiter's ``adf >= 0 ? pf : mf`` select. So this check uses divergent
    (white-noise) velocities and T_old != T."""
    from fesom_jax_b200.adjoint import chain_loss_and_grad
    f = I.make_fields(pi, seed=5, ab2=True, kind="white", sigma=0.02)
    target = torch.from_numpy(np.random.default_rng(8).normal(15.0, 3.0, pi.nod2D))
    c = [_d(torch, x) for x in (f.helem, f.hnode, f.hnode_new)]
    T0, uv = _d(torch, f.tracers[0]), _d(torch, f.uv)
    K = 3
    To0 = _d(torch, f.tracers_old[0])
    loss, gT0, guv = chain_loss_and_grad(pi, T0, uv, *c, target, K, dt=DT, T_old0=To0)
    rng = np.random.default_rng(2024)
    lm = torch.from_numpy(pi.node_layer_mask).cuda()
    em = torch.from_numpy(pi.elem_layer_mask).cuda()[:, :, None]
    worst = 0.0
    for d in range(20):
        if d < 10:
            v = _d(torch, rng.normal(size=T0.shape)) * lm
            eps = 1e-7
            Lp = chain_loss_and_grad(pi, T0 + eps * v, uv, *c, target, K, dt=DT, T_old0=To0)[0]
            Lm = chain_loss_and_grad(pi, T0 - eps * v, uv, *c, target, K, dt=DT, T_old0=To0)[0]
            ad = float((gT0 * v).sum())
        else:
            v = _d(torch, rng.normal(size=uv.shape)) * em
            eps = 1e-7
            Lp = chain_loss_and_grad(pi, T0, uv + eps * v, *c, target, K, dt=DT, T_old0=To0)[0]
            Lm = chain_loss_and_grad(pi, T0, uv - eps * v, *c, target, K, dt=DT, T_old0=To0)[0]
            ad = float((guv * v).sum())
        fd = (Lp - Lm) / (2 * eps)
        rel = abs(fd - ad) / max(abs(ad), 1e-30)
        worst = max(worst, rel)
        assert rel <= 1e-5, (d, fd, ad, rel)


def test_autograd_function_matches_vjp(torch, pi):
    from fesom_jax_b200.adjoint import advect_one_fct_vjp, functions
    AdvectFCT, ComputeW = functions()
    f = I.make_fields(pi, seed=3, ab2=True, n_passive=1)
    lm = pi.node_layer_mask
    wts = _d(torch, np.where(lm, np.random.default_rng(1).normal(size=(3,) + lm.shape), 0.0))
    uv = _d(torch, f.uv).requires_grad_(True)
    T = _d(torch, f.tracers).requires_grad_(True)
    To = _d(torch, f.tracers_old).requires_grad_(True)
    helem, hn, hnn = (_d(torch, x) for x in (f.helem, f.hnode, f.hnode_new))
    w = ComputeW.apply(pi, uv, helem)
    Tn = AdvectFCT.apply(pi, DT, uv, w, helem, hn, hnn, T, To)
    (wts * Tn).sum().backward()
    gT, gTo, guv, gw = advect_one_fct_vjp(pi, uv.detach(), w.detach(), helem, hn, hnn,
                                          T.detach(), To.detach(), wts, dt=DT)
    assert torch.equal(T.grad, gT) and torch.equal(To.grad, gTo)
    from fesom_jax_b200.adjoint import compute_w_vjp
    guv_total = compute_w_vjp(pi, gw, helem, guv.clone())
    assert torch.allclose(uv.grad, guv_total, rtol=1e-12, atol=0)
