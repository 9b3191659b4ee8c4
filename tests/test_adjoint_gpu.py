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


def test_tape_equals_recompute(torch, pi):
    """A taped step's forward (the stage-by-stage kernels) equals fct_forward (the fused
    kernels) to rounding, and its adjoint equals the recomputing adjoint bit for bit; so
    does the K-step chain under both checkpoint modes."""
    from fesom_jax_b200.adjoint import Tape, advect_one_fct_vjp, chain_loss_and_grad
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=5, ab2=True, kind="white", sigma=0.02, n_passive=1)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers), _d(torch, f.tracers_old)
    gTn = _d(torch, np.random.default_rng(3).normal(size=T.shape))
    with Tape(pi, steps=2, ntr=3) as tape:
        Tn = tape.forward(1, *args, T, To, DT)
        Tf = get_plan(pi, 0).forward(*args, T, To, DT)
        assert float((Tn - Tf).abs().max()) <= 1e-13 * float(Tf.abs().max())
        taped = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT, tape=tape, slot=1)
        again = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT, tape=tape, slot=1)
    plain = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT)
    for a, b, c in zip(taped, plain, again):
        assert torch.equal(a, b) and torch.equal(a, c)
    target = torch.from_numpy(np.random.default_rng(8).normal(15.0, 3.0, pi.nod2D))
    c = [_d(torch, x) for x in (f.helem, f.hnode, f.hnode_new)]
    T0, To0, uv = T[0].contiguous(), To[0].contiguous(), args[0]
    r_tape = chain_loss_and_grad(pi, T0, uv, *c, target, 4, dt=DT, T_old0=To0,
                                 checkpoint="tape")
    r_rc = chain_loss_and_grad(pi, T0, uv, *c, target, 4, dt=DT, T_old0=To0,
                               checkpoint="recompute")
    assert r_tape[0] == r_rc[0]
    assert torch.equal(r_tape[1], r_rc[1]) and torch.equal(r_tape[2], r_rc[2])


def test_adjoint_accumulate_bits(torch, pi):
    """fct_adjoint_ex's accumulate bits add the cotangents into the outputs' contents."""
    from fesom_jax_b200.adjoint import (ACC_T, ACC_T_OLD, ACC_UV, ACC_W, _adjoint, _fields,
                                        advect_one_fct_vjp)
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=6, ab2=True)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    gTn = _d(torch, np.random.default_rng(4).normal(size=T.shape))
    ref = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT)
    rng = np.random.default_rng(5)
    base = [_d(torch, rng.normal(size=x.shape)) for x in ref]
    plan = get_plan(pi, 0)
    for acc in (ACC_T | ACC_UV | ACC_W, ACC_T_OLD, ACC_T | ACC_T_OLD | ACC_UV | ACC_W):
        outs = [b.clone() for b in base]
        _adjoint(plan, _fields(pi, *args, T, To), gTn, DT, 1, *outs, None, 0, acc, T.device)
        for bit, o, b, r in zip((ACC_T, ACC_T_OLD, ACC_UV, ACC_W), outs, base, ref):
            assert torch.equal(o, b + r if acc & bit else r), (acc, bit)
    with pytest.raises(RuntimeError, match="accumulate"):   # 16 is FCT_ADJ_DEFER_UV
        _adjoint(plan, _fields(pi, *args, T, To), gTn, DT, 1, *[b.clone() for b in base],
                 None, 0, 32, T.device)


def test_tape_rejects_misuse(torch, pi):
    """Unrecorded slots, another dt, slots out of range and too many tracers are errors."""
    from fesom_jax_b200.adjoint import Tape, advect_one_fct_vjp
    f = I.make_fields(pi, seed=7, ab2=True)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    gTn = torch.ones_like(T)
    with Tape(pi, steps=2) as tape:
        with pytest.raises(RuntimeError, match="no recorded step"):
            advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT, tape=tape, slot=0)
        tape.forward(0, *args, T, To, DT)
        with pytest.raises(RuntimeError, match="dt differs"):
            advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT / 2, tape=tape, slot=0)
        with pytest.raises(RuntimeError, match="slot 2 outside"):
            tape.forward(2, *args, T, To, DT)
        T2, To2 = torch.stack([T, T]), torch.stack([To, To])
        with pytest.raises(RuntimeError, match="outside the tape"):
            tape.forward(1, *args, T2, To2, DT)


def test_tape_reopened_over_the_same_memory(torch, pi):
    """The stateless-handler pattern: a step recorded through one tape is read back through
    a second tape created over the same caller memory (fct_tape_mark_recorded)."""
    import ctypes as C
    from fesom_jax_b200 import _lib
    from fesom_jax_b200.adjoint import Tape, _bind, advect_one_fct_vjp
    f = I.make_fields(pi, seed=8, ab2=True, kind="white", sigma=0.02)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    gTn = _d(torch, np.random.default_rng(9).normal(size=T.shape))
    L = _bind(_lib.lib())
    first = Tape(pi, steps=1)
    first.forward(0, *args, T, To, DT)
    mem, nb = first._mem, Tape.nbytes(pi, 1)
    L.fct_tape_destroy(first._h)
    first._h = C.c_void_p()
    second = Tape.__new__(Tape)
    second.mesh, second.steps, second.ntr, second.device = pi, 1, 1, 0
    second.plan, second._mem = first.plan, mem
    h = C.c_void_p()
    _lib.check(L.fct_tape_create(second.plan.handle, 1, 1, C.c_void_p(mem.data_ptr()), nb,
                                 C.byref(h)))
    second._h = h
    with pytest.raises(RuntimeError, match="no recorded step"):
        advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT, tape=second, slot=0)
    _lib.check(L.fct_tape_mark_recorded(h, 0, DT))
    got = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT, tape=second, slot=0)
    ref = advect_one_fct_vjp(pi, *args, T, To, gTn, dt=DT)
    for a, b in zip(got, ref):
        assert torch.equal(a, b)
    second.close()
    with pytest.raises(RuntimeError, match="256-byte aligned"):
        _lib.check(L.fct_tape_create(second.plan.handle, 1, 1, C.c_void_p(mem.data_ptr() + 8),
                                     nb, C.byref(h)))
    with pytest.raises(RuntimeError, match="needed"):
        _lib.check(L.fct_tape_create(second.plan.handle, 1, 1, C.c_void_p(mem.data_ptr()),
                                     nb - 8, C.byref(h)))


def test_tape_equals_recompute_on_cavity(torch, pi):
    """The same on the cavity mesh (nzmin > 0 under ice shelves): the dry level above a
    cavity's first layer receives the upwind term of interface nzmin in both modes."""
    from fesom_jax_b200.adjoint import Tape, advect_one_fct_vjp
    from tests.golden_cases import cavity_mesh
    cav = cavity_mesh(pi)
    assert (cav.ulevels_nod2D > 1).any()
    f = I.make_fields(cav, seed=4, ab2=True, kind="white", sigma=0.02)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers), _d(torch, f.tracers_old)
    gTn = _d(torch, np.random.default_rng(12).normal(size=T.shape))
    with Tape(cav, steps=1, ntr=2) as tape:
        tape.forward(0, *args, T, To, DT)
        taped = advect_one_fct_vjp(cav, *args, T, To, gTn, dt=DT, tape=tape, slot=0)
    plain = advect_one_fct_vjp(cav, *args, T, To, gTn, dt=DT)
    for a, b in zip(taped, plain):
        assert torch.equal(a, b)
    # the dry level above the first layer of cavity nodes with w < 0 at that interface
    # carries more than dT_new (the upwind term); the other dry levels carry dT_new
    nodes = np.nonzero(cav.ulevels_nod2D > 1)[0]
    ks = cav.ulevels_nod2D[nodes] - 2
    got = taped[0][0].cpu().numpy()[nodes, ks]
    seed = gTn[0].cpu().numpy()[nodes, ks]
    wtop = f.w_e[nodes, ks + 1]
    assert np.any((got != seed) & (wtop < 0))
    assert np.all(got[wtop > 0] == seed[wtop > 0] + 0.0)


def _core2_chain_inputs(torch):
    from fesom_jax_b200 import workloads as W
    mesh = W.make_workload_mesh("batched", seed=0)
    f = I.make_fields(mesh, seed=3, ab2=True, kind="white", sigma=0.002)
    d = [_d(torch, x) for x in (f.tracers[0], f.tracers_old[0], f.uv, f.helem, f.hnode,
                                f.hnode_new)]
    target = torch.from_numpy(np.random.default_rng(7).normal(15.0, 3.0, mesh.nod2D))
    return mesh, f, d, target


def test_chain_grad_dot_product_core2(torch):
    """Dot-product test of the 10-step reverse pass on the CORE2-size mesh (126,990 nodes,
    48 levels) against the oracle's tangent along x = (T0, T_old0).

    The FCT step is positively homogeneous of degree 1 in its tracer inputs: the LO and HO
    fluxes are linear in T, the limiter's bounds are max/min of T-linear values and its
    factors are ratios of T-linear values (the 1e-16 ratio guard and the +-1e3 pads below
    a cell's bottom never decide a max/min for these fields), and every subgradient
    convention (equal split at ties, abs'(0) = 0) is a convex combination of degree-1
    branches. So the tangent of the K-step map along x is the trajectory itself,
    J x = T_K, and for L = sum_n a_n (T_K[n,0] - target_n)^2 the identity

        <gT0, T0> + <gT_old0, T_old0> = sum_n 2 a_n (T_K[n,0] - target_n) T_K[n,0]

    holds exactly; T_K comes from 10 steps of the C oracle. (Central differences at this
    size are lost in the round-off of a loss near 1e15.)"""
    from fesom_jax_b200.adjoint import chain_loss_and_grad
    from fesom_jax_b200.ale import compute_w
    from oracle import fct_c
    mesh, f, (T0, To0, uv, helem, hn, hnn), target = _core2_chain_inputs(torch)
    K, dt = 10, 1800.0
    loss, gT0, guv, gTo0 = chain_loss_and_grad(mesh, T0, uv, helem, hn, hnn, target, K,
                                               dt=dt, T_old0=To0, return_gT_old=True)
    lhs = float((gT0 * T0).sum() + (gTo0 * To0).sum())
    w = compute_w(mesh, uv, helem).cpu().numpy()
    T, To = f.tracers[0], f.tracers_old[0]
    for _ in range(K):
        T, To = fct_c.advect_one_fct(mesh, f.uv, w, f.helem, f.hnode, f.hnode_new, T, To,
                                     dt=dt)
    terms = 2.0 * mesh.areasvol[:, 0] * (T[:, 0] - target.numpy()) * T[:, 0]
    rhs = float(terms.sum())
    assert abs(lhs - rhs) <= 1e-11 * float(np.abs(terms).sum()), (lhs, rhs)
    assert abs(loss - float((mesh.areasvol[:, 0] * (T[:, 0] - target.numpy()) ** 2).sum())) \
        <= 1e-11 * loss


def test_chain_grad_uv_taylor_core2(torch):
    """The uv gradient of the same 10-step loss on the CORE2-size mesh by a Taylor test:
    along a seeded direction v (the size of uv), the remainder
    r(h) = |L(uv + h v) - L(uv) - h <guv, v>| must fall as h^2 (second order: a wrong
    gradient leaves a first-order remainder); kinks crossed by the perturbation (upwind
    sign of w, limiter min/max switches) add O(h) x O(h) in expectation."""
    from fesom_jax_b200.adjoint import chain_loss_and_grad
    mesh, f, (T0, To0, uv, helem, hn, hnn), target = _core2_chain_inputs(torch)
    K, dt = 10, 1800.0
    L0, gT0, guv = chain_loss_and_grad(mesh, T0, uv, helem, hn, hnn, target, K, dt=dt,
                                       T_old0=To0)
    em = torch.from_numpy(mesh.elem_layer_mask).cuda()[:, :, None]
    v = _d(torch, np.random.default_rng(11).normal(0.0, 0.002, uv.shape)) * em
    gv = float((guv * v).sum())
    r = {}
    for h in (1e-2, 3e-3, 1e-3):
        Lh = chain_loss_and_grad(mesh, T0, uv + h * v, helem, hn, hnn, target, K, dt=dt,
                                 T_old0=To0)[0]
        r[h] = abs(Lh - L0 - h * gv)
        print(f"h={h:g} L(h)-L0={Lh - L0:.6e} h<g,v>={h * gv:.6e} r={r[h]:.3e}")
    assert abs(gv) > 0
    # measured on B200: r/|h<g,v>| = 14% at h = 1e-2 (v is as large as uv itself: at
    # h = 1e-1 the remainder is 73%), falling with an observed order of 1.7-1.8; a wrong
    # gradient leaves r/|h<g,v>| constant as h -> 0 (order 1)
    assert r[1e-3] <= 0.05 * abs(1e-3 * gv), r
    assert r[1e-3] <= r[1e-2] / 20.0, r


def test_chain_deferred_uv_equals_per_step_transpose(torch, pi):
    """FCT_ADJ_DEFER_UV + fct_adjoint_flush_uv (the uv cotangent transposed once from the
    sum of the steps' volume-flux cotangents) against a transpose per step: the T
    gradients are the same bits, the uv gradient agrees to rounding; the flush clears the
    sum and checks its arguments."""
    import ctypes as C

    from fesom_jax_b200 import _lib
    from fesom_jax_b200.adjoint import _bind, chain_loss_and_grad
    from fesom_jax_b200.tracer_adv import get_plan
    f = I.make_fields(pi, seed=5, ab2=True, kind="white", sigma=0.02)
    c = [_d(torch, x) for x in (f.helem, f.hnode, f.hnode_new)]
    T0, To0, uv = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0]), _d(torch, f.uv)
    target = torch.from_numpy(np.random.default_rng(8).normal(15.0, 3.0, pi.nod2D))
    for mode in ("tape", "recompute"):
        a = chain_loss_and_grad(pi, T0, uv, *c, target, 4, dt=DT, T_old0=To0, checkpoint=mode,
                                defer_uv=True)
        b = chain_loss_and_grad(pi, T0, uv, *c, target, 4, dt=DT, T_old0=To0, checkpoint=mode,
                                defer_uv=False)
        assert a[0] == b[0] and torch.equal(a[1], b[1])
        # the per-step uv cotangents are larger than their sum and partly cancel, so the
        # two summation orders differ by more than an ulp of the result (6e-13 measured on
        # B200), far inside the 1e-10 of the comparison with the reference's autodiff
        err = float((a[2] - b[2]).abs().max()) / float(b[2].abs().max())
        assert err <= 1e-11, (mode, err)
    # the sum was cleared by the last flush: flushing again adds nothing
    L = _bind(_lib.lib())
    plan = get_plan(pi, 0)
    g = torch.zeros_like(uv)
    s = C.c_void_p(int(torch.cuda.current_stream().cuda_stream))
    assert L.fct_adjoint_flush_uv(plan.handle, C.c_void_p(c[0].data_ptr()),
                                  C.c_void_p(g.data_ptr()), 1, s) == 0
    torch.cuda.synchronize()
    assert float(g.abs().max()) == 0.0
    assert L.fct_adjoint_flush_uv(plan.handle, C.c_void_p(c[0].data_ptr()),
                                  C.c_void_p(g.data_ptr()), 2, s) == -1
    assert L.fct_adjoint_flush_uv(plan.handle, None, C.c_void_p(g.data_ptr()), 0, s) == -1


def test_tape_shared_volume_fluxes(torch, pi):
    """fct_tape_share_vflux: with uv and helem fixed, slots after the first reuse slot 0's
    volume fluxes; the recorded steps and their adjoints are the same bits as without
    sharing, and a sharing tape refuses to record another slot before slot 0."""
    from fesom_jax_b200.adjoint import Tape, advect_one_fct_vjp
    f = I.make_fields(pi, seed=9, ab2=True, kind="white", sigma=0.02)
    args = [_d(torch, x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new)]
    T, To = _d(torch, f.tracers[0]), _d(torch, f.tracers_old[0])
    gTn = _d(torch, np.random.default_rng(13).normal(size=T.shape))
    res = []
    for share in (False, True):
        with Tape(pi, steps=3) as tape:
            if share:
                tape.share_vflux()
                with pytest.raises(RuntimeError, match="slot 0 first"):
                    tape.forward(1, *args, T, To, DT)
            states = [To, T]
            for s in range(3):
                states.append(tape.forward(s, *args, states[-1], states[-2], DT))
            grads = [advect_one_fct_vjp(pi, *args, states[s + 1], states[s], gTn, dt=DT,
                                        tape=tape, slot=s) for s in range(3)]
        res.append((states, grads))
    for a, b in zip(res[0][0], res[1][0]):
        assert torch.equal(a, b)
    for ga, gb in zip(res[0][1], res[1][1]):
        for x, y in zip(ga, gb):
            assert torch.equal(x, y)
