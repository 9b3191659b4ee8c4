"""Reverse mode of the FCT step: the autodiff surface of the reference.

The reference differentiates ``advect_one_fct`` with ``jax.grad`` through its JAX
primitives (fesom_jax/integrate.py:43-169, docs/LIMITER_GRADIENTS.md). Here the
vector-Jacobian product is hand-written CUDA (``fct_adjoint`` in ``libfesom_fct.so``)
and exposed three ways:

* :func:`advect_one_fct_vjp` / :func:`compute_w_vjp` -- explicit VJPs;
* :class:`AdvectFCT` -- a ``torch.autograd.Function`` (forward = ``fct_forward``,
  backward = ``fct_adjoint``), the custom-VJP wrapper: ``loss.backward()`` through the
  CUDA step;
* :func:`chain_loss_and_grad` -- a K-step loss with per-step recomputation
  checkpointing: only the K+1 tracer states are stored; each step's intermediates are
  recomputed inside its adjoint call.

Subgradients follow JAX's conventions (equal split at max/min ties, even split over tied
segment maxima, ``abs'(0) = 0``).
"""

from __future__ import annotations

import ctypes as C

from . import _lib
from .mesh import Mesh
from .tracer_adv import _torch, get_plan


class FctGrads(C.Structure):
    _fields_ = [("gT", C.c_void_p), ("gT_old", C.c_void_p), ("guv", C.c_void_p),
                ("gw_e", C.c_void_p)]


def _bind(L):
    if getattr(L, "_adj_bound", False):
        return L
    L.fct_plan_reserve_adjoint.argtypes = [C.c_void_p, C.c_int]
    L.fct_adjoint.argtypes = [C.c_void_p, C.POINTER(_lib.FctFields), C.c_void_p, C.c_double,
                              C.c_int, C.POINTER(FctGrads), C.c_void_p]
    L.fct_compute_w_adjoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_int, C.c_void_p]
    for n in ("fct_plan_reserve_adjoint", "fct_adjoint", "fct_compute_w_adjoint"):
        getattr(L, n).restype = C.c_int
    L._adj_bound = True
    return L


def _stream(torch, dev):
    return C.c_void_p(int(torch.cuda.current_stream(dev).cuda_stream))


def advect_one_fct_vjp(mesh: Mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, gT_new, *,
                       dt: float, Z3d=None, zbar3=None):
    """Cotangents ``(gT, gT_old, guv, gw_e)`` of one FCT step for the output cotangent
    ``gT_new`` (CUDA float64 tensors; ``T`` may carry a leading tracer axis, in which case
    ``guv``/``gw_e`` are summed over the tracers)."""
    torch = _torch()
    dev = T.device
    plan = get_plan(mesh, dev.index if dev.index is not None else torch.cuda.current_device())
    L = _bind(_lib.lib())
    ntr = 1 if T.dim() == 2 else int(T.shape[0])
    _lib.check(L.fct_plan_reserve_adjoint(plan.handle, ntr))
    T, T_old, gT_new = T.contiguous(), T_old.contiguous(), gT_new.contiguous()
    f = _lib.FctFields()
    f.uv, f.w_e, f.helem = uv.data_ptr(), w_e.data_ptr(), helem.data_ptr()
    f.hnode, f.hnode_new = hnode.data_ptr(), hnode_new.data_ptr()
    f.T, f.T_old, f.T_new = T.data_ptr(), T_old.data_ptr(), None
    f.tracer_stride = mesh.nod2D * mesh.nl
    f.Z3d = Z3d.data_ptr() if Z3d is not None else None
    f.zbar3 = zbar3.data_ptr() if zbar3 is not None else None
    f.w_i = None
    gT, gTo = torch.empty_like(T), torch.empty_like(T)
    guv, gw = torch.empty_like(uv), torch.empty_like(w_e)
    g = FctGrads(gT.data_ptr(), gTo.data_ptr(), guv.data_ptr(), gw.data_ptr())
    with plan._lock:
        _lib.check(L.fct_adjoint(plan.handle, C.byref(f), C.c_void_p(gT_new.data_ptr()),
                                 float(dt), ntr, C.byref(g), _stream(torch, dev)))
    return gT, gTo, guv, gw


def compute_w_vjp(mesh: Mesh, gw, helem, guv=None):
    """Cotangent of ``uv`` for ``w = compute_w(mesh, uv, helem)`` (fesom_jax/ale.py:309-365);
    adds into ``guv`` when given."""
    torch = _torch()
    dev = gw.device
    plan = get_plan(mesh, dev.index if dev.index is not None else torch.cuda.current_device())
    L = _bind(_lib.lib())
    _lib.check(L.fct_plan_reserve_adjoint(plan.handle, 1))
    acc = 1 if guv is not None else 0
    if guv is None:
        guv = torch.empty((mesh.elem2D, mesh.nl, 2), dtype=torch.float64, device=dev)
    gw = gw.contiguous()
    with plan._lock:
        _lib.check(L.fct_compute_w_adjoint(plan.handle, C.c_void_p(gw.data_ptr()),
                                           C.c_void_p(helem.data_ptr()),
                                           C.c_void_p(guv.data_ptr()), acc,
                                           _stream(torch, dev)))
    return guv


def _autograd_function():
    torch = _torch()

    class AdvectFCT(torch.autograd.Function):
        """``T_new = AdvectFCT.apply(mesh, dt, uv, w_e, helem, hnode, hnode_new, T, T_old)``
        with gradients w.r.t. ``uv``, ``w_e``, ``T`` and ``T_old``."""

        @staticmethod
        def forward(ctx, mesh, dt, uv, w_e, helem, hnode, hnode_new, T, T_old):
            plan = get_plan(mesh, T.device.index)
            T_new = plan.forward(uv, w_e, helem, hnode, hnode_new, T.contiguous(),
                                 T_old.contiguous(), dt)
            ctx.mesh, ctx.dt = mesh, dt
            ctx.save_for_backward(uv, w_e, helem, hnode, hnode_new, T, T_old)
            return T_new

        @staticmethod
        def backward(ctx, gT_new):
            uv, w_e, helem, hnode, hnode_new, T, T_old = ctx.saved_tensors
            gT, gTo, guv, gw = advect_one_fct_vjp(ctx.mesh, uv, w_e, helem, hnode, hnode_new,
                                                  T, T_old, gT_new, dt=ctx.dt)
            return None, None, guv, gw, None, None, None, gT, gTo

    class ComputeW(torch.autograd.Function):
        """``w = ComputeW.apply(mesh, uv, helem)`` with gradient w.r.t. ``uv``."""

        @staticmethod
        def forward(ctx, mesh, uv, helem):
            from .ale import compute_w
            ctx.mesh = mesh
            ctx.save_for_backward(helem)
            return compute_w(mesh, uv, helem)

        @staticmethod
        def backward(ctx, gw):
            (helem,) = ctx.saved_tensors
            return None, compute_w_vjp(ctx.mesh, gw, helem), None

    return AdvectFCT, ComputeW


_FUNCS = None


def functions():
    """``(AdvectFCT, ComputeW)`` autograd functions (built on first use)."""
    global _FUNCS
    if _FUNCS is None:
        _FUNCS = _autograd_function()
    return _FUNCS


def chain_loss_and_grad(mesh: Mesh, T0, uv, helem, hnode, hnode_new, target, steps: int, *,
                        dt: float, T_old0=None):
    """Loss ``sum_n areasvol[n,0] * (T_K[n,0] - target_n)^2`` after ``steps`` FCT steps
    with ``w_e = compute_w(uv)`` inside the loss, and its gradients w.r.t. the initial
    ``T0`` and ``uv``. Per-step recomputation checkpointing: the K+1 states are kept,
    every step's intermediates are recomputed in its adjoint call.

    Returns ``(loss, gT0, guv)``; ``T_old0`` defaults to ``T0`` (step-1 convention)."""
    torch = _torch()
    from .ale import compute_w
    plan = get_plan(mesh, T0.device.index)
    w = compute_w(mesh, uv, helem)
    states = [T_old0 if T_old0 is not None else T0, T0]   # [T_{-1}, T_0, T_1, ...]
    for _ in range(steps):
        states.append(plan.forward(uv, w, helem, hnode, hnode_new, states[-1], states[-2], dt))
    TK = states[-1]
    av0 = torch.from_numpy(mesh.areasvol[:, 0].copy()).to(T0.device)
    tgt = target.to(T0.device)
    diff = TK[:, 0] - tgt
    loss = float((av0 * diff * diff).sum().item())
    lam = torch.zeros_like(TK)
    lam[:, 0] = 2.0 * av0 * diff
    guv = torch.zeros_like(uv)
    gw = torch.zeros_like(w)
    carry = torch.zeros_like(TK)   # cotangent reaching T_s through step s+1's T_old input
    for s in range(steps - 1, -1, -1):
        T_s, T_sm1 = states[s + 1], states[s]
        gT, gTo, gu, gww = advect_one_fct_vjp(mesh, uv, w, helem, hnode, hnode_new, T_s, T_sm1,
                                              lam, dt=dt)
        guv += gu
        gw += gww
        lam = gT + carry
        carry = gTo
    gT0 = lam + (carry if T_old0 is None else 0.0)
    compute_w_vjp(mesh, gw, helem, guv)
    return loss, gT0, guv
