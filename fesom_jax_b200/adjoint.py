"""Reverse mode of the FCT step: the autodiff surface of the reference.

The reference differentiates ``advect_one_fct`` with ``jax.grad`` through its JAX
primitives (fesom_jax/integrate.py:43-169, docs/LIMITER_GRADIENTS.md). Here the
vector-Jacobian product is hand-written CUDA (``fct_adjoint`` in ``libfesom_fct.so``)
and exposed three ways:

* :func:`advect_one_fct_vjp` / :func:`compute_w_vjp` -- explicit VJPs;
* :class:`AdvectFCT` -- a ``torch.autograd.Function`` (forward = ``fct_forward``,
  backward = ``fct_adjoint``), the custom-VJP wrapper: ``loss.backward()`` through the
  CUDA step;
* :func:`chain_loss_and_grad` -- a K-step loss. Checkpointing is either a
  :class:`Tape` (every step's forward intermediates are kept, as jax.grad keeps its
  residuals, so the reverse pass only runs the reverse kernels) or per-step
  recomputation (only the K+1 tracer states are kept; each step's intermediates are
  recomputed inside its adjoint call). Both give the same bits.

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
    L.fct_adjoint_ex.argtypes = [C.c_void_p, C.POINTER(_lib.FctFields), C.c_void_p,
                                 C.c_double, C.c_int, C.POINTER(FctGrads), C.c_void_p, C.c_int,
                                 C.c_int, C.c_void_p]
    L.fct_compute_w_adjoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_int, C.c_void_p]
    L.fct_adjoint_flush_uv.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                       C.c_void_p]
    L.fct_tape_bytes.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int64)]
    L.fct_tape_create.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64,
                                  C.POINTER(C.c_void_p)]
    L.fct_tape_destroy.argtypes = [C.c_void_p]
    L.fct_forward_taped.argtypes = [C.c_void_p, C.POINTER(_lib.FctFields), C.c_double, C.c_int,
                                    C.c_void_p, C.c_int, C.c_void_p]
    L.fct_tape_mark_recorded.argtypes = [C.c_void_p, C.c_int, C.c_double]
    L.fct_tape_share_vflux.argtypes = [C.c_void_p]
    for n in ("fct_plan_reserve_adjoint", "fct_adjoint", "fct_adjoint_ex",
              "fct_compute_w_adjoint", "fct_adjoint_flush_uv", "fct_tape_bytes",
              "fct_tape_create", "fct_tape_destroy",
              "fct_forward_taped", "fct_tape_mark_recorded", "fct_tape_share_vflux"):
        getattr(L, n).restype = C.c_int
    L._adj_bound = True
    return L


# accumulate bits of fct_adjoint_ex (include/fesom_fct.h); DEFER_UV: the step's volume-flux
# cotangents go into the plan's running sum (fct_adjoint_flush_uv transposes it once)
ACC_T, ACC_T_OLD, ACC_UV, ACC_W, DEFER_UV = 1, 2, 4, 8, 16


def _fields(mesh: Mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, T_new=None, Z3d=None,
            zbar3=None):
    f = _lib.FctFields()
    f.uv, f.w_e, f.helem = uv.data_ptr(), w_e.data_ptr(), helem.data_ptr()
    f.hnode, f.hnode_new = hnode.data_ptr(), hnode_new.data_ptr()
    f.T, f.T_old = T.data_ptr(), T_old.data_ptr()
    f.T_new = T_new.data_ptr() if T_new is not None else None
    f.tracer_stride = mesh.nod2D * mesh.nl
    f.Z3d = Z3d.data_ptr() if Z3d is not None else None
    f.zbar3 = zbar3.data_ptr() if zbar3 is not None else None
    f.w_i = None
    return f


class Tape:
    """Forward intermediates of up to ``steps`` FCT steps of one mesh (``fct_tape_*``):
    :meth:`forward` runs a step and keeps its intermediates in a slot, and the adjoint of
    that slot (``advect_one_fct_vjp(..., tape=, slot=)``) runs only the reverse kernels.
    The memory (:meth:`nbytes`) comes from torch's caching allocator, so tapes of the same
    size reuse it."""

    def __init__(self, mesh: Mesh, steps: int, ntr: int = 1, device: int | None = None):
        torch = _torch()
        dev = torch.cuda.current_device() if device is None else int(device)
        self.mesh, self.steps, self.ntr, self.device = mesh, int(steps), int(ntr), dev
        self.plan = get_plan(mesh, dev)
        L = _bind(_lib.lib())
        nb = Tape.nbytes(mesh, steps, ntr, dev)
        self._mem = torch.empty(max(nb // 8, 1), dtype=torch.float64,
                                device=torch.device("cuda", dev))
        h = C.c_void_p()
        with self.plan._lock:
            _lib.check(L.fct_tape_create(self.plan.handle, self.ntr, self.steps,
                                         C.c_void_p(self._mem.data_ptr()), nb, C.byref(h)))
        self._h = h

    @staticmethod
    def nbytes(mesh: Mesh, steps: int, ntr: int = 1, device: int = 0) -> int:
        out = C.c_int64()
        L = _bind(_lib.lib())
        _lib.check(L.fct_tape_bytes(get_plan(mesh, device).handle, int(ntr), int(steps),
                                    C.byref(out)))
        return int(out.value)

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def forward(self, slot: int, uv, w_e, helem, hnode, hnode_new, T, T_old, dt: float,
                Z3d=None, zbar3=None, out=None):
        """``fct_forward`` of one step, recorded in ``slot``; returns ``T_new``."""
        torch = _torch()
        ntr = 1 if T.dim() == 2 else int(T.shape[0])
        T, T_old = T.contiguous(), T_old.contiguous()
        if out is None:
            out = torch.empty_like(T)
        f = _fields(self.mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, out, Z3d, zbar3)
        with self.plan._lock:
            _lib.check(_bind(_lib.lib()).fct_forward_taped(
                self.plan.handle, C.byref(f), float(dt), ntr, self._h, int(slot),
                _stream(torch, T.device)))
        return out

    def share_vflux(self) -> None:
        """Every step recorded on this tape uses the same uv and helem: slot 0's forward
        computes the edge volume fluxes and the other slots reuse them
        (``fct_tape_share_vflux``; record slot 0 first)."""
        _lib.check(_bind(_lib.lib()).fct_tape_share_vflux(self._h))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fct_tape_destroy(self._h)
            self._h = C.c_void_p()
        self._mem = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _adjoint(plan, f, gT_new, dt, ntr, gT, gTo, guv, gw, tape=None, slot=0, acc=0, dev=None):
    torch = _torch()
    L = _bind(_lib.lib())
    g = FctGrads(gT.data_ptr(), gTo.data_ptr(), guv.data_ptr() if guv is not None else None,
                 gw.data_ptr())
    with plan._lock:
        _lib.check(L.fct_adjoint_ex(plan.handle, C.byref(f), C.c_void_p(gT_new.data_ptr()),
                                    float(dt), ntr, C.byref(g),
                                    tape.handle if tape is not None else None, int(slot),
                                    int(acc), _stream(torch, dev)))


def _stream(torch, dev):
    return C.c_void_p(int(torch.cuda.current_stream(dev).cuda_stream))


def advect_one_fct_vjp(mesh: Mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, gT_new, *,
                       dt: float, Z3d=None, zbar3=None, tape: Tape | None = None,
                       slot: int = 0):
    """Cotangents ``(gT, gT_old, guv, gw_e)`` of one FCT step for the output cotangent
    ``gT_new`` (CUDA float64 tensors; ``T`` may carry a leading tracer axis, in which case
    ``guv``/``gw_e`` are summed over the tracers). With ``tape``, the step recorded in
    ``slot`` (by :meth:`Tape.forward` with the same inputs) is not recomputed."""
    torch = _torch()
    dev = T.device
    plan = get_plan(mesh, dev.index if dev.index is not None else torch.cuda.current_device())
    L = _bind(_lib.lib())
    ntr = 1 if T.dim() == 2 else int(T.shape[0])
    if tape is None:
        _lib.check(L.fct_plan_reserve_adjoint(plan.handle, ntr))
    T, T_old, gT_new = T.contiguous(), T_old.contiguous(), gT_new.contiguous()
    f = _fields(mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, None, Z3d, zbar3)
    gT, gTo = torch.empty_like(T), torch.empty_like(T)
    guv, gw = torch.empty_like(uv), torch.empty_like(w_e)
    _adjoint(plan, f, gT_new, dt, ntr, gT, gTo, guv, gw, tape, slot, 0, dev)
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


def _tape_fits(torch, mesh: Mesh, steps: int, dev) -> bool:
    """A tape of ``steps`` one-tracer steps fits in half of the memory torch could hand out
    (free device memory plus its cached, unused blocks)."""
    need = Tape.nbytes(mesh, steps, 1, dev.index)
    free, _ = torch.cuda.mem_get_info(dev)
    cached = torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
    return need <= 0.5 * (free + cached)


def chain_loss_and_grad(mesh: Mesh, T0, uv, helem, hnode, hnode_new, target, steps: int, *,
                        dt: float, T_old0=None, checkpoint: str = "auto",
                        return_gT_old: bool = False, defer_uv: bool = True, tape=None):
    """Loss ``sum_n areasvol[n,0] * (T_K[n,0] - target_n)^2`` after ``steps`` FCT steps
    with ``w_e = compute_w(uv)`` inside the loss, and its gradients w.r.t. the initial
    ``T0`` and ``uv``. ``checkpoint``: ``"tape"`` keeps every step's intermediates
    (:class:`Tape`), ``"recompute"`` keeps only the K+1 states and recomputes each step
    inside its adjoint call, ``"auto"`` takes the tape when it fits in half the free
    memory. The cotangents are accumulated in place (``fct_adjoint_ex``). With
    ``defer_uv`` (the default) the steps' volume-flux cotangents are summed on the device
    and transposed into the uv gradient once after the last step (uv and helem are the
    same at every step), instead of once per step; the result agrees to rounding.
    ``tape``: a :class:`Tape` of this mesh with at least ``steps`` slots, reused across
    calls (it stays open); by default tape mode allocates one per call.

    Returns ``(loss, gT0, guv)``; ``T_old0`` defaults to ``T0`` (step-1 convention), and
    then ``gT0`` is the gradient through both inputs. With ``return_gT_old`` and an explicit
    ``T_old0`` the gradient w.r.t. ``T_old0`` is appended: ``(loss, gT0, guv, gT_old0)``."""
    torch = _torch()
    from .ale import compute_w
    dev = T0.device
    plan = get_plan(mesh, dev.index)
    if checkpoint not in ("auto", "tape", "recompute"):
        raise ValueError(f"checkpoint={checkpoint!r}: expected auto, tape or recompute")
    own_tape = False
    if tape is not None:
        if tape.mesh is not mesh or tape.steps < steps or tape.device != dev.index:
            raise ValueError("tape: needs this mesh, this device and >= steps slots")
        checkpoint = "tape"
    elif checkpoint == "auto":
        checkpoint = "tape" if _tape_fits(torch, mesh, steps, dev) else "recompute"
    if tape is None and checkpoint == "tape":
        tape, own_tape = Tape(mesh, steps, 1, dev.index), True
    if tape is not None:
        tape.share_vflux()   # uv and helem are the same at every step of the chain
    if tape is None:
        _lib.check(_bind(_lib.lib()).fct_plan_reserve_adjoint(plan.handle, 1))
    try:
        # loss weights and target on the device first: no host copy between the forward
        # and the reverse pass, which would wait for the forward to finish
        av0 = torch.from_numpy(mesh.areasvol[:, 0].copy()).to(dev)
        tgt = target.to(dev)
        w = compute_w(mesh, uv, helem)
        states = [T_old0 if T_old0 is not None else T0, T0]   # [T_{-1}, T_0, T_1, ...]
        for s in range(steps):
            if tape is not None:
                states.append(tape.forward(s, uv, w, helem, hnode, hnode_new, states[-1],
                                           states[-2], dt))
            else:   # the stage-by-stage kernels: the trajectory the tape would record
                states.append(plan.forward(uv, w, helem, hnode, hnode_new, states[-1],
                                           states[-2], dt, stagewise=True))
        TK = states[-1]
        diff = TK[:, 0] - tgt
        loss_t = (av0 * diff * diff).sum()   # read back after the reverse pass is queued
        lam = torch.zeros_like(TK)
        lam[:, 0] = 2.0 * av0 * diff
        guv = torch.zeros_like(uv)
        gw = torch.zeros_like(w)
        carry = torch.zeros_like(TK)   # cotangent reaching T_s through step s+1's T_old input
        for s in range(steps - 1, -1, -1):
            T_s, T_sm1 = states[s + 1], states[s]
            f = _fields(mesh, uv, w, helem, hnode, hnode_new, T_s, T_sm1)
            gTo = torch.empty_like(TK)
            # gT accumulates into carry: the cotangent of T_s is gT + carry
            _adjoint(plan, f, lam, dt, 1, carry, gTo, None if defer_uv else guv, gw, tape, s,
                     ACC_T | ACC_W | (DEFER_UV if defer_uv else ACC_UV), dev)
            lam, carry = carry, gTo
        gT0 = lam + (carry if T_old0 is None else 0.0)
        if defer_uv:
            with plan._lock:
                _lib.check(_bind(_lib.lib()).fct_adjoint_flush_uv(
                    plan.handle, C.c_void_p(helem.data_ptr()), C.c_void_p(guv.data_ptr()), 1,
                    _stream(torch, dev)))
        compute_w_vjp(mesh, gw, helem, guv)
        loss = float(loss_t.item())
    finally:
        if own_tape:
            tape.close()
    if return_gT_old:
        if T_old0 is None:
            raise ValueError("return_gT_old needs an explicit T_old0")
        return loss, gT0, guv, carry
    return loss, gT0, guv
