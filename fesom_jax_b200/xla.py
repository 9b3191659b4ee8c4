"""The JAX/XLA custom-call surface of the FCT step (``fct_xla_forward`` /
``fct_xla_adjoint`` in ``libfesom_fct.so``, the legacy GPU custom-call ABI).

A JAX program registers the two handlers as custom-call targets and passes the opaque
bytes built here; the reference's ``advect_one_fct`` (fesom_jax/tracer_adv.py:532-578)
and its VJP then run these handlers on XLA's stream with XLA-owned buffers. This module
builds the opaque bytes and the fixed buffer list, and can invoke the handlers the way
XLA does (device pointers, a stream, no allocation inside), which is how they are tested
without JAX.
"""

from __future__ import annotations

import ctypes as C

from . import _lib

Z3D, WI = 1, 2          # FCT_XLA_* flags
FWD_STATUS, ADJ_STATUS = 11, 14


class FctXlaOpaque(C.Structure):
    _fields_ = [("plan", C.c_uint64), ("dt", C.c_double), ("ntr", C.c_int32),
                ("flags", C.c_int32)]


def _bind(L):
    if getattr(L, "_xla_bound", False):
        return L
    for n in ("fct_xla_forward", "fct_xla_adjoint"):
        f = getattr(L, n)
        f.argtypes = [C.c_void_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_size_t]
        f.restype = None
    L._xla_bound = True
    return L


def opaque(plan, dt: float, ntr: int, *, z3d: bool = False, w_i: bool = False) -> bytes:
    """The opaque bytes of a call on ``plan`` (a ``tracer_adv.FctPlan``)."""
    o = FctXlaOpaque(plan.handle.value or 0, float(dt), int(ntr),
                     (Z3D if z3d else 0) | (WI if w_i else 0))
    return bytes(memoryview(o))


def _call(name, stream, ptrs, op: bytes):
    L = _bind(_lib.lib())
    arr = (C.c_void_p * len(ptrs))(*ptrs)
    getattr(L, name)(C.c_void_p(int(stream)), arr, op, len(op))


def forward(plan, uv, w_e, helem, hnode, hnode_new, T, T_old, dt: float, *, Z3d=None,
            zbar3=None, w_i=None, op: bytes | None = None):
    """Run ``fct_xla_forward`` as XLA would; returns ``(T_new, status tensor)``."""
    import torch
    ntr = 1 if T.dim() == 2 else int(T.shape[0])
    dummy = torch.zeros(1, dtype=torch.float64, device=T.device)
    T_new = torch.empty_like(T)
    status = torch.full((1,), 12345, dtype=torch.int32, device=T.device)
    if op is None:
        op = opaque(plan, dt, ntr, z3d=Z3d is not None, w_i=w_i is not None)
    opt = [Z3d if Z3d is not None else dummy, zbar3 if zbar3 is not None else dummy,
           w_i if w_i is not None else dummy]
    ptrs = [x.data_ptr() for x in (uv, w_e, helem, hnode, hnode_new, T, T_old, *opt,
                                   T_new, status)]
    _call("fct_xla_forward", torch.cuda.current_stream(T.device).cuda_stream, ptrs, op)
    return T_new, status


def adjoint(plan, uv, w_e, helem, hnode, hnode_new, T, T_old, gT_new, dt: float, *,
            Z3d=None, zbar3=None, op: bytes | None = None):
    """Run ``fct_xla_adjoint`` as XLA would; returns ``(gT, gT_old, guv, gw_e, status)``."""
    import torch
    ntr = 1 if T.dim() == 2 else int(T.shape[0])
    dummy = torch.zeros(1, dtype=torch.float64, device=T.device)
    gT, gTo = torch.empty_like(T), torch.empty_like(T)
    guv, gw = torch.empty_like(uv), torch.empty_like(w_e)
    status = torch.full((1,), 12345, dtype=torch.int32, device=T.device)
    if op is None:
        op = opaque(plan, dt, ntr, z3d=Z3d is not None)
    opt = [Z3d if Z3d is not None else dummy, zbar3 if zbar3 is not None else dummy]
    ptrs = [x.data_ptr() for x in (uv, w_e, helem, hnode, hnode_new, T, T_old, *opt, gT_new,
                                   gT, gTo, guv, gw, status)]
    _call("fct_xla_adjoint", torch.cuda.current_stream(T.device).cuda_stream, ptrs, op)
    return gT, gTo, guv, gw, status
