"""Implicit vertical tracer diffusion on B200: the reference's call signatures over the
CUDA kernel ``fct_vert_diff`` (fesom_jax/tracer_diff.py:68-141).

``impl_vert_diff_one(mesh, T, Kv, hnode_new, *, dt, bc_surf=None, sw_3d=None, Z3d=None)``
and ``impl_vert_diff(mesh, T, S, Kv, hnode_new, *, dt, bc_T=None, bc_S=None, sw_3d=None,
Z3d=None) -> (T_new, S_new)`` keep the reference's arguments and semantics (per-node
tridiagonal solve, surface BC increment, shortwave divergence on T only, zstar spacings,
dry levels unchanged). ``T`` may carry a leading tracer axis ``[ntr, nod2D, nl]`` (then
``bc_surf`` is ``[ntr, nod2D]`` and ``sw_3d`` applies to tracer 0). Torch CUDA tensors are
computed on the current stream; numpy arrays go to the GPU and back. No CPU fallback.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .mesh import Mesh
from .tracer_adv import DT_DEFAULT, _is_torch, _torch, get_plan


class FctVdiffFields(C.Structure):
    _fields_ = [("T", C.c_void_p), ("T_new", C.c_void_p), ("tracer_stride", C.c_int64),
                ("Kv", C.c_void_p), ("hnode_new", C.c_void_p), ("Z3d", C.c_void_p),
                ("bc_surf", C.c_void_p), ("sw_3d", C.c_void_p), ("sw_tracer", C.c_int)]


def _bind(L):
    if not getattr(L, "_vdiff_bound", False):
        L.fct_vert_diff.argtypes = [C.c_void_p, C.POINTER(FctVdiffFields), C.c_double, C.c_int,
                                    C.c_void_p]
        L.fct_vert_diff.restype = C.c_int
        L._vdiff_bound = True
    return L


def _run(mesh: Mesh, T, Kv, hnode_new, dt, bc_surf, sw_3d, Z3d, sw_tracer=0, out=None):
    torch = _torch()
    host = not _is_torch(T)
    dev = torch.cuda.current_device() if host else (
        T.device.index if T.device.index is not None else torch.cuda.current_device())

    def up(x):
        if x is None:
            return None
        if _is_torch(x):
            return x.contiguous()
        return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(f"cuda:{dev}")

    Td, Kd, hd = up(T), up(Kv), up(hnode_new)
    bd, sd, zd = up(bc_surf), up(sw_3d), up(Z3d)
    N, nl = mesh.nod2D, mesh.nl
    ntr = 1 if Td.dim() == 2 else int(Td.shape[0])
    for x, shape, name in ((Td, (N, nl) if ntr == 1 and Td.dim() == 2 else (ntr, N, nl), "T"),
                           (Kd, (N, nl), "Kv"), (hd, (N, nl), "hnode_new")):
        if tuple(x.shape) != shape or x.dtype != torch.float64 or not x.is_cuda:
            raise ValueError(f"{name}: need float64 CUDA {shape}, got {tuple(x.shape)}")
    if bd is not None and tuple(bd.shape) not in ((ntr, N),) + (((N,),) if ntr == 1 else ()):
        raise ValueError(f"bc_surf: need shape {(ntr, N)}, got {tuple(bd.shape)}")
    for x, name in ((sd, "sw_3d"), (zd, "Z3d")):
        if x is not None and tuple(x.shape) != (N, nl):
            raise ValueError(f"{name}: need shape {(N, nl)}, got {tuple(x.shape)}")
    plan = get_plan(mesh, dev)
    if ntr > plan.info()["max_tracers"]:
        plan.reserve(ntr)
    out = torch.empty_like(Td) if out is None else out
    f = FctVdiffFields()
    f.T, f.T_new, f.tracer_stride = Td.data_ptr(), out.data_ptr(), N * nl
    f.Kv, f.hnode_new = Kd.data_ptr(), hd.data_ptr()
    f.Z3d = zd.data_ptr() if zd is not None else None
    f.bc_surf = bd.data_ptr() if bd is not None else None
    f.sw_3d = sd.data_ptr() if sd is not None else None
    f.sw_tracer = sw_tracer
    L = _bind(_lib.lib())
    s = torch.cuda.current_stream(dev).cuda_stream
    with plan._lock:   # the plan workspace holds the elimination factors
        _lib.check(L.fct_vert_diff(plan.handle, C.byref(f), float(dt), ntr, C.c_void_p(int(s))))
    return out.cpu().numpy() if host else out


def impl_vert_diff_one(mesh: Mesh, T, Kv, hnode_new, *, dt: float = DT_DEFAULT,
                       bc_surf=None, sw_3d=None, Z3d=None):
    """Per-node implicit vertical diffusion of one tracer (fesom_jax/tracer_diff.py:68-123)."""
    return _run(mesh, T, Kv, hnode_new, dt, bc_surf, sw_3d, Z3d)


def impl_vert_diff(mesh: Mesh, T, S, Kv, hnode_new, *, dt: float = DT_DEFAULT,
                   bc_T=None, bc_S=None, sw_3d=None, Z3d=None):
    """T and S with the same ``Kv``; the shortwave divergence on T only
    (fesom_jax/tracer_diff.py:126-141). Returns ``(T_new, S_new)``."""
    return (_run(mesh, T, Kv, hnode_new, dt, bc_T, sw_3d, Z3d),
            _run(mesh, S, Kv, hnode_new, dt, bc_S, None, Z3d))
