"""Sea-ice FCT advection on B200: the reference's call signature over the CUDA kernels
behind ``fct_ice_solve`` (fesom_jax/ice_adv.py:175-194, ``fesom_ice_fct.c``).

``fct_solve(cfg, mesh, a_ice, m_ice, m_snow, u_ice, v_ice, exch=None) -> (a, m, m_snow)``
keeps the reference's arguments and return order; ``cfg`` is any object with
``ice_gamma_fct``, ``ice_diff`` and ``ice_dt`` (the reference's ``IceConfig`` works, and
:class:`IceConfig` here carries the same defaults). Torch CUDA tensors are computed on
the current stream; numpy arrays go to the GPU and back. ``exch`` (sharded halo
refreshes) is not supported on this single-GPU path. No CPU fallback.
"""

from __future__ import annotations

import ctypes as C
from typing import NamedTuple

import numpy as np

from . import _lib
from .mesh import Mesh
from .tracer_adv import _is_torch, _torch, get_plan


class IceConfig(NamedTuple):
    """The FCT part of the reference's ``IceConfig`` (fesom_jax/ice.py:57-62)."""
    ice_gamma_fct: float = 0.5
    ice_diff: float = 10.0
    ice_dt: float = 500.0


class FctIceFields(C.Structure):
    _fields_ = [("tracer", C.c_void_p * 3), ("tracer_new", C.c_void_p * 3),
                ("u_ice", C.c_void_p), ("v_ice", C.c_void_p)]


class FctIceConfig(C.Structure):
    _fields_ = [("dt", C.c_double), ("gamma", C.c_double), ("diff", C.c_double)]


def _bind(L):
    if not getattr(L, "_ice_bound", False):
        L.fct_ice_solve.argtypes = [C.c_void_p, C.POINTER(FctIceFields),
                                    C.POINTER(FctIceConfig), C.c_void_p]
        L.fct_ice_solve.restype = C.c_int
        L._ice_bound = True
    return L


def fct_solve(cfg, mesh: Mesh, a_ice, m_ice, m_snow, u_ice, v_ice, exch=None):
    """One sea-ice FCT step (fesom_jax/ice_adv.py:175-194); returns the advected
    ``(a_ice, m_ice, m_snow)`` before ``cut_off``."""
    if exch is not None:
        raise NotImplementedError("exch (sharded halo refresh) is not supported: the B200 "
                                  "ice FCT runs one mesh per GPU")
    torch = _torch()
    host = not _is_torch(a_ice)
    dev = torch.cuda.current_device() if host else (
        a_ice.device.index if a_ice.device.index is not None else torch.cuda.current_device())

    def up(x):
        if _is_torch(x):
            t = x.contiguous()
        else:
            t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(f"cuda:{dev}")
        if tuple(t.shape) != (mesh.nod2D,) or t.dtype != torch.float64:
            raise ValueError(f"need float64 [{mesh.nod2D}] arrays, got {tuple(t.shape)}")
        return t

    X = [up(a_ice), up(m_ice), up(m_snow)]
    u, v = up(u_ice), up(v_ice)
    out = [torch.empty_like(x) for x in X]
    f = FctIceFields()
    for i in range(3):
        f.tracer[i], f.tracer_new[i] = X[i].data_ptr(), out[i].data_ptr()
    f.u_ice, f.v_ice = u.data_ptr(), v.data_ptr()
    c = FctIceConfig(float(cfg.ice_dt), float(cfg.ice_gamma_fct), float(cfg.ice_diff))
    plan = get_plan(mesh, dev)
    L = _bind(_lib.lib())
    s = torch.cuda.current_stream(dev).cuda_stream
    with plan._lock:   # the plan workspace is the scratch
        _lib.check(L.fct_ice_solve(plan.handle, C.byref(f), C.byref(c), C.c_void_p(int(s))))
    if host:
        return tuple(o.cpu().numpy() for o in out)
    return tuple(out)
