"""The ``w`` producer on the GPU: ``compute_w(mesh, uv, helem)`` (fesom_jax/ale.py:309-365).

Same signature and result as the reference function (vertical velocity at interfaces
``[nod2D, nl]`` from discrete continuity), computed by ``fct_compute_w`` in
``libfesom_fct.so`` on torch CUDA tensors; no CPU fallback.
"""

from __future__ import annotations

import ctypes as C

from . import _lib
from .mesh import Mesh
from .tracer_adv import _torch, get_plan


def compute_w(mesh: Mesh, uv, helem, out=None, stream=None):
    torch = _torch()
    if not (uv.is_cuda and helem.is_cuda):
        raise TypeError("compute_w: uv and helem must be CUDA tensors")
    dev = uv.device.index if uv.device.index is not None else torch.cuda.current_device()
    plan = get_plan(mesh, dev)
    N, E, nl = mesh.nod2D, mesh.elem2D, mesh.nl
    if tuple(uv.shape) != (E, nl, 2) or tuple(helem.shape) != (E, nl):
        raise ValueError("compute_w: uv must be [elem2D, nl, 2] and helem [elem2D, nl]")
    if uv.dtype != torch.float64 or helem.dtype != torch.float64:
        raise TypeError("compute_w: float64 tensors required")
    uv, helem = uv.contiguous(), helem.contiguous()
    if out is None:
        out = torch.empty((N, nl), dtype=torch.float64, device=uv.device)
    s = stream if stream is not None else torch.cuda.current_stream(uv.device).cuda_stream
    _lib.check(_lib.lib().fct_compute_w(plan.handle, C.c_void_p(uv.data_ptr()),
                                        C.c_void_p(helem.data_ptr()),
                                        C.c_void_p(out.data_ptr()), C.c_void_p(int(s))))
    return out
