"""Drop-in FCT tracer advection on B200: the reference's call signature over the CUDA path.

``advect_one_fct(mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, *, dt, exch=None,
Z3d=None, zbar3=None, w_i=None) -> (T_new, T_old_new)`` keeps the signature, argument
meaning and return convention of fesom_jax/tracer_adv.py:532-578: ``T_old_new`` is ``T``
itself (the AB2 ``valuesold`` save, an alias, not a copy). The arithmetic runs in the
CUDA kernels of ``libfesom_fct.so``; there is no CPU fallback.

Arrays may be torch CUDA tensors (float64; computed in place on the current stream, no
host round trip) or numpy arrays (copied to the GPU and the result copied back). ``T``
may also carry a leading tracer axis ``[ntr, nod2D, nl]``: several tracers that share
velocities and thicknesses advance in one launch sequence (T and S of
fesom_jax/step.py:409-416 are ``ntr = 2``).

``exch`` (the sharded halo exchange) is not supported on this single-GPU path and raises
``NotImplementedError``; it never silently falls back.
"""

from __future__ import annotations

import ctypes as C
import threading
import weakref

import numpy as np

from . import _lib
from .mesh import Mesh

DT_DEFAULT = 2400.0  # fesom_jax/config.py:100

_plans: "weakref.WeakKeyDictionary[Mesh, dict]" = weakref.WeakKeyDictionary()
_plans_lock = threading.Lock()


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("fesom_jax_b200 FCT needs a CUDA GPU; there is no CPU fallback")
    return torch


class FctPlan:
    """A mesh uploaded to one GPU plus reserved workspace (``fct_plan_create``)."""

    def __init__(self, mesh: Mesh, device: int = 0, max_tracers: int = 2):
        mesh.validate()
        self.mesh = mesh
        self.device = int(device)
        keep: list = []
        desc = _lib.mesh_desc(mesh, keep)
        h = C.c_void_p()
        _lib.check(_lib.lib().fct_plan_create(C.byref(desc), self.device, int(max_tracers),
                                              C.byref(h)))
        self._h = h
        self._lock = threading.Lock()

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def info(self) -> dict:
        out = (C.c_int64 * 8)()
        _lib.check(_lib.lib().fct_plan_info(self._h, out))
        keys = ("nod2D", "elem2D", "edge2D", "nl", "wet_node_layers", "wet_elem_layers",
                "wet_edge_layers", "max_tracers")
        return dict(zip(keys, [int(v) for v in out]))

    def reserve(self, ntr: int) -> None:
        _lib.check(_lib.lib().fct_plan_reserve(self._h, int(ntr)))

    def health(self, stream=None) -> int:
        """Non-finite ``T_new`` values this plan's forward calls wrote since the previous
        check (``fct_plan_health``; synchronises the stream). The finiteness gate of the
        reference's diagnostics (fesom_jax/diagnostics.py:31-101)."""
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        n = C.c_int64(0)
        _lib.health_status(_lib.lib().fct_plan_health(self._h, C.c_void_p(int(s)), C.byref(n)))
        return int(n.value)

    def fill_workspace(self, byte: int = 0xFF, stream=None) -> None:
        """Debug aid: fill the plan workspace with ``byte`` (0xFF: NaN doubles)."""
        torch = _torch()
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        L = _lib.lib()
        L.fct_plan_fill_workspace.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.fct_plan_fill_workspace.restype = C.c_int
        _lib.check(L.fct_plan_fill_workspace(self._h, int(byte), C.c_void_p(int(s))))

    def set_mapping(self, tracers_per_thread: int, levels_per_thread: int) -> None:
        """Thread mapping of the fused stages (tracers and column levels per thread, each
        1, 2, 4 or 8); a tuning knob, the results do not depend on it."""
        L = _lib.lib()
        L.fct_plan_set_mapping.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.fct_plan_set_mapping.restype = C.c_int
        _lib.check(L.fct_plan_set_mapping(self._h, int(tracers_per_thread),
                                          int(levels_per_thread)))

    def autotune(self, args, dt: float, candidates=((1, 1), (1, 2), (1, 4), (2, 1), (2, 2),
                                                    (2, 4)), reps: int = 20, cache=None) -> dict:
        """Time ``forward(*args, dt)`` (device tensors, the call to be tuned for) under each
        (tracers, levels) per-thread mapping and keep the fastest; returns ``{"TxL": ms}``.
        ``cache`` (a :class:`fesom_jax_b200.tuning.TuningCache`, or ``True`` for the default
        file): an entry for this GPU model, mesh and tracer count is applied without
        timing (returns ``{"cached": "TxL"}``); otherwise the choice is stored."""
        from . import tuning
        if cache is True:
            cache = tuning.TuningCache()
        ck = None
        if cache is not None:
            T = args[5]
            ck = tuning.key("plan", tuning.gpu_name(self.device), [self.mesh],
                            ntr=int(T.shape[0]) if T.dim() == 3 else 1)
            hit = cache.get(ck)
            if hit:
                self.set_mapping(*hit["mapping"])
                return {"cached": f"{hit['mapping'][0]}x{hit['mapping'][1]}"}
        torch = _torch()
        dev = torch.device("cuda", self.device)
        stream = torch.cuda.current_stream(dev)
        out = torch.empty_like(args[5])
        times = {}
        for c, lv in candidates:
            self.set_mapping(c, lv)
            for _ in range(3):
                self.forward(*args, dt, out=out)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(reps):
                self.forward(*args, dt, out=out)
            e1.record(stream)
            e1.synchronize()
            times[(c, lv)] = e0.elapsed_time(e1) / reps
        best = min(times, key=times.get)
        self.set_mapping(*best)
        if cache is not None:
            cache.put(ck, dict(mapping=list(best), ms=times[best]))
        return {f"{c}x{lv}": v for (c, lv), v in times.items()}

    def set_fused(self, fused: bool) -> None:
        """Fused stage kernels (default) or one kernel per reference stage; same bits."""
        _lib.check(_lib.lib().fct_plan_set_fused(self._h, int(bool(fused))))

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            _lib.lib().fct_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def forward(self, uv, w_e, helem, hnode, hnode_new, T, T_old, dt: float, out=None,
                Z3d=None, zbar3=None, w_i=None, stream=None, stagewise: bool = False):
        """One FCT step on device tensors; returns ``T_new`` (same shape as ``T``).
        ``stagewise`` runs one kernel per reference stage (``fct_forward_ex``), the kernels
        the reverse pass recomputes with (needs the plan's adjoint reservation)."""
        torch = _torch()
        m = self.mesh
        N, E, nl = m.nod2D, m.elem2D, m.nl
        ntr = 1 if T.dim() == 2 else int(T.shape[0])
        dev = torch.device("cuda", self.device)

        def chk(x, shape, name):
            if x is None:
                return None
            if not (x.is_cuda and x.dtype == torch.float64 and x.device == dev):
                raise TypeError(f"{name}: need a float64 tensor on {dev}")
            if tuple(x.shape) != tuple(shape):
                raise ValueError(f"{name}: shape {tuple(x.shape)} != {tuple(shape)}")
            if not x.is_contiguous():
                raise ValueError(f"{name}: must be contiguous")
            return x

        tshape = (N, nl) if T.dim() == 2 else (ntr, N, nl)
        chk(uv, (E, nl, 2), "uv"); chk(w_e, (N, nl), "w_e"); chk(helem, (E, nl), "helem")
        chk(hnode, (N, nl), "hnode"); chk(hnode_new, (N, nl), "hnode_new")
        chk(T, tshape, "T"); chk(T_old, tshape, "T_old")
        chk(Z3d, (N, nl), "Z3d"); chk(zbar3, (N, nl), "zbar3"); chk(w_i, (N, nl), "w_i")
        if out is None:
            out = torch.empty_like(T)
        chk(out, tshape, "out")
        if ntr > self.info()["max_tracers"]:
            self.reserve(ntr)
        f = _lib.FctFields()
        f.uv, f.w_e, f.helem = uv.data_ptr(), w_e.data_ptr(), helem.data_ptr()
        f.hnode, f.hnode_new = hnode.data_ptr(), hnode_new.data_ptr()
        f.T, f.T_old, f.T_new = T.data_ptr(), T_old.data_ptr(), out.data_ptr()
        f.tracer_stride = N * nl
        f.Z3d = Z3d.data_ptr() if Z3d is not None else None
        f.zbar3 = zbar3.data_ptr() if zbar3 is not None else None
        f.w_i = w_i.data_ptr() if w_i is not None else None
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        # the library orders calls on one plan on the GPU; the lock keeps the host-side
        # enqueue of concurrent Python threads whole
        L = _lib.lib()
        with self._lock:
            if stagewise:
                L.fct_forward_ex.argtypes = [C.c_void_p, C.POINTER(_lib.FctFields), C.c_double,
                                             C.c_int, C.c_int, C.c_void_p]
                L.fct_forward_ex.restype = C.c_int
                _lib.check(L.fct_forward_ex(self._h, C.byref(f), float(dt), ntr, 1,
                                            C.c_void_p(int(s))))
            else:
                _lib.check(L.fct_forward(self._h, C.byref(f), float(dt), ntr,
                                         C.c_void_p(int(s))))
        return out


def get_plan(mesh: Mesh, device: int = 0) -> FctPlan:
    """The cached plan of ``mesh`` on ``device`` (created on first use)."""
    with _plans_lock:
        per = _plans.setdefault(mesh, {})
        p = per.get(device)
        if p is None:
            p = per[device] = FctPlan(mesh, device, max_tracers=1)   # grows on demand
        return p


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def advect_one_fct(mesh: Mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, *,
                   dt: float = DT_DEFAULT, exch=None, Z3d=None, zbar3=None, w_i=None):
    """One tracer's FCT advection + ALE reconstruction (fesom_jax/tracer_adv.py:532-578).

    Returns ``(T_new, T_old_new)`` with ``T_old_new`` the very ``T`` object passed in.
    """
    if exch is not None:
        raise NotImplementedError("exch (sharded halo exchange) is not supported: the B200 "
                                  "FCT path runs one instance per GPU")
    if (Z3d is None) != (zbar3 is None):
        raise ValueError("Z3d and zbar3 must be given together")
    torch = _torch()
    if _is_torch(T):
        dev = T.device.index if T.device.index is not None else torch.cuda.current_device()
        plan = get_plan(mesh, dev)
        T_new = plan.forward(uv, w_e, helem, hnode, hnode_new, T, T_old, dt,
                             Z3d=Z3d, zbar3=zbar3, w_i=w_i)
        return T_new, T
    # host arrays: upload, compute, download
    dev = torch.cuda.current_device()
    plan = get_plan(mesh, dev)

    def up(x):
        if x is None:
            return None
        return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).to(
            device=f"cuda:{dev}", non_blocking=False)

    args = [up(a) for a in (uv, w_e, helem, hnode, hnode_new, T, T_old)]
    T_new = plan.forward(*args, dt, Z3d=up(Z3d), zbar3=up(zbar3), w_i=up(w_i))
    return T_new.cpu().numpy(), T
