"""Resident ensembles: many FCT instances advanced together on one GPU.

The reference advances one tracer of one model per ``advect_one_fct`` call from a host
time loop (fesom_jax/step.py:497-516, integrate.py:43-169). An :class:`Ensemble` keeps
every member's velocities, thicknesses and three rotating tracer buffers resident in HBM
and advances all members (each with ``ntr`` tracers sharing its velocities, on meshes of
any size) with the batched C ABI (``fct_batch_*``): one launch per stage for all
members of a workspace group, multi-step runs captured once as a CUDA graph.

The AB2 history rotates through the three buffers (step ``p`` reads ``T_old = buf[p%3]``,
``T = buf[(p+1)%3]`` and writes ``buf[(p+2)%3]``), which is exactly the reference's
``(T, T_old) <- advect_one_fct(..., T, T_old)`` carry with ``T_old_new = T``.
"""

from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .mesh import Mesh
from .tracer_adv import FctPlan


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("Ensemble needs a CUDA GPU; there is no CPU fallback")
    return torch


class FctInstance(C.Structure):
    _fields_ = [("plan", C.c_void_p), ("uv", C.c_void_p), ("w_e", C.c_void_p),
                ("helem", C.c_void_p), ("hnode", C.c_void_p), ("hnode_new", C.c_void_p),
                ("buf", C.c_void_p * 3), ("ntr", C.c_int), ("dt", C.c_double),
                ("Kv", C.c_void_p), ("w_derived", C.c_void_p), ("nonfinite", C.c_void_p)]


def _bind_batch(L):
    if getattr(L, "_batch_bound", False):
        return L
    L.fct_batch_create.argtypes = [C.POINTER(FctInstance), C.c_int, C.c_int64, C.POINTER(C.c_void_p)]
    L.fct_batch_destroy.argtypes = [C.c_void_p]
    L.fct_batch_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.fct_batch_prepare.argtypes = [C.c_void_p, C.c_void_p]
    L.fct_batch_step.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.fct_batch_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p]
    L.fct_batch_profile.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.c_int,
                                    C.c_void_p]
    L.fct_stage_name.restype = C.c_char_p
    L.fct_batch_set_chunk.argtypes = [C.c_void_p, C.c_int]
    L.fct_batch_set_mapping.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.fct_batch_set_stage_mapping.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.fct_batch_health.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
    L.fct_batch_fill_workspace.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    for n in ("fct_batch_create", "fct_batch_destroy", "fct_batch_info", "fct_batch_prepare",
              "fct_batch_step", "fct_batch_run", "fct_batch_profile", "fct_batch_set_chunk",
              "fct_batch_health", "fct_batch_fill_workspace", "fct_batch_set_mapping",
              "fct_batch_set_stage_mapping"):
        getattr(L, n).restype = C.c_int
    L._batch_bound = True
    return L


@dataclasses.dataclass
class Member:
    """One ensemble member: a mesh and its ``ntr`` tracers' device state."""

    mesh: Mesh
    ntr: int
    dt: float
    uv: object          # torch [E, nl, 2]
    w_e: object         # torch [N, nl]
    helem: object
    hnode: object
    hnode_new: object
    buf: object         # torch [3, N, nl, ntr] (tracers interleaved innermost)
    Kv: object = None   # torch [N, nl] or None (no vertical diffusion)
    derive_w: bool = False   # w_e recomputed from uv each step (into w_e)


class Ensemble:
    """Members resident on ``device``; see the module docstring."""

    def __init__(self, device: int = 0, workspace_budget: int = 24 << 30):
        self.torch = _torch()
        self.device = int(device)
        self.workspace_budget = int(workspace_budget)
        self.members: list[Member] = []
        self._plans: dict[int, FctPlan] = {}
        self._h = None
        self.phase = 0
        self.chunk = 2          # tracers per thread of the fused stages
        self.levels = 4         # levels per thread
        self.stage_map = [(2, 4)] * 4   # per fused stage (LO, edge, limiter, final)

    # ---------------------------------------------------------------- members
    def plan(self, mesh: Mesh) -> FctPlan:
        p = self._plans.get(id(mesh))
        if p is None:
            p = self._plans[id(mesh)] = FctPlan(mesh, self.device, max_tracers=1)
        return p

    def add_member(self, mesh: Mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, dt: float,
                   Kv=None, derive_w: bool = False) -> int:
        """Add a member (host numpy or device tensors); ``T``/``T_old`` are ``[ntr, N, nl]``.
        With ``Kv`` (``[N, nl]``) every step is followed by the implicit vertical diffusion
        of fesom_jax/tracer_diff.py:68-123 (step.py:452), in the same graph. With
        ``derive_w`` every step first derives ``w_e = compute_w(uv, helem)``
        (fesom_jax/ale.py:309-365, step.py:367) on the GPU and ``w_e`` may be None."""
        if self._h is not None:
            raise RuntimeError("members must be added before the ensemble is built")
        t = self.torch
        dev = t.device("cuda", self.device)

        def d(x):
            if isinstance(x, np.ndarray):
                return t.from_numpy(np.ascontiguousarray(x, np.float64)).to(dev)
            return x.to(device=dev, dtype=t.float64).contiguous()

        T, T_old = d(T), d(T_old)
        if T.dim() == 2:
            T, T_old = T[None], T_old[None]
        ntr = int(T.shape[0])
        N, nl = mesh.nod2D, mesh.nl
        if tuple(T.shape) != (ntr, N, nl) or tuple(T_old.shape) != (ntr, N, nl):
            raise ValueError("T/T_old must be [ntr, nod2D, nl]")
        buf = t.empty((3, N, nl, ntr), dtype=t.float64, device=dev)
        buf[0].copy_(T_old.permute(1, 2, 0))
        buf[1].copy_(T.permute(1, 2, 0))
        buf[2].copy_(T.permute(1, 2, 0))
        self.plan(mesh)
        if derive_w:
            w_e = t.empty((N, nl), dtype=t.float64, device=dev)
        self.members.append(Member(mesh, ntr, float(dt), d(uv), d(w_e), d(helem), d(hnode),
                                   d(hnode_new), buf, d(Kv) if Kv is not None else None,
                                   derive_w))
        return len(self.members) - 1

    # ------------------------------------------------------------------ build
    def build(self) -> None:
        L = _bind_batch(_lib.lib())
        n = len(self.members)
        if n == 0:
            raise ValueError("empty ensemble")
        arr = (FctInstance * n)()
        for i, mb in enumerate(self.members):
            q = arr[i]
            q.plan = self.plan(mb.mesh).handle.value
            q.uv, q.w_e, q.helem = mb.uv.data_ptr(), mb.w_e.data_ptr(), mb.helem.data_ptr()
            q.hnode, q.hnode_new = mb.hnode.data_ptr(), mb.hnode_new.data_ptr()
            for j in range(3):
                q.buf[j] = mb.buf[j].data_ptr()
            q.ntr, q.dt = mb.ntr, mb.dt
            q.Kv = mb.Kv.data_ptr() if mb.Kv is not None else None
            q.w_derived = mb.w_e.data_ptr() if mb.derive_w else None
        h = C.c_void_p()
        _lib.check(L.fct_batch_create(arr, n, self.workspace_budget, C.byref(h)))
        self._h = h
        self.phase = 0
        self.prepare()

    def info(self) -> dict:
        out = (C.c_int64 * 6)()
        _lib.check(_bind_batch(_lib.lib()).fct_batch_info(self._h, out))
        return dict(instances=out[0], groups=out[1], workspace_bytes=out[2],
                    updates_per_step=out[3], workspace_tracers=out[4],
                    launches_per_step=out[5])

    def _stream(self, stream):
        t = self.torch
        return C.c_void_p(int(stream if stream is not None
                              else t.cuda.current_stream(self.device).cuda_stream))

    def prepare(self, stream=None) -> None:
        """Make the dry levels of all three buffers equal (they never change)."""
        _lib.check(_bind_batch(_lib.lib()).fct_batch_prepare(self._h, self._stream(stream)))

    def step(self, stream=None) -> None:
        _lib.check(_bind_batch(_lib.lib()).fct_batch_step(self._h, self.phase % 3,
                                                          self._stream(stream)))
        self.phase += 1

    def run(self, steps: int, stream=None) -> None:
        """``steps`` FCT steps of every member as one CUDA graph launch."""
        _lib.check(_bind_batch(_lib.lib()).fct_batch_run(self._h, self.phase % 3, int(steps),
                                                         self._stream(stream)))
        self.phase += int(steps)

    def health(self, stream=None) -> list:
        """Per-member counts of non-finite ``T_new`` values written since the previous
        check (``fct_batch_health``; synchronises the stream). All zeros for a healthy
        ensemble; the reference's finiteness gate (fesom_jax/diagnostics.py:31-101)."""
        n = len(self.members)
        out = (C.c_int64 * n)()
        _lib.health_status(_bind_batch(_lib.lib()).fct_batch_health(
            self._h, self._stream(stream), out))
        return [int(v) for v in out]

    def fill_workspace(self, byte: int = 0xFF, stream=None) -> None:
        """Debug aid: fill the workspace arena with ``byte`` (0xFF: NaN doubles)."""
        _lib.check(_bind_batch(_lib.lib()).fct_batch_fill_workspace(self._h, int(byte),
                                                                    self._stream(stream)))

    def set_chunk(self, chunk: int) -> None:
        """Tracers per thread of the fused stages (1, 2, 4 or 8)."""
        self.set_mapping(chunk, self.levels)

    def set_mapping(self, tracers_per_thread: int, levels_per_thread: int) -> None:
        """Thread mapping of the fused stages: tracers and column levels per thread (each
        1, 2, 4 or 8; 8 tracers with at most 2 levels). Results do not depend on it."""
        _lib.check(_bind_batch(_lib.lib()).fct_batch_set_mapping(
            self._h, int(tracers_per_thread), int(levels_per_thread)))
        self.chunk, self.levels = int(tracers_per_thread), int(levels_per_thread)
        self.stage_map = [(self.chunk, self.levels)] * 4

    def set_stage_mapping(self, stage: int, tracers_per_thread: int,
                          levels_per_thread: int) -> None:
        """The mapping of one fused stage (0 LO, 1 edge, 2 limiter, 3 final)."""
        _lib.check(_bind_batch(_lib.lib()).fct_batch_set_stage_mapping(
            self._h, int(stage), int(tracers_per_thread), int(levels_per_thread)))
        self.stage_map[int(stage)] = (int(tracers_per_thread), int(levels_per_thread))

    # (tracers per thread, levels per thread) tried by autotune
    MAPPINGS = ((1, 1), (1, 2), (1, 4), (1, 8), (2, 1), (2, 2), (2, 4), (2, 8), (4, 1), (4, 2),
                (4, 4))
    # the fused stages as profile_step names them, in mapping order
    STAGES = ("node_lo", "edge_adf", "node_factors", "node_final")

    def _graph_ms(self, steps: int, reps: int) -> float:
        t = self.torch
        stream = t.cuda.current_stream(self.device)
        self.run(steps)                      # capture + warm
        e0, e1 = t.cuda.Event(enable_timing=True), t.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            self.run(steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    def autotune(self, steps: int = 2, candidates=None, reps: int = 2, cache=None) -> dict:
        """Pick the thread mapping of every fused stage: each (tracers, levels) per-thread
        candidate is timed stage by stage (profile_step) and each stage keeps its fastest;
        the per-stage choice is then timed against the best single mapping for all stages
        as ``steps``-step graph runs, and the faster stays (the member state advances while
        tuning). Returns the per-candidate stage times and the choice.

        ``cache``: a :class:`fesom_jax_b200.tuning.TuningCache` (or ``True`` for the default
        file). An entry for this GPU model, these meshes and this batch shape is applied
        without timing; otherwise the choice is stored there."""
        from . import tuning
        if cache is True:
            cache = tuning.TuningCache()
        ck = None
        if cache is not None:
            ck = tuning.key("ensemble", tuning.gpu_name(self.device),
                            {id(m.mesh): m.mesh for m in self.members}.values(),
                            members=len(self.members),
                            ntr=",".join(str(m.ntr) for m in self.members))
            hit = cache.get(ck)
            if hit:
                for i, (c, lv) in enumerate(hit["stage_map"]):
                    self.set_stage_mapping(i, c, lv)
                return dict(cached=True, key=ck, stage_map=hit["stage_map"])
        out = self._autotune(steps, candidates, reps)
        if cache is not None:
            cache.put(ck, dict(stage_map=[list(m) for m in self.stage_map],
                               per_stage_ms=out["per_stage_ms"], uniform_ms=out["uniform_ms"]))
        return out

    def _autotune(self, steps: int, candidates, reps: int) -> dict:
        ntr_max = max(m.ntr for m in self.members)
        cands = [(c, lv) for c, lv in (candidates or self.MAPPINGS) if c <= ntr_max or c == 1]
        prof = {}
        for c, lv in cands:
            self.set_mapping(c, lv)
            p = [self.profile_step() for _ in range(2)]
            prof[(c, lv)] = {st: min(q[st] for q in p) for st in self.STAGES}
        best_stage = [min(cands, key=lambda m: prof[m][st]) for st in self.STAGES]
        uniform = min(cands, key=lambda m: sum(prof[m].values()))
        self.set_mapping(*uniform)
        t_uniform = self._graph_ms(steps, reps)
        for i, m in enumerate(best_stage):
            self.set_stage_mapping(i, *m)
        t_stage = self._graph_ms(steps, reps)
        if t_uniform < t_stage:
            self.set_mapping(*uniform)
        return dict(stage_ms={f"{c}x{lv}": prof[(c, lv)] for c, lv in cands},
                    per_stage={st: f"{m[0]}x{m[1]}" for st, m in zip(self.STAGES, best_stage)},
                    per_stage_ms=t_stage, uniform=f"{uniform[0]}x{uniform[1]}",
                    uniform_ms=t_uniform,
                    chosen="per_stage" if t_stage <= t_uniform else "uniform")

    def profile_step(self, stream=None) -> dict:
        """Run one step stage by stage (synchronising) and return ``{stage: ms}``."""
        L = _bind_batch(_lib.lib())
        ms = (C.c_double * 16)()
        _lib.check(L.fct_batch_profile(self._h, self.phase % 3, ms, 16, self._stream(stream)))
        self.phase += 1
        out = {}
        for i in range(16):
            name = L.fct_stage_name(i).decode()
            if name:
                out[name] = float(ms[i])
        return out

    # ------------------------------------------------------------------ state
    def state(self, i: int):
        """``(T, T_old)`` of member ``i`` as ``[ntr, N, nl]`` views (device, strided:
        the resident buffers keep the tracers innermost)."""
        b = self.members[i].buf
        p = self.phase
        return b[(p + 1) % 3].permute(2, 0, 1), b[p % 3].permute(2, 0, 1)

    def state_interleaved(self, i: int):
        """``(T, T_old)`` of member ``i`` in the resident ``[N, nl, ntr]`` layout."""
        b = self.members[i].buf
        p = self.phase
        return b[(p + 1) % 3], b[p % 3]

    def set_state(self, i: int, T, T_old, non_blocking: bool = False,
                  interleaved: bool = False) -> None:
        """Copy ``T``/``T_old`` (``[ntr, N, nl]``, or ``[N, nl, ntr]`` when
        ``interleaved``) into member ``i``'s current buffers."""
        Tc, To = self.state_interleaved(i)
        if not interleaved:
            T, T_old = T.permute(1, 2, 0), T_old.permute(1, 2, 0)
        Tc.copy_(T, non_blocking=non_blocking)
        To.copy_(T_old, non_blocking=non_blocking)

    def close(self) -> None:
        if self._h is not None and self._h.value:
            _bind_batch(_lib.lib()).fct_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
