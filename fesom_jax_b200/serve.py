"""Continuous-batching FCT serving on one GPU.

Requests ask to advance one ensemble member, started from a seeded state on a given mesh,
by K FCT steps (optionally followed by an adjoint). The engine keeps every admitted
member's state resident in HBM and runs *iterations*: each iteration is one batched FCT
step (``fct_serve_step``: one launch per stage for all admitted members, any meshes)
over every request still in flight, followed by extra rounds for the requests whose
meshes are much cheaper per step than the largest one in flight (up to ``max_rounds``
steps per iteration), so small requests are not held to the pace of the largest. Requests that arrive while others are on the GPU are
admitted as soon as the HBM budget allows (FIFO), so their steps join the next iteration;
a request leaves the batch after its K-th step and its memory is released once the GPU
has finished with it. Adjoint requests then run the vector-Jacobian product of their last
step (``fct_adjoint``, cotangent of a sea-surface loss) on a second stream, overlapping
the following iterations.

Completion times come from CUDA events (device clock), arrivals from the host clock,
both on one time axis anchored at a start event.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import time
from collections import deque

import numpy as np

from . import _lib
from .ensemble import FctInstance
from .mesh import Mesh
from .tracer_adv import _torch, get_plan


def _bind(L):
    if getattr(L, "_serve_bound", False):
        return L
    L.fct_serve_create.argtypes = [C.c_int, C.c_int, C.c_int64, C.POINTER(C.c_void_p)]
    L.fct_serve_destroy.argtypes = [C.c_void_p]
    L.fct_serve_step.argtypes = [C.c_void_p, C.POINTER(FctInstance), C.POINTER(C.c_int32),
                                 C.c_int, C.c_void_p]
    L.fct_serve_health.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
    for n in ("fct_serve_create", "fct_serve_destroy", "fct_serve_step", "fct_serve_health"):
        getattr(L, n).restype = C.c_int
    L._serve_bound = True
    return L


@dataclasses.dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the run
    mesh: str
    K: int
    adjoint: bool
    seed: int
    # runtime
    steps: int = 0
    admitted: float | None = None
    done: float | None = None
    state: object = None
    nbytes: int = 0
    done_event: object = None
    result: object = None
    grad: object = None
    health: object = None   # device counter of non-finite T_new values of this request
    inst: object = None     # its FctInstance while admitted
    nonfinite: int = 0      # its value after the run


def poisson_requests(rate: float, duration: float, mix=(("pi", 0.6), ("core2", 0.3),
                                                      ("large", 0.1)),
                     kmax: int = 50, p_adjoint: float = 0.2, seed: int = 0,
                     max_requests: int | None = None) -> list[Request]:
    """Seeded Poisson arrivals (mean ``rate`` per second) over ``duration`` seconds; mesh
    drawn from ``mix``, K ~ U{1..kmax}, adjoint with probability ``p_adjoint``."""
    rng = np.random.default_rng(seed)
    names = [m for m, _ in mix]
    w = np.array([p for _, p in mix], float)
    w /= w.sum()
    out, t, rid = [], 0.0, 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration or (max_requests is not None and rid >= max_requests):
            break
        out.append(Request(rid=rid, arrival=t, mesh=str(rng.choice(names, p=w)),
                           K=int(rng.integers(1, kmax + 1)),
                           adjoint=bool(rng.random() < p_adjoint), seed=int(rng.integers(1 << 30))))
        rid += 1
    return out


@dataclasses.dataclass
class MeshEntry:
    mesh: Mesh
    dt: float
    plan: object
    thick: object
    vel: list           # pool of (uv, w_e) device tensors shared by members
    nmask: object
    frac: object
    av0: object


class ServingEngine:
    """See the module docstring. ``budget_bytes`` bounds the member states, the shared
    velocity pools and the workspace arena together."""

    def __init__(self, meshes: dict, dts: dict, budget_bytes: float = 150e9, device: int = 0,
                 ntr: int = 2, workspace_bytes: float | None = None, velocity_pool: int = 2,
                 max_instances: int = 2048, adjoint_meshes=None, sigma: dict | None = None,
                 max_rounds: int = 16):
        from . import workloads as W
        torch = self.torch = _torch()
        self.device = device
        self.dev = torch.device("cuda", device)
        self.ntr = ntr
        self.L = _bind(_lib.lib())
        self.meshes: dict[str, MeshEntry] = {}
        used = 0
        for name, m in meshes.items():
            plan = get_plan(m, device)
            thick = W.rest_thickness_gpu(m, self.dev)
            vel = []
            for j in range(velocity_pool):
                inp = W.member_inputs_gpu(m, seed=7000 + j, ntr=1, device=self.dev, thickness=thick,
                                          sigma=(sigma or {}).get(name, 0.1))
                vel.append((inp["uv"], inp["w_e"]))
                used += inp["uv"].numel() * 8 + inp["w_e"].numel() * 8
            used += 3 * m.nod2D * m.nl * 8
            from .inputs import layer_depth_fraction
            self.meshes[name] = MeshEntry(
                m, float(dts[name]), plan, thick, vel,
                torch.from_numpy(m.node_layer_mask).to(self.dev),
                torch.from_numpy(layer_depth_fraction(m)).to(self.dev)[None, :],
                torch.from_numpy(m.areasvol[:, 0].copy()).to(self.dev))
        self.adjoint_meshes = set(adjoint_meshes if adjoint_meshes is not None else meshes)
        if workspace_bytes is None:
            from ._lib import lib  # noqa: F401
            workspace_bytes = 0.3 * budget_bytes
        self.ws_bytes = int(workspace_bytes)
        self.ws_doubles = self.ws_bytes // 8
        h = C.c_void_p()
        _lib.check(self.L.fct_serve_create(device, max_instances, self.ws_bytes, C.byref(h)))
        self._h = h
        self.max_instances = max_instances
        self.max_rounds = max(1, int(max_rounds))
        self.budget = int(budget_bytes)
        self.static_bytes = used + self.ws_bytes
        self.adj_stream = torch.cuda.Stream(self.dev)
        for name in self.adjoint_meshes:
            from .adjoint import _bind as _bind_adj
            _lib.check(_bind_adj(self.L).fct_plan_reserve_adjoint(self.meshes[name].plan.handle,
                                                                 1))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self.torch.cuda.synchronize(self.dev)
            self.L.fct_serve_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -------------------------------------------------------------- members
    def ws_need(self, r: Request) -> int:
        """Doubles of the fused-stage workspace one instance takes in the arena."""
        m = self.meshes[r.mesh].mesh
        N, Ed, L = m.nod2D, m.edge2D, m.nl
        pad = lambda n: (n + 31) // 32 * 32  # noqa: E731  (fields on 256-byte boundaries)
        return pad(Ed * L) + 4 * pad(self.ntr * N * L) + pad(self.ntr * Ed * L)

    def state_bytes(self, r: Request) -> int:
        m = self.meshes[r.mesh].mesh
        b = 3 * m.nod2D * m.nl * self.ntr * 8
        if r.adjoint and r.mesh in self.adjoint_meshes:   # tracer-0 VJP buffers
            b += 6 * m.nod2D * m.nl * 8 + 2 * m.elem2D * m.nl * 8
        return b

    def init_state(self, r: Request):
        """Seeded member state [3, N, nl, ntr]: T (2-28 degC with depth + noise), S, then
        passive tracers; T_old = T (step-1 convention)."""
        torch = self.torch
        e = self.meshes[r.mesh]
        m = e.mesh
        g = torch.Generator(device=self.dev)
        g.manual_seed(r.seed)
        N, nl = m.nod2D, m.nl
        T = torch.empty((N, nl, self.ntr), dtype=torch.float64, device=self.dev)
        for t in range(self.ntr):
            z = torch.randn((N, nl), generator=g, device=self.dev, dtype=torch.float64)
            if t == 0:
                T[:, :, t] = (28.0 - 26.0 * e.frac + 0.5 * z) * e.nmask
            elif t == 1:
                T[:, :, t] = (34.0 + 2.0 * e.frac + 0.1 * z) * e.nmask
            else:
                T[:, :, t] = torch.rand((N, nl), generator=g, device=self.dev,
                                        dtype=torch.float64) * e.nmask
        buf = torch.empty((3, N, nl, self.ntr), dtype=torch.float64, device=self.dev)
        buf[0].copy_(T)
        buf[1].copy_(T)
        buf[2].copy_(T)
        return buf

    def _instance(self, r: Request) -> FctInstance:
        e = self.meshes[r.mesh]
        uv, w = e.vel[r.seed % len(e.vel)]
        q = FctInstance()
        q.plan = e.plan.handle.value
        q.uv, q.w_e, q.helem = uv.data_ptr(), w.data_ptr(), e.thick.helem.data_ptr()
        q.hnode, q.hnode_new = e.thick.hnode.data_ptr(), e.thick.hnode_new.data_ptr()
        for j in range(3):
            q.buf[j] = r.state[j].data_ptr()
        q.ntr, q.dt = self.ntr, e.dt
        q.nonfinite = r.health.data_ptr() if r.health is not None else None
        return q

    def _adjoint(self, r: Request, stream, after_event):
        """VJP of the request's last step for the loss sum_n areasvol[n,0] T_K[n,0]^2 / 2.
        The loss reads tracer 0 only and the tracers of a step are independent, so the VJP
        runs on tracer 0 (the other tracers' cotangents are zero)."""
        torch = self.torch
        from .adjoint import advect_one_fct_vjp
        e = self.meshes[r.mesh]
        uv, w = e.vel[r.seed % len(e.vel)]
        p = r.K   # phase after K steps
        with torch.cuda.stream(stream):
            stream.wait_event(after_event)
            TK = r.state[(p + 1) % 3][:, :, 0]
            Tm1 = r.state[p % 3][:, :, 0].contiguous()
            Tm2 = r.state[(p + 2) % 3][:, :, 0].contiguous()
            gTn = torch.zeros_like(Tm1)
            gTn[:, 0] = e.av0 * TK[:, 0]
            gT, _, guv, _ = advect_one_fct_vjp(e.mesh, uv, w, e.thick.helem, e.thick.hnode,
                                               e.thick.hnode_new, Tm1, Tm2, gTn, dt=e.dt)
            r.grad = (gT, guv)
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(stream)
        return ev

    def _rounds(self, active: list[Request]) -> list[int]:
        """Steps each active request takes in this iteration: the ratio of the largest
        active mesh's wet node layers to its own (the step cost scales with them), at
        least 1, at most ``max_rounds`` and the steps it has left."""
        wl = [self.meshes[r.mesh].mesh.n_wet_layers for r in active]
        top = max(wl)
        return [max(1, min(self.max_rounds, top // w, r.K - r.steps)) for r, w in zip(active, wl)]

    # ------------------------------------------------------------------ run
    def run(self, requests: list[Request], keep_results: bool = False, max_run_ahead: int = 2,
            time_limit: float | None = None) -> dict:
        """Serve ``requests`` in real time (arrivals on the host clock). Returns statistics;
        every request gets ``admitted``/``done`` times (``done`` None if cut by
        ``time_limit``)."""
        torch = self.torch
        stream = torch.cuda.current_stream(self.dev)
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque[Request] = deque()
        active: list[Request] = []
        finishing: list[Request] = []
        inflight: deque = deque()
        mem = self.static_bytes
        ws_active = 0
        iters, inst_total, multi = 0, 0, 0
        # one non-finite counter per request (read after the run: no host sync per step)
        counters = torch.zeros(max(len(requests), 1), dtype=torch.int64, device=self.dev)
        for i, r in enumerate(requests):
            r.health = counters[i:i + 1]
        torch.cuda.synchronize(self.dev)
        start = torch.cuda.Event(enable_timing=True)
        start.record(stream)
        start.synchronize()
        t0 = time.perf_counter()
        n_total = len(requests)
        n_done = 0
        while n_done < n_total:
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit:
                break
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            while waiting:
                r = waiting[0]
                nb, ws = self.state_bytes(r), self.ws_need(r)
                if mem + nb > self.budget or ws_active + ws > self.ws_doubles or \
                        len(active) >= self.max_instances:
                    break
                waiting.popleft()
                r.state = self.init_state(r)
                r.inst = self._instance(r)   # its buffers stay put until it leaves
                r.nbytes, r.admitted = nb, now
                mem += nb
                ws_active += ws
                active.append(r)
            # release finished requests whose GPU work is over
            keep = []
            for r in finishing:
                if r.done_event.query():
                    r.done = start.elapsed_time(r.done_event) / 1e3
                    if keep_results:
                        p = r.K
                        r.result = r.state[(p + 1) % 3].permute(2, 0, 1).cpu().numpy()
                    r.state, r.inst = None, None
                    mem -= r.nbytes
                    n_done += 1
                else:
                    keep.append(r)
            finishing = keep
            if active:
                # every active request advances one step; requests on meshes far cheaper
                # per step than the dearest active one advance up to ``max_rounds`` steps
                # (one fct_serve_step per round), so a pi-size request does not move at
                # the pace of a 1.3M-node one sharing the iteration
                rounds = self._rounds(active)
                multi += max(rounds) > 1
                for rd in range(max(rounds)):
                    sub = [r for r, n in zip(active, rounds) if n > rd]
                    insts = (FctInstance * len(sub))(*[r.inst for r in sub])
                    phases = (C.c_int32 * len(sub))(*[r.steps for r in sub])
                    _lib.check(self.L.fct_serve_step(self._h, insts, phases, len(sub),
                                                     C.c_void_p(int(stream.cuda_stream))))
                    for r in sub:
                        r.steps += 1
                    inst_total += len(sub)
                ev = torch.cuda.Event(enable_timing=True)
                ev.record(stream)
                iters += 1
                still = []
                for r in active:
                    if r.steps == r.K:
                        ws_active -= self.ws_need(r)
                        if r.adjoint and r.mesh in self.adjoint_meshes:
                            r.done_event = self._adjoint(r, self.adj_stream, ev)
                        else:
                            r.done_event = ev
                        finishing.append(r)
                    else:
                        still.append(r)
                active = still
                inflight.append(ev)
                while len(inflight) > max_run_ahead:
                    inflight.popleft().synchronize()
            elif finishing:
                time.sleep(0.0002)
            elif pending and not waiting:
                time.sleep(max(0.0, min(0.01, pending[0].arrival - (time.perf_counter() - t0))))
        torch.cuda.synchronize(self.dev)
        wall = time.perf_counter() - t0
        counts = counters.cpu().tolist()
        for i, r in enumerate(requests):
            r.nonfinite, r.health = int(counts[i]), None
        done = [r for r in requests if r.done is not None]
        lat = np.array([r.done - r.arrival for r in done]) * 1e3
        upd = sum(r.K * self.ntr * self.meshes[r.mesh].mesh.n_wet_layers for r in done)
        # per mesh class: latency, the wait for admission (arrival -> admitted) and the
        # latency per step of the request (what K steps of that mesh take in the mix)
        by_mesh = {}
        for name in sorted({r.mesh for r in done}):
            rs = [r for r in done if r.mesh == name]
            lm = np.array([r.done - r.arrival for r in rs]) * 1e3
            wait = np.array([r.admitted - r.arrival for r in rs]) * 1e3
            per_step = np.array([(r.done - r.admitted) / r.K for r in rs]) * 1e3
            by_mesh[name] = dict(completed=len(rs), p50_ms=float(np.percentile(lm, 50)),
                                 p99_ms=float(np.percentile(lm, 99)),
                                 wait_p99_ms=float(np.percentile(wait, 99)),
                                 ms_per_step_p50=float(np.percentile(per_step, 50)))
        return dict(requests=n_total, completed=len(done), wall_s=wall, iterations=iters,
                    mean_batch=inst_total / max(iters, 1), multi_round_iterations=multi,
                    p50_ms=float(np.percentile(lat, 50)) if len(lat) else None,
                    p99_ms=float(np.percentile(lat, 99)) if len(lat) else None,
                    throughput_req_s=len(done) / wall, updates_per_s=upd / wall,
                    nonfinite_requests=sum(1 for r in requests if r.nonfinite),
                    by_mesh=by_mesh)

    def run_serial(self, requests: list[Request], time_limit: float | None = None) -> dict:
        """Baseline: the same requests one at a time through the single-instance C ABI
        (fct_forward per step, plain launches, no batching); latency from a FIFO queue of
        the measured service times."""
        torch = self.torch
        service = []
        t_start = time.perf_counter()
        for r in sorted(requests, key=lambda x: x.arrival):
            if time_limit is not None and time.perf_counter() - t_start > time_limit:
                break
            e = self.meshes[r.mesh]
            uv, w = e.vel[r.seed % len(e.vel)]
            st = self.init_state(r)
            T = st[1].permute(2, 0, 1).contiguous()
            To = T.clone()
            Tm2 = To
            torch.cuda.synchronize(self.dev)
            t0 = time.perf_counter()
            for _ in range(r.K):   # one tracer per call, the reference's granularity
                Tn = torch.empty_like(T)
                for t in range(self.ntr):
                    e.plan.forward(uv, w, e.thick.helem, e.thick.hnode, e.thick.hnode_new,
                                   T[t], To[t], e.dt, out=Tn[t])
                Tm2, To, T = To, T, Tn
            if r.adjoint and r.mesh in self.adjoint_meshes:
                from .adjoint import advect_one_fct_vjp
                gTn = torch.zeros_like(T[0])
                gTn[:, 0] = e.av0 * T[0, :, 0]
                advect_one_fct_vjp(e.mesh, uv, w, e.thick.helem, e.thick.hnode,
                                   e.thick.hnode_new, To[0].contiguous(), Tm2[0].contiguous(),
                                   gTn, dt=e.dt)
            torch.cuda.synchronize(self.dev)
            service.append((r, time.perf_counter() - t0))
            del st, T, To
        clock, lat, upd, busy = 0.0, [], 0, 0.0
        for r, s in service:
            start = max(clock, r.arrival)
            clock = start + s
            busy += s
            lat.append((clock - r.arrival) * 1e3)
            upd += r.K * self.ntr * self.meshes[r.mesh].mesh.n_wet_layers
        lat = np.array(lat)
        return dict(requests=len(service), busy_s=busy,
                    p50_ms=float(np.percentile(lat, 50)) if len(lat) else None,
                    p99_ms=float(np.percentile(lat, 99)) if len(lat) else None,
                    throughput_req_s=len(service) / max(clock, 1e-9),
                    updates_per_s=upd / max(busy, 1e-9))
