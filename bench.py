#!/usr/bin/env python
"""FCT tracer-advection benchmark on B200 (one JSON line on rank 0).

Default workload ("batched"): a CORE2-size synthetic mesh (127,000 nodes, 48 levels,
bottom level 5-48), 32 ensemble members x 8 tracers (T, S, 6 passive) with
seed-perturbed velocities, 30 FCT steps (dt = 1800 s) captured as one CUDA graph. One
bench step is one such 30-step graph over all members; ``value`` is node-level updates/s
(one tracer value at one wet node layer advanced one FCT step) over all ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config batched|pi|large]
    python bench.py --impl reference ...   # the CPU arm (C restatement, all host threads)

Multi-GPU: one rank per GPU (torchrun); every rank advances its own 32 members (weak
scaling, no data-path collective); time = max over ranks of the CUDA-event time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FCT node-level updates/s FP64, batched vs plain on 1 B200; serve p50/p99 ms"
UNIT = "node-level updates/s"
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (read + write) per node-level update of the six kernels of the fused FCT step
# (volume fluxes, LO, edge fluxes and their node-gradient lanes, limiter, final), from one
# ncu capture of the small case of the batched workload (2 members x 8 tracers of the
# CORE2-size mesh: 12.53 GB per FCT step / 48.76 M updates). Scaled to a launch by the
# updates it does.
TRAFFIC_B_PER_UPDATE = 257.0
# Warp-instructions per node-level update of the same six kernels in the same capture
# (smsp__inst_executed.sum / updates). The kernels are latency- and issue-limited rather
# than HBM-bound, so the line also reports this issue-rate fraction beside the HBM one:
# achieved warp-instructions/s against 148 SMs x 4 schedulers x the sampled SM clock.
WARP_INST_PER_UPDATE = 46.0
B200_SMS, SCHEDULERS_PER_SM = 148, 4


def peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return dict(hbm_gbs=float(d["hbm_gbs"]), source="measured")
    return dict(hbm_gbs=FALLBACK_HBM_GBS, source="fallback")


def issue_roofline(updates_per_s: float, clk) -> dict:
    """Instruction-issue fraction of the batched step: warp-instructions per update (ncu
    capture constant) x updates/s against every scheduler issuing one per cycle at the
    median SM clock sampled in the timed region (max clock when unsampled)."""
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965.0
    peak = B200_SMS * SCHEDULERS_PER_SM * float(mhz) * 1e6 / 1e9
    achieved = WARP_INST_PER_UPDATE * updates_per_s / 1e9
    return dict(achieved=achieved, peak=peak, unit="G warp-instructions/s",
                frac=achieved / peak, warp_inst_per_update=WARP_INST_PER_UPDATE,
                sm_mhz=float(mhz))


# ------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling (200 ms) of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self) -> dict | None:
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append(dict(sm=float(parts[1]), smax=float(parts[2]), power=float(parts[3]),
                                 hw=parts[5], hwt=parts[6], swt=parts[7], pcap=parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        loaded = [r for r in rows if r["power"] > 250.0] or rows
        reasons = set()
        for r in rows:
            for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                              ("swt", "sw_thermal_slowdown"), ("pcap", "sw_power_cap")):
                if r[key].lower() == "active":
                    reasons.add(name)
        return dict(sm_mhz=float(np.median([r["sm"] for r in loaded])),
                    sm_max_mhz=float(max(r["smax"] for r in rows)), reasons=sorted(reasons),
                    samples=len(rows), power_w_max=float(max(r["power"] for r in rows)))


def gpu_index(local_rank: int) -> int:
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        if local_rank < len(ids) and ids[local_rank].isdigit():
            return int(ids[local_rank])
    return local_rank


# -------------------------------------------------------------------- distributed
class Dist:
    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = False

    def init(self, backend: str):
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
            self.pg = True

    def barrier(self):
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, x: float, device) -> float:
        if not self.pg:
            return x
        import torch
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def weak_value(self, updates_per_rank: float, t_local: float, device) -> tuple:
        """Whole-job rate of a weak-scaling run: every rank did ``updates_per_rank`` in its
        own device time ``t_local``; the job time is the max over ranks.
        Returns ``(updates/s over all ranks, job time)``."""
        t = self.max(t_local, device)
        return updates_per_rank * self.world / t, t

    def close(self):
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()


# -------------------------------------------------------------------- CPU oracle
def cpu_oracle_rate(mesh, fields_host, ntr: int, dt: float, min_seconds: float = 10.0,
                    max_reps: int = 3) -> dict:
    """Time the C restatement (all host threads) on one member's ``ntr`` tracers, one
    FCT step, repeated until ``min_seconds`` or ``max_reps``; returns updates/s."""
    from oracle import fct_c
    keep = []
    from fesom_jax_b200 import _lib as fl
    desc = fl.mesh_desc(mesh, keep)
    f = fields_host
    reps, t_total = 0, 0.0
    while reps < max_reps and (t_total < min_seconds or reps == 0):
        t0 = time.perf_counter()
        for t in range(ntr):
            fct_c.advect_one_fct(mesh, f["uv"], f["w_e"], f["helem"], f["hnode"],
                                 f["hnode_new"], f["T"][t], f["T_old"][t], dt=dt, desc=desc)
        t_total += time.perf_counter() - t0
        reps += 1
    upd = reps * ntr * mesh.n_wet_layers
    return dict(value=upd / t_total, unit=UNIT, cores=fct_c.max_threads(), kind="port",
                sample=f"C loop restatement (OpenMP), {reps} x (1 member x {ntr} tracers x 1 "
                       f"FCT step) on {mesh.name}, {t_total:.1f} s")


# ------------------------------------------------------------------ correctness gates
# per-step parity of the CUDA path against the oracle (max-norm over wet lanes, relative)
GATE_RTOL = 1e-12
# budget closure residual relative to the tracer content
GATE_CLOSURE_RTOL = 1e-13


def run_gates(ens, mesh, cfg, plan, member: int = 0) -> dict:
    """The per-run correctness gates on one member, after the timed region: one more
    batched FCT step of every member, then on ``member``:
    (i) every tracer against the C oracle (fct_ref.c, all host threads) at <= 1e-12
        (max-norm over wet lanes, relative to max|T_oracle|);
    (ii) budget closure of tracer 0 (content change = dt x surface fluxes, from the numpy
        oracle's intermediates) to 1e-13 of the content;
    (iii) no value of tracer 0 outside the limiter's window (fesom_jax/tracer_adv.py:389-418),
        16 ulp slack (oracle.gates.GPU_WINDOW_ULPS);
    (iv) bitwise determinism: the single-instance fused call twice on the same inputs, and
        the batched result of tracer 0 against it.
    With the vertical diffusion epilogue (``Kv``) the reference of (i) is the oracle's FCT
    step followed by the oracle's diffusion (oracle/vdiff_np.py), the single-instance call
    of (iv) is fct_forward followed by fct_vert_diff, and (iii) does not apply (the
    diffusion mixes each column after the limiter's window was enforced).
    The oracle serves as the checker only; nothing here is timed."""
    import torch

    from oracle import fct_c, fct_np, vdiff_np
    from oracle.gates import closure_residual, window_violations
    mb = ens.members[member]
    Kv = mb.Kv.cpu().numpy() if mb.Kv is not None else None
    T, To = (x.cpu().numpy() for x in ens.state(member))
    host = {k: getattr(mb, k).cpu().numpy() for k in ("uv", "w_e", "helem", "hnode",
                                                      "hnode_new")}
    ens.step()
    torch.cuda.synchronize()
    Tn = ens.state(member)[0].cpu().numpy()
    lm = mesh.node_layer_mask
    keep = []
    from fesom_jax_b200 import _lib as fl
    desc = fl.mesh_desc(mesh, keep)
    worst, dry_equal = 0.0, True
    for t in range(mb.ntr):
        ref, _ = fct_c.advect_one_fct(mesh, host["uv"], host["w_e"], host["helem"],
                                      host["hnode"], host["hnode_new"], T[t], To[t],
                                      dt=mb.dt, desc=desc)
        if Kv is not None:
            ref = vdiff_np.impl_vert_diff_one(mesh, ref, Kv, host["hnode_new"], dt=mb.dt)
        worst = max(worst, float(np.max(np.abs(Tn[t][lm] - ref[lm])) /
                                 np.max(np.abs(ref[lm]))))
        dry_equal = dry_equal and bool(np.array_equal(Tn[t][~lm], T[t][~lm]))
    inter = {}
    ref0, _ = fct_np.advect_one_fct(mesh, host["uv"], host["w_e"], host["helem"],
                                    host["hnode"], host["hnode_new"], T[0], To[0], dt=mb.dt,
                                    intermediates=inter)
    closure = closure_residual(mesh, T[0], host["hnode"], host["hnode_new"], Tn[0], inter,
                               mb.dt)
    from oracle.gates import GPU_WINDOW_ULPS
    viol = (int(len(window_violations(mesh, T[0], host["hnode_new"], Tn[0], inter,
                                      GPU_WINDOW_ULPS))) if Kv is None else None)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    args = [d(host[k]) for k in ("uv", "w_e", "helem", "hnode", "hnode_new")]
    a = plan.forward(*args, d(T[0]), d(To[0]), mb.dt)
    b = plan.forward(*args, d(T[0]), d(To[0]), mb.dt)
    det = bool(torch.equal(a, b))
    if Kv is not None:
        from fesom_jax_b200.tracer_diff import impl_vert_diff_one
        a = impl_vert_diff_one(mesh, a, mb.Kv, args[4], dt=mb.dt)
    batched_eq = bool(np.array_equal(a.cpu().numpy(), Tn[0]))
    out = dict(member=member, tracers=mb.ntr, max_rel_err=worst, rtol=GATE_RTOL,
               dry_levels_equal=dry_equal, closure_rel=closure, closure_rtol=GATE_CLOSURE_RTOL,
               window_violations=viol, deterministic=det, batched_equals_plain=batched_eq)
    out["passed"] = bool(worst <= GATE_RTOL and dry_equal and closure <= GATE_CLOSURE_RTOL
                         and (viol is None or viol == 0) and det)
    return out


# ------------------------------------------------------------------------ our arm
def member_seed(rank: int, i: int) -> int:
    """Seed of member ``i`` on ``rank``: replicas advance different members."""
    return 1000 * rank + i


def run_ours(args, D: Dist) -> dict | None:
    import torch

    from fesom_jax_b200 import workloads as W
    from fesom_jax_b200.ensemble import Ensemble

    torch.cuda.set_device(D.local_rank)
    dev = torch.device("cuda", D.local_rank)
    cfg = dict(W.WORKLOADS[args.config])
    if args.members:
        cfg["members"] = args.members
    if args.fct_steps:
        cfg["fct_steps"] = args.fct_steps
    if args.ntr:
        cfg["ntr"] = args.ntr
    mesh = W.make_workload_mesh(args.config, seed=0, node_order=args.node_order)
    thick = W.rest_thickness_gpu(mesh, dev)
    ens = Ensemble(device=D.local_rank, workspace_budget=int(args.workspace_gb * (1 << 30)))
    member_inputs = []
    Kv = None
    if args.vdiff:   # implicit vertical diffusion epilogue (tracer_diff.py:68-123)
        g = torch.Generator(device=dev)
        g.manual_seed(4242)
        from fesom_jax_b200.inputs import layer_depth_fraction
        frac = torch.from_numpy(layer_depth_fraction(mesh)).to(dev)[None, :]
        im = torch.from_numpy(mesh.node_iface_mask).to(dev)
        u = 0.5 + torch.rand(im.shape, generator=g, device=dev, dtype=torch.float64)
        Kv = torch.where(im, 1e-5 + 1e-2 * torch.exp(-5.0 * frac) * u, 0.0).contiguous()
    for i in range(cfg["members"]):
        inp = W.member_inputs_gpu(mesh, seed=member_seed(D.rank, i), ntr=cfg["ntr"], device=dev,
                                  thickness=thick, sigma=cfg["sigma"],
                                  n_vortices=cfg["n_vortices"], kind=cfg["velocity"])
        ens.add_member(mesh, inp["uv"], inp["w_e"], inp["helem"], inp["hnode"],
                       inp["hnode_new"], inp["T"], inp["T_old"], cfg["dt"], Kv=Kv,
                       derive_w=args.derive_w)
        member_inputs.append(inp if i == 0 else None)
        del inp
    torch.cuda.empty_cache()   # hand the input temporaries back before the arena is allocated
    ens.build()
    info = ens.info()
    S = cfg["fct_steps"]
    stream = torch.cuda.current_stream(dev)
    fixed = bool(args.chunk or args.levels or args.stage_mapping)
    tune = ens.autotune(steps=2) if not fixed else None
    if args.stage_mapping:
        for st, m in enumerate(parse_stage_mapping(args.stage_mapping)):
            ens.set_stage_mapping(st, *m)
    elif fixed:
        ens.set_mapping(args.chunk or ens.chunk, args.levels or ens.levels)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        ens.run(S)
    torch.cuda.synchronize()
    D.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(gpu_index(D.local_rank))
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        ens.run(S)
    e1.record(stream)
    torch.cuda.synchronize()
    D.barrier()
    clk = clocks.stop()
    t_local = e0.elapsed_time(e1) / 1e3
    upd_rank = info["updates_per_step"] * S * args.steps
    value, t = D.weak_value(upd_rank, t_local, dev)

    # health: non-finite T_new values written by any member since the build (device
    # counters of the final stage), and the finiteness of every member's state
    nonfinite = ens.health()
    finite = (sum(nonfinite) == 0 and
              all(bool(torch.isfinite(ens.state(i)[0]).all().item())
                  for i in range(len(ens.members))))
    # per-stage breakdown (events on the launching stream, one step, synchronised)
    prof = {}
    for _ in range(3):
        for k, v in ens.profile_step().items():
            prof[k] = prof.get(k, 0.0) + v / 3
    fct_step_ms = t_local / (S * args.steps) * 1e3
    alg = W.algorithmic_bytes(mesh, cfg["ntr"], cfg["members"])
    pk = peaks()
    achieved = alg / (fct_step_ms / 1e3) / 1e9
    info = ens.info()   # after tuning: launches per step depend on tracers per thread
    n_kernels = info["launches_per_step"]
    gates = None
    if D.rank == 0 and not args.no_gates:
        from fesom_jax_b200.tracer_adv import get_plan
        gates = run_gates(ens, mesh, cfg, get_plan(mesh, D.local_rank))
    out = dict(value=value, t=t, info=info, clocks=clk, prof=prof, fct_step_ms=fct_step_ms,
               finite=finite, nonfinite=int(sum(nonfinite)), gates=gates, mesh=mesh, cfg=cfg,
               alg_bytes=alg,
               roofline=dict(bound="hbm", kernel="fused FCT step (k_vflux, k_seg_lo, k_seg_edge, "
                                                 "k_edge_fix, k_seg_limit, k_seg_final)",
                             achieved=achieved, peak=pk["hbm_gbs"], unit="GB/s",
                             frac=achieved / pk["hbm_gbs"], peak_source=pk["source"],
                             traffic=TRAFFIC_B_PER_UPDATE * info["updates_per_step"],
                             traffic_note="ncu DRAM bytes of the step's 6 kernels, small-case "
                                          "capture scaled by updates",
                             alg_bytes_per_step=alg,
                             issue=issue_roofline(value / D.world, clk)),
               gpu_launches=n_kernels * S * args.steps,
               tuning=dict(stage_mapping={st: f"{c}x{lv}" for st, (c, lv) in
                                          zip(ens.STAGES, ens.stage_map)},
                           autotune=tune))

    # plain one-instance-per-launch comparison (the reference's call granularity:
    # one tracer per advect_one_fct call), member 0, one FCT step per call
    if D.rank == 0 and member_inputs[0] is not None:
        from fesom_jax_b200.tracer_adv import get_plan
        inp = member_inputs[0]
        plan = get_plan(mesh, D.local_rank)
        plan.autotune([inp[k] for k in ("uv", "w_e", "helem", "hnode", "hnode_new")] +
                      [inp["T"][0], inp["T_old"][0]], cfg["dt"], reps=3)
        outb = torch.empty_like(inp["T"][0])
        for _ in range(2):
            plan.forward(inp["uv"], inp["w_e"], inp["helem"], inp["hnode"], inp["hnode_new"],
                         inp["T"][0], inp["T_old"][0], cfg["dt"], out=outb)
        torch.cuda.synchronize()
        e0.record(stream)
        reps = 3
        for _ in range(reps):
            for tr in range(cfg["ntr"]):
                plan.forward(inp["uv"], inp["w_e"], inp["helem"], inp["hnode"],
                             inp["hnode_new"], inp["T"][tr], inp["T_old"][tr], cfg["dt"],
                             out=outb)
        e1.record(stream)
        torch.cuda.synchronize()
        tp = e0.elapsed_time(e1) / 1e3
        out["plain"] = dict(value=reps * cfg["ntr"] * mesh.n_wet_layers / tp, unit=UNIT,
                            how="fct_forward, 1 tracer per call, 1 FCT step per call")
    tuned = list(ens.stage_map)
    ens.close()   # the end-to-end run below builds its own ensemble
    del ens
    torch.cuda.empty_cache()
    host = None
    if D.rank == 0 and member_inputs[0] is not None and not args.no_cpu:
        host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v)
                for k, v in member_inputs[0].items()}
    member_inputs.clear()
    torch.cuda.empty_cache()
    if not args.no_e2e:
        # every rank streams its own members; the whole-job rate is all ranks' updates over
        # the slowest rank's time, as for the headline value
        e = e2e_host(args, mesh, cfg, dev, per_thread=tuned, rank=D.rank)
        value_e, t_e = D.weak_value(e["updates"], e["t"], dev)
        if D.rank == 0:
            e.update(value=value_e, t_max_s=t_e, ranks=D.world,
                     h2d_bytes_per_step=e["h2d_bytes_per_step"] * D.world,
                     d2h_bytes_per_step=e["d2h_bytes_per_step"] * D.world)
            out["e2e"] = e
    if host is not None:
        out["cpu_baseline"] = cpu_oracle_rate(mesh, host, cfg["ntr"], cfg["dt"])
    return out


def e2e_host(args, mesh, cfg, dev, per_thread=None, rank: int = 0) -> dict:
    """The same metric through the public ensemble API with HOST buffers: every bench step
    copies each member's inputs (T, T_old, uv, w_e) from pinned host memory, runs the
    FCT steps and copies the final T back; copies are inside the timed region. Members are
    pipelined over three CUDA streams (one single-member ensemble each), so one member's
    copies overlap another's FCT steps, as a user streaming members through the API would."""
    import torch

    from fesom_jax_b200 import workloads as W
    from fesom_jax_b200.ensemble import Ensemble
    nm = min(args.e2e_members, cfg["members"])
    thick = W.rest_thickness_gpu(mesh, dev)
    streams = [torch.cuda.Stream(dev) for _ in range(3)]
    ens, host = [], []
    for i in range(nm):
        inp = W.member_inputs_gpu(mesh, seed=500000 + member_seed(rank, i), ntr=cfg["ntr"],
                                  device=dev,
                                  thickness=thick, sigma=cfg["sigma"], n_vortices=cfg["n_vortices"],
                                  kind=cfg["velocity"])
        e = Ensemble(device=dev.index, workspace_budget=int(args.workspace_gb * (1 << 30)))
        e.add_member(mesh, inp["uv"], inp["w_e"], inp["helem"], inp["hnode"], inp["hnode_new"],
                     inp["T"], inp["T_old"], cfg["dt"])
        h = {k: inp[k].cpu().pin_memory() for k in ("uv", "w_e")}
        # host state in the resident interleaved layout [N, nl, ntr]
        for k in ("T", "T_old"):
            h[k] = inp[k].permute(1, 2, 0).contiguous().cpu().pin_memory()
        h["out"] = torch.empty_like(h["T"]).pin_memory()
        ens.append(e)
        host.append(h)
        del inp
    torch.cuda.empty_cache()
    for e in ens:
        e.build()
        if per_thread:   # the main run's autotuned thread mapping, stage by stage
            for st, m in enumerate(per_thread):
                e.set_stage_mapping(st, *m)
    S = cfg["fct_steps"]
    main = torch.cuda.current_stream(dev)
    h2d = sum(h[k].numel() * 8 for h in host for k in ("T", "T_old", "uv", "w_e"))
    d2h = sum(h["out"].numel() * 8 for h in host)

    def one(first=True, last=True):
        """One bench step: every member in, S FCT steps, out. The streams carry on from
        one step to the next (each member's next copy in is ordered after its copy out on
        its stream), so a run of steps is joined to the main stream only at its end."""
        if first:
            start = torch.cuda.Event()
            start.record(main)
            for st in streams:
                st.wait_event(start)
        for i, (e, h) in enumerate(zip(ens, host)):
            st = streams[i % len(streams)]
            with torch.cuda.stream(st):
                mb = e.members[0]
                e.set_state(0, h["T"], h["T_old"], non_blocking=True, interleaved=True)
                mb.uv.copy_(h["uv"], non_blocking=True)
                mb.w_e.copy_(h["w_e"], non_blocking=True)
                e.run(S, stream=st.cuda_stream)
                h["out"].copy_(e.state_interleaved(0)[0], non_blocking=True)
        if last:
            for st in streams:
                done = torch.cuda.Event()
                done.record(st)
                main.wait_event(done)

    for _ in range(max(1, min(args.warmup, 2))):
        one()
    torch.cuda.synchronize()
    first_out = host[0]["out"].clone()   # every step starts from the same inputs
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(1, min(args.steps, 3))
    w0 = time.perf_counter()
    e0.record(main)
    for r in range(reps):
        one(first=r == 0, last=r == reps - 1)
    e1.record(main)
    torch.cuda.synchronize()
    wall = time.perf_counter() - w0
    t = max(e0.elapsed_time(e1) / 1e3, 1e-9)
    upd = sum(e.info()["updates_per_step"] for e in ens) * S * reps
    # the first member's host result of the timed steps is the warm-up's bit for bit, and
    # every member's is finite
    same = bool(torch.equal(first_out, host[0]["out"]))
    finite = all(bool(torch.isfinite(h["out"]).all()) for h in host)
    for e in ens:
        e.close()
    return dict(value=upd / t, unit=UNIT, h2d_bytes_per_step=h2d, d2h_bytes_per_step=d2h,
                members=nm, steps=reps, wall_s=wall, streams=len(streams), updates=upd, t=t,
                outputs_repeat_bitwise=same, outputs_finite=finite,
                how="Ensemble API, pinned host buffers in/out every step, members pipelined "
                    "over 3 streams")


# ---------------------------------------------------------------- adjoint (config 3)
def run_adjoint(args, D: Dist) -> dict:
    """Gradient of loss = sum_n areasvol[n,0] (T_K[n,0] - target_n)^2 after K = 10 FCT
    steps on the CORE2-size mesh, w.r.t. the initial T and uv, with w_e = compute_w(uv)
    inside the loss (chain_loss_and_grad with a forward tape; the per-step recomputation
    variant is timed beside it). Reports its cost against the forward alone (compute_w +
    K steps), a dot-product test of the T gradients and a Taylor test of the uv gradient.

    The velocities here are white noise (sigma 0.002 m/s, vertical CFL < 1), so w is far
    from the upwind kink at 0 and the gradient is taken at a differentiable point."""
    import torch

    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200 import workloads as W
    from fesom_jax_b200.adjoint import Tape, chain_loss_and_grad
    from fesom_jax_b200.ale import compute_w
    from fesom_jax_b200.tracer_adv import get_plan
    torch.cuda.set_device(D.local_rank)
    dev = torch.device("cuda", D.local_rank)
    mesh = W.make_workload_mesh("batched", seed=0)
    K, dt = 10, 1800.0
    f = I.make_fields(mesh, seed=3 + D.rank, ab2=True, kind="white", sigma=0.002)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    T0, To0, uv = d(f.tracers[0]), d(f.tracers_old[0]), d(f.uv)
    helem, hn, hnn = d(f.helem), d(f.hnode), d(f.hnode_new)
    target = torch.from_numpy(np.random.default_rng(7).normal(15.0, 3.0, mesh.nod2D))
    plan = get_plan(mesh, D.local_rank)
    stream = torch.cuda.current_stream(dev)

    def forward():
        w = compute_w(mesh, uv, helem)
        T, To = T0, To0
        for _ in range(K):
            T, To = plan.forward(uv, w, helem, hn, hnn, T, To, dt), T
        return T

    main_mode = args.checkpoint   # the headline checkpointing; the other is timed beside it
    other = "recompute" if main_mode == "tape" else None

    torch.cuda.empty_cache()   # hand back what earlier measurements left cached
    tape = Tape(mesh, K, 1, D.local_rank) if main_mode == "tape" else None

    def grad(checkpoint=main_mode):
        return chain_loss_and_grad(mesh, T0, uv, helem, hn, hnn, target, K, dt=dt, T_old0=To0,
                                   checkpoint=checkpoint,
                                   tape=tape if checkpoint == "tape" else None)

    def timed(fn, reps):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    D.barrier()
    t_fwd = timed(forward, args.steps)
    t_grad = timed(grad, args.steps)
    t_grad_rc = timed(lambda: grad(other), args.steps) if other else None
    t = D.max(t_grad, dev)
    loss, gT0, guv = grad()
    same_bits = None
    if other:
        _, gT0_rc, guv_rc = grad(other)
        same_bits = bool(torch.equal(gT0, gT0_rc) and torch.equal(guv, guv_rc))
    # gradient checks that hold at this size (central differences are lost in the
    # round-off of a ~1e15 loss): (1) a dot-product test along x = (T0, T_old0): the K-step
    # map is positively homogeneous of degree 1 in its tracer inputs, so its tangent along
    # x is T_K itself and <gT0, T0> + <gT_old0, T_old0> = <dL/dT_K, T_K>; (2) a Taylor test
    # in uv: r(h) = |L(uv + h v) - L - h <guv, v>| falls as h^2 for the right gradient
    checks = None
    if not args.no_fd:
        _, gT, gU, gTo = chain_loss_and_grad(mesh, T0, uv, helem, hn, hnn, target, K, dt=dt,
                                             T_old0=To0, checkpoint=main_mode,
                                             return_gT_old=True,
                                             tape=tape if main_mode == "tape" else None)
        TK = forward()[:, 0]
        av0 = torch.from_numpy(mesh.areasvol[:, 0].copy()).to(dev)
        terms = 2.0 * av0 * (TK - target.to(dev)) * TK
        lhs = float((gT * T0).sum() + (gTo * To0).sum())
        rhs = float(terms.sum())
        em = torch.from_numpy(mesh.elem_layer_mask).to(dev)[:, :, None]
        v = d(np.random.default_rng(11).normal(0.0, 0.002, uv.shape)) * em
        gv = float((gU * v).sum())
        rem = {}
        for h in (1e-2, 1e-3):
            Lh = chain_loss_and_grad(mesh, T0, uv + h * v, helem, hn, hnn, target, K, dt=dt,
                                     T_old0=To0, checkpoint=main_mode,
                                     tape=tape if main_mode == "tape" else None)[0]
            rem[h] = abs(Lh - loss - h * gv)
        checks = dict(dot_T_rel_err=abs(lhs - rhs) / float(terms.abs().sum()),
                      taylor_uv=dict(h=[1e-2, 1e-3], remainder=[rem[1e-2], rem[1e-3]],
                                     first_order=[abs(1e-2 * gv), abs(1e-3 * gv)],
                                     order=float(np.log10(rem[1e-2] / max(rem[1e-3], 1e-300)))))
    if tape is not None:
        tape.close()
    upd = K * mesh.n_wet_layers * D.world
    return dict(value=upd / t, t=t * args.steps, mesh=mesh, t_fwd=t_fwd, t_grad=t_grad,
                cfg=dict(members=1, ntr=1, fct_steps=K, dt=dt),
                adjoint=dict(forward_ms=t_fwd * 1e3, loss_and_grad_ms=t_grad * 1e3,
                             ratio=t_grad / t_fwd, K=K, loss=loss, checkpoint=main_mode,
                             tape_gb=Tape.nbytes(mesh, K, 1, D.local_rank) / 1e9,
                             recompute_loss_and_grad_ms=(t_grad_rc * 1e3 if other else None),
                             recompute_ratio=(t_grad_rc / t_fwd if other else None),
                             tape_equals_recompute=same_bits,
                             gradient_checks=checks, max_cfl_z=float(I.max_cfl_z(
                                 mesh, f.w_e, f.hnode, dt)),
                             how="chain_loss_and_grad (forward x K with the chosen "
                                 "checkpointing, fct_adjoint_ex x K, fct_compute_w_adjoint) vs "
                                 "compute_w + fct_forward x K"))


# ---------------------------------------------------------------- serving (config 5)
def run_serve(args, D: Dist) -> dict:
    """Continuous-batching serving (ServingEngine): Poisson arrivals at 200 req/s mixing
    the pi, CORE2-size and 1.3M-node meshes (0.6/0.3/0.1), each request K ~ U{1..50} FCT
    steps of a resident member (T, S), 20 % with the adjoint of the last step; admission
    by a 150 GB HBM budget. The offered load is far above one GPU's capacity, so the
    stream is bounded (``--serve-seconds`` of arrivals) and the run also reports a
    sustainable-rate stream and the serial plain-launch baseline on the same requests."""
    import torch

    from fesom_jax_b200 import workloads as W
    from fesom_jax_b200.mesh import pi_mesh
    from fesom_jax_b200.serve import ServingEngine, poisson_requests
    torch.cuda.set_device(D.local_rank)
    meshes = {"pi": pi_mesh(), "core2": W.make_workload_mesh("batched", seed=0),
              "large": W.make_workload_mesh("large", seed=0)}
    dts = {"pi": 3600.0, "core2": 1800.0, "large": 600.0}
    eng = ServingEngine(meshes, dts, budget_bytes=150e9, device=D.local_rank, ntr=2,
                        workspace_bytes=45e9, sigma={"large": 0.2},
                        max_rounds=args.serve_rounds)
    out = {}
    reqs = poisson_requests(200.0, args.serve_seconds, seed=1 + D.rank)
    clocks = ClockSampler(gpu_index(D.local_rank))
    clocks.start()
    sat = eng.run(reqs, time_limit=args.serve_limit)
    out["clocks"] = clocks.stop()
    out["saturated"] = dict(rate_req_s=200.0, arrivals_s=args.serve_seconds, **sat)
    cap = sat["throughput_req_s"]
    low = poisson_requests(max(0.5 * cap, 0.2), args.serve_seconds * 4, seed=100 + D.rank)
    out["sustainable"] = dict(rate_req_s=max(0.5 * cap, 0.2),
                              **eng.run(low, time_limit=args.serve_limit))
    out["serial"] = eng.run_serial(reqs, time_limit=args.serve_limit / 2)
    eng.close()
    out["value"] = sat["updates_per_s"] * D.world
    out["t"] = sat["wall_s"]
    return out


# ------------------------------------------------------- side measurements (default run)
def run_side(args, D: Dist) -> dict:
    """Short measurements of the other configurations beside the headline, so a default
    run covers them: config 1 (pi, plain fct_forward, T and S, one step, u, v ~ N(0, 0.1),
    T_old = T) with its parity against the C oracle and the oracle's own rate, and config 3
    (the 10-step adjoint loss gradient on the CORE2-size mesh, its cost against the
    forward; no gradient checks here). Each takes a few seconds."""
    import copy

    import torch

    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200.mesh import pi_mesh
    from fesom_jax_b200.tracer_adv import get_plan
    from oracle import fct_c
    out = {}
    dev = torch.device("cuda", D.local_rank)
    m = pi_mesh()
    f = I.make_fields(m, seed=0, kind="white", sigma=0.1)
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)  # noqa: E731
    a = [d(x) for x in (f.uv, f.w_e, f.helem, f.hnode, f.hnode_new, f.tracers, f.tracers_old)]
    plan = get_plan(m, D.local_rank)
    tune = plan.autotune(a, 3600.0)
    outb = torch.empty_like(a[5])
    for _ in range(20):
        plan.forward(*a, 3600.0, out=outb)
    stream = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 500
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        plan.forward(*a, 3600.0, out=outb)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    got = outb.cpu().numpy()
    lm = m.node_layer_mask
    worst, t_cpu = 0.0, 0.0
    for tr in range(2):
        c0 = time.perf_counter()
        ref, _ = fct_c.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                      f.tracers[tr], f.tracers_old[tr], dt=3600.0)
        t_cpu += time.perf_counter() - c0
        worst = max(worst, float(np.max(np.abs(got[tr][lm] - ref[lm])) / np.max(np.abs(ref[lm]))))
    upd = 2 * m.n_wet_layers
    out["pi_plain"] = dict(value=upd / t, unit=UNIT, ms_per_step=t * 1e3, max_rel_err=worst,
                           cpu_value=upd / t_cpu, cpu_cores=fct_c.max_threads(),
                           tuning_ms=tune,
                           how="fct_forward, T and S in one call, one FCT step, dt 3600")
    a2 = copy.copy(args)
    a2.no_fd, a2.steps, a2.warmup = True, 2, 1
    r = run_adjoint(a2, D)["adjoint"]
    out["adjoint"] = {k: r[k] for k in ("forward_ms", "loss_and_grad_ms", "ratio", "K",
                                        "checkpoint", "recompute_loss_and_grad_ms",
                                        "recompute_ratio", "tape_equals_recompute")}
    return out


# ------------------------------------------------------------------ reference arm
def run_reference(args, D: Dist):
    """CPU arm: the C restatement of the reference algorithm on the box's host cores
    (JAX is not installed, so the reference's own jax.jit CPU path cannot run); rank 0
    only, each step one member x ntr tracers x 1 FCT step of the same workload."""
    if D.rank != 0:
        return
    from fesom_jax_b200 import inputs as I
    from fesom_jax_b200 import workloads as W
    from oracle import fct_c
    cfg = dict(W.WORKLOADS[args.config])
    mesh = W.make_workload_mesh(args.config, seed=0)
    f = I.make_fields(mesh, seed=1, n_passive=max(cfg["ntr"] - 2, 0), ab2=True,
                      sigma=cfg["sigma"], n_vortices=cfg["n_vortices"], kind=cfg["velocity"])
    ntr = cfg["ntr"]
    keep = []
    from fesom_jax_b200 import _lib as fl
    desc = fl.mesh_desc(mesh, keep)

    def step():
        for t in range(ntr):
            fct_c.advect_one_fct(mesh, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                 f.tracers[t], f.tracers_old[t], dt=cfg["dt"], desc=desc)

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    t = time.perf_counter() - t0
    value = args.steps * ntr * mesh.n_wet_layers / t
    cores = fct_c.max_threads()
    sample = (f"C loop restatement (OpenMP, {cores} threads): per step 1 member x {ntr} "
              f"tracers x 1 FCT step on {mesh.name}")
    line = dict(metric=METRIC, value=value, unit=UNIT, impl="reference", n_gpus=args.gpus,
                steps=args.steps, warmup=args.warmup, ms_per_step=t / args.steps * 1e3,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic", config=workload_config(args.config, cfg, mesh),
                cpu_baseline=dict(value=value, unit=UNIT, cores=cores, kind="port",
                                  sample=sample),
                e2e=dict(value=value, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))
    print(json.dumps(line), flush=True)


def side_line(args, D: Dist, r: dict) -> dict:
    """The JSON line of the adjoint and serving workloads."""
    line = dict(metric=METRIC, value=r["value"], unit=UNIT, n_gpus=D.world, steps=args.steps,
                warmup=args.warmup, ms_per_step=r["t"] / max(args.steps, 1) * 1e3,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic (seeded mesh, velocities and tracers)")
    if args.config == "adjoint":
        m = r["mesh"]
        line["config"] = dict(workload=f"adjoint: 10-step loss gradient (T0, uv), {m.name} mesh",
                              nod2D=m.nod2D, nl=m.nl, wet_node_layers=m.n_wet_layers,
                              tracers=1, fct_steps=10, dt=1800.0,
                              value_is="forward-equivalent updates/s of the loss+gradient")
        line["adjoint"] = r["adjoint"]
    else:
        line["config"] = dict(workload="serve: Poisson 200 req/s, pi/CORE2/1.3M mix 0.6/0.3/0.1, "
                                       "K~U{1..50}, 20% adjoint, 150 GB budget, T+S",
                              value_is="node-level updates/s served (saturated stream)",
                              max_steps_per_iteration=args.serve_rounds)
        for k in ("saturated", "sustainable", "serial", "clocks"):
            line[k] = r[k]
    return line


def workload_config(name, cfg, mesh) -> dict:
    from fesom_jax_b200 import workloads as W
    return dict(workload=f"{name}: FCT tracer advection, {mesh.name} mesh", nod2D=mesh.nod2D,
                elem2D=mesh.elem2D, edge2D=mesh.edge2D, nl=mesh.nl,
                wet_node_layers=mesh.n_wet_layers, members=cfg["members"], tracers=cfg["ntr"],
                fct_steps_per_bench_step=cfg["fct_steps"], dt=cfg["dt"],
                velocity=W.velocity_note(name),
                l2="inputs larger than L2 (resident state >> 126 MB)",
                parallelism="replicas: members per GPU, no collective")


def parse_stage_mapping(text):
    """'4x2,2x2,2x1,4x1' -> [(4, 2), (2, 2), (2, 1), (4, 1)] (one pair per fused stage)."""
    out = [tuple(int(v) for v in part.split("x")) for part in text.split(",")]
    if len(out) != 4 or any(len(m) != 2 for m in out):
        raise SystemExit(f"--stage-mapping wants four TRACERSxLEVELS pairs, got {text!r}")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", choices=["batched", "pi", "large", "adjoint", "serve"],
                    default="batched")
    ap.add_argument("--serve-seconds", type=float, default=2.0,
                    help="serve: seconds of Poisson arrivals at 200 req/s")
    ap.add_argument("--serve-rounds", type=int, default=16,
                    help="serve: most steps a request takes per iteration (1 = lockstep)")
    ap.add_argument("--serve-limit", type=float, default=90.0,
                    help="serve: wall-clock cap per stream")
    ap.add_argument("--members", type=int, default=0)
    ap.add_argument("--fct-steps", type=int, default=0)
    ap.add_argument("--ntr", type=int, default=0, help="override tracers per member")
    ap.add_argument("--chunk", type=int, default=0,
                    help="fix the tracers per thread (no autotune)")
    ap.add_argument("--levels", type=int, default=0,
                    help="fix the levels per thread (no autotune)")
    ap.add_argument("--stage-mapping", default="",
                    help="fix the mapping stage by stage (no autotune): tracers x levels per "
                         "thread for LO, edge, limiter, final, e.g. 4x2,2x2,2x1,4x1")
    ap.add_argument("--workspace-gb", type=float, default=40.0)
    ap.add_argument("--e2e-members", type=int, default=8)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-checks", "--no-fd", dest="no_fd", action="store_true",
                    help="adjoint: skip the gradient checks (dot-product and Taylor tests)")
    ap.add_argument("--no-side", action="store_true",
                    help="batched: skip the side measurements of the pi and adjoint configs")
    ap.add_argument("--no-gates", action="store_true",
                    help="skip the per-run correctness gates (oracle parity, closure, window)")
    ap.add_argument("--node-order", choices=["rcm", "raw", "random"], default="rcm",
                    help="synthetic meshes: node numbering (reverse Cuthill-McKee, the "
                         "generator's Fibonacci order, or a seeded shuffle)")
    ap.add_argument("--checkpoint", choices=["tape", "recompute"], default="tape",
                    help="adjoint: keep every step's intermediates (tape; the per-step "
                         "recomputation is timed beside it) or recompute them only")
    ap.add_argument("--derive-w", action="store_true",
                    help="batched/large: derive w_e = compute_w(uv) inside every step's graph")
    ap.add_argument("--vdiff", action="store_true",
                    help="batched/large: implicit vertical diffusion after every FCT step")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    D = Dist()
    if args.impl == "reference":
        run_reference(args, D)
        return
    D.init("nccl")
    try:
        if args.config == "adjoint":
            r = run_adjoint(args, D)
        elif args.config == "serve":
            r = run_serve(args, D)
        else:
            r = run_ours(args, D)
            if r is not None and args.config == "batched" and D.world == 1 and not args.no_side:
                r["side"] = run_side(args, D)
    finally:
        D.close()
    if D.rank != 0 or r is None:
        return
    if args.config in ("adjoint", "serve"):
        print(json.dumps(side_line(args, D, r)), flush=True)
        return
    cfg, mesh = r["cfg"], r["mesh"]
    line = dict(metric=METRIC, value=r["value"], unit=UNIT, n_gpus=D.world, steps=args.steps,
                warmup=args.warmup, ms_per_step=r["t"] / args.steps * 1e3,
                higher_is_better=True, scaling="weak", vs_baseline=None, dtype="f64",
                data="synthetic (seeded mesh, velocities and tracers)",
                config=dict(workload_config(args.config, cfg, mesh), vertical_diffusion=bool(args.vdiff),
                            derive_w=bool(args.derive_w)),
                roofline=r["roofline"],
                clocks=r["clocks"], gpu_launches=r["gpu_launches"],
                fct_step_ms=r["fct_step_ms"], stage_ms=r["prof"], finite=r["finite"],
                nonfinite=r["nonfinite"], gates=r["gates"], batch=r["info"], tuning=r["tuning"])
    for k in ("plain", "e2e", "cpu_baseline", "side"):
        if k in r:
            line[k] = r[k]
    e2e_ok = "e2e" not in r or (r["e2e"]["outputs_finite"] and r["e2e"]["outputs_repeat_bitwise"])
    failed = (not r["finite"] or (r["gates"] is not None and not r["gates"]["passed"])
              or not e2e_ok)
    if failed:   # a state that went non-finite or failed a gate gives no throughput
        line["value"] = None
        line["error"] = ("non-finite state" if not r["finite"] else
                         "end-to-end outputs not finite or not repeatable" if not e2e_ok else
                         "correctness gate failed")
    print(json.dumps(line), flush=True)
    if failed:
        sys.exit(1)


if __name__ == "__main__":
    main()
