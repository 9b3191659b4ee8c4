"""Parity at the measured configurations (the reference pins its FCT on full fields,
fesom_jax/tests/test_tracers.py:573-596):

* the CORE2-size mesh (127,000 nodes, 48 levels) through the batched engine as the
  benchmark runs it: 3 members x 8 tracers, 2 tracers per thread, one member per
  workspace group (3 groups), 30 one-step CUDA graphs; member 0 checked against the C
  oracle every step (every tracer, max-norm over wet lanes <= 1e-12, dry levels equal to
  T bit for bit), the others after the last step, the limiter window of tracer 0 after
  the last step, and a 30-step graph from the same start equal to the 30 single steps;
* the 1.3M-node mesh (70 levels, 10 tracers) for one step with the workspace in chunks
  of 8 + 2 tracers (the large benchmark's layout), every tracer against the C oracle.

Velocities are the benchmark's closed-basin flows (low-order CFL below 1)."""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from fesom_jax_b200 import workloads as W
from oracle import fct_c, fct_np, gates

pytestmark = pytest.mark.gpu
RTOL = 1e-12


@pytest.fixture(scope="module")
def torch():
    import torch
    assert torch.cuda.is_available()
    return torch


def _check(mesh, desc, host, T, To, Tn, dt, tracers):
    lm = mesh.node_layer_mask
    worst = 0.0
    for t in tracers:
        ref, _ = fct_c.advect_one_fct(mesh, host["uv"], host["w_e"], host["helem"],
                                      host["hnode"], host["hnode_new"], T[t], To[t], dt=dt,
                                      desc=desc)
        err = float(np.max(np.abs(Tn[t][lm] - ref[lm])) / np.max(np.abs(ref[lm])))
        worst = max(worst, err)
        assert err <= RTOL, (t, err)
        assert np.array_equal(Tn[t][~lm], T[t][~lm]), t
    return worst


def _members(torch, mesh, cfg, n, ntr):
    thick = W.rest_thickness_gpu(mesh, torch.device("cuda", 0))
    out = []
    for i in range(n):
        inp = W.member_inputs_gpu(mesh, seed=900 + i, ntr=ntr, device=torch.device("cuda", 0),
                                  thickness=thick, sigma=cfg["sigma"],
                                  n_vortices=cfg["n_vortices"], kind=cfg["velocity"])
        out.append(inp)
    return out


def _ws_bytes(mesh, chunk):
    N, Ed, L = mesh.nod2D, mesh.edge2D, mesh.nl
    pad = lambda n: (n + 31) // 32 * 32  # noqa: E731  (fields on 256-byte boundaries)
    return 8 * (pad(Ed * L) + 4 * pad(chunk * N * L) + pad(chunk * Ed * L))


def test_core2_batched_tuned_mapping_30_steps(torch):
    from fesom_jax_b200 import _lib as fl
    from fesom_jax_b200.ensemble import Ensemble
    mesh = W.make_workload_mesh("batched", seed=0)
    cfg = W.WORKLOADS["batched"]
    dt = cfg["dt"]
    inps = _members(torch, mesh, cfg, 3, 8)
    host = [{k: inp[k].cpu().numpy() for k in ("uv", "w_e", "helem", "hnode", "hnode_new")}
            for inp in inps]
    assert I.lo_outflow_cfl(mesh, host[0]["uv"], host[0]["w_e"], host[0]["hnode"], dt) < 1.0

    def build():
        ens = Ensemble(device=0, workspace_budget=_ws_bytes(mesh, 8) + 1024)
        for inp in inps:
            ens.add_member(mesh, inp["uv"], inp["w_e"], inp["helem"], inp["hnode"],
                           inp["hnode_new"], inp["T"], inp["T_old"], dt)
        ens.build()
        ens.set_chunk(2)
        return ens

    ens = build()
    assert ens.info()["groups"] == 3
    keep = []
    desc = fl.mesh_desc(mesh, keep)
    for step in range(30):
        T, To = (x.cpu().numpy() for x in ens.state(0))
        if step == 29:
            prev = [tuple(x.cpu().numpy() for x in ens.state(i)) for i in (1, 2)]
        ens.run(1)
        Tn = ens.state(0)[0].cpu().numpy()
        _check(mesh, desc, host[0], T, To, Tn, dt, range(8))
    for j, i in enumerate((1, 2)):
        _check(mesh, desc, host[i], prev[j][0], prev[j][1], ens.state(i)[0].cpu().numpy(), dt,
               range(8))
    inter = {}
    fct_np.advect_one_fct(mesh, host[0]["uv"], host[0]["w_e"], host[0]["helem"],
                          host[0]["hnode"], host[0]["hnode_new"], T[0], To[0], dt=dt,
                          intermediates=inter)
    assert len(gates.window_violations(mesh, T[0], host[0]["hnode_new"], Tn[0], inter,
                                          gates.GPU_WINDOW_ULPS)) == 0
    assert ens.health() == [0, 0, 0]
    stepped = [ens.state(i)[0].cpu().numpy() for i in range(3)]
    ens.close()
    ens = build()
    ens.run(30)
    for i in range(3):
        assert np.array_equal(ens.state(i)[0].cpu().numpy(), stepped[i]), i
    ens.close()


def test_large_mesh_one_step_chunked(torch):
    from fesom_jax_b200 import _lib as fl
    from fesom_jax_b200.ensemble import Ensemble
    mesh = W.make_workload_mesh("large", seed=0)
    cfg = W.WORKLOADS["large"]
    dt = cfg["dt"]
    inp = _members(torch, mesh, cfg, 1, cfg["ntr"])[0]
    # a budget that holds 8 tracers' workspace but not 10: chunks of 8 + 2
    ens = Ensemble(device=0, workspace_budget=_ws_bytes(mesh, 8) + 1024)
    ens.add_member(mesh, inp["uv"], inp["w_e"], inp["helem"], inp["hnode"], inp["hnode_new"],
                   inp["T"], inp["T_old"], dt)
    ens.build()
    assert ens.info()["workspace_tracers"] == 8
    host = {k: inp[k].cpu().numpy() for k in ("uv", "w_e", "helem", "hnode", "hnode_new")}
    T, To = inp["T"].cpu().numpy(), inp["T_old"].cpu().numpy()
    del inp
    ens.run(1)
    Tn = ens.state(0)[0].cpu().numpy()
    keep = []
    desc = fl.mesh_desc(mesh, keep)
    _check(mesh, desc, host, T, To, Tn, dt, range(cfg["ntr"]))
    assert ens.health() == [0]
    ens.close()
