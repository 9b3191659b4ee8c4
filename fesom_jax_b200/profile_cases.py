"""Each secondary operator of the package, run a few times on the CORE2-size workload mesh
(126,990 nodes, 48 levels, rest thicknesses, closed-basin velocities): a fixed case to
time or profile one kernel family on its own.

    python -m fesom_jax_b200.profile_cases compute_w   # k_compute_w   (ale.compute_w)
    python -m fesom_jax_b200.profile_cases vdiff       # k_vdiff       (tracer_diff, T and S)
    python -m fesom_jax_b200.profile_cases ice         # k_ice_*       (ice_adv.fct_solve)
    python -m fesom_jax_b200.profile_cases wsplit      # k_vert_impl   (advect_one_fct, w_i)

Every call is checked for finite output; the process prints one line with the mean
CUDA-event time per call and exits 0.
"""

import argparse
import json


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["compute_w", "vdiff", "ice", "wsplit"])
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args(argv)

    import torch
    from . import workloads as W
    from .ale import compute_w
    from .ice_adv import IceConfig, fct_solve
    from .tracer_diff import impl_vert_diff

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    mesh = W.make_workload_mesh("batched", seed=0)
    cfg = W.WORKLOADS["batched"]
    thick = W.rest_thickness_gpu(mesh, dev)
    inp = W.member_inputs_gpu(mesh, seed=0, ntr=2, device=dev, thickness=thick,
                              sigma=cfg["sigma"], n_vortices=cfg["n_vortices"],
                              kind=cfg["velocity"])
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    N = mesh.nod2D

    if args.case == "compute_w":
        def call():
            return [compute_w(mesh, inp["uv"], thick.helem)]
    elif args.case == "vdiff":
        im = torch.from_numpy(mesh.node_iface_mask).to(dev)
        Kv = torch.where(im, 1e-5 + 1e-3 * torch.rand(im.shape, generator=g, device=dev,
                                                      dtype=torch.float64), 0.0)
        T, S = inp["T"][0].contiguous(), inp["T"][1].contiguous()

        def call():
            return list(impl_vert_diff(mesh, T, S, Kv, thick.hnode_new, dt=cfg["dt"]))
    elif args.case == "wsplit":
        # the split vertical velocity of tracer_adv.py:487-529: half of w_e explicit, half
        # implicit (w_i), T and S in one call
        from .tracer_adv import advect_one_fct
        w_half = (0.5 * inp["w_e"]).contiguous()
        T, To = inp["T"], inp["T_old"]

        def call():
            return [advect_one_fct(mesh, inp["uv"], w_half, thick.helem, thick.hnode,
                                   thick.hnode_new, T, To, dt=cfg["dt"], w_i=w_half)[0]]
    else:
        a = torch.rand(N, generator=g, device=dev, dtype=torch.float64)
        m = 2.0 * torch.rand(N, generator=g, device=dev, dtype=torch.float64)
        s = 0.3 * torch.rand(N, generator=g, device=dev, dtype=torch.float64)
        u = 0.1 * torch.randn(N, generator=g, device=dev, dtype=torch.float64)
        v = 0.1 * torch.randn(N, generator=g, device=dev, dtype=torch.float64)

        def call():
            return list(fct_solve(IceConfig(), mesh, a, m, s, u, v))

    call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.reps):
        out = call()
    e1.record()
    torch.cuda.synchronize()
    for x in out:
        if not bool(torch.isfinite(x).all()):
            raise SystemExit(f"{args.case}: non-finite output")
    print(json.dumps({"case": args.case, "reps": args.reps, "nodes": N, "nl": mesh.nl,
                      "ms_per_call": e0.elapsed_time(e1) / args.reps}))


if __name__ == "__main__":
    main()
