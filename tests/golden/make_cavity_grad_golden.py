"""Golden gradients of one FCT step on the ice-shelf cavity mesh of
``tests/golden_cases.cavity_arrays``, from the reference itself: the torch-backed ``jax``
stand-in of ``make_grad_golden.py`` runs the reference's unmodified
``tracer_adv.advect_one_fct`` on the cavity copy of the pi mesh (as in
``make_cavity_golden.py``) with autograd; loss = sum(wts * T_new), seeded weights on wet
layers; gradients w.r.t. T, T_old, uv and w_e.

    python tests/golden/make_cavity_grad_golden.py     # needs the reference checkout
"""

from __future__ import annotations

import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

import make_golden as mg  # noqa: E402
from make_grad_golden import DT, import_reference_torch, sample  # noqa: E402

from fesom_jax_b200 import inputs as I  # noqa: E402
from fesom_jax_b200.mesh import pi_mesh  # noqa: E402
from tests.golden_cases import cavity_arrays, cavity_mesh  # noqa: E402

OUT = HERE / "fct_cavity_grad_golden.npz"


def main():
    import torch
    torch.set_default_dtype(torch.float64)
    ta, ale, rmesh = import_reference_torch()
    src = mg.REF / "fesom_jax/data/mesh_pi"
    tmp = Path(tempfile.mkdtemp(prefix="mesh_pi_cavity_")) / "mesh"
    shutil.copytree(src, tmp)
    pi = pi_mesh()
    for name, arr in cavity_arrays(pi).items():
        np.save(tmp / f"{name}.npy", np.asarray(arr, np.load(src / f"{name}.npy").dtype))
    rm = rmesh.load_mesh(tmp)
    m = cavity_mesh(pi)
    lm = m.node_layer_mask
    f = I.make_fields(m, seed=0, ab2=True)
    tt = lambda x: torch.tensor(np.asarray(x), dtype=torch.float64, requires_grad=True)  # noqa
    wts = np.where(lm, np.random.default_rng(99).normal(size=lm.shape), 0.0)
    T, To, uv, w = tt(f.tracers[0]), tt(f.tracers_old[0]), tt(f.uv), tt(f.w_e)
    Tn, _ = ta.advect_one_fct(rm, uv, w, torch.tensor(f.helem), torch.tensor(f.hnode),
                              torch.tensor(f.hnode_new), T, To, dt=DT)
    loss = (torch.tensor(wts) * Tn).sum()
    loss.backward()
    out = {}
    for name, x in (("T", T), ("T_old", To), ("uv", uv), ("w_e", w)):
        s, d = sample(m, x.grad.numpy())
        out[f"step__g_{name}"], out[f"step__g_{name}_digest"] = s, d
    out["step__loss"] = np.array(loss.item())
    np.savez_compressed(OUT, **out)
    print("cavity step: loss", loss.item(), "wrote", OUT, OUT.stat().st_size)


if __name__ == "__main__":
    main()
