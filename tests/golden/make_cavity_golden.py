"""Golden vectors on a mesh with an ice-shelf cavity (layers above a node's ulevels are
dry), from the reference itself: ``fesom_jax.tracer_adv.advect_one_fct``,
``fesom_jax.ale.compute_w`` and ``fesom_jax.tracer_diff.impl_vert_diff_one`` run unmodified
through the numpy-backed ``jax`` stand-in of ``make_golden.py`` on a copy of the shipped pi
mesh whose ``ulevels``/``ulevels_nod2D``/``ulevels_nod2D_max``/``area``/``areasvol`` are
replaced by ``tests/golden_cases.cavity_arrays`` (the reference's own loader derives the
level masks from them).

    python tests/golden/make_cavity_golden.py          # needs the reference checkout
"""

from __future__ import annotations

import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

import make_golden as mg  # noqa: E402

from fesom_jax_b200.mesh import pi_mesh  # noqa: E402
from tests.golden_cases import (CAVITY_GOLDEN, cases, cavity_arrays, cavity_mesh,  # noqa: E402
                                vdiff_cases)

DT = 3600.0


def main():
    ta, ale, rmesh = mg.import_reference()
    import fesom_jax.tracer_diff as td
    src = mg.REF / "fesom_jax/data/mesh_pi"
    tmp = Path(tempfile.mkdtemp(prefix="mesh_pi_cavity_")) / "mesh"
    shutil.copytree(src, tmp)
    pi = pi_mesh()
    for name, arr in cavity_arrays(pi).items():
        ref_dtype = np.load(src / f"{name}.npy").dtype
        np.save(tmp / f"{name}.npy", np.asarray(arr, ref_dtype))
    rm = rmesh.load_mesh(tmp)
    m = cavity_mesh(pi)
    assert np.array_equal(np.asarray(rm.node_layer_mask), m.node_layer_mask)
    out = {}
    cs = cases(m)
    for name in ("T_step1", "T_ab2", "sharp_x5"):
        c = cs[name]
        Tn, _ = ta.advect_one_fct(rm, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                  c["hnode_new"], c["T"], c["T_old"], dt=DT)
        out[f"{name}__T_new"] = np.asarray(Tn)[mg.SAMPLE]
        out[f"{name}__digest"] = mg.field_digest(m, np.asarray(Tn))
        print(f"{name}: max|dT| = {np.max(np.abs(np.asarray(Tn) - c['T'])):.3e}")
    c = cs["T_step1"]
    w = np.asarray(ale.compute_w(rm, c["uv"], c["helem"]))
    out["w_e"] = w[mg.SAMPLE]
    out["w_e__digest"] = mg.field_digest(m, w, m.node_iface_mask)
    v = vdiff_cases(m)["T"]
    Tv = np.asarray(td.impl_vert_diff_one(rm, v["T"], v["Kv"], v["hnode_new"], dt=DT))
    out["vdiff__T_new"] = Tv[mg.SAMPLE]
    out["vdiff__digest"] = mg.field_digest(m, Tv)
    np.savez_compressed(CAVITY_GOLDEN, **out)
    print("wrote", CAVITY_GOLDEN)


if __name__ == "__main__":
    main()
