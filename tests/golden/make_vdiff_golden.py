"""Golden vectors for the implicit vertical tracer diffusion from the reference itself:
``fesom_jax.tracer_diff.impl_vert_diff_one`` (tracer_diff.py:68-123) run unmodified
through the numpy-backed ``jax`` stand-in of ``make_golden.py`` (its ``ops.tdma`` uses
``lax.scan``, which the stand-in runs as a Python loop) on the seeded pi-mesh cases of
``tests/golden_cases.vdiff_cases``; plus ``impl_vert_diff`` (T and S, :126-141).

    python tests/golden/make_vdiff_golden.py          # needs the reference checkout
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

from make_golden import REF, SAMPLE, digest, field_digest, import_reference  # noqa: E402

from fesom_jax_b200.mesh import pi_mesh  # noqa: E402
from tests.golden_cases import VDIFF_GOLDEN, vdiff_cases  # noqa: E402

DT = 3600.0


def main():
    import_reference()
    import fesom_jax.mesh as rmesh
    import fesom_jax.tracer_diff as td
    rm = rmesh.load_mesh(REF / "fesom_jax/data/mesh_pi")
    m = pi_mesh()
    out = {}
    for name, c in vdiff_cases(m).items():
        Tn = np.asarray(td.impl_vert_diff_one(rm, c["T"], c["Kv"], c["hnode_new"], dt=DT,
                                              **c["kw"]))
        out[f"{name}__T_new"] = Tn[SAMPLE]
        out[f"{name}__digest"] = field_digest(m, Tn)
        out[f"{name}__in_digest"] = np.frombuffer(bytes.fromhex(
            digest(c["T"], c["Kv"], c["hnode_new"], *c["kw"].values())), np.uint8)
        print(f"{name:8s} max|dT| = {np.max(np.abs(Tn - c['T'])):.3e}")
    cs = vdiff_cases(m)
    T, S = cs["T"]["T"], cs["S_bc"]["T"]
    Tn, Sn = td.impl_vert_diff(rm, T, S, cs["T"]["Kv"], cs["T"]["hnode_new"], dt=DT,
                               bc_T=cs["S_bc"]["kw"]["bc_surf"] * 2.0,
                               bc_S=cs["S_bc"]["kw"]["bc_surf"], sw_3d=cs["T_sw"]["kw"]["sw_3d"])
    out["pair__T_new"] = np.asarray(Tn)[SAMPLE]
    out["pair__S_new"] = np.asarray(Sn)[SAMPLE]
    out["pair__T_digest"] = field_digest(m, np.asarray(Tn))
    out["pair__S_digest"] = field_digest(m, np.asarray(Sn))
    np.savez_compressed(VDIFF_GOLDEN, **out)
    print("wrote", VDIFF_GOLDEN)


if __name__ == "__main__":
    main()
