"""Golden vectors for the sea-ice FCT advection from the reference itself:
``fesom_jax.ice_adv.fct_solve`` (ice_adv.py:175-194) run unmodified through the
numpy-backed ``jax`` stand-in of ``make_golden.py`` with the reference's ``IceConfig``
(gamma 0.5, ice_diff 10), on the pi mesh and on the seeded coastline mesh of
``make_mesh_golden.py`` (the reference's own ``prepare_mesh.derive``), for the cases of
``tests/golden_cases.ice_cases``.

    python tests/golden/make_ice_golden.py          # needs the reference checkout
"""

from __future__ import annotations

import importlib.util
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(HERE))

import make_golden as mg  # noqa: E402
from make_mesh_golden_params import N_NODES, SEED  # noqa: E402

from fesom_jax_b200 import meshgen  # noqa: E402
from fesom_jax_b200.mesh import pi_mesh  # noqa: E402
from tests.golden_cases import ICE_GOLDEN, ice_cases  # noqa: E402


def main():
    mg.import_reference()
    import fesom_jax.ice_adv as ia
    import fesom_jax.mesh as rmesh
    from fesom_jax.ice import IceConfig
    spec = importlib.util.spec_from_file_location("prepare_mesh", mg.REF / "scripts/prepare_mesh.py")
    pm = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(pm)
    raw = meshgen.generate_raw(N_NODES, pi_mesh().zbar, seed=SEED)
    tmp = Path(tempfile.mkdtemp(prefix="ice_small_"))
    pm.write_mesh(pm.derive(raw), tmp)
    meshes = {"pi": (rmesh.load_mesh(mg.REF / "fesom_jax/data/mesh_pi"), pi_mesh()),
              "small": (rmesh.load_mesh(tmp), None)}
    out = {}
    for mname, (rm, m) in meshes.items():
        nod2D = int(np.asarray(rm.nlevels_nod2D).shape[0])
        coords = np.asarray(rm.coord_nod2D)

        class _M:   # the inputs need coordinates only
            pass
        mm = _M()
        mm.nod2D, mm.coord_nod2D = nod2D, coords
        for name, c in ice_cases(mm).items():
            cfg = IceConfig(ice_dt=c["dt"])
            res = ia.fct_solve(cfg, rm, c["a"], c["m"], c["ms"], c["u"], c["v"])
            for tr, x in zip(("a", "m", "ms"), res):
                out[f"{mname}_{name}__{tr}"] = np.asarray(x)
            print(f"{mname}/{name}: max|da| = {np.max(np.abs(np.asarray(res[0]) - c['a'])):.3e}")
    np.savez_compressed(ICE_GOLDEN, **out)
    print("wrote", ICE_GOLDEN)


if __name__ == "__main__":
    main()
