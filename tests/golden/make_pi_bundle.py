"""Build ``fesom_jax_b200/data/mesh_pi.npz`` from the reference's pi mesh export directory.

The pi mesh (3140 nodes) ships with the reference as one ``.npy`` per array
(fesom_jax/data/mesh_pi, layout in docs/MESH_EXPORT_LAYOUT.md). This script keeps the
arrays the FCT path reads and writes them, unchanged, into one compressed bundle so the
mesh travels with this package:

    python tests/golden/make_pi_bundle.py [<reference checkout>/fesom_jax/data/mesh_pi]

Without an argument it reads the checkout named by FESOM_JAX_REFERENCE (or a
``reference`` directory beside this repository), as the golden generators do.
"""

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
sys.path.insert(0, str(Path(__file__).resolve().parent))
from fesom_jax_b200.mesh import PI_BUNDLE, load_mesh, save_bundle  # noqa: E402


def main(src: str) -> None:
    m = load_mesh(Path(src), name="pi")
    save_bundle(m, PI_BUNDLE)
    back = load_mesh(PI_BUNDLE)
    for f, a in m.arrays().items():
        assert np.array_equal(a, getattr(back, f)), f
    print(f"wrote {PI_BUNDLE} ({PI_BUNDLE.stat().st_size} bytes)")


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    else:
        from make_golden import REF
        main(str(REF / "fesom_jax/data/mesh_pi"))
