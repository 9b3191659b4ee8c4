"""Build ``mesh_pi.npz`` from the reference's pi mesh export directory.

The pi mesh (3140 nodes) ships with the reference as one ``.npy`` per array
(fesom_jax/data/mesh_pi, layout in docs/MESH_EXPORT_LAYOUT.md). This script keeps the
arrays the FCT path reads and writes them, unchanged, into one compressed bundle so the
mesh travels with this package:

    python fesom_jax_b200/data/make_pi_bundle.py /root/reference/fesom_jax/data/mesh_pi
"""

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from fesom_jax_b200.mesh import PI_BUNDLE, load_mesh, save_bundle  # noqa: E402


def main(src: str) -> None:
    m = load_mesh(Path(src), name="pi")
    save_bundle(m, PI_BUNDLE)
    back = load_mesh(PI_BUNDLE)
    for f, a in m.arrays().items():
        assert np.array_equal(a, getattr(back, f)), f
    print(f"wrote {PI_BUNDLE} ({PI_BUNDLE.stat().st_size} bytes)")


if __name__ == "__main__":
    main(sys.argv[1])
