"""Static FESOM2 mesh container for the FCT tracer-advection path.

Holds the subset of the reference ``Mesh`` (fesom_jax/mesh.py:62-123) that the FCT
advection reads, as host numpy arrays with the reference's field names, dtypes and
row-major ``[entity, nl]`` layout, so the same object can be handed to the CUDA plan
(``fesom_jax_b200.tracer_adv``) and to the CPU oracle.

Conventions (fesom_jax/mesh.py:11-33):
  * indices are 0-based int32; ``edge_tri``/``edge_up_dn_tri`` carry -1 for a missing
    neighbour;
  * for node ``n``: layers ``k in [ulevels_nod2D-1, nlevels_nod2D-1)``, interfaces
    ``k in [ulevels_nod2D-1, nlevels_nod2D-1]``; elements likewise with
    ``ulevels``/``nlevels`` (fesom_jax/mesh.py:135-151).

Two on-disk formats load into it:
  * the reference's export layout (one ``<name>.npy`` per array plus ``meta.txt``,
    fesom_jax/mesh.py:225-274);
  * a single ``.npz`` bundle with the same array names plus the scalar counts
    (``fesom_jax_b200/data/mesh_pi.npz`` is the pi mesh in this form).
"""

from __future__ import annotations

import dataclasses
from pathlib import Path

import numpy as np

R_EARTH = 6367500.0  # fesom_jax/config.py:41
CYCLIC_LENGTH_RAD = 2.0 * 3.14159265358979  # fesom_jax/config.py:55 (truncated pi)

DATA_DIR = Path(__file__).resolve().parent / "data"
PI_BUNDLE = DATA_DIR / "mesh_pi.npz"

# Arrays the FCT path reads (plus coordinates, used for locality reordering and the
# orientation check). Name -> (dtype, per-entity trailing shape or None).
FCT_FIELDS = (
    "coord_nod2D",
    "nlevels_nod2D", "nlevels_nod2D_min", "ulevels_nod2D", "ulevels_nod2D_max",
    "area", "areasvol", "nod_in_elem2D_offsets", "nod_in_elem2D",
    "elem_nodes", "nlevels", "ulevels", "elem_area", "elem_cos", "gradient_sca",
    "edges", "edge_tri", "edge_dxdy", "edge_cross_dxdy", "edge_up_dn_tri",
    "zbar", "Z",
)
_INT_FIELDS = {
    "nlevels_nod2D", "nlevels_nod2D_min", "ulevels_nod2D", "ulevels_nod2D_max",
    "nod_in_elem2D_offsets", "nod_in_elem2D", "elem_nodes", "nlevels", "ulevels",
    "edges", "edge_tri", "edge_up_dn_tri",
}


def level_masks(ulevels, nlevels, nl: int):
    """``(layer_mask, iface_mask)`` ``[n, nl]`` bool (fesom_jax/mesh.py:135-151):
    layer ``ulevels-1 <= k < nlevels-1``; interface ``ulevels-1 <= k < nlevels``."""
    u = np.asarray(ulevels).reshape(-1, 1)
    n = np.asarray(nlevels).reshape(-1, 1)
    k = np.arange(nl).reshape(1, -1)
    top = k >= (u - 1)
    return top & (k < (n - 1)), top & (k < n)


@dataclasses.dataclass(eq=False)
class Mesh:
    """FESOM2 mesh arrays used by FCT advection (host numpy, reference names)."""

    coord_nod2D: np.ndarray
    nlevels_nod2D: np.ndarray
    nlevels_nod2D_min: np.ndarray
    ulevels_nod2D: np.ndarray
    ulevels_nod2D_max: np.ndarray
    area: np.ndarray
    areasvol: np.ndarray
    nod_in_elem2D_offsets: np.ndarray
    nod_in_elem2D: np.ndarray
    elem_nodes: np.ndarray
    nlevels: np.ndarray
    ulevels: np.ndarray
    elem_area: np.ndarray
    elem_cos: np.ndarray
    gradient_sca: np.ndarray
    edges: np.ndarray
    edge_tri: np.ndarray
    edge_dxdy: np.ndarray
    edge_cross_dxdy: np.ndarray
    edge_up_dn_tri: np.ndarray
    zbar: np.ndarray
    Z: np.ndarray
    name: str = "mesh"

    def __post_init__(self):
        for f in FCT_FIELDS:
            a = np.asarray(getattr(self, f))
            a = a.astype(np.int32 if f in _INT_FIELDS else np.float64, copy=False)
            setattr(self, f, np.ascontiguousarray(a))
        nl = self.nl
        self.node_layer_mask, self.node_iface_mask = level_masks(
            self.ulevels_nod2D, self.nlevels_nod2D, nl)
        self.elem_layer_mask, self.elem_iface_mask = level_masks(
            self.ulevels, self.nlevels, nl)

    # -- counts (static metadata in the reference Mesh) --
    @property
    def nod2D(self) -> int:
        return int(self.nlevels_nod2D.shape[0])

    @property
    def elem2D(self) -> int:
        return int(self.elem_nodes.shape[0])

    @property
    def edge2D(self) -> int:
        return int(self.edges.shape[0])

    @property
    def myDim_edge2D(self) -> int:
        return int(self.edge_up_dn_tri.shape[0])

    @property
    def nl(self) -> int:
        return int(self.zbar.shape[0])

    # -- workload sizes used by the throughput metric --
    @property
    def n_wet_layers(self) -> int:
        """``N_wl = sum_n (nlevels_nod2D - ulevels_nod2D)``: wet node layers."""
        return int(np.sum(self.nlevels_nod2D.astype(np.int64) - self.ulevels_nod2D))

    @property
    def n_wet_elem_layers(self) -> int:
        return int(np.sum(self.nlevels.astype(np.int64) - self.ulevels))

    def arrays(self) -> dict:
        return {f: getattr(self, f) for f in FCT_FIELDS}

    def validate(self) -> None:
        """Shape/range checks the CUDA plan relies on; raises ``ValueError``."""
        N, E, Ed, nl = self.nod2D, self.elem2D, self.edge2D, self.nl
        shapes = {
            "coord_nod2D": (N, 2), "area": (N, nl), "areasvol": (N, nl),
            "nod_in_elem2D_offsets": (N + 1,), "elem_nodes": (E, 3), "nlevels": (E,),
            "ulevels": (E,), "elem_area": (E,), "elem_cos": (E,), "gradient_sca": (E, 6),
            "edges": (Ed, 2), "edge_tri": (Ed, 2), "edge_dxdy": (Ed, 2),
            "edge_cross_dxdy": (Ed, 4), "edge_up_dn_tri": (Ed, 2), "Z": (nl - 1,),
        }
        for f, s in shapes.items():
            if getattr(self, f).shape != s:
                raise ValueError(f"mesh field {f}: shape {getattr(self, f).shape} != {s}")
        for f in ("nlevels_nod2D", "nlevels_nod2D_min", "ulevels_nod2D", "ulevels_nod2D_max"):
            if getattr(self, f).shape != (N,):
                raise ValueError(f"mesh field {f}: shape {getattr(self, f).shape} != ({N},)")
        if self.nod_in_elem2D.shape != (int(self.nod_in_elem2D_offsets[-1]),):
            raise ValueError("nod_in_elem2D length != offsets[-1]")
        if np.any(self.edges < 0) or np.any(self.edges >= N):
            raise ValueError("edges: node id out of range")
        if np.any(self.elem_nodes < 0) or np.any(self.elem_nodes >= N):
            raise ValueError("elem_nodes: node id out of range")
        for f in ("edge_tri", "edge_up_dn_tri"):
            a = getattr(self, f)
            if np.any(a < -1) or np.any(a >= E):
                raise ValueError(f"{f}: element id out of range")
        if np.any(self.edge_tri[:, 0] < 0):
            raise ValueError("edge_tri[:,0] must be a valid element")
        if np.any(self.nlevels_nod2D > nl) or np.any(self.nlevels > nl):
            raise ValueError("level count exceeds nl")
        if np.any(self.ulevels < 1) or np.any(self.ulevels_nod2D < 1):
            raise ValueError("ulevels must be >= 1")


def _read_meta_txt(path: Path) -> dict:
    out = {}
    for line in path.read_text().splitlines():
        line = line.strip()
        if line:
            k, v = line.split()
            out[k] = float(v)
    return out


def load_mesh(path: str | Path = PI_BUNDLE, *, name: str | None = None) -> Mesh:
    """Load a mesh from an ``.npz`` bundle or a reference-layout ``.npy`` directory."""
    path = Path(path)
    if path.is_dir():
        arrays = {f: np.load(path / f"{f}.npy") for f in FCT_FIELDS}
        meta = _read_meta_txt(path / "meta.txt")
        if int(meta["nl"]) != arrays["zbar"].shape[0]:
            raise ValueError("meta.txt nl disagrees with zbar")
    else:
        with np.load(path) as z:
            arrays = {f: z[f] for f in FCT_FIELDS}
    m = Mesh(**arrays, name=name or path.stem)
    m.validate()
    return m


def save_bundle(mesh: Mesh, path: str | Path) -> None:
    np.savez_compressed(path, **mesh.arrays())


def pi_mesh() -> Mesh:
    """The pi mesh (3140 nodes, 5839 elements, 8986 edges, nl=48)."""
    if not PI_BUNDLE.exists():
        raise FileNotFoundError(f"pi mesh bundle missing: {PI_BUNDLE}")
    return load_mesh(PI_BUNDLE, name="pi")
