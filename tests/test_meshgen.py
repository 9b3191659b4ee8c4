"""Synthetic meshes: geometry pinned to the reference's own derivation (CPU)."""

import hashlib

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from fesom_jax_b200 import meshgen
from fesom_jax_b200.mesh import FCT_FIELDS, Mesh, pi_mesh
from oracle import fct_np
from tests.golden.make_mesh_golden_params import DT, N_NODES, SEED

GOLDEN = "tests/golden/fct_small_mesh_golden.npz"


def _sha(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.digest()


@pytest.fixture(scope="module")
def small():
    g = dict(np.load(GOLDEN))
    raw = meshgen.generate_raw(N_NODES, pi_mesh().zbar, seed=SEED)
    assert _sha(raw["nodes_deg"], raw["elem_nodes"], raw["edges"], raw["edge_tri"],
                raw["nlevels"], raw["nlevels_nod2D"]) == g["raw_digest"].tobytes()
    der = meshgen.derive(raw)
    return g, der, Mesh(**der, name="small")


def test_derive_bit_identical_to_reference(small):
    g, der, _ = small
    for f in FCT_FIELDS:
        a = np.asarray(der[f])
        a = a.astype(np.int32 if a.dtype.kind in "iu" else np.float64)
        assert _sha(a) == g[f"mesh__{f}"].tobytes(), f


def test_mesh_has_coasts_and_cw(small):
    _, _, m = small
    assert np.any(m.edge_tri[:, 1] < 0) and np.any(m.edge_up_dn_tri < 0)
    assert np.all(m.edge_tri[np.flatnonzero(m.edge_tri[:, 1] >= 0), 1] >= 0)
    r, en = m.coord_nod2D, m.elem_nodes
    bx = meshgen._trim(r[en[:, 1], 0] - r[en[:, 0], 0]); by = r[en[:, 1], 1] - r[en[:, 0], 1]
    cx = meshgen._trim(r[en[:, 2], 0] - r[en[:, 0], 0]); cy = r[en[:, 2], 1] - r[en[:, 0], 1]
    assert np.all(bx * cy - by * cx < 0)


def test_numpy_oracle_on_small_mesh_matches_reference(small):
    g, _, m = small
    f = I.make_fields(m, seed=SEED, n_passive=1, ab2=True)
    assert _sha(f.uv, f.w_e, f.tracers, f.tracers_old) == g["in_digest"].tobytes()
    for t, name in enumerate(["T", "S", "P"]):
        T_new, _ = fct_np.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                         f.tracers[t], f.tracers_old[t], dt=DT)
        ref = g[f"{name}__T_new"]
        got = T_new[m.node_layer_mask]
        assert np.max(np.abs(got - ref)) / np.max(np.abs(ref)) < 1e-13


def test_stretched_zbar():
    z = meshgen.stretched_zbar(70)
    assert z.shape == (70,) and z[0] == 0.0 and abs(z[-1] + 6000.0) < 1e-6
    dz = -np.diff(z)
    assert np.all(dz > 0) and np.all(np.diff(dz) > 0) and abs(dz[0] - 5.0) < 0.5


def test_node_orders_renumber_the_same_mesh():
    """rcm, raw and random orders number the same ocean: the same counts and wet layers, a
    valid mesh each, local neighbours for rcm and the Fibonacci order, not for a shuffle."""
    import numpy as np
    from fesom_jax_b200.meshgen import make_mesh
    spans = {}
    meshes = {}
    for order in ("rcm", "raw", "random"):
        m = make_mesh(3000, nl=12, seed=4, bottom=(4, None), node_order=order)
        meshes[order] = m
        spans[order] = float(np.median(np.abs(m.edges[:, 0] - m.edges[:, 1])))
    counts = {(m.nod2D, m.elem2D, m.edge2D, m.n_wet_layers) for m in meshes.values()}
    assert len(counts) == 1
    assert spans["rcm"] < 0.1 * spans["random"] and spans["raw"] < 0.1 * spans["random"]
    with pytest.raises(ValueError, match="node_order"):
        make_mesh(300, nl=12, seed=4, node_order="hilbert")
