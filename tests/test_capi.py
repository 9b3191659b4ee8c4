"""The C-ABI library loads and exports every function ``include/*.h`` declares (CPU)."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(fct_\w+)\s*\(", text, re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for required in ("fct_plan_create", "fct_plan_destroy", "fct_forward", "fct_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    from fesom_jax_b200 import _lib
    lib = _lib.lib()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    assert b"sm_100a" in lib.fct_version()


def test_plan_create_rejects_bad_mesh(pi):
    """Validation runs on the host before any CUDA call (no GPU needed)."""
    from fesom_jax_b200 import _lib
    keep = []
    desc = _lib.mesh_desc(pi, keep)
    bad = keep[[f for f, _ in _lib.FctMeshDesc._fields_[4:]].index("edges")].copy()
    bad[0, 0] = pi.nod2D + 5
    desc.edges = bad.ctypes.data_as(_lib.i32p)
    h = ctypes.c_void_p()
    st = _lib.lib().fct_plan_create(ctypes.byref(desc), 0, 1, ctypes.byref(h))
    assert st == -1 and b"out of range" in _lib.lib().fct_last_error()


def _desc_with(pi, keep, field, mutate):
    from fesom_jax_b200 import _lib
    desc = _lib.mesh_desc(pi, keep)
    names = [f for f, _ in _lib.FctMeshDesc._fields_[4:]]
    arr = keep[names.index(field)].copy()
    mutate(arr)
    keep.append(arr)
    ptype = _lib.i32p if arr.dtype == np.int32 else _lib.f64p
    setattr(desc, field, arr.ctypes.data_as(ptype))
    return desc


@pytest.mark.parametrize("field,mutate,msg", [
    ("elem_nodes", lambda a: a.__setitem__((3, 1), -1), b"elem_nodes"),
    ("edge_tri", lambda a: a.__setitem__((2, 0), -1), b"edge_tri"),
    ("nlevels", lambda a: a.__setitem__(5, 1000), b"level range"),
    ("ulevels_nod2D", lambda a: a.__setitem__(7, 0), b"level range"),
    ("nod_in_elem2D", lambda a: a.__setitem__(0, a[-1]), b"not one of its vertices"),
])
def test_plan_create_rejects_inconsistent_arrays(pi, field, mutate, msg):
    """Host-side validation (before any CUDA call): indices in range, level ranges
    consistent, node->element lists naming cells that contain the node."""
    from fesom_jax_b200 import _lib
    keep = []
    desc = _desc_with(pi, keep, field, mutate)
    h = ctypes.c_void_p()
    st = _lib.lib().fct_plan_create(ctypes.byref(desc), 0, 1, ctypes.byref(h))
    assert st == -1 and msg in _lib.lib().fct_last_error(), _lib.lib().fct_last_error()


def test_plan_create_rejects_too_many_levels(pi):
    from fesom_jax_b200 import _lib
    keep = []
    desc = _lib.mesh_desc(pi, keep)
    desc.nl = 129
    h = ctypes.c_void_p()
    st = _lib.lib().fct_plan_create(ctypes.byref(desc), 0, 1, ctypes.byref(h))
    assert st == -1 and b"nl=129" in _lib.lib().fct_last_error()


def _header_define(name):
    text = (ROOT / "include" / "fesom_fct.h").read_text()
    m = re.search(r"^#define\s+" + name + r"\s+(\d+)", text, re.M)
    assert m, name
    return int(m.group(1))


def test_xla_opaque_and_buffer_layout_agree_with_the_header():
    """The custom-call opaque struct (uint64 plan, double dt, int32 ntr, int32 flags) is 24
    bytes in the header, in fesom_jax_b200.xla and in the struct.pack format a JAX binding
    uses; the status result indices and flags match the header's."""
    import struct
    from fesom_jax_b200 import xla
    assert ctypes.sizeof(xla.FctXlaOpaque) == 24 == struct.calcsize("<Qdii")
    o = xla.FctXlaOpaque(0x1234, 1800.0, 3, xla.Z3D | xla.WI)
    assert bytes(memoryview(o)) == struct.pack("<Qdii", 0x1234, 1800.0, 3, 3)
    assert xla.FWD_STATUS == _header_define("FCT_XLA_FWD_STATUS") == 11
    assert xla.ADJ_STATUS == _header_define("FCT_XLA_ADJ_STATUS") == 14
    assert (xla.Z3D, xla.WI) == (_header_define("FCT_XLA_Z3D"), _header_define("FCT_XLA_WI"))


def test_adjoint_accumulate_bits_agree_with_the_header():
    from fesom_jax_b200.adjoint import ACC_T, ACC_T_OLD, ACC_UV, ACC_W, DEFER_UV
    assert (ACC_T, ACC_T_OLD, ACC_UV, ACC_W, DEFER_UV) == tuple(
        _header_define(n) for n in ("FCT_ACC_T", "FCT_ACC_T_OLD", "FCT_ACC_UV", "FCT_ACC_W",
                                    "FCT_ADJ_DEFER_UV"))


def test_plan_create_rejects_nodes_of_more_than_255_cells():
    """A node's lane record packs its edge and cell counts in 8 bits each: a fan of 300
    triangles around one node is refused on the host, before any CUDA call."""
    from fesom_jax_b200 import _lib
    from fesom_jax_b200.mesh import Mesh
    from fesom_jax_b200.meshgen import _edges_from_triangles, derive, stretched_zbar
    k = 300
    ang = np.linspace(0.0, 2.0 * np.pi, k, endpoint=False)
    nodes = np.concatenate([[[10.0, 0.0]], np.stack([10.0 + np.cos(ang), np.sin(ang)], 1)])
    tri = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int64)
    zbar = stretched_zbar(6)
    edges, edge_tri = _edges_from_triangles(tri, np.radians(nodes[:, 0]), np.radians(nodes[:, 1]))
    raw = dict(nodes_deg=nodes, elem_nodes=tri.astype(np.int32), nl=6, zbar=zbar,
               depth=np.full(k + 1, -zbar[-1]), nlevels_nod2D=np.full(k + 1, 6, np.int32),
               nlevels=np.full(k, 6, np.int32), edges=edges, edge_tri=edge_tri, nod2D=k + 1,
               elem2D=k, coast=np.zeros(k + 1, np.int32))
    m = Mesh(**derive(raw), name="fan")
    m.validate()
    keep = []
    desc = _lib.mesh_desc(m, keep)
    plan = ctypes.c_void_p()
    st = _lib.lib().fct_plan_create(ctypes.byref(desc), 0, 1, ctypes.byref(plan))
    assert st == -1 and not plan.value
    assert b"more than 255" in _lib.lib().fct_last_error()


def test_plan_create_rejects_nodes_of_more_than_24_edges():
    """The segment kernels keep one flag bit per edge slot of a node layer: a fan of 30
    triangles (a node with 30 edges) is refused on the host, before any CUDA call."""
    from fesom_jax_b200 import _lib
    from fesom_jax_b200.mesh import Mesh
    from fesom_jax_b200.meshgen import _edges_from_triangles, derive, stretched_zbar
    k = 30
    ang = np.linspace(0.0, 2.0 * np.pi, k, endpoint=False)
    nodes = np.concatenate([[[10.0, 0.0]], np.stack([10.0 + np.cos(ang), np.sin(ang)], 1)])
    tri = np.array([[0, 1 + i, 1 + (i + 1) % k] for i in range(k)], np.int64)
    zbar = stretched_zbar(6)
    edges, edge_tri = _edges_from_triangles(tri, np.radians(nodes[:, 0]), np.radians(nodes[:, 1]))
    raw = dict(nodes_deg=nodes, elem_nodes=tri.astype(np.int32), nl=6, zbar=zbar,
               depth=np.full(k + 1, -zbar[-1]), nlevels_nod2D=np.full(k + 1, 6, np.int32),
               nlevels=np.full(k, 6, np.int32), edges=edges, edge_tri=edge_tri, nod2D=k + 1,
               elem2D=k, coast=np.zeros(k + 1, np.int32))
    m = Mesh(**derive(raw), name="fan30")
    m.validate()
    keep = []
    desc = _lib.mesh_desc(m, keep)
    plan = ctypes.c_void_p()
    st = _lib.lib().fct_plan_create(ctypes.byref(desc), 0, 1, ctypes.byref(plan))
    assert st == -1 and not plan.value
    assert b"at most 24" in _lib.lib().fct_last_error()
