"""ctypes binding of ``libfesom_fct.so`` (the C ABI in ``include/fesom_fct.h``).

Loading fails loudly when the library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libfesom_fct.so"

FCT_OK = 0
STATUS_NAMES = {0: "FCT_OK", -1: "FCT_ERR_INVALID", -2: "FCT_ERR_CUDA",
                -3: "FCT_ERR_CAPACITY", -4: "FCT_ERR_UNSUPPORTED", -5: "FCT_ERR_NONFINITE"}

i32p = C.POINTER(C.c_int32)
f64p = C.POINTER(C.c_double)


class FctMeshDesc(C.Structure):
    _fields_ = [
        ("nod2D", C.c_int32), ("elem2D", C.c_int32), ("edge2D", C.c_int32), ("nl", C.c_int32),
        ("edges", i32p), ("edge_tri", i32p), ("edge_up_dn_tri", i32p),
        ("edge_cross_dxdy", f64p), ("edge_dxdy", f64p),
        ("elem_nodes", i32p), ("gradient_sca", f64p), ("elem_cos", f64p), ("elem_area", f64p),
        ("nlevels", i32p), ("ulevels", i32p),
        ("nlevels_nod2D", i32p), ("nlevels_nod2D_min", i32p), ("ulevels_nod2D", i32p),
        ("ulevels_nod2D_max", i32p), ("nod_in_elem2D_offsets", i32p), ("nod_in_elem2D", i32p),
        ("area", f64p), ("areasvol", f64p), ("Z", f64p), ("zbar", f64p),
    ]


class FctFields(C.Structure):
    _fields_ = [
        ("uv", C.c_void_p), ("w_e", C.c_void_p), ("helem", C.c_void_p), ("hnode", C.c_void_p),
        ("hnode_new", C.c_void_p), ("T", C.c_void_p), ("T_old", C.c_void_p),
        ("T_new", C.c_void_p), ("tracer_stride", C.c_int64),
        ("Z3d", C.c_void_p), ("zbar3", C.c_void_p), ("w_i", C.c_void_p),
    ]


FCT_ERR_NONFINITE = -5


def health_status(status: int) -> None:
    """Raise for a failed health call; FCT_ERR_NONFINITE is a result, not a failure."""
    if status not in (FCT_OK, FCT_ERR_NONFINITE):
        check(status)


class FctError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def lib() -> C.CDLL:
    """The loaded library (raises ``ImportError`` when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    # FESOM_FCT_LIB: load another build of the same library (e.g. for A/B timing)
    path = Path(os.environ.get("FESOM_FCT_LIB", str(LIB_PATH)))
    if not path.exists():
        raise ImportError(f"{path} is missing: build it with `python -m fesom_jax_b200.build` "
                          "(the FCT path has no CPU fallback)")
    L = C.CDLL(str(path))
    L.fct_last_error.restype = C.c_char_p
    L.fct_version.restype = C.c_char_p
    L.fct_plan_create.argtypes = [C.POINTER(FctMeshDesc), C.c_int, C.c_int, C.POINTER(C.c_void_p)]
    L.fct_plan_destroy.argtypes = [C.c_void_p]
    L.fct_plan_reserve.argtypes = [C.c_void_p, C.c_int]
    L.fct_plan_info.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
    L.fct_plan_set_fused.argtypes = [C.c_void_p, C.c_int]
    L.fct_forward.argtypes = [C.c_void_p, C.POINTER(FctFields), C.c_double, C.c_int, C.c_void_p]
    L.fct_compute_w.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.fct_plan_health.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
    for name in ("fct_plan_create", "fct_plan_destroy", "fct_plan_reserve", "fct_plan_info",
                 "fct_plan_set_fused", "fct_forward", "fct_compute_w", "fct_plan_health"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(status: int) -> None:
    if status != FCT_OK:
        raise FctError(status, lib().fct_last_error().decode())


def mesh_desc(mesh, keep: list) -> FctMeshDesc:
    """Fill an ``FctMeshDesc`` from a ``Mesh``; ``keep`` holds the arrays alive."""
    d = FctMeshDesc()
    d.nod2D, d.elem2D, d.edge2D, d.nl = mesh.nod2D, mesh.elem2D, mesh.edge2D, mesh.nl
    for name, ctype in FctMeshDesc._fields_[4:]:
        arr = getattr(mesh, name)
        arr = np.ascontiguousarray(arr, dtype=np.int32 if ctype is i32p else np.float64)
        keep.append(arr)
        setattr(d, name, arr.ctypes.data_as(ctype))
    return d
