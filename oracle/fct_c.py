"""ctypes binding of the C oracle (``oracle/liboracle_fct.so``); test infrastructure only."""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SO = HERE / "liboracle_fct.so"
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not SO.exists() or SO.stat().st_mtime < (HERE / "fct_ref.c").stat().st_mtime:
            subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
        L = C.CDLL(str(SO))
        L.oracle_fct_forward.restype = C.c_int
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _p(x):
    if x is None:
        return None
    return np.ascontiguousarray(x, dtype=np.float64).ctypes.data_as(C.POINTER(C.c_double))


def advect_one_fct(mesh, uv, w_e, helem, hnode, hnode_new, T, T_old, *, dt,
                   Z3d=None, zbar3=None, w_i=None, threads: int = 0, desc=None):
    """One tracer FCT step through the C oracle; ``threads=0`` uses all OpenMP threads."""
    from fesom_jax_b200 import _lib as fl   # only for the FctMeshDesc struct layout
    keep = []
    d = desc if desc is not None else fl.mesh_desc(mesh, keep)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
            (uv, w_e, helem, hnode, hnode_new, T, T_old)]
    opt = [None if a is None else np.ascontiguousarray(a, dtype=np.float64)
           for a in (Z3d, zbar3, w_i)]
    out = np.empty_like(arrs[5])
    st = lib().oracle_fct_forward(C.byref(d), *[_p(a) for a in arrs], _p(out),
                                  C.c_double(dt), *[_p(a) for a in opt], C.c_int(threads))
    if st != 0:
        raise MemoryError("oracle_fct_forward failed")
    return out, T


def max_threads() -> int:
    return int(lib().oracle_max_threads())
