"""The C-ABI library loads and exports every function ``include/*.h`` declares (CPU)."""

import ctypes
import re
from pathlib import Path

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
