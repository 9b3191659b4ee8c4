"""Build ``libfesom_fct.so`` (the CUDA kernels + C ABI) in-tree for sm_100a.

    python -m fesom_jax_b200.build          # or __graft_entry__.build()

The library is compiled with nvcc directly (no torch extension): it exposes only the
plain C ABI declared in ``include/fesom_fct.h`` and links the CUDA runtime statically.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libfesom_fct.so"
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    deps += list((PKG.parent / "include").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, extra=()) -> Path:
    """Compile every ``csrc/*.cu`` to an object (in parallel), then link the library."""
    if not force and not needs_build():
        return LIB
    import tempfile
    from concurrent.futures import ThreadPoolExecutor
    tmp = LIB.with_suffix(".so.tmp")
    # --fmad=false: no implicit FMA contraction, so every template instantiation (tracer
    # chunk size, layout) rounds identically and results do not depend on the chunking;
    # the kernels state their fused multiply-adds explicitly where they want them
    common = [ARCH, "-O3", "-lineinfo", "-std=c++17", "--fmad=false",
              "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
              "-I", str(PKG.parent / "include"), *extra]
    with tempfile.TemporaryDirectory() as td:
        objs = [Path(td) / (s.stem + ".o") for s in sources()]

        def compile_one(so):
            src, obj = so
            cmd = [nvcc(), *common, "-c", str(src), "-o", str(obj)]
            return cmd, subprocess.run(cmd, capture_output=True, text=True)

        with ThreadPoolExecutor(max_workers=max(1, min(len(objs), os.cpu_count() or 1))) as ex:
            results = list(ex.map(compile_one, zip(sources(), objs)))
        for cmd, r in results:
            if verbose:
                print(" ".join(cmd), flush=True)
            if r.returncode != 0:
                sys.stderr.write(r.stdout + r.stderr)
                raise RuntimeError("nvcc failed building libfesom_fct.so")
            if verbose and (r.stdout or r.stderr):
                sys.stderr.write(r.stdout + r.stderr)
        link = [nvcc(), ARCH, "-shared", "-cudart", "static", *map(str, objs), "-o", str(tmp)]
        r = subprocess.run(link, capture_output=True, text=True)
        if verbose:
            print(" ".join(link), flush=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed linking libfesom_fct.so")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=("-Xptxas", "-v") if "--ptxas" in sys.argv else ())
    print(LIB)
