"""Persistent cache of autotuned thread mappings, per (GPU model, mesh, workload shape).

The autotuners (:meth:`fesom_jax_b200.ensemble.Ensemble.autotune`,
:meth:`fesom_jax_b200.tracer_adv.FctPlan.autotune`) time every candidate mapping of the
fused stages, which takes seconds on a large batch. With a cache they time once per GPU
model, mesh and workload shape, store the choice in a JSON file and apply it directly on
later runs. The mapping only changes speed, never results, so a stale entry costs time,
not correctness.

Default location: ``$FESOM_FCT_TUNING_CACHE``, else
``~/.cache/fesom_jax_b200/tuning.json``.
"""

from __future__ import annotations

import hashlib
import json
import os
import tempfile
from pathlib import Path

import numpy as np


def default_path() -> Path:
    env = os.environ.get("FESOM_FCT_TUNING_CACHE")
    if env:
        return Path(env)
    return Path.home() / ".cache" / "fesom_jax_b200" / "tuning.json"


def mesh_fingerprint(mesh) -> str:
    """A short digest of the mesh's shape, connectivity and level structure: the inputs
    that decide the kernels' segment lists and gathers."""
    h = hashlib.sha1()
    h.update(np.asarray([mesh.nod2D, mesh.elem2D, mesh.edge2D, mesh.nl], np.int64).tobytes())
    for name in ("edges", "elem_nodes", "nlevels_nod2D", "ulevels_nod2D", "nlevels", "ulevels"):
        a = getattr(mesh, name, None)
        if a is not None:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def gpu_name(device: int = 0) -> str:
    import torch
    return torch.cuda.get_device_name(device)


def key(kind: str, gpu: str, meshes, **shape) -> str:
    """Cache key: the tuner (``kind``), the GPU model, the mesh fingerprints and the
    workload shape (tracers, members, ...), in a stable order."""
    fp = ",".join(sorted(mesh_fingerprint(m) for m in meshes))
    sh = ",".join(f"{k}={shape[k]}" for k in sorted(shape))
    return f"{kind}|{gpu}|{fp}|{sh}"


class TuningCache:
    """A JSON file of ``{key: value}`` entries; writes go through a temporary file and a
    rename, so a reader never sees a half-written file."""

    def __init__(self, path=None):
        self.path = Path(path) if path is not None else default_path()

    def _load(self) -> dict:
        try:
            return json.loads(self.path.read_text())
        except (FileNotFoundError, json.JSONDecodeError):
            return {}

    def get(self, k: str):
        return self._load().get(k)

    def put(self, k: str, value) -> None:
        d = self._load()
        d[k] = value
        self.path.parent.mkdir(parents=True, exist_ok=True)
        fd, tmp = tempfile.mkstemp(dir=str(self.path.parent), suffix=".tmp")
        with os.fdopen(fd, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)
