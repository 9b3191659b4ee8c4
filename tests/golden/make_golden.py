"""Generate the golden FCT vectors from the reference code itself.

JAX is not installed here, so the reference's ``fesom_jax`` package is imported with a
minimal numpy-backed stand-in for the handful of ``jax`` entry points it touches
(``jax.numpy`` -> numpy, ``jax.ops.segment_{sum,max,min}`` -> ``np.{add,maximum,minimum}.at``,
``jax.lax.{cumsum,scan}``, ``jax.tree_util.register_dataclass`` -> identity). The
reference's own functions then run unmodified on numpy arrays:

  * ``fesom_jax.tracer_adv.advect_one_fct`` (tracer_adv.py:532-578) -- the primary golden;
  * ``fesom_jax.ale.compute_w`` (ale.py:309-365) -- pins the ``w`` producer;
  * ``_fct_ref`` of fesom_jax/tests/test_tracers.py:325-516 (the reference's own
    loop-based cross-check, extracted from the test file's AST) -- a second opinion.

Inputs are the seeded pi-mesh fields of ``fesom_jax_b200.inputs.make_fields``; the
fixture stores digests of those inputs so a drift in input generation is detected.

    python tests/golden/make_golden.py            # needs the reference checkout
"""

from __future__ import annotations

import ast
import hashlib
import os
import sys
import tempfile
import textwrap
from pathlib import Path

import numpy as np

# the reference checkout (koldunovn/fesom_jax): the FESOM_JAX_REFERENCE environment
# variable, else a ``reference`` directory beside this repository
REF = Path(os.environ.get("FESOM_JAX_REFERENCE",
                          str(Path(__file__).resolve().parents[3] / "reference")))
HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

from fesom_jax_b200 import inputs as I  # noqa: E402
from fesom_jax_b200.mesh import pi_mesh  # noqa: E402

DT = 3600.0

_SHIM = {
    "__init__.py": """
        from . import numpy, lax, ops, tree_util
        import numpy as _np
        Array = _np.ndarray
        class _Cfg:
            def update(self, *a, **k):
                pass
        config = _Cfg()
        def jit(f=None, **k):
            return f if f is not None else (lambda g: g)
        def checkpoint(f=None, **k):
            return f if f is not None else (lambda g: g)
    """,
    "numpy.py": """
        from numpy import *
        import numpy as _np
        max = _np.max
        min = _np.min
        abs = _np.abs
    """,
    "ops.py": """
        import numpy as _np
        def segment_sum(data, segment_ids, num_segments, **k):
            data = _np.asarray(data)
            out = _np.zeros((num_segments,) + data.shape[1:], data.dtype)
            _np.add.at(out, _np.asarray(segment_ids), data)
            return out
        def segment_max(data, segment_ids, num_segments, **k):
            data = _np.asarray(data)
            out = _np.full((num_segments,) + data.shape[1:], -_np.inf)
            _np.maximum.at(out, _np.asarray(segment_ids), data)
            return out
        def segment_min(data, segment_ids, num_segments, **k):
            data = _np.asarray(data)
            out = _np.full((num_segments,) + data.shape[1:], _np.inf)
            _np.minimum.at(out, _np.asarray(segment_ids), data)
            return out
    """,
    "lax.py": """
        import numpy as _np
        def cumsum(x, axis=0, reverse=False):
            x = _np.asarray(x)
            if reverse:
                return _np.flip(_np.cumsum(_np.flip(x, axis), axis=axis), axis)
            return _np.cumsum(x, axis=axis)
        def scan(f, init, xs, reverse=False, length=None):
            leaves = xs if isinstance(xs, tuple) else (xs,)
            n = leaves[0].shape[0]
            order = range(n - 1, -1, -1) if reverse else range(n)
            carry, ys = init, [None] * n
            for i in order:
                x = tuple(l[i] for l in leaves) if isinstance(xs, tuple) else xs[i]
                carry, y = f(carry, x)
                ys[i] = y
            if isinstance(ys[0], tuple):
                return carry, tuple(_np.stack([y[j] for y in ys]) for j in range(len(ys[0])))
            return carry, _np.stack(ys)
        def optimization_barrier(x):
            return x
    """,
    "tree_util.py": """
        def register_dataclass(cls, data_fields=None, meta_fields=None):
            return cls
        def register_pytree_node(*a, **k):
            return None
    """,
}


def import_reference():
    shim = Path(tempfile.mkdtemp(prefix="jaxshim_")) / "jax"
    shim.mkdir()
    for name, src in _SHIM.items():
        (shim / name).write_text(textwrap.dedent(src))
    sys.path.insert(0, str(shim.parent))
    sys.path.insert(1, str(REF))
    import fesom_jax.ale as ale
    import fesom_jax.mesh as rmesh
    import fesom_jax.tracer_adv as ta
    return ta, ale, rmesh


def extract_fct_ref():
    """Compile ``_fct_ref`` (and its module constants) out of the reference test file."""
    path = REF / "fesom_jax/tests/test_tracers.py"
    tree = ast.parse(path.read_text())
    keep = []
    for node in tree.body:
        if isinstance(node, ast.FunctionDef) and node.name == "_fct_ref":
            keep.append(node)
        elif isinstance(node, ast.Assign):
            names = [t.id for t in ast.walk(node.targets[0]) if isinstance(t, ast.Name)]
            if any(n in ("_AB_OLD", "_AB_NEW", "_FLUX_EPS", "_BIG") for n in names):
                keep.append(node)
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {"np": np}
    exec(compile(mod, str(path), "exec"), ns)
    return ns["_fct_ref"]


SAMPLE = slice(0, None, 4)   # every 4th node column is stored in full


def field_digest(m, x, mask=None):
    """``[sum x, sum wts*x, sum |wts*x|, sum x^2]`` over wet lanes; ``wts`` are fixed
    seeded N(0,1) weights, so the digest pins every lane, not only the stored ones."""
    mask = m.node_layer_mask if mask is None else mask
    wts = np.random.default_rng(1234).normal(size=mask.shape)
    xm = np.where(mask, x, 0.0)
    return np.array([xm.sum(), (wts * xm).sum(), np.abs(wts * xm).sum(), (xm * xm).sum()])


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main():
    ta, ale, rmesh = import_reference()
    fct_ref = extract_fct_ref()
    rm = rmesh.load_mesh(REF / "fesom_jax/data/mesh_pi")
    m = pi_mesh()
    lm = m.node_layer_mask
    out = {}

    f = I.make_fields(m, seed=0)
    f_ab2 = I.make_fields(m, seed=0, ab2=True)
    f_white = I.make_fields(m, seed=0, kind="white")
    w_ref = np.asarray(ale.compute_w(rm, f.uv, f.helem))
    out["w_e__digest"] = field_digest(m, w_ref, m.node_iface_mask)
    print("compute_w  ours vs reference max|d| =", np.max(np.abs(w_ref - f.w_e)))

    k = np.arange(m.nl)[None, :]
    sharp = np.where(lm, 10.0 + 5.0 * np.sin(np.arange(m.nod2D)[:, None] * 0.7)
                     * np.cos(k * 1.3), 0.0)
    ten = np.where(lm, 10.0, 0.0)
    const = np.where(lm, 20.0, 0.0)
    # split w (w_split) and live zstar depths for the optional-argument cases
    zbar3 = np.broadcast_to(m.zbar, (m.nod2D, m.nl)).copy()
    zbar3[:, 1:] *= 1.0 + 0.01 * np.sin(np.arange(m.nod2D))[:, None]
    Z3d = np.concatenate([0.5 * (zbar3[:, :-1] + zbar3[:, 1:]), 0.5 * (zbar3[:, -2:-1] + zbar3[:, -1:])], axis=1)
    w_i = 0.3 * f.w_e

    cases = {
        # name: (uv, w, T, T_old, kwargs, run _fct_ref)
        "T_step1": (f.uv, f.w_e, f.tracers[0], f.tracers_old[0], {}, True),
        "S_step1": (f.uv, f.w_e, f.tracers[1], f.tracers_old[1], {}, True),
        "T_ab2": (f_ab2.uv, f_ab2.w_e, f_ab2.tracers[0], f_ab2.tracers_old[0], {}, True),
        "sharp_x5": (f_white.uv * 5.0, f_white.w_e * 5.0, sharp, ten, {}, True),
        "const": (f.uv, f.w_e, const, const, {}, False),
        "T_wsplit_zstar": (f.uv, f.w_e - w_i, f.tracers[0], f_ab2.tracers_old[0],
                           dict(w_i=w_i, Z3d=Z3d, zbar3=zbar3), False),
    }
    meta = []
    for name, (uv, w, T, To, kw, run_loop) in cases.items():
        Tn, Told_new = ta.advect_one_fct(rm, uv, w, f.helem, f.hnode, f.hnode_new, T, To,
                                         dt=DT, **kw)
        Tn = np.asarray(Tn)
        assert Told_new is T
        out[f"{name}__T_new"] = Tn[SAMPLE][lm[SAMPLE]]
        out[f"{name}__digest"] = field_digest(m, Tn)
        out[f"{name}__in_digest"] = np.frombuffer(
            bytes.fromhex(digest(uv, w, T, To, *kw.values())), np.uint8)
        msg = f"{name}: max|T_new-T|={np.max(np.abs(Tn - T)[lm]):.3e}"
        if run_loop:
            Tl = fct_ref(rm, uv, w, f.helem, f.hnode, f.hnode_new, T, To, DT)
            out[f"{name}__loopref_maxdiff"] = np.array(np.max(np.abs(Tn - Tl)[lm]))
            msg += f"  tracer_adv vs _fct_ref max|d|={np.max(np.abs(Tn - Tl)[lm]):.3e}"
        print(msg, flush=True)
        meta.append(name)
    out["cases"] = np.array(meta)
    np.savez_compressed(HERE / "fct_pi_golden.npz", **out)
    print("wrote", HERE / "fct_pi_golden.npz", (HERE / "fct_pi_golden.npz").stat().st_size)


if __name__ == "__main__":
    main()
