"""Golden GRADIENTS of the FCT step, from the reference code itself.

JAX (and so ``jax.grad``) is not installed here. The reference's ``fesom_jax`` package is
imported with a torch-backed stand-in for the ``jax`` entry points it touches
(``jax.numpy`` -> torch ops, ``segment_sum`` -> ``index_add``, ``segment_max/min`` ->
``scatter_reduce`` amax/amin, ``lax.cumsum``), and the reference's unmodified
``tracer_adv.advect_one_fct`` and ``ale.compute_w`` run on float64 torch tensors with
autograd. torch's rules at ties match JAX's in the cases that occur here: ``maximum`` /
``minimum`` split the cotangent equally at a tie, ``amax``/``amin`` and ``scatter_reduce``
amax/amin spread it evenly over tied entries, and ``abs'(0) = 0``.

Cases (pi mesh, seeded inputs of ``fesom_jax_b200.inputs.make_fields``):
  * ``step``: one step, loss = sum(wts * T_new) with seeded N(0,1) weights on wet layers;
    gradients w.r.t. T, T_old, uv, w_e.
  * ``chain``: config-3 style loss = sum_n areasvol[n,0] * (T_K[n,0] - target_n)^2 after
    K = 4 FCT steps with ``w_e = compute_w(uv)`` inside the loss; gradients w.r.t. the
    initial T and uv (T_old = T at step 1).

    python tests/golden/make_grad_golden.py       # needs the reference checkout
"""

from __future__ import annotations

import sys
import tempfile
import textwrap
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

import make_golden as mg  # noqa: E402
from fesom_jax_b200 import inputs as I  # noqa: E402
from fesom_jax_b200.mesh import pi_mesh  # noqa: E402

DT = 3600.0
K_CHAIN = 4
SAMPLE = slice(0, None, 4)

_SHIM = {
    "__init__.py": """
        from . import numpy, lax, ops, tree_util
        import torch as _t
        Array = _t.Tensor
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
        import numpy as _np
        import torch as _t
        float64 = _t.float64
        int32 = _t.int32
        def _c(x):
            if isinstance(x, _t.Tensor):
                return x
            if isinstance(x, _np.ndarray):
                return _t.from_numpy(x)
            return _t.tensor(x, dtype=_t.float64 if isinstance(x, float) else None)
        def asarray(x, dtype=None):
            x = _c(x)
            return x.to(dtype) if dtype is not None else x
        def concatenate(xs, axis=0):
            return _t.cat([_c(x) for x in xs], dim=axis)
        def zeros_like(x):
            return _t.zeros_like(x)
        def zeros(shape, dtype=None):
            return _t.zeros(shape, dtype=dtype if dtype is not None else _t.float64)
        def where(c, a, b):
            return _t.where(_c(c), _c(a), _c(b))
        def abs(x):
            return _t.abs(x)
        def maximum(a, b):
            return _t.maximum(_c(a), _c(b))
        def minimum(a, b):
            return _t.minimum(_c(a), _c(b))
        def max(x, axis=None):
            return _t.amax(x, dim=axis)
        def min(x, axis=None):
            return _t.amin(x, dim=axis)
        def stack(xs, axis=0):
            return _t.stack([_c(x) for x in xs], dim=axis)
        def broadcast_to(x, shape):
            return _t.broadcast_to(_c(x), tuple(shape))
        def arange(n, dtype=None):
            return _t.arange(n, dtype=dtype if dtype is not None else _t.int64)
        def take_along_axis(x, idx, axis):
            return _t.take_along_dim(x, idx.long(), dim=axis)
    """,
    "ops.py": """
        import torch as _t
        def segment_sum(data, segment_ids, num_segments, **k):
            out = _t.zeros((num_segments,) + tuple(data.shape[1:]), dtype=data.dtype)
            return out.index_add(0, segment_ids.long(), data)
        def _seg(data, segment_ids, num_segments, red, init):
            idx = segment_ids.long().reshape((-1,) + (1,) * (data.ndim - 1)).expand(data.shape)
            out = _t.full((num_segments,) + tuple(data.shape[1:]), init, dtype=data.dtype)
            return out.scatter_reduce(0, idx, data, reduce=red, include_self=False)
        def segment_max(data, segment_ids, num_segments, **k):
            return _seg(data, segment_ids, num_segments, "amax", float("-inf"))
        def segment_min(data, segment_ids, num_segments, **k):
            return _seg(data, segment_ids, num_segments, "amin", float("inf"))
    """,
    "lax.py": """
        import torch as _t
        def cumsum(x, axis=0, reverse=False):
            if reverse:
                return _t.flip(_t.cumsum(_t.flip(x, [axis]), dim=axis), [axis])
            return _t.cumsum(x, dim=axis)
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


def import_reference_torch():
    shim = Path(tempfile.mkdtemp(prefix="jaxtorch_")) / "jax"
    shim.mkdir()
    for name, src in _SHIM.items():
        (shim / name).write_text(textwrap.dedent(src))
    sys.path.insert(0, str(shim.parent))
    sys.path.insert(1, str(mg.REF))
    import fesom_jax.ale as ale
    import fesom_jax.mesh as rmesh
    import fesom_jax.tracer_adv as ta
    return ta, ale, rmesh


SAMPLE_E = slice(0, None, 16)


def sample(m, g):
    """Every 4th node's full column of a node field (every 16th element's of an element
    field); plus [sum, sum|.|, sum g*w] digests over the whole field."""
    g = np.asarray(g)
    wts = np.random.default_rng(4321).normal(size=g.shape)
    sl = SAMPLE if g.shape[0] == m.nod2D else SAMPLE_E
    return g[sl], np.array([g.sum(), np.abs(g).sum(), (g * wts).sum()])


def main():
    import torch
    torch.set_default_dtype(torch.float64)
    ta, ale, rmesh = import_reference_torch()
    rm = rmesh.load_mesh(mg.REF / "fesom_jax/data/mesh_pi")
    m = pi_mesh()
    lm = m.node_layer_mask
    f = I.make_fields(m, seed=0, ab2=True)
    out = {}
    tt = lambda x: torch.tensor(np.asarray(x), dtype=torch.float64, requires_grad=True)  # noqa
    wts = np.where(lm, np.random.default_rng(99).normal(size=lm.shape), 0.0)

    # ---- single step
    T, To, uv, w = tt(f.tracers[0]), tt(f.tracers_old[0]), tt(f.uv), tt(f.w_e)
    Tn, _ = ta.advect_one_fct(rm, uv, w, torch.tensor(f.helem), torch.tensor(f.hnode),
                              torch.tensor(f.hnode_new), T, To, dt=DT)
    from oracle import fct_np
    Tn_np, _ = fct_np.advect_one_fct(m, f.uv, f.w_e, f.helem, f.hnode, f.hnode_new,
                                     f.tracers[0], f.tracers_old[0], dt=DT)
    print("torch-run reference vs numpy oracle, forward max|d| =",
          np.max(np.abs(Tn.detach().numpy() - Tn_np)), flush=True)
    loss = (torch.tensor(wts) * Tn).sum()
    loss.backward()
    for name, x in (("T", T), ("T_old", To), ("uv", uv), ("w_e", w)):
        s, d = sample(m, x.grad.numpy())
        out[f"step__g_{name}"], out[f"step__g_{name}_digest"] = s, d
    out["step__loss"] = np.array(loss.item())
    out["step__wts_seed"] = np.array(99)
    print("step: loss", loss.item(), "max|gT|", T.grad.abs().max().item(),
          "max|guv|", uv.grad.abs().max().item(), flush=True)

    # ---- multi-step chain with w = compute_w(uv) inside the loss
    target = np.random.default_rng(7).normal(20.0, 2.0, m.nod2D)
    T0, uv = tt(f.tracers[0]), tt(f.uv)
    helem = torch.tensor(f.helem)
    w = ale.compute_w(rm, uv, helem)
    Tc, Tp = T0, T0
    for _ in range(K_CHAIN):
        Tc, Tp = ta.advect_one_fct(rm, uv, w, helem, torch.tensor(f.hnode),
                                   torch.tensor(f.hnode_new), Tc, Tp, dt=DT)
    av0 = torch.tensor(m.areasvol[:, 0])
    loss = (av0 * (Tc[:, 0] - torch.tensor(target)) ** 2).sum()
    loss.backward()
    for name, x in (("T", T0), ("uv", uv)):
        s, d = sample(m, x.grad.numpy())
        out[f"chain__g_{name}"], out[f"chain__g_{name}_digest"] = s, d
    out["chain__loss"] = np.array(loss.item())
    out["chain__K"] = np.array(K_CHAIN)
    print("chain: loss", loss.item(), "max|gT0|", T0.grad.abs().max().item(),
          "max|guv|", uv.grad.abs().max().item(), flush=True)
    np.savez_compressed(HERE / "fct_pi_grad_golden.npz", **out)
    print("wrote", HERE / "fct_pi_grad_golden.npz", (HERE / "fct_pi_grad_golden.npz").stat().st_size)


if __name__ == "__main__":
    main()
