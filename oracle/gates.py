"""Per-step correctness gates of the FCT step, computed from the numpy oracle's
intermediates (test infrastructure: the checker of the CUDA results, never measured).

* budget closure: ``sum(areasvol * (hnode_new * T_new - hnode * T))`` equals ``dt`` times
  the sum over nodes of the surface fluxes (LO vertical flux + limited antidiffusive
  vertical flux at ``nzmin``): horizontal fluxes cancel edge by edge and interior vertical
  fluxes telescope (fesom_jax/tracer_adv.py:298-313, 469-484), so a step changes the
  tracer content only through the surface;
* monotonicity against the Zalesak window (fesom_jax/tracer_adv.py:389-418): every
  updated lane stays inside ``[window_min, window_max]`` with a slack of 4 ulp (16 for the
  CUDA path's results, GPU_WINDOW_ULPS) of the largest magnitude the update combines (the
  bound, T and LO): ``T_new = T + ((LO * hnode_new - T * hnode) + fluxes + T * (hnode -
  hnode_new)) / hnode_new`` cancels T against LO-sized terms, so its rounding is relative
  to those.
"""

from __future__ import annotations

import numpy as np

from . import fct_np


def closure_residual(m, T, hnode, hnode_new, T_new, inter, dt: float) -> float:
    """|content change - dt x surface fluxes| relative to the content sum |areasvol*hnode*T|."""
    lm = m.node_layer_mask
    av = m.areasvol
    content = np.where(lm, av * hnode * T, 0.0)
    lhs = np.sum(np.where(lm, av * hnode_new * T_new, 0.0)) - np.sum(content)
    n = np.arange(m.nod2D)
    top = m.ulevels_nod2D - 1
    rhs = dt * np.sum(inter["flux_v_lo"][n, top] + inter["adf_v_lim"][n, top])
    return float(abs(lhs - rhs) / np.sum(np.abs(content)))


def window(m, inter):
    """The limiter's admissible window per node-layer (a4, tracer_adv.py:407-418)."""
    k = np.arange(m.nl)[None, :]
    nzmin = (m.ulevels_nod2D - 1)[:, None]
    nzmax = (m.nlevels_nod2D - 1)[:, None]
    own = (k == nzmin) | (k == nzmax - 1)
    tv_max, tv_min = inter["tvert_max"], inter["tvert_min"]
    w_max = np.where(own, tv_max, np.maximum(np.maximum(fct_np.shift_down(tv_max), tv_max),
                                             fct_np.shift_up(tv_max)))
    w_min = np.where(own, tv_min, np.minimum(np.minimum(fct_np.shift_down(tv_min), tv_min),
                                             fct_np.shift_up(tv_min)))
    return w_max, w_min


# Slack of the window check for results of the CUDA path: its fused kernels form every
# quotient as a product with the divisor's reciprocal (up to 1.5 ulp each) and evaluate
# LO, the bounds and the factors themselves, so their update may land a few ulp further
# past the oracle's window than the oracle's own update does.
GPU_WINDOW_ULPS = 16.0


def window_violations(m, T, hnode_new, T_new, inter, ulps: float = 4.0):
    """``[(node, layer)]`` of valid lanes outside the window (``ulps`` slack)."""
    w_max, w_min = window(m, inter)
    valid = m.node_layer_mask & (m.areasvol > 0.0) & (hnode_new > 0.0)
    scale = np.maximum(np.abs(T), np.abs(inter["LO"]))
    with np.errstate(invalid="ignore"):
        hi = w_max + ulps * np.spacing(np.maximum(np.abs(w_max), scale))
        lo = w_min - ulps * np.spacing(np.maximum(np.abs(w_min), scale))
    return np.argwhere(valid & ((T_new > hi) | (T_new < lo)))
