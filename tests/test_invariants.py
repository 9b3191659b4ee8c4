"""Per-step correctness gates beyond the max-norm tolerance, on the oracle (CPU) and on
the CUDA result (GPU):

* budget closure: sum(areasvol * (hnode_new * T_new - hnode * T)) equals
  dt * sum over nodes of the surface fluxes (LO vertical flux + limited antidiffusive
  vertical flux at nzmin): horizontal fluxes cancel edge by edge and interior vertical
  fluxes telescope, so the step changes the tracer content only through the surface;
* monotonicity against the Zalesak window: every updated lane stays inside
  [window_min, window_max] of the limiter (tracer_adv.py:389-418); the violation set must
  be empty for the oracle and for the GPU. The slack is 4 ulp of the largest magnitude the
  update combines (the bound, T and LO): T_new = T + ((LO*hnode_new - T*hnode) + fluxes
  + T*(hnode - hnode_new)) / hnode_new cancels T against LO-sized terms, so its rounding
  is relative to those (the oracle itself lands 6 ulp of a 2.4 bound, 1.5 ulp of T = 9.3,
  past the window on the limiter-active case).

The window and the surface fluxes come from the oracle's intermediates; the GPU result
is checked against them because it equals the oracle's T_new to 1e-12."""

import numpy as np
import pytest

from oracle import fct_np
from tests.golden_cases import DT, cases

CASES = ["T_step1", "S_step1", "T_ab2", "sharp_x5", "const"]
# closure residual relative to the step's total tracer content (sum |areasvol*hnode*T|)
CLOSURE_RTOL = 1e-13


def _oracle(m, c):
    inter = {}
    T_new, _ = fct_np.advect_one_fct(m, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                     c["hnode_new"], c["T"], c["T_old"], dt=DT,
                                     intermediates=inter, **c["kw"])
    return T_new, inter


def closure_residual(m, c, T_new, inter):
    lm = m.node_layer_mask
    av = m.areasvol
    content = np.where(lm, av * c["hnode"] * c["T"], 0.0)
    lhs = np.sum(np.where(lm, av * c["hnode_new"] * T_new, 0.0)) - np.sum(content)
    n = np.arange(m.nod2D)
    top = m.ulevels_nod2D - 1
    rhs = DT * np.sum(inter["flux_v_lo"][n, top] + inter["adf_v_lim"][n, top])
    return abs(lhs - rhs) / np.sum(np.abs(content))


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


def window_violations(m, c, T_new, inter):
    w_max, w_min = window(m, inter)
    valid = m.node_layer_mask & (m.areasvol > 0.0) & (c["hnode_new"] > 0.0)
    scale = np.maximum(np.abs(c["T"]), np.abs(inter["LO"]))
    with np.errstate(invalid="ignore"):
        hi = w_max + 4.0 * np.spacing(np.maximum(np.abs(w_max), scale))
        lo = w_min - 4.0 * np.spacing(np.maximum(np.abs(w_min), scale))
    return np.argwhere(valid & ((T_new > hi) | (T_new < lo)))


@pytest.mark.parametrize("name", CASES)
def test_oracle_closure_and_window(pi, name):
    c = cases(pi)[name]
    T_new, inter = _oracle(pi, c)
    assert closure_residual(pi, c, T_new, inter) <= CLOSURE_RTOL
    assert len(window_violations(pi, c, T_new, inter)) == 0


def test_window_gate_detects_a_planted_overshoot(pi):
    """The gate is not vacuous: an oracle result pushed past its window is caught."""
    c = cases(pi)["sharp_x5"]
    T_new, inter = _oracle(pi, c)
    w_max, _ = window(pi, inter)
    bad = T_new.copy()
    n, k = np.argwhere(pi.node_layer_mask)[1234]
    bad[n, k] = w_max[n, k] + 1e-9 * max(1.0, abs(w_max[n, k]))
    assert [tuple(v) for v in window_violations(pi, c, bad, inter)] == [(n, k)]
    assert closure_residual(pi, c, bad, inter) > 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_gpu_closure_and_window(pi, name):
    from tests.test_fct_gpu import run_gpu
    import torch
    c = cases(pi)[name]
    _, inter = _oracle(pi, c)
    T_gpu = run_gpu(torch, pi, c)
    assert closure_residual(pi, c, T_gpu, inter) <= CLOSURE_RTOL
    assert len(window_violations(pi, c, T_gpu, inter)) == 0
