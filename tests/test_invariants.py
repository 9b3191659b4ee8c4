"""Per-step correctness gates beyond the max-norm tolerance (``oracle/gates.py``), on the
oracle (CPU) and on the CUDA result (GPU):

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

from oracle import fct_np, gates
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
    return gates.closure_residual(m, c["T"], c["hnode"], c["hnode_new"], T_new, inter, DT)


def window(m, inter):
    return gates.window(m, inter)


def window_violations(m, c, T_new, inter, ulps=4.0):
    return gates.window_violations(m, c["T"], c["hnode_new"], T_new, inter, ulps)


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
    assert len(window_violations(pi, c, T_gpu, inter, gates.GPU_WINDOW_ULPS)) == 0
