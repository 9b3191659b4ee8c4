"""The C loop oracle against the numpy oracle and the golden vectors (CPU)."""

import numpy as np
import pytest

from oracle import fct_c, fct_np
from tests.golden_cases import DT, cases, check_against_golden, load_golden


@pytest.fixture(scope="module")
def pi_cases(pi):
    return cases(pi)


@pytest.mark.parametrize("name", ["T_step1", "T_ab2", "sharp_x5", "T_wsplit_zstar"])
def test_c_oracle_matches_golden_and_numpy(pi, pi_cases, name):
    c = pi_cases[name]
    got, _ = fct_c.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                  c["hnode_new"], c["T"], c["T_old"], dt=DT, **c["kw"])
    check_against_golden(pi, load_golden(), name, c, got)
    ref, _ = fct_np.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                   c["hnode_new"], c["T"], c["T_old"], dt=DT, **c["kw"])
    lm = pi.node_layer_mask
    assert np.max(np.abs(got[lm] - ref[lm])) / np.max(np.abs(ref[lm])) < 1e-13
    assert np.array_equal(got[~lm], c["T"][~lm])


def test_c_oracle_thread_count_invariant(pi, pi_cases):
    c = pi_cases["sharp_x5"]
    a, _ = fct_c.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                c["hnode_new"], c["T"], c["T_old"], dt=DT, threads=1)
    b, _ = fct_c.advect_one_fct(pi, c["uv"], c["w_e"], c["helem"], c["hnode"],
                                c["hnode_new"], c["T"], c["T_old"], dt=DT, threads=4)
    assert np.array_equal(a, b)
