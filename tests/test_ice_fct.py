"""Sea-ice FCT advection (fesom_jax/ice_adv.py:175-194): the oracle and the CUDA path
against golden vectors of the reference's own ``fct_solve`` (tests/golden/
make_ice_golden.py) on the pi mesh and a coastline mesh, plus the properties the scheme
guarantees: total ice volume / area (sum of node area x tracer) conserved to round-off
(the Taylor-Galerkin operator and the antidiffusive fluxes both sum to zero), and the
reference test's boundedness (fesom_jax/tests/test_ice_adv.py:65-76)."""

import numpy as np
import pytest

from fesom_jax_b200 import meshgen
from fesom_jax_b200.mesh import Mesh, pi_mesh
from oracle import ice_fct_np
from tests.golden.make_mesh_golden_params import N_NODES, SEED
from tests.golden_cases import ICE_GOLDEN, RTOL, ice_cases

CASES = ["step_500", "fast_3600"]


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(ICE_GOLDEN))


@pytest.fixture(scope="module")
def meshes(pi):
    raw = meshgen.generate_raw(N_NODES, pi_mesh().zbar, seed=SEED)
    return {"pi": pi, "small": Mesh(**meshgen.derive(raw), name="small")}


def _ref(golden, mname, name):
    return [golden[f"{mname}_{name}__{t}"] for t in ("a", "m", "ms")]


def _content(m, x):
    return float(np.sum(m.area[:, 0] * x))


@pytest.mark.parametrize("mname", ["pi", "small"])
@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference(golden, meshes, mname, name):
    m = meshes[mname]
    c = ice_cases(m)[name]
    out = ice_fct_np.fct_solve(m, c["a"], c["m"], c["ms"], c["u"], c["v"], dt=c["dt"])
    for x, ref in zip(out, _ref(golden, mname, name)):
        assert np.max(np.abs(x - ref)) <= 1e-13 * np.max(np.abs(ref))


@pytest.mark.parametrize("name", CASES)
def test_oracle_conserves_and_bounds(meshes, name):
    m = meshes["pi"]
    c = ice_cases(m)[name]
    out = ice_fct_np.fct_solve(m, c["a"], c["m"], c["ms"], c["u"], c["v"], dt=c["dt"])
    for x, x0 in zip(out, (c["a"], c["m"], c["ms"])):
        assert abs(_content(m, x) - _content(m, x0)) <= 1e-12 * abs(_content(m, x0))
    assert out[0].max() - c["a"].max() < 0.05 and c["a"].min() - out[0].min() < 0.05


@pytest.mark.gpu
@pytest.mark.parametrize("mname", ["pi", "small"])
@pytest.mark.parametrize("name", CASES)
def test_gpu_matches_reference_and_oracle(golden, meshes, mname, name):
    import torch
    from fesom_jax_b200.ice_adv import IceConfig, fct_solve
    m = meshes[mname]
    c = ice_cases(m)[name]
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()  # noqa: E731
    cfg = IceConfig(ice_dt=c["dt"])
    out = [x.cpu().numpy() for x in fct_solve(cfg, m, d(c["a"]), d(c["m"]), d(c["ms"]),
                                               d(c["u"]), d(c["v"]))]
    orc = ice_fct_np.fct_solve(m, c["a"], c["m"], c["ms"], c["u"], c["v"], dt=c["dt"])
    for x, ref, o, x0 in zip(out, _ref(golden, mname, name), orc, (c["a"], c["m"], c["ms"])):
        assert np.max(np.abs(x - ref)) <= RTOL * np.max(np.abs(ref))
        assert np.max(np.abs(x - o)) <= RTOL * np.max(np.abs(o))
        assert abs(_content(m, x) - _content(m, x0)) <= 1e-12 * abs(_content(m, x0))
    again = [x.cpu().numpy() for x in fct_solve(cfg, m, d(c["a"]), d(c["m"]), d(c["ms"]),
                                                 d(c["u"]), d(c["v"]))]
    assert all(np.array_equal(a, b) for a, b in zip(out, again))


def test_exch_rejected(pi):
    from fesom_jax_b200.ice_adv import IceConfig, fct_solve
    z = np.zeros(pi.nod2D)
    with pytest.raises(NotImplementedError):
        fct_solve(IceConfig(), pi, z, z, z, z, z, exch=object())
