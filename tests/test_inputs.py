"""The benchmark's closed-basin velocities (inputs.basin_velocities).

The multi-step workloads need a low-order step that stays monotone: the plain
streamfunction of ``kind="psi"`` carries column divergence wherever the bathymetry steps,
which ``compute_w`` turns into a surface ``w`` with a vertical CFL far above 1 (the cause
of non-finite states after several hundred steps). A per-layer streamfunction that
vanishes at every node touching a wall on that layer is discretely divergence-free layer
by layer; the small white-noise part keeps the vertical path exercised.
"""

import numpy as np
import pytest

from fesom_jax_b200 import inputs as I
from fesom_jax_b200 import meshgen


@pytest.fixture(scope="module")
def coast():
    return meshgen.make_mesh(2000, seed=5, name="coast2000")


@pytest.mark.parametrize("which", ["pi", "coast"])
def test_basin_flow_is_divergence_free_layer_by_layer(pi, coast, which):
    m = pi if which == "pi" else coast
    hn, he = I.rest_thickness(m)
    uv = I.basin_velocities(m, np.random.default_rng(1), sigma_div=0.0)
    w = I.compute_w(m, uv, he)
    speed = np.sqrt((uv ** 2).sum(-1))[m.elem_layer_mask]
    assert np.abs(w).max() <= 1e-13 * speed.max()
    assert speed.mean() > 0.05     # a real flow, not a vanished one


@pytest.mark.parametrize("which", ["pi", "coast"])
def test_basin_flow_keeps_the_low_order_step_monotone(pi, coast, which):
    m = pi if which == "pi" else coast
    hn, he = I.rest_thickness(m)
    uv = I.basin_velocities(m, np.random.default_rng(2))
    w = I.compute_w(m, uv, he)
    assert np.abs(w).max() > 1e-6                     # the divergent part reaches w
    assert I.lo_outflow_cfl(m, uv, w, hn, 3600.0) < 1.0
    # the plain streamfunction over the same bathymetry does not
    psi = I.velocities(m, np.random.default_rng(2), kind="psi")
    assert I.lo_outflow_cfl(m, psi, I.compute_w(m, psi, he), hn, 3600.0) > \
        I.lo_outflow_cfl(m, uv, w, hn, 3600.0)


def test_basin_torch_combine_equals_numpy(pi):
    import torch
    a = I.basin_velocities(pi, np.random.default_rng(3), n_vortices=3)
    psi, noise = I.basin_draw(pi, np.random.default_rng(3), 0.1, 3, I.BASIN_SIGMA_DIV)
    b = I.basin_combine(pi, psi, noise, I.wall_rings(pi, I.basin_rings(pi)), torch, "cpu")
    assert b.dtype == torch.float64
    assert np.array_equal(a, b.numpy())


def test_wall_rings_grow_monotonically(coast):
    rings = I.wall_rings(coast, 4)
    for (n0, u0, c0), (n1, u1, c1) in zip(rings, rings[1:]):
        assert np.all(n1 <= n0) and np.all(u1 >= u0) and np.all(c1 >= c0)
    taper = I.basin_taper(rings, coast.nl)
    assert taper.min() == 0.0 and taper.max() == 1.0
