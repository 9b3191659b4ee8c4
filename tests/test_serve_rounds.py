"""Host logic of the serving engine's multi-rate iterations (no GPU): how many steps each
active request takes in one iteration."""

import types

from fesom_jax_b200.serve import Request, ServingEngine


def _engine(max_rounds, wet):
    meshes = {k: types.SimpleNamespace(mesh=types.SimpleNamespace(n_wet_layers=v))
              for k, v in wet.items()}
    return types.SimpleNamespace(meshes=meshes, max_rounds=max_rounds)


def _req(mesh, K, steps=0):
    r = Request(rid=0, arrival=0.0, mesh=mesh, K=K, adjoint=False, seed=0)
    r.steps = steps
    return r


def test_rounds_follow_the_step_cost_ratio():
    eng = _engine(16, {"pi": 100_000, "core2": 3_000_000, "large": 52_000_000})
    active = [_req("large", 50), _req("core2", 50), _req("pi", 50), _req("pi", 3, steps=1)]
    # the largest mesh takes one step; CORE2 17 (capped at 16); pi capped at 16, or its 2
    # remaining steps
    assert ServingEngine._rounds(eng, active) == [1, 16, 16, 2]


def test_rounds_are_one_in_a_single_class_and_respect_the_cap():
    eng = _engine(16, {"pi": 100_000, "core2": 3_000_000})
    assert ServingEngine._rounds(eng, [_req("pi", 9), _req("pi", 9)]) == [1, 1]
    assert ServingEngine._rounds(eng, [_req("core2", 9), _req("pi", 40)]) == [1, 16]
    eng1 = _engine(1, {"pi": 100_000, "core2": 3_000_000})   # lockstep
    assert ServingEngine._rounds(eng1, [_req("core2", 9), _req("pi", 40)]) == [1, 1]
