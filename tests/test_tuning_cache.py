"""The autotuners' persistent cache (fesom_jax_b200.tuning): keys separate GPU models,
meshes and workload shapes and are stable for the same inputs; entries round-trip through
the JSON file; a damaged file reads as empty."""

from fesom_jax_b200 import meshgen, tuning
from fesom_jax_b200.mesh import pi_mesh


def test_keys_separate_meshes_gpus_and_shapes():
    a, b = pi_mesh(), meshgen.make_mesh(600, seed=3, name="small600")
    k = tuning.key("ensemble", "NVIDIA B200", [a], members=32, ntr=8)
    assert k == tuning.key("ensemble", "NVIDIA B200", [pi_mesh()], ntr=8, members=32)
    assert k != tuning.key("ensemble", "NVIDIA B200", [b], members=32, ntr=8)
    assert k != tuning.key("ensemble", "NVIDIA H100", [a], members=32, ntr=8)
    assert k != tuning.key("ensemble", "NVIDIA B200", [a], members=16, ntr=8)
    assert k != tuning.key("plan", "NVIDIA B200", [a], members=32, ntr=8)
    # the mesh order of a mixed batch does not matter
    assert tuning.key("ensemble", "g", [a, b]) == tuning.key("ensemble", "g", [b, a])


def test_cache_round_trip_and_damaged_file(tmp_path):
    path = tmp_path / "sub" / "tuning.json"
    c = tuning.TuningCache(path)
    assert c.get("k") is None
    c.put("k", {"stage_map": [[2, 2], [2, 4], [4, 1], [4, 1]]})
    c.put("k2", {"mapping": [2, 1]})
    c2 = tuning.TuningCache(path)
    assert c2.get("k") == {"stage_map": [[2, 2], [2, 4], [4, 1], [4, 1]]}
    assert c2.get("k2") == {"mapping": [2, 1]}
    assert not list(path.parent.glob("*.tmp"))
    path.write_text("{not json")
    assert tuning.TuningCache(path).get("k") is None


def test_default_path_from_environment(monkeypatch, tmp_path):
    monkeypatch.setenv("FESOM_FCT_TUNING_CACHE", str(tmp_path / "t.json"))
    assert tuning.default_path() == tmp_path / "t.json"
