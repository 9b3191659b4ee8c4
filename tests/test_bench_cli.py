"""bench.py's command line: every --config choice dispatches to a function that exists
(a missing one only shows up as a NameError on the GPU otherwise)."""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_every_config_has_its_runner():
    sys.path.insert(0, str(ROOT))
    import bench
    for name in ("run_ours", "run_adjoint", "run_serve", "run_reference", "e2e_host",
                 "side_line", "workload_config"):
        assert callable(getattr(bench, name, None)), name
    src = (ROOT / "bench.py").read_text()
    for cfg in ("batched", "pi", "large", "adjoint", "serve"):
        assert f'"{cfg}"' in src
