"""The N > 1 path of bench.py on CPU: two ranks over gloo (127.0.0.1), the barrier, the
max-over-ranks job time, the whole-job weak-scaling rate, distinct member seeds per
rank, and the reference arm printing from rank 0 only."""

import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    D = bench.Dist()
    D.init("gloo")
    D.barrier()
    t_local = 1.0 + rank          # rank 1 is the slow one
    value, t = D.weak_value(100.0, t_local, None)
    seeds = [bench.member_seed(rank, i) for i in range(3)]
    D.barrier()
    D.close()
    Path(out_dir, f"r{rank}.json").write_text(json.dumps(dict(value=value, t=t, seeds=seeds)))


def test_two_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    r = [json.loads((tmp_path / f"r{i}.json").read_text()) for i in range(2)]
    for x in r:
        assert x["t"] == 2.0                     # max over ranks
        assert x["value"] == 100.0 * 2 / 2.0     # all ranks' updates / job time
    assert not set(r[0]["seeds"]) & set(r[1]["seeds"])


@pytest.mark.timeout(600)
def test_reference_arm_prints_on_rank0_only():
    """Under torchrun with 2 ranks the CPU reference arm runs and prints on rank 0 only
    (pi workload, one short step); the other rank exits 0 without output."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--config", "pi", "--gpus", "2", "--steps", "1",
           "--warmup", "0"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=500)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
