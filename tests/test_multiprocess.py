"""The N > 1 host logic on CPU (gloo, world size 2).  `bench.py --gpus N`
runs one independent replica per rank (no collective on the data path) and
reports the job's time as the max over ranks; the reference arm runs on rank
0 alone under torchrun while the other ranks exit 0 without work."""
import datetime
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, out):
    import torch.distributed as td

    td.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                          timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench

    # each replica's own time; every rank must see the slowest one
    r = bench.max_over_ranks(1.5 * (rank + 1), "cpu")
    td.barrier()
    td.destroy_process_group()
    with open(f"{out}.{rank}", "w") as f:
        f.write(repr(r))


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "r")
    mp.start_processes(_replica, args=(2, free_port(), out), nprocs=2, start_method="spawn", join=True)
    assert [float(open(f"{out}.{k}").read()) for k in range(2)] == [3.0, 3.0]


def test_max_over_ranks_without_a_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(2.5, "cpu") == 2.5


def test_reference_arm_under_torchrun():
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libref3d_lazy.so")):
        pytest.skip("the reference is not built here (oracle/_ref)")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--bodies", "3000", "--steps", "2", "--warmup", "1", "--cpu-budget", "5"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr[-3000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["steps"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
