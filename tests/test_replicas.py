"""The multi-rank path of bench.py on CPU (gloo, world size 2).  The projector
work is independent replicas, one per GPU, with no collective on the data
path; what ranks share is the timing: every rank takes the same collective
steps, the reported time is the slowest rank's, and rank 0 alone prints."""
import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _max_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # the same two collectives on every rank, in the same order
        a = bench.max_over_ranks(1.5 + rank, world, "cpu")
        b = bench.max_over_ranks(10.0 - rank, world, "cpu")
        with open(os.path.join(out, f"r{rank}.json"), "w") as f:
            json.dump([a, b], f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks(tmp_path):
    import torch.multiprocessing as mp
    mp.start_processes(_max_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        with open(tmp_path / f"r{r}.json") as f:
            assert json.load(f) == [2.5, 10.0]


def test_max_over_ranks_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.25, 1, "cpu") == 3.25


def test_reference_arm_under_torchrun_prints_once():
    """Two ranks launched by torchrun on one node: rank 0 times the
    reference's CPU path and prints one line, rank 1 exits 0 without work."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2", "--master-addr",
           "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "1"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["cores"] >= 1 and d["e2e"]["h2d_bytes_per_step"] == 0
