"""CPU tests of bench.py's multi-rank plumbing: replicas on N GPUs report the
slowest rank's time (max over ranks) after barriers, and only rank 0 of the
reference arm does work. Two gloo ranks on the CPU stand in for GPUs."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.rank_barrier(dist)
        got = bench.rank_max(10.0 * (rank + 1), dist, "cpu")
        bench.rank_barrier(dist)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": got}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        with open(tmp_path / f"rank{r}.json") as f:
            assert json.load(f)["max"] == 20.0


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_max(3.5, None, "cpu") == 3.5
    bench.rank_barrier(None)


def test_reference_arm_runs_on_rank_zero_only():
    """A non-zero rank of the reference arm exits 0 at once and prints nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, timeout=120, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
