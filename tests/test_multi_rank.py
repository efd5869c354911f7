"""Multi-rank plumbing of bench.py on CPU: world size 2 over gloo.

The B200 path runs one process per GPU as independent replicas (no data-path
collective); the only cross-rank operations are the barrier and the
max-over-ranks reduction of the timed region.  These run here with the gloo
backend, as they run with NCCL on GPUs.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, REPO)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # each rank times a different amount; every rank must see the slowest
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max_ms": t}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    port = free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for r in range(2):
        got = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert got["max_ms"] == 15.0


@pytest.mark.slow
def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched like the driver's multi-GPU runs:
    rank 0 times the reference CPU path and prints one JSON line, rank 1 exits 0."""
    port = free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(REPO, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--steps", "1", "--warmup", "3", "--ref-budget", "0.3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=REPO)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2
    assert line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port")
