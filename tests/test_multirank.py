"""The N > 1 launch path on the CPU: two gloo ranks for the bench's
max-over-ranks reduction, per-rank inputs, and the reference arm under
torch.distributed.run with two ranks (rank 0 prints the one line, the other
exits without work).  No GPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], dist)
        ins = bench.rank_inputs(rank, 4)
        dist.barrier()
        with open(f"{out_path}.{rank}", "w") as f:
            json.dump({"max": got, "inputs": ins}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank_inputs_with_gloo(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    out = str(tmp_path / "rank")
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    res = [json.load(open(f"{out}.{r}")) for r in range(2)]
    for r in res:
        assert r["max"] == [2.0, 10.0, 0.5]  # every rank sees the slowest rank's times
    assert res[0]["inputs"] != res[1]["inputs"]  # replicas prove different inputs


def test_max_over_ranks_single_rank():
    import bench

    assert bench.max_over_ranks([3.0, 4.0], None) == [3.0, 4.0]


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_two_ranks():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--log-n", "10"]
    p = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1  # rank 0 alone prints
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
