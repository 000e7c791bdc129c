"""The bench's several-rank path on the host (CPU, gloo, world size 2).

bench.py runs one replica per rank (replicas only: a placement does not shard) and reports the
whole job's throughput against the slowest rank: its per-rank loop and end-to-end times go
through one MAX all-reduce (bench.max_over_ranks). The reference arm runs on rank 0 alone and
the other ranks leave without work. Both are checked here without a GPU: the all-reduce on two
gloo ranks over 127.0.0.1, and the reference arm's rank rule in-process.
"""
import json
import os
import socket
from datetime import timedelta

import pytest

import bench


def free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_worker(rank, world, port, out_dir):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        # rank 0 is slower in the first time, rank 1 in the second
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.25 * rank], world, "cpu")
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump(got, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_single_rank_is_identity():
    assert bench.max_over_ranks([3.5, 7.0], 1, "cpu") == [3.5, 7.0]


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    mp.spawn(_rank_worker, args=(2, free_port(), str(tmp_path)), nprocs=2, join=True)
    for r in range(2):
        with open(tmp_path / f"rank{r}.json") as f:
            assert json.load(f) == [2.0, 10.0, 0.25]


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.argparse.Namespace(workload="small", warmup=1, steps=1, ref_iters=0, gpus=2)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""


@pytest.mark.parametrize("world", [1, 2])
def test_dist_env_reads_the_launcher(monkeypatch, world):
    monkeypatch.setenv("RANK", str(world - 1))
    monkeypatch.setenv("WORLD_SIZE", str(world))
    monkeypatch.setenv("LOCAL_RANK", str(world - 1))
    assert bench.dist_env() == (world - 1, world, world - 1)
