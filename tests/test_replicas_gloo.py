"""The multi-rank path of bench.py (replicas, one box per rank) on CPU: world size 2 over gloo."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        local_ms = 10.0 + 5.0 * rank                 # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, world, "cpu")
        dist.barrier()
        out[rank] = (ms, bench.aggregate_rate(world, 512 ** 3, 20, ms))
    finally:
        dist.destroy_process_group()


def test_replica_timing_takes_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 15.0
    assert res[0][1] == pytest.approx(2 * 512 ** 3 * 20 / 15e-3)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.main() == 0
    assert capsys.readouterr().out == ""
