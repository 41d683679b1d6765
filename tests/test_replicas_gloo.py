"""Multi-process host logic of bench.py on CPU: two gloo ranks, each with its own work (replicas,
no data-path collective); the job time is the slowest rank's and the rate counts every rank's
registrations. The reference arm prints from rank 0 only."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    per_rank_seconds = [2.0, 3.0][rank]
    slowest = bench.max_over_ranks(per_rank_seconds, world, torch.device("cpu"))
    out[rank] = (slowest, bench.replica_rate(world, 5, slowest))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1] == (3.0, 2 * 5 / 3.0)


def test_reference_arm_other_ranks_exit(monkeypatch, capsys):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("LOCAL_RANK", "1")
    class A:
        impl, steps, warmup, seed = "reference", 1, 0, 0
    assert bench.run_reference(A()) == 0
    assert capsys.readouterr().out == ""
