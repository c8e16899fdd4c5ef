"""The multi-GPU path of bench.py is replicas only: each rank steps its own session and the
job's time is the slowest rank's.  Its rank logic runs here as two gloo processes on the CPU."""
import importlib.util
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b = load_bench()
        got = b.max_over_ranks([10.0 * (rank + 1), 7.0 - rank], world, "cpu")
        out[rank] = got
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_gloo_world_2():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(world, free_port(), out), nprocs=world, join=True, start_method="spawn")
        assert dict(out) == {0: [20.0, 7.0], 1: [20.0, 7.0]}


def test_aggregate_value_counts_every_replica():
    b = load_bench()
    assert b.aggregate_value(2, 100, 50.0) == pytest.approx(4000.0)
    assert b.aggregate_value(1, 100, 50.0) == pytest.approx(2000.0)


def test_reference_arm_other_ranks_do_nothing(monkeypatch):
    b = load_bench()
    monkeypatch.setenv("RANK", "1")

    class A:
        steps = 5
        warmup = 1
    assert b.run_reference(A()) == 0  # returns before rendering or running anything
