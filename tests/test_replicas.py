"""The multi-GPU path of the benchmark on the CPU: two ranks over gloo (one process each, rendezvous on
127.0.0.1), each a replica; the job's time is the slowest rank's and the units add up over the ranks."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def replica(rank, world, port, results):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from o_o_solver_b200.replicas import Replicas

    replicas = Replicas("gloo", timeout_s=60.0)
    replicas.barrier()
    slowest = replicas.slowest(1.5 + rank)
    total = replicas.total(10.0 * (rank + 1))
    replicas.close()
    results[rank] = (replicas.rank, replicas.world, slowest, total)


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = free_port()
    processes = [ctx.Process(target=replica, args=(rank, 2, port, results)) for rank in range(2)]
    for p in processes:
        p.start()
    for p in processes:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in processes), [p.exitcode for p in processes]
    assert dict(results) == {0: (0, 2, 2.5, 30.0), 1: (1, 2, 2.5, 30.0)}


def test_one_rank_needs_no_process_group(monkeypatch):
    for name in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(name, raising=False)
    from o_o_solver_b200.replicas import Replicas

    replicas = Replicas("gloo")
    assert (replicas.rank, replicas.world) == (0, 1)
    assert replicas.slowest(3.0) == 3.0 and replicas.total(4.0) == 4.0
    replicas.close()
