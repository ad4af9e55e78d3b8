"""Replica aggregation across ranks (the N>1 bench path), world size 2 on gloo, CPU only."""
import os
import socket

import torch.multiprocessing as mp

from ants_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, v = replicas.aggregate(1.5 + rank, 1000 * (rank + 1))
        out[rank] = (t, v, replicas.pair_seed(rank), replicas.assign_pairs(5, world, rank))
    finally:
        dist.destroy_process_group()


def test_aggregate_max_time_sum_work_two_ranks():
    world = 2
    port = _free_port()
    manager = mp.Manager()
    out = manager.dict()
    mp.start_processes(_worker, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    assert out[0][:2] == out[1][:2] == (2.5, 3000)
    assert out[0][2] != out[1][2]  # each rank registers its own pair
    assert sorted(out[0][3] + out[1][3]) == [0, 1, 2, 3, 4]


def test_aggregate_single_process_is_identity():
    assert replicas.aggregate(2.0, 7) == (2.0, 7)
