"""bench.py's multi-GPU form: one block per rank, no collective on the data
path, time taken as the maximum over ranks and throughput summed over the
replicas.  The aggregation runs here on two CPU ranks over gloo (the GPU runs
use NCCL with the same calls)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = [12.5, 20.0][rank]  # the ranks' own timed regions
        m = bench.replica_max(ms, dist, torch, "cpu")
        v = bench.replica_throughput(1000, 10, m, world)
        out[rank] = (m, v)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_max_and_throughput_over_two_gloo_ranks():
    world = 2
    with mp.Manager() as man:
        out = man.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    m, v = res[0]
    assert m == 20.0
    assert v == pytest.approx(world * 1000 * 10 / 0.020)


def test_single_rank_is_its_own_maximum():
    assert bench.replica_max(3.5, None, torch, "cpu") == 3.5
    assert bench.replica_throughput(8, 2, 4.0, 1) == pytest.approx(8 * 2 / 0.004)
