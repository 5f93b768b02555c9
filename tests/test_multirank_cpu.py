"""The multi-rank logic of bench.py on CPU: two gloo ranks (no GPU).

With N GPUs every rank runs its own replica of the single-system workload, and the batched workload
splits its independent problems across the ranks; the only collectives are the barrier and the
max/sum of the timings and counts over the ranks.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        mine = bench.batch_share(256, world, rank)
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        t_max = bench.ranks_reduce(10.0 + rank, "max", dist, "cpu")
        n_sum = bench.ranks_reduce(len(mine), "sum", dist, "cpu")
        dist.barrier()
        out[rank] = (shares, t_max, n_sum)
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_the_batch_and_reduce():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    shares, t_max, n_sum = res[0]
    assert res[1][0] == shares
    a, b = set(shares[0]), set(shares[1])
    assert not (a & b) and (a | b) == set(range(256))              # disjoint and complete
    rows = {}
    for p in range(256):
        u = bench.uniforms(bench.mt19937_64_stream(4000 + p, 2))
        nx, ny = (32 + int(v * 225) for v in u)
        rows[p] = (nx - 1) * (ny - 1)
    la, lb = sum(rows[p] for p in a), sum(rows[p] for p in b)
    assert abs(la - lb) <= 0.01 * (la + lb)                         # balanced within 1%
    assert t_max == 11.0 and n_sum == 256.0                         # max over ranks, sum of counts
    assert res[1][1] == 11.0


def test_single_rank_is_the_identity():
    assert bench.ranks_reduce(3.5, "max", None, "cpu") == 3.5
    assert bench.batch_share(256, 1, 0) == list(range(256))
