"""Host logic of the multi-GPU benchmark (weak scaling over roots), run as
two gloo ranks on the CPU: the ranks' root shards cover the roots exactly
once, and the cross-rank reductions give the slowest time, the total edges
and the summed harmonic means."""
from __future__ import annotations

import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        roots = list(range(100, 164))
        mine = bench.rank_roots(roots, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        ms, edges, hm = bench.combine_ranks(dist, "cpu", 10.0 + rank, 1000.0 * (rank + 1), 2.5 * (rank + 1))
        out.put((rank, gathered, ms, edges, hm))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding_and_reductions():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, ms, edges, hm in results:
        flat = sorted(r for shard in gathered for r in shard)
        assert flat == list(range(100, 164))
        assert not set(gathered[0]) & set(gathered[1])
        assert ms == 11.0 and edges == 3000.0 and hm == 7.5


def test_single_rank_takes_every_root():
    assert bench.rank_roots([5, 6, 7], 0, 1) == [5, 6, 7]

