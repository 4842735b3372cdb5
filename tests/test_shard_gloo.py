"""Host-side multi-rank logic on CPU with gloo (world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from orbit_b200.shard import orbits_for_rank, met_draw_seed


def _port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from orbit_b200.shard import max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = orbits_for_rank(144, rank, world)
    t = max_over_ranks(10.0 + rank, device="cpu")
    got = [None] * world
    dist.all_gather_object(got, mine)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, got))


def test_partition_covers_disjointly():
    for world in (1, 2, 3, 8):
        parts = [orbits_for_rank(144, r, world) for r in range(world)]
        flat = sorted(x for p in parts for x in p)
        assert flat == list(range(144))
    seeds = {met_draw_seed(2024, r, d) for r in range(8) for d in range(12)}
    assert len(seeds) == 96


def test_gloo_two_ranks_max_and_partition():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, got in out:
        assert t == 11.0
        assert sorted(got[0] + got[1]) == list(range(144))
        assert not set(got[0]) & set(got[1])
