"""The multi-rank path on CPU: two gloo ranks partition the batched
workload (256 independent SDPs) with the package's work-based sharding;
gathered, the shares cover every problem exactly once, agree on every rank
without any exchange, and balance the estimated work; the timing reduction
(max over ranks) gives the slowest rank's time.  No GPU is used."""
import os

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import load_pkg


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        load_pkg()
        import importlib
        P = importlib.import_module("sdpa_dd_b200.problems")
        shard = importlib.import_module("sdpa_dd_b200.shard")
        rng_sizes = [(n, m) for n, m, _ in P.batch(256, seed=4)]
        works = [shard.work_estimate(m, [n]) for n, m in rng_sizes]
        shares = shard.partition_by_work(works, world)
        mine = shares[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        t = torch.tensor([float(rank + 1)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            out.put({"gathered": gathered, "shares": shares, "works": works, "tmax": float(t.item())})
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_two_gloo_ranks_shard_the_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_rank_main, args=(world, port, q), nprocs=world, join=True, start_method="spawn")
    res = q.get()
    gathered, shares, works = res["gathered"], res["shares"], res["works"]
    assert gathered == shares  # every rank computed the same assignment
    flat = sorted(i for s in gathered for i in s)
    assert flat == list(range(256))  # each problem exactly once
    loads = [sum(works[i] for i in s) for s in gathered]
    assert max(loads) / min(loads) < 1.02
    assert res["tmax"] == float(world)


def test_partition_is_deterministic_and_balanced():
    load_pkg()
    import importlib
    shard = importlib.import_module("sdpa_dd_b200.shard")
    works = [float((7 * q) % 23 + 1) for q in range(50)]
    for world in (1, 3, 8):
        s1, s2 = shard.partition_by_work(works, world), shard.partition_by_work(works, world)
        assert s1 == s2 and sorted(i for s in s1 for i in s) == list(range(50))
        loads = [sum(works[i] for i in s) for s in s1]
        assert max(loads) - min(loads) <= max(works)
