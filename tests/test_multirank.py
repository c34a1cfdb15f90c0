"""Multi-GPU host logic on CPU ranks (gloo, world_size 2).

The path shards by independent sea state: each rank owns a disjoint set of
oceans (replicas) and the only collective is the max over ranks of the timed
region. Both are checked here with two CPU processes."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = bench.rank_seeds(rank, 5)
        gathered = [None] * world
        dist.all_gather_object(gathered, seeds)
        mine = 10.0 + rank  # rank 1 is the slow one
        slowest = bench.max_over_ranks(mine, dist, "cpu")
        if rank == 0:
            out.put((gathered, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_seeds_are_disjoint_and_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert not set(gathered[0]) & set(gathered[1])
    assert sorted(gathered[0] + gathered[1]) == list(range(7, 17))
    assert slowest == 11.0


def test_single_rank_defaults():
    assert bench.rank_seeds(0, 3) == [7, 8, 9]
    rank, world, local = bench.dist_env()
    assert world >= 1 and 0 <= rank < world


def _router_worker(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oceanlib_b200 import router, workloads as W

        descs = W.ensemble_64()
        mine = router.assign(descs, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            out.put(gathered)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_router_shares_config4_across_two_ranks_without_exchange():
    # Each rank computes its own share of config 4's 64 sea states from the
    # descriptors alone: the shares, gathered, are disjoint, cover every
    # ocean, and agree with what either rank computes for the other.
    from oceanlib_b200 import router, workloads as W

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_router_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    descs = W.ensemble_64()
    assert gathered == router.assign(descs, 2)
    assert not set(gathered[0]) & set(gathered[1])
    assert sorted(gathered[0] + gathered[1]) == list(range(64))


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_router_balance_bound(world):
    # Longest-processing-time assignment: the busiest rank carries less than
    # the mean load plus one ocean's cost.
    from oceanlib_b200 import router, workloads as W

    descs = W.ensemble_64()
    shares = router.assign(descs, world)
    load = router.loads(descs, shares)
    assert sorted(i for s in shares for i in s) == list(range(64))
    mean = sum(load) / world
    assert max(load) < mean + max(router.ocean_cost(d) for d in descs)
    assert router.assign(descs, world) == shares  # deterministic
