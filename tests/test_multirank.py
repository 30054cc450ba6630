"""The N > 1 logic of bench.py on CPU: two gloo ranks on 127.0.0.1.

Each rank solves its own seeded sites of the same model (weak scaling, no
data-path collective); timings are combined as the maximum over ranks and
the whole-job value counts every rank's solves.
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


class _Args:
    lattice = 16
    sites = 8
    moments = 16


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = bench.make_problem(_Args(), rank)
        sites = [None] * world
        dist.all_gather_object(sites, p.sites.tolist())
        again = bench.make_problem(_Args(), rank).sites.tolist()
        t = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        out.put((rank, sites, again == sites[rank], t, p.N, p.M))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_sites_and_take_max():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, sites, reproducible, t, N, M in res:
        assert reproducible
        assert t == [2.0, 10.0]            # max over ranks, on every rank
        assert N == 16 * 16 * 2 and M == 16
        assert len(sites) == world and all(len(s) == 8 for s in sites)
        assert sites[0] != sites[1]        # each rank its own seeded sites
    assert res[0][1] == res[1][1]          # both ranks see the same shards


def test_reference_arm_only_on_rank_zero():
    class A:
        pass
    assert bench.reference_arm(A(), 2, 1) is None


@pytest.mark.parametrize("world", [1, 2, 4])
def test_whole_job_value_counts_every_rank(world):
    # value = B * steps * world / max-over-ranks time
    B, steps, ms = 64, 5, 2000.0
    assert B * steps * world / (ms / 1e3) == pytest.approx(160.0 * world)
