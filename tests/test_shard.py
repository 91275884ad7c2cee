"""Instance sharding of batched workloads: the nnz-balanced partition, and the
gather / max-over-ranks plumbing on two gloo ranks (CPU, no GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pramana_b200 import generators as G
from pramana_b200.shard import partition


def test_partition_covers_and_balances():
    w = G.uneven_family_sizes(256, 1e4, 5e5, seed=4)
    for world in (1, 2, 3, 4, 8):
        parts = partition(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(loads) / world + max(w) + 1e-9
        assert all(p == sorted(p) for p in parts)
    assert partition(w, 4) == partition(w, 4)


def test_uneven_family_subset_matches_full():
    full = G.uneven_family(6, 1e4, 3e4, seed=9)
    sub = G.uneven_family(6, 1e4, 3e4, seed=9, only=[4, 1])
    for a, b in zip([full[4], full[1]], sub):
        assert a.name == b.name and np.array_equal(a.value, b.value) and np.array_equal(a.index, b.index)


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from pramana_b200.shard import gather, max_over_ranks, partition

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = [5, 1, 1, 3, 2, 8, 1]
        mine = partition(w, world)[rank]
        local = {i: {"status": "Optimal", "iterations": 10 * i, "rank": rank} for i in mine}
        merged = gather(local)
        t = max_over_ranks([0.5 + rank, 2.0 - rank])
        if rank == 0:
            out.put((sorted(merged), [merged[i]["rank"] for i in sorted(merged)], t))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(120)
def test_gather_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(100)
    assert all(p.exitcode == 0 for p in procs)
    keys, owners, t = q.get(timeout=10)
    assert keys == list(range(7))
    assert owners == [0 if i in partition([5, 1, 1, 3, 2, 8, 1], 2)[0] else 1 for i in range(7)]
    assert t == [1.5, 2.0]


def _solve_worker(rank, world, port, out):
    """One rank: its nnz-balanced share of an uneven family, each LP solved
    by the CPU oracle, then the gather on rank 0."""
    import torch.distributed as dist

    from oracle import oracle as O
    from pramana_b200.shard import gather, partition

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = G.uneven_family_sizes(10, 2e3, 2e4, seed=12)
        mine = partition(sizes, world)[rank]
        lps = G.uneven_family(10, 2e3, 2e4, seed=12, only=mine)
        local = {}
        for i, lp in zip(mine, lps):
            r = O.solve(lp, "oracle", tolerance=1e-5, max_iterations=100000)
            local[i] = {"status": r.status, "iterations": r.iterations, "objective": r.objective,
                        "x": r.x.tolist(), "y": r.y.tolist(), "rank": rank}
        merged = gather(local)
        if rank == 0:
            out.put(merged)
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_sharded_solves_equal_one_process_solves(oracle_mod):
    """Two gloo ranks split an uneven family by nonzeros, solve their shares
    and gather: every instance's answer equals the one-process answer (the
    same solver on the same LP), and every instance is solved exactly once."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_solve_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=280)
    for p in procs:
        p.join(60)
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(merged) == list(range(10))
    assert {merged[i]["rank"] for i in merged} == {0, 1}
    for i, lp in enumerate(G.uneven_family(10, 2e3, 2e4, seed=12)):
        r = oracle_mod.solve(lp, "oracle", tolerance=1e-5, max_iterations=100000)
        got = merged[i]
        assert got["status"] == r.status and got["iterations"] == r.iterations
        assert got["objective"] == r.objective
        assert np.array_equal(np.array(got["x"]), r.x) and np.array_equal(np.array(got["y"]), r.y)
