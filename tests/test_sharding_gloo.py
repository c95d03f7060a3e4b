"""Multi-rank host logic of the sweep sharding, run as two gloo ranks on the CPU.
The per-rank compute is replaced by a deterministic stand-in (no GPU here); the
partition, the gather and the global ordering are the code under test."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from sagittasbr_b200 import sharding as S


def test_block_partition_matches_reference_rule():
    # n // world each, remainder to the low ranks (src/app/sweep.cu:172-179)
    for n, world in [(600, 1), (600, 7), (5, 8), (8281, 8), (0, 3)]:
        parts = [S.block_partition(n, world, r) for r in range(world)]
        assert sum(c for _, c in parts) == n
        assert all(parts[r][0] + parts[r][1] == parts[r + 1][0] for r in range(world - 1))
        counts = [c for _, c in parts]
        assert max(counts) - min(counts) <= 1 and counts == sorted(counts, reverse=True)


def test_cost_partition_balances_and_covers():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0, 1.5, 1000)
    for world in (1, 2, 3, 8):
        parts = S.cost_partition(costs, world)
        assert parts[0][0] == 0 and sum(c for _, c in parts) == costs.size
        loads = [costs[s:s + c].sum() for s, c in parts]
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
    assert S.cost_partition([], 4) == [(0, 0)] * 4
    assert sum(c for _, c in S.cost_partition(np.zeros(10), 3)) == 10


def test_aperture_cost_tracks_projected_box():
    lo, hi = [-0.5, -0.5, -0.5], [0.5, 0.5, 0.5]
    c = S.aperture_cost(lo, hi, [0.0, 54.7356], [0.0, 45.0], 100, 100, 2.0)
    # face-on cube: 1 m of 2 m -> ~50 x 50 pixels; body diagonal: wider silhouette
    assert 2500 <= c[0] <= 52 * 52 and c[1] > c[0]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n, nf, balance, q):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        costs = np.linspace(1, 5, n) ** 2
        if balance == "cost":
            start, count = S.cost_partition(costs, world)[rank]
        else:
            start, count = S.block_partition(n, world, rank)
        idx = np.arange(start, start + count)
        # stand-in per-sample result: a function of the global sample index only
        vals = (idx[:, None] * 1.5 + 1j * np.arange(nf)[None, :]).astype(np.complex128)
        # ranks deliver their shard in reverse order to exercise the sort
        merged = S.gather_samples(idx[::-1], vals[::-1], n)
        if rank == 0:
            q.put(merged)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("balance", ["block", "cost"])
def test_two_rank_gather_orders_samples(balance):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, n, nf = 2, 37, 3
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, nf, balance, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    expect = np.arange(n)[:, None] * 1.5 + 1j * np.arange(nf)[None, :]
    np.testing.assert_array_equal(merged, expect)
