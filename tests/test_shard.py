"""Sharding the worlds of a sweep over GPUs (CPU only): the cost-balanced
partition, and the per-rank results gathered on two gloo ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from life_simulation_b200 import workloads as wl
from life_simulation_b200.shard import gather_records, loads, partition, world_cost


def test_partition_covers_every_world_once_and_is_deterministic():
    costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0, 1.0]
    for n in (1, 2, 3, 7, 9):
        shares = partition(costs, n)
        assert len(shares) == n
        assert sorted(i for s in shares for i in s) == list(range(len(costs)))
        assert shares == partition(costs, n)
    # 8 -> r0, 5 -> r1, 3 -> r1, 3 -> r0 (tie: lower rank), 2 -> r1, 1 -> r1, 1 -> r0.
    assert partition(costs, 2) == [[3, 5, 6], [0, 1, 2, 4]]
    assert loads(costs, partition(costs, 2)) == [12.0, 11.0]
    with pytest.raises(ValueError):
        partition(costs, 0)


def test_partition_of_the_512_world_sweep_is_balanced():
    specs, _ = wl.sweep512()
    costs = [world_cost(s["width"], s["height"], s["radius"]) for s in specs]
    total = sum(costs)
    for n in (2, 4, 8):
        ld = loads(costs, partition(costs, n))
        # Largest-first list scheduling: within the largest single world of
        # the even split (a far tighter bound than LPT's 4/3 here).
        assert max(ld) - total / n <= max(costs) + 1e-12, (n, ld)
        assert max(ld) / min(ld) < 1.05


def test_world_cost_picks_the_cheaper_path():
    # Small radius: the direct path's few taps beat the spectral step.
    assert world_cost(256, 256, 2) < 256 * 256 * 10e-12
    # Large radius: the spectral step's per-pixel cost.
    assert world_cost(256, 256, 32) == pytest.approx(256 * 256 * 10e-12)
    assert world_cost(512, 512, 16) == pytest.approx(4 * world_cost(256, 256, 16))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world_size, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world_size)
    try:
        costs = [float(1 + (i * 7) % 5) for i in range(11)]
        mine = partition(costs, world_size)[rank]
        # Each rank "runs" its share and reports one record per world.
        records = [{"world": i, "rank": rank, "value": i * i} for i in mine]
        out[rank] = gather_records(records)
    finally:
        dist.destroy_process_group()


def test_shares_run_on_two_ranks_and_gather_in_world_order():
    world_size = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world_size, _free_port(), out), nprocs=world_size, join=True)
    costs = [float(1 + (i * 7) % 5) for i in range(11)]
    shares = partition(costs, world_size)
    for r in range(world_size):
        got = out[r]
        assert [g["world"] for g in got] == list(range(11))
        assert all(g["value"] == g["world"] ** 2 for g in got)
        assert all(g["world"] in shares[g["rank"]] for g in got)
    assert gather_records([{"world": 2}, {"world": 0}]) == [{"world": 0}, {"world": 2}]
