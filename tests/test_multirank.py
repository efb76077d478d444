"""The multi-GPU path of bench.py on CPU: two gloo ranks.  Regions are independent, so each rank takes
its own shard (no collective on the data path); the job's value is all ranks' cells over the slowest
rank's device time, reduced over the ranks.  In the strong-scaling leg the ranks split one shared
batch by the library's region partitioner: every region on exactly one rank, cells balanced."""
from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, q) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        cells = 1000.0 * (rank + 1)        # per-rank cells per step
        device_ms = 10.0 + rank            # per-rank device time of all steps
        value, ms_per_step = bench.weak_scaling_value(dist, cells, 5, device_ms)
        total = bench.rank_reduce(dist, float(rank + 1), "sum")
        slowest = bench.rank_reduce(dist, float(rank), "max")
        q.put((rank, bench.shard_seed(rank), value, ms_per_step, total, slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_weak_scaling_reduction():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    seeds = {g[1] for g in got}
    assert seeds == {1, 2}                          # each rank its own shard
    want_value = (1000.0 + 2000.0) * 5 / (11.0 / 1e3) / 1e9
    for rank, _, value, ms_per_step, total, slowest in got:
        assert value == pytest.approx(want_value, rel=1e-12)
        assert ms_per_step == pytest.approx(11.0 / 5)
        assert total == 3.0 and slowest == 1.0



def _split_worker(rank: int, world: int, port: int, q) -> None:
    sys.path.insert(0, str(ROOT))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from rovaca_b200 import synth

        shared = synth.config1(40, seed=bench.shard_seed(0))  # every rank builds the same batch
        mine = bench.strong_scaling_regions(shared, rank, world)
        cells = float(shared.subset(mine).cells()) if mine else 0.0
        everyone = [None] * world
        dist.all_gather_object(everyone, mine)
        total = bench.rank_reduce(dist, cells, "sum")
        biggest = bench.rank_reduce(dist, cells, "max")
        largest_region = max(shared.subset([g]).cells() for g in range(shared.n_regions))
        q.put((rank, everyone, total, biggest, float(shared.cells()), float(largest_region)))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_one_batch_by_region_cells():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, everyone, total, biggest, all_cells, largest_region in got:
        regions = [g for part in everyone for g in part]
        assert sorted(regions) == list(range(40))   # every region once, on one rank
        assert total == all_cells
        assert biggest <= all_cells / world + largest_region
    assert got[0][1] == got[1][1]                    # both ranks agree on the split


def test_reference_arm_runs_on_rank_zero_only(capsys):
    """Under torchrun the reference arm's other ranks exit without work or output."""
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        steps, warmup = 1, 3

    bench.run_reference(Args(), rank=1, world=2)
    assert capsys.readouterr().out == ""
