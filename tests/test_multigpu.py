"""Multi-rank host logic on CPU (gloo, world size 2): instance sharding has
no data-path collective, every instance lands on exactly one rank, and the
timing reduction returns the max over ranks."""
import os
import socket

import pytest

import multigpu


def test_lpt_partition_covers_every_instance_once():
    import workloads as W
    sizes = W.log_uniform_sizes(64)
    costs = [multigpu.estimated_cost(int(n)) for n in sizes]
    for nranks in (1, 2, 3, 4, 8):
        parts = multigpu.lpt_partition(costs, nranks)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert multigpu.imbalance(costs, parts) < 1.35


def test_lpt_partition_degenerate_cases():
    assert multigpu.lpt_partition([], 3) == [[], [], []]
    assert multigpu.lpt_partition([5.0], 2) == [[0], []]
    with pytest.raises(ValueError):
        multigpu.lpt_partition([1.0], 0)


def test_weak_scaling_value():
    assert multigpu.weak_scaling_value(1_000_000, 4, 100.0) == pytest.approx(40.0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, costs, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    parts = multigpu.lpt_partition(costs, world)
    mine = parts[rank]
    fake_ms = 10.0 + 5.0 * rank
    mx = multigpu.reduce_max(fake_ms, dist)
    total = multigpu.reduce_sum(len(mine), dist)
    dist.barrier()
    out[rank] = (mine, mx, total)
    dist.destroy_process_group()


def _batched_worker(rank, world, port, out):
    import torch.distributed as dist
    import workloads as W
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    insts = W.batched_instances()
    seen = []

    def run_shard(mine):  # stands in for the engine: records the shard, reports a time from its cost
        seen.extend(mine)
        return 1e-9 * sum(multigpu.instance_cost(insts[i]) for i in mine), len(mine)

    res = multigpu.batched_run(insts, rank, world, run_shard, rhs=8, dist=dist)
    dist.barrier()
    out[rank] = (seen, res["ms"], res["value"], res["imbalance"], res["extra"])
    dist.destroy_process_group()


def test_two_rank_gloo_batched_instances_are_sharded():
    """The batched benchmark's run path (multigpu.batched_run, with the
    engine replaced by a stand-in): on two gloo ranks every one of the 64
    instances is evaluated by exactly one rank, the step time is the slower
    rank's, and the value counts every instance once."""
    import torch.multiprocessing as mp
    import workloads as W
    insts = W.batched_instances()
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_batched_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    a, b = res[0], res[1]
    assert sorted(a[0] + b[0]) == list(range(len(insts))) and not set(a[0]) & set(b[0])
    costs = [multigpu.instance_cost(i) for i in insts]
    slow = max(sum(costs[i] for i in a[0]), sum(costs[i] for i in b[0])) * 1e-9
    assert a[1] == b[1] == pytest.approx(slow)
    npts = sum(i["n"] for i in insts)
    assert a[2] == pytest.approx(npts * 8 / (slow / 1e3) / 1e6)
    assert a[3] == b[3] < 1.05 and a[4] + b[4] == len(insts)


def test_two_rank_gloo_sharding_and_max_timing():
    import torch.multiprocessing as mp
    costs = [multigpu.estimated_cost(n) for n in (10_000, 500_000, 40_000, 250_000, 90_000, 12_000, 330_000)]
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, costs, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    a, b = res[0], res[1]
    assert sorted(a[0] + b[0]) == list(range(len(costs))) and not set(a[0]) & set(b[0])
    assert a[1] == b[1] == 15.0  # max over ranks
    assert a[2] == b[2] == len(costs)
