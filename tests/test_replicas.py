"""Multi-GPU host logic (bounce_b200.replicas) on CPU: the partition of
independent cloths over ranks, and the collectives around the step, run as
two gloo processes."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from bounce_b200 import replicas


def test_plan_covers_every_cloth_once_and_balances():
    rng = __import__("numpy").random.default_rng(5)
    sides = rng.integers(16, 129, size=512)
    work = [int(s) * int(s) for s in sides]
    for world in (1, 2, 3, 4, 8):
        shards = replicas.plan_shards(work, world)
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(len(work)))
        loads = replicas.shard_loads(work, shards)
        # LPT: no rank exceeds the average by more than the largest cloth
        assert max(loads) - sum(loads) / world <= max(work)
        assert max(loads) / min(loads) < 1.01


def test_plan_is_deterministic_and_ties_go_low():
    work = [5, 5, 5, 5]
    assert replicas.plan_shards(work, 2) == [[0, 2], [1, 3]]
    assert replicas.plan_shards(work, 2) == replicas.plan_shards(list(work), 2)
    assert replicas.plan_shards([], 3) == [[], [], []]


def test_plan_budget():
    work = [100, 90, 80, 70]
    replicas.plan_shards(work, 2, bytes_of=[w * 10 for w in work], budget_bytes=1700)
    with pytest.raises(replicas.BudgetError):
        replicas.plan_shards(work, 2, bytes_of=[w * 10 for w in work], budget_bytes=1600)
    with pytest.raises(ValueError):
        replicas.plan_shards(work, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=30))
    try:
        env = replicas.rank_env()
        work = [int(x) for x in (1024, 4096, 256, 16384, 9, 700, 700)]
        shards = replicas.plan_shards(work, world)
        mine = shards[env.rank]
        units = sum(work[k] for k in mine) * 10          # ten steps of the rank's cloths
        seconds = 0.5 + 0.25 * env.rank                  # the rank's device time
        out = {"rank": env.rank, "world": env.world, "mine": mine, "same_plan": replicas.check_same_plan(shards),
               "max_s": replicas.max_over_ranks(seconds), "sum_units": replicas.sum_over_ranks(units),
               "rate": replicas.aggregate_rate(units, seconds)}
        q.put(out)
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    outs.sort(key=lambda o: o["rank"])
    work = [1024, 4096, 256, 16384, 9, 700, 700]
    # the ranks' shards are disjoint and cover every cloth; both computed the same plan
    assert sorted(outs[0]["mine"] + outs[1]["mine"]) == list(range(len(work)))
    assert all(o["same_plan"] for o in outs)
    # timing is the slowest rank; the rate is all units over that time
    for o in outs:
        assert o["max_s"] == pytest.approx(0.75)
        assert o["sum_units"] == pytest.approx(10 * sum(work))
        assert o["rate"] == pytest.approx(10 * sum(work) / 0.75)


def _dropout_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        # this rank leaves between steps, with nothing in flight
        q.put({"rank": 1, "left": True})
        q.close()
        q.join_thread()  # the message is sent before the process ends
        os._exit(0)
    try:
        t = torch.ones(1)
        dist.all_reduce(t)
        q.put({"rank": 0, "error": None})
    except Exception as e:  # the collective ends with an error instead of waiting for good
        q.put({"rank": 0, "error": type(e).__name__})
    q.close()
    q.join_thread()
    os._exit(0)


def test_rank_that_leaves_ends_the_next_collective_with_an_error():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dropout_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = {o["rank"]: o for o in (q.get(timeout=120) for _ in range(world))}
    for p in procs:
        p.join(timeout=60)
    assert outs[1]["left"]
    assert outs[0]["error"] is not None
