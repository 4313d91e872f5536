"""The multi-rank steps of a replica run (bench.py --gpus N), as world-size-2 gloo ranks on CPU.

Every rank must take the same collective steps in the same order: agree on rank 0's settings,
meet at the barriers around the timed region, and report the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from patchtable_b200 import replicas
    replicas.init("gloo", timeout_s=60)
    r, w, local = replicas.env()
    replicas.barrier()
    slow = replicas.max_over_ranks(1.5 + r)                   # rank 1 is the slower one
    chosen = replicas.agree(10 * r + 3)                       # rank 0's choice wins
    rate = replicas.whole_job_rate(1000, slow, w)
    replicas.barrier()
    replicas.finish()
    out.put((r, w, local, slow, chosen, rate))


def test_two_gloo_ranks_agree():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, (rank, w, local, slow, chosen, rate) in enumerate(res):
        assert (rank, w, local) == (r, world, r)
        assert slow == 2.5
        assert chosen == 3.0
        assert rate == pytest.approx(world * 1000 / 2.5)


def test_single_process_needs_no_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from patchtable_b200 import replicas
    replicas.init("gloo")
    assert replicas.env() == (0, 1, 0)
    assert replicas.max_over_ranks(4.0) == 4.0 and replicas.agree(7) == 7.0
    replicas.barrier()
    replicas.finish()


def test_shard_by_cost_covers_every_image_once_and_balances():
    from patchtable_b200 import replicas
    rng = __import__("random").Random(4)
    costs = [rng.randint(1, 4_000_000) for _ in range(64)]
    for world in (1, 2, 3, 8):
        shards = replicas.shard_by_cost(costs, world)
        assert len(shards) == world
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - sum(loads) / world <= max(costs)
    assert replicas.shard_by_cost([5, 5, 5], 2) == [[0, 2], [1]]


def _shard_rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from patchtable_b200 import replicas
    replicas.init("gloo", timeout_s=60)
    r, w, _ = replicas.env()
    costs = [(7 * i) % 11 + 1 for i in range(20)]
    mine = replicas.shard_by_cost(costs, w)[r]
    units = sum(costs[i] for i in mine)
    slow = replicas.max_over_ranks(float(units))          # time stands in as proportional to units
    total = replicas.agree(sum(costs))
    replicas.finish()
    out.put((r, mine, units, slow, total))


def test_two_gloo_ranks_split_a_batch_by_image():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, u0, s0, t0), (_, m1, u1, s1, t1) = res
    assert not set(m0) & set(m1) and sorted(m0 + m1) == list(range(20))
    assert u0 + u1 == t0 == t1 and s0 == s1 == max(u0, u1)
