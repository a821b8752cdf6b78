"""Multi-rank host logic on CPU (gloo, world size 2): sharding of independent problems by rank and the
max-over-ranks timing the benchmark reports. No GPU: the ranks exchange only host data."""
import os
import socket

import numpy as np

from hfk import batch as B


def test_shard_problems_is_a_balanced_partition():
    problems = B.draw_batch(256, seed=4)
    for world in (1, 2, 3, 8):
        shards = [B.shard_problems(problems, r, world) for r in range(world)]
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(len(problems)))  # every problem exactly once
        cost = [sum(3 * (2 * problems[k].n + 1) ** 3 for k in s) for s in shards]
        biggest = max(3 * (2 * q.n + 1) ** 3 for q in problems)
        assert max(cost) - min(cost) <= biggest  # greedy balance bound
        assert shards == [B.shard_problems(problems, r, world) for r in range(world)]  # deterministic


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    problems = B.draw_batch(32, seed=4)
    mine = B.shard_problems(problems, rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    # each rank's "time": the benchmark reports the maximum over ranks
    t = torch.tensor([1.0 + rank], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, gathered, float(t.item())))


def test_two_gloo_ranks_agree_on_shards_and_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, g0, t0), (r1, g1, t1) = res
    assert g0 == g1 and sorted(g0[0] + g0[1]) == list(range(32)) and not set(g0[0]) & set(g0[1])
    assert t0 == t1 == 2.0
