"""Multi-GPU split of batched WaveHoltz solves, exercised on CPU with two gloo ranks.

Each rank computes the same deterministic assignment, "solves" its share (a stand-in
that returns a record derived from the problem), and the records are gathered; both ranks
must end with every problem exactly once.
"""
import os
import socket

import numpy as np
import pytest

from wavedg_b200 import shard


def _costs():
    rng = np.random.default_rng(4)
    out = []
    for _ in range(29):
        n = int(rng.choice([64, 96, 128, 192, 256]))
        P = int(rng.choice([3, 4, 6]))
        om = float(rng.uniform(10, 40))
        out.append(shard.cost(3 * (P + 1) ** 2 * n * n, P + 1, n, om))
    return out


def test_assignment_partitions_and_balances():
    c = _costs()
    for world in (1, 2, 3, 8):
        parts = shard.assign(c, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(c)))
        loads = [sum(c[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(c) + 1e-9
        assert parts == shard.assign(c, world)  # deterministic


def test_cost_follows_the_period_rule():
    # 128 x 128, P = 4, omega = 20: dt0 = 0.5 (2/128) / 25, nt = ceil(2 pi / 20 / dt0) = 1006
    assert shard.cost(1, 5, 128, 20.0) == 1006.0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = _costs()
        mine = shard.assign(c, world)[rank]
        recs = {i: {"rank": rank, "iterations": 10 + i, "residual": 1e-7 * (i + 1), "status": 0} for i in mine}
        merged = shard.gather_records(recs, world)
        q.put((rank, sorted(merged), {i: merged[i]["rank"] for i in merged}))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gather_every_problem():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n = len(_costs())
    parts = shard.assign(_costs(), 2)
    for rank, idx, owner in res:
        assert idx == list(range(n))
        for r in range(2):
            assert all(owner[i] == r for i in parts[r])
