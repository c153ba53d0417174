"""Multi-rank host logic on CPU: two gloo ranks shard seeds and ladders, take
the max of their timings and agree on the global best state."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from __graft_entry__ import load_package

    load_package()
    from no_three_in_line_b200 import shard, state
    from oracle import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        seeds = shard.seed_block(rank, world, 8)
        p, q = state.seeded_population(20, 8, base_seed=seeds.start)
        scores = oracle.score_population(p, q, threads=1)
        b = int(np.argmin(scores))
        cols = state.pq_to_columns(p[b], q[b])
        e, winner, best = shard.global_best(int(scores[b]), cols)
        t = shard.max_over_ranks(0.5 + rank)
        out.put((rank, list(seeds), [list(shard.ladder_block(5, r, world)) for r in range(world)],
                 int(scores.min()), e, winner, best.tolist(), t))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    (r0, s0, lad0, m0, e0, w0, b0, t0), (r1, s1, lad1, m1, e1, w1, b1, t1) = res
    assert s0 == list(range(91001, 91009)) and s1 == list(range(91009, 91017))
    assert lad0 == lad1 == [[0, 1], [2, 3, 4]]
    assert e0 == e1 == min(m0, m1) and w0 == w1 == (0 if m0 <= m1 else 1)
    assert b0 == b1
    from oracle import oracle

    assert oracle.score_columns(np.asarray(b0))[0] == e0
    assert t0 == t1 == 1.5


def test_block_helpers_reject_bad_ranks():
    from no_three_in_line_b200 import shard

    with pytest.raises(ValueError):
        shard.seed_block(2, 2, 4)
    with pytest.raises(ValueError):
        shard.ladder_block(4, -1, 2)
    assert sum(len(shard.ladder_block(32, r, 3)) for r in range(3)) == 32
