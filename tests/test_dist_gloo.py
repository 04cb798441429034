"""The multi-rank path of bench.py on CPU: two gloo ranks, each with its own
weak-scaling workload seed, reduce device-timed seconds by max and evaluated
placements by sum (tetris_ai3_b200/dist.py). No GPU needed."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from tetris_ai3_b200 import workload
    from tetris_ai3_b200.dist import rank_seed, reduce_timing
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    b = workload.generation_batch(islands=1, pop=2, games=3, max_moves=10, seed=rank_seed(1, rank))
    secs = 1.5 + rank                          # rank 1 is the slow one
    units = 1000.0 * (rank + 1)
    t, u, rate = reduce_timing(secs, units)
    q.put((rank, t, u, rate, b.weights[0, :3].tolist(), b.seeds.tolist()))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_max_time_and_sum_units():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, t, u, rate, w3, seeds in res:
        assert t == pytest.approx(2.5) and u == pytest.approx(3000.0) and rate == pytest.approx(1200.0)
    assert res[0][4] != res[1][4] and res[0][5] != res[1][5]      # ranks score different generations


def test_single_process_is_identity():
    from tetris_ai3_b200.dist import reduce_timing
    assert reduce_timing(2.0, 10.0) == (2.0, 10.0, 5.0)
