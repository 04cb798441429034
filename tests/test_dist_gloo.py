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


TRAIN_CFG = dict(islands=4, population=8, gens_per_iteration=3, iterations_per_cycle=2, games=3, max_moves=50)


def _quadratic(w, seeds, max_moves):
    import numpy as np
    target = np.linspace(-1.0, 1.0, w.shape[1])
    base = -((w.astype(np.float64) - target) ** 2).sum(1)
    return (base[:, None] + (seeds % 5)[None, :] * 0.01).astype(np.float32)


def _train_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from tetris_ai3_b200 import trainer as tr
    from tetris_ai3_b200.dist import island_group_score
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    seen = []

    def local(w, seeds, max_moves):            # this rank's "GPU": records the rows it scores
        seen.append(w.shape[0])
        return _quadratic(w, seeds, max_moves)

    t = tr.Trainer(tr.default_config(**TRAIN_CFG), score=island_group_score(local, TRAIN_CFG["islands"]))
    t.run(4)
    champs = [(x.tobytes(), f) for x, f in (t.champion(i) for i in range(4))]
    q.put((rank, champs, seen, t.stats()["evaluations"]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_split_a_training_run_by_island_group():
    """Two ranks, each scoring its own island group (islands 0, 2 / 1, 3) and all-gathering the
    generation: both ranks end with the single-process run's champions bit for bit, the ring
    migration having moved individuals between islands scored on different ranks."""
    from tetris_ai3_b200 import trainer as tr
    one = tr.Trainer(tr.default_config(**TRAIN_CFG), score=_quadratic)
    one.run(4)
    want = [(x.tobytes(), f) for x, f in (one.champion(i) for i in range(4))]
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_train_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, champs, seen, evals in res:
        assert champs == want
        assert evals == one.stats()["evaluations"]
        assert set(seen) == {16}                   # 2 islands x 8 candidates per call on each rank
