"""Multi-rank host logic on CPU: gloo, world size 2 (no GPU)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from blaze_b200.parallel import replica_seed, shard_sims


def test_shard_sims_balances_and_covers():
    cells = [48 ** 3, 64 ** 3, 96 ** 3, 128 * 64 * 64, 64 * 128 * 64] * 13
    for ws in (1, 2, 3, 8):
        parts = shard_sims(cells, ws)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(cells)))
        loads = [sum(cells[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(cells)


def test_shard_sims_deterministic():
    cells = [5, 3, 3, 9, 1, 7]
    assert shard_sims(cells, 2) == shard_sims(list(cells), 2)
    assert shard_sims([], 4) == [[], [], [], []]
    with pytest.raises(ValueError):
        shard_sims(cells, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    from blaze_b200.parallel import max_over_ranks, sum_over_ranks, shard_sims
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank                      # the slower rank sets the time
        t = max_over_ranks(ms)
        steps = sum_over_ranks(3.0)
        mine = shard_sims([100, 50, 50, 25, 25], ws)[rank]
        q.put((rank, t, steps, mine, replica_seed(7, rank)))
    finally:
        dist.destroy_process_group()


def test_two_rank_timing_and_sharding():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]
    assert [o[2] for o in out] == [6.0, 6.0]
    assert sorted(i for o in out for i in o[3]) == [0, 1, 2, 3, 4]
    assert out[0][4] != out[1][4]


def _batch_worker(rank, ws, port, q):
    """The batch benchmark's split of one seeded set of 64 simulations
    (bench.run_batch): each rank takes shard_sims(cells, ws)[rank] and the
    ranks' total cells are summed for the aggregate rate."""
    import datetime
    import torch
    import torch.distributed as dist
    from blaze_b200.parallel import shard_sims, sum_over_ranks
    from blaze_b200.scenes import batch_scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        scenes = batch_scenes(64, seed=4, tol=1e-4, max_iter=20000, check_every=20)
        cells = [s.gridRes[0] * s.gridRes[1] * s.gridRes[2] for s, _ in scenes]
        mine = shard_sims(cells, ws)[rank]
        gathered = [None] * ws
        dist.all_gather_object(gathered, mine)
        total = sum_over_ranks(float(sum(cells[i] for i in mine)))
        q.put((rank, mine, gathered, total, float(sum(cells))))
    finally:
        dist.destroy_process_group()


def test_two_rank_batch_split_covers_the_set_once():
    ws = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_batch_worker, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][2] == out[1][2]                      # both ranks see the same split
    assert sorted(i for o in out for i in o[1]) == list(range(64))
    assert not set(out[0][1]) & set(out[1][1])
    assert out[0][3] == out[0][4] == out[1][3]          # the ranks' cells add up to the whole set
