"""Host side of the multi-GPU path (replicas only), on CPU: the cost-model
sharding of an ensemble and the gloo collectives that gather statistics and
take the max over ranks, with two ranks as separate processes."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import gs_dist


def test_shard_is_a_balanced_partition(gb):
    ps = gb.ensemble_params(gb.GS_DTYPE_F32)
    costs = [gs_dist.sim_cost(p) for p in ps]
    for world in (1, 2, 3, 4, 8):
        parts = gs_dist.shard(costs, world)
        flat = sorted(i for part in parts for i in part)
        assert flat == list(range(len(ps)))
        loads = [sum(costs[i] for i in part) for part in parts]
        # longest-processing-time bound: no rank exceeds the lightest by more than the largest item
        assert max(loads) - min(loads) <= max(costs) + 1e-9
        assert gs_dist.shard(costs, world) == parts  # deterministic


def test_shard_rejects_empty_world():
    with pytest.raises(ValueError):
        gs_dist.shard([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [float(c) for c in np.arange(1, 11)]
        mine = gs_dist.shard(costs, world)[rank]
        local = {i: {"mass": float(i) * 10.0, "rank": rank} for i in mine}
        merged = gs_dist.gather_stats(local, world)
        mx = gs_dist.max_over_ranks(float(rank) + 0.5, world)
        out.put((rank, sorted(merged.items()), mx))
    finally:
        dist.destroy_process_group()


def test_gather_and_max_over_two_gloo_ranks():
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
    res.sort()
    (r0, m0, x0), (r1, m1, x1) = res
    assert m0 == m1  # every rank holds every simulation's stats
    assert [k for k, _ in m0] == list(range(10))
    assert all(v["mass"] == 10.0 * k for k, v in m0)
    assert x0 == x1 == 1.5
