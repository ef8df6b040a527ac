"""Multi-rank host logic on CPU: two gloo ranks split grids and requests
without exchanging data, the split is a partition, and the timing reduction
takes the max over ranks."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from openfpm_data_b200 import shard as S
from openfpm_data_b200 import workloads as W


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        _, radii, _ = W.batch_grids(256)
        weights = [float(r) ** 3 for r in radii]
        grids = S.shard_weighted(weights, rank, world)
        reqs = W.requests(duration=0.2, seed=4)
        mine = [r.rid for r in S.shard_requests(reqs, rank, world)]
        lo, hi = S.shard_range(1000, rank, world)
        gathered = [None] * world
        dist.all_gather_object(gathered, {"grids": grids, "rids": mine, "range": (lo, hi),
                                          "load": sum(weights[i] for i in grids)})
        t = S.max_over_ranks(1.0 + rank)
        if rank == 0:
            out.put((gathered, t, len(reqs), sum(weights)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_partition_the_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered, tmax, nreq, wsum = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    g0, g1 = gathered
    assert sorted(g0["grids"] + g1["grids"]) == list(range(256))
    assert not set(g0["grids"]) & set(g1["grids"])
    assert abs(g0["load"] - g1["load"]) <= 0.05 * wsum  # balanced by active points
    assert sorted(g0["rids"] + g1["rids"]) == list(range(nreq))
    assert g0["range"] == (0, 500) and g1["range"] == (500, 1000)
    assert tmax == 2.0


def _bench_worker(rank, world, port, out):
    """The split bench.py's batched and served runners use, driven from gloo ranks."""
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["WORLD_SIZE"] = str(world)
    os.environ["RANK"] = str(rank)
    d = bench.Dist(world)  # gloo on a CPU-only host
    try:
        all_specs, mine = bench.batched_shard(d.rank, d.world)
        all_reqs, reqs = bench.served_shard(2000.0, 0.5, d.rank, d.world)
        parts = d.gather({"grids": mine, "rids": [r.rid for r in reqs], "nspecs": len(all_specs),
                          "nreqs": len(all_reqs)})
        if rank == 0:
            single_specs, single = bench.batched_shard(0, 1)
            single_reqs, _ = bench.served_shard(2000.0, 0.5, 0, 1)
            out.put((parts, single, [r.rid for r in single_reqs]))
    finally:
        d.close()


def test_bench_runners_split_is_a_partition_of_the_single_gpu_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    parts, single, single_rids = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(parts[0]["grids"] + parts[1]["grids"]) == sorted(single) == list(range(256))
    assert not set(parts[0]["grids"]) & set(parts[1]["grids"])
    assert sorted(parts[0]["rids"] + parts[1]["rids"]) == sorted(single_rids)
    assert not set(parts[0]["rids"]) & set(parts[1]["rids"])
    assert parts[0]["nreqs"] == parts[1]["nreqs"] == len(single_rids)


def test_shard_helpers_single_process():
    assert S.shard_range(10, 0, 1) == (0, 10)
    assert S.shard_weighted([3.0, 1.0, 2.0], 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        S.shard_range(10, 2, 2)
    assert S.max_over_ranks(3.5) == 3.5
