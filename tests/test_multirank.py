"""The multi-GPU path of the benchmark without a GPU: two gloo ranks on CPU.

Ranks are independent replicas (each solves its own frame pair, its own
speckle seed); the only cross-rank step is the aggregation, max time and
summed points, which must give the same whole-job throughput on every rank.
"""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "semper-dic-engine_b200"))
    import bench
    import semper_b200 as sb

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        pts = [1000, 1200][rank]
        ms = [50.0, 80.0][rank]
        value, ms_max = bench.aggregate(pts * 3, ms, 3, dist, "cpu")
        ref, dfm, _prm, _w = sb.config_pair(0, size=64, pair=rank)
        q.put((rank, value, ms_max, int(ref.sum()), int(dfm.sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_and_own_pairs():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expected = (1000 + 1200) / (80.0 / 1000.0)
    for _rank_id, value, ms_max, _r, _d in res:
        assert ms_max == 80.0
        assert abs(value - expected) < 1e-6 * expected
    # every rank has its own frame pair
    assert res[0][3] != res[1][3] and res[0][4] != res[1][4]


def _shard_rank(rank, world, port, q):
    """One rank of a sharded batch: it takes its jobs by semper_b200.shard,
    solves each (the CPU restatement stands in for the device solve on this
    GPU-less machine), and the ranks' point totals are summed over gloo."""
    import datetime
    import hashlib

    import torch
    import torch.distributed as dist

    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "semper-dic-engine_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    import semper_b200 as sb

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        params = sb.batch_job_params(8, seed=5, min_side=160, max_side=288)
        mine = sb.shard([sb.job_cost(p) for p, _ in params], rank, world)
        jobs = sb.batch_jobs(8, seed=5, min_side=160, max_side=288, only=mine)
        out = []
        pts = 0
        for j in jobs:
            o = oracle.Oracle(False)
            o.set_reference(j["ref"], j["mask"])
            p = j["prm"]
            rc, res, _ = o.run(j["dfm"], [0, 0, p.rect_w, p.rect_h, p.step, p.subset_size, p.strain_window, 0],
                               mask=j["mask"])
            out.append((j["index"], int(rc), hashlib.sha1(res.tobytes()).hexdigest()))
            pts += max(int(rc), 0)
        t = torch.tensor([float(pts)], dtype=torch.float64)
        dist.all_reduce(t)
        q.put((rank, out, float(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_a_batch_and_solve_it():
    """A batch split over two ranks by cost: every job is solved by exactly
    one rank, each with the result a single process gives it, and the summed
    point total over the ranks is the single process's."""
    import hashlib

    sys.path.insert(0, os.path.join(REPO, "semper-dic-engine_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    import semper_b200 as sb

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = sorted(sum((r[1] for r in res), []))
    assert [g[0] for g in got] == list(range(8))
    assert res[0][2] == res[1][2]
    whole = []
    for j in sb.batch_jobs(8, seed=5, min_side=160, max_side=288):
        o = oracle.Oracle(False)
        o.set_reference(j["ref"], j["mask"])
        p = j["prm"]
        rc, pts, _ = o.run(j["dfm"], [0, 0, p.rect_w, p.rect_h, p.step, p.subset_size, p.strain_window, 0],
                           mask=j["mask"])
        whole.append((j["index"], int(rc), hashlib.sha1(pts.tobytes()).hexdigest()))
    assert got == whole
    assert res[0][2] == sum(max(w[1], 0) for w in whole) > 0
    costs = [sb.job_cost(p) for p, _ in sb.batch_job_params(8, seed=5, min_side=160, max_side=288)]
    loads = [sum(costs[g[0]] for g in r[1]) for r in res]
    assert max(loads) <= sum(costs) / 2 + max(costs)


def test_shard_covers_every_job_once_and_balances():
    """semper_b200.shard: every index on exactly one rank, the same split on
    every call, the largest jobs spread first (no rank above the mean by more
    than the largest job); batch_jobs with `only` draws the same jobs."""
    sys.path.insert(0, os.path.join(REPO, "semper-dic-engine_b200"))
    import semper_b200 as sb

    jobs = sb.batch_job_params(256, seed=0)
    costs = [sb.job_cost(p) for p, _ in jobs]
    for world in (1, 2, 3, 8):
        parts = [sb.shard(costs, r, world) for r in range(world)]
        assert sorted(sum(parts, [])) == list(range(256))
        assert parts == [sb.shard(costs, r, world) for r in range(world)]
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)
    few = sb.batch_jobs(6, seed=2, min_side=64, max_side=96)
    some = sb.batch_jobs(6, seed=2, min_side=64, max_side=96, only=[4, 1])
    assert [j["index"] for j in some] == [1, 4]
    for j in some:
        k = j["index"]
        assert np.array_equal(j["ref"], few[k]["ref"]) and np.array_equal(j["dfm"], few[k]["dfm"])
        assert (j["mask"] is None) == (few[k]["mask"] is None)
    assert [m for _, m in sb.batch_job_params(6, seed=2, min_side=64, max_side=96)] == \
        [j["mask"] is not None for j in few]
