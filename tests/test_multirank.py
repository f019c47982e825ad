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
