"""Batched uneven solves (semper_b200_batch_run): independent pairs of
different sizes, masks, subsets and steps solved concurrently. Each job must
give exactly what a lone semper_set_reference + semper_run on a fresh handle
gives (results, metrics counts, return code), whatever the worker count and
order. The lone runs themselves are held to the CPU restatement by the
parity tests."""
import numpy as np
import pytest

import semper_b200 as sb

pytestmark = pytest.mark.gpu

COUNT_SLOTS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 15, 16, 19, 20, 21, 22, 23]


def _lone(j):
    e = sb.Engine()
    assert e.set_reference(j["ref"], j.get("mask")) == 0
    return e.run(j["dfm"], j["prm"], capacity=j.get("capacity"), mask=j.get("mask"))


@pytest.fixture(scope="module")
def jobs():
    js = sb.batch_jobs(7, seed=3, min_side=256, max_side=640)
    # uneven extras: a capacity cut, a rect error and a pair with no texture
    js[1]["capacity"] = 8 * 50 + 3
    bad = dict(js[2])
    bad["prm"] = sb.params((0, 0, 64, 64), 8, 20, 21)
    js.append(bad)
    flat = dict(js[3])
    flat["dfm"] = np.full_like(flat["ref"], 128)
    js.append(flat)
    return js


def test_batch_equals_lone_runs(jobs):
    b = sb.Batch(workers=3)
    got = b.run(jobs)
    assert b.last_error == ""
    for j, (rc, pts, met) in zip(jobs, got):
        lrc, lpts, lmet = _lone(j)
        assert rc == lrc
        assert np.array_equal(pts, lpts)
        assert np.array_equal(met[COUNT_SLOTS], lmet[COUNT_SLOTS])
    rcs = [g[0] for g in got]
    assert rcs[1] == 50 and rcs[7] == sb.SEMPER_ERR_INIT and sum(r > 0 for r in rcs) >= 6


def test_batch_independent_of_workers_and_order(jobs):
    a = sb.Batch(workers=1).run(jobs)
    rev = list(reversed(jobs))
    b = list(reversed(sb.Batch(workers=5).run(rev)))
    for (ra, pa, ma), (rb, pb, mb) in zip(a, b):
        assert ra == rb and np.array_equal(pa, pb) and np.array_equal(ma[COUNT_SLOTS], mb[COUNT_SLOTS])


def test_many_workers_mixed_subsets():
    """Engines on many threads launching the same kernels with different
    shared-memory sizes (subsets 15 to 41) at once: every job as when run alone."""
    js = sb.batch_jobs(24, seed=11, min_side=256, max_side=768)
    one = sb.Batch(workers=1).run(js)
    for _ in range(2):
        b = sb.Batch(workers=12)
        many = b.run(js)
        assert b.last_error == ""
        for (ra, pa, _), (rb, pb, _) in zip(one, many):
            assert ra == rb and np.array_equal(pa, pb)


def test_empty_batch():
    assert sb.Batch(workers=2).run([]) == []


def test_batch_on_a_device_list(jobs):
    """Engines created over a device list (every GPU this machine has, each
    listed twice): the jobs as lone runs give them, whichever GPU solves
    them. With one GPU this runs the list's plumbing on device 0."""
    import torch

    devs = [d for d in range(torch.cuda.device_count()) for _ in range(2)]
    b = sb.Batch(workers=4, devices=devs)
    got = b.run(jobs)
    assert b.last_error == ""
    for j, (rc, pts, met) in zip(jobs, got):
        lrc, lpts, _ = _lone(j)
        assert rc == lrc and np.array_equal(pts, lpts)
    assert torch.cuda.current_device() == 0
    b.close()
