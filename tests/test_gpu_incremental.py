"""IncrementalSession on the device against the same session over the CPU
restatement (include/semper/incremental.hpp; tests/integration/
test_incremental.cpp of the reference for the contracts checked here).

The device session (per-node state and steps as kernels, incnode.cu and
inc_session.cpp) and the CPU restatement's session
(oracle/src/incremental_session.hpp) are separate implementations of the
same rules; their solves, reference adoptions and packing agree bit for bit,
so every frame's points, return code and frame info must be identical.
"""
import numpy as np
import pytest

import oracle
import semper_b200 as sb

pytestmark = pytest.mark.gpu

COUNT_SLOTS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 15, 16, 19, 20, 21, 22, 23]


def sequence(n=256, frames=6, seed=31):
    ref = sb.speckle(n, n, seed)
    out = []
    for t in range(1, frames + 1):
        a = 0.004 * t
        w = sb.warp_block(cx=n / 2, cy=n / 2, u0=0.9 * t, v0=-0.5 * t, a=(a, 0.0, 0.0, -0.5 * a))
        out.append(sb.speckle(n, n, seed, w, 1.0, 100 + t))
    return ref, out


def run_both(ref, frames, prm_list, interval, mask=None):
    n = ref.shape[0]
    dev = sb.Incremental()
    ora = oracle.IncrementalOracle()
    assert dev.init(ref, sb.params(*prm_list), interval, mask=mask) == 0
    assert ora.init(ref, [*prm_list[0], prm_list[1], prm_list[2], prm_list[3], 0], interval, mask=mask) == 0
    cap = (n // prm_list[1]) ** 2 * 8
    rows = []
    for f in frames:
        d = dev.process(f, cap)
        o = ora.process(f, cap)
        rows.append((d, o))
    return rows


def assert_same(d, o):
    rc, pts, met, info = d
    orc, opts, omet, oinfo = o
    assert rc == orc
    assert np.array_equal(pts, opts)
    assert np.array_equal(met[COUNT_SLOTS], omet[COUNT_SLOTS])
    got = [info.reference_frame, info.reference_updated, info.tracked_points, info.frame0_points,
           info.taylor_fallbacks, info.lost_this_frame]
    assert got == oinfo.tolist()


@pytest.mark.parametrize("interval", [0, 1, 3])
def test_session_matches_restatement(interval):
    ref, frames = sequence()
    rows = run_both(ref, frames, ((16, 16, 224, 224), 8, 21, 21), interval)
    for d, o in rows:
        assert_same(d, o)
        assert d[0] > 400
    updated = [d[3].reference_updated for d, _ in rows]
    if interval == 0:
        assert not any(updated)
    elif interval == 1:
        assert all(updated)
    else:
        assert updated[2] and updated[5]


def test_masked_session_matches_restatement():
    ref, frames = sequence(seed=17)
    yy, xx = np.mgrid[0:256, 0:256]
    mask = np.full((256, 256), 255, np.uint8)
    mask[(xx - 140) ** 2 + (yy - 120) ** 2 < 30 ** 2] = 0
    rows = run_both(ref, frames[:4], ((16, 16, 224, 224), 8, 21, 21), 2, mask=mask)
    for d, o in rows:
        assert_same(d, o)


def test_interval_zero_is_a_fixed_reference_run():
    ref, frames = sequence(frames=3)
    prm = sb.params((16, 16, 224, 224), 8, 21, 21)
    inc = sb.Incremental()
    assert inc.init(ref, prm, 0) == 0
    e = sb.Engine()
    e.set_global_motion(False)  # the session solves without a global model
    assert e.set_reference(ref) == 0
    for f in frames:
        rc, pts, _met, _info = inc.process(f, 28 * 28 * 8)
        rc2, pts2, _m2 = e.run(f, prm)
        assert rc == rc2 and np.array_equal(pts, pts2)


def test_first_frame_is_a_fixed_reference_run():
    ref, frames = sequence(frames=1)
    prm = sb.params((16, 16, 224, 224), 8, 21, 21)
    inc = sb.Incremental()
    assert inc.init(ref, prm, 1) == 0
    rc, pts, _met, info = inc.process(frames[0], 28 * 28 * 8)
    e = sb.Engine()
    e.set_global_motion(False)
    assert e.set_reference(ref) == 0
    rc2, pts2, _m2 = e.run(frames[0], prm)
    assert rc == rc2 and np.array_equal(pts, pts2)
    assert info.reference_updated == 1 and info.frame0_points == 625


def test_cancel_during_frame():
    """semper_incremental_cancel from inside a frame ends it with
    SEMPER_ERR_CANCELLED and leaves the session as it was: the frame processed
    again gives what an uncancelled session gives. The pair is one whose solve
    runs through thousands of Path B rounds (a masked 1745^2 frame at subset
    31, step 4), so the cancel, raised by the progress callback when seeding
    starts, is seen by a later round."""
    j = sb.batch_jobs(3, seed=0)[2]
    prm = j["prm"]
    cap = (prm.rect_w // prm.step) * (prm.rect_h // prm.step) * 8
    a, b = sb.Incremental(), sb.Incremental()
    assert a.init(j["ref"], prm, 1, mask=j["mask"]) == 0 and b.init(j["ref"], prm, 1, mask=j["mask"]) == 0
    rc, _, _, _ = a.process(j["dfm"], cap, progress=lambda pct, user: a.cancel())
    assert rc == sb.SEMPER_ERR_CANCELLED
    ra, pa, _, ia = a.process(j["dfm"], cap)
    rb, pb, _, ib = b.process(j["dfm"], cap)
    assert ra == rb > 0 and np.array_equal(pa, pb)
    assert ia.reference_frame == ib.reference_frame


def occluder_sequence(n=320, frames=12, seed=41, speed=2.0):
    """Material translating and stretching under a stationary, textureless
    occluder that appears small (frames 2-3), grows (frames 4-7) and goes.
    Nodes beside the small one get anchors (a gap within reach), coast on
    fitted planes while the large one covers them, and when it goes are
    confirmed only by direct matches of those anchors."""
    ref = sb.speckle(n, n, seed)
    out = []
    for t in range(1, frames + 1):
        w = sb.warp_block(cx=n / 2, cy=n / 2, u0=speed * t, v0=-0.5 * t, a=(0.002 * t, 0.0, 0.0, -0.001 * t))
        f = sb.speckle(n, n, seed, w, 1.0, 300 + t)
        if 2 <= t <= 3:
            f[148:172, 148:172] = 128
        if 4 <= t <= 7:
            f[112:208, 112:208] = 128
        out.append(f)
    return ref, out


@pytest.mark.parametrize("interval", [1, 2])
def test_coasting_and_anchor_matches_match_restatement(interval):
    ref, frames = occluder_sequence()
    dev = sb.Incremental()
    ora = oracle.IncrementalOracle()
    assert dev.init(ref, sb.params((16, 16, 288, 288), 8, 21, 21), interval) == 0
    assert ora.init(ref, [16, 16, 288, 288, 8, 21, 21, 0], interval) == 0
    cap = 36 * 36 * 8
    matches = taylor = 0
    for f in frames:
        d = dev.process(f, cap)
        o = ora.process(f, cap)
        assert_same(d, o)
        matches += int(dev.profile()["matches"])
        taylor += d[3].taylor_fallbacks
    print(f"interval {interval}: {matches} anchor matches, {taylor} Taylor samples")
    assert taylor > 0
    assert matches > 0


def test_batched_sequences_match_restatement():
    """Three sequences (own seeds, update intervals and one with a mask)
    advanced together by semper_b200_inc_batch_process, their solves
    interleaved on the device: every frame of every sequence equals the CPU
    restatement's session on that sequence alone, bit for bit."""
    prm = ((16, 16, 224, 224), 8, 21, 21)
    yy, xx = np.mgrid[0:256, 0:256]
    mask = np.full((256, 256), 255, np.uint8)
    mask[(xx - 120) ** 2 + (yy - 140) ** 2 < 25 ** 2] = 0
    setups = [(31, 1, None), (17, 3, mask), (53, 0, None)]
    seqs = [sequence(seed=s, frames=5) for s, _, _ in setups]
    cap = (256 // 8) ** 2 * 8
    b = sb.IncrementalBatch(len(setups))
    oras = []
    for q, ((seed, interval, m), (ref, _)) in enumerate(zip(setups, seqs)):
        assert b.init(q, ref, sb.params(*prm), interval, mask=m) == 0
        o = oracle.IncrementalOracle()
        assert o.init(ref, [*prm[0], prm[1], prm[2], prm[3], 0], interval, mask=m) == 0
        oras.append(o)
    for t in range(5):
        got = b.process({q: seqs[q][1][t] for q in range(len(setups))}, cap)
        for q in range(len(setups)):
            assert_same(got[q], oras[q].process(seqs[q][1][t], cap))
            assert got[q][0] > 300
    # a sequence named twice, or out of range, is refused
    arr = (sb.IncFrame * 2)()
    arr[0].sequence = arr[1].sequence = 0
    assert sb.lib().semper_b200_inc_batch_process(b._h, arr, 2) == sb.SEMPER_ERR_INIT
    arr[1].sequence = 7
    assert sb.lib().semper_b200_inc_batch_process(b._h, arr, 2) == sb.SEMPER_ERR_INIT
    b.close()


def test_batched_sequences_on_a_device_list():
    """Sessions created over a device list (every GPU, each listed twice):
    each sequence as its lone session gives it."""
    import torch

    devs = [d for d in range(torch.cuda.device_count()) for _ in range(2)]
    prm = ((16, 16, 224, 224), 8, 21, 21)
    seqs = [sequence(seed=s, frames=3) for s in (31, 53)]
    cap = (256 // 8) ** 2 * 8
    b = sb.IncrementalBatch(2, devices=devs)
    lone = []
    for q, (ref, _) in enumerate(seqs):
        assert b.init(q, ref, sb.params(*prm), 1) == 0
        s = sb.Incremental()
        assert s.init(ref, sb.params(*prm), 1) == 0
        lone.append(s)
    for t in range(3):
        got = b.process({q: seqs[q][1][t] for q in range(2)}, cap)
        for q in range(2):
            rc, pts, _, _ = lone[q].process(seqs[q][1][t], cap)
            assert got[q][0] == rc > 300 and np.array_equal(got[q][1], pts)
    b.close()
