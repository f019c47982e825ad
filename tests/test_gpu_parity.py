"""Device stages and the device pipeline against the CPU restatement.

The kernels follow the same arithmetic contract as the restatement (32-lane
partial sums + butterfly, explicit FMA placement, FP64 Hessian), so every
comparison here is exact: integer and flag outputs equal, floating-point
outputs bit-identical.
"""
import numpy as np
import pytest

import oracle
import semper_b200 as sb

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _rng_image(h, w, seed):
    return sb.speckle(w, h, seed)


def _mask_circle(h, w, cx, cy, r):
    yy, xx = np.mgrid[0:h, 0:w]
    m = np.full((h, w), 255, np.uint8)
    m[(xx - cx) ** 2 + (yy - cy) ** 2 < r * r] = 0
    return m


def _planes(img, mask=None):
    t = torch.from_numpy(img).cuda()
    mt = None if mask is None else torch.from_numpy(mask).cuda()
    return sb.image_prep(t, mt)


def test_image_prep_bit_exact():
    img = _rng_image(257, 301, 7)
    mask = _mask_circle(257, 301, 150, 120, 40)
    for m in (None, mask):
        I, gx, gy = _planes(img, m)
        oI, ogx, ogy = oracle.prepare(img, m)
        w = img.shape[1]
        assert np.array_equal(I.cpu().numpy()[:, :w], oI)
        assert np.array_equal(gx.cpu().numpy()[:, :w], ogx)
        assert np.array_equal(gy.cpu().numpy()[:, :w], ogy)
        assert not I.cpu().numpy()[:, w:].any()


@pytest.mark.parametrize("subset", [15, 21, 31, 41])
def test_hessian_pool_bit_exact(subset):
    img = _rng_image(300, 320, 11)
    mask = _mask_circle(300, 320, 160, 150, 30)
    planes = _planes(img, mask)
    step = 7
    gw, gh = 320 // step, 300 // step
    skip = torch.zeros(gw * gh, dtype=torch.uint8, device="cuda")
    valid, ms, H, Hs = sb.hessian_pool(planes, 320, skip, (gw, gh), (0, 0), step, subset)
    xy = np.array([(x * step, y * step) for y in range(gh) for x in range(gw)], np.int32)
    ov, oms, oH = oracle.pool(img, xy, subset, mask)
    assert np.array_equal(valid.cpu().numpy().astype(np.int32), ov)
    assert ov.sum() > 0
    sel = ov == 1
    assert np.array_equal(ms.cpu().numpy()[sel], oms[sel])
    assert np.array_equal(H.cpu().numpy()[sel], oH[sel])


def _solve_case(ref, dfm, xy, guess, mode, subset, lm=True, six=False, mask=None):
    rI = _planes(ref, mask)
    dI, _, _ = _planes(dfm)
    h, w = ref.shape
    n = len(xy)
    # pool rows = task index: a 1 x n "grid" of arbitrary centres
    valid = torch.zeros(n, dtype=torch.uint8, device="cuda")
    ms = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    Hs = torch.zeros((n, 21), dtype=torch.float64, device="cuda")
    for k, (x, y) in enumerate(xy):
        sk = torch.zeros(1, dtype=torch.uint8, device="cuda")
        v1, m1, _h1, hs1 = sb.hessian_pool(rI, w, sk, (1, 1), (int(x), int(y)), 1, subset, lm)
        valid[k] = v1[0]
        ms[k] = m1[0]
        Hs[k] = hs1[0]
    tasks = np.zeros(n, sb.TASK_DT)
    tasks["node"] = np.arange(n)
    tasks["cx"] = xy[:, 0]
    tasks["cy"] = xy[:, 1]
    tasks["mode"] = mode
    tasks["g"] = guess
    res = sb.solve(rI, dI, w, (valid, ms, None, Hs), subset, tasks, lm=lm, six=six)
    fo, io = oracle.solve_nodes(ref, dfm, xy, guess, mode, subset, lm=lm, six=six, mask=mask)
    return res, fo, io


def _assert_same(res, fo, io):
    init = (res["flags"] & 1).astype(np.int32)
    assert np.array_equal(init, io[:, 0])
    sel = io[:, 0] == 1
    assert np.array_equal(res["status"][sel], io[sel, 1])
    assert np.array_equal(res["iters"][sel], io[sel, 2])
    assert np.array_equal(res["invalid_ref"][sel], io[sel, 3])
    assert np.array_equal(((res["flags"] >> 1) & 1)[sel], io[sel, 4])
    assert np.array_equal(res["trigger_iters"][sel], io[sel, 5])
    assert np.array_equal(res["p"][sel], fo[sel])


@pytest.mark.parametrize("six", [False, True])
@pytest.mark.parametrize("mode", [sb.INIT_NO_SIMPLEX, sb.INIT_NO_SEARCH, sb.INIT_AUTO_SEARCH])
def test_solve_bit_exact(six, mode):
    n = 256
    warp = sb.warp_block(cx=128, cy=128, u0=1.3, v0=-0.7, a=(0.01, -0.004, 0.003, -0.006))
    ref = sb.speckle(n, n, 5)
    dfm = sb.speckle(n, n, 5, warp, 1.0, 77)
    rng = np.random.default_rng(3)
    xy = rng.integers(20, n - 20, size=(64, 2)).astype(np.int32)
    guess = np.zeros((64, 6), np.float32)
    if mode != sb.INIT_AUTO_SEARCH:
        guess[:, 0] = 1.0
        guess[:, 1] = -0.5
        guess[::5, 0] = 6.0  # far guesses: failures and rescues
    res, fo, io = _solve_case(ref, dfm, xy, guess, mode, 21, six=six)
    _assert_same(res, fo, io)
    assert (io[:, 1] == 0).sum() > 10


@pytest.mark.parametrize("mode", [sb.INIT_NO_SEARCH, sb.INIT_AUTO_SEARCH])
def test_solve_large_subset_bit_exact(mode):
    # subset 47 (more than 64 pixels per lane) is solved by the unstaged kernel
    n = 256
    ref = sb.speckle(n, n, 4)
    dfm = sb.speckle(n, n, 4, sb.warp_block(cx=128, cy=128, u0=0.7, v0=-1.4, a=(0.004, 0.0, 0.0, -0.003)), 1.0, 9)
    rng = np.random.default_rng(8)
    xy = rng.integers(30, n - 30, size=(24, 2)).astype(np.int32)
    guess = np.zeros((24, 6), np.float32)
    if mode == sb.INIT_NO_SEARCH:
        guess[:, 0], guess[:, 1] = 0.5, -1.0
        guess[::4, 0] = 5.0
    res, fo, io = _solve_case(ref, dfm, xy, guess, mode, 47)
    _assert_same(res, fo, io)
    assert (io[:, 1] == 0).sum() > 5


def test_solve_masked_and_edges_bit_exact():
    n = 200
    ref = sb.speckle(n, n, 9)
    dfm = sb.speckle(n, n, 9, sb.warp_block(u0=2.2, v0=1.1), 0.5, 5)
    mask = _mask_circle(n, n, 100, 100, 25)
    xy = np.array([(x, y) for y in range(16, n - 10, 11) for x in range(16, n - 10, 11)], np.int32)
    guess = np.tile(np.array([2.0, 1.0, 0, 0, 0, 0], np.float32), (len(xy), 1))
    res, fo, io = _solve_case(ref, dfm, xy, guess, sb.INIT_NO_SEARCH, 25, mask=mask)
    _assert_same(res, fo, io)
    # some subsets reach the Ghost Wall, some leave the image
    assert (io[:, 3] > 0).any()


def test_median_vsg_bit_exact():
    rng = np.random.default_rng(1)
    gh, gw = 40, 50
    u = (rng.normal(0, 0.02, (gh, gw)) + np.linspace(0, 1, gw)[None, :]).astype(np.float32)
    v = (rng.normal(0, 0.02, (gh, gw)) + np.linspace(0, -0.5, gh)[:, None]).astype(np.float32)
    u[10, 10] += 5.0
    v[20:23, 30:33] -= 4.0
    valid = (rng.random((gh, gw)) > 0.1).astype(np.uint8)
    rej, val, st = oracle.median_vsg(u, v, valid, 6, 21)
    drej, dval, exx, eyy, exy = sb.median_vsg(torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda(),
                                              torch.from_numpy(valid).cuda(), 6, 21)
    assert drej == rej and rej > 0
    assert np.array_equal(dval.cpu().numpy(), val)
    assert np.array_equal(np.stack([exx.cpu().numpy(), eyy.cpu().numpy(), exy.cpu().numpy()], -1), st)


def _run_both(ref, dfm, prm, mask=None, capacity=None):
    """The device engine (global motion on, its default) and the restatement
    given the model the device estimated, as the reference's golden scenarios
    inject their AKAZE model."""
    e = sb.Engine()
    assert e.set_reference(ref, mask) == 0
    rc, pts, met = e.run(dfm, prm, capacity=capacity, mask=mask)
    g = e.last_global_motion()
    o = oracle.Oracle(False)
    o.set_reference(ref, mask)
    p = [prm.rect_x, prm.rect_y, prm.rect_w, prm.rect_h, prm.step, prm.subset_size, prm.strain_window,
         prm.use_6x6_interpolator]
    orc, opts, omet = o.run(dfm, p, capacity=capacity, mask=mask, model_h=g["H"] if g["locked"] else None)
    return (rc, pts, met), (orc, opts, omet)


COUNT_SLOTS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 15, 16, 19, 20, 21, 22, 23]


def _assert_field_equal(d, o):
    assert d[0] == o[0]
    assert np.array_equal(d[1], o[1])
    assert np.array_equal(d[2][COUNT_SLOTS], o[2][COUNT_SLOTS])


def test_pipeline_cfg0_bit_exact():
    ref, dfm, prm, _ = sb.config_pair(0)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 1500
    _assert_field_equal(d, o)


def test_pipeline_golden_inputs_bit_exact():
    for s in (0, 1):
        ref, dfm = oracle.ff_inputs(s)
        d, o = _run_both(ref, dfm, sb.params((0, 0, 320, 320), 12, 21, 48))
        _assert_field_equal(d, o)


def test_pipeline_masked_6x6_and_capacity():
    ref, dfm, _, _ = sb.config_pair(0, size=384)
    mask = _mask_circle(384, 384, 190, 200, 60)
    prm = sb.params((10, 20, 360, 340), 8, 25, 33, six=True)
    d, o = _run_both(ref, dfm, prm, mask=mask)
    _assert_field_equal(d, o)
    d, o = _run_both(ref, dfm, prm, mask=mask, capacity=8 * 100 + 5)
    assert d[0] == o[0] == 100
    _assert_field_equal(d, o)


def test_pipeline_cfg1_small_bit_exact():
    ref, dfm, prm, _ = sb.config_pair(1, size=768)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 20000
    _assert_field_equal(d, o)


def test_return_codes():
    ref, dfm, prm, _ = sb.config_pair(0, size=256)
    e = sb.Engine()
    assert e.run(dfm, prm)[0] == sb.SEMPER_ERR_INIT  # no reference
    assert e.set_reference(ref) == 0
    assert e.run(dfm, sb.params((0, 0, 256, 256), 0, 21, 21))[0] == sb.SEMPER_ERR_ROI
    assert e.run(dfm, sb.params((0, 0, 256, 256), 8, 20, 21))[0] == sb.SEMPER_ERR_INIT
    assert e.run(dfm, sb.params((0, 0, 256, 256), 8, 15, 8))[0] == sb.SEMPER_ERR_STRAIN_WINDOW
    assert e.run(dfm, sb.params((300, 0, 10, 10), 8, 15, 15))[0] == sb.SEMPER_ERR_ROI
    assert e.run(dfm[:100], prm)[0] == sb.SEMPER_ERR_INIT


def test_pipeline_unpadded_width_bit_exact():
    # width not a multiple of 4: the device planes carry a padded pitch
    w, h = 330, 300
    ref = sb.speckle(w, h, 21)
    dfm = sb.speckle(w, h, 21, sb.warp_block(cx=165, cy=150, u0=-1.2, v0=0.6, a=(0.004, 0.0, 0.0, 0.003)), 1.0, 3)
    d, o = _run_both(ref, dfm, sb.params((0, 0, w, h), 9, 21, 27))
    assert o[0] > 100
    _assert_field_equal(d, o)


def test_autotuned_fast_pass_shapes_agree():
    """The engine's autotuner alternates the first four Path A launches
    between the reference read from the planes and staged, then keeps the
    faster: every run of the same frame must give the same field."""
    ref, dfm, prm, _ = sb.config_pair(1, size=768)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    assert e.fast_pass_shape(prm.subset_size) == -1
    runs = [e.run(dfm, prm) for _ in range(5)]
    assert e.fast_pass_shape(prm.subset_size) in (0, 1)
    for rc, pts, met in runs[1:]:
        assert rc == runs[0][0] and np.array_equal(pts, runs[0][1])
        assert np.array_equal(met[COUNT_SLOTS], runs[0][2][COUNT_SLOTS])


def test_run_device_equals_run():
    """semper_b200_run_device (frame and output in device memory) gives the
    points semper_run gives for the same frame."""
    import torch

    ref, dfm, prm, _ = sb.config_pair(0, size=384)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    rc, pts, met = e.run(dfm, prm)
    cap = (prm.rect_w // prm.step) * (prm.rect_h // prm.step) * 8
    d_def = torch.from_numpy(dfm).cuda()
    d_out = torch.zeros(cap, dtype=torch.float32, device="cuda")
    rc2, met2 = e.run_device(d_def, prm, d_out, cap)
    torch.cuda.synchronize()
    assert rc2 == rc > 0
    assert np.array_equal(d_out[: rc * 8].cpu().numpy().reshape(-1, 8), pts)
    assert np.array_equal(met2[COUNT_SLOTS], met[COUNT_SLOTS])


def _long_pair():
    """A pair whose lattice does not reach full quality (a masked 1745^2 frame
    at subset 31, step 4): Path B's rounds take it, some 4,000 of them, so a
    solve lasts hundreds of milliseconds and polls the cancel flag in every
    round."""
    return sb.batch_jobs(3, seed=0)[2]


def test_cancel_during_run():
    """semper_cancel from inside the run (the progress callback, which the
    engine's ticker thread calls as soon as seeding starts) ends it with
    SEMPER_ERR_CANCELLED; the next run on the handle is unaffected, and a
    cancel between runs does not carry over."""
    j = _long_pair()
    e = sb.Engine()
    assert e.set_reference(j["ref"], j["mask"]) == 0
    seen = []

    def cb(pct, user):
        seen.append(pct)
        e.cancel()

    rc, _, _ = e.run(j["dfm"], j["prm"], mask=j["mask"], progress=cb)
    assert seen and rc == sb.SEMPER_ERR_CANCELLED
    rc2, pts, _ = e.run(j["dfm"], j["prm"], mask=j["mask"])
    assert rc2 > 0
    e.cancel()
    rc3, pts3, _ = e.run(j["dfm"], j["prm"], mask=j["mask"])
    assert rc3 == rc2 and np.array_equal(pts3, pts)


def test_pipeline_cfg1_2048_bit_exact():
    """cfg1's field and full solve settings (step 4, subset 31, window 31) on a
    2048^2 frame: 259k grid nodes, bit for bit."""
    ref, dfm, prm, _ = sb.config_pair(1, size=2048)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 230000
    _assert_field_equal(d, o)


def test_pipeline_target_settings_2048_bit_exact():
    """The target settings (step 8, subset 41, window 41) under the cfg1 field
    on a 2048^2 frame, bit for bit."""
    ref, dfm, prm, _ = sb.config_pair(4, size=2048)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 55000
    _assert_field_equal(d, o)


def test_pipeline_cfg1_4096_bit_exact():
    """The headline workload itself: cfg1 at 4096^2 (step 4, subset 31, window
    31; 1,014,049 attempted nodes), the device field against the CPU
    restatement's, bit for bit."""
    ref, dfm, prm, _ = sb.config_pair(1)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 1000000
    _assert_field_equal(d, o)


def test_pipeline_target_settings_4096_bit_exact():
    """The target settings at their full size: 4096^2, step 8, subset 41,
    window 41, bit for bit."""
    ref, dfm, prm, _ = sb.config_pair(4)
    d, o = _run_both(ref, dfm, prm)
    assert o[0] > 240000
    _assert_field_equal(d, o)


def test_batch_cfg2_jobs_against_restatement():
    """Eight pairs of the batched uneven workload (masks, rotations, subsets
    15-41, steps 4 and 8), solved in one batch call, each against the CPU
    restatement given the global model a lone device run estimates."""
    jobs = sb.batch_jobs(8, seed=22, min_side=256, max_side=1024)
    got = sb.Batch(workers=4).run(jobs)
    positive = 0
    for j, (rc, pts, met) in zip(jobs, got):
        e = sb.Engine()
        assert e.set_reference(j["ref"], j["mask"]) == 0
        lrc, _, _ = e.run(j["dfm"], j["prm"], mask=j["mask"])
        assert lrc == rc
        g = e.last_global_motion()
        o = oracle.Oracle(False)
        o.set_reference(j["ref"], j["mask"])
        p = j["prm"]
        orc, opts, omet = o.run(j["dfm"], [p.rect_x, p.rect_y, p.rect_w, p.rect_h, p.step, p.subset_size,
                                           p.strain_window, 0], mask=j["mask"],
                                model_h=g["H"] if g["locked"] else None)
        _assert_field_equal((rc, pts, met), (orc, opts, omet))
        positive += rc > 0
    assert positive >= 5 and sb.SEMPER_ERR_STRAIN_WINDOW in [g[0] for g in got]


def test_tma_wait_that_runs_out_falls_back_bit_exact():
    """The solve's TMA waits given a limit of one poll: the first tile copy of
    (nearly) every warp is still in flight when its wait gives up, so the warp
    samples global memory from then on, and waits for the late copy before it
    exits. The run reports the timeout, and its field is the CPU restatement's,
    bit for bit, as with the default limit."""
    ref, dfm, prm, _ = sb.config_pair(1, size=512)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    rc0, pts0, met0 = e.run(dfm, prm)
    assert e.last_tma_timeout() == 0
    assert e.set_tma_wait_limit(1) == 0
    rc1, pts1, met1 = e.run(dfm, prm)
    assert e.last_tma_timeout() == 1
    assert rc1 == rc0 > 10000
    assert np.array_equal(pts1, pts0)
    assert np.array_equal(met1[COUNT_SLOTS], met0[COUNT_SLOTS])
    g = e.last_global_motion()
    o = oracle.Oracle(False)
    o.set_reference(ref)
    p = [prm.rect_x, prm.rect_y, prm.rect_w, prm.rect_h, prm.step, prm.subset_size, prm.strain_window, 0]
    orc, opts, _ = o.run(dfm, p, model_h=g["H"] if g["locked"] else None)
    assert orc == rc1 and np.array_equal(pts1, opts)
    assert e.set_tma_wait_limit(0) == 0
    rc2, pts2, _ = e.run(dfm, prm)
    assert e.last_tma_timeout() == 0 and np.array_equal(pts2, pts0)


def test_path_c_seed_bit_exact():
    """Path C seeds the field: the anchor lattice's nodes are all masked
    (tests/scenarios.py) and the global-motion front end is off (the
    reference without an AKAZE model), so the routing finds no seed and the
    central search's first converging candidate starts the Path B flood. The
    device field equals the CPU restatement's, bit for bit, with the metrics
    showing no anchor, no Path A point and every point from Path B. With the
    front end on (its default) the model's guess field feeds Path A instead,
    and the two still agree."""
    import scenarios

    ref, dfm, mask, prm = scenarios.lattice_masked_pair()
    e = sb.Engine()
    assert e.set_global_motion(False) == 0
    assert e.set_reference(ref, mask) == 0
    d = e.run(dfm, prm, mask=mask)
    o = oracle.Oracle(False)
    o.set_reference(ref, mask)
    p = [prm.rect_x, prm.rect_y, prm.rect_w, prm.rect_h, prm.step, prm.subset_size, prm.strain_window, 0]
    ores = o.run(dfm, p, mask=mask)
    met = d[2]
    assert d[0] > 2000
    assert met[16] == 0 and met[19] == 0 and met[21] == 0 and met[3] == 0 and met[4] > 3000
    _assert_field_equal(d, ores)
    d2, o2 = _run_both(ref, dfm, prm, mask=mask)
    assert d2[0] > 2000
    _assert_field_equal(d2, o2)
