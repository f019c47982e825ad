"""Global motion on the device: the phase-correlation similarity that stands in
for the reference's AKAZE + RANSAC model (src/pipeline/akaze_features.cpp:
122-182; src/pipeline/full_field_anchors.cpp:204-279 uses it to seed the
anchor lattice).

The estimate itself has no reference counterpart to be bit-exact with: it is
checked against the known warps of synthetic pairs. Its use is checked the
way the reference's own golden scenarios with an AKAZE model are (the model
injected into the CPU restatement): the full-field result with the estimated
model must equal, bit for bit, the restatement's result with that model.
"""
import math

import numpy as np
import pytest

import oracle
import semper_b200 as sb

pytestmark = pytest.mark.gpu

COUNT_SLOTS = [0, 1, 2, 3, 4, 5, 6, 7, 8, 15, 16, 19, 20, 21, 22, 23]


def _pair(deg, s, t, n=1024, seed=5, other_seed=None):
    th = math.radians(deg)
    a = (s * math.cos(th) - 1, -s * math.sin(th), s * math.sin(th), s * math.cos(th) - 1)
    warp = sb.warp_block(cx=n / 2, cy=n / 2, u0=t[0], v0=t[1], a=a)
    ref = sb.speckle(n, n, seed)
    dfm = sb.speckle(n, n, seed if other_seed is None else other_seed, warp, 1.0, 9)
    return ref, dfm, warp


def _estimate(ref, dfm, rect):
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    e.run(dfm, sb.params(rect, 8, 21, 21))
    return e.last_global_motion()


@pytest.mark.parametrize("deg,s,t", [(0, 1.0, (7.3, -4.2)), (20, 1.0, (0.0, 0.0)), (60, 1.0, (25.0, -12.0)),
                                     (135, 1.05, (-30.0, 18.0)), (170, 0.97, (10.0, 40.0)),
                                     (-45, 1.0, (-15.5, 3.25))])
def test_similarity_recovered(deg, s, t):
    ref, dfm, warp = _pair(deg, s, t)
    rect = (128, 128, 768, 768)
    g = _estimate(ref, dfm, rect)
    assert g["locked"], g
    dth = (g["theta"] - math.radians(deg) + math.pi) % (2 * math.pi) - math.pi
    assert abs(dth) < math.radians(0.15), (g["theta"], deg)
    assert abs(g["scale"] - s) < 3e-3
    # the homography carries the ROI corners and centre within a pixel of the true warp
    H = g["H"]
    X = np.array([128, 896, 128, 896, 512], np.float64)
    Y = np.array([128, 128, 896, 896, 512], np.float64)
    u, v = sb.displacement(warp, X, Y)
    P = H @ np.vstack([X, Y, np.ones_like(X)])
    err = np.hypot(P[0] / P[2] - (X + u), P[1] / P[2] - (Y + v))
    assert err.max() < 1.0, err


def test_unrelated_frames_do_not_lock():
    ref, dfm, _ = _pair(0, 1.0, (0.0, 0.0), other_seed=77)
    g = _estimate(ref, dfm, (128, 128, 768, 768))
    assert not g["locked"]
    assert g["peaks"][1] < 0.08


def test_estimate_is_repeatable():
    ref, dfm, _ = _pair(135, 1.05, (-30.0, 18.0))
    a = _estimate(ref, dfm, (128, 128, 768, 768))
    b = _estimate(ref, dfm, (128, 128, 768, 768))
    assert np.array_equal(a["H"], b["H"]) and a["peaks"] == b["peaks"]


def _oracle_run(ref, dfm, prm, model):
    o = oracle.Oracle(False)
    o.set_reference(ref)
    p = [prm.rect_x, prm.rect_y, prm.rect_w, prm.rect_h, prm.step, prm.subset_size, prm.strain_window,
         prm.use_6x6_interpolator]
    return o.run(dfm, p, model_h=model)


@pytest.mark.parametrize("deg", [30.0, 100.0, 170.0])
def test_large_motion_field(deg):
    """Rotation, up to 60 px translation and a smooth random field (the
    large-deformation workload at 1024^2): the estimated model seeds the
    lattice; the field is bit-identical to the restatement's under the same
    model and within 0.02 px RMS of the true displacement. Without a model
    both fail the same way."""
    ref, dfm, prm, warp, _sim = sb.large_motion_pair(1024, angle_deg=deg)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    rc, pts, met = e.run(dfm, prm)
    g = e.last_global_motion()
    assert g["locked"]
    orc, opts, omet = _oracle_run(ref, dfm, prm, g["H"])
    assert rc == orc and rc > 0.8 * (prm.rect_w // prm.step) ** 2
    assert np.array_equal(pts, opts)
    assert np.array_equal(met[COUNT_SLOTS], omet[COUNT_SLOTS])
    assert met[21] == 1.0  # a global model seeded the lattice
    u, v = sb.displacement(warp, pts[:, 0], pts[:, 1])
    err = np.hypot(pts[:, 2] - u, pts[:, 3] - v)
    assert np.sqrt(np.mean(err ** 2)) < 0.02

    e.set_global_motion(False)
    rc0, _, _ = e.run(dfm, prm)
    orc0, _, _ = _oracle_run(ref, dfm, prm, None)
    assert rc0 == orc0 < 0
    assert not e.last_global_motion()["locked"]


def test_injected_model_takes_precedence():
    ref, dfm, prm, warp, (th, tx, ty) = sb.large_motion_pair(1024, angle_deg=75.0)
    n = ref.shape[0]
    c, s = math.cos(th), math.sin(th)
    H = np.array([[c, -s, n / 2 + tx - (c - s) * n / 2], [s, c, n / 2 + ty - (s + c) * n / 2], [0, 0, 1.0]])
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    assert e.set_global_model(H) == 0
    rc, pts, _ = e.run(dfm, prm)
    assert not e.last_global_motion()["locked"]  # no estimate ran
    orc, opts, _ = _oracle_run(ref, dfm, prm, H)
    assert rc == orc > 0 and np.array_equal(pts, opts)


@pytest.mark.parametrize("subset,six", [(21, False), (31, True)])
def test_rotated_field_other_subsets_and_keys6(subset, six):
    """The tiles sized for the model's rotation (about 1.4 times the subset
    side at 45 deg) with the other compiled subset sizes and with the 6x6 Keys
    interpolator: the field bit-identical to the restatement's under the same
    model."""
    ref, dfm, prm0, warp, _sim = sb.large_motion_pair(1024, angle_deg=45.0)
    prm = sb.params((prm0.rect_x, prm0.rect_y, prm0.rect_w, prm0.rect_h), 8, subset, subset, six=six)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    rc, pts, met = e.run(dfm, prm)
    g = e.last_global_motion()
    assert g["locked"]
    orc, opts, omet = _oracle_run(ref, dfm, prm, g["H"])
    assert rc == orc and rc > 0.8 * (prm.rect_w // prm.step) ** 2
    assert np.array_equal(pts, opts)
    assert np.array_equal(met[COUNT_SLOTS], omet[COUNT_SLOTS])


def test_zoomed_field_tiles_capped():
    """A 1.8x zoom: the model's spread (1.87 with the margin) is above the
    tiles' cap of 1.5, so the tiles stay those of 1.5 (inside shared memory
    and the TMA box limit) and the outer samples read global memory; the
    field is bit-identical to the restatement's under the same model."""
    n = 768
    ref = sb.speckle(n, n, 515)
    warp = sb.warp_block(cx=n / 2, cy=n / 2, a=(0.8, 0.0, 0.0, 0.8))
    dfm = sb.speckle(n, n, 515, warp, 1.0, 77)
    prm = sb.params((288, 288, 192, 192), 8, 21, 21)
    e = sb.Engine()
    assert e.set_reference(ref) == 0
    H = np.array([[1.8, 0.0, -0.8 * n / 2], [0.0, 1.8, -0.8 * n / 2], [0.0, 0.0, 1.0]])
    assert e.set_global_model(H) == 0
    rc, pts, met = e.run(dfm, prm)
    orc, opts, omet = _oracle_run(ref, dfm, prm, H)
    assert rc == orc and rc > 100
    assert np.array_equal(pts, opts)
    assert np.array_equal(met[COUNT_SLOTS], omet[COUNT_SLOTS])
