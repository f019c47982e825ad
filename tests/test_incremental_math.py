"""The per-node math of incremental DIC on exact fields: sampling, the coasting
fit, anchors, the node field of a solve and the material-mask warp.

Known answers of the reference's tests/unit/test_incremental_math.cpp, run on
the CPU restatement (oracle/src/incremental_session.hpp) through the oracle
library. The device session (incnode.cu) is a separate implementation, held
to this restatement bit for bit by the GPU incremental tests.
"""
import math

import numpy as np
import pytest

import oracle

A = (1.5, 0.02, -0.01)
B = (-0.75, 0.015, 0.03)


def lin(c, x, y):
    return c[0] + c[1] * x + c[2] * y


def linear_field(gw, gh, rx, ry, step, a=A, b=B):
    f = oracle.NodeField(gw, gh, rx, ry, step)
    for j in range(gh):
        for i in range(gw):
            k = j * gw + i
            x, y = f.node(i, j)
            f.u[k], f.v[k] = lin(a, x, y), lin(b, x, y)
            f.ux[k], f.uy[k], f.vx[k], f.vy[k] = a[1], a[2], b[1], b[2]
    f.corr[:] = 0.01
    return f


def test_sample_on_node_returns_node_exactly():
    f = linear_field(6, 5, 20, 30, 10)
    f.valid[1 * 6 + 3] = 0  # a missing neighbour must not matter on a node
    ok, u, v, _c, taylor = oracle.inc_sample(f, *f.node(2, 1))
    assert ok and not taylor
    assert u == f.u[1 * 6 + 2] and v == f.v[1 * 6 + 2]


def test_sample_bilinear_reproduces_linear_field():
    f = linear_field(6, 5, 20, 30, 10)
    for x in (21.3, 37.9, 64.5):
        for y in (30.2, 55.5, 69.9):
            ok, u, v, _c, taylor = oracle.inc_sample(f, x, y)
            assert ok and not taylor
            assert abs(u - lin(A, x, y)) < 1e-4 and abs(v - lin(B, x, y)) < 1e-4


def test_sample_taylor_fallback_reproduces_linear_field():
    f = linear_field(6, 5, 20, 30, 10)
    f.valid[2 * 6 + 3] = 0  # node (50, 50): the cell around (44, 47) loses a corner
    ok, u, v, _c, taylor = oracle.inc_sample(f, 44.0, 47.0)
    assert ok and taylor
    assert abs(u - lin(A, 44, 47)) < 1e-4 and abs(v - lin(B, 44, 47)) < 1e-4


def test_sample_too_far_from_any_node_is_invalid():
    f = linear_field(4, 4, 100, 100, 10)
    assert oracle.inc_sample(f, 90.0, 95.0)[0]
    assert not oracle.inc_sample(f, 80.0, 100.0)[0]
    assert not oracle.inc_sample(f, 100.0, 160.0)[0]


def test_sample_corr_is_worst_contributor():
    f = linear_field(4, 4, 0, 0, 10)
    f.corr[1 * 4 + 2] = 0.09
    ok, _u, _v, c, _t = oracle.inc_sample(f, 15.0, 15.0)
    assert ok and c == np.float32(0.09)


def test_fit_reproduces_linear_field_across_a_hole():
    f = linear_field(12, 12, 20, 30, 10)
    for j in range(4, 8):
        f.valid[j * 12:(j + 1) * 12] = 0
    for x in (20.0, 73.0, 130.0):
        y = 85.0
        assert not oracle.inc_sample(f, x, y)[0]
        ok, u, v, _c = oracle.inc_fit(f, x, y, 80.0)
        assert ok
        assert abs(u - lin(A, x, y)) < 1e-3 and abs(v - lin(B, x, y)) < 1e-3


def test_fit_too_few_or_collinear_nodes_is_invalid():
    f = linear_field(10, 10, 0, 0, 10)
    f.valid[:] = 0
    f.valid[30:40] = 1  # one row: no spread across it
    assert not oracle.inc_fit(f, 45.0, 50.0, 80.0)[0]
    f.valid[:] = 0
    for k in (43, 47, 25, 65, 23):
        f.valid[k] = 1
    assert not oracle.inc_fit(f, 50.0, 40.0, 80.0)[0]
    f.valid[67] = 1
    ok, u, v, _c = oracle.inc_fit(f, 50.0, 40.0, 80.0)
    assert ok
    assert abs(u - lin(A, 50, 40)) < 1e-3 and abs(v - lin(B, 50, 40)) < 1e-3
    assert not oracle.inc_fit(f, 50.0, 40.0, 5.0)[0]


def test_fit_corr_is_worst_used():
    f = linear_field(8, 8, 0, 0, 10)
    f.corr[2 * 8 + 3] = 0.12  # within the radius of (35, 35)
    f.corr[7 * 8 + 7] = 0.30  # outside it
    ok, _u, _v, c = oracle.inc_fit(f, 35.0, 35.0, 30.0)
    assert ok and c == np.float32(0.12)


def test_anchor_need_drop_refresh_keep():
    f = linear_field(30, 30, 0, 0, 5)
    assert oracle.inc_anchor_need(f, 75.0, 75.0, 21) == "drop"
    assert oracle.inc_anchor_need(f, 75.0, 20.0, 21) == "refresh"
    assert oracle.inc_anchor_need(f, 75.0, 5.0, 21) == "refresh"
    f.valid[23 * 30 + 15] = 0  # a gap 40 px below
    assert oracle.inc_anchor_need(f, 75.0, 75.0, 21) == "refresh"
    f.valid[17 * 30 + 15] = 0  # a hole in its own subset
    assert oracle.inc_anchor_need(f, 75.0, 75.0, 21) == "keep"


def test_node_field_drops_unsolved_and_outliers():
    x, y = np.meshgrid(np.arange(7), np.arange(7))
    u = (1.0 + 0.01 * x).astype(np.float32)
    v = (-0.5 + 0.01 * y).astype(np.float32)
    corr = np.full((7, 7), 0.02, np.float32)
    solved = np.ones((7, 7), np.uint8)
    solved[1, 1] = 0  # never solved
    corr[2, 5] = -1.0  # solved flag but no result
    u[4, 3] += 6.0  # a wrong match
    valid, rejected = oracle.inc_node_field(u, v, corr, solved)
    assert not valid[1, 1] and not valid[2, 5] and not valid[4, 3]
    assert rejected == 1
    assert valid[3, 3]


def rect_mask(w, h, x, y, rw, rh):
    m = np.zeros((h, w), np.uint8)
    m[y:y + rh, x:x + rw] = 255
    return m


def test_mask_warp_zero_displacement_is_identity():
    m0 = rect_mask(240, 200, 60, 50, 100, 80)
    geom = (10, 8, 60, 50, 10)
    n = 80
    w = oracle.inc_warp_mask(m0, geom, np.zeros(n), np.zeros(n), np.ones(n, np.uint8), 40)
    assert np.array_equal(w, m0)


def test_mask_warp_translation_shifts_mask():
    m0 = rect_mask(240, 200, 60, 50, 100, 80)
    geom = (10, 8, 60, 50, 10)
    n = 80
    valid = np.ones(n, np.uint8)
    valid[5] = 0  # a hole in the field is filled, not left empty
    w = oracle.inc_warp_mask(m0, geom, np.full(n, 7.0), np.full(n, -4.0), valid, 40)
    assert np.array_equal(w, rect_mask(240, 200, 67, 46, 100, 80))


def test_mask_warp_stretch_scales_area():
    m0 = rect_mask(320, 240, 80, 60, 120, 100)
    gw, gh, step = 12, 10, 10
    cx = 80 + 60.0
    U = np.array([[0.2 * (80 + i * step - cx) for i in range(gw)] for _ in range(gh)], np.float32)
    w = oracle.inc_warp_mask(m0, (gw, gh, 80, 60, step), U, np.zeros(gw * gh), np.ones(gw * gh, np.uint8), 60)
    ratio = np.count_nonzero(w) / np.count_nonzero(m0)
    assert abs(ratio - 1.2) < 0.012
    xs = np.nonzero(w.any(axis=0))[0]
    bx, bw = xs[0], xs[-1] - xs[0] + 1
    assert abs(bx - (cx - 1.2 * (cx - 80))) <= 1.0
    assert abs(bx + bw - (cx + 1.2 * (80 + 120 - cx))) <= 1.5


def test_mask_warp_large_rotation_is_the_rotated_mask():
    r = (110, 110, 100, 100)
    m0 = rect_mask(320, 320, r[0] - 16, r[1] - 16, r[2] + 32, r[3] + 32)
    gw, gh, step = 20, 20, 5
    c, th = 160.0, math.radians(84.0)
    ct, st = math.cos(th), math.sin(th)
    U = np.zeros((gh, gw), np.float32)
    V = np.zeros((gh, gw), np.float32)
    for j in range(gh):
        for i in range(gw):
            X, Y = r[0] + i * step - c, r[1] + j * step - c
            U[j, i] = ct * X - st * Y - X
            V[j, i] = st * X + ct * Y - Y
    w = oracle.inc_warp_mask(m0, (gw, gh, r[0], r[1], step), U, V, np.ones(gw * gh, np.uint8), 40)
    ratio = np.count_nonzero(w) / np.count_nonzero(m0)
    assert abs(ratio - 1.0) < 0.02
    yy, xx = np.mgrid[0:320, 0:320]
    dx, dy = xx - c, yy - c
    X, Y = ct * dx + st * dy + c, -st * dx + ct * dy + c
    lo, hi = r[0] - 16, r[0] + r[2] + 16
    inside = np.minimum(np.minimum(X - lo, hi - 1 - X), np.minimum(Y - lo, hi - 1 - Y))
    s = w != 0
    assert not (s & (inside < -1.0)).any()
    assert not (~s & (inside > 1.0)).any()


def test_mask_warp_no_valid_node_is_empty():
    m0 = rect_mask(240, 200, 60, 50, 100, 80)
    n = 80
    w = oracle.inc_warp_mask(m0, (10, 8, 60, 50, 10), np.zeros(n), np.zeros(n), np.zeros(n, np.uint8), 40)
    assert not w.any()


def texture(w, h, seed):
    scipy_ndimage = pytest.importorskip("scipy.ndimage")
    rng = np.random.default_rng(seed)
    t = scipy_ndimage.gaussian_filter(rng.normal(0.0, 1.0, (h, w)), 2.0)
    t = (t - t.min()) / (t.max() - t.min()) * 195.0 + 30.0
    return t.astype(np.uint8)


def shifted(img, tx, ty):
    # a whole-pixel shift (reflected borders): no resampling error of its own
    h, w = img.shape
    yy = np.clip(np.arange(h) - ty, -h, 2 * h - 1)
    xx = np.clip(np.arange(w) - tx, -w, 2 * w - 1)
    yy = np.where(yy < 0, -yy - 1, np.where(yy >= h, 2 * h - 1 - yy, yy))
    xx = np.where(xx < 0, -xx - 1, np.where(xx >= w, 2 * w - 1 - xx, xx))
    return img[yy][:, xx]


def test_anchor_matches_the_node_where_it_moved():
    ref = texture(200, 200, 7)
    tx, ty = 12, -7
    dfm = shifted(ref, tx, ty)
    gx, gy = 100.4 + tx + 0.8, 90.7 + ty - 0.6
    rc, x, y, corr, ax, ay, dx, dy = oracle.inc_match(ref, dfm, 100.4, 90.7, 21, gx, gy, 2.0)
    assert (ax, ay) == (100, 91)
    assert abs(dx - 0.4) < 1e-5 and abs(dy + 0.3) < 1e-5
    assert rc == 1
    assert abs(x - (100.4 + tx)) < 0.05 and abs(y - (90.7 + ty)) < 0.05
    assert corr < 0.05
    assert oracle.inc_match(ref, dfm, 100.4, 90.7, 21, gx, gy, 0.5)[0] == 0  # further than allowed
    assert oracle.inc_match(ref, texture(200, 200, 8), 100.4, 90.7, 21, gx, gy, 2.0)[0] == 0  # nothing like it
    assert oracle.inc_match(ref, dfm, 12.0, 100.0, 21, gx, gy, 2.0)[0] == -1  # the patch would leave the image


def test_match_anchor_rejects_unconverged_solve():
    ref = texture(200, 200, 7)
    # most of the subset off the left edge: every start fails the valid-pixel guard
    assert oracle.inc_match(ref, ref, 100.0, 100.0, 21, 3.0, 100.0, 50.0)[0] == 0
    rc, _x, _y, corr = oracle.inc_match(ref, ref, 100.0, 100.0, 21, 100.5, 100.0, 2.0)[:4]
    assert rc == 1 and corr <= 0.15
